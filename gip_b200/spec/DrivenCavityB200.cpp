// GIP's driver (DrivenCavity.cpp:21-43) with the B200 Specification selected.  Build
// variants: -DGIPB200_FUSED_PCG (device-resident PCG per solve) and
// -DGIPB200_FUSED_DNS (the whole integrate() on the fused engine).  Optional second
// argument: number of timesteps (GIP hard-codes 10, GIP_DNS.h:132) -- set through the
// GIP_DNS member the driver reaches by compiling with `private` mapped to `public`.
#include <stdio.h>
#include <stdlib.h>

#include <iostream>
#include <map>
#include <string>
#include <vector>

#include <mpi.h>

#define private public
#include "../../Algorithms/GIP_DNS.h"
#undef private
#include "B200.h"
#ifdef GIPB200_FUSED_PCG
#include "GIP_LinearSolverB200.h"
#endif
#ifdef GIPB200_FUSED_DNS
#include "GIP_DNSB200.h"
#endif

typedef GIP_DNS<GIP_MatrixB200, GIP_VectorB200, GIP_ArchB200, GIP_NonLinearB200> B200DNS;

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cout << "a.out <Mesh_file> [steps]" << std::endl;
    return 0;
  }
  int prov;
  MPI_Init_thread(0, 0, MPI_THREAD_SINGLE, &prov);
  B200DNS driven(argv[1]);
  if (argc >= 3) driven.maxIt = atoi(argv[2]);
  GIP_TimerB200 timer;
  driven.setUp();
  timer.startChannel();
  driven.integrate();
  timer.stopChannel();
  fprintf(stderr, "{\"integrate_s\": %.6f, \"steps\": %d}\n", timer.getTimeL(), driven.maxIt);
  MPI_Finalize();
  return 0;
}
