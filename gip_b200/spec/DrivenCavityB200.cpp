// GIP's driver (DrivenCavity.cpp:21-43) with the B200 Specification selected.  Build
// variants: -DGIPB200_FUSED_PCG (device-resident PCG per solve), -DGIPB200_FUSED_OPS
// (GIP's solver loop on the host over the fused CG calls) and -DGIPB200_FUSED_DNS (the
// whole integrate() on the fused engine).  Optional second
// argument: number of timesteps (GIP hard-codes 10, GIP_DNS.h:132) -- set through the
// GIP_DNS member the driver reaches by compiling with `private` mapped to `public`.
// Optional third argument: how many times integrate() is called (default 1); the run
// ends with a JSON line on stderr holding the integrate time and field checksums.
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
#if defined(GIPB200_FUSED_PCG) || defined(GIPB200_FUSED_OPS)
#include "GIP_LinearSolverB200.h"
#endif
#ifdef GIPB200_FUSED_DNS
#include "GIP_DNSB200.h"
#endif

typedef GIP_DNS<GIP_MatrixB200, GIP_VectorB200, GIP_ArchB200, GIP_NonLinearB200> B200DNS;

// Checksums of a field (sum, and sum weighted by position) at full precision, so runs can
// be compared bit for bit from their stderr.
static void field_sums(const char* name, GIP_VectorB200& v, int n, bool first) {
  const double* h = v.getHostPtr();
  double s = 0.0, sw = 0.0;
  for (int i = 0; i < n; ++i) {
    s += h[i];
    sw += h[i] * (double)(i + 1);
  }
  fprintf(stderr, "%s\"%s\": [%.17g, %.17g]", first ? "" : ", ", name, s, sw);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cout << "a.out <Mesh_file> [steps] [integrate calls]" << std::endl;
    return 0;
  }
  int prov;
  MPI_Init_thread(0, 0, MPI_THREAD_SINGLE, &prov);
  B200DNS driven(argv[1]);
  if (argc >= 3) driven.maxIt = atoi(argv[2]);
  const int calls = argc >= 4 ? atoi(argv[3]) : 1;
  GIP_TimerB200 timer;
  driven.setUp();
  timer.startChannel();
  for (int c = 0; c < calls; ++c) driven.integrate();
  timer.stopChannel();
  fprintf(stderr, "{\"integrate_s\": %.6f, \"steps\": %d, \"calls\": %d, \"fields\": {",
          timer.getTimeL(), driven.maxIt, calls);
  const int n = driven.topoCols.getOwnedSize();
  field_sums("u", driven.u, n, true);
  field_sums("v", driven.v, n, false);
  field_sums("w", driven.w, n, false);
  field_sums("p", driven.p, n, false);
  field_sums("mf", driven.mf, driven.topoFaces.getAllSize(), false);
  fprintf(stderr, "}, \"time\": %.17g}\n", driven.time);
  MPI_Finalize();
  return 0;
}
