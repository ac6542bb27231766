/*
 * Test-infrastructure only: a driver translation unit around GIP's own CPU
 * Specification (src/Specifications/Multicore) and its unmodified templates
 * GIP_DNS (src/Algorithms/GIP_DNS.h) and GIP_LinearSolver
 * (src/Algorithms/GIP_LinearSolver.h).  It is compiled by oracle/Makefile from the
 * reference sources where they lie; nothing here is linked into the product.
 *
 * Compared with GIP's DrivenCavity.cpp:21-43 it adds four things a checker needs:
 *   - the number of timesteps (GIP_DNS hard-codes maxIt=10 at GIP_DNS.h:132),
 *   - the PCG iteration count (GIP_DNS sets maxIt=100 at GIP_DNS.h:183; the environment
 *     variable GIPREF_CG_MAXIT overrides the solver's copy after setUp, so a benchmark
 *     can time a bounded number of GIP's own iterations),
 *   - wall-clock timing of setUp() and integrate() (rank 0 prints one JSON line to
 *     stderr), after GIPREF_WARMUP untimed timesteps when that variable is set (an
 *     extra integrate() call first: it recomputes dt from the current fields, as
 *     GIP_DNS.h:101-102 does at every call),
 *   - an optional dump of the final fields of every rank (u,v,w,p,p0,mf,ax0,ay0,az0)
 *     as raw float64 arrays, so parity tests can compare fields, not only the
 *     printed massr lines.
 * The class members it touches are private in GIP_DNS; the driver reaches them by
 * compiling this one translation unit with `private` redefined as `public`.
 *
 * Usage (cwd must contain InputFiles/):  GIPSHIM_NP=<ranks> gip_ref_cpu <case>
 *        [steps] [dump_prefix] [Re]
 * `Re` sets GIP_DNS::Re and gamma=1/Re, which only enter the CFL limit
 * (GIP_DNS.h:136-137, 406); the viscosity of the momentum equation is baked into D.
 */
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>

#include <iostream>
#include <map>
#include <string>

#include "mpi.h"

#define private public
#define protected public
#include "src/Algorithms/GIP_DNS.h"
#include "src/Specifications/Multicore/Multicore.h"
#undef private
#undef protected

typedef GIP_DNS<GIP_MatrixMulticore, GIP_VectorMulticore, GIP_ArchCPU, GIP_NonLinearMulticore>
    RefDNS;

static void dump_vec(const std::string& prefix, const char* name, int rank, GIP_Vector& v) {
  std::string path = prefix + "." + name + "." + std::to_string(rank) + ".f64";
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "ref_driver: cannot write %s\n", path.c_str());
    exit(3);
  }
  fwrite(v.getHostPtr(), sizeof(double), (size_t)v.getSize(), f);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: gip_ref_cpu <case> [steps] [dump_prefix]\n");
    return 2;
  }
  int prov;
  MPI_Init_thread(0, 0, MPI_THREAD_SINGLE, &prov);
  int rank, nranks;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  nranks = 1;
  {
    const char* np = getenv("GIPSHIM_NP");
    if (np) nranks = atoi(np);
  }

  RefDNS dns(argv[1]);
  if (argc >= 3) dns.maxIt = atoi(argv[2]);
  if (argc >= 5) {
    dns.Re = atof(argv[4]);
    dns.gamma = 1.0 / dns.Re;
  }

  MPI_Barrier(MPI_COMM_WORLD);
  double t0 = omp_get_wtime();
  dns.setUp();
  {
    const char* m = getenv("GIPREF_CG_MAXIT");
    if (m) dns.cg.maxIt = atoi(m);
  }
  MPI_Barrier(MPI_COMM_WORLD);
  const double t_setup = omp_get_wtime() - t0;
  int warmup = 0;
  {
    const char* w = getenv("GIPREF_WARMUP");
    if (w) warmup = atoi(w);
  }
  if (warmup > 0) {
    const int steps = dns.maxIt;
    dns.maxIt = warmup;
    dns.integrate();
    dns.maxIt = steps;
  }
  MPI_Barrier(MPI_COMM_WORLD);
  double t1 = omp_get_wtime();
  dns.integrate();
  MPI_Barrier(MPI_COMM_WORLD);
  double t2 = omp_get_wtime();

  if (argc >= 4 && argv[3][0] != '\0' && std::string(argv[3]) != "-") {
    std::string prefix(argv[3]);
    dump_vec(prefix, "u", rank, dns.u);
    dump_vec(prefix, "v", rank, dns.v);
    dump_vec(prefix, "w", rank, dns.w);
    dump_vec(prefix, "p", rank, dns.p);
    dump_vec(prefix, "p0", rank, dns.p0);
    dump_vec(prefix, "mf", rank, dns.mf);
    dump_vec(prefix, "ax0", rank, dns.ax0);
    dump_vec(prefix, "ay0", rank, dns.ay0);
    dump_vec(prefix, "az0", rank, dns.az0);
  }
  if (rank == 0) {
    fprintf(stderr,
            "{\"ranks\": %d, \"steps\": %d, \"setup_s\": %.6f, \"integrate_s\": %.6f, "
            "\"ms_per_step\": %.6f, \"dt_next\": %.17g, \"time\": %.17g, \"cg_maxit\": %d, "
            "\"warmup\": %d}\n",
            nranks, dns.maxIt, t_setup, t2 - t1, (t2 - t1) * 1e3 / (dns.maxIt > 0 ? dns.maxIt : 1),
            dns.dt, dns.time, dns.cg.maxIt, warmup);
  }
  MPI_Finalize();
  return 0;
}
