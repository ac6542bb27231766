#include "GIP_VectorB200.h"

#include <stdio.h>
#include <stdlib.h>

#include <map>
#include <vector>

#include "GIP_B200Check.h"
#include "gipb200.h"

// GIP_LinearSolver::solve constructs five temporaries per solve
// (GIP_LinearSolver.h:54-61); a size-keyed free list keeps those from turning into
// device allocations and frees on every timestep.
namespace {
std::map<size_t, std::vector<double*> >& pool() {
  static std::map<size_t, std::vector<double*> > p;
  return p;
}
double* pool_get(size_t n) {
  std::vector<double*>& v = pool()[n];
  if (!v.empty()) {
    double* d = v.back();
    v.pop_back();
    return d;
  }
  void* d = 0;
  gipb200_require(gipb200_malloc(&d, n * sizeof(double)), "gipb200_malloc");
  return (double*)d;
}
void pool_put(size_t n, double* d) {
  if (d) pool()[n].push_back(d);
}
}  // namespace

GIP_VectorB200::GIP_VectorB200() : dvec(0) {
  vec = 0;
  size = 0;
  myTopo = 0;
  myArch = 0;
}

GIP_VectorB200::GIP_VectorB200(int n, GIP_Arch* arch) : dvec(0) {
  vec = 0;
  myTopo = 0;
  myArch = arch;
  allocate(n);
}

GIP_VectorB200::GIP_VectorB200(GIP_Topo* topo, GIP_Arch* arch) : dvec(0) {
  vec = 0;
  myTopo = topo;
  myArch = arch;
  allocate(topo->getAllSize());
}

GIP_VectorB200::~GIP_VectorB200() {
  pool_put((size_t)(size > 0 ? size : 1), dvec);
  delete[] vec;
}

void GIP_VectorB200::allocate(int n) {
  size = n;
  vec = new double[n > 0 ? n : 1];
  dvec = pool_get((size_t)(n > 0 ? n : 1));
  // GIP leaves new vectors uninitialised; zeros make runs reproducible
  gipb200_require(gipb200_dfill(n, dvec, 0.0, 0), "gipb200_dfill");
}

void GIP_VectorB200::postConstruct(GIP_Topo* topo, GIP_Arch* arch) {
  myTopo = topo;
  myArch = arch;
  allocate(topo->getAllSize());
}

// GIP_VectorCuda::postConstruct(name,...) (GIP_VectorCuda.cpp:23-59): int32 n then n doubles.
void GIP_VectorB200::postConstruct(string name, GIP_Topo* topo, GIP_Arch* arch) {
  postConstruct(topo, arch);
  FILE* fp = fopen(name.c_str(), "rb");
  if (!fp) {
    fprintf(stderr, "GIP B200 Specification: cannot open scalar field %s\n", name.c_str());
    exit(1);
  }
  int n = 0;
  if (fread(&n, sizeof(int), 1, fp) != 1 || n < 0 || n > size) {
    fprintf(stderr, "GIP B200 Specification: bad length in %s\n", name.c_str());
    exit(1);
  }
  for (int i = 0; i < size; ++i) vec[i] = 0.0;
  if (fread(vec, sizeof(double), n, fp) != (size_t)n) {
    fprintf(stderr, "GIP B200 Specification: truncated scalar field %s\n", name.c_str());
    exit(1);
  }
  fclose(fp);
  gipb200_require(gipb200_memcpy_h2d(dvec, vec, (size_t)size * sizeof(double), 0), "h2d");
}

int GIP_VectorB200::range(enum RUN_DOMAIN r) const {
  switch (r) {
    case _ALL_: return size;
    case _OWNED_: return myTopo->getOwnedSize();
    case _INNER_: return myTopo->getInnerSize();
    default:
      fprintf(stderr, "GIP B200 Specification: unsupported RUN_DOMAIN %d\n", (int)r);
      exit(1);
  }
}

void GIP_VectorB200::axpy(GIP_Vector* x, double alpha, enum RUN_DOMAIN r) {
  gipb200_require(gipb200_daxpy(range(r), dvec, x->getDevicePtr(), alpha, 0), "daxpy");
}

void GIP_VectorB200::axpy(GIP_Vector* x, double alpha, double beta, enum RUN_DOMAIN r) {
  gipb200_require(gipb200_daxpby(range(r), dvec, x->getDevicePtr(), alpha, beta, 0), "daxpby");
}

// GIP_VectorCuda::dot (GIP_VectorCuda.cpp:103-130) without the MPI_Allreduce: one rank.
double GIP_VectorB200::dot(GIP_Vector* x, GIP_Vector*, enum RUN_DOMAIN r) {
  double v = 0.0;
  gipb200_require(gipb200_ddot(range(r), dvec, x->getDevicePtr(), &v, 0), "ddot");
  return v;
}

double GIP_VectorB200::norm(GIP_Vector*, enum RUN_DOMAIN r) {
  double v = 0.0;
  gipb200_require(gipb200_dnorminf(range(r), dvec, &v, 0), "dnorminf");
  return v;
}

void GIP_VectorB200::copyTo(GIP_Vector* x, enum RUN_DOMAIN r) {
  gipb200_require(gipb200_dcopy(range(r), x->getDevicePtr(), dvec, 0), "dcopy");
}

// The halo exchange of GIP_Topo (GIP_VectorCuda.cpp:224-247) is empty at one rank; the
// B200 Specification runs the topology collapsed to one rank and refuses halos.
void GIP_VectorB200::update() {
  if (myTopo && (myTopo->getSendSize() > 0 || myTopo->getRecvSize() > 0)) {
    fprintf(stderr, "GIP B200 Specification: multi-rank halos are not supported; merge the "
                    "operators to one rank\n");
    exit(1);
  }
}

double* GIP_VectorB200::getHostPtr() {
  gipb200_require(gipb200_memcpy_d2h(vec, dvec, (size_t)size * sizeof(double), 0), "d2h");
  return vec;
}

void GIP_VectorB200::operator=(int value) {
  gipb200_require(gipb200_dfill(size, dvec, (double)value, 0), "dfill");
}
