#include "GIP_MatrixB200.h"

#include <stdio.h>

#include "GIP_B200Check.h"
#include "GIP_VectorB200.h"

GIP_MatrixB200::GIP_MatrixB200() : h(0) {
  ss.op = 0;
  ss.maxit = ss.n = ss.n_all = 0;
  ss.pcg = 0;
  ss.work = 0;
  csrValA = 0;
  csrColIndA = 0;
  csrRowIndA = 0;
  num_rows = num_cols = nnz = 0;
  myTopo = 0;
  myArch = 0;
}

GIP_MatrixB200::~GIP_MatrixB200() {
  release_solver_state();
  if (h) gipb200_matrix_destroy(h);
  delete[] csrValA;
  delete[] csrColIndA;
  delete[] csrRowIndA;
}

// Binary CSR reader with GIP's layout (GIP_MatrixCuda::postConstruct,
// GIP_MatrixCuda.cpp:14-53), plus the size checks GIP leaves out.
void GIP_MatrixB200::postConstruct(string name, GIP_Topo* topo, GIP_Arch* arch) {
  FILE* fp = fopen(name.c_str(), "rb");
  if (!fp) {
    fprintf(stderr, "GIP B200 Specification: cannot open operator %s\n", name.c_str());
    exit(1);
  }
  int sizes[5];
  if (fread(sizes, sizeof(int), 5, fp) != 5 || sizes[0] < 0 || sizes[1] < 0 || sizes[2] < 0) {
    fprintf(stderr, "GIP B200 Specification: bad header in %s\n", name.c_str());
    exit(1);
  }
  nnz = sizes[0];
  num_cols = sizes[1];
  num_rows = sizes[2];
  csrValA = new double[nnz > 0 ? nnz : 1];
  csrColIndA = new int[nnz > 0 ? nnz : 1];
  csrRowIndA = new int[num_rows + 1];
  size_t got = fread(csrValA, sizeof(double), nnz, fp);
  got += fread(csrColIndA, sizeof(int), nnz, fp);
  got += fread(csrRowIndA, sizeof(int), num_rows + 1, fp);
  fclose(fp);
  if (got != (size_t)nnz * 2 + num_rows + 1) {
    fprintf(stderr, "GIP B200 Specification: truncated operator %s\n", name.c_str());
    exit(1);
  }
  myTopo = topo;
  myArch = arch;
  upload();
}

void GIP_MatrixB200::upload() {
  // columns may reach past the header's ncols (GIP's per-rank files count only owned
  // cells there); the device gather bound is the largest column present
  int ncols = num_cols;
  for (int k = 0; k < nnz; ++k)
    if (csrColIndA[k] + 1 > ncols) ncols = csrColIndA[k] + 1;
  if (h) gipb200_matrix_destroy(h);
  h = 0;
  gipb200_require(gipb200_matrix_create(num_rows, ncols, nnz, csrRowIndA, csrColIndA, csrValA, &h),
                  "gipb200_matrix_create");
}

void GIP_MatrixB200::spmv(GIP_Vector* x, GIP_Vector* y) {
  gipb200_require(gipb200_matrix_spmv(h, x->getDevicePtr(), y->getDevicePtr(), 0.0, 0.0, 0, 0),
                  "spmv");
}

void GIP_MatrixB200::spmv(GIP_Vector* x, GIP_Vector* y, double alpha, double beta) {
  gipb200_require(gipb200_matrix_spmv(h, x->getDevicePtr(), y->getDevicePtr(), alpha, beta, 1, 0),
                  "spmv");
}

static gipb200_matrix target_handle(GIP_Matrix* t) {
  GIP_MatrixB200* m = dynamic_cast<GIP_MatrixB200*>(t);
  if (!m) {
    fprintf(stderr, "GIP B200 Specification: spmv target is not a GIP_MatrixB200\n");
    exit(1);
  }
  return m->handle();
}

void GIP_MatrixB200::spmv(GIP_Vector* x, GIP_Matrix* target) {
  gipb200_require(gipb200_matrix_spmv_values(h, x->getDevicePtr(), target_handle(target), 0.0,
                                             0.0, 0, 0),
                  "spmv into matrix values");
}

void GIP_MatrixB200::spmv(GIP_Vector* x, GIP_Matrix* target, double alpha, double beta) {
  gipb200_require(gipb200_matrix_spmv_values(h, x->getDevicePtr(), target_handle(target), alpha,
                                             beta, 1, 0),
                  "spmv into matrix values");
}

// The Jacobi diagonal as a one-entry-per-row matrix, as GIP builds it
// (GIP_MatrixMulticore::setUpDiagonal, GIP_MatrixMulticore.cpp:177-210): 1/A_ii, the last
// diagonal entry of a row wins.  A row without a diagonal becomes an empty row.
void GIP_MatrixB200::release_solver_state() {
  if (ss.pcg) gipb200_pcg_destroy(ss.pcg);
  if (ss.work) gipb200_free(ss.work);
  ss.op = 0;
  ss.maxit = ss.n = ss.n_all = 0;
  ss.pcg = 0;
  ss.work = 0;
}

void GIP_MatrixB200::setUpDiagonal(GIP_Matrix* A) {
  release_solver_state();  // a new setUp: the solver's device state is rebuilt on demand
  num_rows = A->getNumRows();
  num_cols = A->getNumRows();
  const double* va = A->getCsrValA();
  const int* ca = A->getCsrColIndA();
  const int* ra = A->getCsrRowIndA();
  double* d = new double[num_rows > 0 ? num_rows : 1];
  bool* has = new bool[num_rows > 0 ? num_rows : 1];
  int count = 0;
  for (int i = 0; i < num_rows; ++i) {
    has[i] = false;
    for (int j = ra[i]; j < ra[i + 1]; ++j)
      if (ca[j] == i) {
        d[i] = 1.0 / va[j];
        has[i] = true;
      }
    count += has[i];
  }
  nnz = count;
  delete[] csrValA;
  delete[] csrColIndA;
  delete[] csrRowIndA;
  csrValA = new double[nnz > 0 ? nnz : 1];
  csrColIndA = new int[nnz > 0 ? nnz : 1];
  csrRowIndA = new int[num_rows + 1];
  int k = 0;
  for (int i = 0; i < num_rows; ++i) {
    csrRowIndA[i] = k;
    if (has[i]) {
      csrValA[k] = d[i];
      csrColIndA[k] = i;
      ++k;
    }
  }
  csrRowIndA[num_rows] = k;
  delete[] d;
  delete[] has;
  myTopo = A->getMyTopo();
  myArch = A->getMyArch();
  upload();
}
