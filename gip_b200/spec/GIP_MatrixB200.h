// Matrix of the B200 Specification (counterpart of GIP_MatrixCuda,
// src/Specifications/Cuda/GIP_MatrixCuda.h).  The host CSR arrays of GIP_Matrix are
// kept (GIP_LinearSolver::setUp builds the Jacobi diagonal from them); the device
// copy is a libgipb200 matrix handle.
#ifndef _gip_matrixb200_
#define _gip_matrixb200_
#include <string>

#include "../../AbstractInterfaces/GIP_Matrix.h"
#include "gipb200.h"

class GIP_MatrixB200 : public GIP_Matrix {
 public:
  GIP_MatrixB200();
  ~GIP_MatrixB200();
  void postConstruct(string name, GIP_Topo*, GIP_Arch*);

  void spmv(GIP_Vector* x, GIP_Vector* y);                                // y = A x
  void spmv(GIP_Vector* x, GIP_Vector* y, double alpha, double beta);     // y = a A x + b y
  void spmv(GIP_Vector* x, GIP_Matrix* target);                           // values of target
  void spmv(GIP_Vector* x, GIP_Matrix* target, double alpha, double beta);
  void setUpDiagonal(GIP_Matrix* A);
  double* getCsrValADevice() { return 0; }
  gipb200_matrix handle() const { return h; }

 protected:
  void upload();
  gipb200_matrix h;
};
#endif
