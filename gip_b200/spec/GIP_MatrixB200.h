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

  // Device state of the fused solver variants.  GIP_LinearSolver owns its Jacobi diagonal
  // as a Matrix member (GIP_LinearSolver.h:20) and builds it in setUp (:40), so a state
  // kept here lives exactly as long as the solver object and is dropped when setUp runs
  // again: no table keyed by addresses, nothing outlives its operator's solver.
  struct SolverState {
    gipb200_matrix op;  // operator the state was built for (the solver's dA)
    int maxit, n, n_all;
    gipb200_pcg pcg;    // device-resident PCG (GIPB200_FUSED_PCG)
    double* work;       // host-driven fused loop (GIPB200_FUSED_OPS): p Ap r z | dinv | scalars
  };
  SolverState& solver_state() { return ss; }
  void release_solver_state();

 protected:
  void upload();
  gipb200_matrix h;
  SolverState ss;
};
#endif
