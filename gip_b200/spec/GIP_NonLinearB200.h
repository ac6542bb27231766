// CFL time step of the B200 Specification (counterpart of GIP_NonLinearCuda,
// src/Specifications/Cuda/GIP_NonLinearCuda.h).
#ifndef _gip_nlinearb200_
#define _gip_nlinearb200_
#include "../../AbstractInterfaces/GIP_NonLinear.h"

class GIP_NonLinearB200 : public GIP_NonLinear {
 public:
  GIP_NonLinearB200() {}
  ~GIP_NonLinearB200() {}
  double getCFL(GIP_Topo*, GIP_Vector*, GIP_Vector*, GIP_Vector*, GIP_Vector*, GIP_Vector*,
                double gamma, double rho);
};
#endif
