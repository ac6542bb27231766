#include "GIP_NonLinearB200.h"

#include "GIP_B200Check.h"

// GIP_NonLinearMulticore::getCFL (GIP_NonLinearMulticore.cpp:3-55) over the inner cells,
// one fused min-reduction on the device.
double GIP_NonLinearB200::getCFL(GIP_Topo* topo, GIP_Vector* u, GIP_Vector* v, GIP_Vector* w,
                                 GIP_Vector* dxs, GIP_Vector*, double gamma, double rho) {
  double dt = 0.0;
  gipb200_require(gipb200_cfl(topo->getInnerSize(), u->getDevicePtr(), v->getDevicePtr(),
                              w->getDevicePtr(), dxs->getDevicePtr(), gamma, rho, &dt, 0),
                  "gipb200_cfl");
  return dt;
}
