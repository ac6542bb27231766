// Vector of the B200 Specification (counterpart of GIP_VectorCuda,
// src/Specifications/Cuda/GIP_VectorCuda.h).  The values live on the device; the host
// array of GIP_Vector is refreshed on getHostPtr().  Ranges follow RUN_DOMAIN
// (src/BasicInterfaces/GIP_Topo.h:19-27).
#ifndef _gip_vectorb200_
#define _gip_vectorb200_
#include <string>

#include "../../AbstractInterfaces/GIP_Vector.h"

class GIP_VectorB200 : public GIP_Vector {
 public:
  GIP_VectorB200();
  GIP_VectorB200(int n, GIP_Arch*);
  GIP_VectorB200(GIP_Topo*, GIP_Arch*);
  ~GIP_VectorB200();

  void postConstruct(GIP_Topo*, GIP_Arch*);
  void postConstruct(string name, GIP_Topo*, GIP_Arch*);

  void axpy(GIP_Vector* x, double alpha, enum RUN_DOMAIN);               // y += a x
  void axpy(GIP_Vector* x, double alpha, double beta, enum RUN_DOMAIN);  // y = a x + b y
  double dot(GIP_Vector* x, GIP_Vector* scratch, enum RUN_DOMAIN);
  double norm(GIP_Vector* scratch, enum RUN_DOMAIN);                       // max |y_i|
  void copyTo(GIP_Vector* x, enum RUN_DOMAIN);
  void update();
  double* getDevicePtr() { return dvec; }
  double* getHostPtr();
  void operator=(int value);

 protected:
  void allocate(int n);
  int range(enum RUN_DOMAIN) const;
  double* dvec;
};
#endif
