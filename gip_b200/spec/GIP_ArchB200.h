// Node of the B200 Specification (counterpart of GIP_ArchGPU,
// src/Specifications/Cuda/GIP_ArchGPU.h): selects the device of this rank.
#ifndef _gip_archb200_
#define _gip_archb200_
#include "../../AbstractInterfaces/GIP_Arch.h"

class GIP_ArchB200 : public GIP_Arch {
 public:
  GIP_ArchB200() : devId(0) {}
  GIP_ArchB200(int numcpus, int numcores, int numdevs);
  ~GIP_ArchB200() {}
  void postConstruct(int numcpus, int numcores, int numdevs);
  void setUp();
  int device() const { return devId; }

 protected:
  int devId;
};
#endif
