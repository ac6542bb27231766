// The B200 Specification: GIP's Node/Matrix/Vector/NonLinear/Timer concrete classes
// implemented over libgipb200 (include/gipb200.h).  Drop this directory into GIP as
// src/Specifications/B200/ and select it in DrivenCavity.cpp with
//   #include "src/Specifications/B200/B200.h"  and the GIP_*B200 typedefs.
#ifndef _gip_b200_spec_
#define _gip_b200_spec_
#include "GIP_ArchB200.h"
#include "GIP_MatrixB200.h"
#include "GIP_NonLinearB200.h"
#include "GIP_TimerB200.h"
#include "GIP_VectorB200.h"
#endif
