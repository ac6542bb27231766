// Timer of the B200 Specification (counterpart of GIP_TimerCuda,
// src/Specifications/Cuda/GIP_TimerCuda.h): CUDA events on the default stream.
#ifndef _gip_timerb200_
#define _gip_timerb200_
#include "../../AbstractInterfaces/GIP_Timer.h"

class GIP_TimerB200 : public GIP_Timer {
 public:
  GIP_TimerB200();
  ~GIP_TimerB200();
  void startChannel();
  void stopChannel();
  void stopAllChannels();

 protected:
  void* start_ev;
  void* stop_ev;
};
#endif
