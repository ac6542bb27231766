#include "GIP_TimerB200.h"

#include "GIP_B200Check.h"

GIP_TimerB200::GIP_TimerB200() : GIP_Timer(), start_ev(0), stop_ev(0) {
  gipb200_require(gipb200_event_create(&start_ev), "event_create");
  gipb200_require(gipb200_event_create(&stop_ev), "event_create");
}

GIP_TimerB200::~GIP_TimerB200() {
  gipb200_event_destroy(start_ev);
  gipb200_event_destroy(stop_ev);
}

void GIP_TimerB200::startChannel() { gipb200_require(gipb200_event_record(start_ev, 0), "record"); }

// GIP_TimerCuda::stopChannel (GIP_TimerCuda.cpp:13-22): seconds, accumulated.
void GIP_TimerB200::stopChannel() {
  float ms = 0.f;
  gipb200_require(gipb200_event_record(stop_ev, 0), "record");
  gipb200_require(gipb200_event_elapsed_ms(start_ev, stop_ev, &ms), "elapsed");
  tm_l = ms / 1000.0f;
  sum_l += tm_l;
  cont += 1;
}

// At one rank the global time equals the local one (GIP_TimerCuda.cpp:23-32 reduces MAX).
void GIP_TimerB200::stopAllChannels() {
  stopChannel();
  tm_g = tm_l;
  sum_g += tm_g;
}
