#include "GIP_ArchB200.h"

#include <mpi.h>
#include <stdlib.h>

#include "GIP_B200Check.h"

// GIP_ArchGPU picks rank % numcpus (GIP_ArchGPU.cpp:3-8), which sends every rank of
// GIP's default Node(1,4,4) to device 0.  Here the device is GIPB200_DEVICE when set,
// else the rank modulo the visible devices is left to the caller's CUDA_VISIBLE_DEVICES.
GIP_ArchB200::GIP_ArchB200(int numcpus, int numcores, int numdevs)
    : GIP_Arch(numcpus, numcores, numdevs), devId(0) {
  const char* env = getenv("GIPB200_DEVICE");
  if (env) devId = atoi(env);
}

void GIP_ArchB200::postConstruct(int numcpus, int numcores, int numdevs) {
  num_cpus = numcpus;
  num_cores = numcores;
  num_devs = numdevs;
}

void GIP_ArchB200::setUp() { gipb200_require(gipb200_set_device(devId), "gipb200_set_device"); }
