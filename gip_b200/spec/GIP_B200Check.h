// Status handling shared by the B200 Specification classes.  GIP's own device
// Specification ignores CUDA errors (src/Specifications/Cuda/Libs/libgpu.cu); these
// classes stop the run with the library's message instead, since GIP's interfaces
// have no error channel.
#ifndef _gip_b200_check_
#define _gip_b200_check_
#include <stdio.h>
#include <stdlib.h>

#include "gipb200.h"

inline void gipb200_require(int status, const char* what) {
  if (status != GIPB200_OK) {
    fprintf(stderr, "GIP B200 Specification: %s failed: %s (%s)\n", what,
            gipb200_status_string(status), gipb200_last_error());
    exit(1);
  }
}
#endif
