/* <perfcounter.h> of the DPU runtime: see dpu_host.h. */
#include "dpu_host.h"
