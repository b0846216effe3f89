#include_next <cuda.h>
#include "gvh_ref_gpu_shim.h"
