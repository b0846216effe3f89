#include_next <cuda_runtime.h>
#include "gvh_ref_gpu_shim.h"
