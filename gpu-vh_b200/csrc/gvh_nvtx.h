// gvh_nvtx.h -- NVTX ranges around the library's device work (host side), so that a profiler
// timeline (Nsight Systems, ncu's NVTX filters) shows each RK stage, serving round and surface
// slab by name. NVTX v3 is header-only: with no tool attached a range costs a check of a
// function pointer. Defining GVH_NO_NVTX compiles the ranges out.
#pragma once

#ifndef GVH_NO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

namespace gvh {

// A named range from construction to destruction on the calling host thread.
class NvtxRange {
 public:
  explicit NvtxRange(const char *name) {
#ifndef GVH_NO_NVTX
    nvtxRangePushA(name);
#else
    (void)name;
#endif
  }
  ~NvtxRange() {
#ifndef GVH_NO_NVTX
    nvtxRangePop();
#endif
  }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace gvh
