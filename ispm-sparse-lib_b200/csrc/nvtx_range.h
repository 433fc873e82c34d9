// Named NVTX ranges around the library's host-side phases (solver set-up,
// solves, reliable updates, value updates, batch calls, plan tuning), so a
// timeline tool shows them and ncu can filter kernels by range.  The NVTX v3
// header is self-contained: without a tool attached the calls return at once.
#ifndef ISPM_NVTX_RANGE_H
#define ISPM_NVTX_RANGE_H

#include <nvtx3/nvToolsExt.h>

namespace ispm {

struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace ispm

#endif
