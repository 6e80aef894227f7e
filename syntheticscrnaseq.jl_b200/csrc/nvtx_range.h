// Named NVTX ranges around the library's compute entry points, so that a profiler's
// timeline (Nsight Systems, or ncu --nvtx with --nvtx-include) shows which call launched
// which kernels.  NVTX v3 is header-only: with no tool attached a range costs an indirect
// call that returns at once.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace scrna {

class NvtxRange {
public:
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace scrna
