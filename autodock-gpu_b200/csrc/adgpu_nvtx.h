// adgpu_nvtx.h -- named NVTX ranges around the library's host entry points
// (a docking, an engine tick, a submission, result processing), so that a
// profiler's timeline shows where each call's kernels belong.  NVTX is
// header-only: without a profiler attached a range costs two calls that
// return at once.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace adgpu {

struct NvtxRange {
	explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
	~NvtxRange() { nvtxRangePop(); }
	NvtxRange(const NvtxRange&) = delete;
	NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace adgpu
