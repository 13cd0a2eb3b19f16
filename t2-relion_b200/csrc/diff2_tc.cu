// tcgen05 split-BF16 coarse diff2 (placeholder until the tensor-core kernel lands).
#include "t2b_internal.cuh"

namespace t2b {

bool tc_supported() { return false; }

void tc_prepare_projections(const Tables&, TcOperands&, cudaStream_t)
{
    throw Error{T2B_ERR_UNSUPPORTED, "split-BF16 contraction not built"};
}

void tc_launch_diff2(const Tables&, const Work&, TcOperands&, cudaStream_t)
{
    throw Error{T2B_ERR_UNSUPPORTED, "split-BF16 contraction not built"};
}

}  // namespace t2b
