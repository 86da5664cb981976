// sfnl_split.cu -- split-precision tcgen05 form (placeholder).
#include "sfnl_internal.h"
#include "sfnl_ops.cuh"
namespace sfnl {
bool split_supported(int, int) { return false; }
int launch_split(const ProgArgs &, int, cudaStream_t) { return set_error(SFNL_ERR_UNSUPPORTED, "split form not built"); }
}  // namespace sfnl
