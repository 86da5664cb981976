// sfnl_fast.cu -- FP64 factored transforms on an internal alias-free grid (placeholder).
#include "sfnl_internal.h"
#include "sfnl_ops.cuh"
namespace sfnl {
int fast_grid_length(int m) { return 3 * m; }
bool fast_supported(int, int, int) { return false; }
int launch_fast(const ProgArgs &, cudaStream_t) { return set_error(SFNL_ERR_UNSUPPORTED, "FAST form not built"); }
}  // namespace sfnl
