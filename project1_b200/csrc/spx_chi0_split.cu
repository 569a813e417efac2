// K2 placeholder: split-precision accumulation is enqueued here.
#include "spx_common.cuh"
namespace spx {
size_t split_workspace_bytes(int64_t, int, int) { return 0; }
int split_chi0_slab(spx_ctx* ctx, const double2*, int64_t, int64_t, int, const double*, int64_t,
                    int, double2*, void*, size_t, cudaStream_t, int*, cudaEvent_t) {
  return set_error(ctx, SPX_ENOTSUP, "split precision not built");
}
}  // namespace spx
