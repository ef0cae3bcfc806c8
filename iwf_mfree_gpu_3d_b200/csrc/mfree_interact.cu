// mfree_interact.cu -- launches of the pair kernel: one launch over the tiles
// of every scene of a table (kernel templates in mfree_interact.cuh).
#include "mfree_interact.cuh"

namespace mfree {

cudaError_t launch_interact_batch(const BatchTable &T, int lpp, bool cspm, int cond, bool prec, int grid,
                                  cudaStream_t s) {
    return with_lpp(lpp, cspm, cond, prec, [&](auto v) { return decltype(v)::batch(T, grid, s); });
}

}  // namespace mfree
