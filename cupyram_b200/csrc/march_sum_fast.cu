// march_sum_fast.cu - the batched partial-fraction march instantiated for one
// precision form (kFast; see march_sum_impl.cuh).
#include "march_sum_impl.cuh"

namespace crk {

cudaError_t sum_launch_fast(const SumArgs& a, int p, int count, cudaStream_t st, bool launch) {
    return launch_p<kFast>(a, p, count, st, launch);
}

cudaError_t sum_queue_fast(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch) {
    return launch_queue_f<kFast>(a, n_tiles, st, ctas, launch);
}

}  // namespace crk
