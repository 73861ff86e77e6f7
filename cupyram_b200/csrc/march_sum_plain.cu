// march_sum_plain.cu - the batched partial-fraction march instantiated for one
// precision form (kPlain; see march_sum_impl.cuh).
#include "march_sum_impl.cuh"

namespace crk {

cudaError_t sum_launch_plain(const SumArgs& a, int p, int count, cudaStream_t st, bool launch) {
    return launch_p<kPlain>(a, p, count, st, launch);
}

cudaError_t sum_queue_plain(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch) {
    return launch_queue_f<kPlain>(a, n_tiles, st, ctas, launch);
}

}  // namespace crk
