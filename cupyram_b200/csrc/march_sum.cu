// march_sum.cu - launchers of the batched partial-fraction march: dispatch on
// the precision form to its translation unit (march_sum_plain.cu,
// march_sum_chosen.cu, march_sum_fast.cu, march_sum_refined.cu; kernels in
// march_sum_impl.cuh).
#include <cuda_runtime.h>

#include "march_sum.cuh"

namespace crk {

cudaError_t sum_launch_plain(const SumArgs& a, int p, int count, cudaStream_t st);
cudaError_t sum_launch_chosen(const SumArgs& a, int p, int count, cudaStream_t st);
cudaError_t sum_launch_fast(const SumArgs& a, int p, int count, cudaStream_t st);
cudaError_t sum_queue_plain(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas);
cudaError_t sum_queue_chosen(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas);
cudaError_t sum_queue_fast(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas);
cudaError_t sum_launch_refined(const SumArgs& a, int p, int count, cudaStream_t st);
cudaError_t sum_queue_refined(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas);

cudaError_t launch_march_sum_queue(const SumArgs& a, int n_tiles, int form, cudaStream_t st, int* ctas) {
    if (n_tiles <= 0) return cudaSuccess;
    return form == CR_C64_REFINED ? sum_queue_refined(a, n_tiles, st, ctas)
           : form == CR_CHOSEN_C64 ? sum_queue_fast(a, n_tiles, st, ctas)
           : form == CR_CHOSEN_C64R ? sum_queue_chosen(a, n_tiles, st, ctas)
                                    : sum_queue_plain(a, n_tiles, st, ctas);
}

cudaError_t launch_march_sum(const SumArgs& a0, const int* tile_P, int n_tiles, int form,
                             const cudaStream_t* streams, int n_streams, int* launches) {
    // tiles are ordered by lanes per ray; one launch per run of equal P
    int begin = 0;
    *launches = 0;
    while (begin < n_tiles) {
        int end = begin + 1;
        while (end < n_tiles && tile_P[end] == tile_P[begin]) ++end;
        SumArgs a = a0;
        a.tile_begin = begin;
        const cudaStream_t st = streams[*launches % n_streams];
        const cudaError_t ce = form == CR_C64_REFINED ? sum_launch_refined(a, tile_P[begin], end - begin, st)
                               : form == CR_CHOSEN_C64 ? sum_launch_fast(a, tile_P[begin], end - begin, st)
                               : form == CR_CHOSEN_C64R ? sum_launch_chosen(a, tile_P[begin], end - begin, st)
                                                        : sum_launch_plain(a, tile_P[begin], end - begin, st);
        if (ce != cudaSuccess) return ce;
        ++*launches;
        begin = end;
    }
    return cudaSuccess;
}

}  // namespace crk
