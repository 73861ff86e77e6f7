// march_sum.cu - launchers of the batched partial-fraction march: dispatch on
// the precision form to its translation unit (march_sum_plain.cu,
// march_sum_chosen.cu, march_sum_fast.cu, march_sum_refined.cu; kernels in
// march_sum_impl.cuh).
#include <cuda_runtime.h>

#include <cstring>

#include "march_sum.cuh"
#include "tensor_map.h"

namespace crk {

namespace {

// Map of an array stored as rows of 32 elements of elem_bytes bytes (rows
// rows), viewed as 8-byte words, in boxes of the first `cols` elements of
// kRB rows: plain tiles, no swizzle, no interleave, zeros outside the array.
// Boxes narrower than a row (the ray columns of a tile) take no L2
// promotion: a wider fetch would read the unused columns from DRAM.
bool rows_map(EncodeTiledFn enc, CUtensorMap* m, const void* base, int elem_bytes, long long rows, int cols) {
    const cuuint64_t dims[2] = {(cuuint64_t)(kTile * elem_bytes / 8), (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)(kTile * elem_bytes)};
    const cuuint32_t box[2] = {(cuuint32_t)(cols * elem_bytes / 8), (cuuint32_t)kRB};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               cols == kTile ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B : CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool encode_sum_maps(SumArgs& a, int form, long long ray_rows, long long lane_rows) {
    std::memset(&a.maps, 0, sizeof a.maps);
    const EncodeTiledFn enc = encode_tiled();
    if (!enc || ray_rows <= 0 || lane_rows <= 0) return false;
    const int vb = form == CR_PLAIN_C128 ? 16 : 8;  // factors and workspace: complex128 or complex64
    const int eb = form == CR_CHOSEN_C64 ? 8 : 16;  // couplings
    const void* lanes[5];
    lanes[kMapG] = a.G;
    lanes[kMapQD] = a.QD;
    lanes[kMapWD] = a.WD;
    lanes[kMapQU] = a.QU;
    lanes[kMapWU] = a.WU;
    bool ok = true;
    for (int i = 0; i < 5; ++i) ok = ok && rows_map(enc, &a.maps.lane[i], lanes[i], vb, lane_rows, kTile);
    for (int P = 1; P <= kMaxP; ++P) {
        const int R = kTile / P;  // rays of a tile whose rays take P lanes
        ok = ok && rows_map(enc, &a.maps.ray[kMapU][P - 1], a.u, 16, ray_rows, R);
        ok = ok && rows_map(enc, &a.maps.ray[kMapED][P - 1], a.ED, eb, ray_rows, R);
        ok = ok && rows_map(enc, &a.maps.ray[kMapEU][P - 1], a.EU, eb, ray_rows, R);
        if (a.E2) ok = ok && rows_map(enc, &a.maps.ray[kMapE2][P - 1], a.E2, 16, ray_rows, R);
    }
    return ok;
}

cudaError_t sum_launch_plain(const SumArgs& a, int p, int count, cudaStream_t st, bool launch);
cudaError_t sum_launch_chosen(const SumArgs& a, int p, int count, cudaStream_t st, bool launch);
cudaError_t sum_launch_fast(const SumArgs& a, int p, int count, cudaStream_t st, bool launch);
cudaError_t sum_launch_refined(const SumArgs& a, int p, int count, cudaStream_t st, bool launch);
cudaError_t sum_queue_plain(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch);
cudaError_t sum_queue_chosen(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch);
cudaError_t sum_queue_fast(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch);
cudaError_t sum_queue_refined(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch);

namespace {

cudaError_t queue_form(const SumArgs& a, int n_tiles, int form, cudaStream_t st, int* ctas, bool launch) {
    return form == CR_C64_REFINED ? sum_queue_refined(a, n_tiles, st, ctas, launch)
           : form == CR_CHOSEN_C64 ? sum_queue_fast(a, n_tiles, st, ctas, launch)
           : form == CR_CHOSEN_C64R ? sum_queue_chosen(a, n_tiles, st, ctas, launch)
                                    : sum_queue_plain(a, n_tiles, st, ctas, launch);
}

cudaError_t launch_form(const SumArgs& a, int p, int count, int form, cudaStream_t st, bool launch) {
    return form == CR_C64_REFINED ? sum_launch_refined(a, p, count, st, launch)
           : form == CR_CHOSEN_C64 ? sum_launch_fast(a, p, count, st, launch)
           : form == CR_CHOSEN_C64R ? sum_launch_chosen(a, p, count, st, launch)
                                    : sum_launch_plain(a, p, count, st, launch);
}

}  // namespace

cudaError_t launch_march_sum_queue(const SumArgs& a, int n_tiles, int form, cudaStream_t st, int* ctas) {
    if (n_tiles <= 0) return cudaSuccess;
    return queue_form(a, n_tiles, form, st, ctas, true);
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
        const cudaError_t ce = launch_form(a, tile_P[begin], end - begin, form, st, true);
        if (ce != cudaSuccess) return ce;
        ++*launches;
        begin = end;
    }
    return cudaSuccess;
}

cudaError_t prepare_march_sum(const int* tile_P, int n_tiles, int form) {
    SumArgs a{};
    a.min_p = kMaxP;
    bool seen[kMaxP + 1] = {};
    for (int t = 0; t < n_tiles; ++t)
        if (tile_P[t] >= 1 && tile_P[t] <= kMaxP) {
            seen[tile_P[t]] = true;
            a.min_p = tile_P[t] < a.min_p ? tile_P[t] : a.min_p;
        }
    cudaError_t ce = n_tiles > 0 ? queue_form(a, n_tiles, form, 0, nullptr, false) : cudaSuccess;
    for (int p = 1; p <= kMaxP && ce == cudaSuccess; ++p)
        if (seen[p]) ce = launch_form(a, p, 0, form, 0, false);
    return ce;
}

}  // namespace crk
