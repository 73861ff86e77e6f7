// mlp.cu - BF16 tensor-core kernels of the learned surrogate (training and
// inference of its MLP ensemble), FP32 accumulation.
//
// Every contraction of the MLP is one kernel, C = A B^T with both operands
// K-contiguous ("TN"):
//     forward        Y[B,N]  = X[B,K]  W[N,K]^T            (+ bias, ReLU)
//     input grad     dX[B,K] = dY[B,N] (W^T)[K,N]^T         (x ReLU mask)
//     weight grad    dW[N,K] = (dY^T)[N,B] (X^T)[K,B]^T
// with transposed BF16 copies of W, dY and X made by a tiled transpose.  The
// tile loop stages 128 x 32 tiles of A and B in shared memory with cp.async
// (two stages, XOR-swizzled 16-byte chunks so that ldmatrix reads are
// conflict-free), and each of 8 warps runs mma.sync m16n8k16 (bf16 x bf16 ->
// f32) on a 64 x 32 piece of the 128 x 128 block.  Shapes must be multiples of
// the tile (M, N of 128, K of 32); the host wrappers check that and the
// 16-byte alignment of every row.
//
// The same contraction also runs on the 5th-generation tensor cores
// (gemm_tn_umma: tcgen05.mma with the accumulator in tensor memory).
//
// Plus the small kernels of a training step: column sums (bias gradients),
// the masked mean-squared-error gradient, Adam, and BF16 conversion.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "../../include/cupyram_b200_mlp.h"
#include "tensor_map.h"

namespace {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void ldsm_x4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared tile: 128 rows x 32 bf16 (four 16-byte chunks per row); chunk c of
// row r is stored at chunk c ^ ((r >> 1) & 3).
__device__ __forceinline__ int swz(int row, int chunk) { return row * BK + ((chunk ^ ((row >> 1) & 3)) << 3); }

struct EpiArgs {
    void* out;
    int ldo;
    const float* bias;
    const __nv_bfloat16* mask;
    int ldm;
};

template <int EPI>
__device__ __forceinline__ void store2(const EpiArgs& e, int row, int col, float v0, float v1) {
    if (EPI == CR_MLP_EPI_BIAS_RELU_BF16) {
        v0 = fmaxf(v0 + e.bias[col], 0.f);
        v1 = fmaxf(v1 + e.bias[col + 1], 0.f);
        *reinterpret_cast<__nv_bfloat162*>((__nv_bfloat16*)e.out + (size_t)row * e.ldo + col) =
            __floats2bfloat162_rn(v0, v1);
    } else if (EPI == CR_MLP_EPI_BIAS_F32) {
        *reinterpret_cast<float2*>((float*)e.out + (size_t)row * e.ldo + col) =
            make_float2(v0 + e.bias[col], v1 + e.bias[col + 1]);
    } else if (EPI == CR_MLP_EPI_F32) {
        *reinterpret_cast<float2*>((float*)e.out + (size_t)row * e.ldo + col) = make_float2(v0, v1);
    } else {  // CR_MLP_EPI_RELU_MASK_BF16: gradient through the ReLU whose output is `mask`
        const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(e.mask + (size_t)row * e.ldm + col);
        v0 = __bfloat162float(m.x) > 0.f ? v0 : 0.f;
        v1 = __bfloat162float(m.y) > 0.f ? v1 : 0.f;
        *reinterpret_cast<__nv_bfloat162*>((__nv_bfloat16*)e.out + (size_t)row * e.ldo + col) =
            __floats2bfloat162_rn(v0, v1);
    }
}

template <int EPI>
__device__ __forceinline__ void store1(const EpiArgs& e, int row, int col, float v) {
    if (EPI == CR_MLP_EPI_BIAS_RELU_BF16) {
        ((__nv_bfloat16*)e.out)[(size_t)row * e.ldo + col] = __float2bfloat16_rn(fmaxf(v + e.bias[col], 0.f));
    } else if (EPI == CR_MLP_EPI_BIAS_F32) {
        ((float*)e.out)[(size_t)row * e.ldo + col] = v + e.bias[col];
    } else if (EPI == CR_MLP_EPI_F32) {
        ((float*)e.out)[(size_t)row * e.ldo + col] = v;
    } else {  // CR_MLP_EPI_RELU_MASK_BF16
        const float m = __bfloat162float(e.mask[(size_t)row * e.ldm + col]);
        ((__nv_bfloat16*)e.out)[(size_t)row * e.ldo + col] = __float2bfloat16_rn(m > 0.f ? v : 0.f);
    }
}

template <int EPI>
__global__ void __launch_bounds__(kThreads) gemm_tn(const __nv_bfloat16* __restrict__ A,
                                                     const __nv_bfloat16* __restrict__ B, int K, int lda, int ldb,
                                                     EpiArgs e) {
    __shared__ __align__(128) __nv_bfloat16 sA[2][BM * BK];
    __shared__ __align__(128) __nv_bfloat16 sB[2][BN * BK];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;  // 2 x 4 warps: 64 rows x 32 columns each
    const int bm = blockIdx.y * BM, bn = blockIdx.x * BN;
    const __nv_bfloat16* Ab = A + (size_t)bm * lda;
    const __nv_bfloat16* Bb = B + (size_t)bn * ldb;

    auto load = [&](int stage, int k0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int c = tid + i * kThreads;  // 512 chunks of 16 bytes per tile
            const int row = c >> 2, ch = c & 3;
            cp_async16(&sA[stage][swz(row, ch)], Ab + (size_t)row * lda + k0 + ch * 8);
            cp_async16(&sB[stage][swz(row, ch)], Bb + (size_t)row * ldb + k0 + ch * 8);
        }
        cp_commit();
    };

    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

    const int nk = K / BK;
    load(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt & 1;
        if (kt + 1 < nk) {
            load(st ^ 1, (kt + 1) * BK);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            uint32_t a[4][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                const int row = wm * 64 + mi * 16 + (lane & 15);
                ldsm_x4(a[mi][0], a[mi][1], a[mi][2], a[mi][3], &sA[st][swz(row, ks * 2 + (lane >> 4))]);
            }
#pragma unroll
            for (int nj = 0; nj < 2; ++nj) {
                const int row = wn * 32 + nj * 16 + (lane & 7) + ((lane >> 4) << 3);
                ldsm_x4(b[2 * nj][0], b[2 * nj][1], b[2 * nj + 1][0], b[2 * nj + 1][1],
                        &sB[st][swz(row, ks * 2 + ((lane >> 3) & 1))]);
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], a[mi], b[ni][0], b[ni][1]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int row = bm + wm * 64 + mi * 16 + (lane >> 2);
            const int col = bn + wn * 32 + ni * 8 + (lane & 3) * 2;
            store2<EPI>(e, row, col, acc[mi][ni][0], acc[mi][ni][1]);
            store2<EPI>(e, row + 8, col, acc[mi][ni][2], acc[mi][ni][3]);
        }
}

// ---------------------------------------------------------------------------
// The same contraction on the 5th-generation tensor cores (tcgen05).
//
// A CTA of 4 warps owns a 128 x 256 block of C; its FP32 accumulator lives in
// tensor memory (128 lanes x 256 columns, so two CTAs share an SM's 512).  A
// tiles of 128 rows and B tiles of 256 rows x 64 bf16 (one 128-byte swizzle
// atom wide) are staged in shared memory by
// cp.async in the canonical K-major SWIZZLE_128B layout - row r at r x 128
// bytes, its 16-byte chunk c at chunk c ^ (r mod 8) - over two stages.  One
// thread issues the four m128 n256 k16 MMAs of a stage and commits them to
// the stage's mbarrier; the stage is refilled once that barrier flips.  The
// epilogue reads the accumulator with tcgen05.ld (warp w: lanes 32w..32w+31,
// i.e. rows 32w..32w+31 of the block), transposes 32 x 32 pieces through
// shared memory so that each store writes 32 consecutive columns of one row,
// and applies the same epilogues as the mma.sync kernel.  Every wait is bounded: a barrier that does not flip in
// time sets *err and the kernel finishes without the result.
// ---------------------------------------------------------------------------
constexpr int UBM = 128, UBN = 256, UBK = 64;
constexpr int kUThreads = 128;
constexpr int kUTileA = UBM * UBK * 2;      // bytes of one stage's A tile
constexpr int kUTileB = UBN * UBK * 2;      // bytes of one stage's B tile
constexpr int kUStage = kUTileA + kUTileB;  // multiple of 1024
constexpr unsigned kUWaitLimit = 1u << 26;

// Shared-memory matrix descriptor of a K-major SWIZZLE_128B tile (rows of
// 128 bytes, 8-row atoms 1024 bytes apart): start address and stride byte
// offset in 16-byte units, descriptor version 1, layout type 2 (128B swizzle).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)(1) << 16;              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;      // stride byte offset: next 8-row atom
    d |= (uint64_t)1 << 46;                // version
    d |= (uint64_t)2 << 61;                // SWIZZLE_128B
    return d;
}
// Instruction descriptor: D f32, A and B bf16, both K-major, M 128, N 128.
constexpr uint32_t kUIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(UBN >> 3) << 17) | ((uint32_t)(UBM >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// true once the barrier's phase with this parity has completed; bounded
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (unsigned it = 0; it < kUWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int EPI>
__global__ void __launch_bounds__(kUThreads) gemm_tn_umma(const __nv_bfloat16* __restrict__ A,
                                                         const __nv_bfloat16* __restrict__ B, int K, int lda, int ldb,
                                                         EpiArgs e, int* err) {
    extern __shared__ __align__(1024) unsigned char usmem[];
    // 1024-byte aligned stage tiles: A0 B0 A1 B1, then barriers and the TMEM address
    unsigned char* base = (unsigned char*)(((uintptr_t)usmem + 1023) & ~(uintptr_t)1023);
    auto tA = [&](int st) { return base + st * kUStage; };
    auto tB = [&](int st) { return base + st * kUStage + kUTileA; };
    uint64_t* bar = (uint64_t*)(base + 2 * kUStage);
    uint32_t* taddr_s = (uint32_t*)(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int bm = blockIdx.y * UBM, bn = blockIdx.x * UBN;
    const __nv_bfloat16* Ab = A + (size_t)bm * lda;
    const __nv_bfloat16* Bb = B + (size_t)bn * ldb;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                     "r"(UBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *taddr_s;

    auto load = [&](int stage, int k0) {
        // rows of 8 chunks of 16 bytes: A 128 rows (8 chunks per thread), B 256 rows (16)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int c = tid + i * kUThreads;
            const int row = c >> 3, ch = c & 7;
            cp_async16(tA(stage) + row * 128 + ((ch ^ (row & 7)) << 4), Ab + (size_t)row * lda + k0 + ch * 8);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = tid + i * kUThreads;
            const int row = c >> 3, ch = c & 7;
            cp_async16(tB(stage) + row * 128 + ((ch ^ (row & 7)) << 4), Bb + (size_t)row * ldb + k0 + ch * 8);
        }
        cp_commit();
    };

    const int nk = K / UBK;
    bool ok = true;
    load(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt & 1;
        if (kt + 1 < nk) {
            // stage st^1 was last read by the MMAs of tile kt-1
            if (kt >= 1) ok &= mbar_wait(&bar[st ^ 1], ((kt - 1) >> 1) & 1);
            load(st ^ 1, (kt + 1) * UBK);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        // make this thread's shared-memory writes visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(tA(st)), sb = smem_u32(tB(st));
#pragma unroll
            for (int k = 0; k < UBK / 16; ++k) {
                // k16 slice: 32 bytes further along the swizzled rows
                const uint64_t da = umma_desc_sw128(sa + k * 32), db = umma_desc_sw128(sb + k * 32);
                const uint32_t acc = (kt > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(kUIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar[st]))
                         : "memory");
        }
    }
    // all MMAs are done once the last commit's barrier flips
    ok &= mbar_wait(&bar[(nk - 1) & 1], ((nk - 1) >> 1) & 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (lane == 0) atomicExch(err, 1);
    } else {
        // 32 columns at a time: lane l reads row 32w + l from tensor memory,
        // the warp transposes the 32 x 32 piece through shared memory (the
        // stage tiles are idle now) and writes it one row per instruction,
        // 32 consecutive columns, so that every store fills whole sectors
        float* stg = reinterpret_cast<float*>(base) + warp * 32 * 33;
#pragma unroll 1
        for (int cc = 0; cc < UBN; cc += 32) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t v[16];
                const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc + 16 * h);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j) stg[lane * 33 + 16 * h + j] = __uint_as_float(v[j]);
            }
            __syncwarp();
#pragma unroll 4
            for (int r = 0; r < 32; ++r) store1<EPI>(e, bm + warp * 32 + r, bn + cc + lane, stg[r * 33 + lane]);
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UBN));
}

constexpr size_t kUSmem = 2 * kUStage + 1024 + 64;

// ---------------------------------------------------------------------------
// The tcgen05 contraction with its operands brought in by the tensor memory
// accelerator (TMA) and its roles split over warps.
//
// Same block (128 x 256, FP32 accumulator in 256 TMEM columns), same
// SWIZZLE_128B K-major tiles and MMAs as gemm_tn_umma, but:
//   * lane 0 of warp 0 issues one cp.async.bulk.tensor per operand tile
//     (tensor maps over this GPU's memory, no multicast) that completes on
//     the stage's "full" mbarrier with the byte count it expects;
//   * lane 0 of warp 1 waits on "full", issues the four k16 MMAs of the
//     stage and commits them to the stage's "empty" mbarrier, which the
//     producer waits on before refilling the stage: no __syncthreads and no
//     thread-issued copies in the main loop;
//   * kTStages stages ring through shared memory;
//   * after the last commit every warp reads its 32 accumulator rows and
//     stores them as gemm_tn_umma does.
// Every wait is bounded; one that gives up sets *err and the kernel finishes
// without the result.
// ---------------------------------------------------------------------------
constexpr int kTStages = 2;  // 2 x 48 KB: two CTAs share an SM (and its 512 TMEM columns)
constexpr size_t kTSmem = (size_t)kTStages * kUStage + 1024 + 256;

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

template <int EPI>
__global__ void __launch_bounds__(kUThreads) gemm_tn_tma(const __grid_constant__ CUtensorMap mapA,
                                                        const __grid_constant__ CUtensorMap mapB, int K, EpiArgs e,
                                                        int* err) {
    extern __shared__ __align__(1024) unsigned char usmem[];
    unsigned char* base = (unsigned char*)(((uintptr_t)usmem + 1023) & ~(uintptr_t)1023);
    auto tA = [&](int st) { return base + st * kUStage; };
    auto tB = [&](int st) { return base + st * kUStage + kUTileA; };
    uint64_t* full = (uint64_t*)(base + kTStages * kUStage);
    uint64_t* empty = full + kTStages;
    uint64_t* done = empty + kTStages;
    uint32_t* taddr_s = (uint32_t*)(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int bm = blockIdx.y * UBM, bn = blockIdx.x * UBN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                     "r"(UBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 32) {
        for (int s = 0; s < kTStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *taddr_s;
    const int nk = K / UBK;
    bool ok = true;

    int issued = 0;  // producer: tiles whose loads were issued
    if (warp == 0 && lane == 0) {
        // producer: stage st is refilled once the MMAs that read it have completed
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int st = kt % kTStages;
            if (kt >= kTStages) ok &= mbar_wait(&empty[st], ((kt / kTStages) - 1) & 1);
            if (!ok) break;
            mbar_expect_tx(&full[st], (unsigned)kUStage);
            tma_load_2d(tA(st), &mapA, kt * UBK, bm, &full[st]);
            tma_load_2d(tB(st), &mapB, kt * UBK, bn, &full[st]);
            issued = kt + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int st = kt % kTStages;
            ok &= mbar_wait(&full[st], (kt / kTStages) & 1);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(tA(st)), sb = smem_u32(tB(st));
#pragma unroll
            for (int k = 0; k < UBK / 16; ++k) {
                const uint64_t da = umma_desc_sw128(sa + k * 32), db = umma_desc_sw128(sb + k * 32);
                const uint32_t acc = (kt > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(kUIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&empty[st]))
                         : "memory");
        }
        // the accumulator is complete once every MMA issued so far is
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(done))
                     : "memory");
    }
    __syncwarp();
    // every thread: wait for the accumulator (bounded), then the epilogue
    ok &= mbar_wait(done, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // a role thread that gave up is seen by the whole CTA
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!ok && warp == 0 && lane == 0) {
        // no copy may still be writing this CTA's shared memory when it exits:
        // wait (bounded) for the last load issued into each stage
        for (int kt = issued - 1; kt >= 0 && kt >= issued - kTStages; --kt)
            mbar_wait(&full[kt % kTStages], (kt / kTStages) & 1);
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        float* stg = reinterpret_cast<float*>(base) + warp * 32 * 33;  // the stage tiles are idle now
#pragma unroll 1
        for (int cc = 0; cc < UBN; cc += 32) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t v[16];
                const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc + 16 * h);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j) stg[lane * 33 + 16 * h + j] = __uint_as_float(v[j]);
            }
            __syncwarp();
#pragma unroll 4
            for (int r = 0; r < 32; ++r) store1<EPI>(e, bm + warp * 32 + r, bn + cc + lane, stg[r * 33 + lane]);
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UBN));
}

// dst[c][r] = src[r][c] for a rows x cols BF16 matrix (32 x 32 tiles).
__global__ void transpose_bf16(const __nv_bfloat16* __restrict__ src, int lds, __nv_bfloat16* __restrict__ dst,
                               int ldd, int rows, int cols) {
    __shared__ __nv_bfloat16 t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[i][threadIdx.x] = src[(size_t)r * lds + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(size_t)c * ldd + r] = t[threadIdx.x][i];
    }
}

// out[c] = sum_r src[r][c] (bias gradients), one thread per column.
__global__ void col_sum_bf16(const __nv_bfloat16* __restrict__ src, int ld, int rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += __bfloat162float(src[(size_t)r * ld + c]);
    out[c] = s;
}

// Masked mean squared error: grad = 2 (pred - y) / n_valid where valid,
// and the sum of squared errors accumulated into *sse.
__global__ void mse_grad(const float* __restrict__ pred, const __nv_bfloat16* __restrict__ y,
                         const unsigned char* __restrict__ valid, long long n, float inv_count,
                         __nv_bfloat16* __restrict__ grad, double* __restrict__ sse) {
    __shared__ double red[256];
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float g = 0.f;
        if (valid[i]) {
            const float d = pred[i] - __bfloat162float(y[i]);
            g = 2.f * d * inv_count;
            acc += (double)d * d;
        }
        grad[i] = __float2bfloat16_rn(g);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(sse, red[0]);
}

// Adam on FP32 master parameters; writes the BF16 copy used by the GEMMs.
__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, __nv_bfloat16* __restrict__ pb, long long n, float lr, float b1,
                          float b2, float eps, float c1, float c2, float wd) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] + wd * p[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        if (pb) pb[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

int grid_for(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 4096 ? (b < 1 ? 1 : b) : 4096);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// The kernel behind cr_mlp_gemm_tc: the TMA-fed one, one block per CTA and
// two CTAs per SM, by default (measured fastest: 515 TFLOP/s on 8192 x 8192 x
// 512, against 392 for the persistent one and 480 for the cp.async-fed one);
// CUPYRAM_B200_GEMM=persistent the persistent one, =cp the cp.async-fed one.
int gemm_feed() {
    const char* v = getenv("CUPYRAM_B200_GEMM");
    if (v && v[0] == 'c') return 0;
    if (v && v[0] == 'p') return 2;
    return 1;
}

// ---------------------------------------------------------------------------
// Persistent TMA-fed tcgen05 contraction with the epilogue overlapped.
//
// One CTA per SM walks the output blocks (128 x 256) in a static round
// robin.  Six warps:
//   * warp 0, lane 0: TMA producer over a kPStages-deep ring of stages;
//   * warp 1, lane 0: MMA issuer, accumulating block i in one of two TMEM
//     accumulators (columns 0..255 or 256..511, by i's parity), committing
//     each stage to its "empty" barrier and each finished block to its
//     accumulator's "full" barrier;
//   * warps 2..5: the epilogue, one TMEM lane quadrant each (quadrant =
//     warp mod 4), reading block i's accumulator while the MMAs of block i+1
//     run in the other one, then releasing it on its "empty" barrier.
// Every wait is bounded; a role that gives up stops, the CTA sets *err, and
// the output is incomplete.
// ---------------------------------------------------------------------------
constexpr int kPStages = 4;
constexpr int kPThreads = 192;
constexpr size_t kPSmem = (size_t)kPStages * kUStage + (size_t)4 * 32 * 33 * 4 + 1024 + 512;

template <int EPI>
__global__ void __launch_bounds__(kPThreads, 1) gemm_tn_persistent(const __grid_constant__ CUtensorMap mapA,
                                                                   const __grid_constant__ CUtensorMap mapB, int M,
                                                                   int N, int K, EpiArgs e, int* err) {
    extern __shared__ __align__(1024) unsigned char usmem[];
    unsigned char* base = (unsigned char*)(((uintptr_t)usmem + 1023) & ~(uintptr_t)1023);
    auto tA = [&](int st) { return base + st * kUStage; };
    auto tB = [&](int st) { return base + st * kUStage + kUTileA; };
    float* stg_all = reinterpret_cast<float*>(base + kPStages * kUStage);
    uint64_t* full = (uint64_t*)(base + kPStages * kUStage + 4 * 32 * 33 * 4);
    uint64_t* empty = full + kPStages;
    uint64_t* acc_full = empty + kPStages;   // [2]
    uint64_t* acc_empty = acc_full + 2;      // [2]
    uint32_t* taddr_s = (uint32_t*)(acc_empty + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nk = K / UBK, nbm = M / UBM, nbn = N / UBN, nblocks = nbm * nbn;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                     "r"(2 * UBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 32) {
        for (int s = 0; s < kPStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 4);  // one arrival per epilogue warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *taddr_s;
    bool ok = true;
    int issued = 0;  // producer: k-tiles whose loads were issued (over all blocks)

    if (warp == 0) {
        if (lane == 0) {
            int g = 0;
            for (int blk = blockIdx.x; blk < nblocks && ok; blk += gridDim.x) {
                const int bm = (blk % nbm) * UBM, bn = (blk / nbm) * UBN;
                for (int kt = 0; kt < nk && ok; ++kt, ++g) {
                    const int st = g % kPStages;
                    if (g >= kPStages) ok &= mbar_wait(&empty[st], ((g / kPStages) - 1) & 1);
                    if (!ok) break;
                    mbar_expect_tx(&full[st], (unsigned)kUStage);
                    tma_load_2d(tA(st), &mapA, kt * UBK, bm, &full[st]);
                    tma_load_2d(tB(st), &mapB, kt * UBK, bn, &full[st]);
                    issued = g + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int g = 0, i = 0;
            for (int blk = blockIdx.x; blk < nblocks && ok; blk += gridDim.x, ++i) {
                const int a = i & 1;
                // the epilogue has drained this accumulator's previous block
                if (i >= 2) ok &= mbar_wait(&acc_empty[a], ((i / 2) - 1) & 1);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_addr = tmem + (uint32_t)(a * UBN);
                for (int kt = 0; kt < nk && ok; ++kt, ++g) {
                    const int st = g % kPStages;
                    ok &= mbar_wait(&full[st], (g / kPStages) & 1);
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(tA(st)), sb = smem_u32(tB(st));
#pragma unroll
                    for (int k = 0; k < UBK / 16; ++k) {
                        const uint64_t da = umma_desc_sw128(sa + k * 32), db = umma_desc_sw128(sb + k * 32);
                        const uint32_t accum = (kt > 0 || k > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                            :
                            : "r"(acc_addr), "l"(da), "l"(db), "r"(kUIdesc), "r"(accum)
                            : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&empty[st]))
                                 : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&acc_full[a]))
                             : "memory");
            }
        }
    } else {
        // epilogue: TMEM lane quadrant q = warp mod 4 holds rows 32q..32q+31
        const int q = warp & 3;
        float* stg = stg_all + (warp - 2) * 32 * 33;
        int i = 0;
        for (int blk = blockIdx.x; blk < nblocks && ok; blk += gridDim.x, ++i) {
            const int a = i & 1;
            const int bm = (blk % nbm) * UBM, bn = (blk / nbm) * UBN;
            ok &= mbar_wait(&acc_full[a], (i / 2) & 1);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int cc = 0; cc < UBN; cc += 32) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    uint32_t v[16];
                    const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * UBN + cc + 16 * h);
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                        "%15}, [%16];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15])
                        : "r"(ta));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 16; ++j) stg[lane * 33 + 16 * h + j] = __uint_as_float(v[j]);
                }
                __syncwarp();
#pragma unroll 4
                for (int r = 0; r < 32; ++r) store1<EPI>(e, bm + q * 32 + r, bn + cc + lane, stg[r * 33 + lane]);
                __syncwarp();
            }
            // this warp's reads of the accumulator are done: release it to the MMAs
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[a])) : "memory");
        }
    }
    __syncwarp();
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!ok && warp == 0 && lane == 0) {
        // no copy may still be writing this CTA's shared memory when it exits
        for (int g = issued - 1; g >= 0 && g >= issued - kPStages; --g)
            mbar_wait(&full[g % kPStages], (g / kPStages) & 1);
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * UBN));
}

using crk::encode_tiled;
using crk::EncodeTiledFn;

// Tensor map of a rows x K bf16 operand (row stride ld elements) in boxes of
// `box_rows` rows x 64 elements, 128-byte swizzle: the layout the MMAs read.
bool operand_map(CUtensorMap* map, const void* ptr, int rows, int K, int ld, int box_rows) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)UBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

extern "C" {

int cr_mlp_gemm(int epi, const void* A, const void* B, int M, int N, int K, int lda, int ldb, void* out, int ldo,
                const float* bias, const void* mask, int ldm, void* stream) {
    if (M <= 0 || N <= 0 || K <= 0 || M % BM || N % BN || K % BK) return CR_MLP_EBADSHAPE;
    if (lda < K || ldb < K || lda % 8 || ldb % 8 || ldo < N || ldo % 2 || !aligned16(A) || !aligned16(B) || !out)
        return CR_MLP_EBADSHAPE;
    if ((epi == CR_MLP_EPI_BIAS_RELU_BF16 || epi == CR_MLP_EPI_BIAS_F32) && !bias) return CR_MLP_EBADSHAPE;
    if (epi == CR_MLP_EPI_RELU_MASK_BF16 && (!mask || ldm < N || ldm % 2)) return CR_MLP_EBADSHAPE;
    EpiArgs e{out, ldo, bias, (const __nv_bfloat16*)mask, ldm};
    const dim3 grid(N / BN, M / BM);
    cudaStream_t st = (cudaStream_t)stream;
    auto a = (const __nv_bfloat16*)A;
    auto b = (const __nv_bfloat16*)B;
    switch (epi) {
        case CR_MLP_EPI_BIAS_RELU_BF16: gemm_tn<CR_MLP_EPI_BIAS_RELU_BF16><<<grid, kThreads, 0, st>>>(a, b, K, lda, ldb, e); break;
        case CR_MLP_EPI_BIAS_F32: gemm_tn<CR_MLP_EPI_BIAS_F32><<<grid, kThreads, 0, st>>>(a, b, K, lda, ldb, e); break;
        case CR_MLP_EPI_F32: gemm_tn<CR_MLP_EPI_F32><<<grid, kThreads, 0, st>>>(a, b, K, lda, ldb, e); break;
        case CR_MLP_EPI_RELU_MASK_BF16: gemm_tn<CR_MLP_EPI_RELU_MASK_BF16><<<grid, kThreads, 0, st>>>(a, b, K, lda, ldb, e); break;
        default: return CR_MLP_EBADSHAPE;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

int cr_mlp_gemm_tc(int epi, const void* A, const void* B, int M, int N, int K, int lda, int ldb, void* out, int ldo,
                   const float* bias, const void* mask, int ldm, int* err, void* stream) {
    if (M <= 0 || N <= 0 || K <= 0 || M % UBM || N % UBN || K % UBK) return CR_MLP_EBADSHAPE;
    if (lda < K || ldb < K || lda % 8 || ldb % 8 || ldo < N || ldo % 2 || !aligned16(A) || !aligned16(B) || !out ||
        !err)
        return CR_MLP_EBADSHAPE;
    if ((epi == CR_MLP_EPI_BIAS_RELU_BF16 || epi == CR_MLP_EPI_BIAS_F32) && !bias) return CR_MLP_EBADSHAPE;
    if (epi == CR_MLP_EPI_RELU_MASK_BF16 && (!mask || ldm < N || ldm % 2)) return CR_MLP_EBADSHAPE;
    EpiArgs e{out, ldo, bias, (const __nv_bfloat16*)mask, ldm};
    const dim3 grid(N / UBN, M / UBM);
    cudaStream_t st = (cudaStream_t)stream;
    auto a = (const __nv_bfloat16*)A;
    auto b = (const __nv_bfloat16*)B;
    cudaError_t ce = cudaSuccess;
    const int feed = gemm_feed();
    if (feed == 2) {
        // persistent: one CTA per SM, operands by the tensor memory accelerator
        CUtensorMap ma, mb;
        if (!operand_map(&ma, A, M, K, lda, UBM) || !operand_map(&mb, B, N, K, ldb, UBN)) return CR_MLP_ECUDA;
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return CR_MLP_ECUDA;
        const int blocks = (M / UBM) * (N / UBN);
        const int ctas = blocks < sms ? blocks : sms;
        switch (epi) {
#define CR_PERS_CASE(E)                                                                                          \
    case E:                                                                                                      \
        ce = cudaFuncSetAttribute(gemm_tn_persistent<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPSmem); \
        if (ce == cudaSuccess) gemm_tn_persistent<E><<<ctas, kPThreads, kPSmem, st>>>(ma, mb, M, N, K, e, err);    \
        break;
            CR_PERS_CASE(CR_MLP_EPI_BIAS_RELU_BF16)
            CR_PERS_CASE(CR_MLP_EPI_BIAS_F32)
            CR_PERS_CASE(CR_MLP_EPI_F32)
            CR_PERS_CASE(CR_MLP_EPI_RELU_MASK_BF16)
#undef CR_PERS_CASE
            default: return CR_MLP_EBADSHAPE;
        }
        if (ce != cudaSuccess) return CR_MLP_ECUDA;
        return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
    }
    if (feed == 1) {
        // operands by the tensor memory accelerator (tensor maps over this GPU's memory)
        CUtensorMap ma, mb;
        if (!operand_map(&ma, A, M, K, lda, UBM) || !operand_map(&mb, B, N, K, ldb, UBN)) return CR_MLP_ECUDA;
        switch (epi) {
#define CR_TMA_CASE(E)                                                                                       \
    case E:                                                                                                  \
        ce = cudaFuncSetAttribute(gemm_tn_tma<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTSmem);   \
        if (ce == cudaSuccess) gemm_tn_tma<E><<<grid, kUThreads, kTSmem, st>>>(ma, mb, K, e, err);            \
        break;
            CR_TMA_CASE(CR_MLP_EPI_BIAS_RELU_BF16)
            CR_TMA_CASE(CR_MLP_EPI_BIAS_F32)
            CR_TMA_CASE(CR_MLP_EPI_F32)
            CR_TMA_CASE(CR_MLP_EPI_RELU_MASK_BF16)
#undef CR_TMA_CASE
            default: return CR_MLP_EBADSHAPE;
        }
        if (ce != cudaSuccess) return CR_MLP_ECUDA;
        return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
    }
    switch (epi) {
#define CR_UMMA_CASE(E)                                                                                    \
    case E:                                                                                                \
        ce = cudaFuncSetAttribute(gemm_tn_umma<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUSmem); \
        if (ce == cudaSuccess) gemm_tn_umma<E><<<grid, kUThreads, kUSmem, st>>>(a, b, K, lda, ldb, e, err);      \
        break;
        CR_UMMA_CASE(CR_MLP_EPI_BIAS_RELU_BF16)
        CR_UMMA_CASE(CR_MLP_EPI_BIAS_F32)
        CR_UMMA_CASE(CR_MLP_EPI_F32)
        CR_UMMA_CASE(CR_MLP_EPI_RELU_MASK_BF16)
#undef CR_UMMA_CASE
        default: return CR_MLP_EBADSHAPE;
    }
    if (ce != cudaSuccess) return CR_MLP_ECUDA;
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

int cr_mlp_transpose(const void* src, int lds, void* dst, int ldd, int rows, int cols, void* stream) {
    if (rows <= 0 || cols <= 0 || lds < cols || ldd < rows) return CR_MLP_EBADSHAPE;
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    transpose_bf16<<<grid, block, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)src, lds, (__nv_bfloat16*)dst, ldd,
                                                              rows, cols);
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

int cr_mlp_col_sum(const void* src, int ld, int rows, int cols, float* out, void* stream) {
    if (rows <= 0 || cols <= 0 || ld < cols) return CR_MLP_EBADSHAPE;
    col_sum_bf16<<<(cols + 255) / 256, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)src, ld, rows, cols, out);
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

int cr_mlp_mse_grad(const float* pred, const void* target, const unsigned char* valid, long long n, float inv_count,
                    void* grad, double* sse, void* stream) {
    if (n <= 0) return CR_MLP_EBADSHAPE;
    mse_grad<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(pred, (const __nv_bfloat16*)target, valid, n, inv_count,
                                                            (__nv_bfloat16*)grad, sse);
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

int cr_mlp_adam(float* p, const float* g, float* m, float* v, void* p_bf16, long long n, float lr, float beta1,
                float beta2, float eps, int step, float weight_decay, void* stream) {
    if (n <= 0 || step < 1) return CR_MLP_EBADSHAPE;
    const float c1 = 1.f / (1.f - powf(beta1, (float)step));
    const float c2 = 1.f / (1.f - powf(beta2, (float)step));
    adam_step<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, (__nv_bfloat16*)p_bf16, n, lr, beta1, beta2,
                                                             eps, c1, c2, weight_decay);
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

int cr_mlp_to_bf16(const float* src, void* dst, long long n, void* stream) {
    if (n <= 0) return CR_MLP_EBADSHAPE;
    to_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, (__nv_bfloat16*)dst, n);
    return cudaGetLastError() == cudaSuccess ? 0 : CR_MLP_ECUDA;
}

}  // extern "C"
