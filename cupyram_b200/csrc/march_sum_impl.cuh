// march_sum_impl.cuh - range march in partial-fraction ("sum") form.
//
// The kernel templates of the batched march.  Each precision form is
// instantiated in its own translation unit (march_sum_plain.cu,
// march_sum_chosen.cu, march_sum_fast.cu, march_sum_refined.cu) so that the
// four compile in parallel; march_sum.cu dispatches on the form.
//
// The split-step Pade operator of one range step is a rational function of
// the Galerkin operator X = M^{-1} D (M: mass matrix, D: Galerkin stiffness +
// wavenumber rows; cupyram/fused_kernel.py:20-69):
//
//     P(X) = prod_j (1 + pd1_j X) / (1 + pd2_j X)          (reference: product form)
//          = c_inf + sum_j c_j / (1 + pd2_j X)             (here: partial fractions)
//
// so u_new = c_inf u + sum_j c_j x_j with (M + pd2_j D) x_j = M u: the np
// tridiagonal solves of a step are independent.  Each lane carries kT = 2
// terms (two independent recurrence chains per row); a ray uses
// P = ceil(np / kT) lanes and a warp holds floor(32 / P) rays.
//
// Per range step each lane runs ONE pass over its column:
//   * the back-substitution of the previous step's solves of its terms,
//   * the combination u_new = c_inf u_old + sum_j c_j x_j for the row: each
//     lane sums its terms, the ray's P lanes exchange their sums by shuffles
//     and add them in a fixed order (FP64, identical in every lane),
//   * the elimination of the next step's solves two rows behind, so that the
//     exchange latency is off the elimination's path,
// alternating the pass direction every step.  Every lane of a warp visits
// the same row index at the same iteration (the warp's deepest ray sets the
// count), so the warp runs in lockstep.  The Thomas factorisation of each
// term (1/den, the coupling factor and w per row, both directions) is
// computed once per change of the operator - profiles, bathymetry index or
// Pade set - and streamed from HBM, with the workspace g and the field, by
// the tensor memory accelerator: one lane issues one bulk tensor copy per
// field and block of kRB rows of the whole tile into a ring of blocks in
// shared memory, completing on the block's mbarrier, which every lane waits
// on before it reads the block; a slot is refilled only after every lane has
// used its rows.  Only 1/den and w are stored per term; the
// elimination's coupling factor -(a1 + pd2 e) / den is rebuilt in FP64 from
// 1/den and the row's Galerkin coupling e (d1 going down, d3 going up,
// complex128), which is stored once per ray row and shared by the ray's
// terms.  The solve loop
// handles kU rows per iteration so that one row's term exchange overlaps the
// next row's recurrences.
//
// The sum form is the reference's rational operator rearranged; on the
// golden cases it matches the product form to <= 5e-8 dB (oracle mode "sum").
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "march_common.cuh"
#include "march_sum.cuh"

namespace crk {

namespace {

constexpr int kSR = 8;                // factor passes: cp.async prefetch depth (rows) per lane
constexpr unsigned kRingWaitLimit = 1u << 22;  // polls of a ring block's mbarrier before giving up
static_assert((kRB & (kRB - 1)) == 0, "kRB must be a power of two");
#ifndef CR_SUM_ROWS
#define CR_SUM_ROWS 2
#endif
constexpr int kU = CR_SUM_ROWS;       // rows per solve-loop iteration
static_assert((kSR & (kSR - 1)) == 0, "kSR must be a power of two");
static_assert(kSR % kU == 0, "the prefetch ring must hold whole iterations");
static_assert(kRB % kU == 0, "a ring block must hold whole iterations");
#ifndef CR_SUM_BLOCK_UNROLL
#define CR_SUM_BLOCK_UNROLL (CR_SUM_RB / CR_SUM_ROWS)
#endif
constexpr int kBlockUnroll = CR_SUM_BLOCK_UNROLL;  // row steps of a steady block unrolled
#ifndef CR_SUM_BLOCK_UNROLL_REFINED
#define CR_SUM_BLOCK_UNROLL_REFINED 2
#endif
// the refined form's rows carry more state: a shorter unrolled body keeps it in registers
constexpr int kBlockUnrollRefined = CR_SUM_BLOCK_UNROLL_REFINED;

enum SumPass { kElimOnly = 0, kFusedP = 1, kBackOnly = 2, kFactor = 3, kRefineUp = 4 };

// Arithmetic forms of the march (template parameter F):
//   kPlain  (0): complex128 factors / workspace, FP64 recurrences;
//   kChosen (1): complex64 factors / workspace, FP32 recurrences, the terms
//                combined in FP64 and the history of the field in FP64;
//   kFast   (2): complex64 factors / workspace and an FP32 inner loop: the
//                elimination's coupling, M u, the term combination and the
//                exchange of the ray's shares all in FP32, the couplings
//                stored as complex64.
// The factorisation itself and the stored field stay FP64 / complex128 in
// every form.
constexpr int kPlain = 0, kChosen = 1, kFast = 2, kRefined = 3;

template <int F>
struct Form;
template <>
struct Form<kPlain> {
    using R = double;
    using V = double2;  // factors / workspace / recurrences
    using H = double2;  // field history and term combination
    using E = double2;  // stored Galerkin coupling
};
template <>
struct Form<kChosen> {
    using R = float;
    using V = float2;
    using H = double2;
    using E = double2;
};
template <>
struct Form<kRefined> {
    using R = float;
    using V = float2;
    using H = double2;
    using E = double2;
};
template <>
struct Form<kFast> {
    using R = float;
    using V = float2;
    using H = float2;
    using E = float2;
};

// Shared memory of a CTA (one warp), from its base:
//   * RingCtl (kCtlBytes): the ring's mbarriers and position, which persist
//     across the tiles a CTA marches;
//   * the solve passes' ring: kNB blocks (ring_blocks of the form), each
//     holding kRB rows of every field a solve pass streams, in 128-byte
//     aligned regions (RingLayout<F, P>): the ray fields u, e (and d1, d2) as
//     [kRB][floor(32 / P)] (the tile's rays), the lane fields w, g, q of each
//     term slot as [kRB][32];
//   * over the ring's bytes, the factor passes' cp.async ring, [kSR][2][32]
//     16-byte slots (f1..f3 and ksq of each lane's ray row): a factor pass
//     runs only between solve passes, whose copies have all landed.
__host__ __device__ constexpr int up128(int n) { return (n + 127) / 128 * 128; }
template <int F, int P>
struct RingLayout {
    using V = typename Form<F>::V;
    using E = typename Form<F>::E;
    static constexpr int R = kTile / P;  // rays of the tile
    static constexpr int kRay = up128(kRB * R * (int)sizeof(double2));  // u, d1, d2
    static constexpr int kE = up128(kRB * R * (int)sizeof(E));
    static constexpr int kLane = kRB * kTile * (int)sizeof(V);
    static constexpr int u = 0;
    static constexpr int e = u + kRay;
    static constexpr int w0 = e + kE;  // term slot t: w at w0 + 3 t kLane, then g, then q
    static constexpr int d1 = w0 + 3 * kT * kLane;
    static constexpr int d2 = d1 + kRay;
    static constexpr int block = F == kRefined ? d2 + kRay : d1;
    static constexpr int kNB = ring_blocks(F);
    static_assert(kLane % 128 == 0, "regions must stay 128-byte aligned");
};
struct RingCtl {
    unsigned long long bar[kNBMax];  // one mbarrier per ring block (arrival count 1 + the copies' bytes)
    unsigned seq;                    // ring blocks this CTA has consumed: slot seq % kNB, phase (seq / kNB) & 1
    unsigned dead;                   // a wait gave up: later waits are skipped and the CTA's rays are flagged
};
constexpr int kCtlBytes = 128;
static_assert(sizeof(RingCtl) <= kCtlBytes, "RingCtl must fit its slot");
constexpr int kFactorRing = kSR * 2 * kTile * (int)sizeof(double2);
// dynamic shared memory of a CTA marching tiles of P lanes per ray
template <int F, int P>
__host__ __device__ constexpr size_t smem_of() {
    using Lay = RingLayout<F, P>;
    return (size_t)kCtlBytes + (size_t)(Lay::kNB * Lay::block > kFactorRing ? Lay::kNB * Lay::block : kFactorRing);
}
struct SumSmem {
    double2 d[1];
};
__device__ __forceinline__ RingCtl* ring_ctl(SumSmem& S) { return reinterpret_cast<RingCtl*>(&S); }
template <int F, int P>
__device__ __forceinline__ unsigned char* ring_block(SumSmem& S, unsigned slot) {
    return reinterpret_cast<unsigned char*>(&S) + kCtlBytes + slot * (unsigned)RingLayout<F, P>::block;
}

__device__ __forceinline__ double2 up2(double2 v) { return v; }
__device__ __forceinline__ double2 up2(float2 v) { return make_double2((double)v.x, (double)v.y); }
template <typename T>
__device__ __forceinline__ T dn2(double2 v);
template <>
__device__ __forceinline__ double2 dn2<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 dn2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

// Prec<R>: the stored precision of the factors / workspace.
template <typename R>
struct Prec;
template <>
struct Prec<double> {
    using V = double2;
    __device__ static __forceinline__ V mk(double2 v) { return v; }
    __device__ static __forceinline__ double2 up(V v) { return v; }
};
template <>
struct Prec<float> {
    using V = float2;
    __device__ static __forceinline__ V mk(double2 v) { return make_float2((float)v.x, (float)v.y); }
    __device__ static __forceinline__ double2 up(V v) { return make_double2((double)v.x, (double)v.y); }
};

struct Lane {
    int lane, k, gbase, P;  // k: lane index within the ray's P lanes
    int rows;               // rows per lane column, common to the warp (its deepest ray's nz + 2)
    int span;               // iterations per pass: rows rounded up to a multiple of kU
    int nzmin;              // shallowest ray of the warp (bounds the unchecked iterations)
    int slot;               // the ray's index in the tile (its ray column)
    int yray, ylane;        // first tensor-map row of the tile's ray columns / lane columns
    unsigned gmask;         // lanes of this ray
    unsigned wmask;         // active lanes of the warp: every pass runs in lockstep over them
    long long rcol;         // ray column base (f1..f3, ksq, u)
    long long lcol;         // lane column base of term slot 0 (G and the factors)
    long long lstride;      // elements between term slots of a lane column
};

struct Ops {
    int nz;
    double cfact, a1, a2;
    double2 pole[kT];  // pd2 of this lane's terms in the active set
    double2 ck[kT];    // partial-fraction residues (0 for slots without a term)
    double2 cinf;      // c_inf of the ray for the active set
    // FP32 copies for the fast form's inner loop
    float a1f, a2f;
    float2 polef[kT], ckf[kT], cinff;
};

template <typename R>
__device__ __forceinline__ const typename Prec<R>::V* fac(const double2* p) {
    return reinterpret_cast<const typename Prec<R>::V*>(p);
}
template <typename R>
__device__ __forceinline__ typename Prec<R>::V* facw(double2* p) {
    return reinterpret_cast<typename Prec<R>::V*>(p);
}

// factor-pass ring slots of prefetch row k: f1..f3 and ksq of the lane's ray row
__device__ __forceinline__ double2* factor_slot(SumSmem& S, int k, int field, int lane) {
    return reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(&S) + kCtlBytes) + (k * 2 + field) * kTile +
           lane;
}
__device__ __forceinline__ float* sfl(SumSmem& S, int k, int lane) { return (float*)factor_slot(S, k, 0, lane); }
__device__ __forceinline__ float2* sks(SumSmem& S, int k, int lane) { return (float2*)factor_slot(S, k, 1, lane); }

// Stream row of iteration k: the same for every lane of the warp.
template <bool DOWN>
__device__ __forceinline__ int row_of(const Lane& L, int k) {
    return DOWN ? k : L.span - 1 - k;
}

// Copies for stream row r of a factor pass (one commit group, empty outside
// the lane's rows).
template <int F, bool DOWN>
__device__ __forceinline__ void sum_issue(const SumArgs& a, const Lane& L, SumSmem& S, int k, int r, int nz) {
    if (r >= 0 && r <= nz + 1) {
        const long long ro = L.rcol + (long long)r * kTile;
        float* f = sfl(S, k, L.lane);
        cp4(f + 0, a.f1 + ro);
        cp4(f + 1, a.f2 + ro);
        cp4(f + 2, a.f3 + ro);
        cp8(sks(S, k, L.lane), a.ksq + ro);
    }
    cp_commit();
}

// Column pointers of one solve pass (element 0 of the lane's columns).
template <int F>
struct PassPtrs {
    using V = typename Form<F>::V;
    using E = typename Form<F>::E;
    double2* u;        // field (ray column)
    const E* e;        // Galerkin coupling of this pass's elimination (ray column)
    const V* w[kT];    // w of the solves being back-substituted (eliminated the other way)
    V* g[kT];          // workspace: read by the back-substitution, rewritten by the elimination
    const V* q[kT];    // 1/den of this pass's elimination
    const double2* d1; // refined form: the Galerkin row's d1 and d2 (ray columns)
    const double2* d2;
};

template <int F, bool DOWN>
__device__ __forceinline__ PassPtrs<F> pass_ptrs(const SumArgs& a, const Lane& L) {
    using R = typename Form<F>::R;
    using E = typename Form<F>::E;
    PassPtrs<F> p;
    p.u = a.u + L.rcol;
    p.e = reinterpret_cast<const E*>(DOWN ? a.ED : a.EU) + L.rcol;
    p.d1 = a.ED + L.rcol;
    p.d2 = a.E2 ? a.E2 + L.rcol : nullptr;
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        const long long lo = L.lcol + t * L.lstride;
        p.w[t] = fac<R>(DOWN ? a.WU : a.WD) + lo;
        p.g[t] = facw<R>(a.G) + lo;
        p.q[t] = fac<R>(DOWN ? a.QD : a.QU) + lo;
    }
    return p;
}

// Lane 0: the bulk tensor copies of block b of a solve pass into ring slot
// `slot`, completing on the slot's mbarrier with the bytes it announces.  The
// block's stream iterations b kRB .. b kRB + kRB - 1 cover the memory rows
// lo .. lo + kRB - 1 (ascending in a DOWN pass, descending in an UP pass); the
// elimination's rows (e, q; d1 and d2 of the residual pass) lie two rows
// behind the stream, one in the refined form's residual pass.  Rows past the
// tile's own belong to neighbouring tiles or read as zeros outside the array:
// they are never used (the CHECK iterations select them away).
template <int F, int P, int PASS, bool DOWN>
__device__ __forceinline__ void ring_issue(const SumArgs& a, const Lane& L, SumSmem& S, int b, unsigned slot) {
    using Lay = RingLayout<F, P>;
    using V = typename Form<F>::V;
    using E = typename Form<F>::E;
    constexpr int R = kTile / P;
    constexpr unsigned kRayBox = kRB * R * sizeof(double2), kEBox = kRB * R * sizeof(E),
                       kLaneBox = kRB * kTile * sizeof(V);
    unsigned bytes = kRayBox;                                      // u
    if (PASS != kBackOnly) bytes += kEBox + kT * kLaneBox;         // e, q
    if (PASS != kElimOnly) bytes += 2 * kT * kLaneBox;             // w, g
    if (PASS == kRefineUp) bytes += 2 * kRayBox;                   // d1, d2
    const int lo = DOWN ? b * kRB : L.span - kRB - b * kRB;
    const int lm = PASS == kRefineUp ? lo + 1 : (DOWN ? lo - 2 : lo + 2);
    unsigned long long* bar = &ring_ctl(S)->bar[slot];
    unsigned char* blk = ring_block<F, P>(S, slot);
    const SumMaps& m = a.maps;
    mbar_expect(bar, bytes);
    tma_2d(blk + Lay::u, &m.ray[kMapU][P - 1], 0, L.yray + lo, bar);
    if (PASS != kBackOnly) tma_2d(blk + Lay::e, &m.ray[DOWN ? kMapED : kMapEU][P - 1], 0, L.yray + lm, bar);
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        const int yl = L.ylane + t * L.rows;
        unsigned char* tb = blk + Lay::w0 + 3 * t * Lay::kLane;
        if (PASS != kElimOnly) {
            tma_2d(tb, &m.lane[DOWN ? kMapWU : kMapWD], 0, yl + lo, bar);
            tma_2d(tb + Lay::kLane, &m.lane[kMapG], 0, yl + lo, bar);
        }
        if (PASS != kBackOnly) tma_2d(tb + 2 * Lay::kLane, &m.lane[DOWN ? kMapQD : kMapQU], 0, yl + lm, bar);
    }
    if constexpr (PASS == kRefineUp) {
        tma_2d(blk + Lay::d1, &m.ray[kMapED][P - 1], 0, L.yray + lm, bar);
        tma_2d(blk + Lay::d2, &m.ray[kMapE2][P - 1], 0, L.yray + lm, bar);
    }
}

// Thomas factorisation of (M + pole_t D) for this lane's terms, one direction.
// The arithmetic is FP64 in every form; 1/den and w are stored in the sweep
// precision, the row's Galerkin coupling in the form's coupling precision.
template <int F, bool DOWN>
__device__ void sum_factor(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o) {
    using R = typename Form<F>::R;
    using E = typename Form<F>::E;
    using P = Prec<R>;
    const int nz = o.nz;
    __threadfence_block();
#pragma unroll 1
    for (int k = 0; k < kSR; ++k) sum_issue<F, DOWN>(a, L, S, k, row_of<DOWN>(L, k), nz);
    EnvRow em{}, ec{}, ep{};
    double2 wp[kT];
#pragma unroll
    for (int t = 0; t < kT; ++t) wp[t] = c2(0.0, 0.0);
    typename P::V* Q = facw<R>(DOWN ? a.QD : a.QU);
    E* Ecol = reinterpret_cast<E*>(DOWN ? a.ED : a.EU);
    typename P::V* W = facw<R>(DOWN ? a.WD : a.WU);
    int seen = 0;  // rows of this lane already streamed
#pragma unroll 1
    for (int k = 0; k < L.span; ++k) {
        const int r = row_of<DOWN>(L, k);  // rows outside 0..nz+1: idle iterations
        const int slot = k & (kSR - 1);
        cp_wait<kSR - 1>();
        EnvRow er;
        {
            const float* f = sfl(S, slot, L.lane);
            er.f1 = f[0];
            er.f2 = f[1];
            er.f3 = f[2];
            er.k = *sks(S, slot, L.lane);
        }
        sum_issue<F, DOWN>(a, L, S, slot, row_of<DOWN>(L, k + kSR), nz);
        if (r < 0 || r > nz + 1) continue;
        if (DOWN) {
            em = ec;
            ec = ep;
            ep = er;
        } else {
            ep = ec;
            ec = em;
            em = er;
        }
        if (++seen < 3) continue;
        const int m = DOWN ? r - 1 : r + 1;
        if (m < 1 || m > nz) continue;
        const Drow d = galerkin3(em, ec, ep, o.cfact);
        if (L.k == 0) Ecol[L.rcol + (long long)m * kTile] = dn2<E>(DOWN ? d.d1 : d.d3);
        if constexpr (F == kRefined) {
            if (DOWN && L.k == 0) a.E2[L.rcol + (long long)m * kTile] = d.d2;
        }
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            const double2 r1 = caxpd(o.a1, o.pole[t], d.d1), r2 = caxpd(o.a2, o.pole[t], d.d2),
                          r3 = caxpd(o.a1, o.pole[t], d.d3);
            const double2 cin = DOWN ? r1 : r3, cout = DOWN ? r3 : r1;
            const double2 q = crcp(cfms(r2, cin, wp[t]));
            wp[t] = cmul(cout, q);
            const long long mo = L.lcol + t * L.lstride + (long long)m * kTile;
            Q[mo] = P::mk(q);
            W[mo] = P::mk(wp[t]);
        }
    }
    cp_wait<0>();
}

// g_m = q (M u)_m + al g_{m-/+1} for every term slot of the lane, with the
// coupling factor al = -(a1 + pole e) q rebuilt from the stored 1/den q and
// the row's Galerkin coupling e (the factorisation's own arithmetic).
// Plain and chosen form M u and the coupling in FP64; the fast form does the
// whole row in FP32 as g = q ((M u) - (a1 + pole e) g_prev).
template <int F>
__device__ __forceinline__ void elim_row(const Ops& o, typename Form<F>::H h3, typename Form<F>::H h2,
                                         typename Form<F>::H h1, typename Form<F>::E fe,
                                         const typename Form<F>::V* fq, typename Form<F>::V* gp) {
    using R = typename Form<F>::R;
    if constexpr (F == kFast) {
        const float mx = fmaf(o.a1f, h3.x + h1.x, o.a2f * h2.x), my = fmaf(o.a1f, h3.y + h1.y, o.a2f * h2.y);
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            // cin = a1 + pole e;  v = M u - cin g_prev;  g = q v
            const float cx = o.a1f + fmaf(o.polef[t].x, fe.x, -o.polef[t].y * fe.y);
            const float cy = fmaf(o.polef[t].x, fe.y, o.polef[t].y * fe.x);
            const float vx = fmaf(-cx, gp[t].x, fmaf(cy, gp[t].y, mx));
            const float vy = fmaf(-cx, gp[t].y, fmaf(-cy, gp[t].x, my));
            float2 g;
            g.x = fmaf(fq[t].x, vx, -fq[t].y * vy);
            g.y = fmaf(fq[t].x, vy, fq[t].y * vx);
            gp[t] = g;
        }
    } else {
        const double2 mud = c2(fma(o.a1, h3.x + h1.x, o.a2 * h2.x), fma(o.a1, h3.y + h1.y, o.a2 * h2.y));
        const R mx = (R)mud.x, my = (R)mud.y;
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            // a1 + pole e cancels strongly for some terms: formed in FP64 like the
            // factorisation, only al is rounded to the sweep precision
            const double2 cin = caxpd(o.a1, o.pole[t], fe);
            const double2 ci = cmul(cin, Prec<R>::up(fq[t]));
            const R ax = (R)(-ci.x), ay = (R)(-ci.y);
            const R tx = fma(fq[t].x, mx, -fq[t].y * my), ty = fma(fq[t].x, my, fq[t].y * mx);
            typename Prec<R>::V g;
            g.x = fma(ax, gp[t].x, fma(-ay, gp[t].y, tx));
            g.y = fma(ax, gp[t].y, fma(ay, gp[t].x, ty));
            gp[t] = g;
        }
    }
}

// One streamed row of a solve pass, in registers.
template <int F>
struct RowF {
    using V = typename Form<F>::V;
    double2 u;
    typename Form<F>::E e;
    V w[kT], g[kT], q[kT];
    double2 d1, d2;  // refined form, pass kRefineUp: the residual row's d1 and d2
};

// Row j (memory order) of a ring block, for this lane: the ray's u and e (d1,
// d2), the lane's w, g, q of each term slot - only what the pass uses.
template <int F, int P, int PASS>
__device__ __forceinline__ void load_row(const unsigned char* blk, int j, const Lane& L, RowF<F>& f) {
    using Lay = RingLayout<F, P>;
    using V = typename Form<F>::V;
    using E = typename Form<F>::E;
    constexpr int R = kTile / P;
    const int ri = j * R + L.slot, li = j * kTile + L.lane;
    f.u = reinterpret_cast<const double2*>(blk + Lay::u)[ri];
    if (PASS != kBackOnly) f.e = reinterpret_cast<const E*>(blk + Lay::e)[ri];
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        const unsigned char* tb = blk + Lay::w0 + 3 * t * Lay::kLane;
        if (PASS != kElimOnly) {
            f.w[t] = reinterpret_cast<const V*>(tb)[li];
            f.g[t] = reinterpret_cast<const V*>(tb + Lay::kLane)[li];
        }
        if (PASS != kBackOnly) f.q[t] = reinterpret_cast<const V*>(tb + 2 * Lay::kLane)[li];
    }
    if constexpr (PASS == kRefineUp) {
        f.d1 = reinterpret_cast<const double2*>(blk + Lay::d1)[ri];
        f.d2 = reinterpret_cast<const double2*>(blk + Lay::d2)[ri];
    }
}

// Carried state of a solve pass.
template <int F>
struct SolveState {
    using V = typename Form<F>::V;
    typename Form<F>::H h1, h2, h3;  // u_new of the last three rows (h1 newest)
    V xp[kT];                        // back-substitution chains
    V xq[kT];                        // refined form: the chains' values one row further back
    V gp[kT];                        // elimination chains
};

template <typename H>
__device__ __forceinline__ H hsel(bool c, H a, H b) {
    H r;
    r.x = c ? a.x : b.x;
    r.y = c ? a.y : b.y;
    return r;
}

// Stream row r of a solve pass.  The elimination of row m = r -/+ 2 uses
// (h3, h2, h1) = (u_{m-/+1}, u_m, u_{m+/-1}) and comes first; then the
// back-substitution x_r = g_r - w_r x_{r-/+1} of each term and this lane's
// share c_inf u_old (lane 0) + sum_t c_t x_t (FP64; FP32 in the fast form),
// and the exchange of the ray's P shares, added in lane order (identical in
// every lane).
// CHECK: rows outside a ray's column are handled with selects and predicated
// stores (branch-free); without CHECK, r and m are interior rows of every
// ray of the warp and r is no ray's first back-substitution row.
template <int F, int P, int PASS, bool DOWN, bool CHECK>
__device__ __forceinline__ void solve_row(const PassPtrs<F>& p, const Lane& L, const Ops& o, const RowF<F>& f,
                                          int r, SolveState<F>& st) {
    using R = typename Form<F>::R;
    using V = typename Form<F>::V;
    using H = typename Form<F>::H;
    const int nz = o.nz;
    const R zr = R(0);
    H hzero;
    hzero.x = 0;
    hzero.y = 0;
    const bool valid = CHECK ? ((r >= 0) & (r <= nz + 1)) : true;
    const bool interior = CHECK ? ((r >= 1) & (r <= nz)) : true;
    if (PASS != kBackOnly) {
        const int m = DOWN ? r - 2 : r + 2;
        const bool mvalid = CHECK ? (valid & (m >= 1) & (m <= nz)) : true;
        V g[kT];
#pragma unroll
        for (int t = 0; t < kT; ++t) g[t] = st.gp[t];
        elim_row<F>(o, st.h3, st.h2, st.h1, f.e, f.q, g);
        const int mo = (CHECK ? (mvalid ? m : 0) : m) * kTile;
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            if (mvalid) p.g[t][mo] = g[t];
            if (CHECK) {
                st.gp[t].x = mvalid ? g[t].x : st.gp[t].x;
                st.gp[t].y = mvalid ? g[t].y : st.gp[t].y;
            } else {
                st.gp[t] = g[t];
            }
        }
    }
    H un;
    if (PASS == kElimOnly) {
        un = interior ? dn2<H>(f.u) : hzero;
    } else {
        const bool first = CHECK ? (DOWN ? (r == 1) : (r == nz)) : false;
        H v;
        if constexpr (F == kFast) {
            const float2 uf = dn2<float2>(f.u);
            v.x = fmaf(o.cinff.x, uf.x, -o.cinff.y * uf.y);
            v.y = fmaf(o.cinff.x, uf.y, o.cinff.y * uf.x);
        } else {
            v = cmul(o.cinf, f.u);
        }
        v = hsel(L.k == 0, v, hzero);  // c_inf u_old is lane 0's share
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            V x;
            x.x = fma(-f.w[t].x, st.xp[t].x, fma(f.w[t].y, st.xp[t].y, f.g[t].x));
            x.y = fma(-f.w[t].x, st.xp[t].y, fma(-f.w[t].y, st.xp[t].x, f.g[t].y));
            if (CHECK) {
                x.x = first ? f.g[t].x : x.x;
                x.y = first ? f.g[t].y : x.y;
                x.x = interior ? x.x : zr;
                x.y = interior ? x.y : zr;
            }
            st.xp[t] = x;
            if constexpr (F == kFast) {
                v.x = fmaf(o.ckf[t].x, x.x, fmaf(-o.ckf[t].y, x.y, v.x));
                v.y = fmaf(o.ckf[t].x, x.y, fmaf(o.ckf[t].y, x.x, v.y));
            } else {
                const double2 xd = Prec<R>::up(x);
                v = c2(fma(o.ck[t].x, xd.x, fma(-o.ck[t].y, xd.y, v.x)),
                       fma(o.ck[t].x, xd.y, fma(o.ck[t].y, xd.x, v.y)));
            }
        }
        H sh[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            sh[j].x = __shfl_sync(L.wmask, v.x, L.gbase + j);
            sh[j].y = __shfl_sync(L.wmask, v.y, L.gbase + j);
        }
        H tot = sh[0];
#pragma unroll
        for (int j = 1; j < P; ++j) {
            tot.x += sh[j].x;
            tot.y += sh[j].y;
        }
        un = interior ? tot : hzero;
        if (interior & (L.k == 0)) p.u[(CHECK ? (interior ? r : 0) : r) * kTile] = up2(un);
    }
    if (CHECK) {
        st.h3 = hsel(valid, st.h2, st.h3);
        st.h2 = hsel(valid, st.h1, st.h2);
        st.h1 = hsel(valid, un, st.h1);
    } else {
        st.h3 = st.h2;
        st.h2 = st.h1;
        st.h1 = un;
    }
}

// Stream row r of the refined form's residual pass (UP, after the main
// solves were eliminated DOWN):
//   * back-substitution of the main solves, x~_r = g_r - w_r x~_{r+1} (FP32),
//     and the partial combination u^p_r = c_inf u_r + sum_t c_t x~_t,r (FP64,
//     exchanged over the ray's lanes), stored over u_r by lane 0;
//   * the FP64 residual of row m = r + 1 of each term,
//       res_m = (M u)_m - [(a1 + p d1) x~_{m-1} + (a2 + p d2) x~_m + (a1 + p d3) x~_{m+1}],
//     from the old field (every lane keeps its last rows) and the row's d1, d2,
//     d3 (d3 is the upward coupling e);
//   * the upward elimination of the correction system (M + p D) d = res with
//     the same complex64 factors, g'_m = q_m (res_m - (a1 + p d3) g'_{m+1}),
//     stored over g.
// The correction's back-substitution runs in the next (DOWN) pass, which adds
// sum_t c_t d_t to u^p.
template <int F, int P, bool CHECK>
__device__ __forceinline__ void refine_row(const PassPtrs<F>& p, const Lane& L, const Ops& o, const RowF<F>& f,
                                           int r, SolveState<F>& st) {
    using R = typename Form<F>::R;
    using V = typename Form<F>::V;
    const int nz = o.nz;
    const R zr = R(0);
    const double2 dz = c2(0.0, 0.0);
    const bool valid = CHECK ? ((r >= 0) & (r <= nz + 1)) : true;
    const bool interior = CHECK ? ((r >= 1) & (r <= nz)) : true;
    const bool first = CHECK ? (r == nz) : false;
    V x[kT];
    double2 v = L.k == 0 ? cmul(o.cinf, f.u) : dz;
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        x[t].x = fma(-f.w[t].x, st.xp[t].x, fma(f.w[t].y, st.xp[t].y, f.g[t].x));
        x[t].y = fma(-f.w[t].x, st.xp[t].y, fma(-f.w[t].y, st.xp[t].x, f.g[t].y));
        if (CHECK) {
            x[t].x = first ? f.g[t].x : x[t].x;
            x[t].y = first ? f.g[t].y : x[t].y;
            x[t].x = interior ? x[t].x : zr;
            x[t].y = interior ? x[t].y : zr;
        }
        const double2 xd = Prec<R>::up(x[t]);
        v = c2(fma(o.ck[t].x, xd.x, fma(-o.ck[t].y, xd.y, v.x)), fma(o.ck[t].x, xd.y, fma(o.ck[t].y, xd.x, v.y)));
    }
    double2 sh[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        sh[j].x = __shfl_sync(L.wmask, v.x, L.gbase + j);
        sh[j].y = __shfl_sync(L.wmask, v.y, L.gbase + j);
    }
    double2 tot = sh[0];
#pragma unroll
    for (int j = 1; j < P; ++j) {
        tot.x += sh[j].x;
        tot.y += sh[j].y;
    }
    if (interior & (L.k == 0)) p.u[(CHECK ? (interior ? r : 0) : r) * kTile] = tot;
    // residual and correction elimination of row m = r + 1
    const double2 uo = interior ? f.u : dz;  // u_r of the old field
    const int m = r + 1;
    const bool mvalid = CHECK ? (valid & (m >= 1) & (m <= nz)) : true;
    const double2 mu = c2(fma(o.a1, uo.x + st.h2.x, o.a2 * st.h1.x), fma(o.a1, uo.y + st.h2.y, o.a2 * st.h1.y));
    const int mo = (CHECK ? (mvalid ? m : 0) : m) * kTile;
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        const double2 r1 = caxpd(o.a1, o.pole[t], f.d1), r2 = caxpd(o.a2, o.pole[t], f.d2),
                      r3 = caxpd(o.a1, o.pole[t], f.e);
        const double2 xm1 = Prec<R>::up(x[t]), xm = Prec<R>::up(st.xp[t]), xp1 = Prec<R>::up(st.xq[t]);
        double2 res = mu;
        res = cfms(res, r1, xm1);
        res = cfms(res, r2, xm);
        res = cfms(res, r3, xp1);
        // g' = q res + al g'_prev, al = -(a1 + p d3) q, as the main elimination
        const double2 ci = cmul(r3, Prec<R>::up(f.q[t]));
        const R ax = (R)(-ci.x), ay = (R)(-ci.y);
        const R rx = (R)res.x, ry = (R)res.y;
        const R tx = fma(f.q[t].x, rx, -f.q[t].y * ry), ty = fma(f.q[t].x, ry, f.q[t].y * rx);
        V g;
        g.x = fma(ax, st.gp[t].x, fma(-ay, st.gp[t].y, tx));
        g.y = fma(ax, st.gp[t].y, fma(ay, st.gp[t].x, ty));
        if (mvalid) p.g[t][mo] = g;
        if (CHECK) {
            st.gp[t].x = mvalid ? g.x : st.gp[t].x;
            st.gp[t].y = mvalid ? g.y : st.gp[t].y;
        } else {
            st.gp[t] = g;
        }
        st.xq[t] = st.xp[t];
        st.xp[t] = x[t];
    }
    if (CHECK) {
        st.h2 = hsel(valid, st.h1, st.h2);
        st.h1 = hsel(valid, uo, st.h1);
    } else {
        st.h2 = st.h1;
        st.h1 = uo;
    }
}

// Position of a solve pass in the CTA's ring.
struct RingPos {
    unsigned seq0;  // ring sequence number of the pass's block 0
    int nblk;       // blocks of the pass
    bool dead;      // a wait gave up (this pass or earlier): wait no more
};

// After the last rows of block b have been used: slot `slot` gets block
// b + kNB.  The bulk copy writes shared memory directly, not through the
// load/store pipeline, so it is not ordered behind loads still queued there
// (other CTAs' shared-memory traffic can hold them back): every lane's loads
// of the block have been consumed by arithmetic before this point, each
// lane's proxy fence orders its reads before the async-proxy writes, and the
// warp synchronises before lane 0 issues.
template <int F, int P, int PASS, bool DOWN>
__device__ __forceinline__ void ring_refill(const SumArgs& a, const Lane& L, SumSmem& S, int b, unsigned slot,
                                            const RingPos& rp) {
    constexpr int NB = RingLayout<F, P>::kNB;
    if (b + NB >= rp.nblk) return;  // warp-uniform
    fence_proxy_async_shared();
    __syncwarp(L.wmask);
    if (L.lane == 0) ring_issue<F, P, PASS, DOWN>(a, L, S, b + NB, slot);
}

// Iterations [k0, k1) of a solve pass, kU rows each.  At the first iteration
// of a block every lane waits for the block's copies; once every lane has
// used the block's last rows, lane 0 refills the slot with block b + kNB.
template <int F, int P, int PASS, bool DOWN, bool CHECK>
__device__ __forceinline__ void solve_iters(const SumArgs& a, const PassPtrs<F>& p, const Lane& L, SumSmem& S,
                                            const Ops& o, int k0, int k1, SolveState<F>& st, RingPos& rp) {
    constexpr int NB = RingLayout<F, P>::kNB;
    // ring slot and mbarrier phase of the block holding iteration k, kept
    // up to date as k crosses block boundaries
    const unsigned q0 = rp.seq0 + (unsigned)(k0 / kRB);
    unsigned slot = q0 % NB, parity = (q0 / NB) & 1u;
#pragma unroll 1
    for (int k = k0; k < k1; k += kU) {
        const int b = k / kRB, jk = k % kRB;
        if (jk == 0 && k != k0 && ++slot == NB) {
            slot = 0;
            parity ^= 1u;
        }
        const unsigned char* blk = ring_block<F, P>(S, slot);
        if (jk == 0 && !rp.dead) rp.dead = !mbar_wait_bounded(&ring_ctl(S)->bar[slot], parity, kRingWaitLimit);
        RowF<F> f[kU];
#pragma unroll
        for (int j = 0; j < kU; ++j) load_row<F, P, PASS>(blk, DOWN ? jk + j : kRB - 1 - jk - j, L, f[j]);
#pragma unroll
        for (int j = 0; j < kU; ++j) {
            if constexpr (PASS == kRefineUp) refine_row<F, P, CHECK>(p, L, o, f[j], row_of<DOWN>(L, k + j), st);
            else solve_row<F, P, PASS, DOWN, CHECK>(p, L, o, f[j], row_of<DOWN>(L, k + j), st);
        }
        if (jk + kU == kRB) ring_refill<F, P, PASS, DOWN>(a, L, S, b, slot, rp);
    }
}

// Whole blocks [b0, b1) of a solve pass whose rows need no checks: one wait
// per block, then its kRB rows, kU per step, with the refill after the last
// rows are used.
template <int F, int P, int PASS, bool DOWN>
__device__ __forceinline__ void solve_blocks(const SumArgs& a, const PassPtrs<F>& p, const Lane& L, SumSmem& S,
                                             const Ops& o, int b0, int b1, SolveState<F>& st, RingPos& rp) {
    constexpr int NB = RingLayout<F, P>::kNB;
    unsigned q = rp.seq0 + (unsigned)b0;
    unsigned slot = q % NB, parity = (q / NB) & 1u;
    unsigned long long* bars = ring_ctl(S)->bar;
#pragma unroll 1
    for (int b = b0; b < b1; ++b) {
        const unsigned char* blk = ring_block<F, P>(S, slot);
        if (!rp.dead) rp.dead = !mbar_wait_bounded(&bars[slot], parity, kRingWaitLimit);
        constexpr int kUnroll = F == kRefined ? kBlockUnrollRefined : kBlockUnroll;
#pragma unroll kUnroll
        for (int jj = 0; jj < kRB; jj += kU) {
            RowF<F> f[kU];
#pragma unroll
            for (int j = 0; j < kU; ++j) load_row<F, P, PASS>(blk, DOWN ? jj + j : kRB - 1 - jj - j, L, f[j]);
#pragma unroll
            for (int j = 0; j < kU; ++j) {
                const int r = row_of<DOWN>(L, b * kRB + jj + j);
                if constexpr (PASS == kRefineUp) refine_row<F, P, false>(p, L, o, f[j], r, st);
                else solve_row<F, P, PASS, DOWN, false>(p, L, o, f[j], r, st);
            }
            if (jj + kU == kRB) ring_refill<F, P, PASS, DOWN>(a, L, S, b, slot, rp);
        }
        if (++slot == NB) {
            slot = 0;
            parity ^= 1u;
        }
    }
}

// One solve pass.  kElimOnly: eliminate from the stored field u.  kFusedP:
// back-substitute the pending solves, combine the terms into u_new (stored
// by lane 0 of the ray), eliminate the next solves.  kBackOnly:
// back-substitute and combine only.  Rows are streamed in the pass
// direction, kU per iteration, in ring blocks of kRB rows.
template <int F, int P, int PASS, bool DOWN>
__device__ void sum_pass(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o) {
    using V = typename Form<F>::V;
    using H = typename Form<F>::H;
    const int nz = o.nz;
    const PassPtrs<F> p = pass_ptrs<F, DOWN>(a, L);
    RingCtl* ctl = ring_ctl(S);
    // The field, the workspace and the factors were last written by generic
    // stores of every lane (the previous pass or factorisation), and the
    // factor ring by cp.async; lane 0's bulk copies read them through the
    // async proxy, from L2.  Each lane's stores must have reached GPU scope
    // (not only this CTA's view) before the copies are issued: the first
    // rows a pass loads are the last ones the previous pass wrote.
    __threadfence();
    fence_proxy_async();
    __syncwarp(L.wmask);
    RingPos rp;
    rp.seq0 = ctl->seq;
    rp.dead = ctl->dead != 0;
    rp.nblk = (L.span + kRB - 1) / kRB;
    if (L.lane == 0) {
        constexpr int NB = RingLayout<F, P>::kNB;
#pragma unroll 1
        for (int b = 0; b < NB && b < rp.nblk; ++b) ring_issue<F, P, PASS, DOWN>(a, L, S, b, (rp.seq0 + b) % NB);
    }
    SolveState<F> st;
    st.h1.x = st.h1.y = 0;
    st.h2 = st.h3 = st.h1;
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        st.xp[t].x = st.xp[t].y = 0;
        st.xq[t].x = st.xq[t].y = 0;
        st.gp[t].x = st.gp[t].y = 0;
    }
    // Iterations whose rows r (and elimination rows) are interior rows of
    // every ray of the warp, and past every first back-substitution row, run
    // unchecked, in whole blocks:  DOWN: 3 <= r <= nzmin;  UP: 1 <= r <= nzmin - 2.
    const int lb = DOWN ? 3 : L.span + 1 - L.nzmin;            // first steady iteration
    const int ub = DOWN ? L.nzmin + 1 - kU : L.span - kU - 1;  // last steady start
    const int b_lo = (max(lb, 0) + kRB - 1) / kRB;
    const int b_hi = max(b_lo, (ub + kU) / kRB);  // blocks [b_lo, b_hi) lie in [lb, ub + kU)
    const int k_lo = min(L.span, b_lo * kRB), k_hi = min(L.span, b_hi * kRB);
    // checked iterations before and after the steady blocks (one copy of
    // the checked loop)
#pragma unroll 1
    for (int seg = 0; seg < 2; ++seg) {
        solve_iters<F, P, PASS, DOWN, true>(a, p, L, S, o, seg ? k_hi : 0, seg ? L.span : k_lo, st, rp);
        if (seg == 0) solve_blocks<F, P, PASS, DOWN>(a, p, L, S, o, k_lo / kRB, k_hi / kRB, st, rp);
    }
    // The last row to eliminate (m = nz DOWN, m = 1 UP) would need stream row
    // nz+2 / -1; its window (u_{m-1}, u_m, u_{m+1}) is already in the history.
    // (The residual pass eliminates one row behind the stream: row 1 came with
    // stream row 0.)
    if (PASS == kElimOnly || PASS == kFusedP) {
        const int m = DOWN ? nz : 1;
        V fq[kT];
#pragma unroll
        for (int t = 0; t < kT; ++t) fq[t] = p.q[t][m * kTile];
        elim_row<F>(o, st.h3, st.h2, st.h1, p.e[m * kTile], fq, st.gp);
#pragma unroll
        for (int t = 0; t < kT; ++t) p.g[t][m * kTile] = st.gp[t];
    }
    (void)sizeof(H);
    // every block of the pass has been waited for: the ring is idle
    const bool dead = __any_sync(L.wmask, rp.dead);
    if (L.lane == 0) {
        ctl->seq = rp.seq0 + (unsigned)rp.nblk;
        ctl->dead = dead ? 1u : 0u;
    }
    __threadfence_block();
    __syncwarp(L.wmask);
}

// TL line / grid and CP line / grid of the field stored in the ray column.
__device__ void sum_outputs(const SumArgs& a, const RayDev& ry, const Lane& L, int tlc, double r, int ir,
                            double dir, int* flag) {
    if (L.k != 0 || tlc < 0 || tlc >= ry.nvr) return;
    auto urow = [&](int i) -> double2 {
        if (i <= 0 || i > ry.nz) return c2(0.0, 0.0);
        return a.u[L.rcol + (long long)i * kTile];
    };
    const double2 ua = urow(ir), ub = urow(ir + 1);
    const double fa = a.f3[L.rcol + (long long)ir * kTile];
    const double fb = a.f3[L.rcol + (long long)(ir + 1) * kTile];
    const double2 cp = c2((1.0 - dir) * fa * ua.x + dir * fb * ub.x, (1.0 - dir) * fa * ua.y + dir * fb * ub.y);
    const double amp = hypot(cp.x, cp.y);
    if (!isfinite(amp)) *flag |= 1;
    a.tll[ry.line_off + tlc] = tl_db(amp, r);
    a.cpl[ry.line_off + tlc] = cp;
    if (a.compute_grids && ry.grid_off >= 0) {
        for (int j = 0; j < ry.nvz; ++j) {
            const int row = (j + 1) * ry.ndz;
            if (row > ry.nz + 1) break;
            const double2 uj = urow(row);
            const double fj = a.f3[L.rcol + (long long)row * kTile];
            const double2 g = c2(uj.x * fj, uj.y * fj);
            const long long o = ry.grid_off + (long long)j * ry.nvr + tlc;
            a.tlg[o] = tl_db(hypot(g.x, g.y), r);
            a.cpg[o] = g;
        }
    }
}

// Poles and residues of this lane's term slots (term j = k + t P) in a set.
__device__ void set_ops(const SumArgs& a, int rid, int set, const Lane& L, Ops* o) {
    const int n = a.pd_n[rid * kSets + set];
    const long long base = ((long long)rid * kSets + set) * CR_MAX_NP;
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        const int j = L.k + t * L.P;
        // slots without a term solve a copy of term 0 with weight 0
        o->pole[t] = a.pd2[base + (j < n ? j : 0)];
        o->ck[t] = j < n ? a.pfc[base + j] : c2(0.0, 0.0);
        o->polef[t] = dn2<float2>(o->pole[t]);
        o->ckf[t] = dn2<float2>(o->ck[t]);
    }
    o->cinf = a.pfcinf[(long long)rid * kSets + set];
    o->cinff = dn2<float2>(o->cinf);
}

template <int F>
__device__ void sum_refactor(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o) {
    sum_factor<F, true>(a, L, S, o);
    sum_factor<F, false>(a, L, S, o);
    __threadfence_block();
    __syncwarp(L.wmask);
}

// Completion of a pending step of the refined form (its main solves were
// eliminated DOWN): the residual pass (UP) back-substitutes them into u^p and
// eliminates the FP64-residual correction; the DOWN pass back-substitutes the
// correction and adds it, u = u^p + sum_t c_t d_t (the combination with
// c_inf = 1 over the stored u^p), and - fused - eliminates the next step
// DOWN, so that every step's main solves run the same way.
template <int F, int P>
__device__ __forceinline__ void refine_step(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o, bool fused) {
    if constexpr (F == kRefined) {
        sum_pass<F, P, kRefineUp, false>(a, L, S, o);
        Ops o1 = o;
        o1.cinf = c2(1.0, 0.0);
        o1.cinff = make_float2(1.0f, 0.0f);
        if (fused) sum_pass<F, P, kFusedP, true>(a, L, S, o1);
        else sum_pass<F, P, kBackOnly, true>(a, L, S, o1);
    }
}

// The whole march of tile t (self-starter, every range step, the outputs) by
// the calling warp; lanes without a ray return at once.
template <int F, int P>
__device__ __forceinline__ void march_tile(const SumArgs& a, SumSmem& S, int t) {
    Lane L;
    L.lane = threadIdx.x;
    L.P = P;
    const int rid = a.tile_ray[t * kTile + L.lane];
    L.wmask = __ballot_sync(0xffffffffu, rid >= 0);
    if (rid < 0 || a.tile_G[t] != P) return;
    L.k = L.lane % L.P;
    L.gbase = L.lane - L.k;
    L.gmask = (L.P >= 32 ? 0xffffffffu : ((1u << L.P) - 1u)) << L.gbase;
    const RayDev ry = a.rays[rid];
    L.rcol = ry.col;
    L.lcol = a.tile_loff[t] + L.lane;
    L.slot = (int)(ry.col % kTile);
    L.yray = (int)(ry.col / kTile);
    L.ylane = (int)(a.tile_loff[t] / kTile);
    // the warp marches in lockstep: every pass covers the deepest ray's rows,
    // the step loop the longest ray's steps
    L.rows = (int)__reduce_max_sync(L.wmask, (unsigned)(ry.nz + 2));
    L.span = (L.rows + kU - 1) / kU * kU;
    L.nzmin = (int)__reduce_min_sync(L.wmask, (unsigned)ry.nz);
    L.lstride = (long long)L.rows * kTile;
    const int nr_max = (int)__reduce_max_sync(L.wmask, (unsigned)ry.nr);
    const EnvPtrs e = env_ptrs(a.envs[ry.env], a.pool);
    const int nz = ry.nz;
    int flag = 0;
    Ops o;
    o.nz = nz;
    o.cfact = 0.5 / (ry.dz * ry.dz);
    o.a1 = ry.k0 * ry.k0 / 6.0;
    o.a2 = 2.0 * ry.k0 * ry.k0 / 3.0;
    o.a1f = (float)o.a1;
    o.a2f = (float)o.a2;

    // initial profiles, split over the ray's lanes (cupyram.py:571-608, profl)
    int iz = max(1, min(nz - 1, (int)floor(e.zb[0] / ry.dz)));
    int ss = 0, sb = 0, bt = 0;
    for (int i = L.k; i <= nz + 1; i += L.P) {
        assemble_rows(ry, e, ss, sb, iz, i, i, a.f1, a.f2, a.f3, a.ksq);
        a.u[L.rcol + (long long)i * kTile] = c2(0.0, 0.0);
    }
    __threadfence_block();
    __syncwarp(L.wmask);
    // self-starter delta (cupyram.py:1008-1022)
    if (L.k == 0) {
        const double si = ry.zs / ry.dz;
        const int is = (int)floor(si);
        const double dis = si - is;
        const double amp = sqrt(2.0 * M_PI / ry.k0);
        const double step = ry.zmax / (double)(nz + 1);
        for (int q = 0; q < 2; ++q) {
            const int i = is + q;
            const double z = (i == nz + 1) ? ry.zmax : (double)i * step;
            const RowProps p = row_props(e, ss, sb, z, ry.lyrw_lambda, ry.attnf);
            const double alpw = sqrt((double)p.cw / ry.c0);
            const double wgt = (q == 0) ? (1.0 - dis) : dis;
            if (i >= 1 && i <= nz) a.u[L.rcol + (long long)i * kTile] = c2(wgt * amp / (ry.dz * alpw), 0.0);
        }
    }
    __threadfence_block();
    __syncwarp(L.wmask);

    const double ri = ry.zr / ry.dz;
    const int ir = (int)floor(ri);
    const double dir = ri - ir;
    int mdr = 0, tlc = -1;

    // The step whose back-substitution is pending (warp-uniform direction);
    // pend_valid is per ray: false once a ray has emitted its last step.
    bool pend_down = true;
    bool pend_valid = false;
    bool pend_out = false;
    double pend_r = 0.0;

    // the output of the pending step is written once its back-substitution
    // has stored the field (pass-level bookkeeping, inlined by hand so that
    // no local escapes into a call and the lane state stays in registers)
#define CR_FINISH_PENDING()                                                 \
    do {                                                                    \
        if (pend_valid && pend_out && ++mdr == ry.ndr) {                    \
            mdr = 0;                                                        \
            ++tlc;                                                          \
            sum_outputs(a, ry, L, tlc, pend_r, ir, dir, &flag);             \
        }                                                                   \
        pend_valid = false;                                                 \
        __syncwarp(L.wmask);                                                \
    } while (0)
#define CR_BACK_ONLY()                                                      \
    do {                                                                    \
        if constexpr (F == kRefined) refine_step<F, P>(a, L, S, o, false);  \
        else if (pend_down) sum_pass<F, P, kBackOnly, false>(a, L, S, o);   \
        else sum_pass<F, P, kBackOnly, true>(a, L, S, o);                   \
        CR_FINISH_PENDING();                                                \
    } while (0)

    // self-starter: two steps of 1/(1-X), one of the ip=2 operator
    set_ops(a, rid, 0, L, &o);
    sum_refactor<F>(a, L, S, o);
    sum_pass<F, P, kElimOnly, true>(a, L, S, o);
    pend_down = true;
    pend_valid = true;
    pend_out = false;
    if constexpr (F == kRefined) {
        refine_step<F, P>(a, L, S, o, true);  // complete step 1, eliminate step 2 (DOWN)
    } else {
        sum_pass<F, P, kFusedP, false>(a, L, S, o);  // back-substitute step 1, eliminate step 2 (UP)
    }
    CR_FINISH_PENDING();
    pend_down = F == kRefined;
    pend_valid = true;
    CR_BACK_ONLY();
    set_ops(a, rid, 1, L, &o);
    sum_refactor<F>(a, L, S, o);
    sum_pass<F, P, kElimOnly, true>(a, L, S, o);
    pend_down = true;
    pend_valid = true;
    pend_out = true;
    pend_r = ry.dr;  // first output at r = dr (cupyram.py:703)

    int set = 2;
    double rs = ry.rs;
    double r = ry.dr;
    bool first_march = true;
    for (int rn = 0; rn < nr_max; ++rn) {
        const bool live = rn < ry.nr;
        // updat (updat.py:38-140) for the step about to be taken
        bool reprofile = false;
        int iz_new = iz;
        int new_set = set;
        bool change = false;
        if (live) {
            if (e.n_bt > 1) {
                while (bt < e.n_bt - 1 && r >= e.rb[bt + 1]) ++bt;
                const int b1 = min(bt + 1, e.n_bt - 1);
                const double r0 = e.rb[bt], r1 = e.rb[b1], z0 = e.zb[bt], z1 = e.zb[b1];
                const double zc = (b1 == bt) ? z0 : z0 + (r + 0.5 * ry.dr - r0) * (z1 - z0) / (r1 - r0);
                iz_new = max(1, min(nz - 1, (int)floor(zc / ry.dz)));
            }
            if (e.n_rss > 1) {
                const int o2 = ss;
                while (ss < e.n_rss - 1 && r >= e.rp_ss[ss + 1]) ++ss;
                reprofile |= (ss != o2);
            }
            if (e.n_rsb > 1) {
                const int o2 = sb;
                while (sb < e.n_rsb - 1 && r >= e.rp_sb[sb + 1]) ++sb;
                reprofile |= (sb != o2);
            }
            if (r >= rs) {  // stability constraints off (cupyram.py:976-999)
                new_set = 3;
                rs = INFINITY;
            }
            change = first_march || reprofile || iz_new != iz || new_set != set;
        }
        const double r_out = (double)(rn + 2) * ry.dr;
        if (__any_sync(L.wmask, change)) {
            // some ray of the warp changes its operator: finish the pending
            // step alone, rebuild where needed, start this step from u
            CR_BACK_ONLY();
            if (change) {
                if (reprofile) {
                    for (int i = L.k; i <= nz + 1; i += L.P) assemble_rows(ry, e, ss, sb, iz_new, i, i, a.f1, a.f2, a.f3, a.ksq);
                } else if (iz_new != iz) {
                    const int lo = min(iz, iz_new) + 1, hi = max(iz, iz_new);
                    for (int i = lo + L.k; i <= hi; i += L.P) assemble_rows(ry, e, ss, sb, iz_new, i, i, a.f1, a.f2, a.f3, a.ksq);
                }
                __threadfence_block();
                __syncwarp(L.gmask);
                iz = iz_new;
                set = new_set;
                set_ops(a, rid, set, L, &o);
                sum_factor<F, true>(a, L, S, o);
                sum_factor<F, false>(a, L, S, o);
                __threadfence_block();
            }
            __syncwarp(L.wmask);
            sum_pass<F, P, kElimOnly, true>(a, L, S, o);
            pend_down = true;
            first_march = false;
        } else {
            // back-substitute the pending step and eliminate this one in one
            // pass (the refined form: its two passes, the second fused)
            if constexpr (F == kRefined) {
                refine_step<F, P>(a, L, S, o, true);
            } else {
                if (pend_down) sum_pass<F, P, kFusedP, false>(a, L, S, o);
                else sum_pass<F, P, kFusedP, true>(a, L, S, o);
            }
            CR_FINISH_PENDING();
            if constexpr (F != kRefined) pend_down = !pend_down;
        }
        pend_valid = live;
        pend_out = live;
        pend_r = r_out;
        r = r_out;
    }
    CR_BACK_ONLY();
    if (ring_ctl(S)->dead) flag |= 2;  // a wait on the ring gave up: the outputs are not to be trusted
    if (L.k == 0) a.flags[rid] = flag;
}

#undef CR_FINISH_PENDING
#undef CR_BACK_ONLY

// The ring's mbarriers, initialised by lane 0 before any copy is issued.
template <int F>
__device__ __forceinline__ void ring_init(SumSmem& S) {
    RingCtl* c = ring_ctl(S);
    if (threadIdx.x == 0) {
        for (int i = 0; i < ring_blocks(F); ++i) mbar_init1(&c->bar[i]);
        c->seq = 0;
        c->dead = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
}

// One tile per CTA (one launch per lanes-per-ray value P).
template <int F, int P>
__global__ void __launch_bounds__(kTile) march_sum_kernel(const __grid_constant__ SumArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SumSmem& S = *reinterpret_cast<SumSmem*>(smem_raw);
    ring_init<F>(S);
    march_tile<F, P>(a, S, a.tile_begin + blockIdx.x);
}

template <int F, int P = 1>
__device__ __forceinline__ void march_tile_p(const SumArgs& a, SumSmem& S, int t, int p) {
    if constexpr (P <= kMaxP) {
        if (p == P) march_tile<F, P>(a, S, t);
        else march_tile_p<F, P + 1>(a, S, t, p);
    }
}

// Persistent march over every batched tile of the engine: each CTA (one
// warp) takes the next tile from the device work queue - an atomic ticket
// over a.queue, the tiles in longest-march-first order - until the queue is
// empty, whatever its lanes per ray.  Taking a ticket never waits.
template <int F>
__global__ void __launch_bounds__(kTile) march_sum_queue_kernel(const __grid_constant__ SumArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SumSmem& S = *reinterpret_cast<SumSmem*>(smem_raw);
    ring_init<F>(S);
    for (;;) {
        int k = 0;
        if (threadIdx.x == 0) k = atomicAdd(a.ticket, 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= a.n_queue) break;
        const int t = a.queue[k];
        march_tile_p<F>(a, S, t, a.tile_G[t]);
        __syncwarp();
    }
}

// Sets the kernel's shared-memory limit; the first such call also loads the
// kernel, which is then not loaded at its first launch (a load while other
// streams' kernels run waits for them).
template <int F, int P>
static cudaError_t prepare_one() {
    return cudaFuncSetAttribute(march_sum_kernel<F, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_of<F, P>());
}

template <int F, int P>
static cudaError_t launch_one(const SumArgs& a, int count, cudaStream_t st) {
    const cudaError_t ce = prepare_one<F, P>();
    if (ce != cudaSuccess) return ce;
    march_sum_kernel<F, P><<<count, kTile, smem_of<F, P>(), st>>>(a);
    return cudaGetLastError();
}

template <int F, int P = 1>
static cudaError_t launch_p(const SumArgs& a, int p, int count, cudaStream_t st, bool launch) {
    if constexpr (P > kMaxP) {
        return cudaErrorInvalidValue;
    } else {
        if (p == P) return launch ? launch_one<F, P>(a, count, st) : prepare_one<F, P>();
        return launch_p<F, P + 1>(a, p, count, st, launch);
    }
}

// shared memory of the persistent launch: the largest need of the tiles' P
// values, i.e. that of the smallest P present
template <int F, int P = 1>
static size_t smem_from_p(int p) {
    if constexpr (P >= kMaxP) return smem_of<F, kMaxP>();
    else return p <= P ? smem_of<F, P>() : smem_from_p<F, P + 1>(p);
}

template <int F>
static cudaError_t launch_queue_f(const SumArgs& a, int n_tiles, cudaStream_t st, int* ctas, bool launch) {
    const size_t smem = smem_from_p<F>(a.min_p);
    cudaError_t ce = cudaFuncSetAttribute(march_sum_queue_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem);
    if (ce != cudaSuccess || !launch) return ce;
    int dev = 0, sms = 0, per_sm = 0;
    ce = cudaGetDevice(&dev);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (ce == cudaSuccess)
        ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, march_sum_queue_kernel<F>, kTile, smem);
    if (ce != cudaSuccess) return ce;
    // every resident slot of the device (or a.max_ctas), and no more CTAs than tiles
    const int slots = a.max_ctas > 0 ? a.max_ctas : std::max(1, per_sm) * sms;
    *ctas = std::max(1, std::min(n_tiles, slots));
    march_sum_queue_kernel<F><<<*ctas, kTile, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

}  // namespace crk
