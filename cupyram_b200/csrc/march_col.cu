// march_col.cu - column-parallel range march for deep grids and few rays.
//
// The batched march (march_sum.cu) gives a ray a few lanes of one warp, so a
// ray advances one depth row at a time: a batch of a handful of rays - a
// single Pekeris run, or the few very long rays of an uneven batch - leaves
// the GPU idle and takes nz x nr dependent row steps.  This kernel spreads
// one ray over a thread-block cluster of C CTAs instead:
//
//   * the column's rows 1..nz are cut into C slices, one per CTA; a CTA
//     keeps the field, the Thomas factors and the workspace of every Pade
//     term for its slice (plus one halo row each side) in shared memory;
//   * a CTA runs one warp per term of the partial-fraction form (the terms
//     of a step are independent solves (M + pd2_k D) x_k = M u), and a
//     warp's 32 lanes cut the slice into 32 segments;
//   * the term's Thomas recurrences - g_m = q_m b_m + al_m g_{m-1} down the
//     column, x_m = g_m - w_m x_{m+1} up - are first-order linear maps, so
//     each segment sweeps its rows from zero (its affine map), the warp
//     scans the 32 maps with shuffles, and the CTAs of the cluster exchange
//     one map per term (distributed shared memory) to fold in the slices
//     above (elimination) or below (back-substitution):
//         sweep 1: segment maps of the elimination; warp scan; cluster fold;
//         sweep 2: true g, stored;
//         sweep 3: segment maps of the back-substitution; scan; fold;
//         sweep 4: true x, stored;
//   * the terms are combined in the CTA, u_new = c_inf u + sum_k c_k x_k
//     (FP64, terms in order), including the two halo rows: the row below
//     the slice from the back-substitution's entry values, the row above
//     from the elimination's entry values and w of that row.  Nothing but
//     the 2 x np maps of a step crosses between CTAs.
//
// The Thomas factorisation of each term (1/den, al = -(a1 + p d1)/den and
// w per row, top-down) is recomputed when the operator changes (profiles,
// bathymetry index, Pade set) by the same segment / scan / fold scheme: the
// recurrence for w is linear in homogeneous coordinates (col_factor), so a
// refactorisation costs about one step, however often a sloping bottom
// moves the bathymetry index.
//
// Range logic, self-starter and outputs follow the batched march
// (cupyram/cupyram.py:273-380 run, :1001-1063 selfs, updat.py:38-140,
// outpt.py:11-57); only the association of the arithmetic differs.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "march_col.cuh"
#include "march_common.cuh"

namespace cg = cooperative_groups;

namespace crk {

namespace {

constexpr int kColMaxTerms = CR_MAX_NP;
constexpr int kColMaxCluster = 16;
constexpr size_t kColSmemLimit = 227 * 1024;

template <typename R>
struct CV;
template <>
struct CV<double> {
    using V = double2;
    __device__ static __forceinline__ V mk(double2 v) { return v; }
    __device__ static __forceinline__ double2 up(V v) { return v; }
};
template <>
struct CV<float> {
    using V = float2;
    __device__ static __forceinline__ V mk(double2 v) { return make_float2((float)v.x, (float)v.y); }
    __device__ static __forceinline__ double2 up(V v) { return make_double2((double)v.x, (double)v.y); }
};

template <typename V>
__device__ __forceinline__ V vmul(V a, V b) {
    V r;
    r.x = fma(a.x, b.x, -a.y * b.y);
    r.y = fma(a.x, b.y, a.y * b.x);
    return r;
}
template <typename V>
__device__ __forceinline__ V vfma(V a, V b, V c) {  // a * b + c
    V r;
    r.x = fma(a.x, b.x, fma(-a.y, b.y, c.x));
    r.y = fma(a.x, b.y, fma(a.y, b.x, c.y));
    return r;
}
template <typename V>
__device__ __forceinline__ V vzero() {
    V r;
    r.x = 0;
    r.y = 0;
    return r;
}
template <typename V>
__device__ __forceinline__ V vone() {
    V r;
    r.x = 1;
    r.y = 0;
    return r;
}

// Slice of a CTA: rows R0..R1 (n rows); lane l owns positions
// [l L, min(n, (l+1) L)), position p being row R0 + p.  Per-row shared
// arrays are stored [j][32] (j: position within the segment) so that a
// warp's accesses at one sweep step are consecutive.
struct Slice {
    int R0, R1, n, L;
    __device__ __forceinline__ int idx(int row) const {
        const int p = row - R0;
        return (p % L) * 32 + p / L;
    }
};

}  // namespace

// Rows of CTA c of a cluster of C over nz rows (near-equal contiguous slices).
void col_slice(int nz, int C, int c, int* R0, int* R1) {
    const int base = nz / C, extra = nz % C;
    *R0 = 1 + c * base + (c < extra ? c : extra);
    *R1 = *R0 + base - 1 + (c < extra ? 1 : 0);
}

namespace {

__device__ __forceinline__ void slice_of(int nz, int C, int c, int& R0, int& R1) {
    const int base = nz / C, extra = nz % C;
    R0 = 1 + c * base + (c < extra ? c : extra);
    R1 = R0 + base - 1 + (c < extra ? 1 : 0);
}

__host__ __device__ inline size_t r16(size_t b) { return (b + 15) & ~(size_t)15; }

// Shared memory of a CTA: P = 32 L slots per per-row array, `terms` warps,
// nmax rows in the cluster's largest slice, vb bytes per stored complex
// value.  Every CTA of a cluster uses the same layout (that of the largest
// slice), so that a remote CTA's tables sit at the same offsets.
__host__ __device__ inline size_t col_bytes(int P, int terms, int nmax, size_t vb) {
    return 2 * r16(2 * 16 * (size_t)terms) + r16(4 * 16 * (size_t)terms) + r16(16 * (size_t)P) +
           4 * r16(vb * (size_t)P * terms) +
           r16(vb * terms) + r16(32 * (size_t)terms) + r16(16 * kColMaxTerms) + r16(16 * 3) +
           r16(4 * (size_t)(nmax + 2));
}

// Shared memory carve-up of a CTA.
template <typename R>
struct ColSmem {
    using V = typename CV<R>::V;
    double2* U;     // field of the slice
    V* Q;           // [term][P] 1/den
    V* AL;          // [term][P] -(a1 + p d1) / den
    V* W;           // [term][P] back-substitution factor
    V* G;           // [term][P] workspace: q (M u), then g, then the term's x
    V* wghost;      // [term] w of row R0 - 1
    double2* fwd;   // [term][2] elimination map of the slice (A, B), read by later CTAs
    double2* bwd;   // [term][2] back-substitution map of the slice, read by earlier CTAs
    double2* fmat;  // [term][4] factorisation map of the slice (2 x 2), read by later CTAs
    double2* xh;    // [term][2] x of the halo rows R0 - 1 and R1 + 1
    double2* ck;    // [kColMaxTerms] residues of the active set
    double2* misc;  // [0] c_inf, [1] u of row R0 - 1, [2] u of row R1 + 1
    float* F3;      // f3 of rows R0 - 1 .. R1 + 1 (output scaling)
};

template <typename R>
__device__ ColSmem<R> carve(unsigned char* base, int P, int terms, int nmax) {
    using V = typename CV<R>::V;
    ColSmem<R> s;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + o;
        o += r16(bytes);
        return p;
    };
    // the tables other CTAs read come first
    s.fwd = (double2*)take(2 * 16 * (size_t)terms);
    s.bwd = (double2*)take(2 * 16 * (size_t)terms);
    s.fmat = (double2*)take(4 * 16 * (size_t)terms);
    s.U = (double2*)take(16 * (size_t)P);
    s.Q = (V*)take(sizeof(V) * (size_t)P * terms);
    s.AL = (V*)take(sizeof(V) * (size_t)P * terms);
    s.W = (V*)take(sizeof(V) * (size_t)P * terms);
    s.G = (V*)take(sizeof(V) * (size_t)P * terms);
    s.wghost = (V*)take(sizeof(V) * terms);
    s.xh = (double2*)take(32 * (size_t)terms);
    s.ck = (double2*)take(16 * kColMaxTerms);
    s.misc = (double2*)take(16 * 3);
    s.F3 = (float*)take(4 * (size_t)(nmax + 2));
    return s;
}

// Inclusive warp scan of affine maps y -> A y + B in lane order (REV: from
// lane 31 down).  (A, B) becomes the lane's inclusive map, (exA, exB) the
// composition of the maps of the earlier lanes (identity for the first).
// The maps are composed in FP64 in both forms: A is a product of up to a
// column's worth of factors, which leaves the FP32 range long before the
// recurrence's own values do.
template <bool REV>
__device__ __forceinline__ void warp_scan(double2& A, double2& B, double2& exA, double2& exB) {
    const int hw = threadIdx.x & 31;
    const int lane = REV ? 31 - hw : hw;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int from = REV ? min(hw + d, 31) : max(hw - d, 0);
        double2 pa, pb;
        pa.x = __shfl_sync(0xffffffffu, A.x, from);
        pa.y = __shfl_sync(0xffffffffu, A.y, from);
        pb.x = __shfl_sync(0xffffffffu, B.x, from);
        pb.y = __shfl_sync(0xffffffffu, B.y, from);
        if (lane >= d) {
            B = vfma(A, pb, B);  // this map after the earlier one
            A = vmul(A, pa);
        }
    }
    const int prev = REV ? min(hw + 1, 31) : max(hw - 1, 0);
    exA.x = __shfl_sync(0xffffffffu, A.x, prev);
    exA.y = __shfl_sync(0xffffffffu, A.y, prev);
    exB.x = __shfl_sync(0xffffffffu, B.x, prev);
    exB.y = __shfl_sync(0xffffffffu, B.y, prev);
    if (lane == 0) {
        exA = vone<double2>();
        exB = vzero<double2>();
    }
}

// Ordered composition of the maps of CTAs lo..hi-1 (REV: hi-1 down to lo)
// of term k applied to 0, by one warp: lane j fetches CTA j's map (one
// remote latency for all of them), the warp composes them in order.
template <bool REV>
__device__ __forceinline__ double2 cluster_fold(cg::cluster_group* cl, double2* table, int k, int lo, int hi) {
    const int hw = threadIdx.x & 31;
    const int n = hi - lo;
    double2 A = vone<double2>(), B = vzero<double2>();
    if (hw < n) {
        const double2* f = cl->map_shared_rank(table, REV ? hi - 1 - hw : lo + hw);
        A = f[2 * k];
        B = f[2 * k + 1];
    }
    // inclusive scan over the lanes in order; lane n - 1 holds the result
#pragma unroll
    for (int d = 1; d < 16; d <<= 1) {
        const int from = max(hw - d, 0);
        double2 pa, pb;
        pa.x = __shfl_sync(0xffffffffu, A.x, from);
        pa.y = __shfl_sync(0xffffffffu, A.y, from);
        pb.x = __shfl_sync(0xffffffffu, B.x, from);
        pb.y = __shfl_sync(0xffffffffu, B.y, from);
        if (hw >= d) {
            B = vfma(A, pb, B);
            A = vmul(A, pa);
        }
    }
    double2 v;
    v.x = __shfl_sync(0xffffffffu, B.x, max(n - 1, 0));
    v.y = __shfl_sync(0xffffffffu, B.y, max(n - 1, 0));
    return n > 0 ? v : vzero<double2>();
}

// Active Pade set of the cluster.
struct ColSet {
    int set = -1, n_active = 0;
};

template <typename R>
struct ColCtx {
    cg::cluster_group* cl;
    const ColArgs* a;
    RayDev ry;
    int rid, C, c, nz, term, lane;
    Slice sl;
    ColSmem<R> sm;
    double cfact, a1, a2;
};

// 2 x 2 complex matrix [[a, b], [c, d]].
struct M2 {
    double2 a, b, c, d;
};
__device__ __forceinline__ double2 cadd(double2 x, double2 y) { return c2(x.x + y.x, x.y + y.y); }
__device__ __forceinline__ M2 m2_mul(const M2& X, const M2& Y) {
    return {cadd(cmul(X.a, Y.a), cmul(X.b, Y.c)), cadd(cmul(X.a, Y.b), cmul(X.b, Y.d)),
            cadd(cmul(X.c, Y.a), cmul(X.d, Y.c)), cadd(cmul(X.c, Y.b), cmul(X.d, Y.d))};
}
// The maps act projectively (w = N / D), so a matrix may be rescaled at will:
// keep its largest component near 1.
__device__ __forceinline__ M2 m2_norm(M2 X) {
    const double m = fmax(fmax(fmax(fabs(X.a.x), fabs(X.a.y)), fmax(fabs(X.b.x), fabs(X.b.y))),
                          fmax(fmax(fabs(X.c.x), fabs(X.c.y)), fmax(fabs(X.d.x), fabs(X.d.y))));
    if (m > 0.0 && isfinite(m)) {
        const double s = 1.0 / m;
        X.a = c2(X.a.x * s, X.a.y * s);
        X.b = c2(X.b.x * s, X.b.y * s);
        X.c = c2(X.c.x * s, X.c.y * s);
        X.d = c2(X.d.x * s, X.d.y * s);
    }
    return X;
}
__device__ __forceinline__ M2 m2_eye() { return {c2(1.0, 0.0), c2(0.0, 0.0), c2(0.0, 0.0), c2(1.0, 0.0)}; }
__device__ __forceinline__ M2 m2_shfl(const M2& X, int from) {
    M2 r;
    r.a = c2(__shfl_sync(0xffffffffu, X.a.x, from), __shfl_sync(0xffffffffu, X.a.y, from));
    r.b = c2(__shfl_sync(0xffffffffu, X.b.x, from), __shfl_sync(0xffffffffu, X.b.y, from));
    r.c = c2(__shfl_sync(0xffffffffu, X.c.x, from), __shfl_sync(0xffffffffu, X.c.y, from));
    r.d = c2(__shfl_sync(0xffffffffu, X.d.x, from), __shfl_sync(0xffffffffu, X.d.y, from));
    return r;
}

// The Galerkin row m of the term (r1, r2, r3 of M + p D) from the f-window.
struct Rrow {
    double2 r1, r2, r3;
};

// Thomas factorisation of every active term's (M + p D), top-down, all rows
// of the slice in parallel.  w_m = r3_m / (r2_m - r1_m w_{m-1}) (w_0 = 0) is
// linear in homogeneous coordinates: (N, D)_m = T_m (N, D)_{m-1} with
// T_m = [[0, r3], [-r1, r2]] and w = N / D.  So, as for the solves: each
// segment multiplies its rows' T (sweep A), the warp scans the segments'
// products, the cluster folds in the slices above, and each segment runs the
// recurrence from its true entry w (sweep B), storing 1/den, al = -r1/den and
// w.  All arithmetic is FP64; the factors are stored in the sweep precision.
// Called by every thread of every CTA (one cluster barrier).
template <typename R>
__device__ void col_factor(ColCtx<R>& x, const ColSet& cs) {
    const ColArgs& a = *x.a;
    const int nz = x.nz, k = x.term, l = x.lane, L = x.sl.L, n = x.sl.n, P = 32 * L;
    const bool active = k < cs.n_active;
    const double2 p = active ? a.pd2[((long long)x.rid * kSets + cs.set) * CR_MAX_NP + k] : c2(0.0, 0.0);
    const int p0 = min(n, l * L), p1 = min(n, p0 + L);
    auto ld = [&](int i) {
        EnvRow r;
        if (i < 0 || i > nz + 1) {
            r.f1 = r.f2 = r.f3 = 0.0f;
            r.k = make_float2(0.0f, 0.0f);
            return r;
        }
        const long long o = x.ry.col + (long long)i * kTile;
        r.f1 = a.f1[o];
        r.f2 = a.f2[o];
        r.f3 = a.f3[o];
        r.k = a.ksq[o];
        return r;
    };
    auto row = [&](const EnvRow& em, const EnvRow& ec, const EnvRow& ep) {
        const Drow d = galerkin3(em, ec, ep, x.cfact);
        return Rrow{caxpd(x.a1, p, d.d1), caxpd(x.a2, p, d.d2), caxpd(x.a1, p, d.d3)};
    };
    M2 Mseg = m2_eye(), ex = m2_eye();
    if (active) {
        // sweep A: T of the segment's rows, last row leftmost
        EnvRow em = ld(x.sl.R0 + p0 - 1), ec = ld(x.sl.R0 + p0), ep;
        int cnt = 0;
        for (int q = p0; q < p1; ++q) {
            const int m = x.sl.R0 + q;
            ep = ld(m + 1);
            const Rrow rr = row(em, ec, ep);
            const M2 T{c2(0.0, 0.0), rr.r3, c2(-rr.r1.x, -rr.r1.y), rr.r2};
            Mseg = m2_mul(T, Mseg);
            if (++cnt == 8) {
                Mseg = m2_norm(Mseg);
                cnt = 0;
            }
            em = ec;
            ec = ep;
        }
        Mseg = m2_norm(Mseg);
        // warp scan in lane order: the product of the earlier lanes' maps
#pragma unroll
        for (int dd = 1; dd < 32; dd <<= 1) {
            const M2 prev = m2_shfl(Mseg, max(l - dd, 0));
            if (l >= dd) Mseg = m2_norm(m2_mul(Mseg, prev));
        }
        ex = m2_shfl(Mseg, max(l - 1, 0));
        if (l == 0) ex = m2_eye();
        if (l == 31) {
            x.sm.fmat[4 * k + 0] = Mseg.a;
            x.sm.fmat[4 * k + 1] = Mseg.b;
            x.sm.fmat[4 * k + 2] = Mseg.c;
            x.sm.fmat[4 * k + 3] = Mseg.d;
        }
    }
    x.cl->sync();
    if (active) {
        // the slices above, in order (lane j holds CTA j's map)
        M2 C = m2_eye();
        if (l < x.c) {
            const double2* f = x.cl->map_shared_rank(x.sm.fmat, l);
            C = {f[4 * k + 0], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]};
        }
#pragma unroll
        for (int dd = 1; dd < 16; dd <<= 1) {
            const M2 prev = m2_shfl(C, max(l - dd, 0));
            if (l >= dd) C = m2_norm(m2_mul(C, prev));
        }
        C = m2_shfl(C, max(x.c - 1, 0));
        if (x.c == 0) C = m2_eye();
        // entry (N, D) of this lane's segment: ex C (0, 1)
        const M2 E = m2_mul(ex, C);
        const double2 N = E.b, D = E.d;
        double2 wp = (N.x == 0.0 && N.y == 0.0) ? c2(0.0, 0.0) : cmul(N, crcp(D));
        if (l == 0) x.sm.wghost[k] = CV<R>::mk(wp);  // w of row R0 - 1
        // sweep B: the recurrence from the true entry
        EnvRow em = ld(x.sl.R0 + p0 - 1), ec = ld(x.sl.R0 + p0), ep;
        int o = l;
        for (int q = p0; q < p1; ++q, o += 32) {
            const int m = x.sl.R0 + q;
            ep = ld(m + 1);
            const Rrow rr = row(em, ec, ep);
            const double2 qq = crcp(cfms(rr.r2, rr.r1, wp));
            wp = cmul(rr.r3, qq);
            const double2 ci = cmul(rr.r1, qq);
            x.sm.Q[k * P + o] = CV<R>::mk(qq);
            x.sm.AL[k * P + o] = CV<R>::mk(c2(-ci.x, -ci.y));
            x.sm.W[k * P + o] = CV<R>::mk(wp);
            em = ec;
            ec = ep;
        }
    }
    __syncthreads();
}

// Switch to Pade set `ns` (when it changes) and refactor every active term.
template <typename R>
__device__ __forceinline__ void col_use_set(ColCtx<R>& x, ColSet& cs, int ns) {
    const ColArgs& a = *x.a;
    if (ns != cs.set) {
        cs.set = ns;
        cs.n_active = a.pd_n[x.rid * kSets + ns];
        const long long base = ((long long)x.rid * kSets + ns) * CR_MAX_NP;
        if (threadIdx.x < kColMaxTerms)
            x.sm.ck[threadIdx.x] = (int)threadIdx.x < cs.n_active ? a.pfc[base + threadIdx.x] : c2(0.0, 0.0);
        if (threadIdx.x == 0) x.sm.misc[0] = a.pfcinf[(long long)x.rid * kSets + ns];
    }
    col_factor<R>(x, cs);
}

// One range step of the active set.
template <typename R>
__device__ __forceinline__ void col_step(ColCtx<R>& x, const ColSet& cs) {
    using V = typename CV<R>::V;
    const int k = x.term, l = x.lane, L = x.sl.L, n = x.sl.n;
    const int P = 32 * L;
    const double2 zero = c2(0.0, 0.0);
    if (k < cs.n_active) {
        V* Q = x.sm.Q + k * P;
        V* AL = x.sm.AL + k * P;
        V* W = x.sm.W + k * P;
        V* G = x.sm.G + k * P;
        const int p0 = min(n, l * L), p1 = min(n, p0 + L);  // positions of this lane
        // neighbours of the segment: the previous lane's last row (or the
        // halo above), the next lane's first row (or the halo below)
        const double2 u_before = p0 >= p1 ? zero : (l == 0 ? x.sm.misc[1] : x.sm.U[(L - 1) * 32 + l - 1]);
        const double2 u_after = p0 >= p1 ? zero : (p1 == n ? x.sm.misc[2] : x.sm.U[l + 1]);
        // sweep 1: stage q (M u) in G; the segment's map g_end = A g_in + B
        double2 A = vone<double2>(), B = vzero<double2>();
        {
            double2 up = u_before, uc = p0 < p1 ? x.sm.U[l] : zero;
            int o = l;
            for (int p = p0; p < p1; ++p, o += 32) {
                const double2 un = p + 1 < p1 ? x.sm.U[o + 32] : u_after;
                V bv;
                bv.x = (R)fma(x.a1, up.x + un.x, x.a2 * uc.x);
                bv.y = (R)fma(x.a1, up.y + un.y, x.a2 * uc.y);
                const V qb = vmul(Q[o], bv);
                G[o] = qb;
                const double2 al = CV<R>::up(AL[o]);
                B = vfma(al, B, CV<R>::up(qb));
                A = vmul(al, A);
                up = uc;
                uc = un;
            }
        }
        double2 eA, eB;
        warp_scan<false>(A, B, eA, eB);
        if (l == 31) {
            x.sm.fwd[2 * k] = A;
            x.sm.fwd[2 * k + 1] = B;
        }
        // the value entering the slice, from the slices above
        x.cl->sync();
        const double2 gin = cluster_fold<false>(x.cl, x.sm.fwd, k, 0, x.c);
        // sweep 2: true g, stored
        V g = CV<R>::mk(vfma(eA, gin, eB));
        {
            int o = l;
            for (int p = p0; p < p1; ++p, o += 32) {
                g = vfma(AL[o], g, G[o]);
                G[o] = g;
            }
        }
        // sweep 3: the segment's map x_first = A x_in + B of x_m = g_m - w_m x_{m+1}
        A = vone<double2>();
        B = vzero<double2>();
        const int olast = l + (p1 - 1 - p0) * 32;
        {
            int o = olast;
            for (int p = p1 - 1; p >= p0; --p, o -= 32) {
                double2 mw = CV<R>::up(W[o]);
                mw.x = -mw.x;
                mw.y = -mw.y;
                B = vfma(mw, B, CV<R>::up(G[o]));
                A = vmul(mw, A);
            }
        }
        warp_scan<true>(A, B, eA, eB);
        if (l == 0) {
            x.sm.bwd[2 * k] = A;
            x.sm.bwd[2 * k + 1] = B;
        }
        x.cl->sync();
        const double2 xin = cluster_fold<true>(x.cl, x.sm.bwd, k, x.c + 1, x.C);
        // sweep 4: true x, stored over g
        V xv = CV<R>::mk(vfma(eA, xin, eB));
        {
            int o = olast;
            for (int p = p1 - 1; p >= p0; --p, o -= 32) {
                V mw = W[o];
                mw.x = -mw.x;
                mw.y = -mw.y;
                xv = vfma(mw, xv, G[o]);
                G[o] = xv;
            }
        }
        // halo rows: x of row R1 + 1 is the entry from below; x of row R0 - 1
        // is g_{R0-1} - w_{R0-1} x_{R0}, g_{R0-1} being the entry from above
        if (l == 0) {
            x.sm.xh[2 * k + 1] = xin;
            double2 mw = CV<R>::up(x.sm.wghost[k]);
            mw.x = -mw.x;
            mw.y = -mw.y;
            x.sm.xh[2 * k] = vfma(mw, CV<R>::up(xv), gin);  // xv: x of row R0 (lane 0, position 0)
        }
    } else {
        // a warp without a term in this set still takes the cluster's barriers
        x.cl->sync();
        x.cl->sync();
    }
    __syncthreads();
    // combine the terms: u_new = c_inf u + sum_k c_k x_k over the slots of
    // the slice (slot o holds position (o % 32) L + o / 32), then the halos
    const double2 ci = x.sm.misc[0];
    const int na = cs.n_active;
    for (int o = threadIdx.x; o < P; o += blockDim.x) {
        if ((o & 31) * L + (o >> 5) >= n) continue;
        typename CV<R>::V xs[kColMaxTerms];
#pragma unroll
        for (int j = 0; j < kColMaxTerms; ++j)
            if (j < na) xs[j] = x.sm.G[j * P + o];
        double2 acc = cmul(ci, x.sm.U[o]);
#pragma unroll
        for (int j = 0; j < kColMaxTerms; ++j) {
            if (j < na) {
                const double2 xd = CV<R>::up(xs[j]);
                const double2 c = x.sm.ck[j];
                acc = c2(fma(c.x, xd.x, fma(-c.y, xd.y, acc.x)), fma(c.x, xd.y, fma(c.y, xd.x, acc.y)));
            }
        }
        x.sm.U[o] = acc;
    }
    if (threadIdx.x < 2) {
        // halo rows outside the column (rows 0 and nz + 1) stay zero
        const int h = threadIdx.x;
        double2 acc = cmul(ci, x.sm.misc[1 + h]);
        for (int j = 0; j < na; ++j) {
            const double2 xd = x.sm.xh[2 * j + h];
            const double2 c = x.sm.ck[j];
            acc = c2(fma(c.x, xd.x, fma(-c.y, xd.y, acc.x)), fma(c.x, xd.y, fma(c.y, xd.x, acc.y)));
        }
        const bool inside = h == 0 ? x.sl.R0 > 1 : x.sl.R1 < x.nz;
        x.sm.misc[1 + h] = inside ? acc : zero;
    }
    __syncthreads();
}

// u of a row in [R0 - 1, R1 + 1] from the CTA's shared memory.
template <typename R>
__device__ __forceinline__ double2 col_u(const ColCtx<R>& x, int row) {
    if (row < 1 || row > x.nz) return c2(0.0, 0.0);
    if (row == x.sl.R0 - 1) return x.sm.misc[1];
    if (row == x.sl.R1 + 1) return x.sm.misc[2];
    return x.sm.U[x.sl.idx(row)];
}

// Outputs of the field after a step (every ndr steps): the complex pressure
// of the line (the CTA holding row max(ir, 1)) and of the grid rows (the CTA
// holding each).  Their transmission loss is computed once at the end of the
// march (col_tl), off the steps' critical path.
template <typename R>
__device__ __forceinline__ void col_emit(ColCtx<R>& x, int& mdr, int& tlc, int ir, double dir) {
    const RayDev& ry = x.ry;
    const ColArgs& a = *x.a;
    if (++mdr != ry.ndr) return;
    mdr = 0;
    ++tlc;
    if (tlc >= ry.nvr) return;
    const int irow = max(ir, 1);
    if (threadIdx.x == 0 && irow >= x.sl.R0 && irow <= x.sl.R1) {
        const double2 ua = col_u(x, ir), ub = col_u(x, ir + 1);
        const double fa = x.sm.F3[ir - (x.sl.R0 - 1)];
        const double fb = x.sm.F3[ir + 1 - (x.sl.R0 - 1)];
        a.cpl[ry.line_off + tlc] =
            c2((1.0 - dir) * fa * ua.x + dir * fb * ub.x, (1.0 - dir) * fa * ua.y + dir * fb * ub.y);
    }
    if (a.compute_grids && ry.grid_off >= 0) {
        // grid rows (j + 1) ndz of the slice (row nz + 1 goes with the last slice)
        const int jlo = max(0, (x.sl.R0 + ry.ndz - 1) / ry.ndz - 1);
        const int rmax = x.sl.R1 == x.nz ? x.nz + 1 : x.sl.R1;
        for (int j = jlo + (int)threadIdx.x; j < ry.nvz; j += blockDim.x) {
            const int row = (j + 1) * ry.ndz;
            if (row > rmax) break;
            if (row < x.sl.R0) continue;
            const double2 uj = col_u(x, row);
            const double fj = x.sm.F3[row - (x.sl.R0 - 1)];
            a.cpg[ry.grid_off + (long long)j * ry.nvr + tlc] = c2(uj.x * fj, uj.y * fj);
        }
    }
}

// Transmission loss of the ray's n_out emitted outputs from their complex
// pressure (outpt.py:11-57): output t was taken at r = (t + 1) ndr dr.  The
// cluster's threads share the line and the grid; a non-finite line value
// flags the ray.
template <typename R>
__device__ void col_tl(ColCtx<R>& x, int n_out) {
    const RayDev& ry = x.ry;
    const ColArgs& a = *x.a;
    const int tid = x.c * blockDim.x + threadIdx.x, nt = x.C * blockDim.x;
    int bad = 0;
    for (int t = tid; t < n_out; t += nt) {
        const double2 cp = a.cpl[ry.line_off + t];
        const double amp = hypot(cp.x, cp.y);
        bad |= !isfinite(amp);
        a.tll[ry.line_off + t] = tl_db(amp, (double)((t + 1) * ry.ndr) * ry.dr);
    }
    if (bad) atomicOr(a.flags + x.rid, 1);
    if (a.compute_grids && ry.grid_off >= 0) {
        const long long total = (long long)ry.nvz * n_out;
        for (long long q = tid; q < total; q += nt) {
            const int j = (int)(q / n_out), t = (int)(q % n_out);
            const long long o = ry.grid_off + (long long)j * ry.nvr + t;
            const double2 g = a.cpg[o];
            a.tlg[o] = tl_db(hypot(g.x, g.y), (double)((t + 1) * ry.ndr) * ry.dr);
        }
    }
}

// f3 of rows max(lo, R0 - 1) .. min(hi, R1 + 1) into shared memory.
template <typename R>
__device__ __forceinline__ void col_load_f3(ColCtx<R>& x, int lo, int hi) {
    const int a0 = max(lo, x.sl.R0 - 1), a1 = min(hi, x.sl.R1 + 1);
    for (int i = a0 + (int)threadIdx.x; i <= a1; i += blockDim.x)
        x.sm.F3[i - (x.sl.R0 - 1)] = x.a->f3[x.ry.col + (long long)i * kTile];
}

}  // namespace

template <typename R>
__global__ void __launch_bounds__(32 * kColMaxTerms) march_col_kernel(ColArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cl = cg::this_cluster();
    ColCtx<R> x;
    x.cl = &cl;
    x.a = &a;
    x.C = (int)cl.num_blocks();
    x.c = (int)cl.block_rank();
    x.rid = a.col_ray[blockIdx.x / x.C];
    x.ry = a.rays[x.rid];
    x.nz = x.ry.nz;
    x.term = threadIdx.x >> 5;
    x.lane = threadIdx.x & 31;
    slice_of(x.nz, x.C, x.c, x.sl.R0, x.sl.R1);
    x.sl.n = x.sl.R1 - x.sl.R0 + 1;
    // the layout of the cluster's largest slice (CTA 0's) in every CTA
    const int nmax = (x.nz + x.C - 1) / x.C;
    x.sl.L = (nmax + 31) / 32;
    const int terms = blockDim.x >> 5;
    x.sm = carve<R>(smem_raw, 32 * x.sl.L, terms, nmax);
    const RayDev& ry = x.ry;
    const int nz = x.nz;
    const EnvPtrs e = env_ptrs(a.envs[ry.env], a.pool);
    x.cfact = 0.5 / (ry.dz * ry.dz);
    x.a1 = ry.k0 * ry.k0 / 6.0;
    x.a2 = 2.0 * ry.k0 * ry.k0 / 3.0;
    const int T = blockDim.x;
    if (x.c == 0 && threadIdx.x == 0) a.flags[x.rid] = 0;

    // initial profiles (cupyram.py:571-608, profl): rows split over the cluster
    int iz = max(1, min(nz - 1, (int)floor(e.zb[0] / ry.dz)));
    int ss = 0, sb = 0, bt = 0;
    for (int i = x.c + x.C * (int)threadIdx.x; i <= nz + 1; i += x.C * T)
        assemble_rows(ry, e, ss, sb, iz, i, i, a.f1, a.f2, a.f3, a.ksq);
    // self-starter delta (cupyram.py:1008-1022)
    for (int p = threadIdx.x; p < 32 * x.sl.L; p += T) x.sm.U[p] = c2(0.0, 0.0);
    if (threadIdx.x == 0) {
        x.sm.misc[1] = c2(0.0, 0.0);
        x.sm.misc[2] = c2(0.0, 0.0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
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
            const double2 v = c2(wgt * amp / (ry.dz * alpw), 0.0);
            if (i >= 1 && i <= nz) {
                if (i >= x.sl.R0 && i <= x.sl.R1) x.sm.U[x.sl.idx(i)] = v;
                else if (i == x.sl.R0 - 1) x.sm.misc[1] = v;
                else if (i == x.sl.R1 + 1) x.sm.misc[2] = v;
            }
        }
    }
    __threadfence();
    cl.sync();
    col_load_f3(x, 0, nz + 1);
    __syncthreads();

    ColSet cs;
    const double ri = ry.zr / ry.dz;
    const int ir = (int)floor(ri);
    const double dir = ri - ir;
    int mdr = 0, tlc = -1;

    // self-starter: two steps of 1/(1-X), one of the ip=2 operator
    col_use_set(x, cs, 0);
    col_step(x, cs);
    col_step(x, cs);
    col_use_set(x, cs, 1);
    col_step(x, cs);
    col_emit(x, mdr, tlc, ir, dir);  // first output at r = dr (cupyram.py:703)

    double rs = ry.rs;
    double r = ry.dr;
    for (int rn = 0; rn < ry.nr; ++rn) {
        // updat (updat.py:38-140) for the step about to be taken
        bool reprofile = false;
        int iz_new = iz, new_set = cs.set == 1 ? 2 : cs.set;
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
        if (reprofile || iz_new != iz) {
            const int lo = reprofile ? 0 : min(iz, iz_new) + 1;
            const int hi = reprofile ? nz + 1 : max(iz, iz_new);
            for (int i = lo + x.c + x.C * (int)threadIdx.x; i <= hi; i += x.C * T)
                assemble_rows(ry, e, ss, sb, iz_new, i, i, a.f1, a.f2, a.f3, a.ksq);
            __threadfence();
            cl.sync();
            col_load_f3(x, lo, hi);
            iz = iz_new;
            col_use_set(x, cs, new_set);
        } else if (new_set != cs.set) {
            col_use_set(x, cs, new_set);
        }
        col_step(x, cs);
        r = (double)(rn + 2) * ry.dr;
        col_emit(x, mdr, tlc, ir, dir);
    }
    __threadfence();
    cl.sync();  // every complex pressure is stored; no CTA still reads another's shared memory
    col_tl(x, min(tlc + 1, ry.nvr));
}

size_t col_smem_bytes(int nz, int cluster, int terms, int chosen) {
    const int nmax = (nz + cluster - 1) / cluster;
    const int L = (nmax + 31) / 32;
    return col_bytes(32 * L, terms, nmax, chosen ? 8 : 16);
}

int col_cluster_size(int nz, int terms, int chosen) {
    for (int C = 1; C <= kColMaxCluster; ++C)
        if (col_smem_bytes(nz, C, terms, chosen) <= kColSmemLimit) return C;
    return 0;
}

template <typename R>
static cudaError_t col_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr, int n_rays, int cluster,
                              int terms, int nz_max, cudaStream_t st) {
    const size_t smem = col_smem_bytes(nz_max, cluster, terms, sizeof(R) == 4);
    cudaError_t ce = cudaFuncSetAttribute(march_col_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce != cudaSuccess) return ce;
    if (cluster > 8) {
        ce = cudaFuncSetAttribute(march_col_kernel<R>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (ce != cudaSuccess) return ce;
    }
    cfg = cudaLaunchConfig_t{};
    cfg.gridDim = dim3((unsigned)(n_rays * cluster), 1, 1);
    cfg.blockDim = dim3((unsigned)(32 * terms), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaSuccess;
}

cudaError_t launch_march_col(const ColArgs& a, int n_rays, int cluster, int terms, int nz_max, int chosen,
                             cudaStream_t st) {
    if (terms < 1 || terms > kColMaxTerms || cluster < 1 || cluster > kColMaxCluster) return cudaErrorInvalidValue;
    if (col_smem_bytes(nz_max, cluster, terms, chosen) > kColSmemLimit) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    cudaError_t ce = chosen ? col_config<float>(cfg, attr, n_rays, cluster, terms, nz_max, st)
                            : col_config<double>(cfg, attr, n_rays, cluster, terms, nz_max, st);
    if (ce != cudaSuccess) return ce;
    ce = chosen ? cudaLaunchKernelEx(&cfg, march_col_kernel<float>, a)
                : cudaLaunchKernelEx(&cfg, march_col_kernel<double>, a);
    if (ce != cudaSuccess) return ce;
    return cudaGetLastError();
}

int col_max_active_clusters(int cluster, int terms, int nz_max, int chosen) {
    if (terms < 1 || terms > kColMaxTerms || cluster < 1 || cluster > kColMaxCluster) return 0;
    if (col_smem_bytes(nz_max, cluster, terms, chosen) > kColSmemLimit) return 0;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    cudaError_t ce = chosen ? col_config<float>(cfg, attr, 1, cluster, terms, nz_max, 0)
                            : col_config<double>(cfg, attr, 1, cluster, terms, nz_max, 0);
    if (ce != cudaSuccess) return 0;
    int n = 0;
    ce = chosen ? cudaOccupancyMaxActiveClusters(&n, march_col_kernel<float>, &cfg)
                : cudaOccupancyMaxActiveClusters(&n, march_col_kernel<double>, &cfg);
    return ce == cudaSuccess ? n : 0;
}

}  // namespace crk
