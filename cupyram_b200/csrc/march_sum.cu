// march_sum.cu - range march in partial-fraction ("sum") form.
//
// The split-step Pade operator of one range step is a rational function of
// the Galerkin operator X = M^{-1} D (M: mass matrix, D: Galerkin stiffness +
// wavenumber rows; cupyram/fused_kernel.py:20-69):
//
//     P(X) = prod_j (1 + pd1_j X) / (1 + pd2_j X)          (reference: product form)
//          = c_inf + sum_k c_k / (1 + pd2_k X)             (here: partial fractions)
//
// so u_new = c_inf u + sum_k c_k x_k with (M + pd2_k D) x_k = M u.  The np
// tridiagonal solves of a step are independent: one lane per term.  A warp
// holds floor(32/G) rays x G terms (G = largest np of its tile).
//
// Per range step each lane runs ONE pass over its column:
//   * the back-substitution of the previous step's solve for its term,
//   * the combination of the G terms of its ray into u_new for the row
//     (shared memory, double-buffered, one __syncwarp of the ray's lanes),
//   * the elimination of the next step's solve one row behind,
// alternating the pass direction every step.  The Thomas factorisation of
// each term (1/den, the coupling factor and w per row, both directions) is
// computed once per change of the operator - profiles, bathymetry index or
// Pade set - and streamed from HBM, together with the lane's workspace g,
// through a per-lane cp.async prefetch ring.
//
// The sum form is the reference's rational operator rearranged; on the
// golden cases it matches the product form to <= 5e-8 dB (oracle mode "sum").
#include <cuda_runtime.h>

#include "march_common.cuh"
#include "march_sum.cuh"

namespace crk {

namespace {

constexpr int kSR = 8;       // prefetch depth (rows) per lane
constexpr int kSFields = 5;  // 16-byte fields per ring slot
static_assert((kSR & (kSR - 1)) == 0, "kSR must be a power of two");

struct SumSmem {
    double2 q[kSR][kSFields][kTile];
    double2 red[2][kTile];
};

enum SumPass { kElimOnly = 0, kFusedP = 1, kBackOnly = 2, kFactor = 3 };

struct Lane {
    int lane, k, gbase, G;
    unsigned gmask;
    long long rcol;  // ray column base (f1..f3, ksq, u)
    long long lcol;  // lane column base (G, factors)
};

struct Ops {
    int nz;
    double cfact, a1, a2;
    double2 pole;   // pd2 of this lane's term in the active set
    double2 ck;     // partial-fraction residue of this lane's term (0 for unused lanes)
    double2 cinf;   // c_inf of the ray for the active set
};

__device__ __forceinline__ float* sfl(SumSmem& S, int slot, int lane) { return (float*)&S.q[slot][0][lane]; }
__device__ __forceinline__ float2* sks(SumSmem& S, int slot, int lane) { return (float2*)&S.q[slot][1][lane]; }

template <int PASS, bool DOWN>
__device__ __forceinline__ void sum_issue(const SumArgs& a, const Lane& L, SumSmem& S, int slot, int r, int nz) {
    if (r >= 0 && r <= nz + 1) {
        const long long ro = L.rcol + (long long)r * kTile;
        const long long lo = L.lcol + (long long)r * kTile;
        if (PASS == kFactor) {
            float* f = sfl(S, slot, L.lane);
            cp4(f + 0, a.f1 + ro);
            cp4(f + 1, a.f2 + ro);
            cp4(f + 2, a.f3 + ro);
            cp8(sks(S, slot, L.lane), a.ksq + ro);
        } else {
            if (PASS == kElimOnly) cp16(&S.q[slot][0][L.lane], a.u + ro);
            else {
                // back-substitution of a solve eliminated in the other direction
                cp16(&S.q[slot][0][L.lane], (DOWN ? a.WU : a.WD) + lo);
                cp16(&S.q[slot][1][L.lane], a.G + lo);
                cp16(&S.q[slot][4][L.lane], a.u + ro);
            }
            const int m = DOWN ? r - 1 : r + 1;
            if (PASS != kBackOnly && m >= 1 && m <= nz) {
                const long long mo = L.lcol + (long long)m * kTile;
                cp16(&S.q[slot][2][L.lane], (DOWN ? a.QD : a.QU) + mo);
                cp16(&S.q[slot][3][L.lane], (DOWN ? a.AD : a.AU) + mo);
            }
        }
    }
    cp_commit();
}

// Thomas factorisation of (M + pole D) for this lane's term, both directions.
template <bool DOWN>
__device__ void sum_factor(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o) {
    const int nz = o.nz;
    __threadfence_block();
#pragma unroll 1
    for (int k = 0; k < kSR; ++k) sum_issue<kFactor, DOWN>(a, L, S, k, DOWN ? k : nz + 1 - k, nz);
    EnvRow em{}, ec{}, ep{};
    double2 wp = c2(0.0, 0.0);
    double2* Q = DOWN ? a.QD : a.QU;
    double2* A = DOWN ? a.AD : a.AU;
    double2* W = DOWN ? a.WD : a.WU;
#pragma unroll 1
    for (int k = 0; k < nz + 2; ++k) {
        const int r = DOWN ? k : nz + 1 - k;
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
        sum_issue<kFactor, DOWN>(a, L, S, slot, DOWN ? k + kSR : nz + 1 - k - kSR, nz);
        if (DOWN) {
            em = ec;
            ec = ep;
            ep = er;
        } else {
            ep = ec;
            ec = em;
            em = er;
        }
        if (k < 2) continue;
        const int m = DOWN ? r - 1 : r + 1;
        if (m < 1 || m > nz) continue;
        const Drow d = galerkin3(em, ec, ep, o.cfact);
        const double2 r1 = caxpd(o.a1, o.pole, d.d1), r2 = caxpd(o.a2, o.pole, d.d2),
                      r3 = caxpd(o.a1, o.pole, d.d3);
        const double2 cin = DOWN ? r1 : r3, cout = DOWN ? r3 : r1;
        const double2 q = crcp(cfms(r2, cin, wp));
        wp = cmul(cout, q);
        const double2 ci = cmul(cin, q);
        const long long mo = L.lcol + (long long)m * kTile;
        Q[mo] = q;
        A[mo] = c2(-ci.x, -ci.y);
        W[mo] = wp;
    }
    cp_wait<0>();
}

// One solve pass.  kElimOnly: eliminate from the stored field u.  kFusedP:
// back-substitute the pending solve, combine the terms into u_new (stored),
// eliminate the next solve.  kBackOnly: back-substitute and combine only.
template <int PASS, bool DOWN>
__device__ void sum_pass(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o) {
    const int nz = o.nz;
    __threadfence_block();
    __syncwarp(L.gmask);
#pragma unroll 1
    for (int k = 0; k < kSR; ++k) sum_issue<PASS, DOWN>(a, L, S, k, DOWN ? k : nz + 1 - k, nz);
    const double2 zero = c2(0.0, 0.0);
    double2 u0 = zero, u1 = zero, u2 = zero;  // u window, oldest first
    double2 xp = zero;                         // back-substitution carry
    double2 gp = zero;                         // elimination carry
#pragma unroll 1
    for (int k = 0; k < nz + 2; ++k) {
        const int r = DOWN ? k : nz + 1 - k;
        const int slot = k & (kSR - 1);
        cp_wait<kSR - 1>();
        const double2 f0 = S.q[slot][0][L.lane];
        double2 f1v = zero, fq = zero, fa = zero, fu = zero;
        if (PASS != kElimOnly) {
            f1v = S.q[slot][1][L.lane];
            fu = S.q[slot][4][L.lane];
        }
        if (PASS != kBackOnly) {
            fq = S.q[slot][2][L.lane];
            fa = S.q[slot][3][L.lane];
        }
        sum_issue<PASS, DOWN>(a, L, S, slot, DOWN ? k + kSR : nz + 1 - k - kSR, nz);
        const bool interior = (r >= 1 && r <= nz);
        double2 un;
        if (PASS == kElimOnly) {
            un = interior ? f0 : zero;
        } else {
            // back-substitution: x_r = g_r - w_r x_{r-/+1}
            double2 x = zero;
            if (interior) {
                const bool first = DOWN ? (r == 1) : (r == nz);
                x = first ? f1v : c2(fma(-f0.x, xp.x, fma(f0.y, xp.y, f1v.x)), fma(-f0.x, xp.y, fma(-f0.y, xp.x, f1v.y)));
            }
            xp = x;
            // combine the G terms of the ray: u_new = c_inf u_old + sum_k c_k x_k
            double2* red = S.red[k & 1];
            red[L.lane] = cmul(o.ck, x);
            __syncwarp(L.gmask);
            double2 acc = cmul(o.cinf, fu);
            for (int j = 0; j < L.G; ++j) {
                const double2 v = red[L.gbase + j];
                acc.x += v.x;
                acc.y += v.y;
            }
            un = interior ? acc : zero;
            if (interior && L.k == 0) a.u[L.rcol + (long long)r * kTile] = un;
        }
        if (PASS == kBackOnly) continue;
        u0 = u1;
        u1 = u2;
        u2 = un;
        if (k < 2) continue;
        const int m = DOWN ? r - 1 : r + 1;
        if (m < 1 || m > nz) continue;
        // (M u)_m = a1 (u_{m-1} + u_{m+1}) + a2 u_m, then g_m = q (M u)_m + al g_{m-/+1}
        const double2 mu = c2(fma(o.a1, u0.x + u2.x, o.a2 * u1.x), fma(o.a1, u0.y + u2.y, o.a2 * u1.y));
        const double2 t = cmul(fq, mu);
        const double2 g = c2(fma(fa.x, gp.x, fma(-fa.y, gp.y, t.x)), fma(fa.x, gp.y, fma(fa.y, gp.x, t.y)));
        gp = g;
        a.G[L.lcol + (long long)m * kTile] = g;
    }
    cp_wait<0>();
    __threadfence_block();
    __syncwarp(L.gmask);
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

__device__ void set_ops(const SumArgs& a, int rid, int set, const Lane& L, Ops* o) {
    const int n = a.pd_n[rid * kSets + set];
    const long long base = ((long long)rid * kSets + set) * CR_MAX_NP;
    const int kk = L.k < n ? L.k : 0;  // unused lanes solve a copy of term 0 with weight 0
    o->pole = a.pd2[base + kk];
    o->ck = L.k < n ? a.pfc[base + kk] : c2(0.0, 0.0);
    o->cinf = a.pfcinf[(long long)rid * kSets + set];
}

__device__ void sum_refactor(const SumArgs& a, const Lane& L, SumSmem& S, const Ops& o) {
    sum_factor<true>(a, L, S, o);
    sum_factor<false>(a, L, S, o);
    __threadfence_block();
    __syncwarp(L.gmask);
}

}  // namespace

__global__ void __launch_bounds__(kTile) march_sum_kernel(SumArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SumSmem& S = *reinterpret_cast<SumSmem*>(smem_raw);
    const int t = blockIdx.x;
    Lane L;
    L.lane = threadIdx.x;
    L.G = a.tile_G[t];
    const int rid = a.tile_ray[t * kTile + L.lane];
    if (rid < 0 || L.G < 1) return;
    L.k = L.lane % L.G;
    L.gbase = L.lane - L.k;
    L.gmask = (L.G >= 32 ? 0xffffffffu : ((1u << L.G) - 1u)) << L.gbase;
    const RayDev ry = a.rays[rid];
    L.rcol = ry.col;
    L.lcol = a.tile_off[t] + L.lane;
    const EnvPtrs e = env_ptrs(a.envs[ry.env], a.pool);
    const int nz = ry.nz;
    int flag = 0;
    Ops o;
    o.nz = nz;
    o.cfact = 0.5 / (ry.dz * ry.dz);
    o.a1 = ry.k0 * ry.k0 / 6.0;
    o.a2 = 2.0 * ry.k0 * ry.k0 / 3.0;

    // initial profiles, split over the ray's lanes (cupyram.py:571-608, profl)
    int iz = max(1, min(nz - 1, (int)floor(e.zb[0] / ry.dz)));
    int ss = 0, sb = 0, bt = 0;
    for (int i = L.k; i <= nz + 1; i += L.G) {
        assemble_rows(ry, e, ss, sb, iz, i, i, a.f1, a.f2, a.f3, a.ksq);
        a.u[L.rcol + (long long)i * kTile] = c2(0.0, 0.0);
    }
    __threadfence_block();
    __syncwarp(L.gmask);
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
    __syncwarp(L.gmask);

    const double ri = ry.zr / ry.dz;
    const int ir = (int)floor(ri);
    const double dir = ri - ir;
    int mdr = 0, tlc = -1;

    // the solve "pending" back-substitution: its direction and the range /
    // output of the step it belongs to
    bool pend_down = true;    // direction of the pending elimination
    bool pend_out = false;    // the pending step is followed by an outpt call
    double pend_r = 0.0;

    auto emit = [&](double r_out) {
        if (++mdr == ry.ndr) {
            mdr = 0;
            ++tlc;
            sum_outputs(a, ry, L, tlc, r_out, ir, dir, &flag);
        }
    };
    auto back_only = [&]() {
        if (pend_down) sum_pass<kBackOnly, false>(a, L, S, o);
        else sum_pass<kBackOnly, true>(a, L, S, o);
        if (pend_out) emit(pend_r);
    };

    // self-starter: two steps of 1/(1-X), one of the ip=2 operator
    set_ops(a, rid, 0, L, &o);
    sum_refactor(a, L, S, o);
    sum_pass<kElimOnly, true>(a, L, S, o);
    pend_down = true;
    pend_out = false;
    sum_pass<kFusedP, false>(a, L, S, o);  // back-substitute step 1, eliminate step 2 (UP)
    pend_down = false;
    back_only();
    set_ops(a, rid, 1, L, &o);
    sum_refactor(a, L, S, o);
    sum_pass<kElimOnly, true>(a, L, S, o);
    pend_down = true;
    pend_out = true;
    pend_r = ry.dr;  // first output at r = dr (cupyram.py:703)

    int set = 2;
    double rs = ry.rs;
    double r = ry.dr;
    bool first_march = true;
    for (int rn = 0; rn < ry.nr; ++rn) {
        // updat (updat.py:38-140) for the step about to be taken
        bool reprofile = false;
        int iz_new = iz;
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
        bool change = first_march || reprofile || iz_new != iz;
        int new_set = set;
        if (r >= rs) {  // stability constraints off (cupyram.py:976-999)
            new_set = 3;
            rs = INFINITY;
            change = true;
        }
        const double r_out = (double)(rn + 2) * ry.dr;
        if (change) {
            back_only();
            if (reprofile) {
                for (int i = L.k; i <= nz + 1; i += L.G) assemble_rows(ry, e, ss, sb, iz_new, i, i, a.f1, a.f2, a.f3, a.ksq);
            } else if (iz_new != iz) {
                const int lo = min(iz, iz_new) + 1, hi = max(iz, iz_new);
                for (int i = lo + L.k; i <= hi; i += L.G) assemble_rows(ry, e, ss, sb, iz_new, i, i, a.f1, a.f2, a.f3, a.ksq);
            }
            __threadfence_block();
            __syncwarp(L.gmask);
            iz = iz_new;
            set = new_set;
            set_ops(a, rid, set, L, &o);
            sum_refactor(a, L, S, o);
            sum_pass<kElimOnly, true>(a, L, S, o);
            pend_down = true;
            first_march = false;
        } else {
            // back-substitute the pending step and eliminate this one in one pass
            if (pend_down) sum_pass<kFusedP, false>(a, L, S, o);
            else sum_pass<kFusedP, true>(a, L, S, o);
            if (pend_out) emit(pend_r);
            pend_down = !pend_down;
        }
        pend_out = true;
        pend_r = r_out;
        r = r_out;
    }
    back_only();
    if (L.k == 0) a.flags[rid] = flag;
}

cudaError_t launch_march_sum(const SumArgs& a, int n_tiles, cudaStream_t st) {
    const size_t smem = sizeof(SumSmem);
    cudaError_t ce = cudaFuncSetAttribute(march_sum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce != cudaSuccess) return ce;
    march_sum_kernel<<<n_tiles, kTile, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace crk
