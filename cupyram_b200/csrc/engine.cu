// engine.cu - B200 split-step Pade range march behind the cupyram_b200.h C ABI.
//
// Work decomposition
//   * A "ray" is one calculation of the reference (an environment at one
//     frequency).  Rays are sorted by work (rows x steps) and packed 32 to a
//     tile; one warp marches one tile, one lane per ray.
//   * Every per-row array of a tile is stored [row][lane] (32 consecutive
//     lanes = 32 consecutive elements), so each load/store of a sweep is a
//     fully coalesced warp access: 128 B (float), 256 B (float2) or 512 B
//     (double2) per instruction.
//   * The whole range march of a tile (self-starter, range-index updates,
//     profile re-assembly, np Pade sweeps per step, receiver / TL-grid
//     extraction) runs inside ONE kernel launch: the range loop is device
//     resident, there is no per-step launch and no per-step host sync
//     (the reference launches ~10 kernels and syncs 3 times per step).
//
// Sweep structure of one range step with n Pade terms (product form,
// term j solves (M + pd2_j D) x = (M + pd1_j D) u):
//   term j eliminates DOWN when j is even and UP when j is odd, so the back-
//   substitution of term j runs in the same direction as the elimination of
//   term j+1 and the two are fused into one pass over the column.  A step is
//   n+1 passes instead of the reference's 2n, the field between terms never
//   touches memory, and the Thomas workspace (w, g) of a row is overwritten
//   in place one row behind the pass.
//
// References for the maths (clapeyre/cupyram):
//   profile interpolation   cupyram/profl.py:8-140, cupyram/cupyram.py:770-803
//   range-index update      cupyram/updat.py:38-140
//   layer selection         cupyram/matrc.py:16-107 (iz == jz branch)
//   Galerkin coefficients   cupyram/fused_kernel.py:20-69
//   Thomas sweeps           cupyram/fused_kernel.py:72-153
//   receiver / TL grid      cupyram/outpt.py:11-57
//   self-starter            cupyram/cupyram.py:1001-1063
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/cupyram_b200.h"
#include "march_col.cuh"
#include "march_common.cuh"
#include "march_sum.cuh"
#include "pade.h"

namespace {

using namespace crk;

// ---------------------------------------------------------------------------
// per-lane prefetch ring
//
// Every pass streams the rows of one column in order.  Each lane copies its
// own elements of the next kRing rows into shared memory with cp.async
// (4/8/16-byte copies; a warp's copies of one row are one coalesced access),
// so the ~1 us global-memory latency overlaps the serial recurrence of the
// rows before.  A lane only ever reads its own slots: no warp-wide sync.
// ---------------------------------------------------------------------------
constexpr int kRing = 32;
constexpr int kRingFields = 6;
static_assert((kRing & (kRing - 1)) == 0, "kRing must be a power of two");

// Per slot and lane, six 16-byte fields.  A lane only touches its own
// column, so the fields are a per-lane union: the on-the-fly passes use
// {W or u, G, (f1, f2, f3), ksq}; the factorised passes use
// {W or u, G, S1, S2, S3, AL}.
struct Ring {
    double2 q[kRing][kRingFields][kTile];
};
constexpr size_t kRingBytes = sizeof(Ring);

enum PassKind { kFirst = 0, kFused = 1, kLast = 2, kEnvOnly = 3 };

__device__ __forceinline__ float* ring_f(Ring& R, int slot, int lane) { return (float*)&R.q[slot][2][lane]; }
__device__ __forceinline__ float2* ring_k(Ring& R, int slot, int lane) { return (float2*)&R.q[slot][3][lane]; }

// Issue the copies of stream row r into ring slot `slot` (one commit group,
// possibly empty when r is outside 0..nz+1).
template <int KIND>
__device__ __forceinline__ void ring_issue(Ring& R, const Col& c, int slot, int r, int nz, int lane) {
    if (r >= 0 && r <= nz + 1) {
        const long long o = (long long)r * kTile;
        if (KIND == kFirst) cp16(&R.q[slot][0][lane], c.u + o);
        else if (KIND != kEnvOnly) {
            cp16(&R.q[slot][0][lane], c.W + o);
            cp16(&R.q[slot][1][lane], c.G + o);
        }
        if (KIND != kLast) {
            float* f = ring_f(R, slot, lane);
            cp4(f + 0, c.f1 + o);
            cp4(f + 1, c.f2 + o);
            cp4(f + 2, c.f3 + o);
            cp8(ring_k(R, slot, lane), c.ksq + o);
        }
    }
    cp_commit();
}

// One pass over the column.
//   kFirst, DOWN : eliminate term (p1, p2) downwards from the stored field u.
//   kFused, DOWN : back-substitute the UP-eliminated term, eliminate (p1, p2) DOWN.
//   kFused, UP   : back-substitute the DOWN-eliminated term, eliminate (p1, p2) UP.
//   kLast        : back-substitute the last term (eliminated opposite to DOWN)
//                  and store the field.
// Stream row r carries W_r, G_r (or u_r) and f1..f3, ksq of row r; the
// elimination runs one row behind the stream so that its 3-row windows of
// field and coefficients are complete.
template <int KIND, bool DOWN>
__device__ void run_pass(const StepCtx& s, Ring& R, double2 p1, double2 p2) {
    const Col& c = s.c;
    const int nz = s.nz;
    const int lane = threadIdx.x;
    const int nrows = nz + 2;
    __threadfence_block();  // order this lane's earlier stores before its cp.async reads
#pragma unroll 1
    for (int k = 0; k < kRing; ++k) ring_issue<KIND>(R, c, k, DOWN ? k : nz + 1 - k, nz, lane);

    EnvRow em{}, ec{}, ep{};
    double2 x0 = c2(0.0, 0.0), x1 = c2(0.0, 0.0), x2 = c2(0.0, 0.0);  // field window, oldest first
    double2 wp = c2(0.0, 0.0), gp = c2(0.0, 0.0);
    const double2 zero = c2(0.0, 0.0);
#pragma unroll 1
    for (int k = 0; k < nrows; ++k) {
        const int r = DOWN ? k : nz + 1 - k;
        const int slot = k & (kRing - 1);
        cp_wait<kRing - 1>();
        double2 av = zero, bv = zero;
        EnvRow er{};
        av = R.q[slot][0][lane];
        if (KIND != kFirst) bv = R.q[slot][1][lane];
        if (KIND != kLast) {
            const float* f = ring_f(R, slot, lane);
            er.f1 = f[0];
            er.f2 = f[1];
            er.f3 = f[2];
            er.k = *ring_k(R, slot, lane);
        }
        ring_issue<KIND>(R, c, slot, DOWN ? k + kRing : nz + 1 - k - kRing, nz, lane);

        // field value x_r of this stream row
        double2 xr;
        if (KIND == kFirst) {
            xr = (r == 0) ? s.u0 : (r == nz + 1 ? zero : av);
        } else if (DOWN) {  // previous term was eliminated UP: x_r = g_r - w_r x_{r-1}
            xr = (r == 0) ? s.u0 : (r == nz + 1 ? zero : (r == 1 ? bv : cfms(bv, av, x2)));
        } else {  // previous term eliminated DOWN: x_r = g_r - w_r x_{r+1}
            xr = (r == nz + 1) ? zero : (r == 0 ? s.u0 : (r == nz ? bv : cfms(bv, av, x2)));
        }
        if (KIND == kLast) {
            if (r >= 1 && r <= nz) c.u[(long long)r * kTile] = xr;
            x2 = xr;
            continue;
        }
        x0 = x1;
        x1 = x2;
        x2 = xr;
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
        // eliminate row m: DOWN m = r-1 with (x_{m-1}, x_m, x_{m+1}) = (x0, x1, x2);
        //                  UP   m = r+1 with (x_{m-1}, x_m, x_{m+1}) = (x2, x1, x0)
        const int m = DOWN ? r - 1 : r + 1;
        if (m < 1 || m > nz) continue;
        const Drow d = galerkin3(em, ec, ep, s.cfact);
        const double2 r1 = caxpd(s.a1, p2, d.d1), r2 = caxpd(s.a2, p2, d.d2), r3 = caxpd(s.a1, p2, d.d3);
        const double2 q1 = caxpd(s.a1, p1, d.d1), q2 = caxpd(s.a2, p1, d.d2), q3 = caxpd(s.a1, p1, d.d3);
        const double2 xlo = DOWN ? x0 : x2, xhi = DOWN ? x2 : x0;
        double2 rhs = cmul(q1, xlo);
        rhs = c2(rhs.x + (q2.x * x1.x - q2.y * x1.y) + (q3.x * xhi.x - q3.y * xhi.y),
                 rhs.y + (q2.x * x1.y + q2.y * x1.x) + (q3.x * xhi.y + q3.y * xhi.x));
        // DOWN: couple to the row above (r1), continue with r3; UP: the reverse
        const double2 cin = DOWN ? r1 : r3, cout = DOWN ? r3 : r1;
        const double2 inv = crcp(cfms(r2, cin, wp));
        wp = cmul(cout, inv);
        gp = cmul(cfms(rhs, cin, gp), inv);
        const long long om = (long long)m * kTile;
        c.W[om] = wp;
        c.G[om] = gp;
    }
    cp_wait<0>();
}

// Term 0 eliminates DOWN from the stored field; term t eliminates DOWN when t
// is even and UP when t is odd, fused with the back-substitution of term t-1.
__device__ void pe_step(const StepCtx& s, Ring& R, const double2* p1, const double2* p2, int n) {
    run_pass<kFirst, true>(s, R, p1[0], p2[0]);
    for (int t = 1; t < n; ++t) {
        if (t & 1) run_pass<kFused, false>(s, R, p1[t], p2[t]);
        else run_pass<kFused, true>(s, R, p1[t], p2[t]);
    }
    // last term eliminated DOWN (n-1 even) -> back-substitute UP, and vice versa
    if (((n - 1) & 1) == 0) run_pass<kLast, false>(s, R, c2(0, 0), c2(0, 0));
    else run_pass<kLast, true>(s, R, c2(0, 0), c2(0, 0));
}

// ---------------------------------------------------------------------------
// factorised march: the operator of a term is fixed until the environment
// (profiles, bathymetry index) or the Pade set changes, so its Thomas
// factorisation - the expensive, strictly serial part with a division per
// row - is computed once per change and every range step only runs
//     g_m = S1 x_{m-1} + S2 x_m + S3 x_{m+1} + AL g_{m-/+1}     (elimination)
//     x_m = g_m - WF x_{m+/-1}                                  (back-substitution)
// with S_k = s_k / den_m, AL = -(coupling) / den_m, WF = w_m.
// ---------------------------------------------------------------------------
struct Fac {
    double2 *S1, *S2, *S3, *AL, *WF;  // already offset to (term, row 0, lane)
};

__device__ __forceinline__ Fac fac_term(const MarchArgs& a, const RayDev& ry, int t) {
    const long long o = ry.ccol + (long long)t * ry.crows * kTile;
    return Fac{a.S1 + o, a.S2 + o, a.S3 + o, a.AL + o, a.WF + o};
}

// Factorise one term (pd1 = p1, pd2 = p2) eliminating DOWN or UP.
template <bool DOWN>
__device__ void factor_pass(const StepCtx& s, Ring& R, double2 p1, double2 p2, const Fac& f) {
    const Col& c = s.c;
    const int nz = s.nz;
    const int lane = threadIdx.x;
    const int nrows = nz + 2;
    __threadfence_block();
#pragma unroll 1
    for (int k = 0; k < kRing; ++k) ring_issue<kEnvOnly>(R, c, k, DOWN ? k : nz + 1 - k, nz, lane);
    EnvRow em{}, ec{}, ep{};
    double2 wp = c2(0.0, 0.0);
#pragma unroll 1
    for (int k = 0; k < nrows; ++k) {
        const int r = DOWN ? k : nz + 1 - k;
        const int slot = k & (kRing - 1);
        cp_wait<kRing - 1>();
        EnvRow er;
        {
            const float* fl = ring_f(R, slot, lane);
            er.f1 = fl[0];
            er.f2 = fl[1];
            er.f3 = fl[2];
            er.k = *ring_k(R, slot, lane);
        }
        ring_issue<kEnvOnly>(R, c, slot, DOWN ? k + kRing : nz + 1 - k - kRing, nz, lane);
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
        const Drow d = galerkin3(em, ec, ep, s.cfact);
        const double2 r1 = caxpd(s.a1, p2, d.d1), r2 = caxpd(s.a2, p2, d.d2), r3 = caxpd(s.a1, p2, d.d3);
        const double2 q1 = caxpd(s.a1, p1, d.d1), q2 = caxpd(s.a2, p1, d.d2), q3 = caxpd(s.a1, p1, d.d3);
        const double2 cin = DOWN ? r1 : r3, cout = DOWN ? r3 : r1;
        const double2 inv = crcp(cfms(r2, cin, wp));
        wp = cmul(cout, inv);
        const long long om = (long long)m * kTile;
        f.S1[om] = cmul(q1, inv);
        f.S2[om] = cmul(q2, inv);
        f.S3[om] = cmul(q3, inv);
        const double2 ci = cmul(cin, inv);
        f.AL[om] = c2(-ci.x, -ci.y);
        f.WF[om] = wp;
    }
    cp_wait<0>();
}

// Stream row r of a factorised pass: field or W of the previous term, G, and
// the elimination factors of row m = r -/+ 1 of the current term.
template <int KIND, bool DOWN>
__device__ __forceinline__ void ring_issue_fac(Ring& R, const Col& c, int slot, int r, int nz, int lane,
                                               const double2* Wprev, const Fac& f) {
    if (r >= 0 && r <= nz + 1) {
        const long long o = (long long)r * kTile;
        if (KIND == kFirst) cp16(&R.q[slot][0][lane], c.u + o);
        else {
            cp16(&R.q[slot][0][lane], Wprev + o);
            cp16(&R.q[slot][1][lane], c.G + o);
        }
        const int m = DOWN ? r - 1 : r + 1;
        if (KIND != kLast && m >= 1 && m <= nz) {
            const long long om = (long long)m * kTile;
            cp16(&R.q[slot][2][lane], f.S1 + om);
            cp16(&R.q[slot][3][lane], f.S2 + om);
            cp16(&R.q[slot][4][lane], f.S3 + om);
            cp16(&R.q[slot][5][lane], f.AL + om);
        }
    }
    cp_commit();
}

// One factorised pass (same stream order and one-row lag as run_pass).
template <int KIND, bool DOWN>
__device__ void run_pass_fac(const StepCtx& s, Ring& R, const double2* Wprev, const Fac& f) {
    const Col& c = s.c;
    const int nz = s.nz;
    const int lane = threadIdx.x;
    const int nrows = nz + 2;
    __threadfence_block();
#pragma unroll 1
    for (int k = 0; k < kRing; ++k)
        ring_issue_fac<KIND, DOWN>(R, c, k, DOWN ? k : nz + 1 - k, nz, lane, Wprev, f);
    double2 x0 = c2(0.0, 0.0), x1 = c2(0.0, 0.0), x2 = c2(0.0, 0.0);
    double2 gp = c2(0.0, 0.0);
    const double2 zero = c2(0.0, 0.0);
#pragma unroll 1
    for (int k = 0; k < nrows; ++k) {
        const int r = DOWN ? k : nz + 1 - k;
        const int slot = k & (kRing - 1);
        cp_wait<kRing - 1>();
        const double2 av = R.q[slot][0][lane];
        double2 bv = zero, s1 = zero, s2 = zero, s3 = zero, al = zero;
        if (KIND != kFirst) bv = R.q[slot][1][lane];
        if (KIND != kLast) {
            s1 = R.q[slot][2][lane];
            s2 = R.q[slot][3][lane];
            s3 = R.q[slot][4][lane];
            al = R.q[slot][5][lane];
        }
        ring_issue_fac<KIND, DOWN>(R, c, slot, DOWN ? k + kRing : nz + 1 - k - kRing, nz, lane, Wprev, f);
        // x_r = g_r - w_r x_prev as two dependent FMAs per component
        const double2 xb = c2(fma(-av.x, x2.x, fma(av.y, x2.y, bv.x)), fma(-av.x, x2.y, fma(-av.y, x2.x, bv.y)));
        double2 xr;
        if (KIND == kFirst) {
            xr = (r == 0) ? s.u0 : (r == nz + 1 ? zero : av);
        } else if (DOWN) {
            xr = (r == 0) ? s.u0 : (r == nz + 1 ? zero : (r == 1 ? bv : xb));
        } else {
            xr = (r == nz + 1) ? zero : (r == 0 ? s.u0 : (r == nz ? bv : xb));
        }
        if (KIND == kLast) {
            if (r >= 1 && r <= nz) c.u[(long long)r * kTile] = xr;
            x2 = xr;
            continue;
        }
        x0 = x1;
        x1 = x2;
        x2 = xr;
        if (k < 2) continue;
        const int m = DOWN ? r - 1 : r + 1;
        if (m < 1 || m > nz) continue;
        const double2 xlo = DOWN ? x0 : x2, xhi = DOWN ? x2 : x0;
        // the two older field values first, then the new one, then the recurrence
        double2 t = c2(fma(s1.x, xlo.x, fma(-s1.y, xlo.y, fma(s2.x, x1.x, -s2.y * x1.y))),
                       fma(s1.x, xlo.y, fma(s1.y, xlo.x, fma(s2.x, x1.y, s2.y * x1.x))));
        t = c2(fma(s3.x, xhi.x, fma(-s3.y, xhi.y, t.x)), fma(s3.x, xhi.y, fma(s3.y, xhi.x, t.y)));
        const double2 g = c2(fma(al.x, gp.x, fma(-al.y, gp.y, t.x)), fma(al.x, gp.y, fma(al.y, gp.x, t.y)));
        gp = g;
        c.G[(long long)m * kTile] = g;
    }
    cp_wait<0>();
}

__device__ void factor_set(const StepCtx& s, Ring& R, const MarchArgs& a, const RayDev& ry,
                           const double2* p1, const double2* p2, int n) {
    for (int t = 0; t < n; ++t) {
        const Fac f = fac_term(a, ry, t);
        if (t & 1) factor_pass<false>(s, R, p1[t], p2[t], f);
        else factor_pass<true>(s, R, p1[t], p2[t], f);
    }
}

__device__ void pe_step_fac(const StepCtx& s, Ring& R, const MarchArgs& a, const RayDev& ry, int n) {
    run_pass_fac<kFirst, true>(s, R, nullptr, fac_term(a, ry, 0));
    for (int t = 1; t < n; ++t) {
        const double2* wprev = fac_term(a, ry, t - 1).WF;
        if (t & 1) run_pass_fac<kFused, false>(s, R, wprev, fac_term(a, ry, t));
        else run_pass_fac<kFused, true>(s, R, wprev, fac_term(a, ry, t));
    }
    const Fac last = fac_term(a, ry, n - 1);
    if (((n - 1) & 1) == 0) run_pass_fac<kLast, false>(s, R, last.WF, last);
    else run_pass_fac<kLast, true>(s, R, last.WF, last);
}

// Receiver line and TL grid after a step (outpt.py:11-57).  The CP grid is
// filled as well (the reference allocates it but never writes it).
__device__ void write_outputs(const MarchArgs& a, const RayDev& ry, const Col& c, double2 u0,
                              int tlc, double r, int ir, double dir, int* flag) {
    auto urow = [&](int i) -> double2 {
        if (i <= 0) return u0;
        if (i > ry.nz) return c2(0.0, 0.0);
        return c.u[(long long)i * kTile];
    };
    const double2 ua = urow(ir), ub = urow(ir + 1);
    const double fa = c.f3[(long long)ir * kTile];
    const double fb = c.f3[(long long)(ir + 1) * kTile];
    const double2 cp = c2((1.0 - dir) * fa * ua.x + dir * fb * ub.x, (1.0 - dir) * fa * ua.y + dir * fb * ub.y);
    const double amp = hypot(cp.x, cp.y);
    if (!isfinite(amp)) *flag |= 1;
    a.tll[ry.line_off + tlc] = tl_db(amp, r);
    a.cpl[ry.line_off + tlc] = cp;
    if (a.compute_grids && ry.grid_off >= 0) {
        for (int k = 0; k < ry.nvz; ++k) {
            const int j = (k + 1) * ry.ndz;
            if (j > ry.nz + 1) break;
            const double2 uj = urow(j);
            const double fj = c.f3[(long long)j * kTile];
            const double2 g = c2(uj.x * fj, uj.y * fj);
            const long long o = ry.grid_off + (long long)k * ry.nvr + tlc;
            a.tlg[o] = tl_db(hypot(g.x, g.y), r);
            a.cpg[o] = g;
        }
    }
}

// ---------------------------------------------------------------------------
// the march kernel: one lane = one ray, all steps
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) march_kernel(MarchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Ring& ring = *reinterpret_cast<Ring*>(smem_raw);
    const int rid = a.tile_ray[blockIdx.x * kTile + threadIdx.x];
    if (rid < 0) return;
    const RayDev ry = a.rays[rid];
    const EnvPtrs e = env_ptrs(a.envs[ry.env], a.pool);
    Col c;
    c.f1 = a.f1 + ry.col;
    c.f2 = a.f2 + ry.col;
    c.f3 = a.f3 + ry.col;
    c.ksq = a.ksq + ry.col;
    c.u = a.u + ry.col;
    c.W = a.W + ry.col;
    c.G = a.G + ry.col;
    const int nz = ry.nz;
    int flag = 0;

    // initial indices (cupyram.py:571-608)
    int iz = (int)floor(e.zb[0] / ry.dz);
    iz = max(1, min(nz - 1, iz));
    int ss = 0, sb = 0, bt = 0;
    assemble_rows(ry, e, ss, sb, iz, 0, nz + 1, a.f1, a.f2, a.f3, a.ksq);

    StepCtx s;
    s.c = c;
    s.nz = nz;
    s.cfact = 0.5 / (ry.dz * ry.dz);
    s.a1 = ry.k0 * ry.k0 / 6.0;
    s.a2 = 2.0 * ry.k0 * ry.k0 / 3.0;

    // self-starter: delta at zs split over two rows, divided by (1-X)^2
    // (two passes of the pd1 = 0, pd2 = -1 operator), then the ip = 2 operator
    for (int i = 0; i <= nz + 1; ++i) c.u[(long long)i * kTile] = c2(0.0, 0.0);
    {
        const double si = ry.zs / ry.dz;
        const int is = (int)floor(si);
        const double dis = si - is;
        const double amp = sqrt(2.0 * M_PI / ry.k0);
        const double step = ry.zmax / (double)(nz + 1);
        for (int k = 0; k < 2; ++k) {
            const int i = is + k;
            const double z = (i == nz + 1) ? ry.zmax : (double)i * step;
            const RowProps p = row_props(e, ss, sb, z, ry.lyrw_lambda, ry.attnf);
            const double alpw = sqrt((double)p.cw / ry.c0);
            const double wgt = (k == 0) ? (1.0 - dis) : dis;
            c.u[(long long)i * kTile] = c2(wgt * amp / (ry.dz * alpw), 0.0);
        }
        s.u0 = c.u[0];
    }
    const double2* pd1 = a.pd1 + (long long)rid * kSets * CR_MAX_NP;
    const double2* pd2 = a.pd2 + (long long)rid * kSets * CR_MAX_NP;
    const int* pn = a.pd_n + rid * kSets;
    pe_step(s, ring, pd1, pd2, pn[0]);
    pe_step(s, ring, pd1, pd2, pn[0]);
    pe_step(s, ring, pd1 + CR_MAX_NP, pd2 + CR_MAX_NP, pn[1]);

    const double ri = ry.zr / ry.dz;
    const int ir = (int)floor(ri);
    const double dir = ri - ir;
    int mdr = 0, tlc = -1;
    double r = ry.dr;
    if (++mdr == ry.ndr) {
        mdr = 0;
        ++tlc;
        if (tlc < ry.nvr) write_outputs(a, ry, c, s.u0, tlc, r, ir, dir, &flag);
    }

    int set = 2;
    double rs = ry.rs;
    const bool factored = a.S1 != nullptr && ry.ccol >= 0;
    bool refactor = true;
    for (int rn = 0; rn < ry.nr; ++rn) {
        // updat (updat.py:38-140): bathymetry index at r + dr/2, profile indices at r
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
            const int o = ss;
            while (ss < e.n_rss - 1 && r >= e.rp_ss[ss + 1]) ++ss;
            reprofile |= (ss != o);
        }
        if (e.n_rsb > 1) {
            const int o = sb;
            while (sb < e.n_rsb - 1 && r >= e.rp_sb[sb + 1]) ++sb;
            reprofile |= (sb != o);
        }
        if (reprofile) {
            assemble_rows(ry, e, ss, sb, iz_new, 0, nz + 1, a.f1, a.f2, a.f3, a.ksq);
            refactor = true;
        } else if (iz_new != iz) {
            // only the rows that change layer
            assemble_rows(ry, e, ss, sb, iz_new, min(iz, iz_new) + 1, max(iz, iz_new), a.f1, a.f2,
                          a.f3, a.ksq);
            refactor = true;
        }
        iz = iz_new;
        if (r >= rs) {  // stability constraints off (cupyram.py:976-999)
            set = 3;
            rs = INFINITY;
            refactor = true;
        }
        if (factored) {
            if (refactor) {
                factor_set(s, ring, a, ry, pd1 + set * CR_MAX_NP, pd2 + set * CR_MAX_NP, pn[set]);
                refactor = false;
            }
            pe_step_fac(s, ring, a, ry, pn[set]);
        } else {
            pe_step(s, ring, pd1 + set * CR_MAX_NP, pd2 + set * CR_MAX_NP, pn[set]);
        }
        r = (double)(rn + 2) * ry.dr;
        if (++mdr == ry.ndr) {
            mdr = 0;
            ++tlc;
            if (tlc < ry.nvr) write_outputs(a, ry, c, s.u0, tlc, r, ir, dir, &flag);
        }
    }
    a.flags[rid] = flag;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
thread_local std::string g_error;

void set_global_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}

}  // namespace

struct cr_engine {
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int n_rays = 0, n_envs = 0, n_tiles = 0;
    int precision = 0, compute_grids = 0;
    long long line_len = 0, grid_len = 0, pool_len = 0;
    long long col_elems = 0;
    double point_updates = 0.0;
    // host copies
    std::vector<RayDev> rays;
    std::vector<EnvDev> envs;
    std::vector<double> pool;
    std::vector<int> tile_ray;
    std::vector<double2> pd1, pd2;
    std::vector<int> pd_n;
    // device buffers
    RayDev* d_rays = nullptr;
    EnvDev* d_envs = nullptr;
    double* d_pool = nullptr;
    int* d_tile_ray = nullptr;
    double2 *d_pd1 = nullptr, *d_pd2 = nullptr;
    int* d_pd_n = nullptr;
    float *d_f1 = nullptr, *d_f2 = nullptr, *d_f3 = nullptr;
    float2* d_ksq = nullptr;
    double2 *d_u = nullptr, *d_W = nullptr, *d_G = nullptr;
    double* d_tll = nullptr;
    double2* d_cpl = nullptr;
    double* d_tlg = nullptr;
    double2* d_cpg = nullptr;
    int* d_flags = nullptr;
    double2 *d_S1 = nullptr, *d_S2 = nullptr, *d_S3 = nullptr, *d_AL = nullptr, *d_WF = nullptr;
    long long fac_elems = 0;
    // partial-fraction (sum form) march
    bool sum_mode = false;
    std::vector<int> tile_G;
    std::vector<long long> tile_off, tile_loff;
    long long lane_elems = 0;
    std::vector<double2> pfc, pfcinf;
    int* d_tile_G = nullptr;
    // device work queue of the batched march: tiles in longest-march-first
    // order and the ticket counter the persistent launch takes them by
    bool queue_mode = true;
    std::vector<int> queue;
    int* d_queue = nullptr;
    int* d_ticket = nullptr;
    long long* d_tile_off = nullptr;
    long long* d_tile_loff = nullptr;
    double2 *d_pfc = nullptr, *d_pfcinf = nullptr;
    double2 *d_QD = nullptr, *d_WD = nullptr, *d_QU = nullptr, *d_WU = nullptr, *d_ED = nullptr, *d_EU = nullptr;
    double2* d_E2 = nullptr;  // refined form: the rows' d2
    // column-parallel march: rays marched by one thread-block cluster each,
    // one launch per (Pade term count) group on its own stream
    struct ColGroup {
        int cluster, terms, nz_max, begin, count;
        cudaStream_t stream;
        cudaEvent_t done;
    };
    std::vector<int> col_ray;
    std::vector<ColGroup> col_groups;
    // batched launches after the first run on their own streams
    std::vector<cudaStream_t> sum_streams;
    std::vector<cudaEvent_t> sum_done;
    std::vector<int> term_capacity;  // Pade terms each ray's lanes / cluster can carry
    int* d_col_ray = nullptr;
    cudaEvent_t ev_fork = nullptr;
    long long device_bytes = 0;
    bool uploaded = false, marched = false;
    cr_stats st{};

    int fail(int code, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        return fail(e == cudaErrorMemoryAllocation ? CR_ENOMEM : CR_ECUDA, "%s: %s", what,
                    cudaGetErrorString(e));
    }
};

namespace {

// Device memory of the engines comes from one stream-ordered pool per device
// that keeps freed memory for the next engine (release threshold: never), so
// that building an engine for every batch - as CuPyRAM.run() does - costs no
// fresh cudaMalloc / cudaFree after the first one.  cr_release_cache() hands
// the pooled memory back to the device.
constexpr int kPoolDevices = 64;
cudaMemPool_t g_pools[kPoolDevices] = {};
std::mutex g_pool_mu;

cudaError_t engine_pool(int dev, cudaMemPool_t* out) {
    if (dev < 0 || dev >= kPoolDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        cudaError_t ce = cudaMemPoolCreate(&pool, &props);
        if (ce != cudaSuccess) return ce;
        unsigned long long keep = ~0ULL;
        ce = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (ce != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return ce;
        }
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return cudaSuccess;
}

template <typename T>
cudaError_t dev_alloc(cr_engine* e, T** p, size_t count) {
    if (count == 0) count = 1;
    const size_t bytes = count * sizeof(T);
    cudaMemPool_t pool = nullptr;
    cudaError_t rc = engine_pool(e->device, &pool);
    if (rc == cudaSuccess) rc = cudaMallocFromPoolAsync((void**)p, bytes, pool, e->stream);
    if (rc == cudaSuccess) e->device_bytes += (long long)bytes;
    return rc;
}

void free_all(cr_engine* e) {
    void* ptrs[] = {e->d_rays, e->d_envs, e->d_pool, e->d_tile_ray, e->d_pd1, e->d_pd2, e->d_pd_n,
                    e->d_f1,   e->d_f2,   e->d_f3,   e->d_ksq,      e->d_u,   e->d_W,   e->d_G,
                    e->d_tll,  e->d_cpl,  e->d_tlg,  e->d_cpg,      e->d_flags, e->d_S1, e->d_S2,
                    e->d_S3,   e->d_AL,   e->d_WF,   e->d_tile_G,  e->d_tile_off, e->d_tile_loff, e->d_pfc, e->d_pfcinf,
                    e->d_QD,   e->d_WD,   e->d_QU,   e->d_WU,      e->d_ED,  e->d_EU, e->d_col_ray,
                    e->d_queue, e->d_ticket, e->d_E2};
    // stream-ordered frees on the engine's stream (every other stream of the
    // engine joins it at the end of each march), back into the pool
    if (e->stream) {
        for (void* p : ptrs)
            if (p) cudaFreeAsync(p, e->stream);
        cudaStreamSynchronize(e->stream);
    }
    for (auto& g : e->col_groups) {
        if (g.done) cudaEventDestroy(g.done);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    for (size_t i = 1; i < e->sum_streams.size(); ++i)
        if (e->sum_streams[i]) cudaStreamDestroy(e->sum_streams[i]);
    for (auto ev : e->sum_done)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : e->ev)
        if (ev) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
}

// Pinned staging of host-to-device copies.  A pageable cudaMemcpy is staged
// by the driver through its own pinned buffers, one host copy at a time; here
// each device has a ring of two pinned chunks, allocated once: while one
// chunk's DMA runs, host threads fill the other, so the host copy and the
// transfer overlap and the copy itself runs on several cores.
constexpr size_t kStageChunk = 16u << 20;  // bytes per chunk
constexpr size_t kStageMin = 4u << 20;     // smaller copies go direct
constexpr int kStageThreads = 4;
struct StageRing {
    unsigned char* buf[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
};
StageRing g_stage[kPoolDevices];
std::mutex g_stage_mu[kPoolDevices];

void copy_parallel(unsigned char* dst, const unsigned char* src, size_t n) {
    if (n < (1u << 20)) {
        memcpy(dst, src, n);
        return;
    }
    std::thread th[kStageThreads - 1];
    const size_t part = (n / kStageThreads + 63) & ~size_t(63);
    for (int t = 1; t < kStageThreads; ++t) {
        const size_t lo = std::min(n, part * t), hi = std::min(n, part * (t + 1));
        th[t - 1] = std::thread([=] { memcpy(dst + lo, src + lo, hi - lo); });
    }
    memcpy(dst, src, std::min(n, part));
    for (auto& x : th) x.join();
}

// Host-to-device copy of `bytes` through the device's pinned ring, ordered on
// `st`.  Returns when the last chunk's copy has been queued (the caller
// synchronises the stream); the ring is held until then.
cudaError_t staged_h2d(int dev, void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (dev < 0 || dev >= kPoolDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_stage_mu[dev]);
    StageRing& R = g_stage[dev];
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < 2 && ce == cudaSuccess; ++k) {
        if (!R.buf[k]) ce = cudaHostAlloc((void**)&R.buf[k], kStageChunk, cudaHostAllocPortable);
        if (ce == cudaSuccess && !R.done[k]) ce = cudaEventCreateWithFlags(&R.done[k], cudaEventDisableTiming);
    }
    const unsigned char* s = (const unsigned char*)src;
    unsigned char* d = (unsigned char*)dst;
    int k = 0;
    for (size_t off = 0; off < bytes && ce == cudaSuccess; off += kStageChunk, k ^= 1) {
        const size_t n = std::min(kStageChunk, bytes - off);
        ce = cudaEventSynchronize(R.done[k]);  // the chunk's previous DMA has finished
        if (ce != cudaSuccess) break;
        copy_parallel(R.buf[k], s + off, n);
        ce = cudaMemcpyAsync(d + off, R.buf[k], n, cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess) ce = cudaEventRecord(R.done[k], st);
    }
    // the ring is reused by the next call only after these copies: wait for them
    for (int j = 0; j < 2 && ce == cudaSuccess; ++j) ce = cudaEventSynchronize(R.done[j]);
    return ce;
}

// Validate the batch; returns an error message or empty string.
std::string validate(const cr_batch* b) {
    char buf[256];
    if (!b) return "batch is NULL";
    if (b->n_rays < 1) return "n_rays must be >= 1";
    if (b->n_envs < 1) return "n_envs must be >= 1";
    if (!b->rays || !b->envs || !b->pool) return "rays, envs and pool must be non-NULL";
    if (b->precision < CR_PLAIN_C128 || b->precision > CR_C64_REFINED) return "unknown precision form";
    for (int k = 0; k < b->n_envs; ++k) {
        const cr_env& v = b->envs[k];
        if (v.n_zss < 1 || v.n_rss < 1 || v.n_zsb < 1 || v.n_rsb < 1 || v.n_bt < 1) {
            snprintf(buf, sizeof buf, "environment %d has an empty profile or bathymetry", k);
            return buf;
        }
        const long long need = (long long)v.n_zss + v.n_rss + (long long)v.n_rss * v.n_zss + v.n_zsb +
                               v.n_rsb + 3LL * v.n_rsb * v.n_zsb + 2LL * v.n_bt;
        if (v.off < 0 || v.off + need > b->pool_len) {
            snprintf(buf, sizeof buf, "environment %d overruns the pool", k);
            return buf;
        }
    }
    for (int i = 0; i < b->n_rays; ++i) {
        const cr_ray& r = b->rays[i];
        auto bad = [&](const char* what) {
            snprintf(buf, sizeof buf, "ray %d: %s", i, what);
            return std::string(buf);
        };
        if (r.env < 0 || r.env >= b->n_envs) return bad("env index out of range");
        if (!(r.freq > 0) || !(r.c0 > 0)) return bad("freq and c0 must be > 0");
        if (!(r.dz > 0) || !(r.dr > 0)) return bad("dz and dr must be > 0");
        if (r.nz < 3) return bad("nz must be >= 3");
        if (r.nr < 0) return bad("nr must be >= 0");
        if (r.np < 1 || r.np > CR_MAX_NP) return bad("np out of range");
        if (r.ns < 0 || r.ns > 2) return bad("ns must be 0, 1 or 2");
        if (r.ndr < 1 || r.ndz < 1) return bad("ndr and ndz must be >= 1");
        if (r.nvr < 0 || r.nvz < 0) return bad("nvr and nvz must be >= 0");
        if (!(r.zs >= 0) || (int)std::floor(r.zs / r.dz) + 1 > r.nz) return bad("source depth outside the grid");
        if (!(r.zr >= 0) || (int)std::floor(r.zr / r.dz) + 1 > r.nz + 1) return bad("receiver depth outside the grid");
        if (r.line_off < 0 || r.line_off + r.nvr > b->line_len) return bad("TL line overruns line_len");
        if (b->compute_grids && r.grid_off >= 0 && r.grid_off + (long long)r.nvz * r.nvr > b->grid_len)
            return bad("TL grid overruns grid_len");
        if ((long long)(r.nvr) * r.ndr > (long long)r.nr + 1) return bad("nvr * ndr exceeds nr + 1 outputs");
    }
    return std::string();
}

// One Pade solve of a batch: (freq, c0, dr, np, ns, ip).
struct PadeJob {
    double freq, c0, dr;
    int np, ns, ip, pad_;
};

// One thread per job: the FP64 Pade construction of pade.h on the device.
// pd1 / pd2 get CR_MAX_NP coefficients per job (zeros past np); status gets
// CR_OK, CR_EPADE (Laguerre did not converge) or CR_EINVAL.
__global__ void pade_batch_kernel(const PadeJob* __restrict__ jobs, int n, double2* __restrict__ pd1,
                                  double2* __restrict__ pd2, int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PadeJob j = jobs[i];
    cr::cd a[CR_MAX_NP], c[CR_MAX_NP];
    const int rc = cr::pade_coefficients(j.freq, j.c0, j.np, j.ns, j.dr, j.ip, a, c);
    status[i] = rc == cr::kPadeOk ? CR_OK : (rc == cr::kPadeNoConverge ? CR_EPADE : CR_EINVAL);
    for (int k = 0; k < CR_MAX_NP; ++k) {
        const bool on = rc == cr::kPadeOk && k < j.np;
        pd1[(size_t)i * CR_MAX_NP + k] = on ? make_double2(a[k].re, a[k].im) : make_double2(0.0, 0.0);
        pd2[(size_t)i * CR_MAX_NP + k] = on ? make_double2(c[k].re, c[k].im) : make_double2(0.0, 0.0);
    }
}

// Solve a batch of Pade jobs on the current device (temporary device memory
// on a private stream; synchronous).  pd1 / pd2: [n][CR_MAX_NP], status: [n].
cudaError_t device_pade(const std::vector<PadeJob>& jobs, std::vector<double2>& pd1, std::vector<double2>& pd2,
                        std::vector<int>& status) {
    const int n = (int)jobs.size();
    pd1.assign((size_t)n * CR_MAX_NP, make_double2(0.0, 0.0));
    pd2.assign((size_t)n * CR_MAX_NP, make_double2(0.0, 0.0));
    status.assign((size_t)n, CR_OK);
    if (n == 0) return cudaSuccess;
    cudaStream_t st = nullptr;
    cudaError_t ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return ce;
    // regions rounded up to 256 bytes: the coefficient arrays are double2 and
    // must start on a 16-byte boundary whatever the number of jobs
    auto r256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t bj = r256(jobs.size() * sizeof(PadeJob)), bp = r256(pd1.size() * sizeof(double2)),
                 bs = r256((size_t)n * sizeof(int));
    unsigned char* d = nullptr;
    ce = cudaMallocAsync((void**)&d, bj + 2 * bp + bs, st);
    if (ce == cudaSuccess) {
        PadeJob* dj = (PadeJob*)d;
        double2* d1 = (double2*)(d + bj);
        double2* d2 = (double2*)(d + bj + bp);
        int* ds = (int*)(d + bj + 2 * bp);
        ce = cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(PadeJob), cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess) {
            // 32 threads a block: the solves are long serial chains, so the
            // jobs are spread over as many SMs as possible
            pade_batch_kernel<<<(n + 31) / 32, 32, 0, st>>>(dj, n, d1, d2, ds);
            ce = cudaGetLastError();
        }
        const size_t np2 = pd1.size() * sizeof(double2);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(pd1.data(), d1, np2, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(pd2.data(), d2, np2, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(status.data(), ds, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st);
        const cudaError_t cf = cudaFreeAsync(d, st);
        if (ce == cudaSuccess) ce = cf;
    }
    const cudaError_t cs = cudaStreamSynchronize(st);
    if (ce == cudaSuccess) ce = cs;
    cudaStreamDestroy(st);
    return ce;
}

// Pade sets for every ray, solved on the device; identical (freq, c0, np,
// ns, dr) share one solve.
int compute_pade_sets(cr_engine* e, const cr_batch* b) {
    using Key = std::tuple<double, double, int, int, double>;
    std::map<Key, int> uniq;
    std::vector<Key> keys;
    std::vector<int> ray_key(b->n_rays);
    for (int i = 0; i < b->n_rays; ++i) {
        const cr_ray& r = b->rays[i];
        Key k{r.freq, r.c0, r.np, r.ns, r.dr};
        auto it = uniq.find(k);
        if (it == uniq.end()) {
            it = uniq.emplace(k, (int)keys.size()).first;
            keys.push_back(k);
        }
        ray_key[i] = it->second;
    }
    const int nk = (int)keys.size();
    // per key: set1 (ip=2, ns), set2 (ip=1, ns), set3 (ip=1, ns=0)
    std::vector<PadeJob> jobs((size_t)nk * 3);
    for (int k = 0; k < nk; ++k) {
        const auto& [freq, c0, np, ns, dr] = keys[k];
        jobs[(size_t)k * 3 + 0] = PadeJob{freq, c0, dr, np, ns, 2, 0};
        jobs[(size_t)k * 3 + 1] = PadeJob{freq, c0, dr, np, ns, 1, 0};
        jobs[(size_t)k * 3 + 2] = PadeJob{freq, c0, dr, np, 0, 1, 0};
    }
    std::vector<double2> r1, r2;
    std::vector<int> status;
    const cudaError_t ce = device_pade(jobs, r1, r2, status);
    if (ce != cudaSuccess)
        return e->fail(ce == cudaErrorMemoryAllocation ? CR_ENOMEM : CR_ECUDA, "cr_create: Pade on the device: %s",
                       cudaGetErrorString(ce));
    for (int k = 0; k < nk; ++k)
        for (int s = 0; s < 3; ++s)
            if (status[(size_t)k * 3 + s] != CR_OK) {
                const auto& [freq, c0, np, ns, dr] = keys[k];
                return e->fail(status[(size_t)k * 3 + s] == CR_EPADE ? CR_EPADE : CR_EINVAL,
                               "Pade coefficients failed (freq=%g c0=%g np=%d ns=%d dr=%g): %s", freq, c0, np, ns,
                               dr, status[(size_t)k * 3 + s] == CR_EPADE ? "Laguerre method not converging"
                                                                          : "bad arguments");
            }
    e->pd1.assign((size_t)b->n_rays * kSets * CR_MAX_NP, make_double2(0.0, 0.0));
    e->pd2.assign((size_t)b->n_rays * kSets * CR_MAX_NP, make_double2(0.0, 0.0));
    e->pd_n.assign((size_t)b->n_rays * kSets, 0);
    for (int i = 0; i < b->n_rays; ++i) {
        const int np = b->rays[i].np;
        double2* p1 = e->pd1.data() + (size_t)i * kSets * CR_MAX_NP;
        double2* p2 = e->pd2.data() + (size_t)i * kSets * CR_MAX_NP;
        p1[0] = make_double2(0.0, 0.0);
        p2[0] = make_double2(-1.0, 0.0);
        e->pd_n[i * kSets + 0] = 1;
        for (int s = 1; s < kSets; ++s) {
            const size_t jb = ((size_t)ray_key[i] * 3 + (s - 1)) * CR_MAX_NP;
            for (int j = 0; j < np; ++j) {
                p1[s * CR_MAX_NP + j] = r1[jb + j];
                p2[s * CR_MAX_NP + j] = r2[jb + j];
            }
            e->pd_n[i * kSets + s] = np;
        }
    }
    return CR_OK;
}

}  // namespace

namespace {
// Named NVTX range over an entry point, for timelines in profilers (no cost
// when no tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace

extern "C" {

int cr_abi_version(void) { return CR_ABI_VERSION; }

int cr_global_error(char* buf, size_t len) {
    if (!buf || len == 0) return CR_EINVAL;
    snprintf(buf, len, "%s", g_error.c_str());
    return CR_OK;
}

int cr_pade(double freq, double c0, int np, int ns, double dr, int ip, double* pd1, double* pd2) {
    if (!pd1 || !pd2 || np < 1 || np > CR_MAX_NP || ns < 0 || ns > 2 || (ip != 1 && ip != 2)) {
        set_global_error("cr_pade: invalid arguments (np=%d ns=%d ip=%d)", np, ns, ip);
        return CR_EINVAL;
    }
    cr::cd a[CR_MAX_NP], b[CR_MAX_NP];
    const int rc = cr::pade_coefficients(freq, c0, np, ns, dr, ip, a, b);
    if (rc == cr::kPadeNoConverge) {
        set_global_error("Laguerre method not converging");
        return CR_EPADE;
    }
    if (rc) {
        set_global_error("cr_pade: invalid arguments (freq=%g c0=%g)", freq, c0);
        return CR_EINVAL;
    }
    for (int j = 0; j < np; ++j) {
        pd1[2 * j] = a[j].re;
        pd1[2 * j + 1] = a[j].im;
        pd2[2 * j] = b[j].re;
        pd2[2 * j + 1] = b[j].im;
    }
    return CR_OK;
}

int cr_pade_batch(int n, const double* freq, const double* c0, const int32_t* np, const int32_t* ns,
                  const double* dr, const int32_t* ip, double* pd1, double* pd2, int32_t* status) {
    NvtxRange nv("cr_pade_batch");
    if (n < 0 || (n > 0 && (!freq || !c0 || !np || !ns || !dr || !ip || !pd1 || !pd2 || !status))) {
        set_global_error("cr_pade_batch: invalid arguments");
        return CR_EINVAL;
    }
    std::vector<PadeJob> jobs((size_t)n);
    for (int i = 0; i < n; ++i) {
        if (np[i] < 1 || np[i] > CR_MAX_NP || ns[i] < 0 || ns[i] > 2 || (ip[i] != 1 && ip[i] != 2)) {
            set_global_error("cr_pade_batch: job %d: invalid arguments (np=%d ns=%d ip=%d)", i, np[i], ns[i], ip[i]);
            return CR_EINVAL;
        }
        jobs[(size_t)i] = PadeJob{freq[i], c0[i], dr[i], np[i], ns[i], ip[i], 0};
    }
    std::vector<double2> r1, r2;
    std::vector<int> st;
    const cudaError_t ce = device_pade(jobs, r1, r2, st);
    if (ce != cudaSuccess) {
        set_global_error("cr_pade_batch: %s", cudaGetErrorString(ce));
        return ce == cudaErrorMemoryAllocation ? CR_ENOMEM : CR_ECUDA;
    }
    int worst = CR_OK;
    for (int i = 0; i < n; ++i) {
        status[i] = st[(size_t)i];
        if (st[(size_t)i] != CR_OK && worst == CR_OK) {
            worst = st[(size_t)i];
            set_global_error("cr_pade_batch: job %d: %s", i,
                             worst == CR_EPADE ? "Laguerre method not converging" : "invalid arguments");
        }
        for (int j = 0; j < CR_MAX_NP; ++j) {  // zeros past np[i]
            pd1[2 * ((size_t)i * CR_MAX_NP + j)] = r1[(size_t)i * CR_MAX_NP + j].x;
            pd1[2 * ((size_t)i * CR_MAX_NP + j) + 1] = r1[(size_t)i * CR_MAX_NP + j].y;
            pd2[2 * ((size_t)i * CR_MAX_NP + j)] = r2[(size_t)i * CR_MAX_NP + j].x;
            pd2[2 * ((size_t)i * CR_MAX_NP + j) + 1] = r2[(size_t)i * CR_MAX_NP + j].y;
        }
    }
    return worst;
}

namespace {

// c_inf = prod_j pd1_j / pd2_j and the residues
// c_k = (1 - pd1_k/pd2_k) prod_{j != k} (1 - pd1_j/pd2_k) / (1 - pd2_j/pd2_k)
// of Pade set `st` of a ray: prod_j (1 + pd1_j X)/(1 + pd2_j X) = c_inf + sum_k c_k/(1 + pd2_k X).
void partial_fractions(cr_engine* e, int ray, int st) {
    const int n = e->pd_n[(size_t)ray * kSets + st];
    const double2* p1 = e->pd1.data() + ((size_t)ray * kSets + st) * CR_MAX_NP;
    const double2* p2 = e->pd2.data() + ((size_t)ray * kSets + st) * CR_MAX_NP;
    auto C = [](double2 v) { return cr::cd{v.x, v.y}; };
    cr::cd cinf{1.0, 0.0};
    for (int j = 0; j < n; ++j) cinf = cinf * (C(p1[j]) / C(p2[j]));
    e->pfcinf[(size_t)ray * kSets + st] = make_double2(cinf.re, cinf.im);
    for (int k = 0; k < CR_MAX_NP; ++k) {
        double2 out = make_double2(0.0, 0.0);
        if (k < n) {
            cr::cd ck = cr::cd{1.0, 0.0} - C(p1[k]) / C(p2[k]);
            for (int j = 0; j < n; ++j)
                if (j != k) ck = ck * ((cr::cd{1.0, 0.0} - C(p1[j]) / C(p2[k])) / (cr::cd{1.0, 0.0} - C(p2[j]) / C(p2[k])));
            out = make_double2(ck.re, ck.im);
        }
        e->pfc[((size_t)ray * kSets + st) * CR_MAX_NP + k] = out;
    }
}

// Device record of a ray (everything but its column placement).
RayDev ray_dev(const cr_ray& r, bool grids) {
    RayDev d{};
    d.k0 = 2.0 * M_PI * r.freq / r.c0;
    d.omega = 2.0 * M_PI * r.freq;
    d.c0 = r.c0;
    d.dz = r.dz;
    d.dr = r.dr;
    d.zmax = r.zmax;
    d.lyrw_lambda = r.lyrw_lambda;
    d.attnf = r.attnf;
    d.rs = r.rs;
    d.zs = r.zs;
    d.zr = r.zr;
    d.nz = r.nz;
    d.nr = r.nr;
    d.np = r.np;
    d.ndr = r.ndr;
    d.ndz = r.ndz;
    d.nvr = r.nvr;
    d.nvz = r.nvz;
    d.env = r.env;
    d.line_off = r.line_off;
    d.grid_off = grids ? r.grid_off : -1;
    d.ccol = -1;
    d.pad_ = 0;
    return d;
}

// Pade terms of a ray's largest set (the warps of its column-kernel CTAs).
int col_terms(const std::vector<int>& pd_n, int ray) {
    int t = 0;
    for (int s = 0; s < kSets; ++s) t = std::max(t, pd_n[(size_t)ray * kSets + s]);
    return t;
}

// Cluster size of each column ray.  The smallest cluster that holds the
// column in shared memory uses the fewest SMs per ray; when the column rays
// leave SMs idle, a ray gets up to SMs / rays CTAs (at most 16, at least 64
// rows per slice) so that its slices, and its steps, are shorter.  Only
// sizes whose clusters can be resident are used.
std::vector<int> column_clusters(const cr_batch* b, const std::vector<int>& pd_n, const std::vector<char>& is_col,
                                 bool chosen) {
    std::vector<int> cl((size_t)b->n_rays, 0);
    int n_col = 0;
    for (char c : is_col) n_col += c ? 1 : 0;
    if (n_col == 0) return cl;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int share = std::max(1, sms / n_col);
    std::map<std::tuple<int, int, int>, bool> runs;
    std::map<std::tuple<int, int, int>, int> dense;  // resident CTAs of a cluster size
    // target CTAs per SM for throughput-bound column launches ("0": keep the
    // smallest cluster)
    const char* env2 = getenv("CUPYRAM_B200_COL2");
    const int per_sm = env2 ? std::max(0, std::min(4, env2[0] - '0')) : 3;
    for (int i = 0; i < b->n_rays; ++i) {
        if (!is_col[(size_t)i]) continue;
        const int nz = b->rays[i].nz, terms = col_terms(pd_n, i);
        const int cmin = crk::col_cluster_size(nz, terms, chosen);
        int C = std::max(cmin, std::min({16, share, std::max(1, nz / 64)}));
        for (; C > cmin; --C) {
            const auto key = std::make_tuple(C, terms, nz);
            auto it = runs.find(key);
            if (it == runs.end()) it = runs.emplace(key, crk::col_max_active_clusters(C, terms, nz, chosen) > 0).first;
            if (it->second) break;
        }
        // many column rays: the launches are throughput-bound.  A larger
        // cluster whose CTAs fit three (else two) to an SM multiplies the
        // warps that hide each other's latencies.
        if (per_sm > 1 && (long long)n_col * cmin > sms) {
            for (int want = per_sm; want >= 2; --want) {
                int found = 0;
                for (int C2 = C + 1; C2 <= 16 && !found; ++C2) {
                    const auto key = std::make_tuple(C2, terms, nz);
                    auto it = dense.find(key);
                    if (it == dense.end())
                        it = dense.emplace(key, crk::col_max_active_clusters(C2, terms, nz, chosen) * C2).first;
                    if (2LL * it->second >= (2LL * want - 1) * sms) found = C2;
                }
                if (found) {
                    C = found;
                    break;
                }
            }
        }
        cl[(size_t)i] = C;
    }
    return cl;
}

// Operator changes a ray's march will see: bathymetry-index moves (the
// bottom's total depth excursion along the track over dz, capped at one per
// step) plus profile updates.
double operator_changes(const cr_batch* b, const cr_ray& r) {
    const cr_env& v = b->envs[r.env];
    const double* q = b->pool + v.off;
    q += v.n_zss + v.n_rss + (long long)v.n_rss * v.n_zss + v.n_zsb + v.n_rsb + 3LL * v.n_rsb * v.n_zsb;
    const double* rb = q;
    const double* zb = q + v.n_bt;
    const double rmax = r.dr * (r.nr + 1);
    double excursion = 0.0;
    for (int k = 0; k + 1 < v.n_bt && rb[k] < rmax; ++k) {
        const double r1 = std::min(rb[k + 1], rmax);
        const double frac = rb[k + 1] > rb[k] ? (r1 - rb[k]) / (rb[k + 1] - rb[k]) : 1.0;
        excursion += std::fabs(zb[k + 1] - zb[k]) * frac;
    }
    return std::min(excursion / r.dz, (double)r.nr) + (double)(v.n_rss - 1) + (double)(v.n_rsb - 1);
}

// Costs of the batched march that the column policy weighs, measured on the
// device by the engine's own tuner (march_costs) unless given explicitly.
struct MarchCosts {
    double row_step_s = 0.0;     // one batched tile alone: one row of one step
    double updates_per_s = 0.0;  // batched kernel over a device-filling batch
    double slots = 0.0;          // batched tiles the device holds at once
};

// The cost rule of the column policy.  A ray's lockstep march in a batched
// tile takes about (nz + 2)(nr + 4 + 4 x operator changes) row steps of one
// warp in sequence; when that alone exceeds the time the whole batch needs at
// the batched kernel's throughput by the margin, the ray would set the
// launch's length, and a cluster of SMs marches it instead.  A row step
// takes the tile's own time alone, or longer when the rays in flight together
// - the batch's, up to what the device's tile slots hold - would exceed the
// batched throughput at that pace.
std::vector<char> cost_rule(const cr_batch* b, const MarchCosts& c) {
    // a ray leaves the batched kernel only when it would clearly outlast the
    // batch: in a homogeneous batch every ray's march is close to the
    // balanced time, and the batched kernel is the efficient one there
    constexpr double kMargin = 1.25;
    std::vector<char> col((size_t)b->n_rays, 0);
    double work = 0.0, per_tile = 0.0;
    for (int i = 0; i < b->n_rays; ++i) {
        work += (double)b->rays[i].nz * b->rays[i].nr;
        per_tile += (double)(kTile / ((b->rays[i].np + crk::kT - 1) / crk::kT));
    }
    per_tile /= std::max(1, b->n_rays);
    const double tau = work / c.updates_per_s;
    const double in_flight = c.slots > 0.0 ? std::min((double)b->n_rays, c.slots * per_tile) : (double)b->n_rays;
    const double row = std::max(c.row_step_s, in_flight / c.updates_per_s);
    for (int i = 0; i < b->n_rays; ++i) {
        const cr_ray& r = b->rays[i];
        // every operator change (bathymetry index, profile update) costs the
        // batched march about four more passes: back-substitution alone, two
        // factorisation passes, elimination alone
        const double steps = (double)(r.nr + 4) + 4.0 * operator_changes(b, r);
        col[(size_t)i] = (double)(r.nz + 2) * steps * row > kMargin * tau;
    }
    return col;
}

MarchCosts march_costs(int device, int precision);
thread_local bool g_in_tuner = false;  // set while the tuner's own batches are created

// Rays marched by the column-parallel kernel instead of the batched one: the
// cost rule with the tuner's measured costs, for rays that fit the shared
// memory of a cluster of at most 16 CTAs.  CUPYRAM_B200_COL: 0 never, 1 every
// ray that fits, unset / other: the cost rule.
std::vector<char> pick_column_rays(const cr_batch* b, const std::vector<int>& pd_n, int precision, int device,
                                   MarchCosts* used) {
    // the column kernel has no refinement: refined rays on it run complex128
    const bool chosen = precision == CR_CHOSEN_C64R || precision == CR_CHOSEN_C64;
    std::vector<char> col((size_t)b->n_rays, 0);
    const char* env = getenv("CUPYRAM_B200_COL");
    const int mode = (env && env[0] == '0') ? 0 : ((env && env[0] == '1') ? 1 : 2);
    if (mode == 0 || g_in_tuner) return col;
    std::vector<char> want((size_t)b->n_rays, 1);
    if (mode == 2) {
        *used = march_costs(device, precision);
        // the rule paces the tiles by all the batch's rays in flight: capping
        // them at the device's tile slots kept 150 more wedge rays batched
        // and measured slower (11.7 s against 9.4 s)
        MarchCosts c = *used;
        c.slots = 0.0;
        want = cost_rule(b, c);
    }
    std::map<std::tuple<int, int, int>, bool> runs;
    for (int i = 0; i < b->n_rays; ++i) {
        if (!want[(size_t)i]) continue;
        const cr_ray& r = b->rays[i];
        const int terms = col_terms(pd_n, i);
        const int cluster = crk::col_cluster_size(r.nz, terms, chosen);
        if (cluster == 0) continue;
        const auto key = std::make_tuple(cluster, terms, r.nz);
        auto it = runs.find(key);
        if (it == runs.end())
            it = runs.emplace(key, crk::col_max_active_clusters(cluster, terms, r.nz, chosen) > 0).first;
        if (it->second) col[(size_t)i] = 1;
    }
    return col;
}

}  // namespace

int cr_create(const cr_batch* b, cr_engine** out) {
    NvtxRange nv("cr_create");
    if (!out) {
        set_global_error("cr_create: out is NULL");
        return CR_EINVAL;
    }
    *out = nullptr;
    const std::string msg = validate(b);
    if (!msg.empty()) {
        set_global_error("cr_create: %s", msg.c_str());
        return CR_EINVAL;
    }
    const auto t_create = std::chrono::steady_clock::now();
    cr_engine* e = new cr_engine();
    cudaGetDevice(&e->device);  // a failure resurfaces at the first device call below
    e->n_rays = b->n_rays;
    e->n_envs = b->n_envs;
    e->precision = b->precision;
    e->compute_grids = b->compute_grids;
    e->line_len = b->line_len;
    e->grid_len = b->compute_grids ? b->grid_len : 0;
    e->pool_len = b->pool_len;
    const auto t_pade = std::chrono::steady_clock::now();
    int rc = compute_pade_sets(e, b);
    e->st.pade_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_pade).count();
    if (rc) {
        set_global_error("%s", e->err.c_str());
        delete e;
        return rc;
    }
    // The partial-fraction march needs the field's surface row to stay zero
    // (true unless a source sits in the first depth cell); CUPYRAM_B200_SUM=0
    // selects the product-form march.
    {
        const char* senv = getenv("CUPYRAM_B200_SUM");
        bool ok = !(senv && senv[0] == '0');
        for (int i = 0; ok && i < b->n_rays; ++i)
            if ((int)std::floor(b->rays[i].zs / b->rays[i].dz) < 1) ok = false;
        e->sum_mode = ok;
    }
    // The reduced forms exist for the partial-fraction march only.  A batch
    // with a source in the first depth cell marches in the product form, in
    // complex128, whatever form was asked for: a drop-in still runs it, more
    // accurately than asked (cr_stats.precision_used says so).
    e->st.precision_used = e->sum_mode ? b->precision : CR_PLAIN_C128;
    if (e->sum_mode) {
        // c_inf and residues c_k of every Pade set (FP64, host)
        e->pfc.assign((size_t)b->n_rays * kSets * CR_MAX_NP, make_double2(0.0, 0.0));
        e->pfcinf.assign((size_t)b->n_rays * kSets, make_double2(0.0, 0.0));
        for (int i = 0; i < b->n_rays; ++i)
            for (int st = 0; st < kSets; ++st) partial_fractions(e, i, st);
    }
    // tiles: rays sorted by work, longest first, 32 per tile
    std::vector<int> order(b->n_rays);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const double wx = (double)(b->rays[x].nz + 2) * (b->rays[x].nr + 3);
        const double wy = (double)(b->rays[y].nz + 2) * (b->rays[y].nr + 3);
        return wx > wy;
    });
    if (e->sum_mode) {
        MarchCosts costs;
        const std::vector<char> is_col = pick_column_rays(b, e->pd_n, b->precision, e->device, &costs);
        e->st.tuner_row_step_s = costs.row_step_s;
        e->st.tuner_updates_per_s = costs.updates_per_s;
        e->st.tuner_slots = costs.slots;
        // batched rays grouped by Pade order, then work; a tile holds
        // floor(32/G) rays of G lanes each, G = the largest np in the tile
        std::vector<int> bord;
        for (int rid : order)
            if (!is_col[(size_t)rid]) bord.push_back(rid);
        // A tile marches in lockstep for its deepest ray's rows and its
        // longest ray's steps, so its rays should agree in both: within a
        // lane count G, rays are sorted by steps, and runs of 16 tiles'
        // worth of rays by depth.
        auto lanes_of = [&](int rid) { return (b->rays[rid].np + crk::kT - 1) / crk::kT; };
        std::stable_sort(bord.begin(), bord.end(), [&](int x, int y) {
            const int gx = lanes_of(x), gy = lanes_of(y);
            if (gx != gy) return gx > gy;
            return b->rays[x].nr > b->rays[y].nr;
        });
        for (size_t q = 0; q < bord.size();) {
            const int G = lanes_of(bord[q]);
            size_t gend = q;
            while (gend < bord.size() && lanes_of(bord[gend]) == G) ++gend;
            const size_t bucket = (size_t)16 * (kTile / G);
            for (size_t k = q; k < gend; k += bucket)
                std::stable_sort(bord.begin() + k, bord.begin() + std::min(gend, k + bucket),
                                 [&](int x, int y) { return b->rays[x].nz > b->rays[y].nz; });
            q = gend;
        }
        e->rays.resize(b->n_rays);
        long long off = 0;
        size_t pos = 0;
        std::vector<double> tile_work;  // lockstep row-steps of each tile
        while (pos < bord.size()) {
            // lanes per ray: each lane carries kT terms of the tile's largest np
            const int G = (b->rays[bord[pos]].np + crk::kT - 1) / crk::kT;
            const int R = kTile / G;
            const size_t end = std::min(bord.size(), pos + (size_t)R);
            int rows = 0;
            for (size_t q = pos; q < end; ++q) rows = std::max(rows, b->rays[bord[q]].nz + 2);
            const int t = (int)e->tile_G.size();
            int nr_tile = 0;
            for (size_t q = pos; q < end; ++q) nr_tile = std::max(nr_tile, b->rays[bord[q]].nr);
            tile_work.push_back((double)rows * (double)(nr_tile + 4));
            e->tile_G.push_back(G);
            e->tile_off.push_back(off);
            e->tile_loff.push_back(e->lane_elems);
            e->lane_elems += (long long)crk::kT * rows * kTile;
            e->tile_ray.resize((size_t)(t + 1) * kTile, -1);
            for (size_t q = pos; q < end; ++q) {
                const int slot = (int)(q - pos);
                const int rid = bord[q];
                for (int k = 0; k < G; ++k) e->tile_ray[(size_t)t * kTile + slot * G + k] = rid;
                RayDev& d = e->rays[rid];
                d = ray_dev(b->rays[rid], b->compute_grids);
                d.col = off + slot;
                d.crows = rows;
                e->point_updates += (double)b->rays[rid].nz * (double)b->rays[rid].nr;
            }
            off += (long long)rows * kTile;
            pos = end;
        }
        e->n_tiles = (int)e->tile_G.size();
        // queue order: the longest lockstep marches first (ties: layout order)
        e->queue.resize((size_t)e->n_tiles);
        std::iota(e->queue.begin(), e->queue.end(), 0);
        std::stable_sort(e->queue.begin(), e->queue.end(),
                         [&](int x, int y) { return tile_work[(size_t)x] > tile_work[(size_t)y]; });
        {
            const char* qenv = getenv("CUPYRAM_B200_QUEUE");
            e->queue_mode = !(qenv && qenv[0] == '0');
        }
        e->term_capacity.assign((size_t)b->n_rays, 0);
        for (int t = 0; t < e->n_tiles; ++t)
            for (int l = 0; l < kTile; ++l) {
                const int rid = e->tile_ray[(size_t)t * kTile + l];
                if (rid >= 0) e->term_capacity[(size_t)rid] = e->tile_G[t] * crk::kT;
            }
        // column rays: grouped by Pade term count (the cluster size), deepest
        // first; their ray columns are packed 32 to a tile after the batched ones
        std::vector<int> cord;
        for (int rid : order)
            if (is_col[(size_t)rid]) cord.push_back(rid);
        auto terms_of = [&](int rid) { return col_terms(e->pd_n, rid); };
        const bool chosen = b->precision == CR_CHOSEN_C64R || b->precision == CR_CHOSEN_C64;
        const std::vector<int> csize = column_clusters(b, e->pd_n, is_col, chosen);
        std::stable_sort(cord.begin(), cord.end(), [&](int x, int y) {
            const int tx = terms_of(x), ty = terms_of(y);
            if (tx != ty) return tx > ty;
            if (csize[(size_t)x] != csize[(size_t)y]) return csize[(size_t)x] > csize[(size_t)y];
            return b->rays[x].nz > b->rays[y].nz;
        });
        for (size_t q = 0; q < cord.size(); q += kTile) {
            const size_t end = std::min(cord.size(), q + (size_t)kTile);
            int rows = 0;
            for (size_t k = q; k < end; ++k) rows = std::max(rows, b->rays[cord[k]].nz + 2);
            for (size_t k = q; k < end; ++k) {
                const int rid = cord[k];
                RayDev& d = e->rays[rid];
                d = ray_dev(b->rays[rid], b->compute_grids);
                d.col = off + (long long)(k - q);
                d.crows = rows;
                e->point_updates += (double)b->rays[rid].nz * (double)b->rays[rid].nr;
            }
            off += (long long)rows * kTile;
        }
        // one launch per run of equal term count and cluster size (rays are
        // sorted by depth within a term count)
        for (size_t q = 0; q < cord.size();) {
            size_t end = q;
            const int terms = terms_of(cord[q]);
            const int nz_max = b->rays[cord[q]].nz;
            const int cluster = csize[(size_t)cord[q]];
            while (end < cord.size() && terms_of(cord[end]) == terms && csize[(size_t)cord[end]] == cluster) ++end;
            e->col_groups.push_back({cluster, terms, nz_max, (int)q, (int)(end - q), nullptr, nullptr});
            q = end;
        }
        for (const auto& g : e->col_groups)
            for (int k = g.begin; k < g.begin + g.count; ++k) e->term_capacity[(size_t)cord[k]] = g.terms;
        e->col_ray = cord;
        e->col_elems = off;
        e->fac_elems = 0;
    } else {
    e->n_tiles = (b->n_rays + kTile - 1) / kTile;
    e->tile_ray.assign((size_t)e->n_tiles * kTile, -1);
    e->rays.resize(b->n_rays);
    // The factorised march stores 5 complex factors per (term, row, ray);
    // CUPYRAM_B200_FACTOR=0 selects the on-the-fly march instead.
    const char* fenv = getenv("CUPYRAM_B200_FACTOR");
    const bool factored = !(fenv && fenv[0] == '0');
    long long col = 0, fcol = 0;
    for (int t = 0; t < e->n_tiles; ++t) {
        int rows = 0, npmax = 0;
        for (int l = 0; l < kTile; ++l) {
            const int k = t * kTile + l;
            if (k < b->n_rays) {
                rows = std::max(rows, b->rays[order[k]].nz + 2);
                npmax = std::max(npmax, b->rays[order[k]].np);
            }
        }
        for (int l = 0; l < kTile; ++l) {
            const int k = t * kTile + l;
            if (k >= b->n_rays) continue;
            const int rid = order[k];
            e->tile_ray[(size_t)t * kTile + l] = rid;
            const cr_ray& r = b->rays[rid];
            RayDev& d = e->rays[rid];
            d.k0 = 2.0 * M_PI * r.freq / r.c0;
            d.omega = 2.0 * M_PI * r.freq;
            d.c0 = r.c0;
            d.dz = r.dz;
            d.dr = r.dr;
            d.zmax = r.zmax;
            d.lyrw_lambda = r.lyrw_lambda;
            d.attnf = r.attnf;
            d.rs = r.rs;
            d.zs = r.zs;
            d.zr = r.zr;
            d.nz = r.nz;
            d.nr = r.nr;
            d.np = r.np;
            d.ndr = r.ndr;
            d.ndz = r.ndz;
            d.nvr = r.nvr;
            d.nvz = r.nvz;
            d.env = r.env;
            d.line_off = r.line_off;
            d.grid_off = b->compute_grids ? r.grid_off : -1;
            d.col = col + l;
            d.ccol = factored ? fcol + l : -1;
            d.crows = rows;
            d.pad_ = 0;
            e->point_updates += (double)r.nz * (double)r.nr;
        }
        col += (long long)rows * kTile;
        if (factored) fcol += (long long)npmax * rows * kTile;
    }
    e->col_elems = col;
    e->fac_elems = fcol;
    }
    e->envs.resize(b->n_envs);
    for (int k = 0; k < b->n_envs; ++k) {
        const cr_env& v = b->envs[k];
        e->envs[k] = EnvDev{v.n_zss, v.n_rss, v.n_zsb, v.n_rsb, v.n_bt, 0, v.off};
    }
    e->pool.assign(b->pool, b->pool + b->pool_len);

    cudaError_t ce = cudaGetDevice(&e->device);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    for (auto& ev : e->ev)
        if (ce == cudaSuccess) ce = cudaEventCreate(&ev);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_rays, e->rays.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_envs, e->envs.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_pool, e->pool.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_tile_ray, e->tile_ray.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_pd1, e->pd1.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_pd2, e->pd2.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_pd_n, e->pd_n.size());
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_f1, (size_t)e->col_elems);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_f2, (size_t)e->col_elems);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_f3, (size_t)e->col_elems);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_ksq, (size_t)e->col_elems);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_u, (size_t)e->col_elems);
    if (ce == cudaSuccess && !e->sum_mode) ce = dev_alloc(e, &e->d_W, (size_t)e->col_elems);
    if (ce == cudaSuccess && !e->sum_mode) ce = dev_alloc(e, &e->d_G, (size_t)e->col_elems);
    if (e->sum_mode) {
        double2** lanecols[] = {&e->d_QD, &e->d_WD, &e->d_QU, &e->d_WU, &e->d_G};
        for (double2** pp : lanecols)
            if (ce == cudaSuccess) ce = dev_alloc(e, pp, (size_t)e->lane_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_ED, (size_t)e->col_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_EU, (size_t)e->col_elems);
        if (ce == cudaSuccess && b->precision == CR_C64_REFINED) ce = dev_alloc(e, &e->d_E2, (size_t)e->col_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_tile_loff, e->tile_loff.size());
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_tile_G, e->tile_G.size());
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_queue, e->queue.size());
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_ticket, (size_t)1);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_tile_off, e->tile_off.size());
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_pfc, e->pfc.size());
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_pfcinf, e->pfcinf.size());
        if (ce == cudaSuccess && !e->col_ray.empty()) ce = dev_alloc(e, &e->d_col_ray, e->col_ray.size());
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
        {
            // one stream per run of equal lanes per ray (the first is the engine's)
            int runs = 0;
            for (int t = 0; t < e->n_tiles; ++t) runs += (t == 0 || e->tile_G[t] != e->tile_G[t - 1]);
            e->sum_streams.assign((size_t)std::max(runs, 1), nullptr);
            e->sum_done.assign(e->sum_streams.size(), nullptr);
            e->sum_streams[0] = e->stream;
            for (size_t i = 1; i < e->sum_streams.size(); ++i)
                if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->sum_streams[i], cudaStreamNonBlocking);
            for (auto& ev : e->sum_done)
                if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        }
        for (auto& g : e->col_groups) {
            if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
            if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
        }
    }
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_tll, (size_t)e->line_len);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_cpl, (size_t)e->line_len);
    if (ce == cudaSuccess && e->compute_grids) ce = dev_alloc(e, &e->d_tlg, (size_t)e->grid_len);
    if (ce == cudaSuccess && e->compute_grids) ce = dev_alloc(e, &e->d_cpg, (size_t)e->grid_len);
    if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_flags, (size_t)e->n_rays);
    if (e->fac_elems > 0) {
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_S1, (size_t)e->fac_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_S2, (size_t)e->fac_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_S3, (size_t)e->fac_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_AL, (size_t)e->fac_elems);
        if (ce == cudaSuccess) ce = dev_alloc(e, &e->d_WF, (size_t)e->fac_elems);
    }
    if (ce == cudaSuccess)
        ce = cudaFuncSetAttribute(march_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRingBytes);
    // the batched march's kernels are loaded now, while the device is idle,
    // not at their first launch beside running column clusters
    if (ce == cudaSuccess && e->sum_mode && e->n_tiles > 0)
        ce = crk::prepare_march_sum(e->tile_G.data(), e->n_tiles, e->precision);
    if (ce != cudaSuccess) {
        set_global_error("cr_create: %s", cudaGetErrorString(ce));
        const int code = ce == cudaErrorMemoryAllocation ? CR_ENOMEM : CR_ECUDA;
        free_all(e);
        delete e;
        return code;
    }
    e->st.point_updates = e->point_updates;
    e->st.tile_rays = kTile;
    e->st.n_tiles = e->n_tiles;
    e->st.device_bytes = e->device_bytes;
    e->st.column_rays = (int)e->col_ray.size();
    e->st.create_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_create).count();
    *out = e;
    return CR_OK;
}

int cr_set_pade(cr_engine* e, int ray, int which, int n, const double* pd1, const double* pd2) {
    if (!e) return CR_EINVAL;
    if (ray < 0 || ray >= e->n_rays || which < 0 || which >= kSets || n < 1 || n > CR_MAX_NP || !pd1 || !pd2)
        return e->fail(CR_EINVAL, "cr_set_pade: invalid arguments");
    if (e->sum_mode && n > e->term_capacity[(size_t)ray])
        return e->fail(CR_EINVAL, "cr_set_pade: %d terms exceed the %d this ray's march was laid out for "
                                  "(create the engine with np >= %d)", n, e->term_capacity[(size_t)ray], n);
    double2* p1 = e->pd1.data() + ((size_t)ray * kSets + which) * CR_MAX_NP;
    double2* p2 = e->pd2.data() + ((size_t)ray * kSets + which) * CR_MAX_NP;
    for (int j = 0; j < CR_MAX_NP; ++j) {
        p1[j] = j < n ? make_double2(pd1[2 * j], pd1[2 * j + 1]) : make_double2(0.0, 0.0);
        p2[j] = j < n ? make_double2(pd2[2 * j], pd2[2 * j + 1]) : make_double2(0.0, 0.0);
    }
    e->pd_n[(size_t)ray * kSets + which] = n;
    if (e->sum_mode) partial_fractions(e, ray, which);
    e->uploaded = false;
    return CR_OK;
}

int cr_upload(cr_engine* e) {
    NvtxRange nv("cr_upload");
    if (!e) return CR_EINVAL;
    cudaError_t ce = cudaSetDevice(e->device);
    float ms = 0.f;
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev[0], e->stream);
    auto cp = [&](void* dst, const void* src, size_t bytes) {
        if (ce != cudaSuccess || !bytes) return;
        // large arrays (the environment pool) go through the pinned staging
        // ring; small tables are copied directly
        ce = bytes >= kStageMin ? staged_h2d(e->device, dst, src, bytes, e->stream)
                                : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, e->stream);
    };
    cp(e->d_rays, e->rays.data(), e->rays.size() * sizeof(RayDev));
    cp(e->d_envs, e->envs.data(), e->envs.size() * sizeof(EnvDev));
    cp(e->d_pool, e->pool.data(), e->pool.size() * sizeof(double));
    cp(e->d_tile_ray, e->tile_ray.data(), e->tile_ray.size() * sizeof(int));
    cp(e->d_pd1, e->pd1.data(), e->pd1.size() * sizeof(double2));
    cp(e->d_pd2, e->pd2.data(), e->pd2.size() * sizeof(double2));
    cp(e->d_pd_n, e->pd_n.data(), e->pd_n.size() * sizeof(int));
    if (e->sum_mode) {
        cp(e->d_tile_G, e->tile_G.data(), e->tile_G.size() * sizeof(int));
        cp(e->d_queue, e->queue.data(), e->queue.size() * sizeof(int));
        cp(e->d_tile_off, e->tile_off.data(), e->tile_off.size() * sizeof(long long));
        cp(e->d_tile_loff, e->tile_loff.data(), e->tile_loff.size() * sizeof(long long));
        cp(e->d_pfc, e->pfc.data(), e->pfc.size() * sizeof(double2));
        cp(e->d_pfcinf, e->pfcinf.data(), e->pfcinf.size() * sizeof(double2));
        cp(e->d_col_ray, e->col_ray.data(), e->col_ray.size() * sizeof(int));
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev[1], e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cr_upload");
    e->st.h2d_ms = ms;
    e->st.h2d_bytes = (long long)(e->rays.size() * sizeof(RayDev) + e->envs.size() * sizeof(EnvDev) +
                                  e->pool.size() * sizeof(double) + e->tile_ray.size() * sizeof(int) +
                                  2 * e->pd1.size() * sizeof(double2) + e->pd_n.size() * sizeof(int));
    e->uploaded = true;
    return CR_OK;
}

int cr_march(cr_engine* e) {
    NvtxRange nv("cr_march");
    if (!e) return CR_EINVAL;
    if (!e->uploaded) return e->fail(CR_ESTATE, "cr_march: call cr_upload first");
    cudaError_t ce = cudaSetDevice(e->device);
    MarchArgs a;
    a.rays = e->d_rays;
    a.tile_ray = e->d_tile_ray;
    a.envs = e->d_envs;
    a.pool = e->d_pool;
    a.pd1 = e->d_pd1;
    a.pd2 = e->d_pd2;
    a.pd_n = e->d_pd_n;
    a.f1 = e->d_f1;
    a.f2 = e->d_f2;
    a.f3 = e->d_f3;
    a.ksq = e->d_ksq;
    a.u = e->d_u;
    a.W = e->d_W;
    a.G = e->d_G;
    a.tll = e->d_tll;
    a.cpl = e->d_cpl;
    a.tlg = e->d_tlg;
    a.cpg = e->d_cpg;
    a.flags = e->d_flags;
    a.compute_grids = e->compute_grids;
    a.S1 = e->d_S1;
    a.S2 = e->d_S2;
    a.S3 = e->d_S3;
    a.AL = e->d_AL;
    a.WF = e->d_WF;
    float ms = 0.f;
    if (ce == cudaSuccess && e->sum_mode) {
        crk::SumArgs sa;
        sa.rays = e->d_rays;
        sa.tile_ray = e->d_tile_ray;
        sa.tile_G = e->d_tile_G;
        sa.tile_off = e->d_tile_off;
        sa.tile_loff = e->d_tile_loff;
        sa.envs = e->d_envs;
        sa.pool = e->d_pool;
        sa.pd1 = e->d_pd1;
        sa.pd2 = e->d_pd2;
        sa.pd_n = e->d_pd_n;
        sa.pfc = e->d_pfc;
        sa.pfcinf = e->d_pfcinf;
        sa.f1 = e->d_f1;
        sa.f2 = e->d_f2;
        sa.f3 = e->d_f3;
        sa.ksq = e->d_ksq;
        sa.u = e->d_u;
        sa.G = e->d_G;
        sa.QD = e->d_QD;
        sa.WD = e->d_WD;
        sa.QU = e->d_QU;
        sa.WU = e->d_WU;
        sa.ED = e->d_ED;
        sa.EU = e->d_EU;
        sa.E2 = e->d_E2;
        sa.tll = e->d_tll;
        sa.cpl = e->d_cpl;
        sa.tlg = e->d_tlg;
        sa.cpg = e->d_cpg;
        sa.flags = e->d_flags;
        sa.compute_grids = e->compute_grids;
        if (e->n_tiles > 0 && !crk::encode_sum_maps(sa, e->precision, e->col_elems / kTile, e->lane_elems / kTile))
            return e->fail(CR_ECUDA, "cr_march: the driver's tensor-map encoder is unavailable or refused a map");
        crk::ColArgs ca;
        ca.rays = e->d_rays;
        ca.col_ray = e->d_col_ray;
        ca.envs = e->d_envs;
        ca.pool = e->d_pool;
        ca.pd2 = e->d_pd2;
        ca.pd_n = e->d_pd_n;
        ca.pfc = e->d_pfc;
        ca.pfcinf = e->d_pfcinf;
        ca.f1 = e->d_f1;
        ca.f2 = e->d_f2;
        ca.f3 = e->d_f3;
        ca.ksq = e->d_ksq;
        ca.tll = e->d_tll;
        ca.cpl = e->d_cpl;
        ca.tlg = e->d_tlg;
        ca.cpg = e->d_cpg;
        ca.flags = e->d_flags;
        ca.compute_grids = e->compute_grids;
        const int chosen = e->precision == CR_CHOSEN_C64R || e->precision == CR_CHOSEN_C64;
        ce = cudaEventRecord(e->ev[0], e->stream);
        int nl = 0;
        // column groups first, each on its own stream (they hold the longest
        // marches), then the batched tiles on the engine's stream
        if (ce == cudaSuccess) ce = cudaEventRecord(e->ev_fork, e->stream);
        for (size_t i = 1; i < e->sum_streams.size(); ++i)
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->sum_streams[i], e->ev_fork, 0);
        for (auto& g : e->col_groups) {
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(g.stream, e->ev_fork, 0);
            crk::ColArgs ga = ca;
            ga.col_ray = e->d_col_ray + g.begin;
            if (ce == cudaSuccess) ce = crk::launch_march_col(ga, g.count, g.cluster, g.terms, g.nz_max, chosen, g.stream);
            if (ce == cudaSuccess) ce = cudaEventRecord(g.done, g.stream);
            ++nl;
        }
        sa.tile_begin = 0;
        sa.ticket = e->d_ticket;
        sa.queue = e->d_queue;
        sa.n_queue = e->n_tiles;
        int nb = 0;
        // Beside column clusters the tiles go in one launch per lane count:
        // the queue's persistent CTAs would hold SMs the clusters wait for,
        // and with one CTA per tile the queue measured slower than these
        // launches on the uneven wedge batch (11.7 s against 9.4 s).
        const bool queue = e->queue_mode && e->col_groups.empty();
        if (queue) {
            // one persistent launch over every batched tile, fed by the queue
            int ctas = 0;
            if (ce == cudaSuccess && e->n_tiles > 0) ce = cudaMemsetAsync(e->d_ticket, 0, sizeof(int), e->stream);
            if (ce == cudaSuccess && e->n_tiles > 0) {
                sa.max_ctas = 0;
                sa.min_p = *std::min_element(e->tile_G.begin(), e->tile_G.end());
                ce = crk::launch_march_sum_queue(sa, e->n_tiles, e->precision, e->stream, &ctas);
                nb = 1;
            }
            e->st.queue_ctas = ctas;
        } else if (ce == cudaSuccess) {
            e->st.queue_ctas = 0;
            ce = crk::launch_march_sum(sa, e->tile_G.data(), e->n_tiles, e->precision, e->sum_streams.data(),
                                       (int)e->sum_streams.size(), &nb);
        }
        for (size_t i = 1; i < e->sum_streams.size(); ++i) {
            if (ce == cudaSuccess) ce = cudaEventRecord(e->sum_done[i], e->sum_streams[i]);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, e->sum_done[i], 0);
        }
        for (auto& g : e->col_groups)
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, g.done, 0);
        e->st.kernel_launches = nl + nb;
        e->st.column_launches = nl;
    } else if (ce == cudaSuccess) {
        ce = cudaEventRecord(e->ev[0], e->stream);
        if (ce == cudaSuccess) {
            march_kernel<<<e->n_tiles, kTile, kRingBytes, e->stream>>>(a);
            ce = cudaGetLastError();
        }
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev[1], e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cr_march");
    e->st.march_ms = ms;
    if (!e->sum_mode) e->st.kernel_launches = 1;
    std::vector<int> fl(e->n_rays);
    ce = cudaMemcpy(fl.data(), e->d_flags, fl.size() * sizeof(int), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cr_march (flags)");
    int failed = 0, timed_out = 0;
    for (int v : fl) {
        failed += (v != 0);
        timed_out += (v & 2) != 0;
    }
    e->st.rays_failed = failed;
    e->marched = true;
    if (timed_out)
        return e->fail(CR_ETIMEOUT, "%d ray(s): a wait for the march's bulk copies gave up", timed_out);
    if (failed) return e->fail(CR_ENAN, "%d ray(s) produced a non-finite field", failed);
    return CR_OK;
}

int cr_download(cr_engine* e, const cr_outputs* out) {
    NvtxRange nv("cr_download");
    if (!e) return CR_EINVAL;
    if (!out || !out->tll || !out->cpl) return e->fail(CR_EINVAL, "cr_download: tll and cpl are required");
    if (!e->marched) return e->fail(CR_ESTATE, "cr_download: nothing marched yet");
    cudaError_t ce = cudaSetDevice(e->device);
    float ms = 0.f;
    long long bytes = 0;
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev[2], e->stream);
    auto cp = [&](void* dst, const void* src, size_t n) {
        if (ce == cudaSuccess && n && dst) {
            ce = cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, e->stream);
            bytes += (long long)n;
        }
    };
    cp(out->tll, e->d_tll, (size_t)e->line_len * sizeof(double));
    cp(out->cpl, e->d_cpl, (size_t)e->line_len * sizeof(double2));
    if (e->compute_grids) {
        cp(out->tlg, e->d_tlg, (size_t)e->grid_len * sizeof(double));
        cp(out->cpg, e->d_cpg, (size_t)e->grid_len * sizeof(double2));
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev[3], e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e->ev[2], e->ev[3]);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cr_download");
    e->st.d2h_ms = ms;
    e->st.d2h_bytes = bytes;
    return CR_OK;
}

namespace {

// TL of cells of sz x sr grid outputs (rows j sz .. j sz + sz - 1, ranges
// c sr .. c sr + sr - 1 of the ray's TL grid): -10 log10 of the mean of
// |cp|^2 / r over the cell, r = (t + 1) ndr dr.  NaN where the ray's grid is
// smaller than the cells asked for.
__global__ void cell_tl_kernel(const RayDev* __restrict__ rays, int n_rays, const double2* __restrict__ cpg, int sz,
                               int sr, int ncz, int ncr, float* __restrict__ out) {
    const long long total = (long long)n_rays * ncz * ncr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int ray = (int)(i / ((long long)ncz * ncr));
        const int rem = (int)(i % ((long long)ncz * ncr));
        const int j = rem / ncr, c = rem % ncr;
        const RayDev& ry = rays[ray];
        if (ry.grid_off < 0 || (j + 1) * sz > ry.nvz || (c + 1) * sr > ry.nvr) {
            out[i] = __int_as_float(0x7fc00000);
            continue;
        }
        double acc = 0.0;
        for (int a = 0; a < sz; ++a) {
            const double2* row = cpg + ry.grid_off + (long long)(j * sz + a) * ry.nvr;
            for (int b = 0; b < sr; ++b) {
                const int t = c * sr + b;
                const double2 p = row[t];
                acc += (p.x * p.x + p.y * p.y) / ((double)((t + 1) * ry.ndr) * ry.dr);
            }
        }
        out[i] = (float)(-10.0 * log10(acc / (double)(sz * sr)));
    }
}

}  // namespace

int cr_cell_tl(cr_engine* e, int sz, int sr, int ncz, int ncr, float* tl_cells) {
    NvtxRange nv("cr_cell_tl");
    if (!e) return CR_EINVAL;
    if (sz < 1 || sr < 1 || ncz < 1 || ncr < 1 || !tl_cells) return e->fail(CR_EINVAL, "cr_cell_tl: invalid arguments");
    if (!e->compute_grids) return e->fail(CR_EINVAL, "cr_cell_tl: the batch computes no TL grid");
    if (!e->marched) return e->fail(CR_ESTATE, "cr_cell_tl: nothing marched yet");
    const size_t n = (size_t)e->n_rays * ncz * ncr;
    float* d_out = nullptr;
    cudaError_t ce = cudaSetDevice(e->device);
    if (ce == cudaSuccess) ce = cudaMallocAsync((void**)&d_out, n * sizeof(float), e->stream);
    if (ce == cudaSuccess) {
        const long long blocks = std::min<long long>(((long long)n + 255) / 256, 65535);
        cell_tl_kernel<<<(unsigned)blocks, 256, 0, e->stream>>>(e->d_rays, e->n_rays, e->d_cpg, sz, sr, ncz, ncr, d_out);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(tl_cells, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream);
    if (d_out) cudaFreeAsync(d_out, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cr_cell_tl");
    return CR_OK;
}

int cr_run(cr_engine* e, const cr_outputs* out) {
    int rc = cr_upload(e);
    if (rc) return rc;
    rc = cr_march(e);
    if (rc) return rc;
    return cr_download(e, out);
}

int cr_ray_flags(cr_engine* e, int32_t* flags, int n) {
    if (!e || !flags || n < e->n_rays) return CR_EINVAL;
    cudaError_t ce = cudaMemcpy(flags, e->d_flags, (size_t)e->n_rays * sizeof(int), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cr_ray_flags");
    return CR_OK;
}

int cr_get_stats(const cr_engine* e, cr_stats* st) {
    if (!e || !st) return CR_EINVAL;
    *st = e->st;
    return CR_OK;
}

int cr_last_error(const cr_engine* e, char* buf, size_t len) {
    if (!e || !buf || len == 0) return CR_EINVAL;
    snprintf(buf, len, "%s", e->err.c_str());
    return CR_OK;
}

void cr_destroy(cr_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_all(e);
    delete e;
}

int cr_plan_columns(const cr_batch* b, double row_step_s, double updates_per_s, double slots, int32_t* is_column) {
    const std::string msg = validate(b);
    if (!msg.empty() || !is_column || !(row_step_s > 0.0) || !(updates_per_s > 0.0)) {
        set_global_error("cr_plan_columns: %s", msg.empty() ? "invalid arguments" : msg.c_str());
        return CR_EINVAL;
    }
    MarchCosts c;
    c.row_step_s = row_step_s;
    c.updates_per_s = updates_per_s;
    c.slots = slots;
    const std::vector<char> col = cost_rule(b, c);
    for (int i = 0; i < b->n_rays; ++i) is_column[i] = col[(size_t)i];
    return CR_OK;
}

}  // extern "C"

namespace {

// The engine's own tuner: the costs of the column policy, measured once per
// device and precision form by marching synthetic batches through the engine
// itself (every ray on the batched kernel):
//   * one tile alone (10 rays of np 6, nz 2000, 30 steps): the time of one
//     row of one step of a lockstep tile when nothing else runs;
//   * two rounds of tiles for every resident slot of the device (nz 200,
//     40 steps): the batched throughput in grid-point updates/s, and the slots
//     (the CTAs of the persistent launch).
// About 0.1 s on first use; CUPYRAM_B200_COSTS="row_step_s,updates_per_s,slots"
// sets them instead (reproducible schedules).
std::mutex g_costs_mu;
std::map<std::pair<int, int>, MarchCosts> g_costs;

// Synthetic batch: isovelocity 100 m water over a 1700 m/s bottom, 100 Hz.
struct SynthBatch {
    std::vector<cr_ray> rays;
    cr_env env{};
    std::vector<double> pool;
    cr_batch b{};
};

void synth_batch(SynthBatch& s, int n_rays, int nz, int nr, int precision) {
    const double D = 100.0, c = 1500.0, rmax = 1.0e5;
    const double dz = (D + 100.0) / (double)(nz + 1);
    // z_ss, rp_ss, cw[1][2], z_sb, rp_sb, cb, rhob, attn [1][2], rb, zb
    s.pool = {0.0, D, 0.0, c, c, D, D + 100.0, 0.0, 1700.0, 1700.0, 1.5, 1.5, 0.5, 0.5, 0.0, rmax, D, D};
    s.env = cr_env{2, 1, 2, 1, 2, 0, 0};
    s.rays.assign((size_t)n_rays, cr_ray{});
    for (int i = 0; i < n_rays; ++i) {
        cr_ray& r = s.rays[(size_t)i];
        r.freq = 100.0;
        r.c0 = c;
        r.zs = r.zr = 20.0;
        r.dz = dz;
        r.dr = 5.0;
        r.zmax = (double)(nz + 1) * dz;
        r.lyrw_lambda = 0.0;
        r.attnf = 10.0;
        r.rs = INFINITY;
        r.nz = nz;
        r.nr = nr;
        r.np = 6;
        r.ns = 1;
        r.ndr = 1;
        r.ndz = 1;
        r.nvr = 1;
        r.nvz = 0;
        r.env = 0;
        r.line_off = i;
        r.grid_off = -1;
    }
    s.b.n_rays = n_rays;
    s.b.n_envs = 1;
    s.b.rays = s.rays.data();
    s.b.envs = &s.env;
    s.b.pool = s.pool.data();
    s.b.pool_len = (int64_t)s.pool.size();
    s.b.precision = precision;
    s.b.compute_grids = 0;
    s.b.line_len = n_rays;
    s.b.grid_len = 0;
}

// Device time (ms) of a warm march of a synthetic batch, or < 0 on failure;
// *ctas: the CTAs of its persistent batched launch.
double synth_march_ms(int n_rays, int nz, int nr, int precision, int* ctas) {
    SynthBatch s;
    synth_batch(s, n_rays, nz, nr, precision);
    cr_engine* e = nullptr;
    if (cr_create(&s.b, &e) != CR_OK) return -1.0;
    std::vector<double> tll((size_t)n_rays), cpl(2 * (size_t)n_rays);
    cr_outputs o{tll.data(), cpl.data(), nullptr, nullptr};
    double ms = -1.0;
    if (cr_run(e, &o) == CR_OK && cr_march(e) == CR_OK) {
        ms = e->st.march_ms;
        *ctas = e->st.queue_ctas;
    }
    cr_destroy(e);
    return ms;
}

MarchCosts march_costs(int device, int precision) {
    MarchCosts c;
    if (const char* v = getenv("CUPYRAM_B200_COSTS")) {
        if (sscanf(v, "%lf,%lf,%lf", &c.row_step_s, &c.updates_per_s, &c.slots) >= 2 && c.row_step_s > 0 &&
            c.updates_per_s > 0)
            return c;
    }
    std::lock_guard<std::mutex> lock(g_costs_mu);
    const auto key = std::make_pair(device, precision);
    auto it = g_costs.find(key);
    if (it != g_costs.end()) return it->second;
    // if a measurement fails: one B200's figures for the plain form
    c.row_step_s = 0.3e-6;
    c.updates_per_s = 1.3e10;
    c.slots = 0.0;
    g_in_tuner = true;
    {
        int sms = 148, ctas = 0, ctas1 = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int nz1 = 2000, nr1 = 30;
        const double t1 = synth_march_ms(10, nz1, nr1, precision, &ctas1);
        const int nz = 200, nr = 40, rays = 10 * 2 * 7 * sms;
        const double t = synth_march_ms(rays, nz, nr, precision, &ctas);
        // a march without operator changes takes about nr + 12 row sweeps
        if (t1 > 0.0) c.row_step_s = t1 * 1e-3 / ((double)(nz1 + 2) * (double)(nr1 + 12));
        if (t > 0.0) c.updates_per_s = (double)rays * nz * nr / (t * 1e-3);
        if (ctas > 0) c.slots = ctas;
    }
    g_in_tuner = false;
    // the tuner's engines leave their memory in the pool: hand it back
    cudaMemPool_t pool = nullptr;
    if (engine_pool(device, &pool) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    g_costs[key] = c;
    return c;
}

}  // namespace

extern "C" {

int cr_release_cache(void) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    for (int d = 0; d < kPoolDevices; ++d) {
        if (!g_pools[d]) continue;
        const cudaError_t ce = cudaMemPoolTrimTo(g_pools[d], 0);
        if (ce != cudaSuccess) {
            set_global_error("cr_release_cache: %s", cudaGetErrorString(ce));
            return CR_ECUDA;
        }
    }
    return CR_OK;
}

}  // extern "C"

// ===========================================================================
// cr_march_static: the march without any allocation.
//
// For callers that cannot allocate device memory when they need a march (a
// real-time loop that forbids allocation after start-up, or a plug-in whose
// host application owns all device memory through its own pool).  Everything
// the march needs besides the caller's inputs and outputs lives in one
// file-scope device array of CR_STATIC_SCRATCH_BYTES; the per-ray tables and
// the Pade sets are built on the device from the raw cr_ray records, so the
// host side needs no heap either.
// ===========================================================================
namespace {

__device__ __align__(256) unsigned char g_static_scratch[CR_STATIC_SCRATCH_BYTES];

static_assert(sizeof(cr_env) == sizeof(EnvDev), "cr_env and EnvDev must share a layout");
static_assert(sizeof(cr_ray) == 136, "cr_ray layout changed");

// Device address of g_static_scratch per device, looked up on the first call
// on that device (host code cannot use the symbol's name as an address).  The
// address belongs to the device's current context: it is stored with that
// context's handle and looked up again when the context changes (after a
// cudaDeviceReset, for example), so a stale address is never used.
constexpr int kMaxDevices = 64;
struct StaticPtr {
    void* ctx = nullptr;
    void* ptr = nullptr;
};
StaticPtr g_static_ptr[kMaxDevices];
std::mutex g_static_mu;

// Handle of the calling thread's current CUDA context, through the driver
// entry point the runtime exposes (nullptr when it is unavailable; the
// address is then looked up on every call).
void* current_context() {
    using Fn = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)
    static Fn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (Fn)p;
    });
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

int static_scratch_ptr(int dev, void** out) {
    if (dev < 0 || dev >= kMaxDevices) return CR_EINVAL;
    std::lock_guard<std::mutex> lock(g_static_mu);
    void* ctx = current_context();
    StaticPtr& c = g_static_ptr[dev];
    if (!c.ptr || !ctx || c.ctx != ctx) {
        void* p = nullptr;
        const cudaError_t ce = cudaGetSymbolAddress(&p, g_static_scratch);
        if (ce != cudaSuccess || !p) {
            set_global_error("cr_march_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(ce));
            return CR_ECUDA;
        }
        c.ptr = p;
        c.ctx = ctx;
    }
    *out = c.ptr;
    return CR_OK;
}

struct StaticLayout {
    size_t rays_raw, envs, pool, rays, tile_ray, pd1, pd2, pd_n, flags, status, f1, f2, f3, ksq, u, W, G;
    size_t total;
    long long col_elems;
    int n_tiles, rows;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

void static_layout(const cr_batch* b, StaticLayout* L) {
    int rows = 0;
    for (int i = 0; i < b->n_rays; ++i) rows = std::max(rows, b->rays[i].nz + 2);
    L->rows = rows;
    L->n_tiles = (b->n_rays + kTile - 1) / kTile;
    L->col_elems = (long long)L->n_tiles * rows * kTile;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = align256(o + bytes);
        return at;
    };
    const size_t nr = (size_t)b->n_rays;
    L->rays_raw = take(nr * sizeof(cr_ray));
    L->envs = take((size_t)b->n_envs * sizeof(cr_env));
    L->pool = take((size_t)b->pool_len * sizeof(double));
    L->rays = take(nr * sizeof(RayDev));
    L->tile_ray = take((size_t)L->n_tiles * kTile * sizeof(int));
    L->pd1 = take(nr * kSets * CR_MAX_NP * sizeof(double2));
    L->pd2 = take(nr * kSets * CR_MAX_NP * sizeof(double2));
    L->pd_n = take(nr * kSets * sizeof(int));
    L->flags = take(nr * sizeof(int));
    L->status = take(sizeof(int));
    const size_t ce = (size_t)L->col_elems;
    L->f1 = take(ce * sizeof(float));
    L->f2 = take(ce * sizeof(float));
    L->f3 = take(ce * sizeof(float));
    L->ksq = take(ce * sizeof(float2));
    L->u = take(ce * sizeof(double2));
    L->W = take(ce * sizeof(double2));
    L->G = take(ce * sizeof(double2));
    L->total = o;
}

// One thread per tile slot: derive RayDev, the tile map and the Pade sets of
// one ray (device FP64 Pade, same code as the host path).  Bit 0 of *status:
// a Pade set failed.
__global__ void static_setup_kernel(const cr_ray* raw, int n_rays, int compute_grids, int rows, RayDev* rays,
                                    int* tile_ray, double2* pd1, double2* pd2, int* pd_n, int* flags, int* status,
                                    int n_slots) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_slots) return;
    if (b >= n_rays) {
        tile_ray[b] = -1;
        return;
    }
    tile_ray[b] = b;
    const cr_ray r = raw[b];
    RayDev d;
    d.k0 = 2.0 * M_PI * r.freq / r.c0;
    d.omega = 2.0 * M_PI * r.freq;
    d.c0 = r.c0;
    d.dz = r.dz;
    d.dr = r.dr;
    d.zmax = r.zmax;
    d.lyrw_lambda = r.lyrw_lambda;
    d.attnf = r.attnf;
    d.rs = r.rs;
    d.zs = r.zs;
    d.zr = r.zr;
    d.nz = r.nz;
    d.nr = r.nr;
    d.np = r.np;
    d.ndr = r.ndr;
    d.ndz = r.ndz;
    d.nvr = r.nvr;
    d.nvz = r.nvz;
    d.env = r.env;
    d.line_off = r.line_off;
    d.grid_off = compute_grids ? r.grid_off : -1;
    d.col = (long long)(b / kTile) * rows * kTile + (b % kTile);
    d.ccol = -1;  // the static path marches on the fly (no factor arrays)
    d.crows = rows;
    d.pad_ = 0;
    rays[b] = d;
    flags[b] = 0;
    double2* p1 = pd1 + (size_t)b * kSets * CR_MAX_NP;
    double2* p2 = pd2 + (size_t)b * kSets * CR_MAX_NP;
    for (int k = 0; k < kSets * CR_MAX_NP; ++k) {
        p1[k] = make_double2(0.0, 0.0);
        p2[k] = make_double2(0.0, 0.0);
    }
    p2[0] = make_double2(-1.0, 0.0);
    pd_n[b * kSets + 0] = 1;
    cr::cd a[CR_MAX_NP], c[CR_MAX_NP];
    const int ips[3] = {2, 1, 1};
    const int nss[3] = {r.ns, r.ns, 0};
    for (int s = 1; s < kSets; ++s) {
        if (cr::pade_coefficients(r.freq, r.c0, r.np, nss[s - 1], r.dr, ips[s - 1], a, c) != cr::kPadeOk) {
            atomicOr(status, 1);
            pd_n[b * kSets + s] = 1;  // keeps the march in bounds; the call reports CR_EPADE
            continue;
        }
        for (int j = 0; j < r.np; ++j) {
            p1[s * CR_MAX_NP + j] = make_double2(a[j].re, a[j].im);
            p2[s * CR_MAX_NP + j] = make_double2(c[j].re, c[j].im);
        }
        pd_n[b * kSets + s] = r.np;
    }
}

// Bit 1 of *status: some ray produced a non-finite field.
__global__ void static_flags_kernel(const int* flags, int n, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flags[i]) atomicOr(status, 2);
}

}  // namespace

extern "C" int cr_march_static(const cr_batch* b, const cr_outputs* out, void* stream_v) {
    NvtxRange nv("cr_march_static");
    const std::string msg = [&]() -> std::string {
        if (!out || !out->tll || !out->cpl) return "dev_out with tll and cpl device pointers is required";
        return std::string();
    }();
    if (!msg.empty()) {
        set_global_error("cr_march_static: %s", msg.c_str());
        return CR_EINVAL;
    }
    const std::string bad = validate(b);
    if (!bad.empty()) {
        set_global_error("cr_march_static: %s", bad.c_str());
        return CR_EINVAL;
    }
    if (b->precision != CR_PLAIN_C128) {
        set_global_error("cr_march_static: only the plain complex128 form is supported");
        return CR_EINVAL;
    }
    if (b->compute_grids && (!out->tlg || !out->cpg)) {
        set_global_error("cr_march_static: compute_grids needs tlg and cpg device pointers");
        return CR_EINVAL;
    }
    StaticLayout L;
    static_layout(b, &L);
    if (L.total > (size_t)CR_STATIC_SCRATCH_BYTES) {
        set_global_error("cr_march_static: batch needs %zu bytes of scratch, the library holds %u "
                         "(CR_STATIC_SCRATCH_BYTES); use cr_create/cr_run or a smaller batch",
                         L.total, (unsigned)CR_STATIC_SCRATCH_BYTES);
        return CR_EINVAL;
    }
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) {
        set_global_error("cr_march_static: %s", cudaGetErrorString(ce));
        return CR_ECUDA;
    }
    void* base_v = nullptr;
    int rc = static_scratch_ptr(dev, &base_v);
    if (rc) return rc;
    unsigned char* base = (unsigned char*)base_v;
    cudaStream_t st = (cudaStream_t)stream_v;
    auto h2d = [&](size_t off, const void* src, size_t bytes) {
        if (ce == cudaSuccess && bytes) ce = cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st);
    };
    h2d(L.rays_raw, b->rays, (size_t)b->n_rays * sizeof(cr_ray));
    h2d(L.envs, b->envs, (size_t)b->n_envs * sizeof(cr_env));
    h2d(L.pool, b->pool, (size_t)b->pool_len * sizeof(double));
    const int n_slots = L.n_tiles * kTile;
    // The status word is cleared on the stream before any thread of the set-up
    // kernel can set a bit in it (no in-kernel clear: blocks run in no fixed order).
    if (ce == cudaSuccess) ce = cudaMemsetAsync(base + L.status, 0, sizeof(int), st);
    if (ce == cudaSuccess) {
        static_setup_kernel<<<(n_slots + 127) / 128, 128, 0, st>>>(
            (const cr_ray*)(base + L.rays_raw), b->n_rays, b->compute_grids, L.rows, (RayDev*)(base + L.rays),
            (int*)(base + L.tile_ray), (double2*)(base + L.pd1), (double2*)(base + L.pd2), (int*)(base + L.pd_n),
            (int*)(base + L.flags), (int*)(base + L.status), n_slots);
        ce = cudaGetLastError();
    }
    MarchArgs a;
    a.rays = (const RayDev*)(base + L.rays);
    a.tile_ray = (const int*)(base + L.tile_ray);
    a.envs = (const EnvDev*)(base + L.envs);
    a.pool = (const double*)(base + L.pool);
    a.pd1 = (const double2*)(base + L.pd1);
    a.pd2 = (const double2*)(base + L.pd2);
    a.pd_n = (const int*)(base + L.pd_n);
    a.f1 = (float*)(base + L.f1);
    a.f2 = (float*)(base + L.f2);
    a.f3 = (float*)(base + L.f3);
    a.ksq = (float2*)(base + L.ksq);
    a.u = (double2*)(base + L.u);
    a.W = (double2*)(base + L.W);
    a.G = (double2*)(base + L.G);
    a.tll = out->tll;
    a.cpl = (double2*)out->cpl;
    a.tlg = b->compute_grids ? out->tlg : nullptr;
    a.cpg = b->compute_grids ? (double2*)out->cpg : nullptr;
    a.flags = (int*)(base + L.flags);
    a.compute_grids = b->compute_grids;
    a.S1 = a.S2 = a.S3 = a.AL = a.WF = nullptr;
    if (ce == cudaSuccess)
        ce = cudaFuncSetAttribute(march_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRingBytes);
    if (ce == cudaSuccess) {
        march_kernel<<<L.n_tiles, kTile, kRingBytes, st>>>(a);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) {
        static_flags_kernel<<<32, 256, 0, st>>>((const int*)(base + L.flags), b->n_rays, (int*)(base + L.status));
        ce = cudaGetLastError();
    }
    int status = 0;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&status, base + L.status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
        set_global_error("cr_march_static: %s", cudaGetErrorString(ce));
        return ce == cudaErrorMemoryAllocation ? CR_ENOMEM : CR_ECUDA;
    }
    if (status & 1) {
        set_global_error("cr_march_static: Laguerre method not converging for a Pade set");
        return CR_EPADE;
    }
    if (status & 2) {
        set_global_error("cr_march_static: a ray produced a non-finite field");
        return CR_ENAN;
    }
    return CR_OK;
}
