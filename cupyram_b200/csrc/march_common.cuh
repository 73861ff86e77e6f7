// march_common.cuh - device-side types and helpers shared by the march kernels.
//
// Everything here lives in namespace crk and is header-only (inline device
// functions, plain structs) so that several translation units can use it.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "../../include/cupyram_b200.h"

namespace crk {

constexpr int kTile = 32;  // rays per tile = lanes per warp

// ---------------------------------------------------------------------------
// device-side descriptors
// ---------------------------------------------------------------------------
struct RayDev {
    double k0, omega, c0, dz, dr, zmax, lyrw_lambda, attnf, rs, zs, zr;
    int nz, nr, np, ndr, ndz, nvr, nvz, env;
    long long line_off, grid_off;
    long long col;   // element index of (row 0, this lane) in the column arrays
    long long ccol;  // element index of (term 0, row 0, this lane) in the factor arrays, -1: none
    int crows;       // rows per term in the factor arrays (the tile's row count)
    int pad_;
};

struct EnvDev {
    int n_zss, n_rss, n_zsb, n_rsb, n_bt, pad;
    long long off;
};

// Pade sets per ray: 0 = (1-X)^-2 starter factor, 1 = starter ip=2,
// 2 = march, 3 = march after the stability range rs.
constexpr int kSets = 4;

struct MarchArgs {
    const RayDev* rays;
    const int* tile_ray;  // [n_tiles * 32] -> ray index or -1
    const EnvDev* envs;
    const double* pool;
    const double2* pd1;  // [ray][set][CR_MAX_NP]
    const double2* pd2;
    const int* pd_n;     // [ray][set]
    float* f1;
    float* f2;
    float* f3;
    float2* ksq;
    double2* u;
    double2* W;
    double2* G;
    double* tll;
    double2* cpl;
    double* tlg;
    double2* cpg;
    int* flags;
    int compute_grids;
    // Factorised march operator, one record per (term, row): the elimination
    // g_m = S1 x_{m-1} + S2 x_m + S3 x_{m+1} + AL g_{m-/+1} and the
    // back-substitution factor WF.  NULL: factor on the fly every step.
    double2* S1;
    double2* S2;
    double2* S3;
    double2* AL;
    double2* WF;
};

// ---------------------------------------------------------------------------
// small complex helpers on double2
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 c2(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return c2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cfms(double2 acc, double2 a, double2 b) {  // acc - a*b
    return c2(acc.x - fma(a.x, b.x, -a.y * b.y), acc.y - fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 crcp(double2 b) {
    const double inv = 1.0 / fma(b.x, b.x, b.y * b.y);
    return c2(b.x * inv, -b.y * inv);
}
// a + p * d  with real a
__device__ __forceinline__ double2 caxpd(double a, double2 p, double2 d) {
    return c2(a + fma(p.x, d.x, -p.y * d.y), fma(p.x, d.y, p.y * d.x));
}

// ---------------------------------------------------------------------------
// profile interpolation (profl)
// ---------------------------------------------------------------------------
struct EnvPtrs {
    const double *z_ss, *rp_ss, *cw, *z_sb, *rp_sb, *cb, *rhob, *attn, *rb, *zb;
    int n_zss, n_rss, n_zsb, n_rsb, n_bt;
};

__device__ __forceinline__ EnvPtrs env_ptrs(const EnvDev& e, const double* pool) {
    EnvPtrs p;
    const double* q = pool + e.off;
    p.n_zss = e.n_zss;
    p.n_rss = e.n_rss;
    p.n_zsb = e.n_zsb;
    p.n_rsb = e.n_rsb;
    p.n_bt = e.n_bt;
    p.z_ss = q; q += p.n_zss;
    p.rp_ss = q; q += p.n_rss;
    p.cw = q; q += (long long)p.n_rss * p.n_zss;
    p.z_sb = q; q += p.n_zsb;
    p.rp_sb = q; q += p.n_rsb;
    p.cb = q; q += (long long)p.n_rsb * p.n_zsb;
    p.rhob = q; q += (long long)p.n_rsb * p.n_zsb;
    p.attn = q; q += (long long)p.n_rsb * p.n_zsb;
    p.rb = q; q += p.n_bt;
    p.zb = q;
    return p;
}

// index idx with arr[idx] <= v < arr[idx+1] (profl.py:8-35 semantics)
__device__ __forceinline__ int seg_search(double v, const double* arr, int n) {
    if (n <= 1 || v <= arr[0]) return 0;
    if (v >= arr[n - 1]) return n - 2;
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (arr[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double lerp_seg(double x, double x0, double x1, double y0, double y1) {
    if (x1 == x0) return y0;
    return y0 + (y1 - y0) * ((x - x0) / (x1 - x0));
}

struct RowProps {
    float cw, cb, rhob, attn;
};

// Interpolated water / seabed properties at depth z for the active profiles,
// rounded to float32 as the reference stores them.
__device__ __forceinline__ RowProps row_props(const EnvPtrs& e, int ss, int sb, double z, double lyrw_lambda,
                              double attnf) {
    RowProps o;
    const double* cwp = e.cw + (long long)ss * e.n_zss;
    const int n1 = e.n_zss;
    double v;
    if (z <= e.z_ss[0]) v = cwp[0];
    else if (z >= e.z_ss[n1 - 1]) v = cwp[n1 - 1];
    else {
        const int k = seg_search(z, e.z_ss, n1);
        v = lerp_seg(z, e.z_ss[k], e.z_ss[k + 1], cwp[k], cwp[k + 1]);
    }
    o.cw = (float)v;
    const int n2 = e.n_zsb;
    const long long so = (long long)sb * n2;
    const double* cbp = e.cb + so;
    const double* rhp = e.rhob + so;
    const double* atp = e.attn + so;
    const double z0 = e.z_sb[0], zl = e.z_sb[n2 - 1];
    const int k = seg_search(z, e.z_sb, n2);
    if (z <= z0) {
        o.cb = (float)cbp[0];
        o.rhob = (float)rhp[0];
    } else if (z >= zl) {
        o.cb = (float)cbp[n2 - 1];
        o.rhob = (float)rhp[n2 - 1];
    } else {
        o.cb = (float)lerp_seg(z, e.z_sb[k], e.z_sb[k + 1], cbp[k], cbp[k + 1]);
        o.rhob = (float)lerp_seg(z, e.z_sb[k], e.z_sb[k + 1], rhp[k], rhp[k + 1]);
    }
    // attenuation with the absorbing layer: profile, then constant over the
    // first 75 % of the layer, then a linear ramp to attnf (profl.py:121-140)
    const double alast = atp[n2 - 1];
    const double zl1 = zl + 0.75 * lyrw_lambda, zl2 = zl + lyrw_lambda;
    if (z <= zl) {
        if (z <= z0) v = atp[0];
        else v = lerp_seg(z, e.z_sb[k], e.z_sb[k + 1], atp[k], atp[k + 1]);
    } else if (z <= zl1) {
        v = alast;
    } else if (z <= zl2) {
        v = lerp_seg(z, zl1, zl2, alast, attnf);
    } else {
        v = attnf;
    }
    o.attn = (float)v;
    return o;
}

// Write the layer-selected coefficients of rows [lo, hi] (matrc.py:16-107
// with iz == jz, preceded by the alpw / alpb / ksqw / ksqb maths of
// cupyram.py:782-803).
__device__ __forceinline__ void assemble_rows(const RayDev& ry, const EnvPtrs& e, int ss, int sb, int iz, int lo,
                              int hi, float* f1, float* f2, float* f3, float2* ksq) {
    const double step = ry.zmax / (double)(ry.nz + 1);
    const double eta = 1.0 / (40.0 * M_PI * 0.43429448190325176);  // 1/(40 pi log10 e)
    const double k02 = ry.k0 * ry.k0;
    for (int i = lo; i <= hi; ++i) {
        const double z = (i == ry.nz + 1) ? ry.zmax : (double)i * step;
        const RowProps p = row_props(e, ss, sb, z, ry.lyrw_lambda, ry.attnf);
        const long long o = ry.col + (long long)i * kTile;
        if (i <= iz) {
            const double alpw = sqrt((double)p.cw / ry.c0);
            const double ow = ry.omega / (double)p.cw;
            f1[o] = (float)(1.0 / alpw);
            f2[o] = 1.0f;
            f3[o] = (float)alpw;
            ksq[o] = make_float2((float)(ow * ow - k02), 0.0f);
        } else {
            const double alpb = sqrt((double)(p.rhob * p.cb) / ry.c0);
            const double ob = ry.omega / (double)p.cb;
            const double ti = ob * eta * (double)p.attn;  // term = ob + i*ti
            f1[o] = (float)((double)p.rhob / alpb);
            f2[o] = (float)(1.0 / (double)p.rhob);
            f3[o] = (float)alpb;
            ksq[o] = make_float2((float)(ob * ob - ti * ti - k02), (float)(2.0 * ob * ti));
        }
    }
}

// ---------------------------------------------------------------------------
// Galerkin row: D_i = (d1, d2, d3) from the 3-row window of f1..f3, ksq
// ---------------------------------------------------------------------------
struct Win {
    float f1c, f2m, f2c, f2p, f3m, f3c, f3p;
    float2 km, kc, kp;
};

struct Drow {
    double2 d1, d2, d3;
};

__device__ __forceinline__ Drow galerkin(const Win& w, double cfact) {
    const double f1 = w.f1c;
    const double c1 = cfact * f1 * ((double)w.f2m + (double)w.f2c) * (double)w.f3m;
    const double c2v = -cfact * f1 * ((double)w.f2m + 2.0 * (double)w.f2c + (double)w.f2p) * (double)w.f3c;
    const double c3 = cfact * f1 * ((double)w.f2c + (double)w.f2p) * (double)w.f3p;
    const double df = 1.0 / 12.0;
    Drow d;
    d.d1 = c2(c1 + df * ((double)w.km.x + (double)w.kc.x), df * ((double)w.km.y + (double)w.kc.y));
    d.d2 = c2(c2v + df * ((double)w.km.x + 6.0 * (double)w.kc.x + (double)w.kp.x),
              df * ((double)w.km.y + 6.0 * (double)w.kc.y + (double)w.kp.y));
    d.d3 = c2(c3 + df * ((double)w.kc.x + (double)w.kp.x), df * ((double)w.kc.y + (double)w.kp.y));
    return d;
}

struct Col {
    const float* f1;
    const float* f2;
    const float* f3;
    const float2* ksq;
    double2* u;
    double2* W;
    double2* G;
};

struct StepCtx {
    Col c;
    int nz;
    double cfact, a1, a2;
    double2 u0;  // field value held at the surface row (non-zero only for zs < dz)
};

// ---------------------------------------------------------------------------
// the passes of one range step
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// cp.async helpers (per-thread asynchronous global -> shared copies)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// Zero-filling variants: when `on` is false no global byte is read and the
// destination is filled with zeros (src-size operand 0), so a copy can be
// issued unconditionally from branch-free code (src must still be a valid
// address; callers clamp it).
__device__ __forceinline__ void cp16z(void* dst, const void* src, bool on) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(on ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp8z(void* dst, const void* src, bool on) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(on ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Bulk tensor copies (cp.async.bulk.tensor, no multicast) completing on an
// mbarrier in shared memory
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init1(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
// arrive once and expect `bytes` more bytes of copies on the current phase
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// true once the phase of this parity has completed; false after `limit`
// polls.  A poll may suspend the thread for up to `suspend_ns` (it resumes
// when the phase completes), so that a waiting warp does not take issue
// slots from the SM's other warps.
#ifndef CR_MBAR_SUSPEND_NS
#define CR_MBAR_SUSPEND_NS 100
#endif
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned limit) {
    for (unsigned it = 0; it < limit; ++it) {
        unsigned done;
        if (CR_MBAR_SUSPEND_NS > 0) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(smem_u32(bar)), "r"(parity), "n"(CR_MBAR_SUSPEND_NS)
                : "memory");
        } else {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(smem_u32(bar)), "r"(parity)
                : "memory");
        }
        if (done) return true;
    }
    return false;
}
// one box of a 2-D tensor map (map: address of a CUtensorMap in parameter,
// constant or global memory) at element coordinates (x, y) into shared memory
__device__ __forceinline__ void tma_2d(void* dst, const void* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
// orders this thread's earlier generic-proxy accesses before later
// async-proxy (bulk copy) accesses, in global and shared memory
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }
// the same, for shared memory only
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

struct EnvRow {
    float f1, f2, f3;
    float2 k;
};

__device__ __forceinline__ Drow galerkin3(const EnvRow& m, const EnvRow& c, const EnvRow& p, double cfact) {
    Win w;
    w.f1c = c.f1;
    w.f2m = m.f2; w.f2c = c.f2; w.f2p = p.f2;
    w.f3m = m.f3; w.f3c = c.f3; w.f3p = p.f3;
    w.km = m.k; w.kc = c.k; w.kp = p.k;
    return galerkin(w, cfact);
}

// Issue the copies of stream row r into ring slot `slot` (one commit group,
// possibly empty when r is outside 0..nz+1).
__device__ __forceinline__ double tl_db(double amp, double r) {
    return -20.0 * log10(amp + 1e-20) + 10.0 * log10(r + 1e-20);
}

}  // namespace crk
