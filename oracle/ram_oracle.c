/*
 * ram_oracle.c - CPU restatement of the CuPyRAM range march (TEST INFRASTRUCTURE).
 *
 * This file is the oracle the engine is checked against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs load
 * it; the product (cupyram_b200) never does.
 *
 * It restates, one ray at a time on the host, the algorithm of the reference
 * (clapeyre/cupyram, a GPU port of PyRAM / RAM v1.5):
 *   profl      cupyram/profl.py:8-140, cupyram/cupyram.py:728-803
 *   updat      cupyram/updat.py:38-140, cupyram/cupyram.py:951-999
 *   matrc      cupyram/matrc.py:16-107 (init_profiles, iz == jz branch)
 *   solve      cupyram/fused_kernel.py:20-153 (Galerkin coefficients + Thomas)
 *   outpt      cupyram/outpt.py:11-57
 *   selfs      cupyram/cupyram.py:1001-1063
 *   run loop   cupyram/cupyram.py:273-317
 *   epade      cupyram/pade.py:17-273
 *
 * Modes (ORACLE_*):
 *   REF    storage rounded exactly where the reference rounds: f1..f3, cw, cb,
 *          rhob, attn in float32, ksq in complex64, the Thomas workspace in
 *          complex64, float32 sums where Numba would form them, the eps=1e-30
 *          additions, and identity Pade terms in the self-starter.
 *   PLAIN  f1..f3 / ksq stored like the reference (float32 / complex64) but
 *          all arithmetic and the workspace in FP64 / complex128.  This is the
 *          engine's plain complex128 form.
 *   F64    everything FP64 (environment too): the FP64 oracle of the
 *          precision study.
 *   SUM    PLAIN arithmetic with each range step in partial-fraction (sum)
 *          form: prod_j (1 + pd1_j X)/(1 + pd2_j X) = c_inf + sum_k c_k/(1 + pd2_k X),
 *          i.e. u_new = c_inf u + sum_k c_k (M + pd2_k D)^{-1} M u.  Same
 *          rational operator as the product form; used to check the engine's
 *          sum-form march against the product form.
 *   CHOSEN, CHOSEN_C32, CHOSEN_F32
 *          models of the engine's chosen form in sum form, rounded where
 *          the batched kernel rounds: 1/den, w and the elimination's
 *          coupling in complex64 (the factorisation recurrence itself in
 *          FP64), M u rounded to complex64, the elimination and the
 *          back-substitution in FP32.  CHOSEN combines the terms in FP64
 *          (the engine's form); CHOSEN_C32 combines them in FP32; CHOSEN_F32
 *          also forms the coupling in FP32 from a complex64 d1 (the model of
 *          the engine's fast form).
 *   REFINED
 *          the engine's refined form: CHOSEN, then per term one
 *          iterative-refinement step - the residual of the complex64 solve
 *          M u - (M + pd2 D) x against the FP64 Galerkin rows, its correction
 *          solved with the same complex64 factors in FP32, added in FP64.
 *   SIM    REF plus the scalar promotions of Numba's CUDA simulator under
 *          NumPy 2 (a Python float times a float32 stays float32), which is
 *          how the golden fixtures were produced: the Galerkin c1..c3 are
 *          formed in float32 and d1..d3 in complex64.  Used only to pin the
 *          oracle to the fixtures at rounding level.
 *
 * Parity pinned against: the .npz fixtures of tests/golden (the reference itself run on CPU
 * under Numba's CUDA simulator) and RAM v1.5's tl_ref.line.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cupyram_b200.h"

#include <pthread.h>

#define ORACLE_REF 0
#define ORACLE_PLAIN 1
#define ORACLE_F64 2
#define ORACLE_SIM 3
#define ORACLE_SUM 4
#define ORACLE_CHOSEN 5
#define ORACLE_CHOSEN_C32 6
#define ORACLE_CHOSEN_F32 7
#define ORACLE_REFINED 8

typedef double complex cd;

/* ------------------------------------------------------------------------- */
/* Pade coefficients (cupyram/pade.py:17-273, RAM's epade)                   */
/* ------------------------------------------------------------------------- */
static cd cpow_int(cd z, int n) {
    cd r = 1.0;
    for (int i = 0; i < n; ++i) r *= z;
    return r;
}

/* Laguerre iteration for one root of a[0..n] (pade.py:95-149).
   Returns 0 on success, -1 when 100 iterations pass without convergence. */
static int guerre(cd* a, int n, cd* zio, double err, int nter) {
    cd az[2 * CR_MAX_NP + 2], azz[2 * CR_MAX_NP + 2];
    const double eps = 1e-20;
    cd z = *zio;
    for (int i = 0; i < n; ++i) az[i] = (double)(i + 1) * a[i + 1];
    for (int i = 0; i < n - 1; ++i) azz[i] = (double)(i + 1) * az[i + 1];
    int iter = 0, jter = 0;
    double adz = INFINITY;
    while (adz > err && iter < nter - 1) {
        cd p = a[n - 1] + a[n] * z;
        for (int i = n - 2; i >= 0; --i) p = a[i] + z * p;
        if (cabs(p) < eps) { *zio = z; return 0; }
        cd pz = az[n - 2] + az[n - 1] * z;
        for (int i = n - 3; i >= 0; --i) pz = az[i] + z * pz;
        cd pzz = azz[n - 3] + azz[n - 2] * z;
        for (int i = n - 4; i >= 0; --i) pzz = azz[i] + z * pzz;
        cd f = pz / p;
        cd g = f * f - pzz / p;
        cd h = csqrt((double)(n - 1) * ((double)n * g - f * f));
        cd dz;
        if (cabs(f + h) > cabs(f - h)) dz = -(double)n / (f + h);
        else dz = -(double)n / (f - h);
        ++iter;
        ++jter;
        if (jter == 9) { jter = 0; dz *= I; }
        z += dz;
        adz = cabs(dz);
        if (iter == 100) { *zio = z; return -1; }
    }
    *zio = z;
    return 0;
}

/* All roots of the degree-n polynomial a[0..n] (pade.py:153-177). */
static int fndrt(cd* a, int n, cd* z) {
    if (n == 1) { z[0] = -a[0] / a[1]; return 0; }
    if (n != 2) {
        for (int k = n - 1; k >= 2; --k) {
            cd root = 0.0;
            if (guerre(a, k + 1, &root, 1e-12, 1000)) return -1;
            if (guerre(a, k + 1, &root, 0.0, 5)) return -1;
            z[k] = root;
            for (int i = k; i >= 0; --i) a[i] += root * a[i + 1];
            for (int i = 0; i <= k; ++i) a[i] = a[i + 1];
        }
    }
    cd disc = csqrt(a[1] * a[1] - 4.0 * a[0] * a[2]);
    z[1] = 0.5 * (-a[1] + disc) / a[2];
    z[0] = 0.5 * (-a[1] - disc) / a[2];
    return 0;
}

int oracle_pade(double freq, double c0, int np, int ns, double dr, int ip, cd* pd1, cd* pd2) {
    const int n = 2 * np;
    double bin[2 * CR_MAX_NP + 1][2 * CR_MAX_NP + 1];
    cd a[2 * CR_MAX_NP + 1][2 * CR_MAX_NP + 1];
    cd b[2 * CR_MAX_NP], dg[2 * CR_MAX_NP + 1], dh1[2 * CR_MAX_NP + 1], dh2[2 * CR_MAX_NP + 1],
        dh3[2 * CR_MAX_NP];
    double fact[2 * CR_MAX_NP + 1];
    if (np < 1 || np > CR_MAX_NP) return -2;
    memset(bin, 0, sizeof bin);
    for (int i = 0; i <= n; ++i) for (int j = 0; j <= n; ++j) a[i][j] = 0.0;
    for (int i = 0; i < n; ++i) { b[i] = 0.0; dh1[i] = dh2[i] = dh3[i] = 0.0; }
    for (int i = 0; i <= n; ++i) dg[i] = 0.0;
    dh1[n] = dh2[n] = 0.0;

    const double k0 = 2.0 * M_PI * freq / c0;
    const double sig = k0 * dr;
    double nu = 0.0, alp = 0.0;
    if (ip != 1) { nu = 1.0; alp = -0.25; }

    fact[0] = 1.0;
    for (int i = 1; i < n; ++i) fact[i] = (double)(i + 1) * fact[i - 1];
    for (int i = 0; i <= n; ++i) { bin[i][0] = 1.0; bin[i][i] = 1.0; }
    for (int i = 2; i <= n; ++i)
        for (int j = 1; j < i; ++j) bin[i][j] = bin[i - 1][j - 1] + bin[i - 1][j];

    /* derivatives of the operator function at x=0 (pade.py:17-43) */
    dh1[0] = 0.5 * I * sig;
    double exp1 = -0.5;
    dh2[0] = alp;
    double exp2 = -1.0;
    dh3[0] = -2.0 * nu;
    double exp3 = -1.0;
    for (int i = 1; i < n; ++i) {
        dh1[i] = dh1[i - 1] * exp1; exp1 -= 1.0;
        dh2[i] = dh2[i - 1] * exp2; exp2 -= 1.0;
        dh3[i] = -nu * dh3[i - 1] * exp3; exp3 -= 1.0;
    }
    dg[0] = 1.0;
    dg[1] = dh1[0] + dh2[0] + dh3[0];
    for (int i = 1; i < n; ++i) {
        dg[i + 1] = dh1[i] + dh2[i] + dh3[i];
        for (int j = 0; j < i; ++j) dg[i + 1] += bin[i][j] * (dh1[j] + dh2[j] + dh3[j]) * dg[i - j];
    }
    /* accuracy constraints (pade.py:229-238) */
    for (int i = 0; i < n; ++i) b[i] = dg[i + 1];
    for (int i = 0; i < n; ++i) {
        if (2 * i <= n - 1) a[i][2 * i] = fact[i];
        for (int j = 0; j <= i; ++j)
            if (2 * j + 1 <= n - 1) a[i][2 * j + 1] = -bin[i + 1][j + 1] * fact[j] * dg[i - j];
    }
    /* stability constraints (pade.py:240-256) */
    if (ns >= 1) {
        cd z1 = -3.0;
        b[n - 1] = -1.0;
        for (int j = 0; j < np; ++j) { a[n - 1][2 * j] = cpow_int(z1, j + 1); a[n - 1][2 * j + 1] = 0.0; }
    }
    if (ns >= 2) {
        cd z1 = -1.5;
        b[n - 2] = -1.0;
        for (int j = 0; j < np; ++j) { a[n - 2][2 * j] = cpow_int(z1, j + 1); a[n - 2][2 * j + 1] = 0.0; }
    }
    /* Gaussian elimination with partial pivoting (pade.py:47-91) */
    for (int i = 0; i < n; ++i) {
        if (i < n - 1) {
            int i0 = i;
            double amp0 = cabs(a[i][i]);
            for (int j = i + 1; j < n; ++j) {
                double amp = cabs(a[j][i]);
                if (amp > amp0) { i0 = j; amp0 = amp; }
            }
            if (i0 != i) {
                cd t = b[i0]; b[i0] = b[i]; b[i] = t;
                for (int j = i; j <= n; ++j) { t = a[i0][j]; a[i0][j] = a[i][j]; a[i][j] = t; }
            }
        }
        a[i][i] = 1.0 / a[i][i];
        b[i] *= a[i][i];
        if (i < n - 1) {
            for (int j = i + 1; j <= n; ++j) a[i][j] *= a[i][i];
            for (int k = i + 1; k < n; ++k) {
                b[k] -= a[k][i] * b[i];
                for (int j = i + 1; j < n; ++j) a[k][j] -= a[k][i] * a[i][j];
            }
        }
    }
    for (int i = n - 2; i >= 0; --i)
        for (int j = i + 1; j < n; ++j) b[i] -= a[i][j] * b[j];

    cd poly[2 * CR_MAX_NP + 1], roots[2 * CR_MAX_NP + 1];
    poly[0] = 1.0;
    for (int j = 0; j < np; ++j) poly[j + 1] = b[2 * j];
    if (fndrt(poly, np, roots)) return -1;
    for (int j = 0; j < np; ++j) pd1[j] = -1.0 / roots[j];
    poly[0] = 1.0;
    for (int j = 0; j < np; ++j) poly[j + 1] = b[2 * j + 1];
    if (fndrt(poly, np, roots)) return -1;
    for (int j = 0; j < np; ++j) pd2[j] = -1.0 / roots[j];
    return 0;
}

/* ------------------------------------------------------------------------- */
/* the march of one ray                                                      */
/* ------------------------------------------------------------------------- */
typedef struct {
    int mode;
    int nz;
    double dz, dr, zmax, k0, omega, c0, lyrw_lambda, attnf;
    /* environment arrays (pool) */
    const double *z_ss, *rp_ss, *cw, *z_sb, *rp_sb, *cb, *rhob, *attn, *rb, *zb;
    int n_zss, n_rss, n_zsb, n_rsb, n_bt;
    /* per-row state */
    double *zg;                 /* depth grid (linspace)                          */
    double *cwr, *cbr, *rhobr, *attnr;  /* interpolated profiles (float-rounded in REF/PLAIN) */
    double *alpw, *alpb;
    double *ksqw;
    cd *ksqb;
    double *f1, *f2, *f3;
    cd *ksq;
    cd *u, *up, *rs;            /* field and Thomas workspace                     */
    int iz, ss_ind, sb_ind, bt_ind;
} ray_state;

static inline double rnd32(int mode, double x) { return mode == ORACLE_F64 ? x : (double)(float)x; }
static inline float f32(double x) { return (float)x; }
static inline cd rnd64c(int mode, cd x) {
    if (mode == ORACLE_F64) return x;
    return (double)(float)creal(x) + I * (double)(float)cimag(x);
}

/* binary search of profl.py:8-35 */
static int bsearch_ref(double val, const double* arr, int count) {
    if (count == 0) return 0;
    if (val <= arr[0]) return 0;
    if (val >= arr[count - 1]) return count - 2;
    int low = 0, high = count - 1;
    while (low < high) {
        int mid = (low + high) / 2;
        if (arr[mid] <= val) {
            if (arr[mid + 1] > val) return mid;
            low = mid + 1;
        } else {
            high = mid;
        }
    }
    return low;
}

static inline double lerp_ref(double x, double x0, double x1, double y0, double y1) {
    if (x1 == x0) return y0;
    double t = (x - x0) / (x1 - x0);
    return y0 + (y1 - y0) * t;
}

/* profl: interpolate the active profiles onto the grid and derive alpw, alpb,
   ksqw, ksqb (profl.py:45-140, cupyram.py:728-803). */
static void profl(ray_state* s) {
    const int mode = s->mode;
    const double* cwp = s->cw + (size_t)s->ss_ind * s->n_zss;
    const double* cbp = s->cb + (size_t)s->sb_ind * s->n_zsb;
    const double* rhp = s->rhob + (size_t)s->sb_ind * s->n_zsb;
    const double* atp = s->attn + (size_t)s->sb_ind * s->n_zsb;
    const int nss = s->n_zss, nsb = s->n_zsb;
    const double zsb_last = s->z_sb[nsb - 1];
    const double attn_last = atp[nsb - 1];
    const double zl1 = zsb_last + 0.75 * s->lyrw_lambda;
    const double zl2 = zsb_last + s->lyrw_lambda;
    const double eta = 1.0 / (40.0 * M_PI * log10(exp(1.0)));
    for (int k = 0; k < s->nz + 2; ++k) {
        const double z = s->zg[k];
        int idx = bsearch_ref(z, s->z_ss, nss);
        double v;
        if (z <= s->z_ss[0]) v = cwp[0];
        else if (z >= s->z_ss[nss - 1]) v = cwp[nss - 1];
        else v = lerp_ref(z, s->z_ss[idx], s->z_ss[idx + 1], cwp[idx], cwp[idx + 1]);
        s->cwr[k] = rnd32(mode, v);
        int isb = bsearch_ref(z, s->z_sb, nsb);
        if (z <= s->z_sb[0]) v = cbp[0];
        else if (z >= s->z_sb[nsb - 1]) v = cbp[nsb - 1];
        else v = lerp_ref(z, s->z_sb[isb], s->z_sb[isb + 1], cbp[isb], cbp[isb + 1]);
        s->cbr[k] = rnd32(mode, v);
        if (z <= s->z_sb[0]) v = rhp[0];
        else if (z >= s->z_sb[nsb - 1]) v = rhp[nsb - 1];
        else v = lerp_ref(z, s->z_sb[isb], s->z_sb[isb + 1], rhp[isb], rhp[isb + 1]);
        s->rhobr[k] = rnd32(mode, v);
        if (z <= zsb_last) {
            if (z <= s->z_sb[0]) v = atp[0];
            else v = lerp_ref(z, s->z_sb[isb], s->z_sb[isb + 1], atp[isb], atp[isb + 1]);
        } else if (z <= zl1) {
            v = attn_last;
        } else if (z <= zl2) {
            v = lerp_ref(z, zl1, zl2, attn_last, s->attnf);
        } else {
            v = s->attnf;
        }
        s->attnr[k] = rnd32(mode, v);
        /* derived quantities (cupyram.py:782-803, single-frequency path) */
        s->alpw[k] = sqrt(s->cwr[k] / s->c0);
        const double rc = (mode == ORACLE_F64) ? s->rhobr[k] * s->cbr[k]
                                                : (double)((float)s->rhobr[k] * (float)s->cbr[k]);
        s->alpb[k] = sqrt(rc / s->c0);
        const double ow = s->omega / s->cwr[k];
        s->ksqw[k] = ow * ow - s->k0 * s->k0;
        const cd term = (s->omega / s->cbr[k]) * (1.0 + I * eta * s->attnr[k]);
        s->ksqb[k] = term * term - s->k0 * s->k0;
    }
}

/* init_profiles with iz == jz (matrc.py:16-107) */
static void init_profiles(ray_state* s) {
    const int mode = s->mode;
    for (int i = 0; i < s->nz + 2; ++i) {
        if (i <= s->iz) {
            s->f1[i] = rnd32(mode, 1.0 / s->alpw[i]);
            s->f2[i] = 1.0;
            s->f3[i] = rnd32(mode, s->alpw[i]);
            s->ksq[i] = rnd64c(mode, s->ksqw[i]);
        } else {
            s->f1[i] = rnd32(mode, s->rhobr[i] / s->alpb[i]);
            s->f2[i] = (mode == ORACLE_SIM) ? (double)(1.0f / (float)s->rhobr[i]) : rnd32(mode, 1.0 / s->rhobr[i]);
            s->f3[i] = rnd32(mode, s->alpb[i]);
            s->ksq[i] = rnd64c(mode, s->ksqb[i]);
        }
    }
}

/* Galerkin row coefficients (fused_kernel.py:20-69).  REF mode reproduces
   Numba's float32 / complex64 intermediate sums. */
static inline void galerkin(const ray_state* s, int i, cd pd1, cd pd2, cd* r, cd* q) {
    const double dz = s->dz;
    const double cfact = 0.5 / (dz * dz);
    const double dfact = 1.0 / 12.0;
    const double* f1 = s->f1;
    const double* f2 = s->f2;
    const double* f3 = s->f3;
    const cd* k = s->ksq;
    double c1, c2, c3;
    cd d1, d2, d3;
    if (s->mode == ORACLE_SIM) {
        /* every product / sum with a Python-float constant stays float32 */
        const float fc = f32(cfact), f1i = f32(f1[i]);
        const float a = f32(f2[i - 1]), bq = f32(f2[i]), cq = f32(f2[i + 1]);
        const float c1f = ((fc * f1i) * (a + bq)) * f32(f3[i - 1]);
        const float c2f = (((-fc) * f1i) * ((a + 2.0f * bq) + cq)) * f32(f3[i]);
        const float c3f = ((fc * f1i) * (bq + cq)) * f32(f3[i + 1]);
        const float dff = f32(dfact);
        float complex km = (float)creal(k[i - 1]) + I * (float)cimag(k[i - 1]);
        float complex kc = (float)creal(k[i]) + I * (float)cimag(k[i]);
        float complex kp = (float)creal(k[i + 1]) + I * (float)cimag(k[i + 1]);
        float complex s1 = km + kc, s2 = (km + 6.0f * kc) + kp, s3 = kc + kp;
        float complex e1 = c1f + dff * s1, e2 = c2f + dff * s2, e3 = c3f + dff * s3;
        d1 = (double)crealf(e1) + I * (double)cimagf(e1);
        d2 = (double)crealf(e2) + I * (double)cimagf(e2);
        d3 = (double)crealf(e3) + I * (double)cimagf(e3);
        (void)c1; (void)c2; (void)c3;
    } else if (s->mode == ORACLE_REF) {
        const double f2a = (double)((float)f2[i - 1] + (float)f2[i]);
        const double f2b = (double)((float)f2[i] + (float)f2[i + 1]);
        c1 = cfact * f1[i] * f2a * f3[i - 1];
        c2 = -cfact * f1[i] * (f2[i - 1] + 2.0 * f2[i] + f2[i + 1]) * f3[i];
        c3 = cfact * f1[i] * f2b * f3[i + 1];
        const cd ka = rnd64c(ORACLE_REF, k[i - 1] + k[i]);
        const cd kb = rnd64c(ORACLE_REF, k[i] + k[i + 1]);
        d1 = c1 + dfact * ka;
        d2 = c2 + dfact * (k[i - 1] + 6.0 * k[i] + k[i + 1]);
        d3 = c3 + dfact * kb;
    } else {
        c1 = cfact * f1[i] * (f2[i - 1] + f2[i]) * f3[i - 1];
        c2 = -cfact * f1[i] * (f2[i - 1] + 2.0 * f2[i] + f2[i + 1]) * f3[i];
        c3 = cfact * f1[i] * (f2[i] + f2[i + 1]) * f3[i + 1];
        d1 = c1 + dfact * (k[i - 1] + k[i]);
        d2 = c2 + dfact * (k[i - 1] + 6.0 * k[i] + k[i + 1]);
        d3 = c3 + dfact * (k[i] + k[i + 1]);
    }
    const double a1 = s->k0 * s->k0 / 6.0;
    const double a2 = 2.0 * s->k0 * s->k0 / 3.0;
    r[0] = a1 + pd2 * d1; r[1] = a2 + pd2 * d2; r[2] = a1 + pd2 * d3;
    q[0] = a1 + pd1 * d1; q[1] = a2 + pd1 * d2; q[2] = a1 + pd1 * d3;
}

/* One range step: n product-form Pade terms, each a Thomas solve in place
   (fused_kernel.py:72-153). */
static void march_step(ray_state* s, int n, const cd* pd1, const cd* pd2) {
    const int nz = s->nz;
    const int ref = s->mode == ORACLE_REF || s->mode == ORACLE_SIM;
    const cd eps = ref ? 1e-30 : 0.0;
    cd* u = s->u;
    cd* up = s->up;
    cd* rs = s->rs;
    for (int j = 0; j < n; ++j) {
        cd r[3], q[3];
        galerkin(s, 1, pd1[j], pd2[j], r, q);
        cd rhs = q[0] * u[0] + q[1] * u[1] + q[2] * u[2] + eps;
        up[1] = r[2] / r[1];
        rs[1] = rhs / r[1];
        if (ref) { up[1] = rnd64c(ORACLE_REF, up[1]); rs[1] = rnd64c(ORACLE_REF, rs[1]); }
        for (int i = 2; i <= nz; ++i) {
            galerkin(s, i, pd1[j], pd2[j], r, q);
            rhs = q[0] * u[i - 1] + q[1] * u[i] + q[2] * u[i + 1] + eps;
            const cd den = r[1] - r[0] * up[i - 1];
            up[i] = r[2] / den;
            rs[i] = (rhs - r[0] * rs[i - 1]) / den + eps;
            if (ref) { up[i] = rnd64c(ORACLE_REF, up[i]); rs[i] = rnd64c(ORACLE_REF, rs[i]); }
        }
        u[nz] = rs[nz];
        for (int i = nz - 1; i >= 1; --i) u[i] = rs[i] - up[i] * u[i + 1] + eps;
    }
}

/* One range step in partial-fraction form (see ORACLE_SUM). */
static void march_step_sum(ray_state* s, int n, const cd* pd1, const cd* pd2) {
    const int nz = s->nz;
    cd cinf = 1.0;
    for (int j = 0; j < n; ++j) cinf *= pd1[j] / pd2[j];
    cd* mu = (cd*)malloc(sizeof(cd) * (size_t)(nz + 2));
    cd* acc = (cd*)malloc(sizeof(cd) * (size_t)(nz + 2));
    cd* x = (cd*)malloc(sizeof(cd) * (size_t)(nz + 2));
    const double a1 = s->k0 * s->k0 / 6.0, a2 = 2.0 * s->k0 * s->k0 / 3.0;
    for (int i = 1; i <= nz; ++i) {
        mu[i] = a1 * (s->u[i - 1] + s->u[i + 1]) + a2 * s->u[i];
        acc[i] = cinf * s->u[i];
    }
    for (int k = 0; k < n; ++k) {
        cd ck = 1.0 - pd1[k] / pd2[k];
        for (int j = 0; j < n; ++j)
            if (j != k) ck *= (1.0 - pd1[j] / pd2[k]) / (1.0 - pd2[j] / pd2[k]);
        const cd zero = 0.0;
        cd r[3], q[3];
        /* Thomas on (M + pd2_k D) x = M u */
        galerkin(s, 1, zero, pd2[k], r, q);
        s->up[1] = r[2] / r[1];
        s->rs[1] = mu[1] / r[1];
        for (int i = 2; i <= nz; ++i) {
            galerkin(s, i, zero, pd2[k], r, q);
            const cd den = r[1] - r[0] * s->up[i - 1];
            s->up[i] = r[2] / den;
            s->rs[i] = (mu[i] - r[0] * s->rs[i - 1]) / den;
        }
        x[nz] = s->rs[nz];
        for (int i = nz - 1; i >= 1; --i) x[i] = s->rs[i] - s->up[i] * x[i + 1];
        for (int i = 1; i <= nz; ++i) acc[i] += ck * x[i];
    }
    for (int i = 1; i <= nz; ++i) s->u[i] = acc[i];
    free(mu);
    free(acc);
    free(x);
}

typedef float complex cf;
static inline cf to_c64(cd z) { return (float)creal(z) + I * (float)cimag(z); }
static inline cd to_c128(cf z) { return (double)crealf(z) + I * (double)cimagf(z); }

/* One range step of the chosen-form models (see ORACLE_CHOSEN): sum form,
   downward elimination, complex64 factors and FP32 recurrences.  comb32:
   terms combined in FP32; coupling32: the coupling -(a1 + pd2 d1)/den
   formed in FP32 from a complex64 d1. */
static void march_step_chosen(ray_state* s, int n, const cd* pd1, const cd* pd2, int comb32, int coupling32,
                              int refine) {
    const int nz = s->nz;
    cd cinf = 1.0;
    for (int j = 0; j < n; ++j) cinf *= pd1[j] / pd2[j];
    cf* mu = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    cd* acc = (cd*)malloc(sizeof(cd) * (size_t)(nz + 2));
    cf* accf = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    cf* g = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    cf* x = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    cf* q = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    cf* w = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    cf* al = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
    const double a1 = s->k0 * s->k0 / 6.0, a2 = 2.0 * s->k0 * s->k0 / 3.0;
    for (int i = 1; i <= nz; ++i) {
        mu[i] = to_c64(a1 * (s->u[i - 1] + s->u[i + 1]) + a2 * s->u[i]);
        acc[i] = cinf * s->u[i];
        accf[i] = to_c64(cinf) * to_c64(s->u[i]);
    }
    for (int k = 0; k < n; ++k) {
        cd ck = 1.0 - pd1[k] / pd2[k];
        for (int j = 0; j < n; ++j)
            if (j != k) ck *= (1.0 - pd1[j] / pd2[k]) / (1.0 - pd2[j] / pd2[k]);
        const cd zero = 0.0;
        cd r[3], rq[3];
        cd wp = 0.0;
        for (int i = 1; i <= nz; ++i) {
            galerkin(s, i, zero, pd2[k], r, rq);
            const cd qd = 1.0 / (r[1] - r[0] * wp);
            wp = r[2] * qd;
            q[i] = to_c64(qd);
            w[i] = to_c64(wp);
            if (coupling32) {
                cd r1[3], q1[3];
                galerkin(s, i, zero, 1.0, r1, q1);  /* a1 + d1 */
                const cf cin = (float)a1 + to_c64(pd2[k]) * to_c64(r1[0] - a1);
                al[i] = -(cin * q[i]);
            } else {
                al[i] = to_c64(-(r[0] * to_c128(q[i])));
            }
        }
        cf gp = 0.0f;
        for (int i = 1; i <= nz; ++i) {
            gp = q[i] * mu[i] + al[i] * gp;
            g[i] = gp;
        }
        x[nz] = g[nz];
        for (int i = nz - 1; i >= 1; --i) x[i] = g[i] - w[i] * x[i + 1];
        const cf ckf = to_c64(ck);
        for (int i = 1; i <= nz; ++i) {
            acc[i] += ck * to_c128(x[i]);
            accf[i] += ckf * x[i];
        }
        if (refine) {
            /* residual of the complex64 solve against the FP64 rows, and its
               correction with the same complex64 factors */
            cf* res = (cf*)malloc(sizeof(cf) * (size_t)(nz + 2));
            for (int i = 1; i <= nz; ++i) {
                galerkin(s, i, zero, pd2[k], r, rq);
                const cd xm = i > 1 ? to_c128(x[i - 1]) : 0.0, xc = to_c128(x[i]),
                         xp = i < nz ? to_c128(x[i + 1]) : 0.0;
                const cd mud = a1 * (s->u[i - 1] + s->u[i + 1]) + a2 * s->u[i];
                res[i] = to_c64(mud - (r[0] * xm + r[1] * xc + r[2] * xp));
            }
            cf gq = 0.0f;
            for (int i = 1; i <= nz; ++i) {
                gq = q[i] * res[i] + al[i] * gq;
                g[i] = gq;
            }
            cf dx = g[nz];
            acc[nz] += ck * to_c128(dx);
            for (int i = nz - 1; i >= 1; --i) {
                dx = g[i] - w[i] * dx;
                acc[i] += ck * to_c128(dx);
            }
            free(res);
        }
    }
    for (int i = 1; i <= nz; ++i) s->u[i] = comb32 ? to_c128(accf[i]) : acc[i];
    free(mu);
    free(acc);
    free(accf);
    free(g);
    free(x);
    free(q);
    free(w);
    free(al);
}

/* updat (updat.py:38-140): returns 1 when the profiles must be re-interpolated. */
static int updat(ray_state* s, double r) {
    int need = 0;
    if (s->n_bt > 1) {
        while (s->bt_ind < s->n_bt - 1 && r >= s->rb[s->bt_ind + 1]) s->bt_ind++;
        const int jz = s->iz;
        const double rc = r + 0.5 * s->dr;
        const int b0 = s->bt_ind;
        const int b1 = b0 + 1 < s->n_bt ? b0 + 1 : b0;
        const double r0 = s->rb[b0], r1 = s->rb[b1], z0 = s->zb[b0], z1 = s->zb[b1];
        const double z = (b1 == b0) ? z0 : z0 + (rc - r0) * (z1 - z0) / (r1 - r0);
        int izn = (int)floor(z / s->dz);
        if (izn < 1) izn = 1;
        if (izn > s->nz - 1) izn = s->nz - 1;
        s->iz = izn;
        if (izn != jz) need = 1;
    }
    if (s->n_rss > 1) {
        const int o = s->ss_ind;
        while (s->ss_ind < s->n_rss - 1 && r >= s->rp_ss[s->ss_ind + 1]) s->ss_ind++;
        if (s->ss_ind != o) need = 1;
    }
    if (s->n_rsb > 1) {
        const int o = s->sb_ind;
        while (s->sb_ind < s->n_rsb - 1 && r >= s->rp_sb[s->sb_ind + 1]) s->sb_ind++;
        if (s->sb_ind != o) need = 1;
    }
    return need;
}

/* outpt (outpt.py:11-57); the CP grid is filled (the reference leaves it 0). */
static void outpt(const ray_state* s, const cr_ray* ry, double r, int* mdr, int* tlc, double* tll,
                  double* cpl, double* tlg, double* cpg) {
    const double eps = 1e-20;
    *mdr += 1;
    if (*mdr != ry->ndr) return;
    *mdr = 0;
    *tlc += 1;
    const int t = *tlc;
    if (t >= ry->nvr) return;
    const double ri = ry->zr / ry->dz;
    const int ir = (int)floor(ri);
    const double dir = ri - ir;
    const cd c = (1.0 - dir) * s->f3[ir] * s->u[ir] + dir * s->f3[ir + 1] * s->u[ir + 1];
    const double temp = 10.0 * log10(r + eps);
    tll[t] = -20.0 * log10(cabs(c) + eps) + temp;
    cpl[2 * t] = creal(c);
    cpl[2 * t + 1] = cimag(c);
    if (tlg) {
        for (int i = 0; i < ry->nvz; ++i) {
            const int j = (i + 1) * ry->ndz;
            if (j > s->nz + 1) break;
            const cd g = s->u[j] * s->f3[j];
            const size_t o = (size_t)i * ry->nvr + t;
            tlg[o] = -20.0 * log10(cabs(g) + eps) + temp;
            if (cpg) { cpg[2 * o] = creal(g); cpg[2 * o + 1] = cimag(g); }
        }
    }
}

static int run_ray(const cr_batch* b, int ib, int mode, double* tll_all, double* cpl_all,
                   double* tlg_all, double* cpg_all) {
    const cr_ray* ry = &b->rays[ib];
    const cr_env* ev = &b->envs[ry->env];
    ray_state s;
    memset(&s, 0, sizeof s);
    s.mode = mode;
    s.nz = ry->nz;
    s.dz = ry->dz;
    s.dr = ry->dr;
    s.zmax = ry->zmax;
    s.c0 = ry->c0;
    s.omega = 2.0 * M_PI * ry->freq;
    s.k0 = s.omega / ry->c0;
    s.lyrw_lambda = ry->lyrw_lambda;
    s.attnf = ry->attnf;
    const double* p = b->pool + ev->off;
    s.n_zss = ev->n_zss; s.n_rss = ev->n_rss; s.n_zsb = ev->n_zsb; s.n_rsb = ev->n_rsb; s.n_bt = ev->n_bt;
    s.z_ss = p; p += s.n_zss;
    s.rp_ss = p; p += s.n_rss;
    s.cw = p; p += (size_t)s.n_rss * s.n_zss;
    s.z_sb = p; p += s.n_zsb;
    s.rp_sb = p; p += s.n_rsb;
    s.cb = p; p += (size_t)s.n_rsb * s.n_zsb;
    s.rhob = p; p += (size_t)s.n_rsb * s.n_zsb;
    s.attn = p; p += (size_t)s.n_rsb * s.n_zsb;
    s.rb = p; p += s.n_bt;
    s.zb = p;

    const int nrow = s.nz + 2;
    double* dbuf = (double*)calloc((size_t)nrow * 12, sizeof(double));
    cd* cbuf = (cd*)calloc((size_t)nrow * 5, sizeof(cd));
    if (!dbuf || !cbuf) { free(dbuf); free(cbuf); return -3; }
    s.zg = dbuf; s.cwr = dbuf + nrow; s.cbr = dbuf + 2 * nrow; s.rhobr = dbuf + 3 * nrow;
    s.attnr = dbuf + 4 * nrow; s.alpw = dbuf + 5 * nrow; s.alpb = dbuf + 6 * nrow;
    s.ksqw = dbuf + 7 * nrow; s.f1 = dbuf + 8 * nrow; s.f2 = dbuf + 9 * nrow; s.f3 = dbuf + 10 * nrow;
    s.ksqb = cbuf; s.ksq = cbuf + nrow; s.u = cbuf + 2 * nrow; s.up = cbuf + 3 * nrow; s.rs = cbuf + 4 * nrow;

    /* depth grid: numpy/cupy linspace(0, zmax, nz+2) (cupyram.py:738) */
    const double step = s.zmax / (double)(nrow - 1);
    for (int k = 0; k < nrow; ++k) s.zg[k] = (double)k * step;
    s.zg[nrow - 1] = s.zmax;

    /* initial indices (cupyram.py:571,601-608) */
    int iz0 = (int)floor(s.zb[0] / s.dz);
    if (iz0 < 1) iz0 = 1;
    if (iz0 > s.nz - 1) iz0 = s.nz - 1;
    s.iz = iz0;
    s.ss_ind = s.sb_ind = s.bt_ind = 0;

    double* tll = tll_all + ry->line_off;
    double* cpl = cpl_all + 2 * ry->line_off;
    double* tlg = (tlg_all && ry->grid_off >= 0) ? tlg_all + ry->grid_off : NULL;
    double* cpg = (cpg_all && ry->grid_off >= 0) ? cpg_all + 2 * ry->grid_off : NULL;

    /* Pade sets */
    const int np = ry->np;
    cd pd1[CR_MAX_NP], pd2[CR_MAX_NP], sp1[CR_MAX_NP], sp2[CR_MAX_NP], mp1[CR_MAX_NP],
        mp2[CR_MAX_NP];
    int rc = 0;
    if (oracle_pade(ry->freq, ry->c0, np, ry->ns, ry->dr, 2, sp1, sp2)) rc = -1;
    if (!rc && oracle_pade(ry->freq, ry->c0, np, ry->ns, ry->dr, 1, mp1, mp2)) rc = -1;
    if (rc) { free(dbuf); free(cbuf); return rc; }

    profl(&s);
    init_profiles(&s);

    /* self-starter (cupyram.py:1001-1063) */
    const double si = ry->zs / s.dz;
    const int is = (int)floor(si);
    const double dis = si - is;
    const double amp = sqrt(2.0 * M_PI / s.k0);
    s.u[is] = (1.0 - dis) * amp / (s.dz * s.alpw[is]);
    s.u[is + 1] = dis * amp / (s.dz * s.alpw[is + 1]);
    /* divide the delta by (1-X)^2: pd1 = 0, pd2 = -1.  The reference runs the
       remaining np-1 terms with pd = 0 (identity solves); REF mode does too. */
    for (int j = 0; j < CR_MAX_NP; ++j) { pd1[j] = 0.0; pd2[j] = 0.0; }
    pd2[0] = -1.0;
    const int nself = (mode == ORACLE_REF || mode == ORACLE_SIM) ? np : 1;
    const int chosen = mode == ORACLE_CHOSEN || mode == ORACLE_CHOSEN_C32 || mode == ORACLE_CHOSEN_F32 ||
                       mode == ORACLE_REFINED;
    const int refine = mode == ORACLE_REFINED;
    const int comb32 = mode == ORACLE_CHOSEN_C32 || mode == ORACLE_CHOSEN_F32, coupling32 = mode == ORACLE_CHOSEN_F32;
    if (chosen) {
        march_step_chosen(&s, 1, pd1, pd2, comb32, coupling32, refine);
        march_step_chosen(&s, 1, pd1, pd2, comb32, coupling32, refine);
        march_step_chosen(&s, np, sp1, sp2, comb32, coupling32, refine);
    } else if (mode == ORACLE_SUM) {
        march_step_sum(&s, 1, pd1, pd2);
        march_step_sum(&s, 1, pd1, pd2);
        march_step_sum(&s, np, sp1, sp2);
    } else {
        march_step(&s, nself, pd1, pd2);
        march_step(&s, nself, pd1, pd2);
        march_step(&s, np, sp1, sp2);
    }

    int mdr = 0, tlc = -1;
    double r = s.dr;
    outpt(&s, ry, r, &mdr, &tlc, tll, cpl, tlg, cpg);

    double rs_lim = ry->rs;
    for (int rn = 0; rn < ry->nr; ++rn) {
        if (updat(&s, r)) profl(&s);
        if (r >= rs_lim) {
            /* stability constraints off (cupyram.py:976-999) */
            if (oracle_pade(ry->freq, ry->c0, np, 0, ry->dr, 1, mp1, mp2)) { rc = -1; break; }
            rs_lim = INFINITY;
        }
        init_profiles(&s);
        if (chosen) march_step_chosen(&s, np, mp1, mp2, comb32, coupling32, refine);
        else if (mode == ORACLE_SUM) march_step_sum(&s, np, mp1, mp2);
        else march_step(&s, np, mp1, mp2);
        r = (double)(rn + 2) * s.dr;
        outpt(&s, ry, r, &mdr, &tlc, tll, cpl, tlg, cpg);
    }
    free(dbuf);
    free(cbuf);
    return rc;
}

typedef struct {
    const cr_batch* b;
    int mode;
    double *tll, *cpl, *tlg, *cpg;
    int next;
    int err;
    pthread_mutex_t mu;
} oracle_job;

static void* oracle_worker(void* arg) {
    oracle_job* job = (oracle_job*)arg;
    for (;;) {
        pthread_mutex_lock(&job->mu);
        const int ib = job->next++;
        pthread_mutex_unlock(&job->mu);
        if (ib >= job->b->n_rays) break;
        const int rc = run_ray(job->b, ib, job->mode, job->tll, job->cpl, job->tlg, job->cpg);
        if (rc) {
            pthread_mutex_lock(&job->mu);
            if (rc < job->err) job->err = rc;
            pthread_mutex_unlock(&job->mu);
        }
    }
    return NULL;
}

/* Run every ray of the batch on nthreads host threads (one ray per thread at
   a time).  Returns 0, or the (negative) status of the worst failing ray. */
int ram_oracle_run(const cr_batch* b, int mode, double* tll, double* cpl, double* tlg, double* cpg,
                   int nthreads) {
    oracle_job job;
    job.b = b;
    job.mode = mode;
    job.tll = tll;
    job.cpl = cpl;
    job.tlg = b->compute_grids ? tlg : NULL;
    job.cpg = b->compute_grids ? cpg : NULL;
    job.next = 0;
    job.err = 0;
    pthread_mutex_init(&job.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (nthreads > b->n_rays) nthreads = b->n_rays > 0 ? b->n_rays : 1;
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < nthreads; ++t)
        if (pthread_create(&th[started], NULL, oracle_worker, &job) == 0) ++started;
    oracle_worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&job.mu);
    return job.err;
}

/* Pade through the oracle (interleaved re/im output), for the tests. */
int ram_oracle_pade(double freq, double c0, int np, int ns, double dr, int ip, double* pd1,
                    double* pd2) {
    cd a[CR_MAX_NP], c[CR_MAX_NP];
    int rc = oracle_pade(freq, c0, np, ns, dr, ip, a, c);
    if (rc) return rc;
    for (int j = 0; j < np; ++j) {
        pd1[2 * j] = creal(a[j]); pd1[2 * j + 1] = cimag(a[j]);
        pd2[2 * j] = creal(c[j]); pd2[2 * j + 1] = cimag(c[j]);
    }
    return 0;
}
