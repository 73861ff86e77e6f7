// pade.h - Pade coefficients of the split-step operator, FP64, host and device.
//
// Computes the product-form rational approximation used by every range step:
//
//     exp(i k0 dr (sqrt(1+X) - 1)) * (1+X)^alp * (1-X)^(2 nu)
//         ~= prod_j (1 + pd1_j X) / (1 + pd2_j X)
//
// with nu = alp = 0 for the march (ip = 1) and nu = 1, alp = -1/4 for the
// self-starter (ip = 2).  Collins' construction (RAM's epade): match the
// Taylor coefficients of the operator at X = 0 (accuracy constraints), replace
// the last one or two by stability constraints at X = -3 and X = -1.5 (ns),
// solve the 2np linear system by Gaussian elimination with partial pivoting,
// then find the roots of the numerator and denominator polynomials by
// Laguerre's method with deflation; pd = -1 / root.
//
// Behaviour follows the reference's cupyram/pade.py:17-273 (same constraint
// rows, the same Laguerre schedule: 1000-iteration search to 1e-12 then a
// 5-iteration polish, a quarter-turn kick every 9 iterations, failure after
// 100 iterations).
#pragma once

#include "cplx.h"

namespace cr {

constexpr int kMaxNp = 10;
constexpr int kMaxN = 2 * kMaxNp;

enum PadeStatus { kPadeOk = 0, kPadeNoConverge = 1, kPadeBadArgs = 2 };

// One root of poly[0..deg] near *z.  err: stop when |step| <= err; nter: cap.
CR_HD int laguerre_root(const cd* poly, int deg, cd* z, double err, int nter) {
    cd d1[kMaxN + 2], d2[kMaxN + 2];
    for (int i = 0; i < deg; ++i) d1[i] = double(i + 1) * poly[i + 1];
    for (int i = 0; i + 1 < deg; ++i) d2[i] = double(i + 1) * d1[i + 1];
    cd x = *z;
    double step = INFINITY;
    int it = 0, kick = 0;
    while (step > err && it < nter - 1) {
        cd p = poly[deg - 1] + poly[deg] * x;
        for (int i = deg - 2; i >= 0; --i) p = poly[i] + x * p;
        if (cabsd(p) < 1e-20) break;
        cd p1 = d1[deg - 2] + d1[deg - 1] * x;
        for (int i = deg - 3; i >= 0; --i) p1 = d1[i] + x * p1;
        cd p2 = d2[deg - 3] + d2[deg - 2] * x;
        for (int i = deg - 4; i >= 0; --i) p2 = d2[i] + x * p2;
        const cd f = p1 / p;
        const cd g = f * f - p2 / p;
        const cd h = csqrt_p(double(deg - 1) * (double(deg) * g - f * f));
        const cd fp = f + h, fm = f - h;
        cd dx = (cabsd(fp) > cabsd(fm)) ? (-double(deg)) / fp : (-double(deg)) / fm;
        ++it;
        if (++kick == 9) {
            kick = 0;
            dx = cd{-dx.im, dx.re};  // multiply by i: leave a limit cycle
        }
        x = x + dx;
        step = cabsd(dx);
        if (it == 100) {
            *z = x;
            return kPadeNoConverge;
        }
    }
    *z = x;
    return kPadeOk;
}

// All deg roots of poly[0..deg] (poly is destroyed by deflation).
CR_HD int poly_roots(cd* poly, int deg, cd* roots) {
    if (deg == 1) {
        roots[0] = -poly[0] / poly[1];
        return kPadeOk;
    }
    for (int k = deg - 1; k >= 2; --k) {
        cd x = cd{0.0, 0.0};
        if (laguerre_root(poly, k + 1, &x, 1e-12, 1000)) return kPadeNoConverge;
        if (laguerre_root(poly, k + 1, &x, 0.0, 5)) return kPadeNoConverge;
        roots[k] = x;
        // synthetic division by (X - x), coefficients shifted down one place
        for (int i = k; i >= 0; --i) poly[i] = poly[i] + x * poly[i + 1];
        for (int i = 0; i <= k; ++i) poly[i] = poly[i + 1];
    }
    const cd disc = csqrt_p(poly[1] * poly[1] - 4.0 * (poly[0] * poly[2]));
    roots[1] = 0.5 * (-poly[1] + disc) / poly[2];
    roots[0] = 0.5 * (-poly[1] - disc) / poly[2];
    return kPadeOk;
}

// pd1[np], pd2[np] for one (freq, c0, np, ns, dr, ip).
CR_HD int pade_coefficients(double freq, double c0, int np, int ns, double dr, int ip, cd* pd1,
                            cd* pd2) {
    if (np < 1 || np > kMaxNp || !(c0 > 0.0) || !(freq > 0.0)) return kPadeBadArgs;
    const int n = 2 * np;
    const double sig = 2.0 * M_PI * freq / c0 * dr;
    const double nu = (ip == 1) ? 0.0 : 1.0;
    const double alp = (ip == 1) ? 0.0 : -0.25;

    // binomial table and (i+1)! factors
    double binom[kMaxN + 1][kMaxN + 1];
    double fct[kMaxN + 1];
    for (int i = 0; i <= n; ++i)
        for (int j = 0; j <= n; ++j) binom[i][j] = (j == 0 || j == i) ? 1.0 : 0.0;
    for (int i = 2; i <= n; ++i)
        for (int j = 1; j < i; ++j) binom[i][j] = binom[i - 1][j - 1] + binom[i - 1][j];
    fct[0] = 1.0;
    for (int i = 1; i < n; ++i) fct[i] = double(i + 1) * fct[i - 1];

    // derivatives at X = 0 of the three log-derivative pieces, then of the
    // operator itself by Leibniz' rule
    cd h1[kMaxN], h2[kMaxN], h3[kMaxN], dg[kMaxN + 1];
    h1[0] = cd{0.0, 0.5 * sig};
    h2[0] = cd{alp, 0.0};
    h3[0] = cd{-2.0 * nu, 0.0};
    double e1 = -0.5, e2 = -1.0, e3 = -1.0;
    for (int i = 1; i < n; ++i) {
        h1[i] = h1[i - 1] * e1;
        h2[i] = h2[i - 1] * e2;
        h3[i] = (-nu * e3) * h3[i - 1];
        e1 -= 1.0;
        e2 -= 1.0;
        e3 -= 1.0;
    }
    dg[0] = cd{1.0, 0.0};
    dg[1] = h1[0] + h2[0] + h3[0];
    for (int i = 1; i < n; ++i) {
        cd acc = h1[i] + h2[i] + h3[i];
        for (int j = 0; j < i; ++j) acc = acc + (binom[i][j] * (h1[j] + h2[j] + h3[j])) * dg[i - j];
        dg[i + 1] = acc;
    }

    // linear system: unknowns are the interleaved numerator / denominator
    // coefficients (even columns: numerator, odd: denominator)
    cd m[kMaxN][kMaxN + 1], rhs[kMaxN];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j <= n; ++j) m[i][j] = cd{0.0, 0.0};
        rhs[i] = dg[i + 1];
        if (2 * i <= n - 1) m[i][2 * i] = cd{fct[i], 0.0};
        for (int j = 0; j <= i; ++j)
            if (2 * j + 1 <= n - 1) m[i][2 * j + 1] = (-binom[i + 1][j + 1] * fct[j]) * dg[i - j];
    }
    const double zst[2] = {-3.0, -1.5};
    for (int c = 0; c < ns && c < 2; ++c) {
        const int row = n - 1 - c;
        rhs[row] = cd{-1.0, 0.0};
        double zp = 1.0;
        for (int j = 0; j < np; ++j) {
            zp *= zst[c];
            m[row][2 * j] = cd{zp, 0.0};
            m[row][2 * j + 1] = cd{0.0, 0.0};
        }
    }

    // Gaussian elimination, partial pivoting, row scaling by the pivot
    for (int i = 0; i < n; ++i) {
        if (i < n - 1) {
            int piv = i;
            double best = cabsd(m[i][i]);
            for (int k = i + 1; k < n; ++k) {
                const double v = cabsd(m[k][i]);
                if (v > best) {
                    best = v;
                    piv = k;
                }
            }
            if (piv != i) {
                const cd t = rhs[piv];
                rhs[piv] = rhs[i];
                rhs[i] = t;
                for (int j = i; j <= n; ++j) {
                    const cd u = m[piv][j];
                    m[piv][j] = m[i][j];
                    m[i][j] = u;
                }
            }
        }
        const cd inv = 1.0 / m[i][i];
        rhs[i] = rhs[i] * inv;
        if (i < n - 1) {
            for (int j = i + 1; j <= n; ++j) m[i][j] = m[i][j] * inv;
            for (int k = i + 1; k < n; ++k) {
                rhs[k] = rhs[k] - m[k][i] * rhs[i];
                for (int j = i + 1; j < n; ++j) m[k][j] = m[k][j] - m[k][i] * m[i][j];
            }
        }
    }
    for (int i = n - 2; i >= 0; --i)
        for (int j = i + 1; j < n; ++j) rhs[i] = rhs[i] - m[i][j] * rhs[j];

    cd poly[kMaxN + 1], roots[kMaxN + 1];
    for (int pass = 0; pass < 2; ++pass) {
        poly[0] = cd{1.0, 0.0};
        for (int j = 0; j < np; ++j) poly[j + 1] = rhs[2 * j + pass];
        if (poly_roots(poly, np, roots)) return kPadeNoConverge;
        cd* out = pass == 0 ? pd1 : pd2;
        for (int j = 0; j < np; ++j) out[j] = -1.0 / roots[j];
    }
    return kPadeOk;
}

}  // namespace cr
