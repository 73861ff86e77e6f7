// cplx.h - minimal complex arithmetic usable on host and device.
//
// The engine stores complex values as CUDA double2 / float2 (re, im) so that
// loads and stores are single 16-byte / 8-byte vector accesses.  These helpers
// keep the arithmetic explicit (no std::complex in device code, no hidden
// temporaries) and let the same Pade code compile for host and device.
#pragma once

#include <cmath>
#include <cuda_runtime.h>

#ifdef __CUDACC__
#define CR_HD __host__ __device__ __forceinline__
#else
#define CR_HD inline
#endif

namespace cr {

struct cd {
    double re, im;
};

// Products and sums are rounded one by one on the device as on the host
// (no fused multiply-add contraction), so that the device's Pade solves take
// the host's path through the Laguerre iterations.
#ifdef __CUDA_ARCH__
#define CR_MUL(a, b) __dmul_rn((a), (b))
#define CR_ADD(a, b) __dadd_rn((a), (b))
#define CR_SUB(a, b) __dsub_rn((a), (b))
#else
#define CR_MUL(a, b) ((a) * (b))
#define CR_ADD(a, b) ((a) + (b))
#define CR_SUB(a, b) ((a) - (b))
#endif

CR_HD cd mk(double re, double im = 0.0) { return cd{re, im}; }
CR_HD cd operator+(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }
CR_HD cd operator-(cd a, cd b) { return cd{a.re - b.re, a.im - b.im}; }
CR_HD cd operator-(cd a) { return cd{-a.re, -a.im}; }
CR_HD cd operator*(cd a, cd b) {
    return cd{CR_SUB(CR_MUL(a.re, b.re), CR_MUL(a.im, b.im)), CR_ADD(CR_MUL(a.re, b.im), CR_MUL(a.im, b.re))};
}
CR_HD cd operator*(double s, cd a) { return cd{s * a.re, s * a.im}; }
CR_HD cd operator*(cd a, double s) { return cd{s * a.re, s * a.im}; }
CR_HD cd operator+(cd a, double s) { return cd{a.re + s, a.im}; }
CR_HD cd operator+(double s, cd a) { return cd{a.re + s, a.im}; }
CR_HD double cabs2(cd a) { return CR_ADD(CR_MUL(a.re, a.re), CR_MUL(a.im, a.im)); }
CR_HD double cabsd(cd a) { return hypot(a.re, a.im); }

// a / b with Smith's scaling (robust when |b| spans many decades, as the
// polynomial values inside Laguerre iteration do).
CR_HD cd operator/(cd a, cd b) {
    if (fabs(b.re) >= fabs(b.im)) {
        const double t = b.im / b.re;
        const double d = CR_ADD(b.re, CR_MUL(b.im, t));
        return cd{CR_ADD(a.re, CR_MUL(a.im, t)) / d, CR_SUB(a.im, CR_MUL(a.re, t)) / d};
    }
    const double t = b.re / b.im;
    const double d = CR_ADD(CR_MUL(b.re, t), b.im);
    return cd{CR_ADD(CR_MUL(a.re, t), a.im) / d, CR_SUB(CR_MUL(a.im, t), a.re) / d};
}
CR_HD cd operator/(double s, cd b) { return cd{s, 0.0} / b; }

// principal square root
CR_HD cd csqrt_p(cd z) {
    if (z.re == 0.0 && z.im == 0.0) return cd{0.0, 0.0};
    const double m = hypot(z.re, z.im);
    const double t = sqrt(0.5 * (fabs(z.re) + m));
    if (z.re >= 0.0) return cd{t, z.im / (2.0 * t)};
    return cd{fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

}  // namespace cr
