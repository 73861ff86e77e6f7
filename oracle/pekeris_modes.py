"""Normal-mode transmission loss of the Pekeris waveguide (test infrastructure).

An isovelocity fluid layer (sound speed c1, density rho1, depth D) under a
pressure-release surface, over a fluid half-space (c2, rho2, attenuation in
dB per wavelength), point source at zs, time dependence exp(-i w t).  The
trapped modes are the standard ones (e.g. Jensen, Kuperman, Porter and
Schmidt, Computational Ocean Acoustics, ch. 2 and 5):

    psi(z) = sin(kz z),                   0 <= z <= D
           = sin(kz D) exp(-g (z - D)),    z > D
    kz = sqrt(k1^2 - kr^2),  g = sqrt(kr^2 - k2^2)  (Re g > 0)

with the interface conditions (continuity of p and p_z / rho) giving

    F(kr) = rho2 kz cos(kz D) + rho1 g sin(kz D) = 0,

normalisation N = (D/2 - sin(2 kz D) / (4 kz)) / rho1 + sin(kz D)^2 / (2 g rho2)
(no conjugates: the modes of the lossy problem are complex), and the field

    p(r, z) = i / (4 rho(zs)) sum_m psi_m(zs) psi_m(z) H0^(1)(kr_m r) / N_m,
    TL = -20 log10(4 pi |p|)   (re 1 m from the source).

The roots are found on the lossless problem (real kr between k2 and k1) and
followed to the lossy k2 by Newton's method.  The continuous spectrum is left
out, so the field is meant for ranges of many water depths.  Used to check
that the march (through the CPU restatement and the engine) reproduces the
Pekeris solution away from interference nulls.
"""
import numpy as np
from scipy.optimize import brentq
from scipy.special import hankel1

DB_PER_NEPER_LAMBDA = 40.0 * np.pi * np.log10(np.e)  # dB/lambda -> imaginary part of k / Re k


def _F(kr, k1, k2, D, rho1, rho2):
    kz = np.sqrt(k1 * k1 - kr * kr + 0j)
    g = np.sqrt(kr * kr - k2 * k2 + 0j)
    if g.real < 0:
        g = -g
    return rho2 * kz * np.cos(kz * D) + rho1 * g * np.sin(kz * D)


def modes(freq, D, c1, c2, rho1, rho2, attn_db_lambda):
    """Complex horizontal wavenumbers of the trapped modes."""
    w = 2.0 * np.pi * freq
    k1 = w / c1
    k2r = w / c2
    k2 = k2r * (1.0 + 1j * attn_db_lambda / DB_PER_NEPER_LAMBDA)
    # lossless roots: sign changes of F on a fine real grid in (k2, k1)
    grid = np.linspace(k2r * (1 + 1e-9), k1 * (1 - 1e-9), 20001)
    vals = np.array([_F(x, k1, k2r, D, rho1, rho2).real for x in grid])
    roots = []
    for a, b, fa, fb in zip(grid[:-1], grid[1:], vals[:-1], vals[1:]):
        if fa == 0.0 or fa * fb < 0.0:
            roots.append(brentq(lambda x: _F(x, k1, k2r, D, rho1, rho2).real, a, b, xtol=1e-15))
    out = []
    for k0 in roots:
        kr = complex(k0)
        for _ in range(60):  # Newton on the lossy problem, numerical derivative
            h = 1e-7 * abs(kr)
            f = _F(kr, k1, k2, D, rho1, rho2)
            df = (_F(kr + h, k1, k2, D, rho1, rho2) - _F(kr - h, k1, k2, D, rho1, rho2)) / (2 * h)
            step = f / df
            kr -= step
            if abs(step) < 1e-15 * abs(kr):
                break
        out.append(kr)
    return np.array(out), k1, k2


def tl(freq, D, c1, c2, rho1, rho2, attn_db_lambda, zs, z, r):
    """Transmission loss (dB) at depth z (< D or > D) and ranges r (m)."""
    krs, k1, k2 = modes(freq, D, c1, c2, rho1, rho2, attn_db_lambda)
    r = np.asarray(r, dtype=np.float64)

    def psi(kr, zz):
        kz = np.sqrt(k1 * k1 - kr * kr + 0j)
        g = np.sqrt(kr * kr - k2 * k2 + 0j)
        if g.real < 0:
            g = -g
        if zz <= D:
            return np.sin(kz * zz), kz, g
        return np.sin(kz * D) * np.exp(-g * (zz - D)), kz, g

    p = np.zeros_like(r, dtype=np.complex128)
    rho_s = rho1 if zs <= D else rho2
    for kr in krs:
        ps, kz, g = psi(kr, zs)
        pz, _, _ = psi(kr, z)
        N = (D / 2.0 - np.sin(2.0 * kz * D) / (4.0 * kz)) / rho1 + np.sin(kz * D) ** 2 / (2.0 * g * rho2)
        p += ps * pz / N * hankel1(0, kr * r)
    p *= 1j / (4.0 * rho_s)
    return -20.0 * np.log10(4.0 * np.pi * np.abs(p))
