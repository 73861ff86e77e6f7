"""Seeded synthetic workloads (the benchmark configurations' inputs).

Every generator returns ``(args, kwargs)`` for ``CuPyRAM(*args, **kwargs)``.
Inputs come from ``numpy.random.Generator(PCG64(seed))``; nothing is read
from disk.

* ``pekeris``      - Pekeris waveguide, one ray (50 Hz, 100 m water over a
                     1700 m/s bottom, rmax 10 km, dr 2 m, dz 0.25 m, np 8)
* ``munk_batch``   - deep-water Munk batch: per-ray frequency and source depth,
                     range-dependent sound speed (Munk + Gaussian-correlated
                     perturbations every 5 km), flat 5000 m bottom
* ``wedge_batch``  - uneven wedge batch: per-ray slope, bottom, frequency,
                     range and Pade order; dr = lambda/4, dz = lambda/8
"""
import numpy as np


def munk_speed(z, axis=1300.0, eps=0.00737, c_axis=1500.0):
    """Canonical Munk profile c(z) = c1 (1 + eps (eta - 1 + exp(-eta))), eta = 2(z - z1)/z1."""
    eta = 2.0 * (np.asarray(z) - axis) / axis
    return c_axis * (1.0 + eps * (eta - 1.0 + np.exp(-eta)))


def pekeris():
    args = [50.0, 50.0, 50.0,
            np.array([0.0, 100.0]), np.array([0.0]), np.array([[1500.0], [1500.0]]),
            np.array([0.0, 200.0]), np.array([0.0]),
            np.array([[1700.0], [1700.0]]), np.array([[1.5], [1.5]]), np.array([[0.5], [0.5]]),
            np.array([[0.0, 100.0], [10000.0, 100.0]])]
    kw = dict(rmax=10000.0, dr=2.0, dz=0.25, np=8, ns=1, lyrw=10, ndr=1, ndz=4, c0=1500.0)
    return args, kw


def _correlated_perturbations(rng, z, n, sigma, corr_len):
    """n Gaussian profiles on grid z with covariance sigma^2 exp(-dz^2 / 2L^2)."""
    dzm = z[:, None] - z[None, :]
    cov = sigma * sigma * np.exp(-0.5 * (dzm / corr_len) ** 2)
    w, v = np.linalg.eigh(cov)
    fac = v * np.sqrt(np.clip(w, 0.0, None))[None, :]
    return (fac @ rng.standard_normal((z.size, n))).T  # [n, nz]


def munk_batch(n_rays=4096, seed=2024, depth=5000.0, rmax=50000.0, dr=25.0, dz=1.0, np_pade=6,
               zr=500.0, update=5000.0, sigma=2.0, corr_len=1000.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    freq = rng.uniform(50.0, 200.0, n_rays)
    zs = rng.uniform(50.0, 1000.0, n_rays)
    z = np.arange(0.0, depth + 1e-9, 10.0)
    rp = np.arange(0.0, rmax, update)
    base = munk_speed(z)
    pert = _correlated_perturbations(rng, z, n_rays * rp.size, sigma, corr_len)
    cw = (base[None, None, :] + pert.reshape(n_rays, rp.size, z.size)).transpose(0, 2, 1)
    cw = np.ascontiguousarray(cw)  # [ray, depth, range]
    args = [freq, zs, np.full(n_rays, zr),
            np.tile(z, (n_rays, 1)), np.tile(rp, (n_rays, 1)), cw,
            np.tile(np.array([0.0, 200.0]), (n_rays, 1)), np.zeros((n_rays, 1)),
            np.full((n_rays, 2, 1), 1600.0), np.full((n_rays, 2, 1), 1.5), np.full((n_rays, 2, 1), 0.5),
            np.tile(np.array([[0.0, depth], [rmax, depth]]), (n_rays, 1, 1))]
    kw = dict(batch_size=n_rays, per_ray=True, rmax=rmax, dr=dr, dz=dz, np=np_pade,
              compute_grids=False)
    return [list(a) if isinstance(a, np.ndarray) and a.ndim > 1 else a for a in args], kw


def wedge_batch(n_rays=10000, seed=7, c_water=1500.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    z0 = rng.uniform(50.0, 400.0, n_rays)
    z1 = rng.uniform(50.0, 400.0, n_rays)
    cb = rng.uniform(1550.0, 1800.0, n_rays)
    rho = rng.uniform(1.3, 2.0, n_rays)
    at = rng.uniform(0.2, 1.0, n_rays)
    freq = np.exp(rng.uniform(np.log(25.0), np.log(500.0), n_rays))
    rmax = rng.uniform(5000.0, 40000.0, n_rays)
    npp = rng.integers(4, 9, n_rays)
    lam = c_water / freq
    zmx = np.maximum(z0, z1)
    zs = np.minimum(0.5 * np.minimum(z0, z1), 30.0)
    args = [freq, zs, zs.copy(),
            [np.array([0.0, zmx[i]]) for i in range(n_rays)], [np.array([0.0])] * n_rays,
            [np.array([[c_water], [c_water]])] * n_rays,
            [np.array([0.0, 100.0])] * n_rays, [np.array([0.0])] * n_rays,
            [np.array([[cb[i]], [cb[i]]]) for i in range(n_rays)],
            [np.array([[rho[i]], [rho[i]]]) for i in range(n_rays)],
            [np.array([[at[i]], [at[i]]]) for i in range(n_rays)],
            [np.array([[0.0, z0[i]], [rmax[i], z1[i]]]) for i in range(n_rays)]]
    kw = dict(batch_size=n_rays, per_ray=True, rmax=rmax, dr=lam / 4.0, dz=lam / 8.0, np=npp,
              c0=np.full(n_rays, c_water), compute_grids=False)
    return args, kw


def build(args, kw, compute_grids=None):
    """Host pipeline only: the packed Batch the engine consumes."""
    from . import batch as _b
    kw = dict(kw)
    if compute_grids is not None:
        kw["compute_grids"] = compute_grids
    envs, p, zs, zr, per_ray = _b.prepare(*args, kw)
    return _b.build_batch(envs, p, zs, zr, per_ray, kw.get("compute_grids", True))
