"""Host input pipeline: reference-style inputs -> packed per-ray batch description.

This is the host half of ``CuPyRAM.__init__`` / ``CuPyRAM.setup`` of the
reference (clapeyre/cupyram ``cupyram/cupyram.py``):

* ``normalize_to_batch``  - ragged lists -> NaN-padded batches (``:56-120``)
* ``valid_slice``         - strip NaN padding (``:123-174``)
* ``check_inputs``        - per-ray validation, ``ValueError`` on bad input (``:382-458``)
* ``derive_params``       - c0, lambda, dr, dz, zmplt, rmax, ns, rs, lyrw (``:460-526``)
* ``build_batch``         - bathymetry extension, seabed offset, grid sizes,
                            output sizes and the packed cr_ray / cr_env / pool
                            arrays of the C ABI (``:528-726``)

Two semantics are supported:

* ``shared`` (the reference's): every calculation is an (environment,
  frequency) pair of the cross product, and all share one grid whose nz,
  dz, dr and absorbing layer come from the maximum frequency and the
  deepest seabed of the batch.
* ``per_ray`` (an extension for uneven batches): calculation i pairs
  environment i with frequency i; source / receiver depth, dr, dz, np and
  rmax may differ per ray and every ray gets its own grid (lambda_i = c0_i /
  f_i).

Deliberate differences from the reference (its defects, not its maths):
range-dependence flags are taken per ray instead of from ray 0
(``cupyram.py:437-442``), and the layer width uses each calculation's own
lambda only in ``per_ray`` mode (shared mode keeps the reference's
max-frequency lambda).
"""
from dataclasses import dataclass, field

import numpy as np

from ._lib import ENV_DTYPE, MAX_NP, RAY_DTYPE

ATTNF = 10.0  # attenuation at the bottom of the absorbing layer (cupyram.py:774)


# ---------------------------------------------------------------------------
# normalisation and NaN padding
# ---------------------------------------------------------------------------
def normalize_to_batch(x, batch_size, name):
    """List -> stacked (or NaN-padded) batch; single array -> tiled batch."""
    if isinstance(x, list):
        if len(x) != batch_size:
            raise ValueError(f"{name}: list length {len(x)} != batch_size {batch_size}")
        arrays = [np.asarray(a) for a in x]
        shapes = {a.shape for a in arrays}
        if len(shapes) == 1:
            return np.stack(arrays, axis=0)
        ndim = arrays[0].ndim
        if any(a.ndim != ndim for a in arrays):
            raise ValueError(f"{name}: list entries differ in dimensionality")
        max_shape = tuple(max(a.shape[i] for a in arrays) for i in range(ndim))
        dtype = arrays[0].dtype
        if np.issubdtype(dtype, np.integer) or dtype == bool:
            dtype = np.float64
        out = np.full((batch_size,) + max_shape, np.nan, dtype=dtype)
        for i, a in enumerate(arrays):
            out[(i,) + tuple(slice(0, s) for s in a.shape)] = a
        return out
    a = np.asarray(x)
    if a.ndim == 0:
        return np.full(batch_size, a)
    return np.tile(a, (batch_size,) + (1,) * a.ndim)


def valid_slice(arr):
    """The non-NaN leading part of a padded 1-D or 2-D array (and its length)."""
    arr = np.asarray(arr)
    if arr.ndim == 1:
        nan = np.isnan(arr)
        if not nan.any():
            return arr, len(arr)
        n = int(np.argmax(nan))
        return (arr[:n], n) if n > 0 else (arr, len(arr))
    if arr.ndim == 2:
        nan = np.isnan(arr)
        rows = int(np.sum(~np.all(nan, axis=1)))
        cols = int(np.sum(~np.all(nan, axis=0)))
        if rows == arr.shape[0] and cols == arr.shape[1]:
            return arr, arr.shape[0]
        return arr[:rows, :cols], rows
    flat = arr.reshape(arr.shape[0], -1)
    bad = np.any(np.isnan(flat), axis=1)
    if not bad.any():
        return arr, len(arr)
    n = int(np.argmax(bad))
    return (arr[:n], n) if n > 0 else (arr, len(arr))


# ---------------------------------------------------------------------------
# per-ray environment record (valid parts only)
# ---------------------------------------------------------------------------
@dataclass
class EnvRecord:
    z_ss: np.ndarray
    rp_ss: np.ndarray
    cw: np.ndarray      # [n_zss, n_rss] (reference layout)
    z_sb: np.ndarray    # relative to the deepest water-profile point (input form)
    rp_sb: np.ndarray
    cb: np.ndarray
    rhob: np.ndarray
    attn: np.ndarray
    rbzb: np.ndarray    # [n_bt, 2]


def check_inputs(n_env, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb):
    """Validate every environment; returns the list of EnvRecord (cupyram.py:382-434).

    zs / zr are arrays of length n_env (the same value repeated in shared mode).
    A batch of stacked (possibly NaN-padded) arrays is checked with whole-batch
    array operations; any other batch, and any batch that fails a check, goes
    through the per-environment loop, which raises the error.
    """
    envs = check_batch(n_env, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb)
    if envs is not None:
        return envs
    return check_each(n_env, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb)


def _lead_len(a):
    """valid_slice's length for every row of a [B, n] array: up to the first NaN
    (the whole row when the first entry is NaN, which then fails the checks)."""
    nan = np.isnan(a)
    k = np.argmax(nan, axis=1)
    return np.where(nan.any(axis=1) & (k > 0), k, a.shape[1])


def _table_dims(a):
    """valid_slice's rows and columns for every [n, m] entry of a [B, n, m] array:
    the counts of rows and of columns that are not entirely NaN."""
    nan = np.isnan(a)
    return (~nan.all(axis=2)).sum(axis=1), (~nan.all(axis=1)).sum(axis=1)


def check_batch(n_env, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb):
    """The checks of check_each over a whole batch at once, or None.

    Applies when the profiles are [n_env, n] arrays and the tables
    [n_env, n, m] arrays (as normalize_to_batch stacks or NaN-pads them).
    Every environment's valid part is found as valid_slice finds it; the
    records are views of those parts.  Returns None when the layout does
    not apply or any check fails (the loop then reports the first failing
    environment).
    """
    vecs = [np.asarray(a) for a in (z_ss, rp_ss, z_sb, rp_sb)]
    tabs = [np.asarray(a) for a in (cw, cb, rhob, attn, rbzb)]
    if any(a.ndim != 2 or a.shape[0] != n_env or a.shape[1] == 0 for a in vecs) or \
            any(a.ndim != 3 or a.shape[0] != n_env or 0 in a.shape[1:] for a in tabs):
        return None
    if any(not (np.issubdtype(a.dtype, np.floating) or np.issubdtype(a.dtype, np.integer)) for a in vecs + tabs):
        return None
    zss, rps, zsb, rpb = (a.astype(np.float64, copy=False) for a in vecs)
    cwb, cbb, rhb, atb, bt = (a.astype(np.float64, copy=False) for a in tabs)
    n_zss, n_rss, n_zsb, n_rsb = (_lead_len(a) for a in (zss, rps, zsb, rpb))
    (cw_r, cw_c), (cb_r, cb_c), (rh_r, rh_c), (at_r, at_c), (bt_r, bt_c) = (
        _table_dims(a) for a in (cwb, cbb, rhb, atb, bt))
    if not (np.array_equal(cw_r, n_zss) and np.array_equal(cw_c, n_rss)):
        return None
    for r, c in ((cb_r, cb_c), (rh_r, rh_c), (at_r, at_c)):
        if not (np.array_equal(r, n_zsb) and np.array_equal(c, n_rsb)):
            return None
    if np.any(bt_c != 2) or np.any(bt_r < 1):
        return None

    def vmask(a, n):
        return np.arange(a.shape[1])[None, :] < n[:, None]

    def tmask(a, r, c):
        return (np.arange(a.shape[1])[None, :, None] < r[:, None, None]) & \
               (np.arange(a.shape[2])[None, None, :] < c[:, None, None])

    masks = [vmask(zss, n_zss), vmask(rps, n_rss), vmask(zsb, n_zsb), vmask(rpb, n_rsb),
             tmask(cwb, cw_r, cw_c), tmask(cbb, cb_r, cb_c), tmask(rhb, rh_r, rh_c), tmask(atb, at_r, at_c),
             tmask(bt, bt_r, bt_c)]
    for a, m in zip((zss, rps, zsb, rpb, cwb, cbb, rhb, atb, bt), masks):
        if not np.all(np.isfinite(a) | ~m):
            return None
    zs = np.asarray(zs, dtype=np.float64)
    zr = np.asarray(zr, dtype=np.float64)
    top, bottom = zss[:, 0], zss[np.arange(n_env), n_zss - 1]
    ok = (top <= zs) & (zs <= bottom) & (top <= zr) & (zr <= bottom)
    ok &= np.where(masks[8][:, :, 1], bt[:, :, 1], -np.inf).max(axis=1) <= bottom
    if not np.all(ok):
        return None
    if np.any((cwb <= 0) & masks[4]) or np.any((cbb <= 0) & masks[5]) or np.any((rhb <= 0) & masks[6]):
        return None
    return [EnvRecord(zss[b, :n_zss[b]], rps[b, :n_rss[b]], cwb[b, :cw_r[b], :cw_c[b]], zsb[b, :n_zsb[b]],
                      rpb[b, :n_rsb[b]], cbb[b, :cb_r[b], :cb_c[b]], rhb[b, :rh_r[b], :rh_c[b]],
                      atb[b, :at_r[b], :at_c[b]], bt[b, :bt_r[b], :bt_c[b]]) for b in range(n_env)]


def check_each(n_env, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb):
    """check_inputs one environment at a time (NaN-padded or ragged batches)."""
    envs = []
    for b in range(n_env):
        zss = valid_slice(z_ss[b])[0].astype(np.float64)
        rps = valid_slice(rp_ss[b])[0].astype(np.float64)
        cwb = valid_slice(np.atleast_2d(cw[b]))[0].astype(np.float64)
        zsb = valid_slice(z_sb[b])[0].astype(np.float64)
        rpb = valid_slice(rp_sb[b])[0].astype(np.float64)
        cbb = valid_slice(np.atleast_2d(cb[b]))[0].astype(np.float64)
        rhb = valid_slice(np.atleast_2d(rhob[b]))[0].astype(np.float64)
        atb = valid_slice(np.atleast_2d(attn[b]))[0].astype(np.float64)
        bt = valid_slice(np.atleast_2d(rbzb[b]))[0].astype(np.float64)
        if not (zss[0] <= zs[b] <= zss[-1]):
            raise ValueError(f"Ray {b}: Source depth {zs[b]}m outside range [{zss[0]}, {zss[-1]}]m")
        if not (zss[0] <= zr[b] <= zss[-1]):
            raise ValueError(f"Ray {b}: Receiver depth {zr[b]}m outside range [{zss[0]}, {zss[-1]}]m")
        if cwb.shape != (zss.size, rps.size):
            raise ValueError(f"Ray {b}: z_ss ({zss.size}), rp_ss ({rps.size}), cw {cwb.shape} inconsistent")
        for prof, name in ((cbb, "cb"), (rhb, "rhob"), (atb, "attn")):
            if prof.shape != (zsb.size, rpb.size):
                raise ValueError(f"Ray {b}: z_sb ({zsb.size}), rp_sb ({rpb.size}), {name} {prof.shape} inconsistent")
        if bt.ndim != 2 or bt.shape[1] != 2:
            raise ValueError(f"Ray {b}: rbzb must have two columns (range, depth)")
        if bt[:, 1].max() > zss[-1]:
            raise ValueError(f"Ray {b}: Max bathy ({bt[:, 1].max()}m) > max SSP depth ({zss[-1]}m)")
        for arr, name in ((zss, "z_ss"), (rps, "rp_ss"), (zsb, "z_sb"), (rpb, "rp_sb"), (cwb, "cw"),
                          (cbb, "cb"), (rhb, "rhob"), (atb, "attn"), (bt, "rbzb")):
            if not np.all(np.isfinite(arr)):
                raise ValueError(f"Ray {b}: {name} contains non-finite values inside its valid part")
        if np.any(cwb <= 0) or np.any(cbb <= 0) or np.any(rhb <= 0):
            raise ValueError(f"Ray {b}: sound speeds and densities must be positive")
        envs.append(EnvRecord(zss, rps, cwb, zsb, rpb, cbb, rhb, atb, bt))
    return envs


# ---------------------------------------------------------------------------
# parameters, grid and packing
# ---------------------------------------------------------------------------
@dataclass
class Params:
    np_pade: np.ndarray     # [n_calc] int
    c0_env: np.ndarray      # [n_env]
    c0_report: object       # 'c0' of the results dict
    freqs: np.ndarray       # [n_freq] shared, or [n_calc] per-ray
    dr: np.ndarray          # [n_calc]
    dz: np.ndarray          # [n_calc]
    ndr: int
    ndz: int
    zmplt: np.ndarray       # [n_calc]
    rmax: np.ndarray        # [n_calc] (before truncation to whole output steps)
    ns: int
    rs: np.ndarray          # [n_calc]
    lyrw: float
    lam: np.ndarray         # [n_calc] wavelength used for the layer width
    ident: object = 0


def _per_calc(v, n, name, dtype=np.float64):
    a = np.asarray(v, dtype=dtype)
    if a.ndim == 0:
        return np.full(n, a, dtype=dtype)
    a = a.reshape(-1)
    if a.size != n:
        raise ValueError(f"{name}: expected a scalar or {n} values, got {a.size}")
    return a


@dataclass
class Batch:
    """Packed description ready for cr_create (plus what run() needs to reshape)."""
    rays: np.ndarray
    envs: np.ndarray
    pool: np.ndarray
    line_len: int
    grid_len: int
    compute_grids: bool
    n_env: int
    n_freq: int
    per_ray: bool
    nz: np.ndarray
    nvr: np.ndarray
    nvz: np.ndarray
    zmax: np.ndarray
    vr: list = field(default_factory=list)
    vz: list = field(default_factory=list)

    @property
    def n_rays(self):
        return len(self.rays)

    @property
    def point_updates(self):
        return float(np.sum(self.rays["nz"].astype(np.float64) * self.rays["nr"]))


def derive_params(envs, freqs, per_ray, kwargs, np_default=8, dzf=0.1, ndr_default=1,
                  ndz_default=1, ns_default=1, lyrw_default=20, id_default=0):
    """c0, lambda, dr, dz, zmplt, rmax, ns, rs (cupyram.py:460-526).

    In shared mode every array is the same value repeated over the
    n_env * n_freq calculations; in per-ray mode calculation i is env i.
    """
    n_env = len(envs)
    n_freq = 1 if per_ray else len(freqs)
    n_calc = n_env * n_freq
    npp = _per_calc(kwargs.get("np", np_default), n_env if per_ray else 1, "np", np.int64)
    if np.any(npp < 1) or np.any(npp > MAX_NP):
        raise ValueError(f"np must be in 1..{MAX_NP}")
    if "c0" in kwargs:
        c0_env = _per_calc(kwargs["c0"], n_env, "c0")
        c0_report = kwargs["c0"]
    else:
        c0_env = np.array([np.nanmean(e.cw[:, 0]) for e in envs])
        c0_report = float(np.mean(c0_env))
    if per_ray:
        f = np.asarray(freqs, dtype=np.float64)
        lam = c0_env / f
        np_calc = npp if npp.size == n_env else np.full(n_env, int(npp[0]))
        dr = _per_calc(kwargs["dr"], n_env, "dr") if "dr" in kwargs else np_calc * 1500.0 / f
        dz = _per_calc(kwargs["dz"], n_env, "dz") if "dz" in kwargs else dzf * 1500.0 / f
        zmplt = (_per_calc(kwargs["zmplt"], n_env, "zmplt") if "zmplt" in kwargs
                 else np.array([e.rbzb[:, 1].max() for e in envs]))
        rmax = (_per_calc(kwargs["rmax"], n_env, "rmax") if "rmax" in kwargs
                else np.array([max(e.rp_ss.max(), e.rp_sb.max(), e.rbzb[:, 0].max()) for e in envs]))
    else:
        fmax = float(np.max(freqs))
        c0_shared = float(np.mean(c0_env)) if "c0" not in kwargs else float(np.mean(c0_env))
        np_calc = np.full(n_calc, int(npp[0]))
        lam = np.full(n_calc, c0_shared / fmax)
        dr = np.full(n_calc, float(kwargs.get("dr", int(npp[0]) * 1500.0 / fmax)))
        dz = np.full(n_calc, float(kwargs.get("dz", dzf * 1500.0 / fmax)))
        zmplt = np.full(n_calc, float(kwargs.get("zmplt", max(e.rbzb[:, 1].max() for e in envs))))
        rmax_default = max(max(e.rp_ss.max(), e.rp_sb.max(), e.rbzb[:, 0].max()) for e in envs)
        rmax = np.full(n_calc, float(kwargs.get("rmax", rmax_default)))
    if np.any(dr <= 0) or np.any(dz <= 0):
        raise ValueError("dr and dz must be positive")
    if per_ray and (np.ndim(kwargs.get("ndr", 1)) or np.ndim(kwargs.get("ndz", 1))):
        # per-ray output decimation (an extension of per_ray mode)
        ndr = _per_calc(kwargs.get("ndr", ndr_default), n_env, "ndr", np.int64)
        ndz = _per_calc(kwargs.get("ndz", ndz_default), n_env, "ndz", np.int64)
        if np.any(ndr < 1) or np.any(ndz < 1):
            raise ValueError("ndr and ndz must be >= 1")
    else:
        ndr = int(kwargs.get("ndr", ndr_default))
        ndz = int(kwargs.get("ndz", ndz_default))
        if ndr < 1 or ndz < 1:
            raise ValueError("ndr and ndz must be >= 1")
    ns = int(kwargs.get("ns", ns_default))
    if ns not in (0, 1, 2):
        raise ValueError("ns must be 0, 1 or 2")
    rs = _per_calc(kwargs["rs"], n_calc, "rs") if "rs" in kwargs else rmax + dr
    lyrw = float(kwargs.get("lyrw", lyrw_default))
    return Params(np_calc, c0_env, c0_report, np.asarray(freqs, dtype=np.float64), dr, dz, ndr, ndz,
                  zmplt, rmax, ns, rs, lyrw, lam, kwargs.get("id", id_default))


def pack_pool(envs, zsb_abs, bt_ext):
    """cr_env records and the float64 pool; per environment the sections
    z_ss, rp_ss, cw[n_rss][n_zss], z_sb (absolute), rp_sb, cb, rhob, attn
    (each [n_rsb][n_zsb]), rb, zb, laid end to end from record.off.

    Equal-shaped environments (the extended bathymetry may still differ by
    its last point) are packed by one scatter; others one at a time.
    """
    n_env = len(envs)
    env_arr = np.zeros(n_env, dtype=ENV_DTYPE)
    if n_env == 0:
        return env_arr, np.zeros(1)
    shape0 = tuple(getattr(envs[0], f).shape for f in ("z_ss", "rp_ss", "z_sb", "rp_sb", "rbzb"))
    uniform = all(tuple(getattr(e, f).shape for f in ("z_ss", "rp_ss", "z_sb", "rp_sb", "rbzb")) == shape0
                  for e in envs)
    uniform = uniform and all(b.shape[0] - e.rbzb.shape[0] in (0, 1) for e, b in zip(envs, bt_ext))
    if not uniform:
        return _pack_each(envs, zsb_abs, bt_ext, env_arr)
    front = np.concatenate([np.stack([e.z_ss for e in envs]), np.stack([e.rp_ss for e in envs]),
                            np.stack([e.cw.T.reshape(-1) for e in envs]), np.stack(zsb_abs),
                            np.stack([e.rp_sb for e in envs]), np.stack([e.cb.T.reshape(-1) for e in envs]),
                            np.stack([e.rhob.T.reshape(-1) for e in envs]),
                            np.stack([e.attn.T.reshape(-1) for e in envs])], axis=1).astype(np.float64, copy=False)
    n_front = front.shape[1]
    bt = np.stack([e.rbzb for e in envs]).astype(np.float64, copy=False)  # [n_env, n_bt, 2]
    n_bt = bt.shape[1]
    ext = np.array([b.shape[0] > n_bt for b in bt_ext])
    n_bt_k = n_bt + ext.astype(np.int64)
    size = n_front + 2 * n_bt_k
    off = np.cumsum(size) - size
    pool = np.empty(int(size.sum()))
    pool[off[:, None] + np.arange(n_front)] = front
    rb0 = off + n_front
    zb0 = rb0 + n_bt_k
    pool[rb0[:, None] + np.arange(n_bt)] = bt[:, :, 0]
    pool[zb0[:, None] + np.arange(n_bt)] = bt[:, :, 1]
    if ext.any():
        last = np.array([b[-1] for b, x in zip(bt_ext, ext) if x])
        pool[rb0[ext] + n_bt] = last[:, 0]
        pool[zb0[ext] + n_bt] = last[:, 1]
    env_arr["n_zss"], env_arr["n_rss"] = shape0[0][0], shape0[1][0]
    env_arr["n_zsb"], env_arr["n_rsb"] = shape0[2][0], shape0[3][0]
    env_arr["n_bt"] = n_bt_k
    env_arr["off"] = off
    return env_arr, pool


def _pack_each(envs, zsb_abs, bt_ext, env_arr):
    chunks = []
    off = 0
    for k, e in enumerate(envs):
        parts = [e.z_ss, e.rp_ss, e.cw.T.reshape(-1), zsb_abs[k], e.rp_sb, e.cb.T.reshape(-1),
                 e.rhob.T.reshape(-1), e.attn.T.reshape(-1), bt_ext[k][:, 0], bt_ext[k][:, 1]]
        env_arr[k] = (e.z_ss.size, e.rp_ss.size, zsb_abs[k].size, e.rp_sb.size, bt_ext[k].shape[0], 0, off)
        for q in parts:
            chunks.append(np.ascontiguousarray(q, dtype=np.float64))
            off += q.size
    return env_arr, np.concatenate(chunks)


def output_axis(n, d, nd):
    """Output ranges (or depths) (1..n_b) * d_b * nd_b of every calculation b, one array each."""
    n = np.asarray(n, dtype=np.int64)
    d = np.asarray(d, dtype=np.float64)
    nd = np.asarray(nd)
    out = [None] * n.size
    order = np.argsort(n, kind="stable")
    for idx in np.split(order, np.flatnonzero(np.diff(n[order])) + 1):
        if idx.size == 0:
            continue
        rows = np.arange(1, n[idx[0]] + 1)[None, :] * d[idx, None] * nd[idx, None]
        for j, b in enumerate(idx):
            out[b] = rows[j]
    return out


def build_batch(envs, p: Params, zs, zr, per_ray, compute_grids):
    """Grid sizes, output sizes and the packed C-ABI arrays (cupyram.py:528-726).

    zs, zr: per-environment arrays.
    """
    n_env = len(envs)
    n_freq = 1 if per_ray else len(p.freqs)
    n_calc = n_env * n_freq
    # seabed depths are given relative to the deepest water-profile point
    zsb_abs = [e.z_sb + e.z_ss[-1] for e in envs]
    # bathymetry extended to rmax (the value before output truncation)
    bt_ext = []
    for k, e in enumerate(envs):
        r_ext = p.rmax[k * n_freq]
        bt = e.rbzb
        if bt[-1, 0] < r_ext:
            bt = np.vstack([bt, [r_ext, bt[-1, 1]]])
        bt_ext.append(bt)
    if per_ray:
        zmax = np.array([zsb_abs[k].max() for k in range(n_env)]) + p.lyrw * p.lam
    else:
        zmax = np.full(n_calc, max(z.max() for z in zsb_abs) + p.lyrw * p.lam[0])
    nz = (np.floor(zmax / p.dz) - 1).astype(np.int64)
    nzplt = np.floor(p.zmplt / p.dz).astype(np.int64)
    nvr = np.floor(p.rmax / (p.dr * p.ndr)).astype(np.int64)
    rmax_t = nvr * p.dr * p.ndr
    nvz = (nzplt // p.ndz).astype(np.int64)
    nr = (np.round(rmax_t / p.dr) - 1).astype(np.int64)
    if np.any(nz < 3):
        raise ValueError("depth grid has fewer than 3 interior points; reduce dz")
    if np.any(nvr < 1) or np.any(nr < 0):
        raise ValueError("rmax must cover at least one output range step")

    env_arr, pool = pack_pool(envs, zsb_abs, bt_ext)

    e_of = np.arange(n_calc) // n_freq
    zs = np.asarray(zs, dtype=np.float64)
    zr = np.asarray(zr, dtype=np.float64)
    rays = np.zeros(n_calc, dtype=RAY_DTYPE)
    rays["freq"] = p.freqs if per_ray else np.tile(p.freqs, n_env)
    rays["c0"] = p.c0_env[e_of]
    rays["zs"] = zs[e_of]
    rays["zr"] = zr[e_of]
    rays["dz"] = p.dz
    rays["dr"] = p.dr
    rays["zmax"] = zmax
    rays["lyrw_lambda"] = p.lyrw * p.lam
    rays["attnf"] = ATTNF
    rays["rs"] = p.rs
    rays["nz"] = nz
    rays["nr"] = nr
    rays["np"] = p.np_pade
    rays["ns"] = p.ns
    ndr_b = np.broadcast_to(p.ndr, (n_calc,))
    ndz_b = np.broadcast_to(p.ndz, (n_calc,))
    rays["ndr"] = ndr_b
    rays["ndz"] = ndz_b
    rays["nvr"] = nvr
    rays["nvz"] = nvz
    rays["env"] = e_of
    ends = np.cumsum(nvr)
    rays["line_off"] = ends - nvr
    line_off = int(ends[-1]) if n_calc else 0
    if compute_grids:
        cells = nvz * nvr
        ends = np.cumsum(cells)
        rays["grid_off"] = ends - cells
        grid_off = int(ends[-1]) if n_calc else 0
    else:
        rays["grid_off"] = -1
        grid_off = 0
    below = np.floor(zs[e_of] / p.dz) + 1 > nz
    if below.any():
        raise ValueError(f"Ray {int(np.argmax(below))}: source depth below the computational grid")
    vr = output_axis(nvr, p.dr, ndr_b)
    vz = output_axis(nvz, p.dz, ndz_b)
    return Batch(rays, env_arr, pool, line_off, grid_off, bool(compute_grids), n_env, n_freq,
                 per_ray, nz, nvr, nvz, zmax, vr, vz)


def prepare(freq, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb, kwargs):
    """Full host pipeline; returns (envs, Params, zs_env, zr_env, per_ray)."""
    per_ray = bool(kwargs.get("per_ray", False))
    batch_size = int(kwargs.get("batch_size", 1))
    if batch_size < 1:
        raise ValueError("batch_size must be >= 1")
    if np.isscalar(freq):
        freqs = np.array([freq], dtype=np.float64)
    else:
        freqs = np.array(freq, dtype=np.float64).reshape(-1)
    if freqs.size == 0 or np.any(~np.isfinite(freqs)) or np.any(freqs <= 0):
        raise ValueError("freq must be positive")
    if per_ray:
        freqs = _per_calc(freqs if freqs.size > 1 else freqs[0], batch_size, "freq")
    zs_env = _per_calc(zs, batch_size, "zs")
    zr_env = _per_calc(zr, batch_size, "zr")
    if not per_ray and (np.ndim(zs) or np.ndim(zr)):
        raise ValueError("zs and zr must be scalars unless per_ray=True")
    norm = [normalize_to_batch(x, batch_size, n) for x, n in
            ((z_ss, "z_ss"), (rp_ss, "rp_ss"), (cw, "cw"), (z_sb, "z_sb"), (rp_sb, "rp_sb"),
             (cb, "cb"), (rhob, "rhob"), (attn, "attn"), (rbzb, "rbzb"))]
    envs = check_inputs(batch_size, zs_env, zr_env, *norm)
    p = derive_params(envs, freqs, per_ray, kwargs)
    return envs, p, zs_env, zr_env, per_ray
