"""Learned surrogate of the march, with fallback to the march.

An ensemble of small MLPs maps an environment - a 32-point sound-speed
profile, water depth at the source and at 20 km (a linear slope), bottom
sound speed, density and attenuation, frequency and source depth - to a
coarse transmission-loss field TL(r, z) on 128 ranges x 64 depths.  It is
trained only on fields this package's march computes, by this package's own
BF16 tensor-core kernels (include/cupyram_b200_mlp.h): forward and backward
passes, Adam, all on the GPU.  At inference the members' mean is served
where they agree; where their spread exceeds 1 dB the request falls back to
the march.  PyTorch only holds device buffers and streams.

Training fields and fallback fields come from the march's chosen form
(complex64 sweeps; <= 0.01 dB RMS from complex128 on every measured
workload, far below the network's own error), whose half-size shared
footprint lets the column-parallel kernel take the deep, high-frequency
columns of this distribution.  The judge reruns use the plain complex128
march.

Coarse field.  Cell (i, j) covers ranges (i, i+1] x 156.25 m and depths
(j, j+1] x D0 / 64 (D0: water depth at the source).  Its TL is
-10 log10 of the mean of |p|^2 over a 4 x 4 sub-grid of march outputs in the
cell, p = cp / sqrt(r) (cp: the march's complex pressure output), clipped to
[20, 150] dB; the incoherent cell average keeps the field learnable where
point values interfere.

Requests (seeded, numpy PCG64):
* sound speed: Munk profile c(z) (axis 1300 m) on 32 points from 0 to the
  track's deepest water, plus 4 Gaussian bumps, amplitude N(0, 3 m/s),
  centre U[0, depth], width U[50, 500] m;
* depth U[100, 4000] m at the source, slope U[-3, 3] deg (at least 20 m);
* bottom: 200 m of sediment, cb U[1500, 1900] m/s, rhob U[1.2, 2.0],
  attenuation U[0.1, 1.0] dB/lambda;
* frequency log-U[25, 400] Hz, source depth U[5, 200] m (at most 0.9 D0,
  at least 0.11 lambda: below the march's first depth cell);
* rmax 20 km; np 6 Pade terms; dr <= 6 lambda, dz <= lambda / 10 chosen so
  that the outputs fall on the 4 x 4 sub-grid of every cell.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import batch as _b
from .engine import Engine
from .workloads import munk_speed

NR_OUT, NZ_OUT, SUB = 128, 64, 4
RMAX = 20000.0
DR_CELL = RMAX / NR_OUT
N_FEAT = 40
D_IN = 128  # features padded to the kernels' tile
TL_LO, TL_HI = 20.0, 150.0
TL_MID, TL_SCALE = 90.0, 25.0
NP_PADE = 6

# ---------------------------------------------------------------------------
# kernels
# ---------------------------------------------------------------------------
_SIGS = {
    "cr_mlp_gemm": [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                    ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                    ctypes.c_int, ctypes.c_void_p],
    "cr_mlp_transpose": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                         ctypes.c_void_p],
    "cr_mlp_col_sum": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "cr_mlp_mse_grad": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_float,
                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "cr_mlp_adam": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                    ctypes.c_longlong, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                    ctypes.c_float, ctypes.c_void_p],
    "cr_mlp_to_bf16": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p],
    "cr_mlp_gemm_tc": [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                       ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
}
# Contractions with N a multiple of 256 and K of 64 run on the tcgen05 tensor
# cores (cr_mlp_gemm_tc); the others on the mma.sync kernel (cr_mlp_gemm).
USE_TCGEN05 = True
_err = None
EPI_BIAS_RELU_BF16, EPI_BIAS_F32, EPI_F32, EPI_RELU_MASK_BF16 = 0, 1, 2, 3
_mlp = None


def kernels():
    """The tensor-core kernels of the native library (no fallback)."""
    global _mlp
    if _mlp is None:
        lib = _lib.load()
        for name, args in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = args
        _mlp = lib
    return _mlp


def _ok(code, what):
    if code != 0:
        raise RuntimeError(f"{what} failed with status {code}")


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def tc_error_flag():
    """The device flag the tcgen05 GEMM sets when one of its bounded waits gives up."""
    global _err
    if _err is None:
        import torch
        _err = torch.zeros(1, dtype=torch.int32, device="cuda")
    return _err


def check_tc_flag():
    """Raise if a tcgen05 GEMM gave up one of its bounded waits (its output is then
    incomplete).  The flag is sticky: it is only ever cleared by the caller."""
    if _err is not None and int(_err.item()) != 0:
        raise RuntimeError("cr_mlp_gemm_tc: a bounded wait gave up (pipeline stalled); "
                           "the GEMM results since the flag was last cleared are invalid")


def gemm(epi, A, B, out, bias=None, mask=None, tc=None):
    """out = epilogue(A B^T); A [M, K], B [N, K] bf16 (K-contiguous rows).  tc: use the tcgen05 kernel
    (default: USE_TCGEN05 where N is a multiple of 256 and K of 64)."""
    M, K = A.shape
    N = B.shape[0]
    assert B.shape[1] == K
    if tc is None:
        tc = USE_TCGEN05 and N % 256 == 0 and K % 64 == 0
    ldm = mask.stride(0) if mask is not None else 0
    if tc:
        _ok(kernels().cr_mlp_gemm_tc(epi, _p(A), _p(B), M, N, K, A.stride(0), B.stride(0), _p(out), out.stride(0),
                                     _p(bias), _p(mask), ldm, _p(tc_error_flag()), _stream()), "cr_mlp_gemm_tc")
    else:
        _ok(kernels().cr_mlp_gemm(epi, _p(A), _p(B), M, N, K, A.stride(0), B.stride(0), _p(out), out.stride(0),
                                  _p(bias), _p(mask), ldm, _stream()), "cr_mlp_gemm")


def transpose(src, dst):
    r, c = src.shape
    _ok(kernels().cr_mlp_transpose(_p(src), src.stride(0), _p(dst), dst.stride(0), r, c, _stream()),
        "cr_mlp_transpose")


# ---------------------------------------------------------------------------
# the MLP
# ---------------------------------------------------------------------------
class MLP:
    """Fully connected ReLU network in BF16 with FP32 accumulation and FP32
    master weights; dims = [d_in, hidden..., d_out], all multiples of 128."""

    def __init__(self, dims, seed=0, device="cuda"):
        import torch
        self.dims = list(dims)
        for d in self.dims:
            if d % 128:
                raise ValueError("MLP widths must be multiples of 128")
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        self.W, self.b, self.Wb, self.WTb, self.mW, self.vW, self.mb, self.vb = ([] for _ in range(8))
        for din, dout in zip(self.dims[:-1], self.dims[1:]):
            w = (torch.randn(dout, din, generator=g) * math.sqrt(2.0 / din)).to(device)
            self.W.append(w)
            self.b.append(torch.zeros(dout, device=device))
            self.Wb.append(torch.empty(dout, din, dtype=torch.bfloat16, device=device))
            self.WTb.append(torch.empty(din, dout, dtype=torch.bfloat16, device=device))
            for lst, shape in ((self.mW, (dout, din)), (self.vW, (dout, din)), (self.mb, (dout,)), (self.vb, (dout,))):
                lst.append(torch.zeros(shape, device=device))
        self.gW = [torch.empty_like(w) for w in self.W]
        self.gb = [torch.empty_like(b) for b in self.b]
        self.t = 0
        self._sync_bf16()
        self._bufs = {}

    def _sync_bf16(self):
        for l, w in enumerate(self.W):
            _ok(kernels().cr_mlp_to_bf16(_p(w), _p(self.Wb[l]), w.numel(), _stream()), "cr_mlp_to_bf16")
            transpose(self.Wb[l], self.WTb[l])

    def _buffers(self, B):
        import torch
        if B not in self._bufs:
            dev = self.W[0].device
            H = [None] + [torch.empty(B, d, dtype=torch.bfloat16, device=dev) for d in self.dims[1:-1]]
            out = torch.empty(B, self.dims[-1], dtype=torch.float32, device=dev)
            dH = [torch.empty(B, d, dtype=torch.bfloat16, device=dev) for d in self.dims[1:]]
            T = torch.empty(max(self.dims) * B, dtype=torch.bfloat16, device=dev)
            T2 = torch.empty(max(self.dims) * B, dtype=torch.bfloat16, device=dev)
            self._bufs[B] = (H, out, dH, T, T2)
        return self._bufs[B]

    def forward(self, X):
        """X: [B, d_in] bf16 (B a multiple of 128) -> output [B, d_out] f32 (a reused buffer)."""
        B = X.shape[0]
        H, out, _, _, _ = self._buffers(B)
        H[0] = X
        L = len(self.W)
        for l in range(L):
            if l < L - 1:
                gemm(EPI_BIAS_RELU_BF16, H[l], self.Wb[l], H[l + 1], bias=self.b[l])
            else:
                gemm(EPI_BIAS_F32, H[l], self.Wb[l], out, bias=self.b[l])
        return out

    def backward(self, dout):
        """dout: [B, d_out] bf16 gradient of the loss at the output; fills gW, gb."""
        B = dout.shape[0]
        H, _, dH, T, T2 = self._buffers(B)
        L = len(self.W)
        if dH[L - 1].data_ptr() != dout.data_ptr():
            dH[L - 1].copy_(dout)
        for l in range(L - 1, -1, -1):
            d_out, d_in = self.dims[l + 1], self.dims[l]
            g = dH[l]
            # dW = g^T X: both transposed to K(=batch)-contiguous rows
            gT = T[: d_out * B].view(d_out, B)
            xT = T2[: d_in * B].view(d_in, B)
            transpose(g, gT)
            transpose(H[l], xT)
            gemm(EPI_F32, gT, xT, self.gW[l])
            _ok(kernels().cr_mlp_col_sum(_p(g), g.stride(0), B, d_out, _p(self.gb[l]), _stream()), "cr_mlp_col_sum")
            if l > 0:
                # dX = g W through the ReLU whose output was H[l]
                gemm(EPI_RELU_MASK_BF16, g, self.WTb[l], dH[l - 1], mask=H[l])

    def step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.t += 1
        k = kernels()
        for l in range(len(self.W)):
            _ok(k.cr_mlp_adam(_p(self.W[l]), _p(self.gW[l]), _p(self.mW[l]), _p(self.vW[l]), _p(self.Wb[l]),
                              self.W[l].numel(), lr, beta1, beta2, eps, self.t, weight_decay, _stream()), "adam")
            _ok(k.cr_mlp_adam(_p(self.b[l]), _p(self.gb[l]), _p(self.mb[l]), _p(self.vb[l]), None,
                              self.b[l].numel(), lr, beta1, beta2, eps, self.t, 0.0, _stream()), "adam")
            transpose(self.Wb[l], self.WTb[l])

    def grad_buffer(self, B):
        """The bf16 buffer backward() reads the output gradient from."""
        return self._buffers(B)[2][-1]


def mse_grad(pred, target, valid, count, grad, sse):
    """grad = d(mean squared error over `count` valid entries)/d pred; sse += squared errors."""
    _ok(kernels().cr_mlp_mse_grad(_p(pred), _p(target), _p(valid), pred.numel(), 1.0 / max(float(count), 1.0),
                                  _p(grad), _p(sse), _stream()), "cr_mlp_mse_grad")


# ---------------------------------------------------------------------------
# requests and their march fields
# ---------------------------------------------------------------------------
@dataclass
class Requests:
    freq: np.ndarray
    zs: np.ndarray
    d0: np.ndarray
    d1: np.ndarray
    slope: np.ndarray
    cb: np.ndarray
    rhob: np.ndarray
    attn: np.ndarray
    ssp_z: np.ndarray  # [n, 32]
    ssp_c: np.ndarray  # [n, 32]

    def __len__(self):
        return self.freq.size

    def take(self, idx):
        return Requests(*(getattr(self, f)[idx] for f in self.__dataclass_fields__))


def requests(n, seed):
    """n seeded requests of the surrogate's input distribution."""
    rng = np.random.Generator(np.random.PCG64(seed))
    d0 = rng.uniform(100.0, 4000.0, n)
    slope = rng.uniform(-3.0, 3.0, n)
    d1 = np.maximum(20.0, d0 + RMAX * np.tan(np.radians(slope)))
    cb = rng.uniform(1500.0, 1900.0, n)
    rhob = rng.uniform(1.2, 2.0, n)
    attn = rng.uniform(0.1, 1.0, n)
    freq = np.exp(rng.uniform(np.log(25.0), np.log(400.0), n))
    # below the first depth cell of the march (dz <= lambda / 10), which the
    # partial-fraction march needs
    zs = np.maximum(np.minimum(rng.uniform(5.0, 200.0, n), 0.9 * d0), 0.11 * 1500.0 / freq)
    dmax = np.maximum(d0, d1)
    ssp_z = np.linspace(0.0, 1.0, 32)[None, :] * dmax[:, None]
    amp = rng.normal(0.0, 3.0, (n, 4))
    cen = rng.uniform(0.0, 1.0, (n, 4)) * dmax[:, None]
    wid = rng.uniform(50.0, 500.0, (n, 4))
    bumps = np.sum(amp[:, None, :] * np.exp(-0.5 * ((ssp_z[:, :, None] - cen[:, None, :]) / wid[:, None, :]) ** 2),
                   axis=2)
    ssp_c = munk_speed(ssp_z) + bumps
    return Requests(freq, zs, d0, d1, slope, cb, rhob, attn, ssp_z, ssp_c)


def features(q: Requests):
    """[n, 128] float32 network inputs (40 features, zero padded)."""
    n = len(q)
    f = np.zeros((n, D_IN), np.float32)
    f[:, :32] = (q.ssp_c - 1500.0) / 30.0
    f[:, 32] = q.d0 / 2000.0 - 1.0
    f[:, 33] = q.d1 / 2000.0 - 1.0
    f[:, 34] = q.slope / 3.0
    f[:, 35] = (q.cb - 1700.0) / 200.0
    f[:, 36] = (q.rhob - 1.6) / 0.4
    f[:, 37] = (q.attn - 0.55) / 0.45
    f[:, 38] = np.log(q.freq / 100.0) / np.log(4.0)
    f[:, 39] = q.zs / 100.0 - 1.0
    return f


def march_inputs(q: Requests, compute_grids=True):
    """CuPyRAM per-ray inputs whose TL grid falls on the 4 x 4 sub-grid of every cell."""
    n = len(q)
    lam = 1500.0 / q.freq
    sub_r = DR_CELL / SUB
    sub_z = q.d0 / NZ_OUT / SUB
    ndr = np.maximum(1, np.ceil(sub_r / (NP_PADE * lam))).astype(np.int64)
    ndz = np.maximum(1, np.ceil(sub_z / (0.1 * lam))).astype(np.int64)
    dr = sub_r / ndr
    dz = sub_z / ndz
    args = [q.freq, q.zs, q.zs.copy(),
            [q.ssp_z[i] for i in range(n)], [np.array([0.0])] * n,
            [q.ssp_c[i][:, None] for i in range(n)],
            [np.array([0.0, 200.0])] * n, [np.array([0.0])] * n,
            [np.array([[q.cb[i]], [q.cb[i]]]) for i in range(n)],
            [np.array([[q.rhob[i]], [q.rhob[i]]]) for i in range(n)],
            [np.array([[q.attn[i]], [q.attn[i]]]) for i in range(n)],
            [np.array([[0.0, q.d0[i]], [RMAX, q.d1[i]]]) for i in range(n)]]
    # outputs to just below D0: 64 x 4 sub-depths, 128 x 4 sub-ranges
    kw = dict(batch_size=n, per_ray=True, rmax=RMAX + 0.25 * dr, dr=dr, dz=dz, ndr=ndr, ndz=ndz,
              np=NP_PADE, c0=np.full(n, 1500.0), zmplt=q.d0 + 0.5 * dz, compute_grids=compute_grids)
    return args, kw


def march_work(q: Requests):
    """Grid-point updates the march needs for each request (nz * nr)."""
    args, kw = march_inputs(q, compute_grids=False)
    envs, p, zs, zr, pr = _b.prepare(*args, dict(kw))
    b = _b.build_batch(envs, p, zs, zr, pr, False)
    return b.rays["nz"].astype(np.float64) * b.rays["nr"]


def coarse_tl_host(b, cpg):
    """[n, 64, 128] coarse TL of every ray of batch b from its downloaded complex-pressure grid
    (the host form of Engine.cell_tl, used to check it)."""
    n = b.n_rays
    out = np.empty((n, NZ_OUT, NR_OUT), np.float32)
    for i in range(n):
        ray = b.rays[i]
        nvz, nvr = int(ray["nvz"]), int(ray["nvr"])
        r = (np.arange(NR_OUT * SUB) + 1.0) * int(ray["ndr"]) * float(ray["dr"])
        g = cpg[ray["grid_off"]: ray["grid_off"] + nvz * nvr].reshape(nvz, nvr)[: NZ_OUT * SUB, : NR_OUT * SUB]
        p2 = (g.real ** 2 + g.imag ** 2) / r[None, :]
        m = p2.reshape(NZ_OUT, SUB, NR_OUT, SUB).mean(axis=(1, 3))
        out[i] = -10.0 * np.log10(m)
    return out


def march_tl(q: Requests, chunk=4096, precision="chosen"):
    """Coarse TL fields of the requests from the march: (tl [n, 64, 128] clipped to [20, 150] dB,
    seconds of march, grid-point updates).  The cells are reduced on the device (Engine.cell_tl)."""
    n = len(q)
    tl = np.empty((n, NZ_OUT, NR_OUT), np.float32)
    secs, work = 0.0, 0.0
    for s in range(0, n, chunk):
        sub = q.take(np.arange(s, min(n, s + chunk)))
        args, kw = march_inputs(sub)
        envs, p, zs, zr, pr = _b.prepare(*args, dict(kw))
        b = _b.build_batch(envs, p, zs, zr, pr, True)
        with Engine(b, precision=precision) as eng:
            eng.upload()
            eng.march()
            st = eng.stats()
            cells = eng.cell_tl(SUB, SUB, NZ_OUT, NR_OUT)
        if not np.all(np.isfinite(cells) | np.isposinf(cells)):
            raise RuntimeError("a request's output grid does not cover the 64 x 128 cells")
        secs += st["march_ms"] * 1e-3
        work += st["point_updates"]
        tl[s: s + len(sub)] = np.clip(np.nan_to_num(cells, posinf=TL_HI), TL_LO, TL_HI)
    return tl, secs, work


# ---------------------------------------------------------------------------
# ensemble
# ---------------------------------------------------------------------------
def default_dims(width=512, layers=4):
    return [D_IN] + [width] * (layers - 1) + [NZ_OUT * NR_OUT]


class Ensemble:
    """Members trained from different initialisations, each on its own
    bootstrap resample of the training fields (so that their spread reflects
    the data's uncertainty, not only the initialisation)."""

    def __init__(self, n_models=4, dims=None, seed=0):
        self.models = [MLP(dims or default_dims(), seed=seed + 7919 * k) for k in range(n_models)]

    def train(self, X, Y, epochs=10, batch=512, lr=1e-3, seed=0, log=None):
        """X: [n, 128] bf16, Y: [n, 8192] bf16 normalised TL (device tensors).  Returns the last-epoch losses."""
        import torch
        n = X.shape[0]
        steps_per_epoch = n // batch
        total = epochs * steps_per_epoch
        dev = X.device
        valid = torch.ones(batch * Y.shape[1], dtype=torch.uint8, device=dev)
        sse = torch.zeros(1, dtype=torch.float64, device=dev)
        losses = []
        for k, m in enumerate(self.models):
            g = torch.Generator(device=dev).manual_seed(int(seed) * 1000 + k)
            boot = torch.randint(0, n, (n,), generator=g, device=dev)
            step = 0
            for ep in range(epochs):
                perm = boot[torch.randperm(n, generator=g, device=dev)]
                sse.zero_()
                for s in range(steps_per_epoch):
                    idx = perm[s * batch:(s + 1) * batch]
                    xb = X.index_select(0, idx)
                    yb = Y.index_select(0, idx)
                    out = m.forward(xb)
                    mse_grad(out, yb, valid, valid.numel(), m.grad_buffer(batch), sse)
                    m.backward(m.grad_buffer(batch))
                    frac = step / max(total - 1, 1)
                    m.step(lr * 0.5 * (1.0 + math.cos(math.pi * frac)))
                    step += 1
                mse = float(sse.item()) / (steps_per_epoch * batch * Y.shape[1])
                check_tc_flag()
                if log:
                    log(f"model {k} epoch {ep}: rms {math.sqrt(mse) * TL_SCALE:.2f} dB")
            losses.append(math.sqrt(mse) * TL_SCALE)
        return losses

    def predict(self, X, chunk=8192, check=True):
        """TL mean and spread over the members, [n, 64, 128] each (dB, float32 device tensors).
        check: synchronise and raise if a tensor-core GEMM gave up a wait (callers that
        synchronise anyway pass False and call check_tc_flag themselves)."""
        import torch
        n = X.shape[0]
        mean = torch.empty(n, NZ_OUT * NR_OUT, device=X.device)
        spread = torch.empty(n, NZ_OUT * NR_OUT, device=X.device)
        for s in range(0, n, chunk):
            xb = X[s: s + chunk]
            preds = torch.stack([m.forward(xb).clone() for m in self.models]) * TL_SCALE + TL_MID
            preds.clamp_(TL_LO, TL_HI)
            mean[s: s + chunk] = preds.mean(0)
            spread[s: s + chunk] = preds.std(0, unbiased=False)
        if check:
            check_tc_flag()
        return mean.view(n, NZ_OUT, NR_OUT), spread.view(n, NZ_OUT, NR_OUT)


def to_device_inputs(feat, tl=None, device="cuda"):
    """Network inputs (and normalised targets) as bf16 device tensors, rows padded to 128."""
    import torch
    n = feat.shape[0]
    npad = (n + 127) // 128 * 128
    X = torch.zeros(npad, D_IN, dtype=torch.bfloat16, device=device)
    X[:n] = torch.from_numpy(feat).to(device).to(torch.bfloat16)
    if tl is None:
        return X
    Y = torch.from_numpy(((tl.reshape(n, -1) - TL_MID) / TL_SCALE).astype(np.float32)).to(device).to(torch.bfloat16)
    return X, Y


@dataclass
class Served:
    tl: np.ndarray          # [n, 64, 128] served fields
    fallback: np.ndarray    # [n] bool: served by the march
    spread_db: np.ndarray   # [n] RMS over cells of the members' standard deviation
    t_net: float            # seconds of network inference (device events)
    t_march: float          # seconds of fallback marches
    march_work: float       # grid-point updates of the fallback marches
    t_wall: float           # host wall clock of the whole call (features in, fields out)


def serve(ens: Ensemble, q: Requests, threshold_db=1.0):
    """Answer requests with the ensemble, falling back to the march where its spread exceeds the threshold."""
    import torch
    tw = time.perf_counter()
    n = len(q)
    X = to_device_inputs(features(q))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    mean, spread = ens.predict(X, check=False)
    e1.record()
    torch.cuda.synchronize()
    check_tc_flag()
    t_net = e0.elapsed_time(e1) * 1e-3
    srms = torch.sqrt((spread[:n] ** 2).mean(dim=(1, 2))).cpu().numpy()
    tl = mean[:n].cpu().numpy()
    fb = srms > threshold_db
    t_march = work = 0.0
    if fb.any():
        idx = np.nonzero(fb)[0]
        tl_fb, t_march, work = march_tl(q.take(idx))
        tl[idx] = tl_fb
    return Served(tl, fb, srms, t_net, t_march, work, time.perf_counter() - tw)


# ---------------------------------------------------------------------------
# the whole pipeline (bench.py --config surrogate)
# ---------------------------------------------------------------------------
def pipeline(n_train=200_000, n_infer=65_536, judge_frac=0.01, epochs=60, batch=512, lr=1e-3, n_models=4,
             width=512, layers=4, threshold_db=1.0, seed=2024, log=print):
    """Generate the training fields with the march, train the ensemble with the
    tensor-core kernels, serve n_infer seeded requests with fallback, and judge
    the served fields against march reruns of a seeded judge_frac sample."""
    import torch
    t0 = time.perf_counter()
    q_train = requests(n_train, seed)
    tl_train, t_gen, w_gen = march_tl(q_train)
    t_gen_wall = time.perf_counter() - t0
    log(f"training fields: {n_train} marches, {w_gen:.3e} updates, {t_gen:.1f} s of march ({t_gen_wall:.1f} s wall)")
    X, Y = to_device_inputs(features(q_train), tl_train)
    del tl_train
    ens = Ensemble(n_models, default_dims(width, layers), seed=seed)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    rms = ens.train(X[:n_train - n_train % batch], Y[:n_train - n_train % batch], epochs=epochs, batch=batch, lr=lr,
                    seed=seed, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    log(f"training: {n_models} members x {epochs} epochs in {t_train:.1f} s, last-epoch rms {rms}")
    del X, Y
    q = requests(n_infer, seed + 1)
    served = serve(ens, q, threshold_db)
    # the march's cost for every request, at the rate the march ran on the training fields
    rate = w_gen / t_gen
    w_all = float(march_work(q).sum())
    t_ram_all = w_all / rate
    t_served = served.t_net + served.t_march
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    idx = np.sort(rng.choice(n_infer, size=max(1, int(round(judge_frac * n_infer))), replace=False))
    tl_judge, _, _ = march_tl(q.take(idx), precision="plain")
    err = served.tl[idx] - tl_judge
    req_rms = np.sqrt(np.mean(err.reshape(len(idx), -1) ** 2, axis=1))
    # the same over the cells the march puts below 100 dB (the precision study's mask)
    lit = (tl_judge < 100.0).reshape(len(idx), -1)
    e2 = np.where(lit, err.reshape(len(idx), -1) ** 2, 0.0)
    req_rms_lit = np.sqrt(e2.sum(axis=1) / np.maximum(lit.sum(axis=1), 1))
    net_idx = ~served.fallback[idx]
    res = {
        "n_train": n_train, "n_infer": n_infer, "n_judge": int(len(idx)), "members": n_models,
        "layers": layers, "width": width, "epochs": epochs, "batch": batch,
        "train_rms_db": rms, "train_seconds": t_train,
        "gen_seconds_march": t_gen, "gen_updates": w_gen, "march_updates_per_s": rate,
        "fallback_rate": float(served.fallback.mean()), "spread_threshold_db": threshold_db,
        "spread_db_median": float(np.median(served.spread_db)),
        "net_seconds": served.t_net, "fallback_march_seconds": served.t_march,
        "served_requests_per_s": n_infer / t_served,
        "march_requests_per_s": n_infer / t_ram_all,
        "speedup_vs_march": t_ram_all / t_served,
        "net_only_speedup_vs_march": t_ram_all / max(served.t_net, 1e-12),
        "equivalent_updates_per_s": w_all / t_served,
        "equivalent_updates_per_s_wall": w_all / served.t_wall,
        "serve_wall_seconds": served.t_wall,
        "judge_rms_db_mean": float(req_rms.mean()),
        "judge_rms_db_net_served": float(req_rms[net_idx].mean()) if net_idx.any() else None,
        "judge_within_1db": float(np.mean(req_rms <= 1.0)),
        "judge_rms_db_mean_tl_below_100": float(req_rms_lit.mean()),
        "judge_within_1db_tl_below_100": float(np.mean(req_rms_lit <= 1.0)),
        "judge_rms_db_fallback_served": float(req_rms[~net_idx].mean()) if (~net_idx).any() else None,
        "judge_spread_db_net_served": float(served.spread_db[idx][net_idx].mean()) if net_idx.any() else None,
        "gemm": "tcgen05" if USE_TCGEN05 else "mma.sync",
        "judge_max_abs_db": float(np.abs(err).max()),
    }
    log(str(res))
    return res
