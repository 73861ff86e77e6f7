"""The learned surrogate: tensor-core kernels against numpy and the MLP oracle,
the device cell reduction against the host one, and what a trained ensemble
gains over the method without it."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def _bf(a):
    import torch
    return torch.from_numpy(np.asarray(a, np.float32)).cuda().to(torch.bfloat16)


def test_gemm_epilogues_vs_numpy(cuda_device):
    import torch
    from cupyram_b200 import surrogate as S
    rng = np.random.default_rng(0)
    M, N, K = 256, 384, 96
    A, B = rng.normal(size=(M, K)), rng.normal(size=(N, K))
    bias = rng.normal(size=N)
    mask = rng.normal(size=(M, N))
    ref = MO.to_bf16(A) @ MO.to_bf16(B).T
    Ab, Bb, mb = _bf(A), _bf(B), _bf(mask)
    bt = torch.from_numpy(bias.astype(np.float32)).cuda()
    scale = np.abs(ref).max()
    out = torch.empty(M, N, device="cuda")
    S.gemm(S.EPI_F32, Ab, Bb, out)
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-5 * scale * K
    S.gemm(S.EPI_BIAS_F32, Ab, Bb, out, bias=bt)
    assert np.abs(out.cpu().numpy() - (ref + bias.astype(np.float32))).max() < 1e-5 * scale * K
    ob = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    S.gemm(S.EPI_BIAS_RELU_BF16, Ab, Bb, ob, bias=bt)
    want = np.maximum(ref + bias.astype(np.float32), 0)
    assert np.abs(ob.float().cpu().numpy() - want).max() <= 2 ** -7 * np.abs(want).max() + 1e-3
    S.gemm(S.EPI_RELU_MASK_BF16, Ab, Bb, ob, mask=mb)
    want = np.where(MO.to_bf16(mask) > 0, ref, 0.0)
    assert np.abs(ob.float().cpu().numpy() - want).max() <= 2 ** -7 * scale + 1e-3
    with pytest.raises(RuntimeError):
        S.gemm(S.EPI_F32, _bf(A[:100]), Bb, out)  # M not a multiple of 128


@pytest.mark.parametrize("feed,M,N,K", [("cp", 256, 512, 192), ("tma", 256, 512, 192), ("tma", 384, 768, 640),
                                         ("persistent", 256, 512, 192), ("persistent", 384, 768, 640),
                                         ("persistent", 2560, 38 * 256, 128)])
def test_gemm_tcgen05_vs_numpy(cuda_device, monkeypatch, feed, M, N, K):
    """The tcgen05 kernels (accumulator in tensor memory) on every epilogue, and their wait
    flag clear: operands fed by per-thread cp.async (CUPYRAM_B200_GEMM=cp), by the tensor
    memory accelerator one block per CTA (the default), or by the persistent kernel
    (=persistent: one CTA per SM, a TMA producer warp, an MMA warp and four epilogue warps
    overlapping two tensor-memory accumulators).  K of 192 and 640 run a ring through 3 and 10 tiles;
    20 x 38 blocks give every CTA of the persistent kernel several blocks."""
    import torch
    from cupyram_b200 import surrogate as S
    monkeypatch.setenv("CUPYRAM_B200_GEMM", {"cp": "cp", "tma": "", "persistent": "persistent"}[feed])
    rng = np.random.default_rng(4)
    A, B = rng.normal(size=(M, K)), rng.normal(size=(N, K))
    bias = rng.normal(size=N)
    mask = rng.normal(size=(M, N))
    ref = MO.to_bf16(A) @ MO.to_bf16(B).T
    Ab, Bb, mb = _bf(A), _bf(B), _bf(mask)
    bt = torch.from_numpy(bias.astype(np.float32)).cuda()
    scale = np.abs(ref).max()
    S.tc_error_flag().zero_()
    out = torch.empty(M, N, device="cuda")
    S.gemm(S.EPI_F32, Ab, Bb, out, tc=True)
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-5 * scale * K
    S.gemm(S.EPI_BIAS_F32, Ab, Bb, out, bias=bt, tc=True)
    assert np.abs(out.cpu().numpy() - (ref + bias.astype(np.float32))).max() < 1e-5 * scale * K
    ob = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    S.gemm(S.EPI_BIAS_RELU_BF16, Ab, Bb, ob, bias=bt, tc=True)
    want = np.maximum(ref + bias.astype(np.float32), 0)
    assert np.abs(ob.float().cpu().numpy() - want).max() <= 2 ** -7 * np.abs(want).max() + 1e-3
    S.gemm(S.EPI_RELU_MASK_BF16, Ab, Bb, ob, mask=mb, tc=True)
    want = np.where(MO.to_bf16(mask) > 0, ref, 0.0)
    assert np.abs(ob.float().cpu().numpy() - want).max() <= 2 ** -7 * scale + 1e-3
    assert int(S.tc_error_flag().item()) == 0


def test_mlp_gradients_vs_oracle(cuda_device):
    """One forward/backward of the kernels against the oracle's float64 backward
    with the same bfloat16 storage points."""
    import torch
    from cupyram_b200 import surrogate as S
    rng = np.random.default_rng(1)
    dims, B = [128, 128, 128, 128, 256], 128
    m = S.MLP(dims, seed=5)
    X = rng.normal(size=(B, dims[0]))
    Y = rng.normal(size=(B, dims[-1]))
    Xb, Yb = _bf(X), _bf(Y)
    valid = torch.ones(B * dims[-1], dtype=torch.uint8, device="cuda")
    sse = torch.zeros(1, dtype=torch.float64, device="cuda")
    out = m.forward(Xb)
    S.mse_grad(out, Yb, valid, valid.numel(), m.grad_buffer(B), sse)
    m.backward(m.grad_buffer(B))
    torch.cuda.synchronize()
    W = [w.cpu().numpy().astype(np.float64) for w in m.W]
    b = [v.cpu().numpy().astype(np.float64) for v in m.b]
    loss, dW, db = MO.loss_and_grads(X, Y, W, b, bf16=True)
    assert abs(float(sse.item()) / (B * dims[-1]) - loss) < 1e-3 * loss
    for l in range(len(W)):
        g = m.gW[l].cpu().numpy()
        assert np.linalg.norm(g - dW[l]) < 2e-2 * np.linalg.norm(dW[l]), l
        gb = m.gb[l].cpu().numpy()
        assert np.linalg.norm(gb - db[l]) < 2e-2 * np.linalg.norm(db[l]) + 1e-6, l


def test_cell_tl_matches_host_reduction(cuda_device):
    from cupyram_b200 import batch as Bt, surrogate as S
    from cupyram_b200.engine import Engine
    q = S.requests(6, seed=3)
    args, kw = S.march_inputs(q)
    envs, p, zs, zr, pr = Bt.prepare(*args, dict(kw))
    b = Bt.build_batch(envs, p, zs, zr, pr, True)
    with Engine(b) as eng:
        out = eng.run()
        dev = eng.cell_tl(S.SUB, S.SUB, S.NZ_OUT, S.NR_OUT)
    host = S.coarse_tl_host(b, out["cpg"])
    fin = np.isfinite(host)
    assert fin.mean() > 0.99
    assert np.abs(dev[fin] - host[fin]).max() < 1e-3


def test_trained_ensemble_beats_the_method_without_it(cuda_device):
    """A small ensemble trained on march fields predicts held-out fields far
    better than the best field-independent guess (the training mean), and
    answers a request much faster than the march."""
    import time
    import torch
    from cupyram_b200 import surrogate as S
    q_tr, q_te = S.requests(1536, seed=11), S.requests(256, seed=12)
    tl_tr, t_march, _ = S.march_tl(q_tr)
    tl_te, _, _ = S.march_tl(q_te)
    X, Y = S.to_device_inputs(S.features(q_tr), tl_tr)
    ens = S.Ensemble(2, [128, 256, 256, 256, 8192], seed=3)
    ens.train(X, Y, epochs=40, batch=128, lr=2e-3, seed=3)
    Xt = S.to_device_inputs(S.features(q_te))
    ens.predict(Xt)  # first call allocates the members' buffers
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mean, spread = ens.predict(Xt)
    torch.cuda.synchronize()
    t_net = time.perf_counter() - t0
    pred = mean[: len(q_te)].cpu().numpy()
    rms_net = np.sqrt(np.mean((pred - tl_te) ** 2))
    rms_mean = np.sqrt(np.mean((tl_tr.mean(axis=0)[None] - tl_te) ** 2))
    assert rms_net < 0.8 * rms_mean, (rms_net, rms_mean)
    assert t_net / len(q_te) < 0.1 * t_march / len(q_tr), (t_net, t_march)
