"""The learned surrogate (needs a GPU): the tensor-core GEMM against torch, the network's loss and
gradients against a float64 CPU restatement (tests/mlp_reference.py), the element-wise kernels,
training on sweep-generated data, the ensemble gate, the inverse fit, and what the network gains
over plain Monte Carlo at equal cost."""

from __future__ import annotations

import math
import time

import numpy as np
import pytest

import tissuemc_b200 as tmc
from mlp_reference import bf16, forward_backward

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 128), (4096, 66, 512), (4096, 512, 512),
                                   (513, 1000, 192)])
def test_tensor_core_gemm_matches_fp32_reference(M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    D = tmc.gemm_bf16(A, B, bias)
    ref = A.double() @ B.double().T + bias.double()
    rel = ((D.double() - ref).abs().max() / ref.abs().max()).item()
    assert rel < 2e-6, rel  # FP32 accumulation of exact BF16 products


@pytest.mark.parametrize("M,N,K,splits", [(512, 512, 4096, 8), (130, 72, 192, 3), (128, 128, 64, 1)])
def test_split_k_weight_gradient_product(M, N, K, splits):
    """D = A B^T with K cut into splits (the weight-gradient shape: long K, small M x N)."""
    import ctypes

    from tissuemc_b200 import surrogate as S

    g = torch.Generator(device="cuda").manual_seed(K + splits)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    D = torch.empty(M, N, device="cuda")
    work = torch.empty(splits * M * N, device="cuda")
    S._call("tmc_b200_nn_matmul_f32_splitk", S._p(A), S._p(B), S._p(D), S._p(work), M, N, K, splits,
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    ref = A.double() @ B.double().T
    assert ((D.double() - ref).abs().max() / ref.abs().max()).item() < 2e-6
    with pytest.raises(tmc.ConfigError, match="split-K"):
        S._call("tmc_b200_nn_matmul_f32_splitk", S._p(A), S._p(B), S._p(D), S._p(work), M, N, K, 5,
                ctypes.c_void_p(0))


def test_gemm_rejects_k_not_multiple_of_64():
    A = torch.zeros(128, 32, device="cuda", dtype=torch.bfloat16)
    with pytest.raises(tmc.ConfigError, match="multiple of 64"):
        tmc.gemm_bf16(A, A)


def test_a_wait_that_runs_out_reports_device_timeout_and_leaves_the_device_usable():
    """The GEMM kernel's producer is told to issue no loads, so the MMA issuer's bounded wait (4096
    polls) runs out with nothing outstanding: the kernel skips its epilogue, frees its tensor memory
    and raises its status word, which the host turns into TMC_DEVICE_TIMEOUT. A normal product on
    the same device afterwards is still exact."""
    rc, msg = tmc.probe_wait_timeout(4096)
    assert rc == tmc.DEVICE_TIMEOUT, (rc, msg)
    assert "gave up" in msg
    rc, msg = tmc.probe_wait_timeout(4096)  # and again: the status word was cleared
    assert rc == tmc.DEVICE_TIMEOUT, (rc, msg)
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn(256, 128, device="cuda", generator=g).bfloat16()
    B = torch.randn(192, 128, device="cuda", generator=g).bfloat16()
    D = tmc.gemm_bf16(A, B)
    ref = A.double() @ B.double().T
    assert ((D.double() - ref).abs().max() / ref.abs().max()).item() < 2e-6


def _member_numpy(m):
    Ws = [bf16(w.cpu().numpy()) for w in m.W]
    bs = [b.cpu().numpy().astype(np.float64) for b in m.b]
    return Ws, bs


def test_gradients_match_the_float64_cpu_restatement():
    from tissuemc_b200 import surrogate as S

    B = 128
    m = S.Member(B, seed=3)
    rng = np.random.default_rng(0)
    for b in m.b:  # non-zero biases exercise the bias paths
        b.copy_(torch.from_numpy(rng.normal(0, 0.1, b.shape[0]).astype(np.float32)))
    Xn = np.zeros((B, S.K_IN), np.float32)
    Xn[:, :S.N_FEAT] = rng.normal(size=(B, S.N_FEAT))
    Y = rng.normal(size=(B, S.N_OUT)).astype(np.float32)
    X = torch.from_numpy(Xn).cuda().bfloat16()
    Yd = torch.from_numpy(Y).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    scale = 1.0 / (B * S.N_OUT)
    m.forward(X, B, stream)
    m.backward(X, Yd, stream, scale)
    torch.cuda.synchronize()
    Ws, bs = _member_numpy(m)
    loss, gW, gb, pred = forward_backward(bf16(Xn), Ws, bs, Y.astype(np.float64), S.N_OUT, scale)
    assert math.isclose(m.loss.item(), loss, rel_tol=1e-4)
    # a BF16 activation may round to the neighbouring value when the FP32 sums differ in the last
    # bit, so outputs agree to a fraction of a BF16 step, not bit for bit
    zp = m.Z[-1].cpu().numpy()
    assert np.abs(zp - pred).max() <= 1e-2 * np.abs(pred).max()
    for li in range(len(Ws)):
        g_gpu, g_ref = m.gW[li].cpu().numpy(), gW[li]
        assert np.abs(g_gpu - g_ref).max() <= 2e-2 * np.abs(g_ref).max() + 1e-9, li
        assert np.abs(m.gb[li].cpu().numpy() - gb[li]).max() <= 2e-2 * np.abs(gb[li]).max() + 1e-9, li
        # gradients of the zero-padded inputs and outputs stay exactly zero
    assert not m.gW[0][:, S.N_FEAT:].any() and not m.gW[-1][S.N_OUT:].any()


def test_adam_transpose_and_colsum_kernels():
    from tissuemc_b200 import surrogate as S

    rows, cols = 96, 200
    w = torch.randn(rows, cols, device="cuda")
    g = torch.randn(rows, cols, device="cuda")
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    wb = torch.empty(rows, cols, dtype=torch.bfloat16, device="cuda")
    wt = torch.empty(cols, rows, dtype=torch.bfloat16, device="cuda")
    w0 = w.clone()
    s = torch.cuda.current_stream().cuda_stream
    import ctypes

    S._call("tmc_b200_nn_adam", S._p(w), S._p(g), S._p(m), S._p(v), rows, cols, ctypes.c_float(0.01), S._p(None),
            ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), ctypes.c_float(0.0), S._p(wb),
            S._p(wt), S._p(None), ctypes.c_float(0.0), ctypes.c_void_p(s))
    torch.cuda.synchronize()
    mi = 0.1 * g
    vi = 0.001 * g * g
    ref = w0 - 0.01 * mi / (vi.sqrt() + 1e-8)
    assert torch.allclose(w, ref, rtol=1e-5, atol=1e-6)
    assert torch.equal(wb, w.bfloat16()) and torch.equal(wt, w.bfloat16().t())
    x = torch.randn(300, 70, device="cuda").bfloat16()
    y = torch.empty(70, 300, dtype=torch.bfloat16, device="cuda")
    S._call("tmc_b200_nn_transpose", S._p(x), S._p(y), 300, 70, ctypes.c_void_p(s))
    work = torch.empty(tmc.lib().tmc_b200_nn_colsum_work(70), device="cuda")
    db = torch.empty(70, device="cuda")
    S._call("tmc_b200_nn_colsum", S._p(x), S._p(db), 300, 70, S._p(work), ctypes.c_void_p(s))
    torch.cuda.synchronize()
    assert torch.equal(y, x.t())
    assert torch.allclose(db, x.float().sum(0), rtol=1e-5, atol=1e-4)


def test_step_size_from_device_memory_and_fused_averaging_give_the_same_bits():
    """Adam reading its step size from device memory, with the Polyak average fused, equals Adam
    with the step size as an argument followed by the separate averaging pass, bit for bit; the
    bias-gradient column sum is the same on every call (no atomics)."""
    import ctypes

    from tissuemc_b200 import surrogate as S

    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rows, cols = 130, 257
    gen = torch.Generator(device="cuda").manual_seed(9)
    w = torch.randn(rows, cols, device="cuda", generator=gen)
    g = torch.randn(rows, cols, device="cuda", generator=gen)
    m = 0.1 * torch.randn(rows, cols, device="cuda", generator=gen)
    v = torch.rand(rows, cols, device="cuda", generator=gen)
    avg = torch.randn(rows, cols, device="cuda", generator=gen)
    lr_dev = torch.tensor([3e-3], device="cuda")
    a = [t.clone() for t in (w, m, v, avg)]
    b = [t.clone() for t in (w, m, v, avg)]
    wb_a, wb_b = (torch.empty(rows, cols, dtype=torch.bfloat16, device="cuda") for _ in range(2))
    S._call("tmc_b200_nn_adam", S._p(a[0]), S._p(g), S._p(a[1]), S._p(a[2]), rows, cols, ctypes.c_float(0.0),
            S._p(lr_dev), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), ctypes.c_float(1e-4),
            S._p(wb_a), S._p(None), S._p(a[3]), ctypes.c_float(0.999), s)
    S._call("tmc_b200_nn_adam", S._p(b[0]), S._p(g), S._p(b[1]), S._p(b[2]), rows, cols, ctypes.c_float(3e-3),
            S._p(None), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), ctypes.c_float(1e-4),
            S._p(wb_b), S._p(None), S._p(None), ctypes.c_float(0.0), s)
    S._call("tmc_b200_nn_ema", S._p(b[0]), S._p(b[3]), rows * cols, ctypes.c_float(0.999), s)
    torch.cuda.synchronize()
    for x, y in zip(a, b, strict=True):
        assert torch.equal(x, y)
    assert torch.equal(wb_a, wb_b)
    assert not torch.equal(a[3], avg)  # the average moved

    dz = torch.randn(4096, 512, device="cuda", generator=gen).bfloat16()
    work = torch.empty(tmc.lib().tmc_b200_nn_colsum_work(512), device="cuda")
    sums = []
    for _ in range(3):
        db = torch.empty(512, device="cuda")
        S._call("tmc_b200_nn_colsum", S._p(dz), S._p(db), 4096, 512, S._p(work), s)
        sums.append(db)
    torch.cuda.synchronize()
    assert torch.equal(sums[0], sums[1]) and torch.equal(sums[0], sums[2])
    assert torch.allclose(sums[0], dz.double().sum(0).float(), rtol=1e-4, atol=1e-3)


def test_many_tensor_adam_equals_one_call_per_tensor():
    """One launch over a table of parameter tensors (ragged sizes, some without bf16 copies or
    averages) gives the same bits as one adam call per tensor."""
    import ctypes

    from tissuemc_b200 import surrogate as S

    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gen = torch.Generator(device="cuda").manual_seed(11)
    shapes = [(130, 257), (1, 513), (64, 64), (3, 1)]
    sets = []
    for _ in range(2):
        torch.cuda.manual_seed(0)
        sets.append([dict(w=torch.randn(r, c, device="cuda", generator=gen.manual_seed(7 + k)),
                          g=torch.randn(r, c, device="cuda", generator=gen.manual_seed(70 + k)),
                          m=torch.zeros(r, c, device="cuda"), v=torch.full((r, c), 0.5, device="cuda"),
                          avg=torch.ones(r, c, device="cuda") if k % 2 == 0 else None,
                          wb=torch.empty(r, c, dtype=torch.bfloat16, device="cuda") if k != 1 else None,
                          wt=torch.empty(c, r, dtype=torch.bfloat16, device="cuda") if k != 1 else None)
                     for k, (r, c) in enumerate(shapes)])
    lr_dev = torch.tensor([2e-3], device="cuda")
    for k, ((r, c), t) in enumerate(zip(shapes, sets[0], strict=True)):
        S._call("tmc_b200_nn_adam", S._p(t["w"]), S._p(t["g"]), S._p(t["m"]), S._p(t["v"]), r, c, ctypes.c_float(0.0),
                S._p(lr_dev), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8),
                ctypes.c_float(1e-4 * k), S._p(t["wb"]), S._p(t["wt"]), S._p(t["avg"]), ctypes.c_float(0.99), s)
    rows = [tmc.CAdamTensor(t["w"].data_ptr(), t["g"].data_ptr(), t["m"].data_ptr(), t["v"].data_ptr(),
                            0 if t["wb"] is None else t["wb"].data_ptr(), 0 if t["wt"] is None else t["wt"].data_ptr(),
                            0 if t["avg"] is None else t["avg"].data_ptr(), r, c, 1e-4 * k, 0)
            for k, ((r, c), t) in enumerate(zip(shapes, sets[1], strict=True))]
    arr = (tmc.CAdamTensor * len(rows))(*rows)
    blocks = tmc.lib().tmc_b200_nn_adam_plan(arr, len(rows))
    assert blocks == sum((r * c + 255) // 256 for r, c in shapes)
    assert [x.first_block for x in arr] == [0, 131, 134, 150]
    dev = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).cuda()
    S._call("tmc_b200_nn_adam_multi", S._p(dev), len(rows), blocks, ctypes.c_float(0.0), S._p(lr_dev),
            ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), ctypes.c_float(0.99), s)
    torch.cuda.synchronize()
    for a, b in zip(sets[0], sets[1], strict=True):
        for key in ("w", "m", "v", "avg", "wb", "wt"):
            if a[key] is not None:
                assert torch.equal(a[key], b[key]), key
    assert tmc.lib().tmc_b200_nn_adam_plan(arr, 0) == -1


def test_graph_captured_training_equals_host_launched_training():
    """Training with the optimiser step captured once as a CUDA graph and replayed gives the same
    weights and Adam moments, bit for bit, as launching every kernel from the host (the reported loss
    is summed with atomics, so it agrees to rounding)."""
    from tissuemc_b200 import surrogate as S

    rng = np.random.default_rng(6)
    X = rng.normal(size=(3 * 4096 + 100, S.N_FEAT))
    Y = rng.normal(size=(len(X), S.N_OUT))
    runs = []
    for graph in (False, True):
        ens = S.Ensemble(members=2, batch=4096, seed=5)
        hist = ens.train(X, Y, epochs=3, lr=2e-3, ema=0.99, weight_decay=1e-4, graph=graph)
        hist += ens.train(X[:4096], Y[:4096], epochs=2, lr=1e-3, graph=graph)  # Adam's step count carries over
        torch.cuda.synchronize()
        runs.append((hist, [[t.clone() for t in m.W + m.b + m.Wb + m.WT + m.mW + m.vW] for m in ens.members]))
    (h0, p0), (h1, p1) = runs
    np.testing.assert_allclose(h0, h1, rtol=1e-5)
    for a, b in zip(p0, p1, strict=True):
        for x, y in zip(a, b, strict=True):
            assert torch.equal(x, y)
    assert h0[2] < h0[0]  # and it trains


@pytest.fixture(scope="module")
def trained():
    """A small ensemble trained on 2^14 sweep solves at 1e4 photons (fast; the full-size run is in
    bench.py --workload surrogate)."""
    from tissuemc_b200 import surrogate as S

    cfgs, X, Y = S.generate(16384, 10_000, master_seed=41)
    _, Xv, Yv = S.generate(2048, 10_000, master_seed=42)
    ens = S.Ensemble(members=4, batch=4096, seed=1)
    hist = ens.train(X, Y, epochs=30, lr=2e-3)
    return S, ens, hist, (Xv, Yv)


def test_training_reduces_the_loss_and_generalises(trained):
    S, ens, hist, (Xv, Yv) = trained
    assert hist[-1] < 0.2 * hist[0], hist
    pred = ens.predict(Xv)
    ynorm = (Yv - ens.norm.y_mean) / ens.norm.y_std
    pnorm = (pred - ens.norm.y_mean) / ens.norm.y_std
    mse = float(((pnorm - ynorm) ** 2).mean())
    assert mse < 0.15, mse  # held-out error well below the variance of the targets (1.0)


def test_gate_flags_disagreement_out_of_distribution(trained):
    S, ens, _, (Xv, _) = trained
    inside = S.gate(ens.predict_members(Xv)).mean()
    far = Xv.copy()
    far[:, 0] += 3.0  # mu_a 1000x beyond the training range
    outside = S.gate(ens.predict_members(far)).mean()
    assert outside > inside


def test_inverse_fit_recovers_parameters_through_the_surrogate(trained):
    S, ens, _, (Xv, _) = trained
    two = Xv[S.present(Xv, 1) & ~S.present(Xv, 2)][:64].copy()  # two-layer configurations
    assert len(two) >= 16
    obs = ens.predict(two)[:, :S.N_RD]  # noise-free, self-consistent observations
    mask = (obs > -3.5).astype(float)
    start = two.copy()
    free = [0, 1, 4, 5]  # log10 mu_a, log10 mu_s' of both layers
    start[:, free] += np.random.default_rng(3).normal(0, 0.15, (len(two), 4))
    fit, res = S.lm_fit(ens, start, obs, mask, free, iters=40)
    err_before = np.abs(start[:, free] - two[:, free]).mean()
    err_after = np.abs(fit[:, free] - two[:, free]).mean()
    assert err_after < 0.5 * err_before, (err_before, err_after)


def test_surrogate_beats_monte_carlo_at_equal_cost(trained):
    """What the network gains: served in batches, one surrogate query costs less GPU time than
    tracing even 1,000 photons, and its R_d(r) (trained on 1e4-photon solves) is closer to a
    1e5-photon solve than a 1,000-photon Monte Carlo run is."""
    S, ens, _, _ = trained
    cfgs, X, _ = S.generate(512, 100_000, master_seed=43)  # reference solves
    n_q = 65536
    Xq = np.tile(X, (n_q // len(X), 1))
    ens.predict(Xq[:4096])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred_q = ens.predict(Xq)
    t_sur = (time.perf_counter() - t0) / n_q
    cheap = (tmc.CSweepConfig * len(cfgs))(*cfgs)
    for c in cheap:
        c.photons = 1000
    mc = tmc.sweep_run(cheap, tmc.sweep_options())
    t_mc = mc.seconds / len(cfgs)
    ref = tmc.sweep_run((tmc.CSweepConfig * len(cfgs))(*cfgs), tmc.sweep_options())
    Yref = S.targets(ref.summary)
    inner = slice(0, 16)
    pred = pred_q[: len(X)]
    err_sur = np.abs(pred[:, inner] - Yref[:, inner]).mean()
    err_mc = np.abs(S.targets(mc.summary)[:, inner] - Yref[:, inner]).mean()
    print(f"surrogate {t_sur * 1e6:.2f} us/query, err {err_sur:.4f}; MC(1e3 photons) {t_mc * 1e6:.2f} us/solve, "
          f"err {err_mc:.4f}")
    assert err_sur < err_mc, (err_sur, err_mc)
    assert t_sur < t_mc, (t_sur, t_mc)


def _check_fused_against_layered(S, ens, X):
    fs = S.FusedServer(ens)
    spreads: list = []
    y, rd, route = fs(X, spreads)
    pm = ens.predict_members(X)  # every member through the per-layer GEMM kernels
    ref_y = pm.mean(0)
    # activations are rounded to BF16 in both paths; a last-bit difference in an FP32 sum can round
    # one activation to its neighbour, so outputs agree to a fraction of a BF16 step
    assert np.abs(y - ref_y).max() <= 1e-2 * np.abs(ref_y).max()
    ref_rd = S.rd_total(pm).mean(0)
    np.testing.assert_allclose(rd, ref_rd, rtol=2e-2)
    ref_sp = S.spread(pm)
    sp = spreads[0]
    assert np.abs(sp - ref_sp).max() <= 2e-3 + 0.05 * ref_sp.max()
    near = np.abs(ref_sp - fs.threshold) < 2e-3
    assert np.array_equal(route[~near], (ref_sp > fs.threshold)[~near])
    # the per-layer serving path (encode kernel, member GEMMs, gate kernel) agrees as well
    sp_l: list = []
    y_l, rd_l, route_l = S.Server(ens, chunk=65536)(X, sp_l)
    assert np.abs(y_l - ref_y).max() <= 1e-2 * np.abs(ref_y).max()
    np.testing.assert_allclose(rd_l, ref_rd, rtol=2e-2)
    assert np.abs(sp_l[0] - ref_sp).max() <= 2e-3 + 0.05 * ref_sp.max()
    assert np.array_equal(route_l[~near], (ref_sp > fs.threshold)[~near])


def test_fused_ensemble_kernel_matches_the_layered_path_random_weights():
    """Three untrained members with non-zero biases, 300 queries (a partial last tile)."""
    from tissuemc_b200 import surrogate as S

    ens = S.Ensemble(members=3, batch=4096, seed=5)
    rng = np.random.default_rng(7)
    for m in ens.members:
        for b in m.b:
            b.copy_(torch.from_numpy(rng.normal(0, 0.05, b.shape[0]).astype(np.float32)))
    y_mean = np.concatenate([np.full(S.N_RD, -2.0), [0.05, 0.6]])
    y_std = np.concatenate([np.full(S.N_RD, 0.3), [0.02, 0.1]])
    ens.norm = S.Norm(np.zeros(S.N_FEAT), np.ones(S.N_FEAT), y_mean, y_std)
    X = rng.normal(size=(300, S.N_FEAT))
    _check_fused_against_layered(S, ens, X)


def test_fused_ensemble_kernel_matches_the_layered_path_trained(trained):
    """The trained ensemble on 40,000 queries: more tiles of 128 than SMs, so every CTA of the
    persistent kernel walks several tiles."""
    S, ens, _, (Xv, _) = trained
    X = np.tile(Xv, (20, 1))[:40_000]
    _check_fused_against_layered(S, ens, X)


def test_fused_ensemble_rejects_bad_shapes():
    from tissuemc_b200 import surrogate as S
    import ctypes

    dummy = torch.zeros(16, device="cuda")
    p = S._p(dummy)
    with pytest.raises(tmc.ConfigError, match="1-8 members"):
        S._call("tmc_b200_nn_ensemble_infer", p, p, 9, p, 10, 13, p, p, 66, p, p, p, 64, ctypes.c_float(0.01),
                p, p, p, p, ctypes.c_void_p(0))
    with pytest.raises(tmc.ConfigError, match="R_d bins"):
        S._call("tmc_b200_nn_ensemble_infer", p, p, 4, p, 10, 13, p, p, 66, p, p, p, 65, ctypes.c_float(0.01),
                p, p, p, p, ctypes.c_void_p(0))
