"""Kernels of the learned frequency screen against their CPU restatement
(oracle/screen_ref.py): the phase-folded features, the BF16 tensor-core
GEMM with every operand layout the network uses, and the network's
forward/backward pass (loss and gradients), plus a training sanity check."""
import numpy as np
import pytest

from conftest import prepared

pytestmark = pytest.mark.gpu


def test_features_match_cpu_restatement():
    from oracle import screen_ref
    from ps_claude_opt_b200 import screen

    obj = prepared("mixed")
    freqs = screen.frequencies(obj)                                    # 1/hour
    freqs = np.concatenate([freqs, np.linspace(0.01, 0.5, 45)])       # plus periods 2 .. 100 h
    got = screen.features(obj, freqs)
    ref = screen_ref.features(obj.tim, obj.brightness, obj.curve_len, 24.0 * freqs)
    assert got.shape == (len(freqs), 88)
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - ref)) < 1e-4
    # fixed-point bin sums: the same features on every run
    assert np.array_equal(screen.features(obj, freqs), got)


def _bf16(rng, *shape):
    from oracle import screen_ref

    return screen_ref.bf16_round(rng.standard_normal(shape).astype(np.float32))


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (37, 29, 70), (130, 67, 300), (64, 256, 1024)])
def test_gemm_bf16_all_layouts(M, N, K):
    import ctypes as C

    import torch

    from ps_claude_opt_b200 import native, screen

    rng = np.random.default_rng(M + N + K)
    a, b = _bf16(rng, M, K), _bf16(rng, K, N)
    ref = a.astype(np.float64) @ b.astype(np.float64)
    bias = rng.standard_normal(N).astype(np.float32)
    for ta in (False, True):
        for tb in (False, True):
            A = torch.from_numpy(np.ascontiguousarray(a.T if ta else a)).cuda().to(torch.bfloat16)
            B = torch.from_numpy(np.ascontiguousarray(b.T if tb else b)).cuda().to(torch.bfloat16)
            sam, sak = (1, M) if ta else (K, 1)
            sbk, sbn = (1, K) if tb else (N, 1)
            Cd = torch.zeros((M, N), dtype=torch.float32, device="cuda")
            Cb = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
            bd = torch.from_numpy(bias).cuda()
            native._check(screen._lib().ps_gemm_bf16(M, N, K, C.c_void_p(A.data_ptr()), sam, sak,
                                                     C.c_void_p(B.data_ptr()), sbk, sbn, C.c_void_p(Cd.data_ptr()),
                                                     N, 0, C.c_void_p(bd.data_ptr()), 1, C.c_void_p(Cb.data_ptr()),
                                                     N, None))
            torch.cuda.synchronize()
            want = np.maximum(ref + bias, 0.0)
            got = Cd.cpu().numpy()
            assert np.allclose(got, want, rtol=1e-5, atol=1e-4 * np.sqrt(K))
            assert np.allclose(Cb.float().cpu().numpy(), got, rtol=1e-2, atol=1e-6)


def test_network_gradients_match_cpu_restatement():
    import torch

    from oracle import screen_ref
    from ps_claude_opt_b200 import screen

    rng = np.random.default_rng(4)
    net = screen.Mlp(sizes=(64, 48, 40, 1), seed=3)
    x = rng.standard_normal((150, 64)).astype(np.float32)
    with pytest.raises(ValueError):
        net.forward(torch.zeros((4, 63), dtype=torch.bfloat16, device="cuda"))
    y = rng.standard_normal(150).astype(np.float32)
    W = [w.cpu().numpy() for w in net.W]
    b = [v.cpu().numpy().astype(np.float64) for v in net.b]
    xb = torch.from_numpy(x).cuda().to(torch.bfloat16)
    yd = torch.from_numpy(y).cuda()
    yhat = net.forward(xb)
    diff = yhat - yd
    gW, gb = net.backward((2.0 / len(y)) * diff)
    loss_ref, yhat_ref, gW_ref, gb_ref = screen_ref.mlp_forward_backward(x, y.astype(np.float64), W, b)
    assert np.allclose(yhat.cpu().numpy(), yhat_ref, rtol=2e-2, atol=2e-2)
    loss = float((diff * diff).mean())
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    for g, r in zip(gW + gb, gW_ref + gb_ref):
        g = g.cpu().numpy()
        assert np.linalg.norm(g - r) <= 3e-2 * np.linalg.norm(r)


def test_training_reduces_the_loss():
    import torch

    from ps_claude_opt_b200 import screen

    rng = np.random.default_rng(9)
    x = rng.standard_normal((4096, screen.N_FEATURES)).astype(np.float32)
    y = (np.tanh(x[:, 0] - 0.5 * x[:, 3]) + 0.3 * x[:, 7] * x[:, 8]).astype(np.float32)
    net = screen.Mlp(seed=1)
    xb = torch.from_numpy(x).cuda().to(torch.bfloat16)
    yd = torch.from_numpy(y).cuda()
    first = net.train_step(xb[:1024], yd[:1024], 1e-3)
    for ep in range(30):
        for i in range(0, 4096, 512):
            net.train_step(xb[i:i + 512], yd[i:i + 512], 1e-3)
    pred = net.predict(x)
    assert float(np.mean((pred - y) ** 2)) < 0.2 * first
