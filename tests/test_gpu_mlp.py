"""The learned warm start's tensor-core kernels (B200).

- The tcgen05 BF16 GEMM against a float64 product of the same BF16 inputs
  (FP32 accumulation: agreement to FP32 rounding), with its fused bias,
  tanh and BF16 epilogue, on ragged row counts, several N tiles and K chunks.
- The network's gradients against the numpy restatement (oracle/mlp_ref.py),
  which rounds to BF16 where the GPU does: relative error of each gradient
  tensor below 1e-3 (FP32 summation order, and a BF16 rounding it flips).
- Training on the GPU fits a smooth map.
- A completion wait that runs out (every wait bounded to no rounds) raises
  the timeout status and stores nothing; the next unbounded GEMM on the same
  device is correct (the drained MMAs left the context usable).
"""

import numpy as np
import pytest

from espice_b200 import mlp
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available(), "a CUDA device is required"
    return torch


# the last: the learned step's inference shape (a 32,768-point chunk through
# a 512-wide hidden layer)
@pytest.mark.parametrize("M,N,K", [(200, 96, 48), (1000, 512, 512), (128, 16, 16), (333, 272, 80),
                                   (32768, 512, 512)])
def test_gemm_matches_float64(M, N, K):
    torch = _torch()
    g = torch.Generator().manual_seed(M + N + K)
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    c = torch.zeros(M, N, device="cuda")
    h = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    mlp.gemm_bf16(a.data_ptr(), K, b.data_ptr(), K, M, N, K, c.data_ptr(), N, d_bias=bias.data_ptr(),
                  d_h=h.data_ptr(), ldh=N, act=1)
    torch.cuda.synchronize()
    ref = a.double().cpu() @ b.double().cpu().T + bias.double().cpu()
    got = c.double().cpu()
    scale = (a.double().abs().cpu() @ b.double().abs().cpu().T).max()
    assert float((got - ref).abs().max()) <= 1e-6 * float(scale) + 1e-6
    # the BF16 tanh copy: the device's tanhf and the host's may differ in the
    # last FP32 bit, which flips a BF16 rounding now and then: one BF16 ulp,
    # on a handful of the elements at most
    th = torch.tanh(c.cpu()).to(torch.bfloat16).float()
    hb = h.cpu().float()
    assert torch.allclose(hb, th, rtol=2.0 ** -7, atol=0.0)
    assert float((hb != th).float().mean()) <= 1e-5


def test_gemm_without_bias_or_copy():
    torch = _torch()
    M, N, K = 130, 32, 32
    a = torch.randn(M, K).to(torch.bfloat16).cuda()
    b = torch.randn(N, K).to(torch.bfloat16).cuda()
    c = torch.zeros(M, N, device="cuda")
    torch.cuda.synchronize()
    mlp.gemm_bf16(a.data_ptr(), K, b.data_ptr(), K, M, N, K, c.data_ptr(), N)
    torch.cuda.synchronize()
    ref = a.double().cpu() @ b.double().cpu().T
    assert float((c.double().cpu() - ref).abs().max()) < 1e-4


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_gradients_match_reference():
    torch = _torch()
    rng = np.random.default_rng(3)
    n_in, n_out, rows = 16, 40, 64
    net = mlp.Mlp(n_in, 64, 3, n_out, seed=5)
    in_mu, in_sig = rng.normal(size=n_in).astype(np.float32), rng.uniform(0.5, 2, n_in).astype(np.float32)
    out_mu, out_sig = rng.normal(size=n_out).astype(np.float32), rng.uniform(0.5, 2, n_out).astype(np.float32)
    net.set_scaling(in_mu, in_sig, out_mu, out_sig)
    x = rng.normal(size=(rows, n_in)).astype(np.float32)
    y = rng.normal(size=(rows, n_out)).astype(np.float32)
    dx, dy = torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")
    torch.cuda.synchronize()
    loss, grads = net.gradients(dx.data_ptr(), dy.data_ptr(), rows)
    layers = net.weights()
    loss_ref, grads_ref = mlp_ref.gradients(layers, x, y, in_mu, in_sig, out_mu, out_sig)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    for (gw, gb), (rw, rb) in zip(grads, grads_ref):
        assert _rel(gw, rw) < 1e-3
        assert _rel(gb, rb) < 1e-3
    net.close()


def test_training_fits_a_smooth_map():
    torch = _torch()
    rng = np.random.default_rng(11)
    n_in, n_out, n = 4, 24, 4096
    A = rng.normal(size=(n_in, n_out))
    x = rng.uniform(-1, 1, size=(n, n_in)).astype(np.float32)
    y = np.sin(x @ A).astype(np.float32)
    net = mlp.Mlp(n_in, 128, 3, n_out, seed=2)
    net.set_scaling(x.mean(0), x.std(0), y.mean(0), y.std(0))
    dx, dy = torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")
    torch.cuda.synchronize()
    loss = net.train(dx.data_ptr(), dy.data_ptr(), n, epochs=60, batch=256, lr=2e-3)
    assert loss[-1] < 0.05 * loss[0]
    out = torch.zeros(n, n_out, device="cuda")
    net.predict(dx.data_ptr(), n, out.data_ptr())
    torch.cuda.synchronize()
    err = np.abs(out.cpu().numpy() - y).mean()
    assert err < 0.1
    net.close()


def test_gemm_wait_runs_out_and_stores_nothing():
    torch = _torch()
    M, N, K = 256, 128, 192
    g = torch.Generator().manual_seed(7)
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    c = torch.full((M, N), 12345.0, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(mlp.MlpError) as err:
        mlp.gemm_bf16(a.data_ptr(), K, b.data_ptr(), K, M, N, K, c.data_ptr(), N, wait_rounds=mlp.GEMM_NO_WAIT)
    assert err.value.code == mlp.MLP_TIMEOUT
    torch.cuda.synchronize()
    assert bool((c == 12345.0).all()), "a timed-out GEMM stored results"
    mlp.gemm_bf16(a.data_ptr(), K, b.data_ptr(), K, M, N, K, c.data_ptr(), N)
    torch.cuda.synchronize()
    ref = a.double().cpu() @ b.double().cpu().T
    assert torch.allclose(c.double().cpu(), ref, rtol=1e-5, atol=1e-4)
