# SPDX-License-Identifier: Apache-2.0
"""The warm-start network's tensor-core kernels (tcgen05) against a plain PyTorch FP32 reference of the same network.

The kernels round the MMA operands to BF16 (features, hidden activations, weights and, in training, the
back-propagated dZ) and accumulate in FP32; the reference rounds the same operands at the same places. The kernels'
SiLU uses the hardware tanh approximation (relative error about 2^-11), so forward outputs agree to 3e-3 of the
output scale and gradients to the BF16 rounding of the back-propagated terms (2e-2 of each block's largest entry)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from alloy_b200.solvers.sph.warmstart import N_PARAMS, Network, init_params, unpack

pytestmark = pytest.mark.gpu


def _bf(x: torch.Tensor) -> torch.Tensor:
    return x.to(torch.bfloat16).to(torch.float32)


def _reference(p: np.ndarray, x: torch.Tensor):
    """The network in FP32 with the kernels' BF16 operand rounding; parameters are leaf tensors for autograd."""
    u = {k: torch.tensor(v, dtype=torch.float32, requires_grad=True) for k, v in unpack(p).items()}
    z1 = _bf(x) @ _bf(u["w1"]).T + u["b1"]
    h1 = z1 * torch.sigmoid(z1)
    z2 = _bf(h1) @ _bf(u["w2"]).T + u["b2"]
    h2 = z2 * torch.sigmoid(z2)
    return h2 @ u["w3"].T + u["b3"], u


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 40_000])
def test_forward_matches_reference(cuda, n):
    rng = np.random.default_rng(n)
    p = init_params(seed=n)
    p[64 * 16:64 * 16 + 64] = rng.normal(0, 0.1, 64)  # non-zero biases
    net = Network(p)
    x = torch.from_numpy(rng.normal(0.0, 1.0, (n, 16)).astype(np.float32))
    y = net.forward(x.to(cuda)).cpu()
    torch.cuda.synchronize()
    net.status()
    ref, _ = _reference(p, x)
    ref = ref.detach()
    scale = float(ref.abs().max()) + 1e-6
    assert torch.isfinite(y).all()
    np.testing.assert_allclose(y.numpy(), ref.numpy(), rtol=0, atol=3e-3 * scale)


@pytest.mark.parametrize("batch", [64, 300, 5000])
def test_gradient_matches_autograd(cuda, batch):
    rng = np.random.default_rng(batch)
    N = 7000
    p = init_params(seed=1)
    p[64 * 16:64 * 16 + 64] = rng.normal(0, 0.1, 64)
    p[64 * 16 + 64 + 64 * 64:64 * 16 + 64 + 64 * 64 + 64] = rng.normal(0, 0.1, 64)
    net = Network(p)
    x = torch.from_numpy(rng.normal(0.0, 1.0, (N, 16)).astype(np.float32))
    t = torch.from_numpy(rng.normal(0.0, 1.0, (N, 2)).astype(np.float32))
    idx = torch.from_numpy(rng.permutation(N)[:batch].astype(np.int32))
    g, loss = net.gradient(x.to(cuda), t.to(cuda), idx.to(cuda))
    net.status()
    xb, tb = x[idx.long()], t[idx.long()]
    y, u = _reference(p, xb)
    L = ((y - tb) ** 2).sum() / (2 * batch)
    L.backward()
    assert loss == pytest.approx(float(L.detach()), rel=2e-3)
    ref = np.concatenate([u[k].grad.numpy().ravel() for k in ("w1", "b1", "w2", "b2", "w3", "b3")])
    assert ref.size == N_PARAMS
    ours = unpack(g)
    for k, r in unpack(ref).items():
        tol = 2e-2 * float(np.abs(r).max()) + 1e-9
        np.testing.assert_allclose(ours[k], r, rtol=0, atol=tol, err_msg=k)


def test_adam_training_fits_a_smooth_map(cuda):
    """Twenty epochs of Adam on the tensor cores fit a smooth 16 -> 2 map far below its variance; the loss falls
    monotonically across epochs and the parameters stay finite."""
    rng = np.random.default_rng(7)
    N = 65_536
    x = rng.normal(0.0, 1.0, (N, 16)).astype(np.float32)
    t = np.stack([np.tanh(x[:, 0] + 0.5 * x[:, 1] * x[:, 2]), 0.3 * x[:, 3] - np.sin(x[:, 4])], axis=1)
    t = ((t - t.mean(0)) / t.std(0)).astype(np.float32)
    net = Network(init_params(seed=3))
    xd, td = torch.from_numpy(x).to(cuda), torch.from_numpy(t).to(cuda)
    gen = torch.Generator(device=cuda).manual_seed(0)
    losses = []
    for ep in range(20):
        perm = torch.randperm(N, generator=gen, device=cuda).to(torch.int32)
        ls = [net.train_step(xd, td, perm[b:b + 8192].contiguous(), 3e-3, want_loss=True) for b in range(0, N, 8192)]
        losses.append(float(np.mean(ls)))
    net.status()
    assert np.isfinite(net.params()).all()
    assert losses[-1] < 0.1 * losses[0], losses
    assert losses[-1] < 0.1, losses
    assert all(b < a * 1.05 for a, b in zip(losses, losses[1:])), losses


def test_an_expired_tensor_core_wait_sets_the_status_and_the_context_survives(cuda):
    """The MMA waits give up after a poll limit; a limit of 0 polls makes every one give up at once. Each kernel then
    waits for the MMAs it committed, frees its tensor memory and returns: the status reports the expiry (ADF_ERR_STATE,
    a RuntimeError here), and after the status is cleared and the limit restored the same network computes the
    reference's outputs again on the same context."""
    from alloy_b200 import _lib

    L = _lib.lib()
    rng = np.random.default_rng(7)
    p = init_params(seed=7)
    net = Network(p)
    x = torch.from_numpy(rng.normal(0.0, 1.0, (3000, 16)).astype(np.float32))
    t = torch.from_numpy(rng.normal(0.0, 1.0, (3000, 2)).astype(np.float32))
    idx = torch.arange(3000, dtype=torch.int32)
    _lib.check(L.adf_mlp_set_wait_limit(net.handle, 0))
    net.forward(x.to(cuda))
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match="tensor-core wait expired"):
        net.status()
    _lib.check(L.adf_mlp_clear_status(net.handle))
    net.gradient(x.to(cuda), t.to(cuda), idx.to(cuda))  # the gradient kernel's waits expire the same way
    with pytest.raises(RuntimeError, match="tensor-core wait expired"):
        net.status()
    _lib.check(L.adf_mlp_clear_status(net.handle))
    _lib.check(L.adf_mlp_set_wait_limit(net.handle, 1 << 22))
    y = net.forward(x.to(cuda)).cpu()
    torch.cuda.synchronize()
    net.status()
    ref, _ = _reference(p, x)
    ref = ref.detach()
    np.testing.assert_allclose(y.numpy(), ref.numpy(), rtol=0, atol=3e-3 * (float(ref.abs().max()) + 1e-6))
