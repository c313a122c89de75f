"""Tensor-core MLP kernels against the CPU oracle (oracle/mlp_ref.py)."""
import numpy as np
import pytest
import torch

from magpackage_b200.mlp import MLP, init_params
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _case(n, seed):
    rng = np.random.default_rng(seed)
    p = init_params(seed)
    p[256:320] = rng.normal(0, 0.1, 64)  # nonzero biases exercise every path
    x = rng.normal(0, 1, (n, 4)).astype(np.float32)
    t = rng.normal(0, 1, n).astype(np.float32)
    return p, x, t


@pytest.mark.parametrize("n", [128, 300, 4096])
def test_forward_matches_oracle(n):
    p, x, _ = _case(n, 1)
    net = MLP(p)
    y, _ = net.forward(torch.as_tensor(x, device="cuda"))
    net.check()
    y_ref, _ = mlp_ref.forward(p, x)
    y = y.cpu().numpy()
    # FP32 accumulation order differs from the float64 oracle; BF16 rounding points match
    assert np.max(np.abs(y - y_ref)) <= 2e-3 * (1 + np.max(np.abs(y_ref)))
    assert np.corrcoef(y, y_ref)[0, 1] > 0.99999


@pytest.mark.parametrize("use_rows", [True, False])
def test_predict_nu_scatter_and_clamp(use_rows):
    """mag_mlp_predict_nu: nu = clamp(exp(y * scale + shift), nu_min, nu_max), scattered to
    d_nu[d_rows[i]] (d_rows NULL: d_nu[i]); y is the inference output of the same network,
    checked against the oracle like the forward test. Rows not named keep their values."""
    n = 5000
    p, x, _ = _case(n, 4)
    net = MLP(p)
    xd = torch.as_tensor(x, device="cuda")
    y, _ = net.forward(xd)
    y = y.cpu().numpy().astype(np.float64)
    scale, shift = 0.7, 3.0
    lo = float(np.exp(np.quantile(y, 0.1) * scale + shift))
    hi = float(np.exp(np.quantile(y, 0.9) * scale + shift))
    m = n + 17  # the output is longer than the rows: the extra entries are not touched
    perm = np.random.default_rng(5).permutation(m)[:n].astype(np.int32)
    rows = torch.as_tensor(perm, device="cuda") if use_rows else None
    nu = torch.full((m,), -1.0, dtype=torch.float64, device="cuda")
    net.predict_nu(xd, rows, nu, scale, shift, lo, hi)
    net.check()
    got = nu.cpu().numpy()
    idx = perm if use_rows else np.arange(n)
    want = np.clip(np.exp(y * scale + shift), lo, hi)
    np.testing.assert_allclose(got[idx], want, rtol=1e-13, atol=0)
    assert np.sum(want == lo) > 0 and np.sum(want == hi) > 0  # both bounds were hit
    untouched = np.ones(m, dtype=bool)
    untouched[idx] = False
    assert np.all(got[untouched] == -1.0)
    y_ref, _ = mlp_ref.forward(p, x)
    want_ref = np.clip(y_ref * scale + shift, np.log(lo), np.log(hi))
    assert np.max(np.abs(np.log(got[idx]) - want_ref)) <= scale * 2e-3 * (1 + np.max(np.abs(y_ref)))


@pytest.mark.parametrize("n", [256, 1000])
def test_gradient_matches_oracle(n):
    p, x, t = _case(n, 2)
    net = MLP(p)
    y, g = net.gradient(torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda"), 2.0 / n)
    net.check()
    y_ref, g_ref = mlp_ref.gradient(p, x, t, 2.0 / n)
    g = g.cpu().numpy()
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert rel < 1e-2, rel
    # every parameter block individually
    for a, b in ((0, 256), (256, 320), (320, 4416), (4416, 4480), (4480, 8576), (8576, 8640), (8640, 8704)):
        r = np.linalg.norm(g[a:b] - g_ref[a:b]) / max(np.linalg.norm(g_ref[a:b]), 1e-12)
        assert r < 2e-2, (a, b, r)


def test_training_reduces_loss():
    rng = np.random.default_rng(3)
    n = 16384
    x = rng.normal(0, 1, (n, 4)).astype(np.float32)
    t = (np.tanh(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * x[:, 3]).astype(np.float32)
    net = MLP(init_params(3))
    xd, td = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    y0, _ = net.forward(xd)
    l0 = float(((y0 - td) ** 2).mean())
    for ep in range(30):
        for i in range(0, n, 4096):
            net.train_step(xd[i:i + 4096].contiguous(), td[i:i + 4096].contiguous(), 3e-3)
    net.check()
    y1, _ = net.forward(xd)
    l1 = float(((y1 - td) ** 2).mean())
    assert l1 < 0.1 * l0, (l0, l1)


def test_bounded_wait_gives_up_and_recovers():
    """A tensor-core completion wait limited to one non-blocking poll runs out (the MMA
    is still in flight right after it is issued): the kernels drain their MMAs, free tensor
    memory, report MAG_E_TIMEOUT through mag_mlp_check once, and the next call with the
    default bound is exact again."""
    from magpackage_b200 import _lib

    p, x, t = _case(8192, 3)
    net = MLP(p)
    xd, td = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    net.set_spin_limit(1)
    net.forward(xd)
    with pytest.raises(_lib.MagError) as ei:
        net.check()
    assert ei.value.code == -5  # MAG_E_TIMEOUT
    net.gradient(xd, td, 2.0 / len(t))
    with pytest.raises(_lib.MagError) as ei:
        net.check()
    assert ei.value.code == -5
    net.set_spin_limit(0)
    y, _ = net.forward(xd)
    net.check()  # the status was cleared when it was reported
    y_ref, _ = mlp_ref.forward(p, x)
    assert np.max(np.abs(y.cpu().numpy() - y_ref)) <= 2e-3 * (1 + np.max(np.abs(y_ref)))


def test_train_epoch_equals_train_steps():
    """mag_mlp_train_epoch (minibatches gathered on the device in the permutation's order)
    leaves the same parameters, bit for bit, as train_step on host-gathered minibatches; its
    loss sum is the minibatches' squared errors."""
    rng = np.random.default_rng(4)
    n, batch = 10000, 2048
    x = torch.as_tensor(rng.normal(0, 1, (n, 4)).astype(np.float32), device="cuda")
    t = torch.as_tensor(rng.normal(0, 1, n).astype(np.float32), device="cuda")
    perm = torch.as_tensor(rng.permutation(n), dtype=torch.int64, device="cuda")
    a, b = MLP(init_params(5)), MLP(init_params(5))
    y = torch.empty(batch, dtype=torch.float32, device="cuda")
    z = torch.empty((batch, 3, 64), dtype=torch.float32, device="cuda")
    xb = torch.empty((batch, 4), dtype=torch.float32, device="cuda")
    tb = torch.empty(batch, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    a.train_epoch(x, t, perm, batch, 3e-3, xb, tb, y, z, loss)
    a.check()
    ref = 0.0
    for i in range(0, n - batch + 1, batch):
        idx = perm[i:i + batch]
        xi, ti = x[idx].contiguous(), t[idx].contiguous()
        yi = b.train_step(xi, ti, 3e-3)
        ref += float(((yi - ti) ** 2).sum())
    b.check()
    assert np.array_equal(a.params().view(np.int32), b.params().view(np.int32))
    assert abs(float(loss[0]) - ref) <= 1e-4 * ref
