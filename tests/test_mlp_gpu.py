"""The scheduler MLP's hand-written GPU kernels against the float64 CPU oracle."""
import ctypes

import numpy as np
import pytest

from custingeralg_b200 import native as N
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def init_params(seed=1):
    p = np.zeros(N.MLP_PARAMS, np.float32)
    N.check(N.lib().tc_mlp_init(p.ctypes.data, seed))
    return p


def data(n, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.uniform(0, 1, (n, N.MLP_IN)).astype(np.float32)
    X[:, :2] *= 16
    s = rng.integers(0, N.MLP_OUT, n).astype(np.int32)
    y = (X[:, 0] * 0.3 - X[:, 1] * 0.1 + s + rng.normal(0, 0.1, n)).astype(np.float32)
    return X, s, y


@pytest.mark.parametrize("n", [1, 31, 33, 1000, 5000])
def test_forward_matches_oracle(n):
    import torch
    p = init_params(3)
    X, _, _ = data(n)
    y = torch.zeros(n, N.MLP_OUT, dtype=torch.float32, device="cuda")
    dp, dx = _t(p), _t(X)  # keep the device tensors alive across the call
    N.check(N.lib().tc_mlp_forward(dp.data_ptr(), dx.data_ptr(), n, y.data_ptr(), None))
    ref, _ = M.forward(p, X)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("n", [1, 40, 3000])
def test_gradient_matches_oracle(n):
    import torch
    p = init_params(5)
    X, s, lab = data(n, seed=n)
    g = torch.zeros(N.MLP_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    dp, dx, ds, dl = _t(p), _t(X), _t(s), _t(lab)
    N.check(N.lib().tc_mlp_backward(dp.data_ptr(), dx.data_ptr(), ds.data_ptr(), dl.data_ptr(), n,
                                    g.data_ptr(), loss.data_ptr(), None))
    ref_loss, ref_g = M.loss_and_grad(p, X, s, lab)
    assert abs(loss.item() - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    # fp32 accumulation vs float64: relative to the gradient's scale
    scale = np.abs(ref_g).max()
    np.testing.assert_allclose(g.cpu().numpy(), ref_g, rtol=2e-3, atol=2e-4 * scale)


def test_training_reduces_loss():
    import torch
    p = init_params(7)
    X, s, lab = data(4000, seed=11)
    dp, dx, ds, dl = _t(p), _t(X), _t(s), _t(lab)
    l0, _ = M.loss_and_grad(p, X, s, lab)
    out = ctypes.c_float()
    N.check(N.lib().tc_mlp_train(dp.data_ptr(), dx.data_ptr(), ds.data_ptr(), dl.data_ptr(), 4000, 400,
                                 3e-3, ctypes.byref(out), None))
    l1, _ = M.loss_and_grad(dp.cpu().numpy(), X, s, lab)
    assert abs(out.value - l1) < 1e-3 * max(1, l1)
    assert l1 < 0.2 * l0
