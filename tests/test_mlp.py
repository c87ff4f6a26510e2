"""The learned schedule's network (bfm_mlp_*): bf16 tensor-core forward and
backward passes with fp32 accumulation and an Adam step, checked against
the numpy oracle (oracle/mlp_oracle.py), whose backward formulas are in
turn checked against finite differences in exact arithmetic.

Tolerances: the device rounds the same operands to bf16 as the oracle, so
the only differences are fp32 versus fp64 accumulation and the rare bf16
rounding flips that follow from them; outputs agree to 1e-3 relative,
gradient vectors to 2e-3 in relative norm."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

I, H, O = 6, 128, 4


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, I)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + x[:, 1] * x[:, 2], np.cos(x[:, 3]), x[:, 4] ** 2 - 1, np.tanh(x[:, 5])], 1)
    return x, t.astype(np.float32)


def _params(seed=1):
    rng = np.random.default_rng(seed)
    n = H * I + H + H * H + H + O * H + O
    return (rng.normal(size=n) * 0.15).astype(np.float32)


def test_oracle_backward_matches_finite_differences():
    mo.ROUND = False
    try:
        x, t = _data(8)
        p = _params().astype(np.float64)
        w = np.array([1.0, 0.5, 2.0, 1.0])
        loss, g = mo.gradients(p, x, t, w, I, H, O)
        rng = np.random.default_rng(3)
        for k in rng.choice(p.size, 40, replace=False):
            e = np.zeros_like(p)
            e[k] = 1e-6
            lp, _ = mo.gradients(p + e, x, t, w, I, H, O)
            lm, _ = mo.gradients(p - e, x, t, w, I, H, O)
            assert abs((lp - lm) / 2e-6 - g[k]) < 1e-6 + 1e-5 * abs(g[k])
    finally:
        mo.ROUND = True


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3], np.float32)
    r = mo.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 1e-3) < 1e-3 * 2 ** -8


def test_network_needs_the_gpu():
    from pscbfm_b200.mlp import MLP
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(RuntimeError):
        MLP()


@pytest.mark.gpu
def test_forward_matches_oracle():
    from pscbfm_b200.mlp import MLP
    m = MLP(I, H, O, seed=5)
    p = _params()
    m.set_params(p)
    assert np.array_equal(m.params(), p)
    x, _ = _data(1000, seed=2)
    y = m.forward(x)
    want, _ = mo.forward(p, x, I, H, O)
    np.testing.assert_allclose(y, want, rtol=1e-3, atol=1e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [16, 100, 4096])
def test_gradients_match_oracle(batch):
    from pscbfm_b200.mlp import MLP
    m = MLP(I, H, O, seed=5)
    p = _params()
    m.set_params(p)
    x, t = _data(batch, seed=batch)
    w = np.array([1.0, 0.5, 2.0, 1.0], np.float32)
    loss, g = m.gradients(x, t, w)
    wl, wg = mo.gradients(p, x, t, w, I, H, O)
    assert abs(loss - wl) <= 1e-4 * abs(wl) + 1e-6
    off = 0
    for shape in ((H, I), (H,), (H, H), (H,), (O, H), (O,)):
        k = int(np.prod(shape))
        a, b = g[off:off + k], wg[off:off + k]
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-7, shape
        off += k


@pytest.mark.gpu
def test_adam_step_matches_oracle_and_training_learns():
    from pscbfm_b200.mlp import MLP
    m = MLP(I, H, O, seed=5)
    p = _params()
    m.set_params(p)
    x, t = _data(512, seed=9)
    _, g = m.gradients(x, t)
    m.train_step(x, t, lr=1e-3)
    want, _, _ = mo.adam(p.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1, 1e-3)
    np.testing.assert_allclose(m.params(), want, rtol=1e-5, atol=1e-6)
    # a fresh network learns the smooth target
    m2 = MLP(I, H, O, seed=11)
    xs, ts = _data(4096, seed=10)
    first = m2.gradients(xs, ts)[0]
    hist = m2.fit(xs, ts, epochs=60, batch=256, lr=2e-3)
    assert hist[-1] < 0.1 * first
    xv, tv = _data(1024, seed=12)
    assert float(np.mean((m2.forward(xv) - tv) ** 2).sum()) < 0.2 * first


@pytest.mark.gpu
def test_steps_in_one_launch_equal_single_steps():
    """bfm_mlp_train_steps runs several Adam steps in one cooperative launch;
    they must equal the same steps launched one by one, bit for bit (the
    cross-CTA gradient sums run in a fixed order), including a last step of
    fewer rows than the others."""
    from pscbfm_b200.mlp import MLP
    x, t = _data(700, seed=21)
    w = np.array([1.0, 0.5, 2.0, 1.0], np.float32)
    rng = np.random.default_rng(4)
    idx = rng.permutation(700).astype(np.uint32)
    rows = [256, 256, 188]
    a = MLP(I, H, O, seed=7)
    b = MLP(I, H, O, seed=7)
    la = a.train_steps(x, t, idx, rows, w, lr=3e-3)
    lb, o = [], 0
    for r in rows:
        sel = idx[o:o + r]
        lb.append(b.train_step(x[sel], t[sel], w, lr=3e-3))
        o += r
    assert np.array_equal(a.params(), b.params())
    assert np.array_equal(la, np.array(lb, np.float32))


@pytest.mark.gpu
def test_network_shapes_outside_the_kernel_are_refused():
    from pscbfm_b200.mlp import MLP
    for shape in ((17, 128, 4), (6, 64, 4), (6, 128, 17)):
        with pytest.raises(ValueError):
            MLP(*shape)
