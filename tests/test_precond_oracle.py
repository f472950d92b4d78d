"""CPU checks of the preconditioner oracle: its operator equals the C oracle's,
its BF16 rounding equals torch's, and its parameter gradient equals central
finite differences of its own float64 loss; the training checkpoint format
round-trips and rejects malformed files."""
import numpy as np
import pytest

import oracle as O
from oracle import precond_oracle as P


def test_operator_matches_c_oracle():
    rng = np.random.default_rng(0)
    nx, ny = 13, 9
    mu = rng.uniform(1, 10, nx * ny)
    a = rng.standard_normal(nx * ny)
    y = O.mag2d_apply(nx, ny, mu, a)
    np.testing.assert_allclose(P.k_apply(a.reshape(ny, nx), (1 / mu).reshape(ny, nx)).ravel(), y, rtol=1e-14,
                               atol=1e-14)
    diag = O.mag2d_diagonal(nx, ny, mu)
    np.testing.assert_allclose(1.0 / P.dinv_of((1 / mu).reshape(ny, nx)).ravel(), diag, rtol=1e-14)


def test_bf16_rounding_matches_torch():
    import torch
    v = np.random.default_rng(1).standard_normal(4096).astype(np.float32) * 1e3
    assert np.array_equal(P.bf16(v), torch.from_numpy(v).bfloat16().float().numpy())


def _batch():
    import similie_b200.magnetostatics as mag
    rng = np.random.default_rng(0)
    out = []
    for n in (21, 36):
        pr = mag.synthetic_problem(rng, n)
        nu = 1.0 / pr.node_mu().reshape(n, n)
        b = pr.rhs().reshape(n, n)
        x, _, _ = O.mag2d_cg(n, n, pr.node_mu(), b.ravel(), tol=1e-12)
        out.append((nu, b, x.reshape(n, n)))
    return out


def test_gradient_matches_finite_differences():
    samples = _batch()
    params = P.init_params(1).astype(np.float64)
    loss, per, g = P.loss_and_grad(params, samples, emulate=False)
    assert all(0.0 <= v <= 1.0 for v in per)
    rng = np.random.default_rng(2)
    for _ in range(3):
        d = rng.standard_normal(P.NUM_PARAMS)
        eps = 1e-6
        lp = P.loss_and_grad(params + eps * d, samples, emulate=False)[0]
        lm = P.loss_and_grad(params - eps * d, samples, emulate=False)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ d) <= 1e-6 * max(abs(fd), 1e-3), (fd, g @ d)


def test_depth_and_pooling_shapes():
    assert P.depth_of(15, 200) == 1 and P.depth_of(16, 16) == 2 and P.depth_of(512, 512) == 7
    x = np.arange(5 * 7, dtype=np.float64).reshape(5, 7, 1)
    c = P.pool(P.pad(x))
    assert c.shape == (3, 4, 1)
    assert c[0, 0, 0] == (0 + 1 + 7 + 8) / 4 and c[2, 3, 0] == x[4, 6, 0] / 4


def test_checkpoint_round_trip_and_rejections(tmp_path):
    from similie_b200.precond import read_checkpoint, write_checkpoint
    rng = np.random.default_rng(3)
    params = rng.standard_normal(1234).astype(np.float32)
    path = str(tmp_path / "ck.bin")
    write_checkpoint(path, params, step=700, seed=9, extra={"lr": 1e-3, "steps": 2000})
    p2, step, seed, extra = read_checkpoint(path)
    np.testing.assert_array_equal(p2, params)
    assert (step, seed, extra) == (700, 9, {"lr": 1e-3, "steps": 2000})
    data = open(path, "rb").read()
    for bad in (b"XXXXXXXX" + data[8:], data[:-4], data + b"\0"):
        open(path, "wb").write(bad)
        with pytest.raises(ValueError):
            read_checkpoint(path)


def test_checkpoint_with_optimizer_state(tmp_path):
    from similie_b200.precond import read_checkpoint, write_checkpoint
    rng = np.random.default_rng(4)
    p, m, v = (rng.standard_normal(50).astype(np.float32) for _ in range(3))
    path = str(tmp_path / "ck2.bin")
    write_checkpoint(path, p, 12, 1, {"adam_steps": 12}, m=m, v=v)
    p2, step, seed, extra, m2, v2 = read_checkpoint(path, with_optimizer=True)
    np.testing.assert_array_equal(p2, p)
    np.testing.assert_array_equal(m2, m)
    np.testing.assert_array_equal(v2, v)
    assert step == 12 and extra["adam_steps"] == 12
