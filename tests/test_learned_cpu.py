"""CPU checks of the learned-plasticity CPU reference (oracle/mlp_oracle.c): its
backward pass against finite differences, the strain-bound check against the
exact return map (plasticityOps.wgsl:7-48), and the training targets."""
import numpy as np


def test_oracle_gradient_matches_finite_differences(oracle_mod):
    rng = np.random.default_rng(0)
    P = rng.normal(0, 0.2, oracle_mod.MLP_PARAMS).astype(np.float32)
    x = rng.normal(0, 1, (7, 12)).astype(np.float32)
    t = rng.normal(0, 0.5, (7, 10)).astype(np.float32)
    # f64 mode (no BF16 rounding) and no uncertainty term: a smooth loss
    _, g = oracle_mod.mlp_gradient(P, x, t, 0.0, bf16=False)
    for i in rng.choice(P.size, 40, replace=False):
        p1, p2 = P.copy(), P.copy()
        p1[i] += np.float32(1e-3)
        p2[i] -= np.float32(1e-3)
        l1, _ = oracle_mod.mlp_gradient(p1, x, t, 0.0, bf16=False)
        l2, _ = oracle_mod.mlp_gradient(p2, x, t, 0.0, bf16=False)
        fd = (l1 - l2) / (float(p1[i]) - float(p2[i]))
        assert abs(fd - g[i]) <= 1e-4 * (abs(g[i]) + 1e-3), (i, fd, g[i])


def test_uncertainty_gradient_is_the_held_error(oracle_mod):
    """The uncertainty head regresses the error norm of the other outputs,
    held constant: its bias gradient is (2w/B) sum (y10 - e)."""
    rng = np.random.default_rng(1)
    P = rng.normal(0, 0.2, oracle_mod.MLP_PARAMS).astype(np.float32)
    x = rng.normal(0, 1, (5, 12)).astype(np.float32)
    t = rng.normal(0, 0.5, (5, 10)).astype(np.float32)
    y = oracle_mod.mlp_forward(P, x, bf16=False)
    e = np.sqrt(((y[:, :10] - t) ** 2).sum(1))
    _, g = oracle_mod.mlp_gradient(P, x, t, 0.25, bf16=False)
    want = (2 * 0.25 / 5) * (y[:, 10] - e).sum()
    assert abs(g[oracle_mod.MLP_PARAMS - 1] - want) <= 1e-9 + 1e-9 * abs(want)


def _random_trial(rng, theta_c, theta_s, spread):
    R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    V, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    s = rng.uniform(1 - theta_c - spread, 1 + theta_s + spread, 3)
    F = R @ np.diag(s) @ V.T
    return np.ascontiguousarray(F.T.reshape(9), np.float32)   # column-major, as stored


def test_strain_bound_check_is_sound(oracle_mod):
    """Whenever the check clears a trial state, the exact map returns it
    unchanged, bit for bit; states well outside the band are never cleared."""
    rng = np.random.default_rng(2)
    cleared = 0
    for _ in range(4000):
        tc = float(rng.uniform(0.015, 0.035))
        Fe = _random_trial(rng, tc, 7.5e-3, 0.01)
        ok, x, t, fe2, fp2 = oracle_mod.mlp_pair(Fe, np.eye(3, dtype=np.float32).reshape(9), 1e-4, tc, 7.5e-3)
        if oracle_mod.cert_elastic(Fe, tc, 7.5e-3):
            cleared += 1
            assert np.array_equal(fe2.view(np.uint32), Fe.view(np.uint32))
            assert np.all(t == 0.0)
    assert cleared > 200
    Fe = np.ascontiguousarray((np.eye(3) * 1.05).T.reshape(9), np.float32)
    assert not oracle_mod.cert_elastic(Fe, 0.025, 7.5e-3)


def test_pair_targets_encode_the_exact_map(oracle_mod):
    rng = np.random.default_rng(3)
    R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    F = R @ np.diag([0.96, 1.0, 1.02]) @ R.T      # a symmetric stretch outside the band
    Fe = np.ascontiguousarray(F.T.reshape(9), np.float32)
    Fp = np.ascontiguousarray(np.eye(3, dtype=np.float32).reshape(9))
    ok, x, t, fe2, fp2 = oracle_mod.mlp_pair(Fe, Fp, 1e-4, 0.025, 7.5e-3)
    assert ok
    assert np.allclose(x[:9], (Fe - np.eye(3, dtype=np.float32).reshape(9)) * 20)
    assert np.allclose(Fe + t[:9] / 100, fe2, atol=1e-6)
    assert np.isclose(t[9] / 100, np.log(np.linalg.det(fp2.reshape(3, 3).astype(np.float64))), atol=1e-5)
