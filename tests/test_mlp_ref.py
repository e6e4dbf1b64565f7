"""The CPU reference of the preconditioner MLP against finite differences (no GPU)."""
import numpy as np

from oracle import mlp_ref
from risq_b200.learned import PrecondMLP, normalise, raw_features
from risq_b200.fcidump import dets_from_ints, synthetic_integrals


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 3.1415927], dtype=np.float32)
    r = mlp_ref.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0          # exactly half an ulp: to even
    assert r[2] == np.float32(1.0 + 4 * 2**-8)  # above half: up
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-7


def test_reference_gradient_by_finite_differences():
    n_in, H = 6, 8
    rng = np.random.default_rng(0)
    m = PrecondMLP.init(2, hidden=H, seed=1)
    # exercise the gradient away from BF16 rounding effects: use weights exact in BF16
    p = mlp_ref.bf16_round(m.params)
    X = rng.standard_normal((20, n_in))
    t = rng.uniform(0.5, 2.0, 20)
    w = rng.uniform(0.1, 1.0, 20)
    loss, g = mlp_ref.loss_and_grad(p, X, t, w, n_in, H)
    # biases are not rounded: finite differences on them are exact in the model
    o = H * n_in
    for k in list(range(o, o + H)) + [len(p) - 1]:
        eps = 1e-3
        pp = p.astype(np.float64).copy(); pp[k] += eps
        pm = p.astype(np.float64).copy(); pm[k] -= eps
        lp = mlp_ref.loss_and_grad(pp.astype(np.float32), X, t, w, n_in, H)[0]
        lm = mlp_ref.loss_and_grad(pm.astype(np.float32), X, t, w, n_in, H)[0]
        assert abs((lp - lm) / (2 * eps) - g[k]) < 1e-3 * max(1.0, abs(g[k]))


def test_features_layout():
    ints = synthetic_integrals(6, 0)
    dets = dets_from_ints([(0b000111, 0b001011)])
    f = raw_features(dets, np.array([-3.0]), -4.0, ints)
    assert f.shape == (1, 14)
    np.testing.assert_array_equal(f[0, :6], [1, 1, 1, -1, -1, -1])
    np.testing.assert_array_equal(f[0, 6:12], [1, 1, -1, 1, -1, -1])
    assert f[0, 12] == 1.0
    hpp = [ints.h(k, k) for k in range(6)]
    assert abs(f[0, 13] - (hpp[0] + hpp[1] + hpp[2] + hpp[0] + hpp[1] + hpp[3])) < 1e-5
    g = normalise(f, np.array([1.0, 2.0, 0.0, 0.5], dtype=np.float32))
    assert g[0, 12] == 0.0 and abs(g[0, 13] - 0.5 * f[0, 13]) < 1e-6


def test_reference_factors_are_spin_flip_symmetric():
    norb, H = 5, 16
    m = PrecondMLP.init(norb, hidden=H, seed=2)
    rng = np.random.default_rng(3)
    m.params = (m.params + 0.1 * rng.standard_normal(m.params.shape)).astype(np.float32)
    X = rng.standard_normal((50, 2 * norb + 2)).astype(np.float32)
    f = mlp_ref.factors(m.params, X, m.n_in, H)
    fs = mlp_ref.factors(m.params, mlp_ref.swap_spins(X, norb), m.n_in, H)
    np.testing.assert_array_equal(f, fs)
    assert np.all((f >= 0.25) & (f <= 4.0))


def test_target_factors():
    from risq_b200.learned import target_factors
    diag = np.array([-1.0, 0.0, 1.0, 1.0, 1.0, 3.0])
    E = -1.0
    # gap: 0 (-> 1), 1, 2, 2, 2, 4
    S = np.array([-5.0, 0.0, -1.0, -1.9, -100.0, -3.0])
    f = target_factors(diag, S, E)
    assert f[0] == 1.0                      # H_ii <= E: no correction
    assert f[1] == 1.0                      # no coupling: DPR
    assert abs(f[2] - np.sqrt(2.0)) < 1e-6  # sqrt(gap / (gap - |S|))
    assert abs(f[3] - 4.0) < 1e-6           # denominator held at gap / 16 -> clip end
    assert f[4] == 4.0
    assert abs(f[5] - 2.0) < 1e-6


def test_adapted_network_equals_universal_network():
    """A universal-layout network (orbitals by h_pp rank, mean occupied h_pp) and its
    adaptation to one system's native layout give the same factors."""
    from risq_b200 import learned
    rng = np.random.default_rng(3)
    for norb, nel in [(12, 6), (24, 10)]:
        ints = synthetic_integrals(norb, 4)
        rows = []
        for _ in range(300):
            up = sum(1 << int(b) for b in rng.choice(norb, nel, replace=False))
            dn = sum(1 << int(b) for b in rng.choice(norb, nel, replace=False))
            rows.append((up, dn))
        dets = dets_from_ints(rows)
        diag = rng.uniform(-5.0, 5.0, len(dets))
        u = PrecondMLP.init(learned.NMAX, seed=2, fnorm=[0.5, 0.7, -3.0, 0.4])
        u.params = (u.params + 0.05 * rng.standard_normal(u.params.shape)).astype(np.float32)
        a = learned.adapt(u, ints, 2 * nel)
        assert a.n_in == 2 * norb + 2
        Xu = normalise(learned.universal_features(dets, diag, -1.0, ints), u.fnorm)
        Xa = normalise(raw_features(dets, diag, -1.0, ints), a.fnorm)
        fu = mlp_ref.factors(u.params, Xu, u.n_in, u.hidden)
        fa = mlp_ref.factors(a.params, Xa, a.n_in, a.hidden)
        # the same sums up to FP32 order (an activation may round to the neighbouring BF16 value)
        np.testing.assert_allclose(fa, fu, rtol=2e-3, atol=1e-6)
        assert np.std(fu) > 1e-3
