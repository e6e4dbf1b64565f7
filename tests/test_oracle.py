"""The CPU oracle against the reference's own golden vectors and invariants (no GPU)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H


def _popcount_parity(n):
    return 1 - 2 * (bin(n).count("1") & 1)


def test_parity_known_answers():
    # src/utils/bits.rs:197-211
    for v in [14, 15, 27, 1919, 4958202, 15 << 64, 1 << 127, (1 << 126) + (1 << 65)]:
        lo, hi = v & (2**64 - 1), v >> 64
        assert O.lib().or_parity(lo, hi) == _popcount_parity(v)


def test_combine_4_symmetry():
    rng = np.random.default_rng(1)
    for _ in range(200):
        p, q, r, s = (int(x) for x in rng.integers(1, 40, 4))
        ref = O.lib().or_combine_4(p, q, r, s)
        for perm in [(q, p, r, s), (p, q, s, r), (r, s, p, q), (s, r, q, p)]:
            assert O.lib().or_combine_4(*perm) == ref
        assert O.combine_4(p, q, r, s) == ref


@pytest.mark.parametrize("name", ["be", "he2", "li2", "be2"])
def test_golden_energy(name):
    # tests/integration_test_suite.rs:13 (tolerance) and :34/:44/:64/:74 (values)
    gold = H.golden_energies()["systems"][name]["e_var"]
    e, dets, coeffs, diag, log = H.oracle_hci(name)
    assert abs(e - gold) < 1e-6
    assert abs(e - gold) < 1e-9  # the restatement is much closer than the tolerance


def test_golden_energy_f2():
    # tests/integration_test_suite.rs:84 (the reference skips it as too slow for CI)
    gold = H.golden_energies()["systems"]["f2"]["e_var"]
    e, dets, *_ = H.oracle_hci("f2")
    assert abs(e - gold) < 1e-6
    assert len(dets) == 69028


def test_reproducible():
    # tests/integration_test_suite.rs:413-440: identical energy and det count across runs
    ints, p = H.golden_system("be")
    runs = []
    for _ in range(2):
        hci = O.Hci(H.oracle_ham(ints, p["norb_core"]), p["nup"], p["ndn"], p["eps_var"])
        runs.append((hci.run(20), hci.ndets))
    assert runs[0] == runs[1]


def _csr(sp):
    rp, cols, vals, diag = sp.export()
    return H.csr_to_dict(rp, cols, vals)


def test_grouped_singles_match_bruteforce():
    # fast_ham.rs:473-517 scans all N for each new det; the grouped scan visits the same pairs
    _, dets, _, diag, _ = H.oracle_hci("be2")
    ints, p = H.golden_system("be2")
    h = H.oracle_ham(ints, p["norb_core"])
    a = O.Sparse().build(h, dets, diag, 0, builder=1, grouped_singles=False)
    b = O.Sparse().build(h, dets, diag, 0, builder=1, grouped_singles=True)
    assert _csr(a) == _csr(b)


@pytest.mark.parametrize("name", ["be", "li2"])
def test_legacy_and_fast_builders_agree(name):
    # ham_gen.rs (n <= 100) and fast_ham.rs store the same set on spin-flip-closed sets,
    # except singles with 0 < |H| <= 1e-12 which only the legacy builder keeps
    _, dets, _, diag, _ = H.oracle_hci(name)
    ints, p = H.golden_system(name)
    h = H.oracle_ham(ints, p["norb_core"])
    fast = _csr(O.Sparse().build(h, dets, diag, 0, builder=1))
    legacy = _csr(O.Sparse().build(h, dets, diag, 0, builder=2))
    assert set(fast) <= set(legacy)
    for k in set(legacy) - set(fast):
        assert abs(legacy[k]) <= 1e-12
    for k in fast:
        assert fast[k] == legacy[k]


def test_incremental_build_equals_full_fast():
    _, dets, _, diag, log = H.oracle_hci("be2")
    ints, p = H.golden_system("be2")
    h = H.oracle_ham(ints, p["norb_core"])
    n1 = log[1]["ndets"]
    inc = O.Sparse().build(h, dets[:n1], diag[:n1], 0, builder=1)
    inc.build(h, dets, diag, n1, builder=1)
    full = O.Sparse().build(h, dets, diag, 0, builder=1)
    assert _csr(inc) == _csr(full)


def test_hci_sparse_is_symmetric_and_complete():
    """Every pair at degree 1-2 with a non-zero element is stored once (upper triangle)."""
    _, dets, _, diag, _ = H.oracle_hci("li2")
    ints, p = H.golden_system("li2")
    h = H.oracle_ham(ints, p["norb_core"])
    got = _csr(O.Sparse().build(h, dets, diag, 0, builder=1))
    n = len(dets)
    i, j = np.triu_indices(n, 1)
    vals = h.off_diag(dets[i], dets[j])
    want = {}
    for a, b, v in zip(i, j, vals):
        if v != 0.0:
            want[(int(a), int(b))] = v
    # singles with |H| <= 1e-12 are dropped by the fast builder only
    assert set(got) <= set(want)
    for k in set(want) - set(got):
        assert abs(want[k]) <= 1e-12
    for k, v in got.items():
        assert v == want[k]


def test_davidson_matches_dense_eigh():
    _, dets, _, diag, _ = H.oracle_hci("be2")
    ints, p = H.golden_system("be2")
    sp = O.Sparse().build(H.oracle_ham(ints, p["norb_core"]), dets, diag, 0)
    rp, cols, vals, dg = sp.export()
    n = len(dg)
    A = np.diag(dg)
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            A[r, cols[k]] = A[cols[k], r] = vals[k]
    w = np.linalg.eigvalsh(A)
    rc, ev, vec, st = sp.davidson(1, None, 1e-4, 1e-8, 50)
    assert rc == 0 and st["converged"]
    assert abs(ev[0] - w[0]) < 1e-6
    x = np.random.default_rng(0).standard_normal(n)
    np.testing.assert_allclose(sp.mv(x), A @ x, rtol=1e-12, atol=1e-12)


def test_mgs_orthonormality():
    # modified_gram_schmidt.rs:45-67
    rng = np.random.default_rng(3)
    ok, B = O.mgs(rng.random((20, 20)), 0, 20)
    assert ok
    assert np.allclose(B.T @ B, np.eye(20), atol=1e-8)
    arr = np.array([[1.0, 1.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 2.0]])
    ok, B = O.mgs(arr, 1, 3)
    assert ok
    assert np.allclose(B.T @ B, np.eye(3), atol=1e-8)


def test_sym_eig_matches_numpy():
    rng = np.random.default_rng(4)
    for n in (1, 2, 5, 11, 12):
        M = rng.standard_normal((n, n))
        M = M + M.T
        w, Y = O.sym_eig(M)
        np.testing.assert_allclose(w, np.linalg.eigvalsh(M), atol=1e-12)
        np.testing.assert_allclose(M @ Y, Y * w, atol=1e-10)


def test_dense_davidson_two_roots():
    rng = np.random.default_rng(5)
    n = 300
    A = np.diag(np.arange(n, dtype=float)) + 0.01 * rng.standard_normal((n, n))
    A = (A + A.T) / 2
    rc, ev, vec, st = O.davidson_dense(A, 2, None, 1e-8, 1e-12, 200)
    assert rc == 0
    np.testing.assert_allclose(ev, np.linalg.eigvalsh(A)[:2], atol=1e-9)


def test_parallel_oracle_matches_serial():
    # the multi-threaded build and sigma of the CPU baseline: the serial fast builder's
    # pairs and values, and the same energy
    _, dets, coeffs, diag, _ = H.oracle_hci("f2")
    ints, p = H.golden_system("f2")
    ham = H.oracle_ham(ints, p["norb_core"])
    s1 = O.Sparse().build(ham, dets, diag, 0, builder=1)
    s2 = O.Sparse().build_par(ham, dets, diag)
    for a, b in zip(s1.export(), s2.export()):
        assert np.array_equal(a, b)
    x = np.random.default_rng(5).standard_normal(len(dets))
    y1, y2 = s1.mv(x), s2.mv_par(x)
    assert np.max(np.abs(y1 - y2)) <= 1e-12 * np.max(np.abs(y1))
    r1 = s1.davidson(1, coeffs, 1e-4, 1e-8, 200)
    r2 = s2.davidson(1, coeffs, 1e-4, 1e-8, 200, parallel=True)
    assert r1[0] == 0 and r2[0] == 0
    assert abs(r1[1][0] - r2[1][0]) < 1e-10


def test_reference_davidson_stays_in_the_spin_flip_even_sector():
    """On the synthetic n24 10a10b integrals the lowest state of an HCI space is odd
    under spin flip, while the reference's start vectors (determinants 0 and 1,
    generate_subspace, davidson.rs:318-338) are even: in exact arithmetic its DPR
    Davidson stays in the even sector and converges to the second eigenvalue.  A solve
    whose rounding breaks the symmetry (FP32 sums) can reach the lower, odd state."""
    import scipy.sparse as sps
    import scipy.sparse.linalg as sla
    from risq_b200.fcidump import synthetic_integrals
    ints = synthetic_integrals(24, 0)
    oh = O.Ham.from_arrays(ints.norb, 0, ints.nuc, ints.one_body, ints.two_body)
    hci = O.Hci(oh, 10, 10, 1e-2).set_options(2000)
    for _ in range(3):
        hci.step()
    dets, coeffs, diag = hci.export()
    n = len(dets)
    sp = O.Sparse().build(oh, dets, diag, 0)
    rp, cols, vals, dg = sp.export()
    U = sps.csr_matrix((vals, (np.repeat(np.arange(n), np.diff(rp)), cols)), shape=(n, n))
    w, V = sla.eigsh(U + U.T + sps.diags(dg), k=2, which="SA", v0=np.random.default_rng(0).standard_normal(n),
                     tol=1e-12)
    order = np.argsort(w)
    w, V = w[order], V[:, order]
    key = {tuple(int(v) for v in d): i for i, d in enumerate(dets)}
    flip = np.array([key[(int(d[2]), int(d[3]), int(d[0]), int(d[1]))] for d in dets])
    rc, ev, vec, st = sp.davidson(1, None, 1e-4, 1e-8, 2000)
    assert abs(ev[0] - w[1]) < 1e-7                    # the reference converges to the second state
    assert w[0] < w[1] - 0.1                           # a lower state exists
    assert V[:, 0] @ V[flip, 0] < -0.999               # odd under spin flip
    assert V[:, 1] @ V[flip, 1] > 0.999                # the reference's state is even
    assert abs(V[0, 0]) < 1e-12 and abs(V[1, 0]) < 1e-12  # no overlap with the start vectors
