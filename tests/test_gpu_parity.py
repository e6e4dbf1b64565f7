"""CUDA path against the CPU oracle: elements, connection set, sigma, Davidson."""
import numpy as np
import pytest

from oracle import oracle as O
from risq_b200 import GpuHam, _capi
from risq_b200.fcidump import synthetic_integrals
from tests import helpers as H

pytestmark = pytest.mark.gpu

GOLDEN = ["he2", "be", "li2", "be2"]


def _gpu(ints):
    return GpuHam(ints, 0)


@pytest.mark.parametrize("name", GOLDEN + ["f2"])
def test_elements_bitwise(name):
    ints, p = H.golden_system(name)
    _, dets, _, _, _ = H.oracle_hci(name)
    oh = H.oracle_ham(ints, p["norb_core"])
    rng = np.random.default_rng(7)
    d1, d2 = H.random_connected_pairs(dets[: min(len(dets), 400)], rng, 3000, ints.norb)
    with _gpu(ints) as g:
        np.testing.assert_array_equal(g.ham_off_diag_no_excite(d1, d2), oh.off_diag(d1, d2))
        np.testing.assert_array_equal(g.ham_diag(dets[:500]), oh.diag(dets[:500]))


@pytest.mark.parametrize("norb", [12, 70, 100])
def test_elements_bitwise_synthetic(norb):
    """norb 70 and 100 exercise the two-word (u128) strings."""
    ints = synthetic_integrals(norb, 2)
    oh = H.oracle_ham(ints, 0)
    rng = np.random.default_rng(norb)
    rows = []
    for _ in range(60):
        up = sum(1 << int(b) for b in rng.choice(norb, 5, replace=False))
        dn = sum(1 << int(b) for b in rng.choice(norb, 5, replace=False))
        rows.append((up, dn))
    from risq_b200.fcidump import dets_from_ints
    base = dets_from_ints(rows)
    d1, d2 = H.random_connected_pairs(base, rng, 2000, norb)
    with _gpu(ints) as g:
        np.testing.assert_array_equal(g.ham_off_diag_no_excite(d1, d2), oh.off_diag(d1, d2))
        np.testing.assert_array_equal(g.ham_diag(base), oh.diag(base))


def _check_csr(g_csr, o_csr):
    grp, gcols, gvals, gdiag = g_csr
    orp, ocols, ovals, odiag = o_csr
    np.testing.assert_array_equal(grp, orp)         # same row counts
    np.testing.assert_array_equal(gcols, ocols)     # same connection set
    assert np.max(np.abs(gvals - ovals), initial=0.0) <= 1e-12
    np.testing.assert_array_equal(np.sign(gvals), np.sign(ovals))
    np.testing.assert_array_equal(gdiag, odiag)
    return np.mean(gvals == ovals) if len(gvals) else 1.0


@pytest.mark.parametrize("name", GOLDEN + ["f2"])
def test_connection_set_matches_oracle(name):
    ints, p = H.golden_system(name)
    _, dets, _, diag, _ = H.oracle_hci(name)
    sp = O.Sparse().build(H.oracle_ham(ints, p["norb_core"]), dets, diag, 0, builder=0)
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        st = g.build(_capi.FP64, _capi.BUILDER_AUTO)
        assert st["nnz_upper"] == sp.nnz
        frac = _check_csr(g.export_upper(), sp.export())
        assert frac == 1.0  # elements are bitwise equal, not only within 1e-12


def test_connection_set_synthetic():
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-4)
    sp = O.Sparse().build(H.oracle_ham(ints, 0), dets, diag, 0, builder=0)
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        assert _check_csr(g.export_upper(), sp.export()) == 1.0


@pytest.mark.parametrize("name", ["be", "li2", "be2", "f2"])
def test_incremental_build_matches_reference_history(name):
    """Replay the HCI growth: each build extends the stored H exactly like
    sparse_optimize does across iterations (legacy rule while N <= 100)."""
    ints, p = H.golden_system(name)
    hci = O.Hci(H.oracle_ham(ints, p["norb_core"]), p["nup"], p["ndn"], p["eps_var"])
    hci.run(20)
    dets, _, diag = hci.export()
    sizes = [l["ndets"] for l in hci.log()]
    ref = O.Sparse()
    ref.ptr = O.lib().or_hci_sparse(hci.ptr)  # borrowed: keep hci alive
    o_csr = ref.export()
    ref.ptr = None
    with _gpu(ints) as g:
        prev = 0
        for n in sizes:
            if n == prev:
                continue
            g.set_dets(dets[:n], prev, diag[:n])
            g.build(_capi.FP64, _capi.BUILDER_AUTO)
            prev = n
        assert _check_csr(g.export_upper(), o_csr) == 1.0


@pytest.mark.parametrize("name", ["li2", "be2"])
def test_legacy_builder_rule(name):
    ints, p = H.golden_system(name)
    _, dets, _, diag, _ = H.oracle_hci(name)
    sp = O.Sparse().build(H.oracle_ham(ints, p["norb_core"]), dets, diag, 0, builder=2)
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64, _capi.BUILDER_LEGACY)
        assert _check_csr(g.export_upper(), sp.export()) == 1.0


@pytest.mark.parametrize("name", ["be2", "f2"])
def test_sigma_matches_oracle(name):
    ints, p = H.golden_system(name)
    _, dets, coeffs, diag, _ = H.oracle_hci(name)
    sp = O.Sparse().build(H.oracle_ham(ints, p["norb_core"]), dets, diag, 0)
    rng = np.random.default_rng(1)
    X = np.column_stack([coeffs, rng.standard_normal(len(dets))])
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        Y = g.matrix_matrix_prod(X)
        for c in range(X.shape[1]):
            ref = sp.mv(X[:, c])
            assert np.max(np.abs(Y[:, c] - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref)))
        g.build(_capi.MIXED)
        y = g.matrix_vector_prod(X[:, 1])
        ref = sp.mv(X[:, 1])
        assert np.max(np.abs(y - ref)) <= 1e-11 * np.max(np.abs(ref))  # FP32 + remainder ~ FP64


@pytest.mark.parametrize("name", GOLDEN + ["f2"])
def test_davidson_matches_golden(name):
    """Davidson on the final HCI set, started from the previous coefficients the
    way sparse_optimize does (var/davidson.rs:69-96)."""
    gold = H.golden_energies()["systems"][name]["e_var"]
    ints, p = H.golden_system(name)
    e_or, dets, coeffs, diag, _ = H.oracle_hci(name)
    sp = O.Sparse().build(H.oracle_ham(ints, p["norb_core"]), dets, diag, 0)
    rc, ev_or, _, st_or = sp.davidson(1, None, 1e-4, 1e-8, 50)
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        r = g.davidson(1, None, 1e-4, 1e-8, 50)
        assert r.converged
        assert abs(r.eigenvalues[0] - ev_or[0]) < 1e-6        # 1 uHa vs the oracle Davidson
        assert abs(r.eigenvalues[0] - gold) < 1e-6            # golden E_var, tests/integration_test_suite.rs:13
        v = r.eigenvectors[:, 0]
        assert abs(np.linalg.norm(v) - 1) < 1e-8
        assert abs(abs(v @ coeffs) - 1) < 1e-4
        # mixed precision on the same set: within 1 uHa of FP64
        g.build(_capi.MIXED)
        m = g.davidson(1, None, 1e-4, 1e-8, 50, mode=_capi.MODE_MIXED)
        assert m.converged
        assert abs(m.eigenvalues[0] - r.eigenvalues[0]) < 1e-6
        assert m.stats["n_sigma_fp64"] < m.stats["n_sigma"]


def test_sparse_optimize_entry_point():
    ints, p = H.golden_system("be2")
    e_or, dets, coeffs, diag, log = H.oracle_hci("be2")
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        e, c, hs, ds = g.sparse_optimize(coeffs, 1e-4, 1e-8)
        assert abs(e - e_or) < 1e-6
        assert hs["nnz_upper"] > 0 and ds["converged"] == 1


def test_two_roots_against_dense():
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-4)
    sp = O.Sparse().build(H.oracle_ham(ints, 0), dets, diag, 0)
    n = len(dets)
    if n > 6000:
        dets, diag = dets[:6000], diag[:6000]
        sp = O.Sparse().build(H.oracle_ham(ints, 0), dets, diag, 0)
        n = 6000
    rp, cols, vals, dg = sp.export()
    A = np.diag(dg)
    for r in range(n):
        A[r, cols[rp[r]:rp[r + 1]]] = vals[rp[r]:rp[r + 1]]
    A = np.triu(A) + np.triu(A, 1).T
    w = np.linalg.eigvalsh(A)[:2]
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        r = g.davidson(2, None, 1e-6, 1e-10, 200)
        assert r.converged
        np.testing.assert_allclose(r.eigenvalues, w, atol=1e-8)


def test_invalid_inputs_are_rejected():
    ints, p = H.golden_system("be")
    _, dets, _, diag, _ = H.oracle_hci("be")
    with _gpu(ints) as g:
        bad = dets.copy()
        bad[0, 0] |= np.uint64(1) << np.uint64(ints.norb)  # orbital index == norb
        with pytest.raises(_capi.RisqGpuError):
            g.set_dets(bad, 0, diag)
        dup = np.vstack([dets, dets[:1]])
        with pytest.raises(_capi.RisqGpuError):
            g.set_dets(dup, 0, np.append(diag, diag[0]))
        g.set_dets(dets, 0, diag)
        with pytest.raises(_capi.RisqGpuError):
            g.matrix_vector_prod(np.ones(len(dets)))  # before build
        with pytest.raises(_capi.RisqGpuError):
            g.davidson(1, mode=_capi.MODE_MIXED)  # before build
        g.build(_capi.FP64)
        with pytest.raises(_capi.RisqGpuError):
            g.davidson(1, mode=_capi.MODE_MIXED)  # FP64 storage cannot run the FP32 sigma
        with pytest.raises(_capi.RisqGpuError):
            g.set_dets(dets[:5], 3, diag[:5])  # n_stored_h must equal the previous size


@pytest.mark.parametrize("name", ["be2", "f2"])
def test_columns_only_build_and_recomputed_sigma(name):
    """COLS storage keeps the columns; sigma recomputes the FP64 elements, which are
    bitwise the stored ones, so export and sigma match the FP64 build."""
    ints, p = H.golden_system(name)
    _, dets, coeffs, diag, _ = H.oracle_hci(name)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(len(dets))
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        ref_csr = g.export_upper()
        ref_y = g.matrix_vector_prod(x)
        r64 = g.davidson(1, None, 1e-4, 1e-8, 50)
        g.build(_capi.COLS)
        csr = g.export_upper()
        for a, b in zip(csr, ref_csr):
            np.testing.assert_array_equal(a, b)
        y = g.matrix_vector_prod(x)
        assert np.max(np.abs(y - ref_y)) <= 1e-12 * np.max(np.abs(ref_y))
        r = g.davidson(1, None, 1e-4, 1e-8, 50)
        assert abs(r.eigenvalues[0] - r64.eigenvalues[0]) < 1e-9
        # FP32 storage: FP32 stage + closing sweeps with the recomputed FP64 elements
        g.build(_capi.FP32)
        m = g.davidson(1, None, 1e-4, 1e-8, 50, mode=_capi.MODE_MIXED)
        assert m.converged and abs(m.eigenvalues[0] - r64.eigenvalues[0]) < 1e-6
        assert 0 < m.stats["n_sigma_fp64"] < m.stats["n_sigma"]
        f = g.davidson(1, None, 1e-4, 1e-8, 50, mode=_capi.MODE_FP32)
        assert f.converged and f.stats["n_sigma_fp64"] == 0


@pytest.mark.parametrize("name", ["be2", "f2"])
def test_upper_triangle_storage(name):
    """FP64_UPPER / MIXED_UPPER store each pair once (SparseMatUpperTri's layout),
    regrouped into row-panel x column-window tiles: same set and values as the
    both-triangle build, same sigma to rounding."""
    ints, p = H.golden_system(name)
    _, dets, coeffs, diag, _ = H.oracle_hci(name)
    x = np.random.default_rng(9).standard_normal(len(dets))
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        ref_csr = g.export_upper()
        ref_y = g.matrix_vector_prod(x)
        r64 = g.davidson(1, None, 1e-4, 1e-8, 50)
        st = g.build(_capi.FP64_UPPER)
        assert st["nnz_upper"] == len(ref_csr[1])
        for a, b in zip(g.export_upper(), ref_csr):
            np.testing.assert_array_equal(a, b)
        y = g.matrix_vector_prod(x)
        assert np.max(np.abs(y - ref_y)) <= 1e-12 * np.max(np.abs(ref_y))
        r = g.davidson(1, None, 1e-4, 1e-8, 50)
        assert abs(r.eigenvalues[0] - r64.eigenvalues[0]) < 1e-9
        g.build(_capi.MIXED_UPPER)
        m = g.davidson(1, None, 1e-4, 1e-8, 50, mode=_capi.MODE_MIXED)
        assert m.converged and abs(m.eigenvalues[0] - r64.eigenvalues[0]) < 1e-6
        g.build(_capi.FP32_UPPER)
        f = g.davidson(1, None, 1e-4, 1e-8, 50, mode=_capi.MODE_FP32)
        assert f.converged and abs(f.eigenvalues[0] - r64.eigenvalues[0]) < 1e-4
        with pytest.raises(_capi.RisqGpuError):
            g.davidson(1, None, 1e-4, 1e-8, 50, mode=_capi.MODE_MIXED)  # FP32 upper has no FP64 sigma
        with pytest.raises(_capi.RisqGpuError):
            g.set_dets(dets, len(dets), diag)  # no incremental extension of an upper build


def test_upper_triangle_sigma_on_large_alpha_groups():
    """Upper-triangle sigma on a set whose alpha groups hold more than 1024
    determinants (n20 8a8b, eps 1e-3, 551,147 determinants): FP64 against the
    both-triangle kernel (checked against the oracle above), FP32 and the FP32 +
    remainder storage against the same reference."""
    from risq_b200.fcidump import synthetic_integrals
    ints = synthetic_integrals(20, 0)
    with _gpu(ints) as g:
        e, dets, c, diag, log = g.variational(8, 8, 1e-3, dav_max_iter=2000)
        up = dets[:, 0]
        _, counts = np.unique(up, return_counts=True)
        assert counts.max() > 1024  # groups larger than a warp's and a block's share of rows
        x = np.random.default_rng(3).standard_normal(len(dets))
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        ref = g.matrix_vector_prod(x)
        scale = np.max(np.abs(ref))
        g.build(_capi.FP64_UPPER)
        y = g.matrix_vector_prod(x)
        assert np.max(np.abs(y - ref)) <= 1e-12 * scale
        g.build(_capi.MIXED_UPPER)
        y = g.matrix_vector_prod(x)  # FP64 sigma over FP32 value + FP32 remainder
        assert np.max(np.abs(y - ref)) <= 1e-11 * scale
        import torch
        perm_free = torch.tensor(x, dtype=torch.float32, device="cuda")  # FP32 sigma, internal order
        y32 = torch.empty_like(perm_free)
        g.build(_capi.FP32)
        g.sigma_device(perm_free.data_ptr(), y32.data_ptr(), 1)
        ref32 = y32.double().cpu().numpy()
        g.build(_capi.FP32_UPPER)
        g.sigma_device(perm_free.data_ptr(), y32.data_ptr(), 1)
        assert np.max(np.abs(y32.double().cpu().numpy() - ref32)) <= 1e-5 * np.max(np.abs(ref32))


@pytest.mark.parametrize("prec", [_capi.FP64, _capi.FP64_UPPER])
def test_connection_set_with_table_search(prec):
    """Alpha partner groups larger than 256 determinants are searched through the
    (alpha group, beta string) table instead of scanned (build_h.cu): on a set with
    such groups (n12 6a6b eps 1e-3, 30,925 dets, groups up to 591) the stored set and
    every element equal the oracle's sparse H bitwise."""
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-3)
    _, counts = np.unique(dets[:, 0], return_counts=True)
    assert (counts > 256).sum() > 0
    sp = O.Sparse().build(H.oracle_ham(ints, 0), dets, diag, 0)
    orp, ocols, ovals, _ = sp.export()
    with _gpu(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(prec)
        rp, cols, vals, _ = g.export_upper()
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(cols, ocols)
    np.testing.assert_array_equal(vals, ovals)
