"""Matrix-free storage (RISQGPU_MATRIX_FREE): sigma finds and evaluates every row's
elements itself, with nothing stored.  Checked against the oracle's sparse H and the
stored FP64 build: the same elements, so the same sigma to rounding and the same
Davidson energies; one warp per row with a private sum, so bitwise reproducible."""
import numpy as np
import pytest

from oracle import oracle as O
from risq_b200 import GpuHam, _capi, learned
from risq_b200.fcidump import synthetic_integrals, dets_from_ints
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b)))


@pytest.mark.parametrize("name", ["be2", "f2"])
def test_matrix_free_sigma_matches_oracle(name):
    ints, p = H.golden_system(name)
    _, dets, coeffs, diag, _ = H.oracle_hci(name)
    sp = O.Sparse().build(H.oracle_ham(ints, p["norb_core"]), dets, diag, 0)
    rng = np.random.default_rng(11)
    X = np.column_stack([coeffs, rng.standard_normal(len(dets))])
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        ref = g.matrix_matrix_prod(X)
        hs = g.build(_capi.MATRIX_FREE)
        assert hs["nnz_upper"] == 0 and g.memory_used()[0] > 0
        Y = g.matrix_matrix_prod(X)
        for c in range(X.shape[1]):
            assert _rel(Y[:, c], sp.mv(X[:, c])) <= 1e-11   # the oracle's SparseMatUpperTri product
            assert _rel(Y[:, c], ref[:, c]) <= 1e-13        # the stored FP64 sigma, other sum order
        # one private sum per row: the same bits every call and after a rebuild
        np.testing.assert_array_equal(g.matrix_matrix_prod(X), Y)
        g.build(_capi.MATRIX_FREE)
        np.testing.assert_array_equal(g.matrix_matrix_prod(X), Y)


@pytest.mark.parametrize("name", ["be2", "f2"])
def test_matrix_free_davidson_matches_golden(name):
    gold = H.golden_energies()["systems"][name]["e_var"]
    ints, p = H.golden_system(name)
    _, dets, coeffs, diag, _ = H.oracle_hci(name)
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        r64 = g.davidson(1, None, 1e-4, 1e-8, 50)
        g.build(_capi.MATRIX_FREE)
        r = g.davidson(1, None, 1e-4, 1e-8, 50)
        assert r.converged and abs(r.stats["iters"] - r64.stats["iters"]) <= 1
        assert abs(r.eigenvalues[0] - r64.eigenvalues[0]) < 1e-10
        assert abs(r.eigenvalues[0] - gold) < 1e-6   # tests/integration_test_suite.rs:34-84
        r2 = g.davidson(1, None, 1e-4, 1e-8, 50)
        assert r2.eigenvalues[0] == r.eigenvalues[0]
        np.testing.assert_array_equal(r2.eigenvectors, r.eigenvectors)


def test_matrix_free_with_table_search():
    """Alpha partner groups of more than 256 determinants go through the determinant
    table in the search (n12 6a6b eps 1e-3, groups up to 591): sigma against the
    oracle's sparse H."""
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-3)
    _, counts = np.unique(dets[:, 0], return_counts=True)
    assert (counts > 256).sum() > 0
    sp = O.Sparse().build(H.oracle_ham(ints, 0), dets, diag, 0)
    x = np.random.default_rng(2).standard_normal(len(dets))
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.MATRIX_FREE)
        y = g.matrix_vector_prod(x)
    assert _rel(y, sp.mv(x)) <= 1e-11


def test_matrix_free_two_word_strings():
    """norb 70: two-word (u128) strings through the same search."""
    norb = 70
    ints = synthetic_integrals(norb, 3)
    rng = np.random.default_rng(70)
    rows = []
    for _ in range(40):
        up = sum(1 << int(b) for b in rng.choice(12, 5, replace=False)) | (1 << 66)
        dn = sum(1 << int(b) for b in rng.choice(12, 5, replace=False)) | (1 << 65)
        rows.append((up, dn))
    base = dets_from_ints(rows)
    d1, d2 = H.random_connected_pairs(base, rng, 600, norb)
    dets = np.unique(np.vstack([base, d1, d2]), axis=0)
    oh = H.oracle_ham(ints, 0)
    diag = oh.diag(dets)
    sp = O.Sparse().build(oh, dets, diag, 0)
    x = rng.standard_normal(len(dets))
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.MATRIX_FREE)
        y = g.matrix_vector_prod(x)
    assert _rel(y, sp.mv(x)) <= 1e-11


def test_matrix_free_rejects_what_needs_stored_elements():
    ints, p = H.golden_system("be")
    _, dets, coeffs, diag, _ = H.oracle_hci("be")
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.MATRIX_FREE)
        for call in (lambda: g.davidson(1, mode=_capi.MODE_MIXED), g.export_upper,
                     lambda: g.export_rows(np.arange(3)), lambda: learned.self_energy(g, -14.6)):
            with pytest.raises(_capi.RisqGpuError) as ei:
                call()
            assert ei.value.code == _capi.ERR_INVALID
        assert g.davidson(1, coeffs, 1e-4, 1e-8, 50).converged  # the handle stays usable


def test_variational_falls_back_to_matrix_free():
    """A memory bound below what the final set's columns need drives precision -1 down
    the whole chain (FP64 rows, upper triangle, columns, matrix-free) to the same
    wavefunction."""
    ints, p = H.golden_system("f2")
    kw = dict(ncore=p["norb_core"], max_iter=20, dav_max_iter=50)
    with GpuHam(ints) as g:
        e0, d0, c0, _, log0 = g.variational(p["nup"], p["ndn"], p["eps_var"], precision=-1, **kw)
    with GpuHam(ints) as g:
        g.variational(p["nup"], p["ndn"], p["eps_var"], precision=_capi.COLS, **kw)
        cols_used, _ = g.memory_used()
    with GpuHam(ints) as g:
        g.variational(p["nup"], p["ndn"], p["eps_var"], precision=_capi.MATRIX_FREE, **kw)
        mf_used, _ = g.memory_used()
    assert mf_used < cols_used
    with GpuHam(ints) as g:
        g.set_memory_limit(cols_used - 1)
        e1, d1, c1, _, log1 = g.variational(p["nup"], p["ndn"], p["eps_var"], precision=-1, **kw)
        assert g.memory_used()[0] <= cols_used
    assert log1[-1]["storage"] == _capi.MATRIX_FREE
    assert log0[-1]["storage"] == _capi.FP64
    assert np.array_equal(d0, d1)
    assert abs(e0 - e1) < 1e-9
