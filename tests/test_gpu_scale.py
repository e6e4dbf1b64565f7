"""Parity at the benchmarked scale, and reproducibility of the upper-triangle path.

The benchmark's set (bench.py config 1: n20 8a8b eps_var 5e-5, 9,150,723
determinants, 1.1e10 stored pairs) is far too large to export whole, so a sample
of its rows is checked against the oracle's brute-force rows over the full set
(every determinant tested, no lookup tables: a method independent of the GPU's
grouped search), and the energy of an earlier HCI iteration's space, which the
CPU oracle solves in seconds, against the oracle's Davidson.  The reference pins
bit-identical energies across runs (tests/integration_test_suite.rs:413-440); the
upper-triangle FP64 sigma sums in 64-bit fixed point, and so does the FP32 one of a
handle set reproducible, so repeated solves must agree bitwise.
"""
import numpy as np
import pytest

from oracle import oracle as O
from risq_b200 import GpuHam, _capi
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config1():
    import bench
    return bench.det_set(1, 0, log=lambda *a: None)


def _rows_by_row(r, c, v, rows):
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    out = {}
    lo = np.searchsorted(r, rows, side="left")
    hi = np.searchsorted(r, rows, side="right")
    for row, a, b in zip(rows, lo, hi):
        out[int(row)] = (c[a:b], v[a:b])
    return out


def test_config1_sampled_rows_match_oracle(config1):
    ints, dets, diag, e, vlog = config1
    assert len(dets) > 5_000_000
    oh = O.Ham.from_arrays(ints.norb, 0, ints.nuc, ints.one_body, ints.two_body)
    rows = np.random.default_rng(7).choice(len(dets), 256, replace=False)
    ref = O.rows_bruteforce(oh, dets, rows)
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        for prec in (_capi.FP64_UPPER, _capi.MIXED_UPPER):
            g.build(prec)
            got = _rows_by_row(*g.export_rows(rows), rows)
            for row, (oc, ov) in zip(rows, ref):
                gc, gv = got[int(row)]
                np.testing.assert_array_equal(gc, oc)  # the connection set, bitwise
                if prec == _capi.FP64_UPPER:
                    np.testing.assert_array_equal(gv, ov)  # FP64 Slater-Condon, bitwise
                else:  # FP32 value + FP32 remainder carries 48 bits of the FP64 element
                    assert np.all(np.abs(gv - ov) <= 2.0 ** -46 * np.abs(ov) + 1e-300)


def test_config1_prefix_energy_matches_oracle(config1):
    import bench
    ints, dets, diag, e, vlog = config1
    k, n = bench.sample_iteration([int(r["n_dets"]) for r in vlog])
    assert 10_000 < n < len(dets)
    sd, sg = dets[:n], diag[:n]
    oh = O.Ham.from_arrays(ints.norb, 0, ints.nuc, ints.one_body, ints.two_body)
    sp = O.Sparse().build_par(oh, sd, sg)
    rc, ev, _, st = sp.davidson(1, None, 1e-4, 1e-8, bench.DAV_MAX_ITER, parallel=True)
    assert rc == 0
    with GpuHam(ints) as g:
        g.set_dets(sd, 0, sg)
        for prec in (_capi.FP64, _capi.FP64_UPPER):
            g.build(prec)
            assert g.nnz()[0] == sp.nnz
            r = g.davidson(1, None, 1e-4, 1e-8, bench.DAV_MAX_ITER)
            assert r.converged and abs(r.eigenvalues[0] - ev[0]) < 1e-6


@pytest.mark.parametrize("prec,mode", [(_capi.FP64_UPPER, _capi.MODE_FP64), (_capi.MIXED_UPPER, _capi.MODE_MIXED)])
def test_upper_triangle_solves_are_bitwise_reproducible(prec, mode):
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-3)
    x = np.random.default_rng(4).standard_normal(len(dets))
    with GpuHam(ints) as g:
        g.set_reproducible(True)  # the FP32 stage of MIXED sums in fixed point too
        g.set_dets(dets, 0, diag)
        g.build(prec)
        y1 = g.matrix_vector_prod(x)
        r1 = g.davidson(1, None, 1e-4, 1e-8, 500, mode=mode)
        g.build(prec)  # a fresh build: the tiles are filled in a run-dependent order
        y2 = g.matrix_vector_prod(x)
        r2 = g.davidson(1, None, 1e-4, 1e-8, 500, mode=mode)
    np.testing.assert_array_equal(y1, y2)
    assert r1.converged and r1.eigenvalues[0] == r2.eigenvalues[0]
    np.testing.assert_array_equal(r1.eigenvectors, r2.eigenvectors)


def test_thick_restart_reaches_the_same_energy():
    # a larger search space with a thick restart (risqgpu_set_subspace) changes the
    # iteration count, not the answer
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-3)
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        ref = g.davidson(1, None, 1e-4, 1e-8, 2000)
        g.set_subspace(32, 8)
        thick = g.davidson(1, None, 1e-4, 1e-8, 2000)
        g.build(_capi.MIXED)
        mixed = g.davidson(1, None, 1e-4, 1e-8, 2000, mode=_capi.MODE_MIXED)
    assert ref.converged and thick.converged and mixed.converged
    assert abs(thick.eigenvalues[0] - ref.eigenvalues[0]) < 1e-6
    assert abs(mixed.eigenvalues[0] - ref.eigenvalues[0]) < 1e-6
    assert thick.stats["iters"] < ref.stats["iters"]
