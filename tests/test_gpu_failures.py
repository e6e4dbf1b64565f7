"""Failure paths, driven without faulting the GPU.

The reference reports a failed solve by keeping the old energy
(src/var/davidson.rs:109-111; DavidsonError, src/var/eigenvalues/algorithms/davidson.rs:81-90).
The library returns status codes instead of aborting; these tests provoke each
failure on the host side (a memory bound on the handle, a non-finite input, a
device wait that is made to run out) and check the status, the message, that no
device memory is left behind, and that the handle stays usable afterwards.
"""
import os

import numpy as np
import pytest

from risq_b200 import GpuHam, _capi, learned
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _err(fn, *a, **k):
    with pytest.raises(_capi.RisqGpuError) as ei:
        fn(*a, **k)
    return ei.value


def test_stalled_tensor_core_wait_returns_error_and_handle_recovers():
    # The tcgen05 inference kernel bounds every mbarrier wait.  RISQGPU_TEST_MMA_STALL=1
    # makes its first wait watch a barrier that nothing arrives on (1 ms limit): the call
    # must return ERR_CUDA with a message, free its TMEM and leave the handle usable.
    ints, _, dets, _, diag, _ = H.synthetic_hci(12, 6, 1e-3)
    m = learned.PrecondMLP.init(ints.norb, hidden=128, seed=2, fnorm=[1.0, 0.5, -10.0, 0.1])
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        learned.install(g, m)
        E = float(diag.min()) - 0.3
        before = learned.device_factors(g, E)
        os.environ["RISQGPU_TEST_MMA_STALL"] = "1"
        try:
            e = _err(learned.device_factors, g, E)
        finally:
            del os.environ["RISQGPU_TEST_MMA_STALL"]
        assert e.code == _capi.ERR_CUDA and "timed out" in str(e)
        after = learned.device_factors(g, E)
        np.testing.assert_array_equal(before, after)
        # a Davidson solve with the learned preconditioner still runs on this handle
        g.build(_capi.MIXED)
        r = g.davidson(1, None, 1e-4, 1e-8, 500, mode=_capi.MODE_MIXED, precond=_capi.PRECOND_LEARNED)
        assert r.converged


def test_memory_limit_gives_oom_without_leaks():
    ints, p = H.golden_system("f2")
    _, dets, coeffs, diag, _ = H.oracle_hci("f2")
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        base, _ = g.memory_used()
        assert base > 0
        # no room for any matrix
        g.set_memory_limit(base + 4096)
        e = _err(g.build, _capi.FP64)
        assert e.code == _capi.ERR_OOM and "limit" in str(e)
        assert g.memory_used()[0] == base
        g.set_memory_limit(0)
        g.build(_capi.FP64)
        used, _ = g.memory_used()
        # sigma and Davidson need work buffers: with none left they fail and release what they took
        g.set_memory_limit(used + 8 * len(dets))
        e = _err(g.matrix_vector_prod, coeffs)
        assert e.code == _capi.ERR_OOM
        assert g.memory_used()[0] == used
        e = _err(g.davidson, 1, coeffs, 1e-4, 1e-8, 50)
        assert e.code == _capi.ERR_OOM
        assert g.memory_used()[0] == used
        g.set_memory_limit(0)
        r = g.davidson(1, coeffs, 1e-4, 1e-8, 50)
        assert r.converged and g.memory_used()[0] == used


def test_variational_storage_fallback_under_memory_limit():
    # variational with precision -1 stores both FP64 triangles while they fit, then the upper
    # triangle, then columns only (the fallback chain of risqgpu_variational); a bound on the
    # handle's memory must drive it down the chain to the same wavefunction
    ints, p = H.golden_system("f2")
    kw = dict(ncore=p["norb_core"], max_iter=20, dav_max_iter=50)
    with GpuHam(ints) as g:
        e0, d0, c0, _, _ = g.variational(p["nup"], p["ndn"], p["eps_var"], precision=-1, **kw)
        nnz_u, nnz_f = g.nnz()
        full_used, _ = g.memory_used()
    with GpuHam(ints) as g:
        g.variational(p["nup"], p["ndn"], p["eps_var"], precision=_capi.FP64_UPPER, **kw)
        upper_used, _ = g.memory_used()
    assert upper_used < full_used
    with GpuHam(ints) as g:
        # half way between the two: both FP64 triangles of the final set do not fit, the
        # upper triangle does, with room for the Davidson work space
        g.set_memory_limit((upper_used + full_used) // 2)
        e1, d1, c1, _, _ = g.variational(p["nup"], p["ndn"], p["eps_var"], precision=-1, **kw)
        assert g.memory_used()[0] <= g.memory_used()[1]
        nu1, nf1 = g.nnz()
    assert np.array_equal(d0, d1)
    assert nu1 == nnz_u
    assert abs(e0 - e1) < 1e-9


def test_non_finite_inputs_are_rejected():
    ints, p = H.golden_system("be")
    _, dets, coeffs, diag, _ = H.oracle_hci("be")
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        bad = coeffs.copy()
        bad[len(bad) // 2] = np.nan
        e = _err(g.matrix_vector_prod, bad)
        assert e.code == _capi.ERR_INVALID and "non-finite" in str(e)
        bad[len(bad) // 2] = np.inf
        e = _err(g.davidson, 1, bad, 1e-4, 1e-8, 50)
        assert e.code == _capi.ERR_INVALID and "non-finite" in str(e)
        r = g.davidson(1, coeffs, 1e-4, 1e-8, 50)
        assert r.converged
