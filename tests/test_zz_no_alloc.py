"""risqgpu_sigma_noalloc: sigma for callers that cannot let the library allocate.

A host code whose pool allocator owns the device memory, or a Davidson loop that
overlaps work on several streams, cannot accept the cudaMalloc/cudaFree (and the
device-wide synchronisation of cudaFree) that risqgpu_sigma performs on every call.
The no-alloc variant keeps its two work vectors in a fixed 16 MiB device array
(at most 2^20 determinants) and takes caller-owned device buffers.  This file is
collected last so that a failure here stops a run only after every other test.
"""
import ctypes

import numpy as np
import pytest

from risq_b200 import GpuHam, _capi
from risq_b200.fcidump import synthetic_integrals
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _noalloc(g, xd, yd):
    lib = _capi.lib()
    return lib.risqgpu_sigma_noalloc(g._h, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()))


@pytest.mark.parametrize("prec", [_capi.FP64, _capi.FP64_UPPER, _capi.MIXED_UPPER, _capi.MATRIX_FREE])
def test_sigma_noalloc_matches_sigma_on_two_calls(prec):
    import torch

    ints, p = H.golden_system("be2")
    _, dets, coeffs, diag, _ = H.oracle_hci("be2")
    rng = np.random.default_rng(11)
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(prec)
        for x in (coeffs, rng.standard_normal(len(dets))):
            ref = g.matrix_vector_prod(x)  # risqgpu_sigma, the allocating entry point
            xd = torch.tensor(x, dtype=torch.float64, device="cuda")
            yd = torch.full_like(xd, float("nan"))
            torch.cuda.synchronize()
            rc = _noalloc(g, xd, yd)
            assert rc == _capi.OK, _capi.lib().risqgpu_last_error(g._h)
            y = yd.cpu().numpy()
            # the same stored elements and the same kernels on the same vector; checked to
            # the sigma tolerance used elsewhere
            assert np.max(np.abs(y - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_sigma_noalloc_in_place_on_the_callers_stream():
    # x produced on the caller's stream and the handle routed onto that stream with
    # risqgpu_set_stream: no explicit synchronisation is needed, and y may overwrite x
    import torch

    ints, p = H.golden_system("be2")
    _, dets, coeffs, diag, _ = H.oracle_hci("be2")
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        ref = g.matrix_vector_prod(coeffs)
        s = torch.cuda.Stream()
        g.set_stream(s.cuda_stream)
        host = torch.tensor(coeffs, dtype=torch.float64).pin_memory()
        with torch.cuda.stream(s):
            xd = torch.empty(len(dets), dtype=torch.float64, device="cuda")
            xd.copy_(host, non_blocking=True)
            xd.mul_(1.0)
        rc = _noalloc(g, xd, xd)
        assert rc == _capi.OK, _capi.lib().risqgpu_last_error(g._h)
        y = xd.cpu().numpy()
        g.set_stream(None)
        assert np.max(np.abs(y - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_sigma_noalloc_argument_checks():
    ints, p = H.golden_system("be")
    _, dets, _, diag, _ = H.oracle_hci("be")
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        lib = _capi.lib()
        one = ctypes.c_void_p(1)
        assert lib.risqgpu_sigma_noalloc(g._h, one, one) == _capi.ERR_INVALID  # before build
        g.build(_capi.FP64)
        assert lib.risqgpu_sigma_noalloc(g._h, None, one) == _capi.ERR_INVALID


def test_sigma_noalloc_rejects_fp32_only_upper_storage():
    import torch

    ints, p = H.golden_system("be2")
    _, dets, coeffs, diag, _ = H.oracle_hci("be2")
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP32_UPPER)  # FP32 values only: no FP64 sigma exists for this storage
        xd = torch.tensor(coeffs, dtype=torch.float64, device="cuda")
        yd = torch.zeros_like(xd)
        torch.cuda.synchronize()
        rc = _noalloc(g, xd, yd)
        assert rc == _capi.ERR_INVALID
        assert b"FP64" in _capi.lib().risqgpu_last_error(g._h)


def test_sigma_noalloc_rejects_sets_above_its_capacity():
    import torch

    # 2^20 + 1000 distinct determinants of 14 orbitals, 6 + 6 electrons, columns-only build
    rng = np.random.default_rng(3)
    n = (1 << 20) + 1000
    from itertools import combinations
    strings = np.array([sum(1 << i for i in c) for c in combinations(range(14), 6)], dtype=np.uint64)
    pick = rng.choice(len(strings) ** 2, size=n, replace=False)
    dets = np.zeros((n, 4), dtype=np.uint64)
    dets[:, 0] = strings[pick // len(strings)]
    dets[:, 2] = strings[pick % len(strings)]
    with GpuHam(synthetic_integrals(14, 0)) as g:
        g.set_dets(dets)
        g.build(_capi.COLS)
        xd = torch.zeros(n, dtype=torch.float64, device="cuda")
        yd = torch.zeros_like(xd)
        torch.cuda.synchronize()
        rc = _noalloc(g, xd, yd)
        assert rc == _capi.ERR_CAPACITY
        assert b"1048576" in _capi.lib().risqgpu_last_error(g._h)
