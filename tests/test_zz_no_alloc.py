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
from tests import helpers as H

pytestmark = pytest.mark.gpu


def test_sigma_noalloc_matches_sigma_on_two_calls():
    import torch

    ints, p = H.golden_system("be2")
    _, dets, coeffs, diag, _ = H.oracle_hci("be2")
    rng = np.random.default_rng(11)
    with GpuHam(ints) as g:
        g.set_dets(dets, 0, diag)
        g.build(_capi.FP64)
        lib = _capi.lib()
        for x in (coeffs, rng.standard_normal(len(dets))):
            ref = g.matrix_vector_prod(x)  # risqgpu_sigma, the allocating entry point
            xd = torch.tensor(x, dtype=torch.float64, device="cuda")
            yd = torch.full_like(xd, float("nan"))
            torch.cuda.synchronize()
            rc = lib.risqgpu_sigma_noalloc(g._h, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()))
            assert rc == _capi.OK, lib.risqgpu_last_error(g._h)
            y = yd.cpu().numpy()
            # the same sums in the same order: equal to within the sigma tolerance used elsewhere
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
