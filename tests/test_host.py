"""Host-side pieces without a GPU: FCIDUMP I/O, synthetic integrals, the C ABI surface."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from risq_b200 import _capi
from risq_b200.fcidump import (combine_4, dets_from_ints, dets_to_ints, hf_det, packed_sizes, read_fcidump,
                               synthetic_integrals, write_fcidump)
from tests import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_packed_sizes():
    assert packed_sizes(32) == (561, 157641)
    assert packed_sizes(20) == (231, 26796)


def test_synthetic_integrals_symmetry_and_psd():
    n = 8
    ints = synthetic_integrals(n, 0)
    # dense 4-index tensor from the packed table
    eri = np.zeros((n, n, n, n))
    for p in range(n):
        for q in range(n):
            for r in range(n):
                for s in range(n):
                    eri[p, q, r, s] = ints.two_body[combine_4(p + 1, q + 1, r + 1, s + 1)]
    M = eri.reshape(n * n, n * n)
    assert np.allclose(M, M.T)
    assert np.linalg.eigvalsh(M).min() > -1e-10  # sum_L B^L B^L is PSD
    h = np.array([[ints.h(p, q) for q in range(n)] for p in range(n)])
    assert np.allclose(h, h.T)
    np.testing.assert_allclose(np.diag(h), -3.0 + 4.0 * np.arange(n) / (n - 1))
    assert ints.nuc == 0.0
    again = synthetic_integrals(n, 0)
    assert np.array_equal(again.two_body, ints.two_body)
    assert not np.array_equal(synthetic_integrals(n, 1).two_body, ints.two_body)


def test_fcidump_roundtrip_is_exact(tmp_path):
    ints = synthetic_integrals(10, 3)
    p = tmp_path / "FCIDUMP"
    write_fcidump(str(p), ints, nelec=10)
    back = read_fcidump(str(p), 10)
    assert back.nuc == ints.nuc
    assert np.array_equal(back.one_body, ints.one_body)
    assert np.array_equal(back.two_body, ints.two_body)
    oh = O.Ham.from_fcidump(str(p), 10, 0)
    nuc, ob, tb = oh.arrays()
    assert np.array_equal(ob, ints.one_body) and np.array_equal(tb, ints.two_body)


def test_fcidump_errors(tmp_path):
    p = tmp_path / "bad"
    p.write_text(" &FCI NORB=2,\n &END\n 0.5 1 1 3 1\n")
    with pytest.raises(ValueError):
        read_fcidump(str(p), 2)
    with pytest.raises(ValueError):
        O.Ham.from_fcidump(str(p), 2, 0)


def test_det_packing_roundtrip():
    rows = [(0b1011, 0b0111), ((1 << 100) | 3, (1 << 64) | 1)]
    d = dets_from_ints(rows)
    assert d.dtype == np.uint64 and d.shape == (2, 4)
    assert dets_to_ints(d) == rows
    assert dets_to_ints(hf_det(3, 2)[None]) == [(7, 3)]


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "risqgpu.h")).read()
    return sorted(set(re.findall(r"RISQGPU_API[^;(]*?\b(risqgpu_\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    syms = _declared_symbols()
    assert len(syms) >= 16
    lib = ctypes.CDLL(_capi.LIB_PATH)
    for s in syms:
        assert hasattr(lib, s), s
    bound = {name for name, _, _ in _capi.SIGNATURES}
    assert set(syms) == bound


def test_calls_without_device():
    L = _capi.lib()
    assert L.risqgpu_version().startswith(b"risq_b200")
    n = L.risqgpu_device_count()
    assert n >= 0
    # argument validation happens before any device work
    h = ctypes.c_void_p()
    ob = np.zeros(3)
    tb = np.zeros(6)
    assert L.risqgpu_create(1, _capi.ptr(ob, _capi._dp), 3, _capi.ptr(tb, _capi._dp), 7, 0.0, 0,
                            ctypes.byref(h)) == _capi.ERR_INVALID
    assert L.risqgpu_create(0, _capi.ptr(ob, _capi._dp), 1, _capi.ptr(tb, _capi._dp), 1, 0.0, 0,
                            ctypes.byref(h)) == _capi.ERR_INVALID
    if n == 0:
        n1, n2 = packed_sizes(1)
        ob, tb = np.zeros(n1), np.zeros(n2)
        assert L.risqgpu_create(1, _capi.ptr(ob, _capi._dp), n1, _capi.ptr(tb, _capi._dp), n2, 0.0, 0,
                                ctypes.byref(h)) == _capi.ERR_NO_DEVICE


def test_oracle_hci_log_shape():
    e, dets, coeffs, diag, log = H.oracle_hci("be")
    assert [l["ndets"] for l in log] == sorted(l["ndets"] for l in log)
    assert log[-1]["ndets"] == len(dets)
    assert abs(np.linalg.norm(coeffs) - 1.0) < 1e-10


def _rank_main(rank, world, port, out):
    import os

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each replica reports its own step time; every rank must see the slowest one
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, world)
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_the_max_over_ranks():
    """bench.py --gpus N runs one replica per rank and reports the slowest rank's time
    (two gloo ranks on the CPU)."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == 15.0 and out[1] == 15.0
    import bench
    assert bench.max_over_ranks(7.5, 1) == 7.5  # one GPU: no collective


def _reduce_rank(rank, world, port, out):
    import ctypes
    import os

    import numpy as np
    import torch.distributed as dist

    from risq_b200 import distributed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank's partial fixed-point sums, wrapping in int64 as the library's do
        part = np.arange(10, dtype=np.int64) * (rank + 1) + np.int64(2**62) * rank
        fn = distributed.make_allreduce(host_buffers=True)
        rc = fn(part.ctypes.data_as(ctypes.c_void_p), part.size, None, None)
        out[rank] = (rc, part.tolist())
    finally:
        dist.destroy_process_group()


def test_partition_allreduce_sums_int64_partials_across_ranks():
    """The all-reduce a partitioned handle calls after every sigma (risqgpu_set_partition)
    adds the ranks' int64 partial sums exactly, wrap-around included (two gloo ranks on
    the CPU, host buffers)."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_reduce_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    want = (np.arange(10, dtype=np.int64) * 3 + np.int64(2**62)).tolist()
    assert out[0] == (0, want) and out[1] == (0, want)
