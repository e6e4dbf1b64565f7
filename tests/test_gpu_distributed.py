"""Row-block partition of sigma (risqgpu_set_partition), two ranks.

Two processes share the one GPU of this test; each holds its half of the row panels
and the partial sums are added through gloo on the host, so no kernel waits on
another process.  Integer fixed-point sums are exact: the two-rank sigma and the
Davidson solves on it must equal the single-rank results bit for bit."""
import os
import socket

import numpy as np
import pytest

from risq_b200 import GpuHam, _capi
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _solve(g, prec, mode, x):
    g.build(prec)
    y = g.matrix_vector_prod(x)
    r = g.davidson(1, None, 1e-4, 1e-8, 2000, mode=mode)
    return y, r.eigenvalues[0], r.eigenvectors[:, 0], r.stats["iters"], g.nnz()[0]


def _rank(rank, world, port, path):
    import torch.distributed as dist

    from risq_b200 import distributed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-3)
        x = np.random.default_rng(8).standard_normal(len(dets))
        res = {}
        with GpuHam(ints) as g:
            g.set_partition(rank, world, distributed.make_allreduce())
            g.set_dets(dets, 0, diag)
            for name, prec, mode in (("fp64", _capi.FP64_UPPER, _capi.MODE_FP64),
                                     ("mixed", _capi.MIXED_UPPER, _capi.MODE_MIXED)):
                y, ev, vec, iters, nnz = _solve(g, prec, mode, x)
                res.update({f"{name}_y": y, f"{name}_e": ev, f"{name}_v": vec, f"{name}_it": iters,
                            f"{name}_nnz": nnz})
        np.savez(os.path.join(path, f"rank{rank}.npz"), **res)
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_equals_one_rank_bitwise(tmp_path):
    import torch.multiprocessing as mp
    ints, e, dets, coeffs, diag, log = H.synthetic_hci(12, 6, 1e-3)
    x = np.random.default_rng(8).standard_normal(len(dets))
    ref = {}
    with GpuHam(ints) as g:
        g.set_reproducible(True)  # fixed-point FP32 sums, as every partitioned handle uses
        g.set_dets(dets, 0, diag)
        for name, prec, mode in (("fp64", _capi.FP64_UPPER, _capi.MODE_FP64),
                                 ("mixed", _capi.MIXED_UPPER, _capi.MODE_MIXED)):
            ref[name] = _solve(g, prec, mode, x)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(600)
        assert p.exitcode == 0
    outs = [np.load(tmp_path / f"rank{r}.npz") for r in range(2)]
    for name in ("fp64", "mixed"):
        y, ev, vec, iters, nnz = ref[name]
        assert outs[0][f"{name}_nnz"] + outs[1][f"{name}_nnz"] == nnz  # the pairs are split, none repeated
        assert min(outs[0][f"{name}_nnz"], outs[1][f"{name}_nnz"]) > 0
        for o in outs:
            np.testing.assert_array_equal(o[f"{name}_y"], y)
            assert float(o[f"{name}_e"]) == ev and int(o[f"{name}_it"]) == iters
            np.testing.assert_array_equal(o[f"{name}_v"], vec)
