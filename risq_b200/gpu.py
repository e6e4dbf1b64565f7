"""Python mirror of the reference's hot-path interface, over librisqgpu.so.

Reference names kept (aaholmes/risq):
  Ham.ham_diag / Ham.ham_off_diag_no_excite   src/ham/mod.rs:92-124, :256-303
  SparseHam.matrix_vector_prod / matrix_matrix_prod / diagonal
                                              src/var/sparse.rs:64-93 (MatrixOperations)
  SparseHam.davidson                          src/var/eigenvalues/algorithms/davidson.rs:106-277
  sparse_optimize                             src/var/davidson.rs:43-113
Determinants are uint64[N, 4] rows {up_lo, up_hi, dn_lo, dn_hi} (Config, src/wf/det.rs:16-19).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _capi as A
from .fcidump import Integrals, packed_sizes


def device_count() -> int:
    return A.lib().risqgpu_device_count()


@dataclasses.dataclass
class DavidsonResult:
    eigenvalues: np.ndarray
    eigenvectors: np.ndarray  # N x nroots
    stats: dict
    converged: bool


class GpuHam:
    """One device handle: integrals, determinant set, sparse H and Davidson."""

    def __init__(self, ints: Integrals, device: int = 0):
        self.norb = ints.norb
        n1, n2 = packed_sizes(ints.norb)
        ob = np.ascontiguousarray(ints.one_body, dtype=np.float64)
        tb = np.ascontiguousarray(ints.two_body, dtype=np.float64)
        if ob.size != n1 or tb.size != n2:
            raise ValueError("integral arrays are not in the packed layout for norb")
        h = C.c_void_p()
        rc = A.lib().risqgpu_create(ints.norb, A.ptr(ob, A._dp), n1, A.ptr(tb, A._dp), n2, float(ints.nuc), device,
                                    C.byref(h))
        A.check(rc)
        self._h = h
        self.n = 0

    def close(self):
        if getattr(self, "_h", None):
            A.lib().risqgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- Slater-Condon elements -------------------------------------------------
    def ham_diag(self, dets) -> np.ndarray:
        d = np.ascontiguousarray(dets, dtype=np.uint64).reshape(-1, 4)
        out = np.zeros(d.shape[0])
        A.check(A.lib().risqgpu_ham_diag(self._h, A.ptr(d, A._u64p), d.shape[0], A.ptr(out, A._dp)), self._h)
        return out

    def ham_off_diag_no_excite(self, d1, d2) -> np.ndarray:
        a = np.ascontiguousarray(d1, dtype=np.uint64).reshape(-1, 4)
        b = np.ascontiguousarray(d2, dtype=np.uint64).reshape(-1, 4)
        if a.shape != b.shape:
            raise ValueError("d1 and d2 must have the same shape")
        out = np.zeros(a.shape[0])
        A.check(A.lib().risqgpu_ham_off_diag(self._h, A.ptr(a, A._u64p), A.ptr(b, A._u64p), a.shape[0],
                                             A.ptr(out, A._dp)), self._h)
        return out

    # --- variational space and sparse H ----------------------------------------
    def set_dets(self, dets, n_stored_h: int = 0, diag=None):
        d = np.ascontiguousarray(dets, dtype=np.uint64).reshape(-1, 4)
        dg = None
        if diag is not None:
            dg = np.ascontiguousarray(diag, dtype=np.float64)
            if dg.size != d.shape[0]:
                raise ValueError("diag length differs from the number of determinants")
        A.check(A.lib().risqgpu_set_dets(self._h, A.ptr(d, A._u64p), d.shape[0], n_stored_h,
                                         A.ptr(dg, A._dp) if dg is not None else None), self._h)
        self.n = d.shape[0]
        return self

    def build(self, precision=A.FP64, builder=A.BUILDER_AUTO) -> dict:
        st = A.HStats()
        A.check(A.lib().risqgpu_build_h(self._h, precision, builder, C.byref(st)), self._h)
        return st.as_dict()

    def nnz(self):
        u, f = C.c_uint64(), C.c_uint64()
        A.check(A.lib().risqgpu_nnz(self._h, C.byref(u), C.byref(f)), self._h)
        return u.value, f.value

    def export_upper(self):
        """(rowptr, cols, vals, diag) of the stored upper triangle, caller indices, rows sorted."""
        nu, _ = self.nnz()
        rp = np.zeros(self.n + 1, dtype=np.int64)
        cols = np.zeros(max(nu, 1), dtype=np.int64)
        vals = np.zeros(max(nu, 1))
        diag = np.zeros(self.n)
        A.check(A.lib().risqgpu_export_upper(self._h, A.ptr(rp, A._i64p), A.ptr(cols, A._i64p), A.ptr(vals, A._dp),
                                             nu, A.ptr(diag, A._dp)), self._h)
        return rp, cols[:nu], vals[:nu], diag

    def export_rows(self, rows, cap=None):
        """Stored elements of the given caller rows in both triangles: arrays (row, col, val)
        in no particular order (risqgpu_export_rows)."""
        r = np.ascontiguousarray(rows, dtype=np.int64)
        if cap is None:
            cap = max(1, 20000 * len(r))
        out_r = np.zeros(cap, dtype=np.int64)
        out_c = np.zeros(cap, dtype=np.int64)
        out_v = np.zeros(cap)
        cnt = C.c_size_t()
        A.check(A.lib().risqgpu_export_rows(self._h, A.ptr(r, A._i64p), len(r), A.ptr(out_r, A._i64p),
                                            A.ptr(out_c, A._i64p), A.ptr(out_v, A._dp), cap, C.byref(cnt)), self._h)
        k = cnt.value
        return out_r[:k], out_c[:k], out_v[:k]

    def matrix_vector_prod(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.n:
            raise ValueError("vector length differs from the number of determinants")
        y = np.zeros(self.n)
        A.check(A.lib().risqgpu_sigma(self._h, A.ptr(x, A._dp), A.ptr(y, A._dp), 1), self._h)
        return y

    def matrix_matrix_prod(self, X) -> np.ndarray:
        """Columns of X (N x k) -> H X (N x k)."""
        X = np.asarray(X, dtype=np.float64)
        Xc = np.ascontiguousarray(X.T)  # k x N, each column contiguous
        Y = np.zeros_like(Xc)
        A.check(A.lib().risqgpu_sigma(self._h, A.ptr(Xc, A._dp), A.ptr(Y, A._dp), Xc.shape[0]), self._h)
        return Y.T.copy()

    def sigma_noalloc(self, x_ptr: int, y_ptr: int):
        """y = H x on caller-owned device buffers (caller order) with no allocation in the call
        (at most 2^20 determinants; see risqgpu_sigma_noalloc in include/risqgpu.h)."""
        A.check(A.lib().risqgpu_sigma_noalloc(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)), self._h)

    def sigma_device(self, x_ptr: int, y_ptr: int, dtype: int = 0):
        A.check(A.lib().risqgpu_sigma_device(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), dtype), self._h)

    def davidson(self, nroots=1, init=None, tol=1e-4, etol=1e-8, max_iter=50, mode=A.MODE_FP64,
                 precond=A.PRECOND_DPR) -> DavidsonResult:
        ev = np.zeros(nroots)
        vecs = np.zeros((nroots, self.n))
        st = A.DStats()
        ip = None
        ninit = 0
        if init is not None:
            init = np.asarray(init, dtype=np.float64)
            if init.ndim == 1:
                init = init[:, None]
            ninit = init.shape[1]
            initc = np.ascontiguousarray(init.T)
            ip = A.ptr(initc, A._dp)
        rc = A.lib().risqgpu_davidson(self._h, nroots, ip, ninit, tol, etol, max_iter, mode, precond,
                                      A.ptr(ev, A._dp), A.ptr(vecs, A._dp), C.byref(st))
        if rc not in (A.OK, A.ERR_NOT_CONVERGED):
            A.check(rc, self._h)
        return DavidsonResult(ev, vecs.T.copy(), st.as_dict(), rc == A.OK)

    def set_precond_mlp(self, w1, b1, w2, b2, w3, b3, feat_norm=(0.0, 1.0, 0.0, 1.0)):
        """Load the learned-preconditioner network (risqgpu_set_precond_mlp).  feat_norm =
        (shift, scale) for the H_ii - E feature, then for the occupied-h_pp feature."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (w1, b1, w2, b2, w3, b3, feat_norm)]
        hidden, n_in = arrs[0].shape
        A.check(A.lib().risqgpu_set_precond_mlp(self._h, n_in, hidden, *[A.ptr(a, A._fp) for a in arrs]), self._h)

    # --- HCI selection and the variational loop --------------------------------
    def find_new_dets(self, coeffs, eps, singles, ncore=0):
        """One selection step over the current set (find_new_dets, src/wf/mod.rs:1418-1631):
        returns (new dets uint64[M, 4], their diagonals) in the reference's push order."""
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        if c.size != self.n:
            raise ValueError("coefficient vector length differs from the number of determinants")
        m = C.c_size_t()
        A.check(A.lib().risqgpu_find_new_dets(self._h, A.ptr(c, A._dp), eps, 1 if singles else 0, ncore,
                                              C.byref(m)), self._h)
        d = np.zeros((m.value, 4), dtype=np.uint64)
        g = np.zeros(m.value)
        A.check(A.lib().risqgpu_get_new_dets(self._h, A.ptr(d, A._u64p), A.ptr(g, A._dp), m.value), self._h)
        return d, g

    def variational(self, nup, ndn, eps_var, ncore=0, max_iter=20, dav_max_iter=50, precision=A.FP64,
                    mode=A.MODE_FP64, precond=A.PRECOND_DPR):
        """init_var_wf + variational (src/wf/mod.rs:1687-1740, src/var/mod.rs:59-134) on the device.
        Returns (energy, dets, coeffs, diag, log)."""
        e = C.c_double()
        n = C.c_uint64()
        A.check(A.lib().risqgpu_variational(self._h, nup, ndn, ncore, 1, eps_var, max_iter, dav_max_iter, precision,
                                            mode, precond, C.byref(e), C.byref(n)), self._h)
        N = n.value
        d = np.zeros((N, 4), dtype=np.uint64)
        c = np.zeros(N)
        g = np.zeros(N)
        A.check(A.lib().risqgpu_get_wf(self._h, A.ptr(d, A._u64p), A.ptr(c, A._dp), A.ptr(g, A._dp), N), self._h)
        k = C.c_int()
        A.lib().risqgpu_var_log(self._h, None, 0, C.byref(k))
        recs = (A.VarIter * max(k.value, 1))()
        A.lib().risqgpu_var_log(self._h, recs, k.value, C.byref(k))
        self.n = N
        return e.value, d, c, g, [recs[i].as_dict() for i in range(k.value)]

    def set_subspace(self, max_space: int = 0, keep: int = 0):
        """Davidson search space and restart size of this handle's solves; (0, 0) is the
        reference's nroots + 10 with a restart to the nroots Ritz vectors
        (risqgpu_set_subspace)."""
        A.check(A.lib().risqgpu_set_subspace(self._h, int(max_space), int(keep)), self._h)

    def set_reproducible(self, on: bool = True):
        """FP32 sigma of upper-triangle storage in 64-bit fixed point (bitwise reproducible)
        instead of FP32 atomic sums (risqgpu_set_reproducible)."""
        A.check(A.lib().risqgpu_set_reproducible(self._h, 1 if on else 0), self._h)

    def set_partition(self, rank: int, nranks: int, reduce_fn=None):
        """Row-block partition over nranks GPUs (risqgpu_set_partition): the next
        upper-triangle build keeps this rank's share of the row panels and sigma adds the
        ranks' partial sums with reduce_fn (risq_b200.distributed.make_allreduce)."""
        fn = reduce_fn if reduce_fn is not None else A.ALLREDUCE_FN()
        A.check(A.lib().risqgpu_set_partition(self._h, int(rank), int(nranks), fn, None), self._h)
        self._reduce_fn = fn  # the library keeps the pointer: keep the callback alive

    def set_memory_limit(self, nbytes: int):
        """Bound the device memory the handle may hold (0 = no bound); allocations past it
        fail with ERR_OOM (risqgpu_set_memory_limit)."""
        A.check(A.lib().risqgpu_set_memory_limit(self._h, int(nbytes)), self._h)

    def memory_used(self):
        """(bytes held by the handle, its bound or 0)."""
        u, l = C.c_size_t(), C.c_size_t()
        A.check(A.lib().risqgpu_memory_used(self._h, C.byref(u), C.byref(l)), self._h)
        return u.value, l.value

    def set_stream(self, stream_ptr):
        """Issue the handle's work on a caller cudaStream_t (int address); None = own stream."""
        A.check(A.lib().risqgpu_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None), self._h)

    def sparse_optimize(self, init_coeffs=None, coeff_eps=1e-4, energy_eps=1e-8, max_iter=50, precision=A.FP64,
                        mode=A.MODE_FP64, precond=A.PRECOND_DPR):
        """Build (or extend) H for the current set and run Davidson for the ground state.

        Returns (energy, coeffs, hstats, dstats); raises RisqGpuError(ERR_NOT_CONVERGED)
        when Davidson fails, as the reference reports DavidsonError (var/davidson.rs:109-111).
        """
        e = C.c_double()
        c = np.zeros(self.n)
        hs, ds = A.HStats(), A.DStats()
        ip = None
        if init_coeffs is not None:
            init_coeffs = np.ascontiguousarray(init_coeffs, dtype=np.float64)
            ip = A.ptr(init_coeffs, A._dp)
        A.check(A.lib().risqgpu_sparse_optimize(self._h, ip, coeff_eps, energy_eps, max_iter, precision, mode,
                                                precond, C.byref(e), A.ptr(c, A._dp), C.byref(hs), C.byref(ds)),
                self._h)
        return e.value, c, hs.as_dict(), ds.as_dict()
