"""ctypes front end of the CPU oracle (``liboracle.so``, built from risq_oracle.c).

TEST INFRASTRUCTURE. Only the test suite, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module, always as the checker of the
CUDA path, never as a stand-in for it.

Determinant strings cross the ABI as ``uint64[N, 4]`` rows ``{up_lo, up_hi,
dn_lo, dn_hi}`` (the reference's ``Config{up: u128, dn: u128}``,
src/wf/det.rs:16-19).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_ip = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compile liboracle.so in place with the committed Makefile."""
    src = os.path.join(_HERE, "risq_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s", "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.or_ham_read_fcidump.restype = C.c_void_p
        L.or_ham_read_fcidump.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int]
        L.or_ham_from_arrays.restype = C.c_void_p
        L.or_ham_from_arrays.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp]
        L.or_ham_free.argtypes = [C.c_void_p]
        L.or_ham_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        L.or_ham_copy.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.or_ham_orbs.argtypes = [C.c_void_p, _ip, _ip]
        L.or_ham_orbs.restype = C.c_int
        L.or_ham_diag_batch.argtypes = [C.c_void_p, _u64p, C.c_size_t, _dp]
        L.or_ham_off_diag_batch.argtypes = [C.c_void_p, _u64p, _u64p, C.c_size_t, _dp]
        L.or_parity.argtypes = [C.c_uint64, C.c_uint64]
        L.or_parity.restype = C.c_int
        L.or_permute.argtypes = [C.c_uint64] * 4
        L.or_permute.restype = C.c_int
        L.or_combine_4.argtypes = [C.c_int] * 4
        L.or_combine_4.restype = C.c_size_t
        L.or_sparse_new.restype = C.c_void_p
        L.or_sparse_free.argtypes = [C.c_void_p]
        L.or_sparse_build.argtypes = [C.c_void_p, C.c_void_p, _u64p, C.c_size_t, C.c_size_t, _dp, C.c_int, C.c_int]
        L.or_sparse_build.restype = C.c_int
        L.or_sparse_nnz.argtypes = [C.c_void_p]
        L.or_sparse_nnz.restype = C.c_size_t
        L.or_sparse_n.argtypes = [C.c_void_p]
        L.or_sparse_n.restype = C.c_size_t
        L.or_sparse_export.argtypes = [C.c_void_p, _i64p, _i64p, _dp, _dp]
        L.or_sparse_mv.argtypes = [C.c_void_p, _dp, _dp]
        L.or_sym_eig.argtypes = [C.c_int, _dp, _dp, _dp]
        L.or_mgs.argtypes = [_dp, C.c_size_t, C.c_int, C.c_int]
        L.or_mgs.restype = C.c_int
        L.or_davidson.argtypes = [C.c_void_p, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _dp, _ip]
        L.or_davidson.restype = C.c_int
        L.or_davidson_par.argtypes = [C.c_void_p, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _dp, _ip]
        L.or_davidson_par.restype = C.c_int
        L.or_sparse_build_par.argtypes = [C.c_void_p, C.c_void_p, _u64p, C.c_size_t, _dp]
        L.or_sparse_build_par.restype = C.c_int
        L.or_sparse_mv_par.argtypes = [C.c_void_p, _dp, _dp]
        L.or_num_threads.restype = C.c_int
        L.or_rows_bruteforce.argtypes = [C.c_void_p, _u64p, C.c_size_t, _i64p, C.c_size_t, _i64p, _i64p, _dp,
                                         C.c_size_t]
        L.or_rows_bruteforce.restype = C.c_int
        L.or_hci_set_options.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_davidson_dense.argtypes = [_dp, C.c_size_t, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _dp, _ip]
        L.or_davidson_dense.restype = C.c_int
        L.or_hci_new.restype = C.c_void_p
        L.or_hci_new.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int]
        L.or_hci_free.argtypes = [C.c_void_p]
        L.or_hci_step_bounded.argtypes = [C.c_void_p, C.c_size_t]
        L.or_hci_step_bounded.restype = C.c_int
        L.or_hci_step.argtypes = [C.c_void_p]
        L.or_hci_step.restype = C.c_int
        L.or_hci_run.argtypes = [C.c_void_p, C.c_int]
        L.or_hci_run.restype = C.c_double
        for f in ("or_hci_ndets", "or_hci_nstored"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = C.c_size_t
        L.or_hci_energy.argtypes = [C.c_void_p]
        L.or_hci_energy.restype = C.c_double
        L.or_hci_eps.argtypes = [C.c_void_p]
        L.or_hci_eps.restype = C.c_double
        L.or_hci_converged.argtypes = [C.c_void_p]
        L.or_hci_converged.restype = C.c_int
        L.or_hci_export.argtypes = [C.c_void_p, _u64p, _dp, _dp]
        L.or_hci_sparse.argtypes = [C.c_void_p]
        L.or_hci_sparse.restype = C.c_void_p
        L.or_hci_log.argtypes = [C.c_void_p, _dp, _dp, _u64p, _u64p, _ip]
        L.or_hci_log.restype = C.c_int
        L.or_excite_gen_max.argtypes = [C.c_void_p, _dp]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def combine_2(p: int, q: int) -> int:
    """1-based triangular packing (src/utils/ints.rs:38-46)."""
    i, j = abs(p), abs(q)
    return (i * (i - 1)) // 2 + j if i > j else (j * (j - 1)) // 2 + i


def combine_4(p, q, r, s) -> int:
    a, b = combine_2(p, q), combine_2(r, s)
    return (a * (a - 1)) // 2 + b if a > b else (b * (b - 1)) // 2 + a


def packed_sizes(norb: int):
    return combine_2(norb + 1, norb + 1), combine_4(norb + 1, norb + 1, norb + 1, norb + 1)


class Ham:
    """Integrals in the reference's packed 1-based layout (src/ham/read_ints.rs:33-42)."""

    def __init__(self, ptr, norb):
        self.ptr = ptr
        self.norb = norb

    @classmethod
    def from_fcidump(cls, path: str, norb: int, ncore: int = 0) -> "Ham":
        err = C.create_string_buffer(512)
        p = lib().or_ham_read_fcidump(path.encode(), norb, ncore, err, 512)
        if not p:
            raise ValueError(err.value.decode())
        return cls(p, norb)

    @classmethod
    def from_arrays(cls, norb, ncore, nuc, one_body, two_body) -> "Ham":
        ob = np.ascontiguousarray(one_body, dtype=np.float64)
        tb = np.ascontiguousarray(two_body, dtype=np.float64)
        n1, n2 = packed_sizes(norb)
        assert ob.size == n1 and tb.size == n2
        return cls(lib().or_ham_from_arrays(norb, ncore, float(nuc), _p(ob, _dp), _p(tb, _dp)), norb)

    def arrays(self):
        n1, n2 = C.c_size_t(), C.c_size_t()
        lib().or_ham_sizes(self.ptr, C.byref(n1), C.byref(n2))
        ob = np.zeros(n1.value)
        tb = np.zeros(n2.value)
        nuc = C.c_double()
        lib().or_ham_copy(self.ptr, C.byref(nuc), _p(ob, _dp), _p(tb, _dp))
        return nuc.value, ob, tb

    def orbs(self):
        core = np.zeros(self.norb, dtype=np.int32)
        val = np.zeros(self.norb, dtype=np.int32)
        nc = lib().or_ham_orbs(self.ptr, _p(core, _ip), _p(val, _ip))
        return core[:nc].copy(), val[: self.norb - nc].copy()

    def diag(self, dets: np.ndarray) -> np.ndarray:
        d = np.ascontiguousarray(dets, dtype=np.uint64)
        out = np.zeros(d.shape[0])
        lib().or_ham_diag_batch(self.ptr, _p(d, _u64p), d.shape[0], _p(out, _dp))
        return out

    def off_diag(self, d1: np.ndarray, d2: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(d1, dtype=np.uint64)
        b = np.ascontiguousarray(d2, dtype=np.uint64)
        out = np.zeros(a.shape[0])
        lib().or_ham_off_diag_batch(self.ptr, _p(a, _u64p), _p(b, _u64p), a.shape[0], _p(out, _dp))
        return out

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.or_ham_free(self.ptr)
            self.ptr = None


class Sparse:
    """SparseMatUpperTri (src/var/sparse.rs:24-36) built by the oracle."""

    def __init__(self):
        self.ptr = lib().or_sparse_new()

    def build(self, ham: Ham, dets, diag, n_stored_h=0, builder=0, grouped_singles=True):
        d = np.ascontiguousarray(dets, dtype=np.uint64)
        dg = np.ascontiguousarray(diag, dtype=np.float64)
        r = lib().or_sparse_build(self.ptr, ham.ptr, _p(d, _u64p), d.shape[0], n_stored_h, _p(dg, _dp),
                                  builder, 1 if grouped_singles else 0)
        if r != 0:
            raise RuntimeError(f"oracle sparse build failed ({r})")
        return self

    def build_par(self, ham: Ham, dets, diag):
        """The fast builder's pairs and values for the whole set, on every host core."""
        d = np.ascontiguousarray(dets, dtype=np.uint64)
        dg = np.ascontiguousarray(diag, dtype=np.float64)
        if lib().or_sparse_build_par(self.ptr, ham.ptr, _p(d, _u64p), d.shape[0], _p(dg, _dp)) != 0:
            raise RuntimeError("oracle parallel build needs an empty matrix")
        return self

    def mv_par(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        lib().or_sparse_mv_par(self.ptr, _p(x, _dp), _p(y, _dp))
        return y

    @property
    def n(self):
        return lib().or_sparse_n(self.ptr)

    @property
    def nnz(self):
        return lib().or_sparse_nnz(self.ptr)

    def export(self):
        """Upper triangle as (rowptr, cols, vals, diag), each row sorted by column."""
        n, z = self.n, self.nnz
        rp = np.zeros(n + 1, dtype=np.int64)
        cols = np.zeros(z, dtype=np.int64)
        vals = np.zeros(z)
        diag = np.zeros(n)
        lib().or_sparse_export(self.ptr, _p(rp, _i64p), _p(cols, _i64p), _p(vals, _dp), _p(diag, _dp))
        return rp, cols, vals, diag

    def mv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        lib().or_sparse_mv(self.ptr, _p(x, _dp), _p(y, _dp))
        return y

    def davidson(self, nvalues=1, init=None, tol=1e-4, etol=1e-8, max_iters=50, parallel=False):
        n = self.n
        ev = np.zeros(nvalues)
        vec = np.zeros((nvalues, n))
        st = np.zeros(4, dtype=np.int32)
        ip = None
        if init is not None:
            init = np.ascontiguousarray(init, dtype=np.float64)
            ip = _p(init, _dp)
        fn = lib().or_davidson_par if parallel else lib().or_davidson
        r = fn(self.ptr, nvalues, ip, tol, etol, max_iters, _p(ev, _dp), _p(vec, _dp), _p(st, _ip))
        return r, ev, vec, dict(iters=int(st[0]), n_sigma=int(st[1]), converged=bool(st[2]), reason=int(st[3]))

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.or_sparse_free(self.ptr)
            self.ptr = None


def rows_bruteforce(ham: Ham, dets, rows, cap=None):
    """Full rows of the given determinants against the whole set by brute force: a list of
    (cols, vals) per row, columns ascending (the fast builder's rule and values)."""
    d = np.ascontiguousarray(dets, dtype=np.uint64)
    r = np.ascontiguousarray(rows, dtype=np.int64)
    if cap is None:
        cap = 20000 * len(r) + 1
    off = np.zeros(len(r) + 1, dtype=np.int64)
    cols = np.zeros(cap, dtype=np.int64)
    vals = np.zeros(cap)
    rc = lib().or_rows_bruteforce(ham.ptr, _p(d, _u64p), d.shape[0], _p(r, _i64p), len(r), _p(off, _i64p),
                                  _p(cols, _i64p), _p(vals, _dp), cap)
    if rc != 0:
        raise RuntimeError(f"row capacity {cap} too small ({off[-1]} entries)")
    return [(cols[off[i]:off[i + 1]].copy(), vals[off[i]:off[i + 1]].copy()) for i in range(len(r))]


def num_threads() -> int:
    """Threads the oracle's multi-threaded paths use (OpenMP)."""
    return lib().or_num_threads()


def davidson_dense(A, nvalues=1, init=None, tol=1e-4, etol=1e-8, max_iters=50):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    ev = np.zeros(nvalues)
    vec = np.zeros((nvalues, n))
    st = np.zeros(4, dtype=np.int32)
    ip = None
    if init is not None:
        init = np.ascontiguousarray(init, dtype=np.float64)
        ip = _p(init, _dp)
    r = lib().or_davidson_dense(_p(A, _dp), n, nvalues, ip, tol, etol, max_iters, _p(ev, _dp), _p(vec, _dp),
                                _p(st, _ip))
    return r, ev, vec, dict(iters=int(st[0]), n_sigma=int(st[1]), converged=bool(st[2]), reason=int(st[3]))


def sym_eig(A):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    w = np.zeros(n)
    Y = np.zeros((n, n))
    lib().or_sym_eig(n, _p(A, _dp), _p(w, _dp), _p(Y, _dp))
    return w, Y


def mgs(B, start, end):
    """MGS::orthonormalize on columns of B (N x k); returns (ok, B')."""
    Bc = np.asfortranarray(B, dtype=np.float64).copy(order="F")
    flat = Bc.reshape(-1, order="F")
    flat = np.ascontiguousarray(flat)
    ok = lib().or_mgs(_p(flat, _dp), B.shape[0], start, end)
    return bool(ok), flat.reshape(B.shape, order="F")


class Hci:
    """init_var_wf + variational (src/wf/mod.rs:1687-1740, src/var/mod.rs:59-134)."""

    def __init__(self, ham: Ham, nup, ndn, eps_var, z_sym=1, builder=0, grouped_singles=True):
        self.ham = ham
        self.ptr = lib().or_hci_new(ham.ptr, nup, ndn, z_sym, eps_var, builder, 1 if grouped_singles else 0)
        if not self.ptr:
            raise ValueError("unsupported HCI start")

    def set_options(self, dav_max_iter=50, parallel=False):
        """Davidson cap of each solve (the reference fixes 50) and the multi-threaded
        build and sigma."""
        lib().or_hci_set_options(self.ptr, int(dav_max_iter), 1 if parallel else 0)
        return self

    def run(self, max_iter=20) -> float:
        return lib().or_hci_run(self.ptr, max_iter)

    def step(self) -> bool:
        return bool(lib().or_hci_step(self.ptr))

    def step_bounded(self, max_dets) -> int:
        """One iteration unless its selection takes the space past max_dets: 0 done, 1 converged,
        2 stopped after the selection (the state then only serves the earlier export)."""
        return int(lib().or_hci_step_bounded(self.ptr, int(max_dets)))

    @property
    def energy(self):
        return lib().or_hci_energy(self.ptr)

    @property
    def ndets(self):
        return lib().or_hci_ndets(self.ptr)

    def export(self):
        n = self.ndets
        dets = np.zeros((n, 4), dtype=np.uint64)
        coeffs = np.zeros(n)
        diag = np.zeros(n)
        lib().or_hci_export(self.ptr, _p(dets, _u64p), _p(coeffs, _dp), _p(diag, _dp))
        return dets, coeffs, diag

    def log(self):
        eps = np.zeros(64)
        en = np.zeros(64)
        nd = np.zeros(64, dtype=np.uint64)
        nz = np.zeros(64, dtype=np.uint64)
        dv = np.zeros((64, 4), dtype=np.int32)
        k = lib().or_hci_log(self.ptr, _p(eps, _dp), _p(en, _dp), _p(nd, _u64p), _p(nz, _u64p), _p(dv, _ip))
        return [dict(eps=eps[i], energy=en[i], ndets=int(nd[i]), nnz=int(nz[i]), dav=dv[i].tolist()) for i in range(k)]

    def excite_gen_max(self):
        out = np.zeros(3)
        lib().or_excite_gen_max(self.ptr, _p(out, _dp))
        return out

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.or_hci_free(self.ptr)
            self.ptr = None


def dets_from_orbs(rows):
    """[(up_orbs, dn_orbs), ...] -> uint64[N, 4]."""
    out = np.zeros((len(rows), 4), dtype=np.uint64)
    for k, (u, d) in enumerate(rows):
        up = sum(1 << int(b) for b in u)
        dn = sum(1 << int(b) for b in d)
        out[k] = [up & (2**64 - 1), up >> 64, dn & (2**64 - 1), dn >> 64]
    return out
