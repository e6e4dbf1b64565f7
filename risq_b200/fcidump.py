"""FCIDUMP integrals in the reference's packed layout, and the synthetic generator.

Packed layout (src/utils/ints.rs:38-68, src/ham/read_ints.rs:79-80): 1-based
orbital indices, one_body[combine_2(p, q)] = h_pq and
two_body[combine_4(p, q, r, s)] = (pq|rs), with the 8-fold symmetry folded in.

``read_fcidump`` follows read_ints (src/ham/read_ints.rs:73-190): a line whose
first token does not parse as a float is a header line and is skipped; then
``value p q r s``: all zero -> nuclear repulsion, r = s = 0 -> one-body,
otherwise two-body; indices outside [0, norb] are an error; later lines
overwrite earlier ones that map to the same packed entry.  The core / valence
split is the ascending h_ii order (stable), lowest ``ncore`` are core.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


def combine_2(p: int, q: int) -> int:
    i, j = abs(p), abs(q)
    return (i * (i - 1)) // 2 + j if i > j else (j * (j - 1)) // 2 + i


def combine_4(p: int, q: int, r: int, s: int) -> int:
    return combine_2(combine_2(p, q), combine_2(r, s))


def packed_sizes(norb: int):
    n1 = combine_2(norb + 1, norb + 1)
    return n1, combine_2(n1, n1)


@dataclasses.dataclass
class Integrals:
    norb: int
    nuc: float
    one_body: np.ndarray  # float64[n1]
    two_body: np.ndarray  # float64[n2]

    def h(self, p: int, q: int) -> float:
        """One-body h_pq, 0-based indices (Ham::one_body, src/ham/mod.rs:65-67)."""
        return float(self.one_body[combine_2(p + 1, q + 1)])

    def core_valence(self, ncore: int):
        """Core/valence split by ascending h_ii, stable (src/ham/read_ints.rs:161-184)."""
        order = sorted(range(self.norb), key=lambda i: self.h(i, i))
        return order[:ncore], order[ncore:]


def _is_float_token(tok: str):
    try:
        v = float(tok)
    except ValueError:
        return None
    low = tok.lower()
    if "inf" in low or "nan" in low or "x" in low:
        return None
    return v


def read_fcidump(path: str, norb: int) -> Integrals:
    n1, n2 = packed_sizes(norb)
    ob = np.zeros(n1)
    tb = np.zeros(n2)
    nuc = 0.0
    with open(path) as f:
        for lineno, line in enumerate(f, 1):
            toks = line.split()
            if not toks:
                raise ValueError(f"line {lineno}: Missing integral value")
            v = _is_float_token(toks[0])
            if v is None:
                continue
            if len(toks) < 5:
                raise ValueError(f"line {lineno}: Missing index")
            try:
                p, q, r, s = (int(t) for t in toks[1:5])
            except ValueError as e:
                raise ValueError(f"line {lineno}: Invalid index") from e
            for x in (p, q, r, s):
                if x < 0 or x > norb:
                    raise ValueError(f"line {lineno}: Index out of range [0, {norb}]: {x}")
            if p == q == r == s == 0:
                nuc = v
            elif r == 0 and s == 0:
                ob[combine_2(p, q)] = v
            else:
                tb[combine_4(p, q, r, s)] = v
    return Integrals(norb, nuc, ob, tb)


def write_fcidump(path: str, ints: Integrals, nelec: int, ms2: int = 0) -> None:
    """Unique entries only (p>=q, r>=s, pq>=rs), %.17g so a read gives the same doubles."""
    n = ints.norb
    with open(path, "w") as f:
        f.write(f" &FCI NORB={n:4d},NELEC={nelec:3d},MS2={ms2},\n")
        f.write("  ORBSYM=" + "1," * n + "\n")
        f.write("  ISYM=1,\n &END\n")
        for p in range(1, n + 1):
            for q in range(1, p + 1):
                pq = combine_2(p, q)
                for r in range(1, n + 1):
                    for s in range(1, r + 1):
                        rs = combine_2(r, s)
                        if rs > pq:
                            continue
                        v = ints.two_body[combine_2(pq, rs)]
                        if v != 0.0:
                            f.write(f" {float(v)!r} {p} {q} {r} {s}\n")
        for p in range(1, n + 1):
            for q in range(1, p + 1):
                v = ints.one_body[combine_2(p, q)]
                if v != 0.0:
                    f.write(f" {float(v)!r} {p} {q} 0 0\n")
        f.write(f" {float(ints.nuc)!r} 0 0 0 0\n")


def synthetic_integrals(n: int, seed: int = 0) -> Integrals:
    """Seeded synthetic molecule-like integrals.

    h_pp = -3 + 4 p / (n - 1); h_pq = 0.08 g_pq exp(-|p-q|/4) for p < q (symmetric);
    (pq|rs) = sum_{L < 2n} B^L_pq B^L_rs with B^L symmetric,
    B^L_pq = 0.25 g^L_pq exp(-|p-q|/3), which makes the ERI tensor 8-fold
    symmetric and positive semi-definite; E_core = 0; g ~ N(0, 1) drawn from
    numpy's default_rng(seed): first an n x n block for h (upper triangle used),
    then one n x n block per L (upper triangle incl. diagonal used).
    """
    rng = np.random.default_rng(seed)
    idx = np.arange(n)
    dist = np.abs(idx[:, None] - idx[None, :])
    g = rng.standard_normal((n, n))
    h = 0.08 * g * np.exp(-dist / 4.0)
    h = np.triu(h, 1)
    h = h + h.T
    h[idx, idx] = -3.0 + 4.0 * idx / (n - 1)
    L = 2 * n
    B = np.empty((L, n, n))
    for l in range(L):
        gl = rng.standard_normal((n, n))
        b = np.triu(0.25 * gl * np.exp(-dist / 3.0))
        B[l] = b + np.triu(b, 1).T
    # pair index (p >= q, 1-based combine_2) -> B^L_pq
    pairs_p, pairs_q = np.tril_indices(n)
    c2 = ((pairs_p + 1) * pairs_p) // 2 + (pairs_q + 1)  # combine_2(p+1, q+1) for p >= q
    Bp = B[:, pairs_p, pairs_q]  # L x npair
    V = Bp.T @ Bp  # npair x npair, (pq|rs)
    n1, n2 = packed_sizes(n)
    ob = np.zeros(n1)
    ob[c2] = h[pairs_p, pairs_q]
    tb = np.zeros(n2)
    a = c2[:, None]
    b = c2[None, :]
    big = np.maximum(a, b)
    small = np.minimum(a, b)
    c4 = (big * (big - 1)) // 2 + small
    tb[c4.ravel()] = V.ravel()
    return Integrals(n, 0.0, ob, tb)


def hf_det(nup: int, ndn: int) -> np.ndarray:
    """Lowest nup/ndn orbitals occupied (src/wf/mod.rs:1697-1698)."""
    up = (1 << nup) - 1
    dn = (1 << ndn) - 1
    return dets_from_ints([(up, dn)])[0]


def dets_from_ints(rows) -> np.ndarray:
    """[(up, dn) python ints] -> uint64[N, 4] {up_lo, up_hi, dn_lo, dn_hi}."""
    out = np.zeros((len(rows), 4), dtype=np.uint64)
    m = (1 << 64) - 1
    for k, (u, d) in enumerate(rows):
        out[k] = (u & m, u >> 64, d & m, d >> 64)
    return out


def dets_to_ints(dets: np.ndarray):
    return [(int(r[0]) | (int(r[1]) << 64), int(r[2]) | (int(r[3]) << 64)) for r in np.asarray(dets)]


def bytes_per_ints(norb: int) -> int:
    n1, n2 = packed_sizes(norb)
    return 8 * (n1 + n2)


__all__ = ["Integrals", "read_fcidump", "write_fcidump", "synthetic_integrals", "combine_2", "combine_4",
           "packed_sizes", "hf_det", "dets_from_ints", "dets_to_ints", "math"]
