"""Shared fixtures: golden systems, synthetic systems and oracle runs (cached)."""
from __future__ import annotations

import functools
import json
import os

import numpy as np

from oracle import oracle as O
from risq_b200.fcidump import Integrals, synthetic_integrals

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_energies():
    with open(os.path.join(GOLDEN_DIR, "reference_energies.json")) as f:
        return json.load(f)


@functools.lru_cache(maxsize=None)
def golden_system(name):
    z = np.load(os.path.join(GOLDEN_DIR, f"{name}_ints.npz"))
    ints = Integrals(int(z["norb"]), float(z["nuc"]), z["one_body"].copy(), z["two_body"].copy())
    params = dict(norb=int(z["norb"]), norb_core=int(z["norb_core"]), nup=int(z["nup"]), ndn=int(z["ndn"]),
                  eps_var=float(z["eps_var"]))
    return ints, params


def oracle_ham(ints: Integrals, ncore=0):
    return O.Ham.from_arrays(ints.norb, ncore, ints.nuc, ints.one_body, ints.two_body)


@functools.lru_cache(maxsize=None)
def oracle_hci(name):
    """Oracle HCI run on a golden system: (energy, dets, coeffs, diag, log)."""
    ints, p = golden_system(name)
    h = oracle_ham(ints, p["norb_core"])
    hci = O.Hci(h, p["nup"], p["ndn"], p["eps_var"])
    e = hci.run(20)
    dets, coeffs, diag = hci.export()
    return e, dets, coeffs, diag, hci.log()


@functools.lru_cache(maxsize=None)
def synthetic_hci(n, nel, eps, seed=0, max_iter=20):
    """Oracle HCI on seeded synthetic integrals (n orbitals, nel up + nel down)."""
    ints = synthetic_integrals(n, seed)
    h = oracle_ham(ints, 0)
    hci = O.Hci(h, nel, nel, eps)
    e = hci.run(max_iter)
    dets, coeffs, diag = hci.export()
    return ints, e, dets, coeffs, diag, hci.log()


def random_connected_pairs(dets, rng, n_pairs, norb):
    """Random (d1, d2) pairs: dets of the set and single/double/triple excitations of them
    within the norb orbitals."""
    from risq_b200.fcidump import dets_from_ints, dets_to_ints
    base = dets_to_ints(dets)
    out1, out2 = [], []
    for _ in range(n_pairs):
        u, d = base[rng.integers(len(base))]
        kind = rng.integers(6)
        u2, d2 = u, d

        def move(x, k):
            for _ in range(k):
                occ = [i for i in range(norb) if x >> i & 1]
                vir = [i for i in range(norb) if not x >> i & 1]
                x = (x & ~(1 << int(rng.choice(occ)))) | (1 << int(rng.choice(vir)))
            return x
        if kind == 0:
            u2 = move(u, 1)
        elif kind == 1:
            d2 = move(d, 1)
        elif kind == 2:
            u2 = move(u, 2)
        elif kind == 3:
            d2 = move(d, 2)
        elif kind == 4:
            u2, d2 = move(u, 1), move(d, 1)
        else:
            u2, d2 = move(u, 2), move(d, 1)
        out1.append((u, d))
        out2.append((u2, d2))
    return dets_from_ints(out1), dets_from_ints(out2)


def csr_to_dict(rp, cols, vals):
    d = {}
    for i in range(len(rp) - 1):
        for k in range(rp[i], rp[i + 1]):
            d[(i, int(cols[k]))] = float(vals[k])
    return d
