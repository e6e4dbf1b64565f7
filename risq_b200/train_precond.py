"""Train the learned Davidson preconditioner on synthetic systems (run on a GPU).

    python -m risq_b200.train_precond --norb 20 --nel 8 --eps 1e-3 --seeds 1-8 \
        --out risq_b200/data/precond_mlp_n20.npz

Training systems: seeded synthetic integrals (risq_b200.fcidump.synthetic_integrals)
with the given orbitals / electrons, their HCI determinant sets made by this
library's device variational stage, and per-determinant target factors from the
second-order self-energy at the converged FP64 Davidson energy, with features taken
at the Ritz values of the FP64 DPR trajectory (risq_b200.learned).  The network is then evaluated on seed 0
(held out): Davidson iterations and time with and without it.

--universal trains a network of the orbital-count-independent layout
(risq_b200.learned.adapt), which can be evaluated on a system of another size:

    python -m risq_b200.train_precond --universal --norb 20 --nel 8 --eps 1e-3 --seeds 1-8 \
        --eval-norb 24 --eval-nel 10 --eval-eps 1e-3
"""
from __future__ import annotations

import argparse
import json
import time

from . import _capi as A
from . import learned
from .fcidump import synthetic_integrals
from .gpu import GpuHam


def parse_seeds(s):
    if "-" in s:
        a, b = s.split("-")
        return list(range(int(a), int(b) + 1))
    return [int(x) for x in s.split(",")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--norb", type=int, default=20)
    ap.add_argument("--nel", type=int, default=8)
    ap.add_argument("--eps", type=float, default=1e-3)
    ap.add_argument("--seeds", default="1-8")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--n-energies", type=int, default=12)
    ap.add_argument("--per-energy", type=int, default=50000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=None)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--universal", action="store_true", help="orbital-count-independent layout")
    ap.add_argument("--eval-norb", type=int, default=None)
    ap.add_argument("--eval-nel", type=int, default=None)
    ap.add_argument("--eval-eps", type=float, default=None)
    args = ap.parse_args()
    t0 = time.time()
    systems = []
    for s in parse_seeds(args.seeds):
        ints = synthetic_integrals(args.norb, s)
        with GpuHam(ints, args.device) as g:
            e, dets, c, diag, log = g.variational(args.nel, args.nel, args.eps, dav_max_iter=2000, precision=-1)
        print(f"# seed {s}: {len(dets)} dets, E = {e:.8f}", flush=True)
        systems.append((ints, dets, diag))
    model, hist = learned.train_from_systems(systems, args.norb, epochs=args.epochs, lr=args.lr,
                                             n_energies=args.n_energies, per_energy=args.per_energy,
                                             device=args.device, universal=args.universal)
    print("# loss per epoch:", " ".join(f"{x:.4g}" for x in hist), flush=True)
    out = args.out or (learned.universal_model_path() if args.universal else learned.default_model_path(args.norb))
    model.save(out)
    # held-out evaluation on seed 0 (another orbital count for a universal network)
    en, ee = args.eval_norb or args.norb, args.eval_nel or args.nel
    eps = args.eval_eps or args.eps
    ints = synthetic_integrals(en, 0)
    res = {}
    with GpuHam(ints, args.device) as g:
        e, dets, c, diag, log = g.variational(ee, ee, eps, dav_max_iter=2000, precision=-1)
        g.set_dets(dets, 0, diag)
        learned.install(g, learned.adapt(model, ints, 2 * ee) if args.universal else model)
        for prec, mode, pc, name in [(A.FP64, A.MODE_FP64, A.PRECOND_DPR, "fp64_dpr"),
                                     (A.FP64, A.MODE_FP64, A.PRECOND_LEARNED, "fp64_learned"),
                                     (A.MIXED, A.MODE_MIXED, A.PRECOND_DPR, "mixed_dpr"),
                                     (A.MIXED, A.MODE_MIXED, A.PRECOND_LEARNED, "mixed_learned")]:
            g.build(prec)
            t = time.perf_counter()
            r = g.davidson(1, None, 1e-4, 1e-8, 2000, mode=mode, precond=pc)
            res[name] = dict(iters=r.stats["iters"], ms=1e3 * (time.perf_counter() - t),
                             energy=float(r.eigenvalues[0]), fallbacks=r.stats["learned_fallbacks"],
                             converged=r.converged)
    e0 = res["fp64_dpr"]["energy"]
    for v in res.values():
        v["dE_uHa"] = abs(v["energy"] - e0) * 1e6
    print(json.dumps({"held_out_seed": 0, "eval": dict(norb=en, nel=ee, eps=eps), "universal": args.universal,
                      "n_dets": int(len(dets)), "train_seconds": time.time() - t0, "results": res}))


if __name__ == "__main__":
    main()
