"""Generate the committed golden fixtures from the reference checkout.

Run in a container that has the reference checkout, giving its path:
    python tests/golden/make_fixtures.py /path/to/reference

For each example system with a pinned variational energy in the reference's
integration tests (tests/integration_test_suite.rs:28-93) this stores the
integrals of examples/<name>/FCIDUMP in the reference's packed layout (read by
the CPU oracle, cross-checked against risq_b200.fcidump.read_fcidump) together
with the system parameters of examples/<name>/in.json, as
tests/golden/<name>_ints.npz.  The golden energies themselves are written to
tests/golden/reference_energies.json with the line they come from.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from risq_b200.fcidump import read_fcidump  # noqa: E402

# name -> (E_var, source line in tests/integration_test_suite.rs, test status there)
GOLDEN = {
    "be": (-14.6168425934, 34, "run"),
    "he2": (-5.5565366249, 44, "run"),
    "li2": (-14.6198472544, 64, "run"),
    "be2": (-28.6608360148, 74, "run"),
    "f2": (-199.0913503137, 84, "ignored as slow (:277)"),
}


def main(ref: str) -> None:
    energies = {"tolerance": 1e-6, "tolerance_source": "tests/integration_test_suite.rs:13", "systems": {}}
    for name, (e, line, status) in GOLDEN.items():
        cfg = json.load(open(os.path.join(ref, "examples", name, "in.json")))
        path = os.path.join(ref, "examples", name, "FCIDUMP")
        h = O.Ham.from_fcidump(path, cfg["norb"], cfg["norb_core"])
        nuc, ob, tb = h.arrays()
        py = read_fcidump(path, cfg["norb"])
        assert py.nuc == nuc and np.array_equal(py.one_body, ob) and np.array_equal(py.two_body, tb), name
        np.savez_compressed(os.path.join(HERE, f"{name}_ints.npz"), one_body=ob, two_body=tb, nuc=np.float64(nuc),
                            norb=cfg["norb"], norb_core=cfg["norb_core"], nup=cfg["nup"], ndn=cfg["ndn"],
                            eps_var=cfg["eps_var"])
        energies["systems"][name] = {"e_var": e, "source": f"tests/integration_test_suite.rs:{line}",
                                     "status": status, "norb": cfg["norb"], "norb_core": cfg["norb_core"],
                                     "nup": cfg["nup"], "ndn": cfg["ndn"], "eps_var": cfg["eps_var"]}
        print(name, "ok")
    with open(os.path.join(HERE, "reference_energies.json"), "w") as f:
        json.dump(energies, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py /path/to/reference")
    main(sys.argv[1])
