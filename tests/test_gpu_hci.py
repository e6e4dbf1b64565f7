"""Device HCI selection and the variational loop against the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from risq_b200 import GpuHam, _capi
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["be", "li2", "be2", "f2"])
def test_find_new_dets_matches_oracle_step(name):
    """Each selection step returns the reference's new determinants, in its push order,
    with bitwise-equal diagonals (iterate_excites + push_and_spin_flipped)."""
    ints, p = H.golden_system(name)
    hci = O.Hci(H.oracle_ham(ints, p["norb_core"]), p["nup"], p["ndn"], p["eps_var"])
    states = []
    while True:
        d, c, g = hci.export()
        states.append((d, c, g))
        if hci.step() or len(states) > 20:
            break
    d_fin, _, g_fin = hci.export()
    log = hci.log()
    with GpuHam(ints) as gpu:
        for k in range(min(len(log), len(states))):
            d, c, g = states[k]
            eps = log[k]["eps"]
            n0 = len(d)
            n1 = log[k]["ndets"]
            gpu.set_dets(d, 0, g)
            nd, ng = gpu.find_new_dets(c, eps, eps == p["eps_var"], p["norb_core"])
            np.testing.assert_array_equal(nd, d_fin[n0:n1])
            np.testing.assert_array_equal(ng, g_fin[n0:n1])


@pytest.mark.parametrize("name", ["he2", "be", "li2", "be2", "f2"])
def test_variational_on_device_matches_golden(name):
    gold = H.golden_energies()["systems"][name]["e_var"]
    ints, p = H.golden_system(name)
    e_or, d_or, c_or, g_or, log_or = H.oracle_hci(name)
    with GpuHam(ints) as gpu:
        e, d, c, g, log = gpu.variational(p["nup"], p["ndn"], p["eps_var"], ncore=p["norb_core"])
    assert abs(e - gold) < 1e-6                       # tests/integration_test_suite.rs:13
    assert abs(e - e_or) < 1e-9
    assert len(d) == len(d_or)
    np.testing.assert_array_equal(d, d_or)            # same determinants in the same order
    np.testing.assert_array_equal(g, g_or)
    assert [l["n_dets"] for l in log] == [l["ndets"] for l in log_or]


def test_variational_synthetic_small():
    ints, e_or, d_or, c_or, g_or, log_or = H.synthetic_hci(10, 4, 1e-3)
    with GpuHam(ints) as gpu:
        e, d, c, g, log = gpu.variational(4, 4, 1e-3)
    assert abs(e - e_or) < 1e-6
    assert len(d) == len(d_or)
