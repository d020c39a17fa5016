"""The restated uiuc_7sp table against the reference's mechanism file.

``tests/golden/uiuc_7sp_mechanism.json`` holds the numbers of
mirgecom/mechanisms/uiuc_7sp.yaml as the file states them (made by
tests/golden/make_mechanism_fixture.py).  This test converts them here,
independently of the library's YAML reader, into the SI table the kernels
use (kg, kmol, m, s, K) and compares every entry of ``UIUC_7SP``:
molecular weights from the compositions, NASA-7 ranges and coefficients,
stoichiometry, forward orders (explicit orders, else the stoichiometric
coefficients), reversibility, and the rate constants (A converted from
(cm^3/mol)^(n-1)/s, Ea from cal/mol to an activation temperature).
"""

import json
import os

import numpy as np

from mirgecom_b200.thermochemistry import (ATOMIC_WEIGHTS, GAS_CONSTANT, UIUC_7SP,
                                           load_cantera_yaml)

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                       "uiuc_7sp_mechanism.json")


def _fixture():
    with open(FIXTURE) as f:
        return json.load(f)


def _side(text, names):
    """Stoichiometric vector of one side of an equation ('CO + 0.5 O2')."""
    nu = np.zeros(len(names))
    for term in text.split("+"):
        parts = term.split()
        coef, name = (float(parts[0]), parts[1]) if len(parts) == 2 else (1.0, parts[0])
        nu[names.index(name)] += coef
    return nu


def test_species_and_thermo_match_reference_file():
    fx = _fixture()
    m = UIUC_7SP
    assert fx["units"] == {"length": "cm", "quantity": "mol", "activation-energy": "cal/mol"}
    assert list(m.species) == fx["species_order"]
    for k, name in enumerate(m.species):
        sp = fx["species"][name]
        assert sp["model"] == "NASA7"
        mw = sum(ATOMIC_WEIGHTS[el] * n for el, n in sp["composition"].items())
        assert m.molecular_weights[k] == mw, name
        tr = sp["temperature_ranges"]
        assert len(tr) == 3 and m.t_mid[k] == tr[1], name
        assert np.array_equal(m.nasa_low[k], np.array(sp["data"][0])), name
        assert np.array_equal(m.nasa_high[k], np.array(sp["data"][1])), name


def test_reactions_match_reference_file():
    fx = _fixture()
    m = UIUC_7SP
    names = list(m.species)
    assert m.nreactions == len(fx["reactions"])
    for i, r in enumerate(fx["reactions"]):
        eq = r["equation"].split("#")[0]
        rev = "<=>" in eq
        lhs, rhs = eq.split("<=>" if rev else "=>")
        nu_r, nu_p = _side(lhs, names), _side(rhs, names)
        assert np.array_equal(m.nu_reac[i], nu_r), i
        assert np.array_equal(m.nu_prod[i], nu_p), i
        assert bool(m.reversible[i]) == rev, i
        orders = nu_r.copy()
        for name, o in r["orders"].items():
            orders[names.index(name)] = float(o)
        assert np.array_equal(m.orders_fwd[i], orders), i
        # A in (cm^3/mol)^(n-1)/s with n the total forward order; 1 cm^3/mol is
        # 1e-3 m^3/kmol
        n = orders.sum()
        a_si = float(r["A"]) * 1e-3 ** (n - 1)
        assert abs(np.exp(m.log_a[i]) - a_si) <= 1e-13 * a_si, i
        assert m.beta[i] == float(r["b"]), i
        ta = float(r["Ea"]) * 4.184 * 1000.0 / GAS_CONSTANT
        assert abs(m.t_act[i] - ta) <= 1e-13 * ta, i


def test_yaml_reader_reproduces_table():
    """The library's reader, given a YAML text written from the fixture's
    numbers, yields the same table as the restatement."""
    import yaml
    fx = _fixture()
    doc = {"units": fx["units"],
           "phases": [{"name": "gas", "species": fx["species_order"]}],
           "species": [{"name": n, "composition": s["composition"],
                        "thermo": {"model": s["model"],
                                   "temperature-ranges": s["temperature_ranges"],
                                   "data": s["data"]}}
                       for n, s in fx["species"].items()],
           "reactions": [{"equation": r["equation"],
                          "rate-constant": {"A": r["A"], "b": r["b"], "Ea": r["Ea"]},
                          **({"orders": r["orders"]} if r["orders"] else {})}
                         for r in fx["reactions"]]}
    m = load_cantera_yaml(yaml.safe_dump(doc))
    for attr in ("molecular_weights", "t_mid", "nasa_low", "nasa_high", "nu_reac", "nu_prod",
                 "orders_fwd", "reversible", "log_a", "beta", "t_act"):
        assert np.array_equal(getattr(m, attr), getattr(UIUC_7SP, attr)), attr
