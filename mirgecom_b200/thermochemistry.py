"""Thermochemistry data for the mixture EOS and the Arrhenius source terms.

The reference takes these from a Cantera-format YAML mechanism through
pyrometheus (mirgecom/thermochemistry.py:51-183, mirgecom/eos.py:540-888,
mirgecom/mechanisms/__init__.py:66-79).  Here a mechanism is a plain table in
SI units (kg, kmol, m, s, K), the units pyrometheus generates code in:

* species molecular weights from IUPAC conventional atomic weights
  (H 1.008, C 12.011, N 14.007, O 15.999 -- the values Cantera uses);
* NASA 7-coefficient polynomials, low range below ``T_mid``, high range
  above it (``T > T_mid`` picks the high range);
* reactions with forward orders, optional reversibility (reverse rate from
  the equilibrium constant built on the NASA-7 Gibbs energies at
  p0 = 1 atm), and modified-Arrhenius rate constants
  ``k = A T^b exp(-Ta / T)`` with ``A`` converted from the file's
  (cm, mol) units and ``Ta = Ea / R``.

``UIUC_7SP`` is the reduced ethylene/air mechanism of
mirgecom/mechanisms/uiuc_7sp.yaml:1-154 (species order from line 11, NASA-7
data lines 19-143, reactions lines 146-154), restated as numbers; the table
must agree with that file, and ``load_cantera_yaml`` reads the same subset of
the Cantera YAML format so the two can be compared.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GAS_CONSTANT = 8314.46261815324      # J / (kmol K)
ONE_ATM = 101325.0                   # Pa
CAL_TO_J = 4.184

ATOMIC_WEIGHTS = {"H": 1.008, "C": 12.011, "N": 14.007, "O": 15.999}


@dataclass
class Mechanism:
    name: str
    species: list                 # names, in conserved-variable order
    molecular_weights: np.ndarray  # (Ns,) kg/kmol
    t_mid: np.ndarray             # (Ns,)
    nasa_low: np.ndarray          # (Ns, 7)
    nasa_high: np.ndarray         # (Ns, 7)
    # reactions
    nu_reac: np.ndarray           # (Nr, Ns) reactant stoichiometry
    nu_prod: np.ndarray           # (Nr, Ns) product stoichiometry
    orders_fwd: np.ndarray        # (Nr, Ns) forward concentration exponents
    reversible: np.ndarray        # (Nr,) bool
    log_a: np.ndarray             # (Nr,) ln(A) in SI (kmol, m^3, s)
    beta: np.ndarray              # (Nr,) temperature exponent
    t_act: np.ndarray             # (Nr,) activation temperature Ea/R  [K]

    @property
    def nspecies(self):
        return len(self.species)

    @property
    def nreactions(self):
        return self.nu_reac.shape[0]

    @property
    def nu_net(self):
        return self.nu_prod - self.nu_reac

    def species_index(self, name):
        return self.species.index(name)


def _molecular_weight(composition):
    return sum(ATOMIC_WEIGHTS[el] * n for el, n in composition.items())


def _build(name, species, compositions, thermo, reactions, units_cgs=True):
    ns = len(species)
    mw = np.array([_molecular_weight(compositions[s]) for s in species])
    tmid = np.array([thermo[s][0][1] for s in species], dtype=np.float64)
    low = np.array([thermo[s][1] for s in species], dtype=np.float64)
    high = np.array([thermo[s][2] for s in species], dtype=np.float64)
    nr = len(reactions)
    nu_r = np.zeros((nr, ns))
    nu_p = np.zeros((nr, ns))
    orders = np.zeros((nr, ns))
    rev = np.zeros(nr, dtype=bool)
    log_a = np.zeros(nr)
    beta = np.zeros(nr)
    t_act = np.zeros(nr)
    for i, rxn in enumerate(reactions):
        for s, n in rxn["reactants"].items():
            nu_r[i, species.index(s)] = n
        for s, n in rxn["products"].items():
            nu_p[i, species.index(s)] = n
        orders[i] = nu_r[i]
        for s, n in rxn.get("orders", {}).items():
            orders[i, species.index(s)] = n
        rev[i] = rxn["reversible"]
        a = rxn["A"]
        total_order = orders[i].sum()
        if units_cgs:
            # (cm^3/mol)^(order-1) / s  ->  (m^3/kmol)^(order-1) / s
            a = a * (1e-3) ** (total_order - 1.0)
        log_a[i] = np.log(a)
        beta[i] = rxn["b"]
        t_act[i] = rxn["Ea_cal"] * CAL_TO_J * 1000.0 / GAS_CONSTANT
    return Mechanism(name=name, species=list(species), molecular_weights=mw,
                     t_mid=tmid, nasa_low=low, nasa_high=high, nu_reac=nu_r,
                     nu_prod=nu_p, orders_fwd=orders, reversible=rev,
                     log_a=log_a, beta=beta, t_act=t_act)


_UIUC7_SPECIES = ["C2H4", "O2", "CO2", "CO", "H2O", "H2", "N2"]
_UIUC7_COMPOSITION = {
    "C2H4": {"C": 2, "H": 4}, "O2": {"O": 2}, "CO2": {"C": 1, "O": 2},
    "CO": {"C": 1, "O": 1}, "H2O": {"H": 2, "O": 1}, "H2": {"H": 2},
    "N2": {"N": 2},
}
# name: ((T_low, T_mid, T_high), low-range a0..a6, high-range a0..a6)
_UIUC7_THERMO = {
    "O2": ((200.0, 1000.0, 3500.0),
           [3.78245636, -2.99673416e-03, 9.84730201e-06, -9.68129509e-09,
            3.24372837e-12, -1063.94356, 3.65767573],
           [3.28253784, 1.48308754e-03, -7.57966669e-07, 2.09470555e-10,
            -2.16717794e-14, -1088.45772, 5.45323129]),
    "H2O": ((200.0, 1000.0, 3500.0),
            [4.19864056, -2.0364341e-03, 6.52040211e-06, -5.48797062e-09,
             1.77197817e-12, -3.02937267e+04, -0.849032208],
            [3.03399249, 2.17691804e-03, -1.64072518e-07, -9.7041987e-11,
             1.68200992e-14, -3.00042971e+04, 4.9667701]),
    "CO": ((200.0, 1000.0, 3500.0),
           [3.57953347, -6.1035368e-04, 1.01681433e-06, 9.07005884e-10,
            -9.04424499e-13, -1.4344086e+04, 3.50840928],
           [2.71518561, 2.06252743e-03, -9.98825771e-07, 2.30053008e-10,
            -2.03647716e-14, -1.41518724e+04, 7.81868772]),
    "CO2": ((200.0, 1000.0, 3500.0),
            [2.35677352, 8.98459677e-03, -7.12356269e-06, 2.45919022e-09,
             -1.43699548e-13, -4.83719697e+04, 9.90105222],
            [3.85746029, 4.41437026e-03, -2.21481404e-06, 5.23490188e-10,
             -4.72084164e-14, -4.8759166e+04, 2.27163806]),
    "C2H4": ((200.0, 1000.0, 3500.0),
             [3.95920148, -7.57052247e-03, 5.70990292e-05, -6.91588753e-08,
              2.69884373e-11, 5089.77593, 4.09733096],
             [2.03611116, 0.0146454151, -6.71077915e-06, 1.47222923e-09,
              -1.25706061e-13, 4939.88614, 10.3053693]),
    "N2": ((300.0, 1000.0, 5000.0),
           [3.298677, 1.4082404e-03, -3.963222e-06, 5.641515e-09,
            -2.444854e-12, -1020.8999, 3.950372],
           [2.92664, 1.4879768e-03, -5.68476e-07, 1.0097038e-10,
            -6.753351e-15, -922.7977, 5.980528]),
    "H2": ((300.0, 1000.0, 5000.0),
           [2.34433112, 7.98052075e-03, -1.9478151e-05, 2.01572094e-08,
            -7.37611761e-12, -917.935173, 0.683010238],
           [3.3372792, -4.94024731e-05, 4.99456778e-07, -1.79566394e-10,
            2.00255376e-14, -950.158922, -3.20502331]),
}
_UIUC7_REACTIONS = [
    {"reactants": {"C2H4": 1, "O2": 1}, "products": {"CO": 2, "H2": 2},
     "orders": {"C2H4": 0.5, "O2": 0.65}, "reversible": False,
     "A": 1.0e+10, "b": 0.0, "Ea_cal": 36000.0},
    {"reactants": {"CO": 1, "O2": 0.5}, "products": {"CO2": 1},
     "reversible": True, "A": 1.1e+07, "b": 0.7, "Ea_cal": 11000.0},
    {"reactants": {"H2": 1, "O2": 0.5}, "products": {"H2O": 1},
     "orders": {"H2": 0.75, "O2": 0.5}, "reversible": False,
     "A": 7.0e+08, "b": 0.0, "Ea_cal": 12000.0},
]

UIUC_7SP = _build("uiuc_7sp", _UIUC7_SPECIES, _UIUC7_COMPOSITION,
                  _UIUC7_THERMO, _UIUC7_REACTIONS)


def get_mechanism(name="uiuc_7sp"):
    if name in ("uiuc_7sp", "uiuc7"):
        return UIUC_7SP
    raise ValueError(f"unknown mechanism {name!r}")


def _parse_equation(eq):
    """Split 'A + 0.5 B <=> C' into (reactants, products, reversible)."""
    if "<=>" in eq:
        lhs, rhs = eq.split("<=>")
        rev = True
    elif "=>" in eq:
        lhs, rhs = eq.split("=>")
        rev = False
    else:
        lhs, rhs = eq.split("=")
        rev = True

    def side(text):
        out = {}
        for term in text.split(" + "):
            parts = term.split()
            if len(parts) == 2:
                out[parts[1]] = out.get(parts[1], 0.0) + float(parts[0])
            else:
                out[parts[0]] = out.get(parts[0], 0.0) + 1.0
        return out
    return side(lhs.strip()), side(rhs.strip()), rev


def load_cantera_yaml(path_or_text, name=None):
    """Read the NASA-7/elementary-reaction subset of a Cantera YAML file."""
    import os

    import yaml
    text = path_or_text
    if os.path.exists(str(path_or_text)):
        with open(path_or_text) as f:
            text = f.read()
    doc = yaml.safe_load(text)
    units = doc.get("units", {})
    if units.get("length", "cm") != "cm" or units.get("quantity", "mol") != "mol" \
            or units.get("activation-energy", "cal/mol") != "cal/mol":
        raise ValueError("only cm/mol/cal-mol mechanisms are supported")
    phase = doc["phases"][0]
    species = list(phase["species"])
    comp = {}
    thermo = {}
    for sp in doc["species"]:
        comp[sp["name"]] = sp["composition"]
        th = sp["thermo"]
        if th["model"] != "NASA7":
            raise ValueError("only NASA7 thermo is supported")
        thermo[sp["name"]] = (tuple(th["temperature-ranges"]), th["data"][0],
                              th["data"][1])
    reactions = []
    for r in doc["reactions"]:
        reac, prod, rev = _parse_equation(r["equation"].split("#")[0])
        rc = r["rate-constant"]
        reactions.append({"reactants": reac, "products": prod,
                          "orders": r.get("orders", {}), "reversible": rev,
                          "A": float(rc["A"]), "b": float(rc["b"]),
                          "Ea_cal": float(rc["Ea"])})
    return _build(name or "mechanism", species, comp, thermo, reactions)
