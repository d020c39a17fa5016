"""Extract the numbers of the reference's uiuc_7sp mechanism into a fixture.

Reads mirgecom/mechanisms/uiuc_7sp.yaml of the reference checkout (Cantera
YAML, units cm / mol / cal/mol) with a plain YAML parse and writes
``uiuc_7sp_mechanism.json`` next to this script: the species order, each
species' elemental composition, NASA-7 temperature ranges and coefficient
rows, and each reaction's equation text, rate constant (A, b, Ea) and
explicit orders, exactly as the file states them (no unit conversion).
``tests/test_mechanism_fixture.py`` compares the library's restated table
against this fixture.  Run once where the reference is present::

    python tests/golden/make_mechanism_fixture.py [path/to/uiuc_7sp.yaml]
"""

import json
import os
import sys

import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT = "/root/reference/mirgecom/mechanisms/uiuc_7sp.yaml"


def extract(path):
    with open(path) as f:
        doc = yaml.safe_load(f)
    phase = doc["phases"][0]
    species = {}
    for sp in doc["species"]:
        th = sp["thermo"]
        species[sp["name"]] = {"composition": sp["composition"], "model": th["model"],
                               "temperature_ranges": th["temperature-ranges"],
                               "data": th["data"]}
    reactions = []
    for r in doc["reactions"]:
        rc = r["rate-constant"]
        reactions.append({"equation": r["equation"].strip(), "A": rc["A"], "b": rc["b"],
                          "Ea": rc["Ea"], "orders": r.get("orders", {})})
    return {"source": "mirgecom/mechanisms/uiuc_7sp.yaml", "units": doc["units"],
            "species_order": list(phase["species"]), "species": species,
            "reactions": reactions}


def main(argv):
    path = argv[1] if len(argv) > 1 else DEFAULT
    out = os.path.join(HERE, "uiuc_7sp_mechanism.json")
    with open(out, "w") as f:
        json.dump(extract(path), f, indent=1)
    print(out)


if __name__ == "__main__":
    main(sys.argv)
