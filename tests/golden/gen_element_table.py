#!/usr/bin/env python3
"""Regenerate elements.json from the reference's element table.

The scattering data (IT92 / Cromer-Mann x-ray coefficients and bound coherent
neutron lengths) are physical constants that must be identical to the ones the
reference uses, so they are taken from thatstar/sqcalc's generated module
src/sqc_element_data.f90 rather than retyped.  Run from the repository root,
given the reference's element module:

    python tests/golden/gen_element_table.py /path/to/sqcalc/src/sqc_element_data.f90

It writes sqcalc_b200/data/elements.json.
"""
import json
import os
import re
import sys


def parse(path):
    text = open(path).read()
    text = re.sub(r"&\s*\n\s*", " ", text)  # join continuation lines
    arrays = {}
    for m in re.finditer(r"parameter, public :: (\w+)\([^)]*\)\s*=\s*(reshape\()?\[(.*?)\]", text):
        name, body = m.group(1), m.group(3)
        items = [x.strip() for x in body.split(",")]
        vals = []
        for it in items:
            if it.startswith('"'):
                vals.append(it.strip('"').strip())
            elif it in (".true.", ".false."):
                vals.append(it == ".true.")
            else:
                vals.append(float(it.replace("d", "e")) if ("." in it or "d" in it) else int(it))
        arrays[name] = vals
    return arrays


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: gen_element_table.py <sqcalc>/src/sqc_element_data.f90")
    src = sys.argv[1]
    a = parse(src)
    ns = len(a["species_label"])
    xa = a["species_xray_a"]
    xb = a["species_xray_b"]
    table = {
        "source": "thatstar/sqcalc src/sqc_element_data.f90 (IT92 x-ray, NN92 neutron)",
        "element_symbol": a["element_symbol"],
        "element_neutron_b": a["element_neutron_b"],
        "element_has_neutron": a["element_has_neutron"],
        "element_neutral_species": a["element_neutral_species"],
        "species_label": a["species_label"],
        "species_element": a["species_element"],
        "species_xray": [xa[4 * i:4 * i + 4] + xb[4 * i:4 * i + 4] + [a["species_xray_c"][i]]
                         for i in range(ns)],
        "species_alias": dict(zip(a["species_alias_from"], a["species_alias_to"])),
    }
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    out = os.path.join(root, "sqcalc_b200", "data", "elements.json")
    with open(out, "w") as fh:
        json.dump(table, fh, separators=(",", ":"))
    print("wrote", out, "species", ns, "elements", len(a["element_symbol"]))


if __name__ == "__main__":
    main()
