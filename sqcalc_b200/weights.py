"""Scattering weights of the ``-w unit|neutron|xray`` / ``-m TYPE:LABEL`` options.

Host-side restatement of thatstar/sqcalc src/sqc_weights.f90 and the species
lookup of src/sqc_elements.f90 (table_find_species :304-352,
split_species_name :360-405, parse_charge_suffix :408-446).  The data table
(IT92 x-ray rows, bound coherent neutron lengths) is the reference's own,
regenerated into data/elements.json by data/gen_element_table.py.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

WEIGHT_UNIT, WEIGHT_NEUTRON, WEIGHT_XRAY = 0, 1, 2

_TABLE = None


def table():
    global _TABLE
    if _TABLE is None:
        with open(os.path.join(os.path.dirname(__file__), "data", "elements.json")) as fh:
            _TABLE = json.load(fh)
    return _TABLE


class MappingError(ValueError):
    pass


def scheme_from_name(name):
    """scheme_from_name (src/sqc_weights.f90:212-229)."""
    t = name.strip().lower()
    if t in ("unit", "none", "1"):
        return WEIGHT_UNIT
    if t in ("neutron", "n"):
        return WEIGHT_NEUTRON
    if t in ("xray", "x-ray", "x_ray", "x"):
        return WEIGHT_XRAY
    raise MappingError('unknown weighting scheme "%s"' % name)


def _normalise(sym):
    sym = sym.strip()[:2]
    return sym[:1].upper() + sym[1:2].lower() if sym else ""


def _element_index(sym):
    s = _normalise(sym)
    try:
        return table()["element_symbol"].index(s) + 1
    except ValueError:
        return 0


def _parse_suffix(text):
    """parse_charge_suffix: '', 'val', '2-', '1+', '+' -> (charge, valence, ok)."""
    t = text.strip().lower()
    if not t:
        return 0, False, True
    if t == "val":
        return 0, True, True
    digits = ""
    i = 0
    while i < len(t) and t[i].isdigit():
        digits += t[i]
        i += 1
    if i != len(t) - 1 or t[i] not in "+-":
        return 0, False, False
    if digits and int(digits) == 0:
        return 0, False, False
    q = int(digits) if digits else 1
    return (q if t[i] == "+" else -q), False, True


def _split(text):
    """split_species_name: the longest symbol that leaves a valid suffix."""
    text = text.strip()
    if len(text) >= 2 and _element_index(text[:2]) > 0:
        c, v, ok = _parse_suffix(text[2:])
        if ok:
            return _normalise(text[:2]), c, v, True
    if _element_index(text[:1]) == 0:
        return "", 0, False, False
    c, v, ok = _parse_suffix(text[1:])
    if not ok:
        return "", 0, False, False
    return _normalise(text[:1]), c, v, True


def find_species(text):
    """Resolve 'Si', 'O2-', 'Cval' to (species index (1-based, 0 if none),
    element index (1-based), canonical label)."""
    T = table()
    wanted = text.strip()
    for a, b in T["species_alias"].items():
        if a.lower() == wanted.lower():
            wanted = b
    sym, charge, val, ok = _split(wanted)
    if not ok:
        raise MappingError('unknown element symbol "%s" in the element mapping' % text.strip())
    el = _element_index(sym)
    if charge == 0 and not val:
        return T["element_neutral_species"][el - 1], el, sym
    canon = sym + "val" if val else "%s%d%s" % (sym, abs(charge), "+" if charge > 0 else "-")
    for idx, lab in enumerate(T["species_label"]):
        if lab.lower() == canon.lower():
            return idx + 1, el, lab
    states = ", ".join(lab for lab, e in zip(T["species_label"], T["species_element"]) if e == el)
    raise MappingError('element "%s" has no charge state "%s"; available: %s'
                       % (sym, text.strip(), states))


@dataclass
class WeightScheme:
    """weight_scheme_t (src/sqc_weights.f90:21-43)."""
    kind: int = WEIGHT_UNIT
    species: dict = field(default_factory=dict)        # type id -> label
    species_index: dict = field(default_factory=dict)  # type id -> x-ray species (1-based)
    element: dict = field(default_factory=dict)        # type id -> element (1-based)

    @classmethod
    def from_options(cls, weight="unit", mapping=None):
        s = cls(kind=scheme_from_name(weight) if isinstance(weight, str) else int(weight))
        if mapping:
            s.set_mapping(mapping)
        return s

    def set_mapping(self, spec):
        """scheme_set_mapping (:46-90): "1:Si,2:O"."""
        items = [x.strip() for x in spec.split(",") if x.strip()]
        if not items:
            raise MappingError("empty element mapping")
        for item in items:
            if ":" not in item or item.index(":") == 0 or item.endswith(":"):
                raise MappingError('cannot parse mapping entry "%s" (expected TYPE:SYMBOL)' % item)
            left, right = item.split(":", 1)
            try:
                t = int(left.strip())
            except ValueError:
                t = 0
            if t < 1:
                raise MappingError('invalid atom type id "%s" in the element mapping' % left)
            idx, el, lab = find_species(right)
            self.species[t] = lab
            self.species_index[t] = idx
            self.element[t] = el

    def mapped_types(self):
        return max(self.species) if self.species else 0

    def amplitude(self, t, q):
        """scheme_amplitude (:136-154)."""
        if self.kind == WEIGHT_NEUTRON:
            el = self.element.get(t, 0)
            return table()["element_neutron_b"][el - 1] if el else 0.0
        if self.kind == WEIGHT_XRAY:
            idx = self.species_index.get(t, 0)
            if idx < 1:
                return 0.0
            c = table()["species_xray"][idx - 1]
            stol2 = (q / (4.0 * math.acos(-1.0))) ** 2
            f = c[8]
            for i in range(4):
                f = f + c[i] * math.exp(-c[4 + i] * stol2)
            return f
        return 1.0

    def neutron_b(self, ntypes):
        return np.array([self.amplitude(t, 0.0) if self.kind == WEIGHT_NEUTRON else 1.0
                         for t in range(1, ntypes + 1)])

    def xray_rows(self, ntypes):
        """(ntypes, 9) rows a1..a4, b1..b4, c (zeros for a type without a row)."""
        out = np.zeros((ntypes, 9))
        for t in range(1, ntypes + 1):
            idx = self.species_index.get(t, 0)
            if idx >= 1:
                out[t - 1] = table()["species_xray"][idx - 1]
        return out

    def pair_label(self, ia, ib):
        """scheme_pair_label (:190-209)."""
        sa, sb = self.species.get(ia, ""), self.species.get(ib, "")
        if sa and sb:
            return "%s-%s" % (sa, sb)
        return "%d-%d" % (ia, ib)
