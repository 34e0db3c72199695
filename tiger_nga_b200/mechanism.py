"""Mechanism tables as the product sees them.

A mechanism is data (one JSON table per mechanism, generated from the reference's Fortran by
:mod:`tiger_nga_b200.mechgen`) instead of a linked ``PRODRATES`` symbol
(combustion/mechanism.f90:17-108 is the reference's link-time template). This module turns
the table into numbers under a literal mode:

* ``'f32'`` -- the reference build: default-real literals rounded to float32 and widened
  (Makefile.in:23-24 carries no default-real promotion flag);
* ``'f64'`` -- every literal read as a double.

It also derives what the kernels need beyond the reference's own arrays: net stoichiometric
coefficients per (species, slot), and the element composition of every species, parsed from
its name and checked against the mechanism's molar mass (GETMOLARMASS, e.g.
combustion/grimech30F.f90 getter block) -- used by the conservation projection.
"""
from __future__ import annotations

import json
import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

from .mechgen import literal_value

MECH_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mechanisms")
BUILTIN = ("hydrogen", "grimech30", "dme39")

# Aliases used in the DME39 species list (combustion/DME39F.f90:18-23) and the GRI subset.
_ALIASES = {
    "CH2X": "CH2",
    "RO2": "CH3OCH2O2",
    "ROH": "CH3OCH2OH",
    "QOOH": "CH2OCH2O2H",
    "O2QOOH": "O2CH2OCH2O2H",
    "HO2QHO": "HO2CH2OCHO",
}
ELEMENTS = ("C", "H", "O", "N", "AR")
_ATOMIC = {"C": 12.011, "H": 1.008, "O": 16.0, "N": 14.01, "AR": 39.948}


def composition(name: str) -> dict[str, int]:
    """Element counts from a species name such as ``CH3OCH2O2`` or ``CH2*-CH2``."""
    base = _ALIASES.get(name, name)
    base = base.split("*")[0]
    if base == "AR":
        return {"AR": 1}
    out: dict[str, int] = {}
    for el, cnt in re.findall(r"(AR|C|H|O|N)(\d*)", base):
        out[el] = out.get(el, 0) + (int(cnt) if cnt else 1)
    if "".join(f"{e}{c}" for e, c in re.findall(r"(AR|C|H|O|N)(\d*)", base)) != base:
        raise ValueError(f"cannot parse species formula {name!r}")
    return out


@dataclass
class Arrh:
    """``A*exp(n*LT + E/RT)`` with signs folded into n and E (E here is the signed numerator)."""

    A: float
    n: float | None
    E: float | None


@dataclass
class Slot:
    index: int
    name: str
    kind: str  # 'arrhenius' | 'falloff'
    arr: Arrh | None = None
    k0: Arrh | None = None
    kinf: Arrh | None = None
    fc: list = field(default_factory=list)  # [(a, form, x)], form 0: exp(-T/x), 1: exp(-x/T)
    fc_key: tuple = ()
    M_fall: int = -1
    C: list = field(default_factory=list)  # reactant species (with multiplicity)
    M: int = -1  # third-body set multiplying W, or -1
    reverse: bool = False  # a fitted reverse-rate slot (name ends with B)


class Mechanism:
    def __init__(self, name: str, literal_mode: str = "f32", path: str | None = None):
        if literal_mode not in ("f32", "f64"):
            raise ValueError("literal_mode must be 'f32' or 'f64'")
        self.name = name
        self.literal_mode = literal_mode
        path = path or os.path.join(MECH_DIR, name + ".json")
        with open(path) as fh:
            tab = json.load(fh)
        if tab.get("format") != "tiger-chem-mechanism/1":
            raise ValueError(f"{path}: not a mechanism table")
        self.table = tab
        L = self.lit
        self.ns = tab["n_species"]
        self.nslot = tab["n_slots"]
        self.nm = tab["n_thirdbody"]
        self.species = list(tab["species"])
        self.wmol = np.array([L(x) for x in tab["molar_mass"]])
        # transport fits (GETMUCOEFF / GETKOVEREPS, e.g. HYDROGENF.f90:453-497)
        self.mucoeff = np.array([L(x) for x in tab["mucoeff"]])
        self.koveps = np.array([L(x) for x in tab["koveps"]])
        self.rgas = L(tab["rgas"])
        self.tmid = L(tab["thermo"]["tmid"])
        self.third_body = [[(s, L(c)) for s, c in terms] for terms in tab["third_body"]]

        def arrh(d):
            return Arrh(L(d["A"]), L(d["n"]) if d["n"] is not None else None, L(d["E"]) if d["E"] is not None else None)

        self.slots: list[Slot] = []
        for i, (k, w) in enumerate(zip(tab["k"], tab["w"])):
            nm = tab["slot_names"][i]
            s = Slot(index=i, name=nm, kind=k["type"], C=list(w["C"]), M=w["M"], reverse=nm.endswith("B"))
            if k["type"] == "falloff":
                s.k0, s.kinf = arrh(k["k0"]), arrh(k["kinf"])
                s.fc = [(L(t["a"]), 0 if t["form"] == "T_over" else 1, L(t["x"])) for t in k["fc"]]
                s.fc_key = tuple(s.fc)
                s.M_fall = k["M"]
            else:
                s.arr = arrh(k)
            self.slots.append(s)

        # net stoichiometry nu[k][r] from the ordered CDOT term lists
        nu = np.zeros((self.ns, self.nslot))
        for k, terms in enumerate(tab["cdot"]):
            for sgn, c, r in terms:
                nu[k, r] += sgn * L(c)
        self.nu = nu

        def thermo(rng):
            out = np.zeros((self.ns, 12))
            for k, e in enumerate(tab["thermo"][rng]):
                out[k] = [L(e["c0"])] + [L(a) for a in e["a"]] + [L(e["a6"])] + [L(b) for b in e["b"]]
            return out

        self.th_hi = thermo("hi")
        self.th_lo = thermo("lo")
        self.troe = {k: L(v) for k, v in (("c_n0", "0.75"), ("c_n1", "1.27"), ("c_c0", "0.4"), ("c_c1", "0.67"),
                                          ("c_d", "0.14"), ("kmin", "1.0D-60"), ("one", "1.0"))}
        comp = [composition(s) for s in self.species]
        self.elements = [e for e in ELEMENTS if any(e in c for c in comp)]
        self.elem = np.array([[c.get(e, 0) for c in comp] for e in self.elements], dtype=np.float64)

    def lit(self, text: str) -> float:
        return literal_value(text, self.literal_mode)

    def check_composition(self, rel: float = 2e-3) -> None:
        """Element composition parsed from names must reproduce the molar masses."""
        for k, s in enumerate(self.species):
            w = sum(_ATOMIC[e] * n for e, n in composition(s).items())
            if abs(w - self.wmol[k]) > rel * self.wmol[k]:
                raise ValueError(f"{self.name}: {s} composition mass {w} != W {self.wmol[k]}")

    def slot_ln_range(self) -> float:
        return max(abs(math.log(s.arr.A)) for s in self.slots if s.arr is not None and s.arr.A > 0)


def load(name: str, literal_mode: str = "f32") -> Mechanism:
    return Mechanism(name, literal_mode)
