"""The implicit solver's generated tables (tiger_nga_b200/codegen.py: solver_tables).

The solver reads its per-slot, per-falloff, per-F_cent, per-third-body-set and per-species
records lane-parallel from shared memory: lane i reads record i. With 8-byte words in 16 bank
pairs, the 16 lanes of a half-warp hit distinct bank pairs exactly when the record stride (in
doubles) is odd. These tests pin the record strides and sizes against csrc/solver_layout.h, the
bank property, the slot order the kernels rely on, and that every record holds the mechanism's
values with zero padding.
"""
import math

import numpy as np
import pytest

from tiger_nga_b200 import codegen as cg
from tiger_nga_b200 import mechanism as M

MECHS = ["hydrogen", "grimech30", "dme39"]


def _half_warp_conflict_free(stride):
    return len({(stride * i) % 16 for i in range(16)}) == 16


@pytest.mark.parametrize("stride_name", ["SLOT_REC", "FO_REC", "FC_REC", "TH_STRIDE"])
def test_record_strides_are_conflict_free(stride_name):
    assert _half_warp_conflict_free(getattr(cg, stride_name))


@pytest.mark.parametrize("mech", MECHS)
def test_table_sizes_follow_the_record_strides(mech):
    t = cg.solver_tables(mech)
    sz, hd = t["sizes"], t["hd"]
    ns, nslot, nfo, nfc, nm = sz["ns"], sz["nslot"], sz["nfo"], sz["nfc"], sz["nm"]
    for lm in (0, 1):
        assert len(hd["slot"][lm]) == cg.SLOT_REC * (nslot - nfo)
        assert len(hd["fo"][lm]) == cg.FO_REC * nfo
        assert len(hd["fc"][lm]) == cg.FC_REC * nfc
        assert len(hd["eff"][lm]) == max(nm, 1) * (ns | 1)
        assert len(hd["th"][lm]) == cg.TH_STRIDE * ns
    assert _half_warp_conflict_free(ns | 1)  # efficiency rows


@pytest.mark.parametrize("mech", MECHS)
def test_records_hold_the_mechanism_values(mech):
    t = cg.solver_tables(mech)
    m = M.load(mech, "f64")  # index 1 of each table holds the f64-literal values
    hd, sz, order = t["hd"], t["sizes"], t["order"]
    ns, nfo = sz["ns"], sz["nfo"]
    th = np.array(hd["th"][1]).reshape(ns, cg.TH_STRIDE)
    assert np.array_equal(th[:, :12], np.asarray(m.th_hi, dtype=float))
    assert np.array_equal(th[:, 12:24], np.asarray(m.th_lo, dtype=float))
    assert not th[:, 24:].any()
    eff = np.array(hd["eff"][1]).reshape(-1, ns | 1)
    assert not eff[:, ns:].any()
    # slot order: falloff slots first, then Arrhenius, then constants
    def kind(s):
        if s.kind == "falloff":
            return 0
        return 2 if (s.arr.n is None and s.arr.E is None) else 1
    kinds = [kind(m.slots[r]) for r in order]
    assert kinds == sorted(kinds) and kinds.count(0) == nfo
    # plain records: (ln A, E, n) for Arrhenius slots, (A, 0, 0) for constant slots
    rec = np.array(hd["slot"][1]).reshape(-1, cg.SLOT_REC)
    for p, r in enumerate(order[nfo:]):
        a = m.slots[r].arr
        if kind(m.slots[r]) == 2:
            assert rec[p, 0] == a.A and rec[p, 1] == 0.0 and rec[p, 2] == 0.0
        else:
            assert rec[p, 0] == math.log(a.A)
            assert rec[p, 1] == (a.E or 0.0) and rec[p, 2] == (a.n or 0.0)
    fo = np.array(hd["fo"][1]).reshape(-1, cg.FO_REC)
    assert not fo[:, 6:].any()
    fc = np.array(hd["fc"][1]).reshape(-1, cg.FC_REC)
    assert not fc[:, 6:].any()
