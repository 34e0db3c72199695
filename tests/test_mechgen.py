"""Mechanism table generator and the committed tables."""
import json
import os

import numpy as np
import pytest

from tiger_nga_b200 import mechgen
from tiger_nga_b200.mechanism import BUILTIN, composition, load

from oracle.f90_to_c import reference_combustion_dir  # noqa: E402

REF = reference_combustion_dir()

MINI_H = """
     integer, parameter ::   SN2 = 1, SH = 2 , SO2 = 3, SOH = 4 , SEND = 5
      integer, parameter ::   R1F = 1, R1B = 2 , R2F = 3, R2B = 4 , R3 = 5, REND = 6
     integer, parameter ::   MM1 = 1, MEND = 2
"""

MINI_F90 = """
subroutine PRODRATES( CDOT, W, K, C, M, TEMP, PRESSURE)
      implicit none
      include 'MINI.h'
      real(DP) :: CDOT(4), W(5), K(5), &
      C(4), M(1), TEMP, PRESSURE
      real(DP) :: GETLINDRATECOEFF, LT, RT
      real(DP), parameter ::  RGAS = 8314.34, CONCDEFAULT = -1.0
      real(DP) ::  KINFTROE, K0TROE
      real(DP) ::  FCTROE
      LT = DLOG( TEMP )
      RT = RGAS * TEMP
      M(MM1) = C(SN2) + 2.5 * C(SH) &
	    + C(SO2)
      M(MM1) = M(MM1) + 12 * C(SOH)
      K(R1F) = 2.0000000000D+13 &
	   * exp(-0.5 * LT - 1000 / RT)
      K(R1B) = 3.0000000000D+10 * exp(1.5 * LT + 2.5e3 / RT)
      K0TROE = 6.0000000000D+14 * exp(-1.4 * LT)
      KINFTROE = 5.0000000000D+09
      FCTROE = 0.5 * EXP( -TEMP / 94 ) &
	   + 0.5 * EXP( -5182 / TEMP )
      K(R2F) = GETLINDRATECOEFF( TEMP, PRESSURE, K0TROE, KINFTROE &
	   , FCTROE, M(mM1) )
      K0TROE = 1.0000000000D+15 * exp(-2000 / RT)
      KINFTROE = 1.0000000000D+10 * exp(-3000 / RT)
      K(R2B) = GETLINDRATECOEFF( TEMP, PRESSURE, K0TROE, KINFTROE &
	   , FCTROE, M(mM1) )
      K(R3) = 4.0000000000D+10
      W(R1F) = K(R1F) * C(SH) * C(SO2)
      W(R1B) = K(R1B) * C(SOH) * M(MM1)
      W(R2F) = K(R2F) * C(SH) * C(SO2)
      W(R2B) = K(R2B) * C(SOH)
      W(R3) = K(R3) * C(SH) * C(SH)
      CDOT(SN2) = 0.0_DP
      CDOT(SH) = - W(R1F) + W(R1B) &
	    - W(R2F) + W(R2B) - 2 * W(R3)
      CDOT(SO2) = - W(R1F) + W(R1B) - W(R2F) + W(R2B)
      CDOT(SOH) = W(R1F) - W(R1B) + W(R2F) - W(R2B)
      END

      DOUBLE PRECISION FUNCTION GETLINDRATECOEFF( TEMP, PRESSURE, &
	   K0, KINF, FC, CONCIN )
      IMPLICIT NONE
      INTEGER ITROE
      DOUBLE PRECISION TEMP, PRESSURE, K0, KINF, FC
      DOUBLE PRECISION R
      PARAMETER (R = 8314.34)
      DOUBLE PRECISION NTMP,CCOEFF,DCOEFF,LGKNULL
      DOUBLE PRECISION KL
      DOUBLE PRECISION F
      DOUBLE PRECISION CONC, CONCIN
      ITROE = 1
      IF (CONCIN.GT.0.0) THEN
        CONC = CONCIN
      ELSE
        CONC = PRESSURE / ( R * TEMP )
      END IF
      NTMP = 0.75 - 1.27 * DLOG10( FC )
      IF (ITROE.EQ.1) THEN
        CCOEFF = - 0.4 - 0.67 * DLOG10( FC )
        DCOEFF = 0.14
        K0 = K0 * CONC / MAX(KINF, 1.0D-60)
        LGKNULL = DLOG10( K0 )
        F=(LGKNULL+CCOEFF)/(NTMP-DCOEFF*(LGKNULL+CCOEFF))
        F = FC**(1.0 / ( F * F + 1.0 ))
        GETLINDRATECOEFF = KINF * F * K0 / ( 1.0 + K0 )
      ELSE
        GETLINDRATECOEFF = KINF
      END IF
      END

      SUBROUTINE GETMOLARMASS( MM )
      IMPLICIT NONE
      DOUBLE PRECISION MM(4)
      INCLUDE 'MINI.h'
      MM(SN2) =  2.80200000e+01
      MM(SH) =  1.00800000e+00
      MM(SO2) =  3.20000000e+01
      MM(SOH) =  1.70080000e+01
      END

      SUBROUTINE GETSPECIESNAMES( NAMES )
      IMPLICIT NONE
      CHARACTER *20 NAMES(4)
      INCLUDE 'MINI.h'
      NAMES(SN2)='N2                  '
      NAMES(SH)='H                   '
      NAMES(SO2)='O2                  '
      NAMES(SOH)='OH                  '
      END

      SUBROUTINE GETNREACTIONS( NREACTIONS )
      IMPLICIT NONE
      INTEGER NREACTIONS
      NREACTIONS = 5
      END

      SUBROUTINE GETMUCOEFF( MUCOEFF )
      implicit none
      include 'MINI.h'
      real(DP) :: MUCOEFF(4)
      MUCOEFF(SN2) =  1.0e-06
      MUCOEFF(SH) =  1.0e-06
      MUCOEFF(SO2) =  1.0e-06
      MUCOEFF(SOH) =  1.0e-06
      END

      SUBROUTINE GETKOVEREPS( KOVEREPS )
      implicit none
      include 'MINI.h'
      real(DP) :: KOVEREPS(4)
      KOVEREPS(SN2) =  1.0e-02
      KOVEREPS(SH) =  1.0e-02
      KOVEREPS(SO2) =  1.0e-02
      KOVEREPS(SOH) =  1.0e-02
      END

@THERMO@
"""


def _thermo_block():
    def one(sp, a1, a6):
        return (f"      H({sp}) =  2.0e+02_DP * ( &\n\t   T * (  {a1}_DP + T * (  1.0e-04_DP &\n"
                f"\t   + T * ( -1.0e-07_DP + T * (  1.0e-11_DP &\n\t   + T * ( -1.0e-15_DP ) ) ) ) ) {a6}_DP )\n"
                f"      CP({sp}) =  2.0e+02_DP * ( &\n\t    {a1}_DP + T * (  2.0e-04_DP &\n"
                f"\t   + T * ( -3.0e-07_DP + T * (  4.0e-11_DP &\n\t   + T * ( -5.0e-15_DP ) ) ) ) )\n")
    sps = ("SN2", "SH", "SO2", "SOH")
    return ("      SUBROUTINE COMPTHERMODATA( H, CP, T )\n      implicit none\n      include 'MINI.h'\n"
            "      real(DP) :: H(4), CP(4), T\n      IF (T.GT.1000.0_DP) THEN\n"
            + "".join(one(sp, "3.0e+00", "-9.0e+02") for sp in sps) + "      ELSE\n"
            + "".join(one(sp, "3.5e+00", "+9.0e+02") for sp in sps) + "      END IF\n      END\n")


def _mini(tmp_path):
    h = tmp_path / "MINI.h"
    f = tmp_path / "MINI.f90"
    h.write_text(MINI_H)
    f.write_text(MINI_F90.replace("@THERMO@", _thermo_block()))
    return str(f), str(h)


def test_literal_kinds():
    assert mechgen.literal_kind("2.6400000000D+13") == "f64"
    assert mechgen.literal_kind("2.96728765e+02_DP") == "f64"
    assert mechgen.literal_kind("-0.67") == "f32"
    assert mechgen.literal_kind("1e-30") == "f32"
    assert mechgen.literal_kind("71300000") == "int"
    assert mechgen.literal_value("8314.34") == 8314.33984375
    assert mechgen.literal_value("8314.34", "f64") == 8314.34
    assert mechgen.literal_value("2.6400000000D+13") == 2.64e13


def test_parser_on_handwritten_mechanism(tmp_path):
    f, h = _mini(tmp_path)
    tab = mechgen.parse_mechanism(f, h, "mini")
    assert tab["n_species"] == 4 and tab["n_slots"] == 5 and tab["n_thirdbody"] == 1
    assert tab["third_body"][0] == [[0, "1"], [1, "2.5"], [2, "1"], [3, "12"]]
    k = tab["k"]
    assert k[0]["A"] == "2.0000000000D+13" and k[0]["n"] == "-0.5" and k[0]["E"] == "-1000"
    assert k[1]["n"] == "1.5" and k[1]["E"] == "2.5e3"
    assert k[2]["type"] == "falloff" and k[2]["kinf"] == {"A": "5.0000000000D+09", "n": None, "E": None}
    assert k[2]["fc"] == [{"a": "0.5", "form": "T_over", "x": "94"}, {"a": "0.5", "form": "over_T", "x": "5182"}]
    assert k[3]["type"] == "falloff" and k[3]["fc"] == k[2]["fc"]  # Fc reused by the reverse slot
    assert k[4] == {"A": "4.0000000000D+10", "n": None, "E": None, "type": "arrhenius", "line": k[4]["line"]}
    assert tab["w"][1] == {"C": [3], "M": 0, "line": tab["w"][1]["line"]}
    assert tab["cdot"][0] == []
    assert tab["cdot"][1][-1] == [-1, "2", 4]
    assert tab["thermo"]["hi"][0]["a6"] == "-9.0e+02_DP" and tab["thermo"]["lo"][0]["a6"] == "9.0e+02_DP"


def test_parser_rejects_reused_k0(tmp_path):
    f, h = _mini(tmp_path)
    text = open(f).read().replace("      K0TROE = 1.0000000000D+15 * exp(-2000 / RT)\n", "")
    open(f, "w").write(text)
    with pytest.raises(ValueError, match="K0TROE"):
        mechgen.parse_mechanism(f, h, "mini")


@pytest.mark.parametrize("name", BUILTIN)
def test_committed_tables_consistent(name):
    m = load(name)
    m.check_composition()
    assert np.all(m.elem @ m.nu == 0.0)  # every slot conserves elements
    assert m.ns == len(m.species) == len(m.wmol)
    sizes = {"hydrogen": (9, 50, 5), "grimech30": (36, 422, 32), "dme39": (39, 350, 20)}[name]
    assert (m.ns, m.nslot, m.nm) == sizes
    assert composition("CH2*-CH2") == {"C": 1, "H": 2}


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not mounted")
@pytest.mark.parametrize("name", BUILTIN)
def test_tables_regenerate_identically(name):
    f90, h = mechgen.BUILTIN[name]
    tab = mechgen.parse_mechanism(os.path.join(REF, f90), os.path.join(REF, h), name)
    with open(os.path.join(os.path.dirname(mechgen.__file__), "mechanisms", name + ".json")) as fh:
        assert json.load(fh) == json.loads(json.dumps(tab))
