"""Recipe: build the reference's own mechanism arithmetic, run here, into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports, links or runs this file or its
outputs; only tests, the smoke check and the CPU-baseline leg of the benchmark may.

The reference's chemistry rates live in three self-contained generated Fortran files
(combustion/HYDROGENF.f90, combustion/grimech30F.f90, combustion/DME39F.f90, each with its
``*F90.h`` parameter header). No Fortran compiler exists in this image, so this recipe
transliterates the routines on the path -- ``PRODRATES``, ``GETLINDRATECOEFF``,
``COMPTHERMODATA``, ``GETMOLARMASS`` and the transport fits ``GETMUCOEFF`` / ``GETKOVEREPS`` --
statement by statement into C, keeping:

* the statement order and each expression's operator order (C and Fortran both associate
  ``+ - * /`` left to right; the C file is compiled with ``-ffp-contract=off`` so no FMA is
  introduced, matching the reference's ``-xAVX`` target, which has no FMA);
* the Fortran literal kinds of the reference build (Makefile.in:23-24, no default-real
  promotion): ``D`` exponents and ``_DP`` suffixes stay double, default-real literals become
  C ``float`` literals that are widened on use, integer literals are exact;
* the by-reference argument passing (``GETLINDRATECOEFF`` overwrites its ``K0`` argument).

The same recipe compiles the reference's own C file library (library/fileio_c.c, unchanged,
into ``oracle/_ref/libref_fileio.so``): the writer and reader behind its data files
(tools/init_flow/param.f90:113-148), used to pin the library's data-file reader and writer.

The transliteration is mechanical and shares no code with the product's table generator, so
it pins that generator and the table-driven oracle independently. Outputs (C sources and the
shared library) go to ``oracle/_ref/`` only; they are git-ignored and are rebuilt from the
reference tree by ``python oracle/f90_to_c.py <reference combustion dir>``.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

MECHS = {
    "hydrogen": ("HYDROGENF.f90", "HYDROGENF90.h"),
    "grimech30": ("grimech30F.f90", "grimech30F90.h"),
    "dme39": ("DME39F.f90", "DME39F90.h"),
}
ROUTINES = ("PRODRATES", "GETLINDRATECOEFF", "COMPTHERMODATA", "GETMOLARMASS", "GETMUCOEFF", "GETKOVEREPS")
INTRINSICS = {"EXP": "exp", "DLOG": "log", "DLOG10": "log10", "MAX": "fmax", "DSQRT": "sqrt", "LOG": "log"}


def statements(path):
    stmts, cur = [], ""
    for raw in open(path, errors="replace"):
        line = raw.rstrip("\n")
        cut = []
        quote = None
        for ch in line:
            if quote:
                cut.append(ch)
                quote = None if ch == quote else quote
            elif ch in "'\"":
                quote = ch
                cut.append(ch)
            elif ch == "!":
                break
            else:
                cut.append(ch)
        s = "".join(cut).rstrip()
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        cur += s
        if cur.strip():
            stmts.append(" ".join(cur.split()))
        cur = ""
    return stmts


def header_params(path):
    out = []
    for st in statements(path):
        if re.match(r"(?i)integer\s*,\s*parameter", st):
            for item in st.split("::", 1)[1].split(","):
                if "=" in item:
                    n, v = (x.strip() for x in item.split("="))
                    if re.fullmatch(r"\d+", v):
                        out.append((n.upper(), int(v)))
    return out


TOK = re.compile(r"\s*((?:\d+\.\d*|\.\d+|\d+)(?:[eEdD][+-]?\d+)?(?:_DP)?|\.[A-Za-z]+\.|[A-Za-z_]\w*|\*\*|'[^']*'|\S)")


def tokens(s):
    pos, out = 0, []
    while pos < len(s):
        m = TOK.match(s, pos)
        if not m:
            break
        out.append(m.group(1))
        pos = m.end()
    return out


def c_literal(t):
    """Fortran numeric literal -> C literal of the same kind and value."""
    if t.upper().endswith("_DP"):
        return t[:-3]
    if re.search(r"[dD]", t):
        return t.replace("D", "E").replace("d", "e")
    if "." in t or "e" in t.lower():
        return t + "f"  # default real: float32, widened to double where it meets a double
    return t + ".0"  # integer literal: exact (no integer/integer division occurs in these files)


class Routine:
    def __init__(self, name, args, body, is_func):
        self.name, self.args, self.body, self.is_func = name, args, body, is_func
        self.arrays, self.locals, self.consts = set(), [], []


def split_routines(stmts):
    out = {}
    cur = None
    for st in stmts:
        u = st.upper()
        m = re.match(r"(DOUBLE PRECISION\s+FUNCTION|SUBROUTINE)\s+(\w+)\s*\(([^)]*)\)", u)
        if m and cur is None:
            args = [a.strip() for a in m.group(3).split(",") if a.strip()]
            cur = Routine(m.group(2), args, [], m.group(1) != "SUBROUTINE")
            continue
        if cur is not None:
            if u == "END":
                out[cur.name] = cur
                cur = None
            else:
                cur.body.append(st)
    return out


def translate_expr(toks, r, mech):
    """Token list -> C expression string for routine r."""
    out = []
    i = 0
    while i < len(toks):
        t = toks[i]
        u = t.upper()
        nxt = toks[i + 1] if i + 1 < len(toks) else None
        if re.match(r"^(\d|\.\d)", t):
            out.append(c_literal(t))
        elif u in (".GT.", ".LT.", ".GE.", ".LE.", ".EQ.", ".NE."):
            out.append({".GT.": ">", ".LT.": "<", ".GE.": ">=", ".LE.": "<=", ".EQ.": "==", ".NE.": "!="}[u])
        elif re.match(r"[A-Za-z_]", t):
            if nxt == "(" and u in INTRINSICS:
                out.append(INTRINSICS[u])
            elif nxt == "(" and u == "GETLINDRATECOEFF":
                # by-reference call: collect the argument groups
                depth, j, args, cur = 0, i + 1, [], []
                while True:
                    tk = toks[j]
                    if tk == "(":
                        depth += 1
                        if depth > 1:
                            cur.append(tk)
                    elif tk == ")":
                        depth -= 1
                        if depth == 0:
                            args.append(cur)
                            break
                        cur.append(tk)
                    elif tk == "," and depth == 1:
                        args.append(cur)
                        cur = []
                    else:
                        cur.append(tk)
                    j += 1
                cargs = []
                for a in args:
                    ca = translate_expr(a, r, mech)
                    if len(a) == 1 and a[0].upper() in r.args:
                        cargs.append("p_" + a[0].upper())
                    else:
                        cargs.append("&" + ca)
                out.append(f"ref_{mech}_getlindratecoeff(" + ", ".join(cargs) + ")")
                i = j + 1
                continue
            elif u in r.args and nxt == "(":
                # array dummy: A(i) -> p_A[(i)-1]
                depth, j, inner = 0, i + 1, []
                while True:
                    tk = toks[j]
                    if tk == "(":
                        depth += 1
                        if depth > 1:
                            inner.append(tk)
                    elif tk == ")":
                        depth -= 1
                        if depth == 0:
                            break
                        inner.append(tk)
                    else:
                        inner.append(tk)
                    j += 1
                out.append(f"p_{u}[({translate_expr(inner, r, mech)})-1]")
                i = j + 1
                continue
            elif u in r.args:
                out.append(f"(*p_{u})")
            elif u == r.name and r.is_func:
                out.append("result")
            else:
                out.append(u)
        elif t == "**":
            # base ** (group): rewrite the previous operand and the following group as pow()
            base = out.pop()
            depth, j, inner = 0, i + 1, []
            assert toks[j] == "(", "exponent must be parenthesised"
            while True:
                tk = toks[j]
                if tk == "(":
                    depth += 1
                elif tk == ")":
                    depth -= 1
                inner.append(tk)
                if depth == 0:
                    break
                j += 1
            out.append(f"pow({base}, {translate_expr(inner, r, mech)})")
            i = j + 1
            continue
        else:
            out.append(t)
        i += 1
    return " ".join(out)


def translate_routine(r, mech):
    lines = []
    decl = []
    body = []
    pnames = set()
    for st in r.body:
        m = re.match(r"^PARAMETER\s*\((\w+)\s*=", st.upper())
        if m:
            pnames.add(m.group(1))
    for st in r.body:
        u = st.upper()
        if re.match(r"^(IMPLICIT|INCLUDE)\b", u):
            continue
        m = re.match(r"^(REAL\(DP\)|DOUBLE PRECISION|INTEGER|CHARACTER[^:]*)\s*(,\s*PARAMETER)?\s*(::)?\s*(.*)$", u)
        if m and not re.match(r"^(REAL|DOUBLE|INTEGER)\w*\s*=", u):
            ctype = "int" if m.group(1).startswith("INTEGER") else "double"
            items = re.split(r",(?![^(]*\))", m.group(4))
            for it in items:
                it = it.strip()
                if not it:
                    continue
                if "=" in it:
                    n, v = (x.strip() for x in it.split("=", 1))
                    decl.append(f"  const {ctype} {n} = {translate_expr(tokens(v), r, mech)};")
                    continue
                n = re.match(r"(\w+)", it).group(1)
                if n in r.args or n == r.name or n in pnames:
                    continue
                decl.append(f"  {ctype} {n};")
            continue
        m = re.match(r"^PARAMETER\s*\((\w+)\s*=\s*(.*)\)$", u)
        if m:
            decl.append(f"  const double {m.group(1)} = {translate_expr(tokens(m.group(2)), r, mech)};")
            continue
        m = re.match(r"^IF\s*\((.*)\)\s*THEN$", st, re.I)
        if m:
            body.append(f"  if ({translate_expr(tokens(m.group(1)), r, mech)}) {{")
            continue
        if u == "ELSE":
            body.append("  } else {")
            continue
        if u in ("END IF", "ENDIF"):
            body.append("  }")
            continue
        if "=" in st:
            toks = tokens(st)
            depth = 0
            for k, t in enumerate(toks):
                depth += t == "("
                depth -= t == ")"
                if t == "=" and depth == 0:
                    break
            lhs = translate_expr(toks[:k], r, mech)
            rhs = translate_expr(toks[k + 1:], r, mech)
            body.append(f"  {lhs} = {rhs};")
            continue
        raise ValueError(f"untranslated statement in {r.name}: {st}")
    cname = f"ref_{mech}_{r.name.lower()}"
    params = ", ".join(f"double *p_{a}" for a in r.args)
    if r.is_func:
        lines.append(f"double {cname}({params}) {{")
        lines.append("  double result;")
    else:
        lines.append(f"void {cname}({params}) {{")
    lines += decl + body
    if r.is_func:
        lines.append("  return result;")
    lines.append("}")
    return "\n".join(lines)


def transliterate(src_dir, mech):
    f90, h = MECHS[mech]
    params = header_params(os.path.join(src_dir, h))
    routines = split_routines(statements(os.path.join(src_dir, f90)))
    out = [f"/* Generated by oracle/f90_to_c.py from combustion/{f90} (+ {h}). Not committed. */",
           "#include <math.h>", f"enum {{"]
    out += [f"  {n} = {v}," for n, v in params]
    out.append("};")
    out.append(f"double ref_{mech}_getlindratecoeff(double*, double*, double*, double*, double*, double*);")
    for name in ROUTINES:
        out.append(translate_routine(routines[name], mech))
    nspec = dict(params)["SEND"] - 1
    nslot = dict(params)["REND"] - 1
    nm = dict(params)["MEND"] - 1
    out.append(f"int ref_{mech}_sizes(int *ns, int *nr, int *nm) {{ *ns = {nspec}; *nr = {nslot}; *nm = {nm}; return 0; }}")
    # finitechem_compute_rhs (finitechem.f90:93-175, low-Mach branch) over a species-major batch,
    # OpenMP over cells like one MPI rank per core; the mechanism routines are the transliterated ones.
    out.append(f"""
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif
void ref_{mech}_rhs_batch(const double *sol, double p, double *rhs, int64_t ncells, int64_t ld, int nthreads) {{
  double W_sp[{nspec}];
  ref_{mech}_getmolarmass(W_sp);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < ncells; ++i) {{
    double s[{nspec + 1}], h[{nspec}], cp[{nspec}], conc[{nspec}], cd[{nspec}], K[{nslot}], W[{nslot}], M[{max(nm, 1)}];
    for (int v = 0; v <= {nspec}; ++v) s[v] = sol[v * ld + i];
    double rho = 0.0;
    for (int k = 0; k < {nspec}; ++k) rho = rho + s[k];
    double T = s[{nspec}] / rho, P = p;
    ref_{mech}_compthermodata(h, cp, &T);
    double cpmix = 0.0;
    for (int k = 0; k < {nspec}; ++k) cpmix = cpmix + (s[k] / rho) * cp[k];
    for (int k = 0; k < {nspec}; ++k) conc[k] = s[k] / W_sp[k];
    ref_{mech}_prodrates(cd, W, K, conc, M, &T, &P);
    double tmp = 0.0;
    for (int k = 0; k < {nspec}; ++k) {{
      double r = cd[k] * W_sp[k];
      rhs[k * ld + i] = r;
      tmp = tmp - h[k] * r;
    }}
    rhs[{nspec} * ld + i] = tmp / cpmix;
  }}
}}
""")
    # finitechem_W + finitechem_density (finitechem.f90:65-74, :324-345), finitechem_viscosity
    # (:351-406), finitechem_diffusivity (:412-461) with finitechem_omegamu (:467-487) and
    # finitechem_Cp (:79-88), per cell in the reference's statement order over the transliterated
    # getters and COMPTHERMODATA (called inside the species loop, as :428-432 does); Fortran's
    # x**-0.5 / **0.5 / **0.25 are pow calls and (..)**2 a product.
    out.append(f"""
static double ref_{mech}_omegamu(double temp) {{
  const double m1 = 3.3530622607, m2 = 2.53272006, m3 = 2.9024238575, m4 = 0.11186138893, m5 = 0.8662326188;
  const double m6 = 1.3913958626, m7 = 3.158490576, m8 = 0.18973411754, m9 = 0.00018682962894;
  double num = m1 + temp * (m2 + temp * (m3 + temp * m4));
  double den = m5 + temp * (m6 + temp * (m7 + temp * (m8 + temp * m9)));
  return num / den;
}}
static double ref_{mech}_w(const double *sc, double *W_sp) {{
  double a = 0.0, b = 0.0;
  for (int k = 0; k < {nspec}; ++k) {{
    double t = fmin(fmax(sc[k], 0.0), 1.0);
    a = a + t;
  }}
  for (int k = 0; k < {nspec}; ++k) {{
    double t = fmin(fmax(sc[k], 0.0), 1.0);
    b = b + t / W_sp[k];
  }}
  return a / b;
}}
void ref_{mech}_props_batch(const double *y, const double *Tin, int64_t ncells, int64_t ld, double P_thermo,
                            const double *lewis, double *wmix, double *rho, double *visc, double *diff, int nthreads) {{
  const double R_cst = 8314.34, Tmin = 50.0, Tmax = 5000.0;
  double W_sp[{nspec}], mucoeff[{nspec}], kOverEps[{nspec}];
  ref_{mech}_getmolarmass(W_sp);
  ref_{mech}_getmucoeff(mucoeff);
  ref_{mech}_getkovereps(kOverEps);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t c = 0; c < ncells; ++c) {{
    double sc[{nspec}], eta[{nspec}], cond[{nspec}], h_sp[{nspec}], Cp_sp[{nspec}];
    double phi[{nspec}][{nspec}];
    for (int k = 0; k < {nspec}; ++k) sc[k] = y[k * ld + c];
    const double T = Tin[c];
    const double W_mix = ref_{mech}_w(sc, W_sp);
    if (wmix) wmix[c] = W_mix;
    if (rho) rho[c] = P_thermo * W_mix / (R_cst * T);
    double temp = fmin(fmax(T, Tmin), Tmax);
    if (visc) {{
      for (int n = 0; n < {nspec}; ++n) {{
        double om = ref_{mech}_omegamu(temp * kOverEps[n]);
        eta[n] = mucoeff[n] * sqrt(temp) / om;
      }}
      for (int k = 0; k < {nspec}; ++k)
        for (int j = 0; j < {nspec}; ++j) {{
          phi[k][j] = (1.0 / sqrt(8.0)) * pow(1.0 + (W_sp[k] / W_sp[j]), -0.5);
          double temp1 = pow(eta[k] / eta[j], 0.5) * pow(W_sp[j] / W_sp[k], 0.25);
          phi[k][j] = phi[k][j] * ((1.0 + temp1) * (1.0 + temp1));
        }}
      double sum_2 = 0.0;
      for (int k = 0; k < {nspec}; ++k) {{
        double sum_1 = 0.0;
        for (int j = 0; j < {nspec}; ++j)
          if (j != k) sum_1 = sum_1 + (sc[j] * W_mix * phi[k][j] / W_sp[j]);
        sum_1 = sum_1 + sc[k] * W_mix / W_sp[k];
        if (sc[k] > 0.0) sum_2 = sum_2 + (sc[k] * W_mix * eta[k] / (W_sp[k] * sum_1));
      }}
      visc[c] = sum_2;
    }}
    if (diff) {{
      for (int n = 0; n < {nspec}; ++n) {{
        double om = ref_{mech}_omegamu(temp * kOverEps[n]);
        eta[n] = mucoeff[n] * sqrt(temp) / om;
        ref_{mech}_compthermodata(h_sp, Cp_sp, &temp);
        cond[n] = eta[n] * (Cp_sp[n] + 1.25 * R_cst / W_sp[n]);
      }}
      double sum_1 = 0.0, sum_2 = 0.0;
      for (int n = 0; n < {nspec}; ++n) {{
        sum_1 = sum_1 + (sc[n] * W_mix / (cond[n] * W_sp[n]));
        sum_2 = sum_2 + (sc[n] * cond[n] * W_mix / W_sp[n]);
      }}
      double lambda = 0.5 * (sum_2 + (1.0 / sum_1));
      ref_{mech}_compthermodata(h_sp, Cp_sp, &temp);
      double Cp_mix = 0.0;
      for (int n = 0; n < {nspec}; ++n) Cp_mix = Cp_mix + sc[n] * Cp_sp[n];
      for (int n = 0; n < {nspec}; ++n) diff[n * ld + c] = (lambda / Cp_mix) / (lewis ? lewis[n] : 1.0);
      diff[{nspec} * ld + c] = lambda / Cp_mix;
    }}
  }}
}}
""")
    # the variable names (SN2, R1F, ...) collide between mechanisms, so each goes to its own file
    return "\n".join(out) + "\n"


def build_fileio(src_dir, out_dir=OUT, cc="gcc"):
    """The reference's own binary file library (library/fileio_c.c, C, compiled unchanged from
    where it lies) into oracle/_ref/libref_fileio.so: the writer and reader of its data files."""
    lib_src = os.path.join(os.path.dirname(os.path.abspath(src_dir)), "library", "fileio_c.c")
    so = os.path.join(out_dir, "libref_fileio.so")
    if os.path.exists(lib_src):
        subprocess.check_call([cc, "-O2", "-fPIC", "-shared", "-o", so, lib_src])
    return so


def build(src_dir, out_dir=OUT, cc="gcc"):
    os.makedirs(out_dir, exist_ok=True)
    build_fileio(src_dir, out_dir, cc)
    cfiles = []
    for mech in MECHS:
        path = os.path.join(out_dir, f"ref_{mech}.c")
        with open(path, "w") as fh:
            fh.write(transliterate(src_dir, mech))
        cfiles.append(path)
    so = os.path.join(out_dir, "libref_mech.so")
    cmd = [cc, "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-o", so] + cfiles + ["-lm"]
    subprocess.check_call(cmd)
    return so


def reference_combustion_dir() -> str:
    """The reference's ``combustion/`` directory that this recipe reads: under the project root
    named by the environment variable TNG_REFERENCE_DIR, else under the read-only mount of the
    reference project in the build container. The directory may be absent (e.g. on a GPU host);
    callers check for it."""
    return os.path.join(os.environ.get("TNG_REFERENCE_DIR", "/root/reference"), "combustion")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else reference_combustion_dir()
    print(build(src))
