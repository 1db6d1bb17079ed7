"""Generates the committed golden fixtures of the test suite.

1. coefficients.json -- constants read as TEXT from the reference's Fortran
   sources (no Fortran compiler exists here, so the reference cannot be run):
     * the RK4(3)5[2R+]C coefficients ACOFRK/BCOFRK/BHATRK(1..5), the
       non-comment assignments of src/dtinit.f:78-94, as exact rationals;
     * every derivative coefficient assigned in src/dfinit.f (interior
       10th-order first/second/mixed schemes and the one-sided closures),
       evaluated from the source expressions in order.
   The oracle's own constants are checked against these (test_oracle_kat).
2. oracle_<case>.npz -- small seeded states (fields, T, ITNDEX) with the
   oracle's right-hand side and its state after two RK steps: a regression
   pin of the oracle, and a GPU parity fixture that needs no oracle at run
   time.

Run from the repository root:
  python tests/golden/make_golden.py <reference_root>
(or with SENGA_REFERENCE_ROOT set; it reads the reference's Fortran sources
under <reference_root>/src. The GPU box never runs this script.)
"""
import json
import os
import re
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SENGA_REFERENCE_ROOT", ""), "src")
sys.path.insert(0, os.path.join(ROOT, "senga-versiona_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _code_lines(path):
    """Non-comment statement lines of a fixed-form Fortran file."""
    out = []
    with open(path) as f:
        for no, line in enumerate(f, 1):
            if not line.strip() or line[0] in "Cc*!":
                continue
            out.append((no, line.rstrip("\n")))
    return out


def _dexp(tok):
    mant, exp = tok.upper().split("D")
    return Fraction(mant) * Fraction(10) ** int(exp)


def rk_coefficients():
    pat = re.compile(r"^\s+(ACOFRK|BCOFRK|BHATRK)\((\d)\)\s*=\s*(.+?)\s*$")
    got = {}
    for no, line in _code_lines(os.path.join(REF, "dtinit.f")):
        m = pat.match(line)
        if not m:
            continue
        name, i, expr = m.group(1), int(m.group(2)), m.group(3)
        if expr.upper() == "ZERO":
            val = Fraction(0)
        else:
            num, den = expr.split("/")
            val = _dexp(num) / _dexp(den)
        got[f"{name}({i})"] = {"num": val.numerator, "den": val.denominator, "value": float(val),
                               "line": f"src/dtinit.f:{no}"}
    return got


_TOK = re.compile(r"\s*(?:(\d+\.\d*D[+-]?\d+|\d+\.\d*|\d+)|([A-Z][A-Z0-9]*)|(.))")


def _eval(expr, env):
    """Evaluates +,-,*,/ and parentheses over Fortran literals and names."""
    toks = []
    for num, name, op in _TOK.findall(expr.upper()):
        if num:
            toks.append(("n", _dexp(num) if "D" in num else Fraction(num)))
        elif name:
            if name not in env:
                raise KeyError(name)
            toks.append(("n", env[name]))
        elif op.strip():
            toks.append(("o", op))
    pos = 0

    def atom():
        nonlocal pos
        kind, v = toks[pos]
        if kind == "o" and v == "(":
            pos += 1
            r = add()
            pos += 1  # ')'
            return r
        if kind == "o" and v == "-":
            pos += 1
            return -atom()
        pos += 1
        return v

    def mul():
        nonlocal pos
        r = atom()
        while pos < len(toks) and toks[pos] in (("o", "*"), ("o", "/")):
            op = toks[pos][1]
            pos += 1
            r = r * atom() if op == "*" else r / atom()
        return r

    def add():
        nonlocal pos
        r = mul()
        while pos < len(toks) and toks[pos] in (("o", "+"), ("o", "-")):
            op = toks[pos][1]
            pos += 1
            r = r + mul() if op == "+" else r - mul()
        return r

    return add()


def fd_coefficients():
    pat = re.compile(r"^\s+([A-Z][A-Z0-9]*)\s*=\s*(.+?)\s*$")
    env = {"ONE": Fraction(1), "ZERO": Fraction(0)}
    src = {}
    for no, line in _code_lines(os.path.join(REF, "dfinit.f")):
        m = pat.match(line)
        if not m:
            continue
        try:
            env[m.group(1)] = _eval(m.group(2), env)
            src[m.group(1)] = f"src/dfinit.f:{no}"
        except (KeyError, IndexError, ValueError, ZeroDivisionError):
            continue
    return {k: {"value": float(v), "line": src[k]} for k, v in env.items() if k in src}


CASES = {
    # name: (make_case name, shape (nx, ny, nz), seed)
    "h2_mavt": ("h2_kernels", (12, 10, 8), 41),
    "onestep": ("ignition32", (12, 10, 8), 42),
}


def oracle_fixtures():
    import cases
    from oracle import Oracle

    for key, (name, (nx, ny, nz), seed) in CASES.items():
        c = cases.make_case(name, n=12, seed=seed)
        # non-cubic crop of the seeded state: keeps the fixture small and
        # exercises nx != ny != nz (periodic wrap on the crop)
        f = np.ascontiguousarray(c["fields"][:, :nz, :ny, :nx])
        t = np.ascontiguousarray(c["T"][:nz, :ny, :nx])
        itn = np.ascontiguousarray(c["itn"][:nz, :ny, :nx])
        lengths = (c["lengths"][0] * (nx - 1) / 11, c["lengths"][1] * (ny - 1) / 11, c["lengths"][2] * (nz - 1) / 11)
        o = Oracle((nx, ny, nz), lengths, c["chem"], c["diff"], c["dt"])
        o.upload(f, t, itn)
        rhs, trhs, prhs = o.rhs()
        o.upload(f, t, itn)
        o.step(2)
        f2, t2, itn2 = o.download()
        np.savez_compressed(os.path.join(HERE, f"oracle_{key}.npz"), shape=np.array([nx, ny, nz]),
                            lengths=np.array(lengths), dt=np.array(c["dt"]), fields=f, T=t, itn=itn, rhs=rhs,
                            T_rhs=trhs, p_rhs=prhs, fields_2=f2, T_2=t2, itn_2=itn2,
                            chem=np.array(os.path.basename(c["chem"])),
                            diff=np.array(os.path.basename(c["diff"]) if c["diff"] else ""))
        print("wrote", key)


def casefile_dump():
    """The reference's formatted restart inputs: its 1-step case
    (src/casefiles/1step/dmpi0000000.dat, 1001 x 1 x 1 points, 2 species),
    copied as a parser fixture, and its 21-step H2/air case
    (src/casefiles/21step/dmpi0000000.dat, the same grid, 9 species: a
    freely propagating 1D flame that the case restarts from with inflow at
    2.05 m/s, NSCBC I3/O1 x faces and every transport switch on), and the
    1-step and 4-step cases' mechanisms (with the 4-step restart state), and
    the 25-step and 68-step methane cases' mechanisms and restart states
    (16 and 18 species: the reference compiles these with NSPCMX = 16/18,
    NSTPMX = 35/68, src/casefiles/{25,68}step/com_senga2.h)."""
    import shutil

    shutil.copyfile(os.path.join(REF, "casefiles", "1step", "dmpi0000000.dat"),
                    os.path.join(HERE, "dmpi_1step_1001.dat"))
    shutil.copyfile(os.path.join(REF, "casefiles", "21step", "dmpi0000000.dat"),
                    os.path.join(HERE, "dmpi_21step_1001.dat"))
    # the same case's constant-Lewis-number flame (dmpi0000000_cle.dat)
    shutil.copyfile(os.path.join(REF, "casefiles", "21step", "dmpi0000000_cle.dat"),
                    os.path.join(HERE, "dmpi_21step_cle_1001.dat"))
    # the 1-step and 4-step cases' own mechanisms and the 4-step restart state
    for src, dst in (("1step/chem.dat", "casefile_1step_chem.dat"), ("4step/chem.dat", "casefile_4step_chem.dat"),
                     ("4step/diff.dat", "casefile_4step_diff.dat"), ("4step/dmpi0000000.dat", "dmpi_4step_1001.dat")):
        shutil.copyfile(os.path.join(REF, "casefiles", src), os.path.join(HERE, dst))
    for case in ("25step", "68step"):
        for src, dst in (("chem.dat", f"casefile_{case}_chem.dat"), ("diff.dat", f"casefile_{case}_diff.dat"),
                         ("dmpi0000000.dat", f"dmpi_{case}_1001.dat")):
            shutil.copyfile(os.path.join(REF, "casefiles", case, src), os.path.join(HERE, dst))


def main():
    casefile_dump()
    coeffs = {"rk": rk_coefficients(), "fd": fd_coefficients()}
    with open(os.path.join(HERE, "coefficients.json"), "w") as f:
        json.dump(coeffs, f, indent=1, sort_keys=True)
    print("rk", len(coeffs["rk"]), "fd", len(coeffs["fd"]))
    oracle_fixtures()


if __name__ == "__main__":
    main()
