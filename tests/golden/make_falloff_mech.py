"""Writes chem_h2_troe_sri.dat, a test mechanism whose falloff steps use the
Troe and SRI forms of CHRATE (src/chrate.f:312-375, :387-434), which no
mechanism shipped with the reference uses.

It is the project's H2/air chem.dat (senga-versiona_b200/data/chem_h2.dat,
the reference's input/chem.dat) with its two Lindemann steps moved, in the
chem.dat record layout of src/chemin.f:290-339:
  * step 9 to the Troe form: the same low-pressure Arrhenius triple, alpha
    0.7, T*** 100 K, T* 1500 K, T** 5000 K, c = -0.4 - 0.67 log10 Fcent,
    n = 0.75 - 1.27 log10 Fcent, d = 0.14;
  * step 15 to the SRI form: the low-pressure pre-exponential raised 1e8
    times so that the reduced pressure Pr stays above 10 on the test states
    (the SRI branch as coded takes log10(log10 Pr), finite only for Pr > 1),
    a = 0.5, b = 600 K, c = 1000 K, d = 1.0, e = 0 (the coded branch computes
    and drops the T**e factor).

Run from the repository root:  python tests/golden/make_falloff_mech.py
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "..", "senga-versiona_b200", "data", "chem_h2.dat")
DST = os.path.join(HERE, "chem_h2_troe_sri.dat")


def e12(v):
    return f"{v:12.4E}"


def main():
    with open(SRC) as fh:
        lines = fh.read().splitlines()
    i = lines.index(" Lindemann step-list:")
    nstep = 21
    lind = lines[i + 2:i + 2 + nstep]
    data = lines[i + 2 + nstep + 1:i + 2 + nstep + 3]
    assert lines[i + 2 + nstep] == " Lindemann step rate data:" and len(data) == 2
    k0_9 = [float(data[0][5 + 12 * k:17 + 12 * k]) for k in range(3)]
    k0_15 = [float(data[1][5 + 12 * k:17 + 12 * k]) for k in range(3)]
    out = lines[:i]
    out += [" Lindemann step-list:", f"{0:5d}", " Lindemann step rate data:"]
    out += [" Troe step-list:", f"{1:5d}"]
    out += [f"{s:5d}{(1 if s == 9 else 0):8d}" for s in range(1, nstep + 1)]
    out += [" Troe step rate data:",
            f"{1:5d}" + "".join(e12(v) for v in (k0_9[0], k0_9[1], k0_9[2], 0.7, 100.0, 1500.0)),
            f"{1:5d}" + "".join(e12(v) for v in (5000.0, -0.4, -0.67, 0.75, -1.27, 0.14))]
    out += [" SRI step-list:", f"{1:5d}"]
    out += [f"{s:5d}{(1 if s == 15 else 0):8d}" for s in range(1, nstep + 1)]
    out += [" SRI step rate data:",
            f"{1:5d}" + "".join(e12(v) for v in (k0_15[0] * 1.0e8, k0_15[1], k0_15[2])),
            f"{1:5d}" + "".join(e12(v) for v in (0.5, 600.0, 1000.0, 1.0, 0.0))]
    out += [" End of file"]
    del lind
    with open(DST, "w") as fh:
        fh.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
