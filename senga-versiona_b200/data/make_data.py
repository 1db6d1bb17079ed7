"""Regenerates the mechanism input files of the named workloads.

* chem_h2.dat / diff_h2.dat: the reference project's own input/chem.dat and
  input/diff.dat (H2/air, 9 species, 21 steps; ppchem/ppdiff output), copied
  verbatim because the 128^3 and 256^3 workloads are defined on them.
* radn_h2.dat: the reference project's input/radn.dat (Planck-mean
  absorption polynomial of H2O for the same 9-species list), copied verbatim
  for the radiation tests.
* chem_1step.dat: the single-step irreversible R -> P mechanism of the 32^3
  and batched workloads, written in the same chem.dat record layout
  (src/chemin.f:146-344): A = 1e9 1/s, Ea/R = 15000 K, equal molar mass 29
  and constant cp = 3.5 R/W for both species, product enthalpy of formation
  lowered by 5250 K * R/W so that T_ad = 300 + 5250/3.5 = 1800 K at constant
  pressure, unit Lewis numbers.

Usage: python make_data.py <reference_root>   (or SENGA_REFERENCE_ROOT set)
Without a reference root only chem_1step.dat is rewritten.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

RGUNIV = 8.3142e3


def species_block(idx, wmol, clewis, a6):
    lines = [f"{idx:5d}{wmol:12.4E}", f"{clewis:12.4E}", f"{2:5d}"]
    for lo, hi in ((3.0e2, 1.0e3), (1.0e3, 5.0e3)):
        lines.append(f"{lo:12.4E}{hi:12.4E}{7:5d}")
        for c in (3.5, 0.0, 0.0, 0.0, 0.0, a6, 0.0):
            lines.append(f"{c:15.7E}")
    return lines


def one_step_chem():
    e_act = 1.5e4 * RGUNIV  # activation energy [J/kmol]; CHEMIN divides by RGUNIV
    out = [" *****************************", " *  single-step R -> P        *",
           " *  1-step ignition workloads *", " *                           *",
           " *****************************", " Species list:", f"{2:5d}",
           f"{1:5d}   R         ", f"{2:5d}   P         ", " Species data:", "  1.0000E+05"]
    out += species_block(1, 29.0, 1.0, 0.0)
    out += species_block(2, 29.0, 1.0, -5250.0)
    out += [" Step rate data:", f"{1:5d}", f"{1:5d}{1.0e9:12.4E}{0.0:12.4E} {e_act:11.5E}"]
    out += [" Step species-list:", f"{1:5d}{2:5d}", f"{1:5d}{1:5d}{1:8d}", f"{1:5d}{2:5d}{2:8d}"]
    out += [" Step reactant-list:", f"{1:5d}{1:5d}", f"{1:5d}{1:5d}{1:8d}"]
    out += [" Step product-list:", f"{1:5d}{1:5d}", f"{1:5d}{1:5d}{2:8d}"]
    out += [" Step reactant coefficient-list:", f"{1:5d}{0:5d}"]
    out += [" Step product coefficient-list:", f"{1:5d}{0:5d}"]
    out += [" Species delta-list:", f"{1:5d}{1:5d}{-1.0:5.1f}", f"{1:5d}{2:5d}{1.0:5.1f}"]
    out += [" Third-body list:", f"{0:5d}", " Third-body step-list:", " Third-body efficiencies:"]
    out += [" Gibbs step-list:", f"{0:5d}"]
    out += [" Lindemann step-list:", f"{0:5d}", " Lindemann step rate data:"]
    out += [" Troe step-list:", f"{0:5d}", " Troe step rate data:"]
    out += [" SRI step-list:", f"{0:5d}", " SRI step rate data:", " End of file"]
    return "\n".join(out) + "\n"


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SENGA_REFERENCE_ROOT", "")
    with open(os.path.join(HERE, "chem_1step.dat"), "w") as fh:
        fh.write(one_step_chem())
    for src, dst in (("input/chem.dat", "chem_h2.dat"), ("input/diff.dat", "diff_h2.dat"),
                     ("input/radn.dat", "radn_h2.dat")):
        path = os.path.join(ref, src)
        if ref and os.path.exists(path):
            shutil.copyfile(path, os.path.join(HERE, dst))


if __name__ == "__main__":
    main()
