"""Optically thin radiation heat loss: RADCIN's reading of radn.dat
(src/radcin.f:80-220) and RADCAL (src/radcal.f:45-119, called from
src/rhscal.f:810).

CPU: the C ABI reader against the file's own numbers, bad files, and the
oracle's energy sink on uniform states against the closed form
  ERHS(on) - ERHS(off) = -4 STEFBO a(T) rho Y_H2O R_H2O T (T^4 - TREFRN^4),
a(T) the Horner polynomial of the file. GPU: the product RHS and steps with
radiation on against the oracle (field-normalised relative L-infinity 1e-10,
as for every state comparison), and the same closed form on the device."""
import os

import numpy as np
import pytest

from conftest import rel_linf

STEFBO = 5.67037321e-08  # src/com_senga2.h:222
# radn.dat of the H2/air mechanism: species 3 (H2O), six coefficients
AK_H2O = [6.869480e-04, -1.523490e-06, 1.417848e-09, -6.620996e-13, 1.524150e-16, -1.373456e-20]


def _sink(fields, T, rg_h2o, trefrn):
    a = 0.0
    for c in reversed(AK_H2O):
        a = a * T + c
    return -4.0 * STEFBO * a * fields[5 + 2] * rg_h2o * T * (T ** 4 - trefrn ** 4)


def _uniform(T0, shape=(12, 12, 12), p=101325.0):
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_H2)
    nx, ny, nz = shape
    shp = (nz, ny, nx)
    Y = [0.01, 0.12, 0.14, 0.0, 0.002, 0.0, 0.0, 0.0]
    Y.append(1.0 - sum(Y))
    z = np.zeros(shp)
    fields, itn = cases.conserved(chem, np.full(shp, p), np.full(shp, T0), z, z, z,
                                  np.array([np.full(shp, y) for y in Y]))
    return chem, fields, np.full(shp, T0), itn


def test_radn_reader_takes_the_file_numbers():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_H2)
    r = senga.Radn(cases.RADN_H2, chem, trefrn=300.0)
    assert r.species == [3]
    assert r.coefficients(0) == AK_H2O
    assert r.t.trefrn == 300.0


def test_radn_reader_rejects_bad_files(tmp_path):
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_H2)
    with pytest.raises(senga.SengaError):
        senga.Radn(str(tmp_path / "missing.dat"), chem)
    text = open(cases.RADN_H2).read().splitlines()
    at = next(i for i, l in enumerate(text) if l.split() == ["3", "6"])
    for bad in (["12", "6"], ["3", "7"]):  # species past NSPEC; more than NCFRMX coefficients
        lines = list(text)
        lines[at] = "    " + "    ".join(bad)
        p = tmp_path / "bad.dat"
        p.write_text("\n".join(lines) + "\n")
        with pytest.raises(senga.SengaError):
            senga.Radn(str(p), chem)
    lines = text[:at + 1]  # coefficients cut off
    p = tmp_path / "short.dat"
    p.write_text("\n".join(lines) + "\n")
    with pytest.raises(senga.SengaError):
        senga.Radn(str(p), chem)


@pytest.mark.parametrize("T0", [900.0, 1800.0, 2400.0])
def test_oracle_radiation_sink_on_a_uniform_state(T0):
    import cases
    from oracle import Oracle

    chem, fields, T, itn = _uniform(T0)
    rg = chem.table("rgspec")[2]
    o = Oracle((12, 12, 12), (1e-3,) * 3, cases.CHEM_H2, cases.DIFF_H2, 1e-9)
    o.upload(fields, T, itn)
    off, _, _ = o.rhs()
    o.set_radiation(cases.RADN_H2, 300.0)
    o.upload(fields, T, itn)  # the oracle's RHS overwrites the U register
    on, _, _ = o.rhs()
    assert np.array_equal(on[:4], off[:4]) and np.array_equal(on[5:], off[5:])
    want = _sink(fields, T, rg, 300.0)
    assert np.all(want < 0.0)
    assert rel_linf(on[4] - off[4], want) <= 1e-12


def test_oracle_radiation_vanishes_at_the_reference_temperature():
    import cases
    from oracle import Oracle

    chem, fields, T, itn = _uniform(1200.0)
    o = Oracle((12, 12, 12), (1e-3,) * 3, cases.CHEM_H2, cases.DIFF_H2, 1e-9)
    o.upload(fields, T, itn)
    off, _, _ = o.rhs()
    o.set_radiation(cases.RADN_H2, 1200.0)
    o.upload(fields, T, itn)  # the oracle's RHS overwrites the U register
    on, _, _ = o.rhs()
    assert np.array_equal(on, off)
    o.set_radiation(None)
    o.upload(fields, T, itn)
    again, _, _ = o.rhs()
    assert np.array_equal(again, off)


# ------------------------------------------------------------------ GPU
def _pair(c, trefrn=300.0):
    import cases
    import senga
    from oracle import Oracle

    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.set_radiation(senga.Radn(cases.RADN_H2, chem, trefrn))
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    ref.set_radiation(cases.RADN_H2, trefrn)
    if "bc" in c:
        box.set_nscbc(c["bc"])
        ref.set_bc(c["bc"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    return box, ref


@pytest.mark.gpu
def test_gpu_radiation_rhs_matches_oracle():
    import cases

    c = cases.make_case("h2_kernels", n=16, seed=21)
    box, ref = _pair(c)
    r, t, p = box.rhs()
    rr, tr, pr = ref.rhs()
    for fl in range(r.shape[0]):
        assert rel_linf(r[fl], rr[fl]) <= 1e-10, fl


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["h2_kernels", "flame_inout"])
def test_gpu_radiation_steps_match_oracle(case):
    import cases

    c = cases.make_case(case, n=16, seed=22)
    box, ref = _pair(c)
    box.step(3)
    ref.step(3)
    f, t, _ = box.download()
    fr, tr, _ = ref.download()
    for fl in range(f.shape[0]):
        assert rel_linf(f[fl], fr[fl]) <= 1e-10, fl
    assert rel_linf(t, tr) <= 1e-10


@pytest.mark.gpu
def test_gpu_radiation_sink_on_a_uniform_state():
    import cases
    import senga

    chem, fields, T, itn = _uniform(2000.0, shape=(16, 16, 16))
    diff = senga.Diff(cases.DIFF_H2, chem)
    box = senga.Box((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-9)
    box.upload(fields, T, itn)
    off, _, _ = box.rhs()
    box.set_radiation(senga.Radn(cases.RADN_H2, chem, 300.0))
    box.upload(fields, T, itn)
    on, _, _ = box.rhs()
    want = _sink(fields, T, chem.table("rgspec")[2], 300.0)
    assert rel_linf(on[4] - off[4], want) <= 1e-12
    box.set_radiation(None)
    box.upload(fields, T, itn)
    again, _, _ = box.rhs()
    assert np.array_equal(again, off)
