"""CHRATE's Troe and SRI falloff branches (src/chrate.f:312-375, :387-434),
which no mechanism shipped with the reference uses, on the test mechanism
tests/golden/chem_h2_troe_sri.dat (the H2/air mechanism with its Lindemann
steps moved to the Troe and SRI forms; tests/golden/make_falloff_mech.py).

CPU: the device library's chem.dat reader and the oracle's agree on the
falloff tables after CHEMIN's derived pass (ln A, E/R, the inverted Troe
temperatures, the negated SRI constants; src/chemin.f:838-857), and the
branches change the rates. GPU: the table-driven thermochemistry kernel
against the oracle, RATE, the RHS and three RK steps (a tenth of the CFL
step: the raised SRI rate makes the chemistry stiffer), field-normalised
relative L-infinity 1e-10."""
import os

import numpy as np
import pytest

from conftest import rel_linf

MECH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "chem_h2_troe_sri.dat")
TOL = 1e-10


def _case():
    import cases

    c = cases.make_case("h2_pool", seed=7, shape=(12, 10, 8))
    c["chem"] = MECH
    c["dt"] = c["dt"] / 10.0
    return c


def test_falloff_tables_read_alike():
    import senga
    from oracle import OracleChem

    dev = senga.Chem(MECH)
    orc = OracleChem(MECH)
    assert (dev.t.nlind, dev.t.ntroe, dev.t.nsrif) == (0, 1, 1)
    for name in ("mtlist", "mslist", "mllist"):
        assert np.array_equal(dev.table(name), orc.table(name)), name
    for name in ("rctroe", "rcsrif"):
        assert np.array_equal(dev.table(name), orc.table(name)), name
    # the derived pass: T*** and T* stored as -1/T, SRI b and c as -b, -1/c
    t = dev.table("rctroe")[0]
    assert t[4] == -1.0 / 100.0 and t[6] == -1.0 / 5000.0 and t[5] == 1500.0
    r = dev.table("rcsrif")[0]
    assert r[4] == -600.0 and r[5] == -1.0 / 1000.0


def test_falloff_branches_change_the_rates():
    import cases
    from oracle import Oracle

    c = _case()
    a = Oracle(c["shape"], c["lengths"], MECH, c["diff"], c["dt"])
    b = Oracle(c["shape"], c["lengths"], cases.CHEM_H2, c["diff"], c["dt"])
    for o in (a, b):
        o.upload(c["fields"], c["T"], c["itn"])
    ra, rb = a.chrate(), b.chrate()
    assert np.isfinite(ra).all()
    assert max(rel_linf(ra[k], rb[k]) for k in range(9) if np.max(np.abs(rb[k])) > 0) > 1e-2


@pytest.mark.gpu
def test_falloff_rates_rhs_and_steps_match_oracle():
    import senga
    from oracle import Oracle

    c = _case()
    chem = senga.Chem(MECH)
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    assert box.info()["mech"] == 0  # the table-driven kernel
    ref = Oracle(c["shape"], c["lengths"], MECH, c["diff"], c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    got, want = box.chrate(), ref.chrate()
    for k in range(want.shape[0]):
        if np.max(np.abs(want[k])) > 0:
            assert rel_linf(got[k], want[k]) <= TOL, f"RATE species {k}"
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    r, t, _ = box.rhs()
    rr, tr, _ = ref.rhs()
    for k in range(rr.shape[0]):
        assert rel_linf(r[k], rr[k]) <= TOL, f"RHS field {k}"
    # rhs() leaves R(U) in the U register: start the steps from the state
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    assert np.isfinite(o).all()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL, f"state field {k}"
    assert rel_linf(tg, to) <= TOL
