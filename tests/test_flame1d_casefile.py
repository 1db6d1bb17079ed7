"""The reference's own 1D restart cases (src/casefiles/{1step,4step,21step,
25step,68step}:
cont.dat, chem.dat, diff.dat and the formatted restart dump, copied under
tests/golden/): 1001 x 1 x 1 points over 10 mm, NSCBC I3 inflow and O1
outflow (p_inf 1e5 Pa, sigma 0.287, eta 1e-3), one-point periodic y and z,
adaptive steps. 1step: single-step R -> P, constant-Lewis transport, inflow
0.39 m/s. 4step: 8-species 6-step mechanism, mixture-averaged transport
with the molar-mass, pressure, Soret and Dufour switches on, inflow 0.5
m/s. 21step: the H2/air mechanism of the named workloads, every switch on,
inflow 2.05 m/s. 25step and 68step: methane/air with 16 and 18 species
(ITNDEX in two words per point), every switch on, inflow 0.39 m/s.

CPU: the bisection start-up temperature agrees with the oracle's TEMPER.
GPU: RHS, fixed-step and adaptive-step runs against the oracle, field-
normalised relative L-infinity 1e-10. A converged flame makes its momentum
RHS a small residual (21step: max ~30) of terms near 6e4 (the pressure
gradient against the convective flux), so rounding-level differences in
the state move it by ~1e-7 of its own maximum: the RHS check allows each
field ten times the change that the oracle itself shows under a one-ulp
random perturbation of the input state, or 1e-10, whichever is larger."""
import os

import numpy as np
import pytest

from conftest import rel_linf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHAPE, LENGTHS, NEND = (1001, 1, 1), (1.0e-2, 1.0e-3, 1.0e-3), (1, 1, 2, 2, 2, 2)
ALL = dict(mixw=True, mixp=True, soret=True, dufour=True, wmltdr=5.0)

# per case: chem, diff, dump, inflow velocity RXLPRM(1), default mass
# fractions (cont.dat "mass fractions"), transport switches
CASES = {
    "1step": ("casefile_1step_chem.dat", None, "dmpi_1step_1001.dat", 0.39, {0: 1.0}, None),
    "4step": ("casefile_4step_chem.dat", "casefile_4step_diff.dat", "dmpi_4step_1001.dat", 0.5,
              {0: 5.5045872e-2, 1: 2.20183486e-1, 7: 7.24770642e-1}, ALL),
    "21step": (None, None, "dmpi_21step_1001.dat", 2.05,
               {0: 2.8312571e-2, 1: 2.26500566e-1, 8: 7.45186863e-1}, ALL),
    # methane/air, 16 and 18 species: ITNDEX takes two words per point
    "25step": ("casefile_25step_chem.dat", "casefile_25step_diff.dat", "dmpi_25step_1001.dat", 0.39,
               {0: 5.5045872e-2, 1: 2.20183486e-1, 15: 7.24770642e-1}, ALL),
    "68step": ("casefile_68step_chem.dat", "casefile_68step_diff.dat", "dmpi_68step_1001.dat", 0.39,
               {0: 5.5045872e-2, 1: 2.20183486e-1, 17: 7.24770642e-1}, ALL),
}


def _paths(name):
    import cases

    chem, diff, dump, u_in, yin, sw = CASES[name]
    chem = os.path.join(GOLD, chem) if chem else cases.CHEM_H2
    diff = os.path.join(GOLD, diff) if diff else (cases.DIFF_H2 if name == "21step" else None)
    return chem, diff, os.path.join(GOLD, dump), u_in, yin, sw


def _case(name):
    import cases
    import senga

    chem_p, diff_p, dump, u_in, yin, sw = _paths(name)
    f, sc = senga.dump_read(dump, formatted=True)
    chem = senga.Chem(chem_p)
    T, itn = cases.temperature_from_state(chem, f)
    ns = chem.nspec
    rg = chem.table("rgspec")[:ns]
    y = np.zeros(ns)
    for k, v in yin.items():
        y[k] = v
    rho_in = 1.0e5 / (300.0 * float((rg * y).sum()))  # PRIN / (R_mix TRIN)
    bc = dict(xl=13, xr=21, u_in=u_in, rho_in=rho_in, y_in=tuple(y), p_inf=1.0e5, sigma=0.287, eta=1.0e-3,
              pio=0, bet_local=0)
    return f, sc, T, itn, bc


def _oracle(name, bc, dt, adaptive=False):
    from oracle import Oracle

    chem_p, diff_p, _, _, _, sw = _paths(name)
    o = Oracle(SHAPE, LENGTHS, chem_p, diff_p, dt, nend=NEND)
    o.set_bc(bc)
    if sw:
        o.set_transport(**sw)
    if adaptive:
        o.set_adaptive(True)
    return o


@pytest.mark.parametrize("name", list(CASES))
def test_startup_temperature_matches_temper(name):
    f, sc, T, itn, bc = _case(name)
    assert f.shape[1:] == (1, 1, 1001)
    assert 299.0 < T.min() < 301.0 and T.max() > 1800.0
    o = _oracle(name, bc, sc["tstep"])
    o.upload(f, T, itn)
    _, t2, p = o.rhs()
    assert float(np.abs(t2 - T).max()) <= 1e-8
    assert abs(float(p.min()) / 1.0e5 - 1.0) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("adaptive", [False, True], ids=["fixed", "adaptive"])
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_casefile_flame_matches_oracle(name, adaptive):
    import senga

    f, sc, T, itn, bc = _case(name)
    chem_p, diff_p, _, _, _, sw = _paths(name)
    chem = senga.Chem(chem_p)
    diff = senga.Diff(diff_p, chem)
    box = senga.Box(SHAPE, LENGTHS, chem, diff, sc["tstep"], nend=NEND, adaptive=adaptive)
    box.set_nscbc(bc)
    if sw:
        box.set_transport(**sw)
    ref = _oracle(name, bc, sc["tstep"], adaptive)
    box.upload(f, T, itn)
    ref.upload(f, T, itn)
    if not adaptive:
        r, _, _ = box.rhs()
        rr, _, _ = ref.rhs()
        rng = np.random.default_rng(7)
        g = f * (1.0 + 2.2e-16 * rng.choice([-1.0, 1.0], size=f.shape))
        pert = _oracle(name, bc, sc["tstep"])
        pert.upload(g, T, itn)
        rp, _, _ = pert.rhs()
        for fl in range(r.shape[0]):
            if np.max(np.abs(rr[fl])) == 0.0:
                assert np.max(np.abs(r[fl])) == 0.0, fl
                continue
            tol = max(1e-10, 10.0 * rel_linf(rp[fl], rr[fl]))
            assert rel_linf(r[fl], rr[fl]) <= tol, (fl, rel_linf(r[fl], rr[fl]), tol)
        box.upload(f, T, itn)
        ref.upload(f, T, itn)
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    w, tw, _ = ref.download()
    for fl in range(g.shape[0]):
        if np.max(np.abs(w[fl])) == 0.0:
            assert np.max(np.abs(g[fl])) == 0.0, fl
            continue
        assert rel_linf(g[fl], w[fl]) <= 1e-10, fl
    assert rel_linf(tg, tw) <= 1e-10
    if adaptive:
        (dg, eg, ig), (dw, ew, iw) = box.tstep(), ref.tstep()
        assert abs(dg / dw - 1.0) <= 1e-8 and ig == iw
