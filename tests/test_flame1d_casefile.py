"""The reference's own 21-step H2/air restart case (src/casefiles/21step:
cont.dat and dmpi0000000.dat, copied as tests/golden/dmpi_21step_1001.dat):
a 1D flame on 1001 x 1 x 1 points, 10 mm, NSCBC I3 inflow at 2.05 m/s and O1
outflow (p_inf 1e5 Pa, sigma 0.287, eta 1e-3), one-point periodic y and z,
mixture-averaged transport with the molar-mass, pressure, Soret and Dufour
switches on (light-species limit 5.0), adaptive steps.

CPU: the bisection start-up temperature agrees with the oracle's TEMPER.
GPU: RHS, fixed-step and adaptive-step runs against the oracle, field-
normalised relative L-infinity 1e-10. This converged flame makes its
momentum RHS a small residual (max ~30) of terms near 6e4 (the pressure
gradient against the convective flux), so rounding-level differences in
the state move it by ~1e-7 of its own maximum: the RHS check allows each
field ten times the change that the oracle itself shows under a one-ulp
random perturbation of the input state, or 1e-10, whichever is larger."""
import os

import numpy as np
import pytest

from conftest import rel_linf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dmpi_21step_1001.dat")
SHAPE, LENGTHS, NEND = (1001, 1, 1), (1.0e-2, 1.0e-3, 1.0e-3), (1, 1, 2, 2, 2, 2)
SWITCHES = dict(mixw=True, mixp=True, soret=True, dufour=True, wmltdr=5.0)


def _case():
    import cases
    import senga

    f, sc = senga.dump_read(GOLD, formatted=True)
    chem = senga.Chem(cases.CHEM_H2)
    T, itn = cases.temperature_from_state(chem, f)
    rg = chem.table("rgspec")[:9]
    yin = np.zeros(9)
    yin[0], yin[1], yin[8] = 2.8312571e-2, 2.26500566e-1, 7.45186863e-1  # cont.dat mass fractions
    rho_in = 1.0e5 / (300.0 * float((rg * yin).sum()))
    bc = dict(xl=13, xr=21, u_in=2.05, rho_in=rho_in, y_in=tuple(yin), p_inf=1.0e5, sigma=0.287, eta=1.0e-3,
              pio=0, bet_local=0)
    return f, sc, T, itn, bc


def _oracle(bc, dt, adaptive=False):
    import cases
    from oracle import Oracle

    o = Oracle(SHAPE, LENGTHS, cases.CHEM_H2, cases.DIFF_H2, dt, nend=NEND)
    o.set_bc(bc)
    o.set_transport(**SWITCHES)
    if adaptive:
        o.set_adaptive(True)
    return o


def test_startup_temperature_matches_temper():
    f, sc, T, itn, bc = _case()
    assert f.shape == (14, 1, 1, 1001)
    assert 299.0 < T.min() < 301.0 and 2300.0 < T.max() < 2400.0
    o = _oracle(bc, sc["tstep"])
    o.upload(f, T, itn)
    _, t2, p = o.rhs()
    assert float(np.abs(t2 - T).max()) <= 1e-8
    assert abs(float(p.min()) / 1.0e5 - 1.0) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("adaptive", [False, True])
def test_gpu_casefile_flame_matches_oracle(adaptive):
    import cases
    import senga

    f, sc, T, itn, bc = _case()
    chem = senga.Chem(cases.CHEM_H2)
    diff = senga.Diff(cases.DIFF_H2, chem)
    box = senga.Box(SHAPE, LENGTHS, chem, diff, sc["tstep"], nend=NEND, adaptive=adaptive)
    box.set_nscbc(bc)
    box.set_transport(**SWITCHES)
    ref = _oracle(bc, sc["tstep"], adaptive)
    box.upload(f, T, itn)
    ref.upload(f, T, itn)
    if not adaptive:
        r, _, _ = box.rhs()
        rr, _, _ = ref.rhs()
        rng = np.random.default_rng(7)
        g = f * (1.0 + 2.2e-16 * rng.choice([-1.0, 1.0], size=f.shape))
        pert = _oracle(bc, sc["tstep"])
        pert.upload(g, T, itn)
        rp, _, _ = pert.rhs()
        for fl in range(r.shape[0]):
            tol = max(1e-10, 10.0 * rel_linf(rp[fl], rr[fl]))
            assert rel_linf(r[fl], rr[fl]) <= tol, (fl, rel_linf(r[fl], rr[fl]), tol)
        box.upload(f, T, itn)
        ref.upload(f, T, itn)
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    w, tw, _ = ref.download()
    for fl in range(g.shape[0]):
        assert rel_linf(g[fl], w[fl]) <= 1e-10, fl
    assert rel_linf(tg, tw) <= 1e-10
    if adaptive:
        (dg, eg, ig), (dw, ew, iw) = box.tstep(), ref.tstep()
        assert abs(dg / dw - 1.0) <= 1e-8 and ig == iw
