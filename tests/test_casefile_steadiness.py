"""The reference's converged 1D flames are steady under this discretisation.

src/casefiles/1step/dmpi0000000.dat (constant Lewis numbers) and
src/casefiles/21step/dmpi0000000.dat (mixture-averaged with every switch)
are restart states the reference ran to convergence with the cont.dat of
their case; 21step/dmpi0000000_cle.dat is the same flame converged with
constant Lewis numbers. Evaluating the oracle's RHS on such a state gives
the front's velocity in the lab frame, -(dY/dt)/(dY/dx) at the mid-level of
the product mass fraction: a correct restatement of the reference's
equations finds it a small fraction of the inflow velocity (the flame
stands still in the frame where the reference converged it), while the
other transport model moves it by 15-25% of the inflow speed. This pins the
oracle (chemistry, transport, NSCBC faces, derivative closures) against
outputs of the reference itself, at the level of the flame speed; the GPU
test repeats the check through the product's C ABI."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALL = dict(mixw=True, mixp=True, soret=True, dufour=True, wmltdr=5.0)


def _front_velocity(chem_p, diff_p, dump, u_in, yin, switches, device=False):
    import cases
    import senga
    from oracle import Oracle

    f, _ = senga.dump_read(os.path.join(GOLD, dump), formatted=True)
    chem = senga.Chem(chem_p)
    T, itn = cases.temperature_from_state(chem, f)
    ns = chem.nspec
    rg = chem.table("rgspec")[:ns]
    y = np.zeros(ns)
    for k, v in yin.items():
        y[k] = v
    bc = dict(xl=13, xr=21, u_in=u_in, rho_in=1.0e5 / (300.0 * float((rg * y).sum())), y_in=tuple(y),
              p_inf=1.0e5, sigma=0.287, eta=1.0e-3, pio=0, bet_local=0)
    if device:  # the product path through the C ABI
        o = senga.Box((1001, 1, 1), (1.0e-2, 1.0e-3, 1.0e-3), chem, senga.Diff(diff_p, chem), 1.0e-8,
                      nend=(1, 1, 2, 2, 2, 2))
        o.set_nscbc(bc)
    else:
        o = Oracle((1001, 1, 1), (1.0e-2, 1.0e-3, 1.0e-3), chem_p, diff_p, 1.0e-8, nend=(1, 1, 2, 2, 2, 2))
        o.set_bc(bc)
    if switches:
        o.set_transport(**switches)
    o.upload(f, T, itn)
    r, _, _ = o.rhs()
    x = np.arange(1001) * 1.0e-5
    rho = f[0, 0, 0]
    ys = f[5:, 0, 0] / rho
    k = int(np.argmax(np.abs(ys[:, -1] - ys[:, 0])))  # the product that changes most across the flame
    yk = ys[k]
    dydt = (r[5 + k, 0, 0] - yk * r[0, 0, 0]) / rho
    half = 0.5 * (yk[0] + yk[-1])
    i = int(np.argmax(np.abs(yk - yk[0]) > abs(half - yk[0])))
    return -dydt[i] / np.gradient(yk, x)[i]


H2_IN = {0: 2.8312571e-2, 1: 2.26500566e-1, 8: 7.45186863e-1}


@pytest.mark.parametrize("dump,model,steady", [
    ("dmpi_21step_1001.dat", "mavt", True),
    ("dmpi_21step_1001.dat", "lewis", False),
    ("dmpi_21step_cle_1001.dat", "lewis", True),
    ("dmpi_21step_cle_1001.dat", "mavt", False),
])
def test_h2_flames_stand_still_under_their_own_transport_model(dump, model, steady):
    import cases

    v = _front_velocity(cases.CHEM_H2, cases.DIFF_H2 if model == "mavt" else None, dump, 2.05, H2_IN,
                        ALL if model == "mavt" else None)
    if steady:
        assert abs(v) < 0.05 * 2.05, v
    else:
        assert abs(v) > 0.1 * 2.05, v


def test_one_step_flame_stands_still():
    v = _front_velocity(os.path.join(GOLD, "casefile_1step_chem.dat"), None, "dmpi_1step_1001.dat", 0.39, {0: 1.0},
                        None)
    assert abs(v) < 0.01 * 0.39, v


@pytest.mark.gpu
def test_device_holds_the_reference_flames_still():
    import cases

    v = _front_velocity(cases.CHEM_H2, cases.DIFF_H2, "dmpi_21step_1001.dat", 2.05, H2_IN, ALL, device=True)
    assert abs(v) < 0.05 * 2.05, v
    v = _front_velocity(os.path.join(GOLD, "casefile_1step_chem.dat"), None, "dmpi_1step_1001.dat", 0.39, {0: 1.0},
                        None, device=True)
    assert abs(v) < 0.01 * 0.39, v

