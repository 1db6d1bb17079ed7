"""Synthetic turbulent inflow velocity (src/inflow.f; BCUTXL NXLPRM(1) = 4)
on the I3 x-left face of a small inflow/outflow H2 flame, against the
oracle's own restatement: the random planes (RAN1, drawn on the host in the
reference's order), the Gaussian filters, the temporal correlation, the
mean removal, and the face values and time derivatives the I3 conditions
take, over several steps (field-normalised L-infinity 1e-10)."""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-10

SETS = [
    dict(urms=0.5, coflow=0.0, lnx=30, lny=30, lnz=30, nfy=60, nfz=60, itime=1),  # the reference's PARAMETERs
    dict(urms=0.3, coflow=0.1, lnx=8, lny=3, lnz=2, nfy=6, nfz=4, itime=5),
]


@pytest.mark.parametrize("adaptive", [False, True], ids=["fixed", "adaptive"])
@pytest.mark.parametrize("p", SETS, ids=["default-filters", "small-filters"])
def test_synthetic_inflow_matches_oracle(p, adaptive):
    import cases
    import senga
    from oracle import Oracle

    c = cases.make_case("flame_inout", seed=13, shape=(24, 8, 12))
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"], adaptive=adaptive)
    box.set_nscbc(c["bc"])
    box.set_synthetic_inflow(**p)
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    ref.set_bc(c["bc"])
    if adaptive:
        ref.set_adaptive(True)
    ref.set_synth(p["urms"], p["coflow"], p["lnx"], p["lny"], p["lnz"], p["nfy"], p["nfz"], p["itime"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    assert box.status() == 0
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL, f"state field {k}"
    assert rel_linf(tg, to) <= TOL
    # the inflow plane carries the fluctuations, with the face mean of u at
    # u_in + coflow
    face_v = g[2][:, :, 0] / g[0][:, :, 0]
    face_u = g[1][:, :, 0] / g[0][:, :, 0]
    assert np.std(face_v) > 1e-4 * p["urms"]  # amplitude ~ urms sqrt(2 dt / theta) at these steps
    assert abs(face_u.mean() - (c["bc"]["u_in"] + p["coflow"])) < 1e-10 * c["bc"]["u_in"]


def test_synthetic_inflow_needs_an_i3_inflow():
    import cases
    import senga

    c = cases.make_case("h2_pool", seed=5, shape=(16, 8, 8))
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    with pytest.raises(senga.SengaError):
        box.set_synthetic_inflow(0.5)
