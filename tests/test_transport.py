"""Molar-mass, pressure, Soret and Dufour terms of mixture-averaged transport
(cont.dat transport switches; src/diffin.f:384-406, src/rhscal.f:946-1003,
1352-1403, 1552-1564, 1966-3765).

CPU (oracle): the branches vanish where their driving gradient does (uniform
composition and pressure; no second light species for the thermal diffusion
ratio), Dufour touches only the energy equation, every branch adds the same
amount to its species source and to the correction-velocity divergence (so
sum_k YRHS_k = DRHS still holds), and the switches need mixture-averaged
transport. GPU: the product RHS and steps against the oracle, field-normalised
relative L-infinity 1e-10 as for every state comparison."""
import numpy as np
import pytest

from conftest import rel_linf

ALL = dict(mixw=True, mixp=True, soret=True, dufour=True)
SWITCHES = [dict(mixw=True), dict(mixp=True), dict(soret=True), dict(dufour=True), ALL]


def _oracle_rhs(c, **sw):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    if sw:
        o.set_transport(**sw)
    o.upload(c["fields"], c["T"], c["itn"])
    r, _, _ = o.rhs()
    return r


def _field_rel(a, b):
    return max(rel_linf(a[f], b[f]) if np.max(np.abs(b[f])) > 0 else float(np.max(np.abs(a[f])))
               for f in range(a.shape[0]))


@pytest.mark.parametrize("sw", SWITCHES[:4], ids=["mixw", "mixp", "soret", "dufour"])
def test_branches_vanish_without_their_gradients(sw):
    """h2_kernels: uniform H2/air composition and pressure, no H atoms: the
    molar-mass and pressure gradients are rounding noise and TDRMIX is zero."""
    import cases

    c = cases.make_case("h2_kernels", n=12, seed=4)
    off = _oracle_rhs(c)
    on = _oracle_rhs(c, **sw)
    assert _field_rel(on, off) <= 1e-13


def test_dufour_changes_only_the_energy_equation():
    import cases

    c = cases.make_case("h2_pool", n=12, seed=6)
    off = _oracle_rhs(c)
    on = _oracle_rhs(c, dufour=True)
    assert np.array_equal(on[:4], off[:4]) and np.array_equal(on[5:], off[5:])
    assert rel_linf(on[4], off[4]) > 1e-6


@pytest.mark.parametrize("sw", SWITCHES, ids=["mixw", "mixp", "soret", "dufour", "all"])
def test_branches_are_active_and_keep_species_sum_equal_to_continuity(sw):
    import cases

    c = cases.make_case("h2_pool", n=12, seed=6)
    off = _oracle_rhs(c)
    on = _oracle_rhs(c, **sw)
    assert _field_rel(on, off) > 1e-6
    assert rel_linf(on[5:].sum(axis=0), on[0]) <= 1e-12


def test_switches_need_mixture_averaged_transport():
    import cases
    from oracle import Oracle

    c = cases.make_case("ignition32", n=12, seed=3)
    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    with pytest.raises(RuntimeError):
        o.set_transport(mixw=True)


# ------------------------------------------------------------------ GPU
def _pair(c, sw):
    import senga
    from oracle import Oracle

    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    if "bc" in c:
        box.set_nscbc(c["bc"])
        ref.set_bc(c["bc"])
    box.set_transport(**sw)
    ref.set_transport(**sw)
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    return box, ref


@pytest.mark.gpu
@pytest.mark.parametrize("sw", SWITCHES, ids=["mixw", "mixp", "soret", "dufour", "all"])
def test_gpu_transport_rhs_matches_oracle(sw):
    import cases

    c = cases.make_case("h2_pool", n=16, seed=31)
    box, ref = _pair(c, sw)
    r, _, _ = box.rhs()
    rr, _, _ = ref.rhs()
    for fl in range(r.shape[0]):
        assert rel_linf(r[fl], rr[fl]) <= 1e-10, fl


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["h2_pool", "flame_inout"])
def test_gpu_transport_steps_match_oracle(case):
    import cases

    c = cases.make_case(case, n=16, seed=32)
    box, ref = _pair(c, ALL)
    box.step(3)
    ref.step(3)
    f, t, _ = box.download()
    fr, tr, _ = ref.download()
    for fl in range(f.shape[0]):
        assert rel_linf(f[fl], fr[fl]) <= 1e-10, fl
    assert rel_linf(t, tr) <= 1e-10


@pytest.mark.gpu
def test_gpu_transport_switch_off_restores_the_plain_path():
    import cases
    import senga

    c = cases.make_case("h2_pool", n=16, seed=33)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    plain, _, _ = box.rhs()
    box.set_transport(**ALL)
    box.upload(c["fields"], c["T"], c["itn"])
    on, _, _ = box.rhs()
    assert _field_rel(on, plain) > 1e-6
    box.set_transport()
    box.upload(c["fields"], c["T"], c["itn"])
    again, _, _ = box.rhs()
    assert np.array_equal(again, plain)
    chem1 = senga.Chem(cases.CHEM_1STEP)
    c1 = cases.make_case("ignition32", n=12, seed=3)
    b1 = senga.Box(c1["shape"], c1["lengths"], chem1, senga.Diff(None, chem1), c1["dt"])
    with pytest.raises(senga.SengaError):
        b1.set_transport(mixw=True)
