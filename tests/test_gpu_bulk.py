"""The three ways of filling the stencil tiles of an all-periodic box of
even nx against the oracle: per-element cp.async (SENGA_STAGE=cpasync), rows
copied by the TMA engine (bulk), one tensor copy per buffer on tiles away
from the wrap (tma); the library reads SENGA_STAGE at every launch, and by
default fills flow's tiles by rows and the species kernels' by cp.async.

Each staged row spans the tile's x range plus six points on either side; in a
periodic box it is cut where x wraps, and a box narrower than one row wraps
several times, so these shapes exercise rows of one, two and many pieces,
partial tiles in every direction, and the hydrogen and one-step mechanisms.
The status word must stay clear (bit 3 would mean a copy did not complete in
time). Bounds as in the other parity tests: field-normalised relative
L-infinity 1e-10 for the RHS and the state after two steps."""
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-10

CASES = [("h2_pool", (10, 12, 8)), ("h2_pool", (34, 9, 7)), ("h2_pool", (46, 12, 6)), ("h2_pool", (2, 14, 10)),
         ("h2_pool", (96, 40, 6)), ("ignition32", None)]


@pytest.mark.parametrize("mode", ["cpasync", "bulk", "tma"])
@pytest.mark.parametrize("name,shape", CASES, ids=[f"{n}-{'x'.join(map(str, s)) if s else '20^3'}" for n, s in CASES])
def test_bulk_staged_tiles_match_oracle(name, shape, mode, monkeypatch):
    monkeypatch.setenv("SENGA_STAGE", mode)
    import cases
    import senga
    from oracle import Oracle

    c = cases.make_case(name, seed=71, shape=shape) if shape else cases.make_case(name, n=20, seed=71)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    r, t, _ = box.rhs()
    rr, tr, _ = ref.rhs()
    assert box.status() == 0
    assert rel_linf(t, tr) <= TOL
    for k in range(rr.shape[0]):
        assert rel_linf(r[k], rr[k]) <= TOL, f"RHS field {k}"
    # rhs() leaves R(U) in the U register: start the steps from the state
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(2, graph=True)
    ref.step(2)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    assert box.status() == 0
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL, f"state field {k}"
    assert rel_linf(tg, to) <= TOL


ZCASES = [("h2_pool", (96, 40, 70)), ("h2_pool", (10, 12, 8)), ("h2_pool", (46, 20, 33)), ("ignition32", None)]


@pytest.mark.parametrize("name,shape", ZCASES, ids=[f"{n}-{'x'.join(map(str, s)) if s else '20^3'}" for n, s in ZCASES])
def test_z_marching_species_rk_matches_oracle(name, shape, monkeypatch):
    """The species + RK update marching along z (SENGA_SPECRK=z): chunks of
    32 planes with a partial last one, columns away from and at the wrap,
    the RHS-only and RK forms."""
    monkeypatch.setenv("SENGA_SPECRK", "z")
    import cases
    import senga
    from oracle import Oracle

    c = cases.make_case(name, seed=73, shape=shape) if shape else cases.make_case(name, n=20, seed=73)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    r, _, _ = box.rhs()
    rr, _, _ = ref.rhs()
    for k in range(rr.shape[0]):
        assert rel_linf(r[k], rr[k]) <= TOL, f"RHS field {k}"
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(2, graph=True)
    ref.step(2)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    assert box.status() == 0
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL, f"state field {k}"
    assert rel_linf(tg, to) <= TOL


FCASES = [("h2_pool", (46, 20, 12)), ("ignition32", None), ("ensemble", None)]


@pytest.mark.parametrize("fuse", ["1", "0"], ids=["fused", "separate"])
@pytest.mark.parametrize("name,shape", FCASES, ids=[f"{n}-{'x'.join(map(str, s)) if s else 'default'}" for n, s in FCASES])
def test_species_kernels_fused_and_separate_match_oracle(name, shape, fuse, monkeypatch):
    """The species kernel and the species+RK kernel as one launch (SENGA_FUSE=1:
    rates, correction velocity, VTMP and energy RHS kept on chip between the
    two passes) and as two (the default):
    RHS-only and RK forms against the oracle. The 48 x 96 x 48 ensemble box
    runs 576 CTAs, so RK passes of some tiles overlap the species passes of
    their neighbours: the species pass must not read U, which those RK passes
    rewrite (it reads the thermochemistry kernel's copy of the momentum)."""
    monkeypatch.setenv("SENGA_FUSE", fuse)
    import cases
    import senga
    from oracle import Oracle

    if name == "ensemble":
        c = cases.make_case(name, seed=21)
    else:
        c = cases.make_case(name, seed=77, shape=shape) if shape else cases.make_case(name, n=20, seed=77)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    assert box.species_fused() == (fuse == "1")
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    r, _, _ = box.rhs()
    rr, _, _ = ref.rhs()
    for k in range(rr.shape[0]):
        assert rel_linf(r[k], rr[k]) <= TOL, f"RHS field {k}"
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(2, graph=True)
    ref.step(2)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    assert box.status() == 0
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL, f"state field {k}"
    assert rel_linf(tg, to) <= TOL
