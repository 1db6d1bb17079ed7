"""The no-slip walls on the x faces.

W1 (NSBCW1, adiabatic): flags and integration ranges bcinit.f:702-735; wall
state boundt.f:243-356 (x-left), 657-768 (x-right) and bountt.f:290-428,
767-; wave amplitudes bounds.f:917-1056, 1833-1974; wall flux terms
rhscal.f:610-660 (FxxCNW) and 1698-1760 (FxxDFW); zero-gradient mass
fractions lincom.f:171-210, fincom.f:171-210.
W2 (NSBCW2, isothermal): flags and ranges bcinit.f:822-855; the wall
temperature RXxPRM(1) imposed by boundt.f:358-470 and bountt.f:429-560 (and
their x-right blocks); the same wave amplitudes (bounds.f:1058-1190, 1975-),
wall diffusion flux and zero-gradient mass fractions as W1; neither momentum
nor energy integrated on the wall.

CPU (oracle): the mirror image of the two-wall box (x -> L - x, u -> -u) has
the mirror image of the RHS and of the state after three steps; on the wall
planes the momentum stays zero, the temperature is the fourth-order
zero-gradient extrapolation of the four planes inward (W1) or the imposed
one (W2), every mass fraction the clipped extrapolation of the updated
state, and the energy the internal energy at that temperature, while the
density is integrated. With the transport switches on, the molar-mass,
pressure and Soret branches add their own wall terms (rhscal.f:2116-2175,
2512-2571, 2925-2984): the mirror symmetry still holds, and so does
sum_k YRHS_k = DRHS on every plane, since each wall term enters a species
rate and VTMP alike. GPU: two walls of either kind, a W1 and a W2 wall, and
a wall with an O1 outflow opposite, with the base transport and with the
switches, against the oracle (RHS and three RK steps, field-normalised
relative L-infinity 1e-10)."""
import numpy as np
import pytest

from conftest import rel_linf

TOL = 1e-10


def _mirror(a):
    m = np.ascontiguousarray(a[..., ::-1])
    m[1] = -m[1]
    return m


TWALL = (760.0, 830.0)


def _case(shape=(16, 8, 6), seed=5, kind=31):
    import cases

    c = cases.make_case("wall_box", seed=seed, shape=shape)
    return c, dict(c["bc"], xl=kind, xr=kind, t_wall=TWALL)


def _mirrored(c, bc):
    cm = dict(c, fields=_mirror(c["fields"]), T=np.ascontiguousarray(c["T"][..., ::-1]),
              itn=np.ascontiguousarray(c["itn"][..., ::-1]))
    tw = bc.get("t_wall", (0.0, 0.0))
    return cm, dict(bc, xl=bc["xr"], xr=bc["xl"], t_wall=(tw[1], tw[0]))


def _oracle(c, bc):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    o.upload(c["fields"], c["T"], c["itn"])
    return o


@pytest.mark.parametrize("kind", [31, 32], ids=["W1", "W2"])
def test_wall_mirror_symmetry_in_the_oracle(kind):
    c, bc = _case(kind=kind)
    cm, bcm = _mirrored(c, bc)
    ra, ta, _ = _oracle(c, bc).rhs()
    rb, tb, _ = _oracle(cm, bcm).rhs()
    assert rel_linf(tb, ta[..., ::-1]) <= 1e-12
    for fl in range(ra.shape[0]):
        assert rel_linf(rb[fl], _mirror(ra)[fl]) <= 1e-12, fl
    a = _oracle(c, bc)
    a.step(3)
    b = _oracle(cm, bcm)
    b.step(3)
    fa, _, _ = a.download()
    fb, _, _ = b.download()
    for fl in range(fa.shape[0]):
        assert rel_linf(fb[fl], _mirror(fa)[fl]) <= 1e-12, fl


@pytest.mark.parametrize("kind", [31, 32], ids=["W1", "W2"])
def test_wall_planes_after_steps(kind):
    import cases
    from oracle import OracleChem

    c, bc = _case(kind=kind)
    o = _oracle(c, bc)
    r, _, _ = o.rhs()
    for fl in (1, 2, 3, 4):  # BOUNDS: momentum and energy RHS vanish on the walls
        assert np.max(np.abs(r[fl][..., 0])) == 0.0 and np.max(np.abs(r[fl][..., -1])) == 0.0
    o = _oracle(c, bc)
    o.step(3)
    f, t, itn = o.download()
    chem = OracleChem(c["chem"])
    rg = chem.table("rgspec")
    for w, st in ((0, 1), (-1, -1)):
        d = f[0][..., w]
        assert np.max(np.abs(d - c["fields"][0][..., w])) > 0.0  # the density is integrated
        for fl in (1, 2, 3):
            assert np.max(np.abs(f[fl][..., w])) == 0.0
        if kind == 31:
            tt = [t[..., w + k * st] for k in range(1, 5)]
            tw = (48.0 * tt[0] - 36.0 * tt[1] + 16.0 * tt[2] - 3.0 * tt[3]) / 25.0
            assert np.array_equal(t[..., w], tw)
        else:  # TRUN keeps TEMPER's value, converged onto the imposed temperature
            tw = np.full_like(d, TWALL[0 if w == 0 else 1])
            assert np.allclose(t[..., w], tw, rtol=0, atol=1e-6)
        y = f[5:] / f[0]
        yy = [y[:, ..., w + k * st] for k in range(1, 5)]
        yw = np.float32(12.0 / 25.0).astype(np.float64) * (
            4.0 * yy[0] - 3.0 * yy[1] + np.float32(4.0 / 3.0).astype(np.float64) * yy[2] - 0.25 * yy[3])
        yw = np.clip(yw, 0.0, 1.0)
        assert np.allclose(f[5:][..., w], d * yw, rtol=1e-14, atol=1e-300)
        assert np.array_equal(itn[..., w], cases.interval_index(chem, tw))
        e = np.zeros_like(d)
        for s in range(chem.nspec):
            e = e + (cases.species_enthalpy(chem, s, tw, itn[..., w]) - rg[s] * tw) * f[5 + s][..., w]
        assert rel_linf(f[4][..., w], e) <= 1e-13


ALL = dict(mixw=True, mixp=True, soret=True, dufour=True)
SWITCHES = [("mixw", dict(mixw=True)), ("mixp", dict(mixp=True)), ("soret", dict(soret=True)), ("all", ALL)]


def _oracle_sw(c, bc, sw):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    o.set_transport(**sw)
    o.upload(c["fields"], c["T"], c["itn"])
    return o


OCASES = [(31, "mixw", dict(mixw=True)), (31, "mixp", dict(mixp=True)), (31, "soret", dict(soret=True)),
          (32, "all", ALL)]


@pytest.mark.parametrize("kind,name,sw", OCASES, ids=[f"W{k - 30}-{n}" for k, n, _ in OCASES])
def test_wall_branch_terms_mirror_and_species_sum_in_the_oracle(kind, name, sw):
    c, bc = _case(kind=kind)
    cm, bcm = _mirrored(c, bc)
    ra, _, _ = _oracle_sw(c, bc, sw).rhs()
    rb, _, _ = _oracle_sw(cm, bcm, sw).rhs()
    for fl in range(ra.shape[0]):
        assert rel_linf(rb[fl], _mirror(ra)[fl]) <= 1e-12, fl
    # every wall term enters one species rate and VTMP alike
    assert rel_linf(ra[5:].sum(axis=0), ra[0]) <= 1e-10
    # the switches change the wall plane's species right-hand side
    r0, _, _ = _oracle(c, bc).rhs()
    assert rel_linf(ra[5:, ..., 0], r0[5:, ..., 0]) > 1e-8


O1 = dict(p_inf=101325.0, sigma=0.287, eta=1.0e-3)
CASES = [("W1-W1", dict(xl=31, xr=31)), ("W1-O1", dict(xl=31, xr=21, **O1)), ("W2-W2", dict(xl=32, xr=32)),
         ("W2-W1", dict(xl=32, xr=31)), ("W2-O1", dict(xl=32, xr=21, **O1))]


@pytest.mark.gpu
@pytest.mark.parametrize("name,faces", CASES, ids=[n for n, _ in CASES])
@pytest.mark.parametrize("mirrored", [False, True], ids=["as-is", "mirrored"])
def test_gpu_walls_match_oracle(name, faces, mirrored):
    import senga

    c, bc = _case(shape=(24, 10, 8), seed=9)
    bc = dict(bc, **faces)
    if mirrored:
        c, bc = _mirrored(c, bc)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.set_nscbc(bc)
    box.upload(c["fields"], c["T"], c["itn"])
    ref = _oracle(c, bc)
    r, t, _ = box.rhs()
    rr, tr, _ = ref.rhs()
    assert rel_linf(t, tr) <= TOL
    for fl in range(rr.shape[0]):
        assert rel_linf(r[fl], rr[fl]) <= TOL, f"RHS field {fl}"
    box.upload(c["fields"], c["T"], c["itn"])
    ref = _oracle(c, bc)
    box.step(3)
    ref.step(3)
    g, tg, ig = box.download()
    o, to, io = ref.download()
    assert box.status() == 0
    for fl in range(o.shape[0]):
        assert rel_linf(g[fl], o[fl]) <= TOL, f"state field {fl}"
    assert rel_linf(tg, to) <= TOL
    assert np.array_equal(ig, io)


@pytest.mark.gpu
def test_gpu_wall_refusals():
    """A W2 face without its temperature is refused by the library."""
    import senga

    c, bc = _case(shape=(16, 8, 6), kind=32)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    with pytest.raises(RuntimeError, match="t_wall"):
        box.set_nscbc(dict(bc, t_wall=(0.0, 800.0)))
    box.set_nscbc(bc)
    box.set_transport(mixw=True)  # walls run with the transport switches too


WCASES = [("W1-W1", dict(xl=31, xr=31)), ("W2-O1", dict(xl=32, xr=21, **O1))]


@pytest.mark.gpu
@pytest.mark.parametrize("name,faces", WCASES, ids=[n for n, _ in WCASES])
@pytest.mark.parametrize("sname,sw", SWITCHES, ids=[n for n, _ in SWITCHES])
@pytest.mark.parametrize("mirrored", [False, True], ids=["as-is", "mirrored"])
def test_gpu_walls_with_transport_switches_match_oracle(name, faces, sname, sw, mirrored):
    import senga

    c, bc = _case(shape=(24, 10, 8), seed=9)
    bc = dict(bc, **faces)
    if mirrored:
        c, bc = _mirrored(c, bc)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.set_nscbc(bc)
    box.set_transport(**sw)
    box.upload(c["fields"], c["T"], c["itn"])
    r, t, _ = box.rhs()
    rr, tr, _ = _oracle_sw(c, bc, sw).rhs()
    assert rel_linf(t, tr) <= TOL
    for fl in range(rr.shape[0]):
        assert rel_linf(r[fl], rr[fl]) <= TOL, f"RHS field {fl}"
    box.upload(c["fields"], c["T"], c["itn"])
    ref = _oracle_sw(c, bc, sw)
    box.step(3)
    ref.step(3)
    g, tg, ig = box.download()
    o, to, io = ref.download()
    assert box.status() == 0
    for fl in range(o.shape[0]):
        assert rel_linf(g[fl], o[fl]) <= TOL, f"state field {fl}"
    assert rel_linf(tg, to) <= TOL
    assert np.array_equal(ig, io)
