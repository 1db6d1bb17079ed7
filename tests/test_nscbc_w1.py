"""The W1 wall (NSBCW1, adiabatic no-slip): flags and integration ranges
bcinit.f:702-735; wall state boundt.f:243-356 (x-left), 657-768 (x-right)
and bountt.f:290-428, 767-; wave amplitudes bounds.f:917-1056, 1833-1974;
wall flux terms rhscal.f:610-660 (FxxCNW) and 1698-1760 (FxxDFW); zero-
gradient mass fractions lincom.f:171-210, fincom.f:171-210.

CPU (oracle): the mirror image of the two-wall box (x -> L - x, u -> -u) has
the mirror image of the RHS and of the state after three steps; on the wall
planes the momentum stays zero, the temperature is the fourth-order
zero-gradient extrapolation of the four planes inward, every mass fraction
the clipped extrapolation of the updated state, and the energy the
internal energy at that temperature, while the density is integrated. The
molar-mass, pressure and thermal-diffusion branches have wall terms of
their own that are not restated, so both sides refuse them with a wall.
GPU: two walls, and a wall with an O1 outflow opposite, against the oracle
(RHS and three RK steps, field-normalised relative L-infinity 1e-10)."""
import numpy as np
import pytest

from conftest import rel_linf

TOL = 1e-10


def _mirror(a):
    m = np.ascontiguousarray(a[..., ::-1])
    m[1] = -m[1]
    return m


def _case(shape=(16, 8, 6), seed=5):
    import cases

    c = cases.make_case("wall_box", seed=seed, shape=shape)
    return c, dict(c["bc"])


def _mirrored(c, bc):
    cm = dict(c, fields=_mirror(c["fields"]), T=np.ascontiguousarray(c["T"][..., ::-1]),
              itn=np.ascontiguousarray(c["itn"][..., ::-1]))
    return cm, dict(bc, xl=bc["xr"], xr=bc["xl"])


def _oracle(c, bc):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    o.upload(c["fields"], c["T"], c["itn"])
    return o


def test_w1_mirror_symmetry_in_the_oracle():
    c, bc = _case()
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


def test_w1_wall_planes_after_steps():
    import cases
    from oracle import OracleChem

    c, bc = _case()
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
        tt = [t[..., w + k * st] for k in range(1, 5)]
        tw = (48.0 * tt[0] - 36.0 * tt[1] + 16.0 * tt[2] - 3.0 * tt[3]) / 25.0
        assert np.array_equal(t[..., w], tw)
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


def test_w1_refuses_the_transport_branches_without_restated_wall_terms():
    from oracle import Oracle

    c, bc = _case()
    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    with pytest.raises(RuntimeError, match="W1"):
        o.set_transport(mixw=True)
    o2 = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o2.set_transport(soret=True)
    with pytest.raises(RuntimeError, match="W1"):
        o2.set_bc(bc)


CASES = [("walls", dict(xl=31, xr=31)), ("wall-outflow", dict(xl=31, xr=21, p_inf=101325.0, sigma=0.287,
                                                                      eta=1.0e-3))]


@pytest.mark.gpu
@pytest.mark.parametrize("name,faces", CASES, ids=[n for n, _ in CASES])
@pytest.mark.parametrize("mirrored", [False, True], ids=["as-is", "mirrored"])
def test_gpu_w1_matches_oracle(name, faces, mirrored):
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
