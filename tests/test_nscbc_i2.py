"""The I2 inflow (NSBCI2, subsonic reflecting inflow with specified
temperature: src/bounds.f:522-608 x-left, 1600-1684 x-right; boundt.f:81-176,
495-; bountt.f:84-200, 590-; integration ranges bcinit.f:458-480) with an O1
outflow on the other x face.

CPU (oracle): the mirror image of the I2/O1 flame (x -> L - x, u -> -u) has
the mirror image of the RHS and of the state after three steps; the inflow
plane keeps T = TRIN, u = u_in and the inflow mass fractions while its
density evolves. GPU: both pairings against the oracle (RHS and three RK
steps, field-normalised relative L-infinity 1e-10)."""
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

    c = cases.make_case("flame_inout", seed=seed, shape=shape)
    bc = dict(c["bc"], xl=12, t_in=300.0)
    return c, bc


def _mirrored(c, bc):
    cm = dict(c, fields=_mirror(c["fields"]), T=np.ascontiguousarray(c["T"][..., ::-1]),
              itn=np.ascontiguousarray(c["itn"][..., ::-1]))
    return cm, dict(bc, xl=21, xr=12, u_in=-bc["u_in"])


def _oracle(c, bc):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    o.upload(c["fields"], c["T"], c["itn"])
    return o


def test_i2_mirror_symmetry_in_the_oracle():
    c, bc = _case()
    cm, bcm = _mirrored(c, bc)
    ra, _, _ = _oracle(c, bc).rhs()
    rb, _, _ = _oracle(cm, bcm).rhs()
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


def test_i2_inflow_plane_keeps_its_imposed_state():
    c, bc = _case()
    o = _oracle(c, bc)
    o.step(3)
    f, t, _ = o.download()
    d = f[0][..., 0]
    assert np.allclose(t[..., 0], bc["t_in"], rtol=0, atol=1e-8)
    assert np.allclose(f[1][..., 0] / d, bc["u_in"], rtol=1e-14)
    assert np.max(np.abs(f[2][..., 0])) == 0.0 and np.max(np.abs(f[3][..., 0])) == 0.0
    for s in range(9):
        assert np.allclose(f[5 + s][..., 0] / d, bc["y_in"][s], rtol=1e-13, atol=1e-16)
    assert np.max(np.abs(d - c["fields"][0][..., 0])) > 0.0  # the density is integrated


@pytest.mark.gpu
@pytest.mark.parametrize("mirrored", [False, True], ids=["I2-left", "I2-right"])
def test_gpu_i2_flame_matches_oracle(mirrored):
    import senga

    c, bc = _case(shape=(24, 10, 8), seed=9)
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
