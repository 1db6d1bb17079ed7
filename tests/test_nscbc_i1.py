"""The I1 inflow (NSBCI1, subsonic non-reflecting laminar inflow: flags
src/bcinit.f:396-407; wave amplitudes src/bounds.f:387-520 x-left,
1465-1598 x-right) with an O1 outflow on the other x face. Nothing is
imposed on the inflow plane: the incoming wave carries only the chemistry
source (COBCxx is set by BCINIT for O1 faces alone, so it is zero here) and
every conserved field is integrated there.

CPU (oracle): the mirror image of the I1/O1 flame (x -> L - x, u -> -u) has
the mirror image of the RHS and of the state after three steps, and every
field of the inflow plane evolves. GPU: both pairings against the oracle (RHS
and three RK steps, field-normalised relative L-infinity 1e-10)."""
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
    return c, dict(c["bc"], xl=11)


def _mirrored(c, bc):
    cm = dict(c, fields=_mirror(c["fields"]), T=np.ascontiguousarray(c["T"][..., ::-1]),
              itn=np.ascontiguousarray(c["itn"][..., ::-1]))
    return cm, dict(bc, xl=21, xr=11)


def _oracle(c, bc):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    o.upload(c["fields"], c["T"], c["itn"])
    return o


def test_i1_mirror_symmetry_in_the_oracle():
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


def test_i1_inflow_plane_is_integrated():
    c, bc = _case()
    o = _oracle(c, bc)
    o.step(3)
    f, _, _ = o.download()
    for fl in range(f.shape[0]):  # nothing is held: every field of the plane moves
        assert np.max(np.abs(f[fl][..., 0] - c["fields"][fl][..., 0])) > 0.0, fl


@pytest.mark.gpu
@pytest.mark.parametrize("mirrored", [False, True], ids=["I1-left", "I1-right"])
def test_gpu_i1_flame_matches_oracle(mirrored):
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
