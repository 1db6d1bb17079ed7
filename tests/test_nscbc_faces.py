"""Both built NSCBC kinds on either x face: I3 inflow (13) and O1 outflow (21)
(src/bounds.f:213-372 O1 x-left, 610-675 I3 x-left, 1296-1450 O1 x-right,
1688- I3 x-right; boundt.f/bountt.f for the inflow plane on either side).

CPU (oracle): the mirror image of the inflow/outflow flame (x -> L - x,
u -> -u, inflow through x-right, outflow at x-left) has the mirror image of
its RHS and of its state after a step; a quiescent uniform box between two
O1 faces stays at rest. GPU: the mirrored flame and an outflow-outflow box
against the oracle (field-normalised relative L-infinity 1e-10)."""
import numpy as np
import pytest

from conftest import rel_linf


def _mirror(a, momentum_first=True):
    """x -> L - x of a (nc, nz, ny, nx) state or RHS; the x momentum changes sign."""
    m = np.ascontiguousarray(a[..., ::-1])
    if momentum_first:
        m[1] = -m[1]
    return m


def _flame(n=16, seed=5):
    import cases

    return cases.make_case("flame_inout", seed=seed, shape=(n, 8, 6))


def _oracle(c, bc):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    return o


def test_mirrored_flame_has_the_mirrored_rhs_and_step():
    c = _flame()
    a = _oracle(c, c["bc"])
    a.upload(c["fields"], c["T"], c["itn"])
    ra, _, _ = a.rhs()
    bcm = dict(c["bc"], xl=21, xr=13, u_in=-c["bc"]["u_in"])
    fm, tm, im = _mirror(c["fields"]), np.ascontiguousarray(c["T"][..., ::-1]), np.ascontiguousarray(c["itn"][..., ::-1])
    b = _oracle(c, bcm)
    b.upload(fm, tm, im)
    rb, _, _ = b.rhs()
    want = _mirror(ra)
    for fl in range(ra.shape[0]):
        assert rel_linf(rb[fl], want[fl]) <= 1e-12, fl
    a = _oracle(c, c["bc"])
    a.upload(c["fields"], c["T"], c["itn"])
    a.step(2)
    b = _oracle(c, bcm)
    b.upload(fm, tm, im)
    b.step(2)
    fa, _, _ = a.download()
    fb, _, _ = b.download()
    want = _mirror(fa)
    for fl in range(fa.shape[0]):
        assert rel_linf(fb[fl], want[fl]) <= 1e-12, fl


def test_quiescent_box_between_outflow_faces_stays_at_rest():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_H2)
    shp = (6, 8, 16)
    y = np.zeros((9,) + shp)
    y[1], y[8] = 0.233, 0.767
    z = np.zeros(shp)
    fields, itn = cases.conserved(chem, np.full(shp, 1.0e5), np.full(shp, 300.0), z, z, z, y)
    c = dict(shape=(16, 8, 6), lengths=(1e-2, 5e-3, 4e-3), chem=cases.CHEM_H2, diff=cases.DIFF_H2, dt=1e-8,
             nend=(1, 1, 2, 2, 2, 2))
    bc = dict(xl=21, xr=21, u_in=0.0, rho_in=1.0, y_in=tuple(y[:, 0, 0, 0]), p_inf=1.0e5, sigma=0.287, eta=1.0e-3,
              pio=0, bet_local=0)
    o = _oracle(c, bc)
    o.upload(fields, np.full(shp, 300.0), itn)
    r, _, _ = o.rhs()
    scale = np.abs(fields).max(axis=(1, 2, 3))
    for fl in range(r.shape[0]):
        assert float(np.abs(r[fl]).max()) <= 1e-9 * max(scale[fl], 1.0), fl


@pytest.mark.gpu
@pytest.mark.parametrize("faces", [(21, 13), (21, 21)], ids=["outflow-inflow", "outflow-outflow"])
def test_gpu_faces_match_oracle(faces):
    import senga

    c = _flame(n=24, seed=9)
    xl, xr = faces
    if xr == 13:  # the mirrored flame: inflow through x-right
        f, t, it = _mirror(c["fields"]), np.ascontiguousarray(c["T"][..., ::-1]), np.ascontiguousarray(c["itn"][..., ::-1])
        bc = dict(c["bc"], xl=21, xr=13, u_in=-c["bc"]["u_in"])
    else:
        f, t, it = c["fields"], c["T"], c["itn"]
        bc = dict(c["bc"], xl=21, xr=21)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.set_nscbc(bc)
    ref = _oracle(c, bc)
    box.upload(f, t, it)
    ref.upload(f, t, it)
    r, _, _ = box.rhs()
    rr, _, _ = ref.rhs()
    for fl in range(r.shape[0]):
        assert rel_linf(r[fl], rr[fl]) <= 1e-10, fl
    box.upload(f, t, it)
    ref.upload(f, t, it)
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    w, tw, _ = ref.download()
    for fl in range(g.shape[0]):
        assert rel_linf(g[fl], w[fl]) <= 1e-10, fl
    assert rel_linf(tg, tw) <= 1e-10
