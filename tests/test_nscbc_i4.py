"""The I4 inflow (NSBCI4, after Lodato et al.: flags src/bcinit.f:653-658;
wave amplitudes src/bounds.f:686-845, coded for the x-left face only) with an
O1 outflow at x-right. Nothing is imposed: the waves L2..L5 and LY are
relaxed towards the targets u_in, v = w = 0, t_in, y_in with the
coefficients NRIETA2..6 over XGDLEN, plus the transverse terms TT2..TT6.

CPU (oracle): the face correction is affine in the coefficients (R(a) +
R(b) - R(0) = R(a + b) on the inflow plane, the rest of the box unchanged),
and an I4 face on x-right is refused, as the reference codes it for x-left
only. GPU: RHS and three RK steps against the oracle for two coefficient
sets (field-normalised relative L-infinity 1e-10), and the same refusal."""
import numpy as np
import pytest

from conftest import rel_linf

TOL = 1e-10
NRI = [(0.0, 0.5, 0.3, 0.3, 0.8, 0.5), (0.0, 2.0, 0.0, 1.0, 0.25, 3.0)]


def _case(shape=(16, 8, 6), seed=5, nri=NRI[0]):
    import cases

    c = cases.make_case("flame_inout", seed=seed, shape=shape)
    return c, dict(c["bc"], xl=14, t_in=300.0, nrieta=nri)


def _oracle(c, bc):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    o.set_bc(bc)
    o.upload(c["fields"], c["T"], c["itn"])
    return o


def test_i4_correction_is_affine_in_the_coefficients():
    c, bc = _case()
    a = np.array(NRI[0])
    b = np.array(NRI[1])
    r = {}
    for key, nri in (("0", np.zeros(6)), ("a", a), ("b", b), ("ab", a + b)):
        r[key], _, _ = _oracle(c, dict(bc, nrieta=tuple(nri))).rhs()
    for fl in range(r["0"].shape[0]):
        lhs = r["a"][fl] + r["b"][fl] - r["0"][fl]
        assert rel_linf(lhs, r["ab"][fl]) <= 1e-11, fl
        # only the inflow plane depends on the coefficients
        assert np.array_equal(r["a"][fl][..., 1:], r["0"][fl][..., 1:]), fl
    assert np.max(np.abs(r["a"][0][..., 0] - r["0"][0][..., 0])) > 0.0


def test_i4_on_x_right_is_refused():
    c, bc = _case()
    with pytest.raises(RuntimeError, match="x-left"):
        _oracle(c, dict(bc, xl=21, xr=14))


@pytest.mark.gpu
@pytest.mark.parametrize("nri", NRI, ids=["eta-a", "eta-b"])
def test_gpu_i4_flame_matches_oracle(nri):
    import senga

    c, bc = _case(shape=(24, 10, 8), seed=9, nri=nri)
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
def test_gpu_i4_on_x_right_is_refused():
    import senga

    c, bc = _case(shape=(16, 8, 6))
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    with pytest.raises(RuntimeError, match="x-left"):
        box.set_nscbc(dict(bc, xl=21, xr=14))
