"""Bounded x direction with NSCBC faces (I3 inflow at x-left, O1 outflow at
x-right; y, z periodic) on the GPU against the oracle, through the C ABI.

Tolerances as in test_gpu_parity: field-normalised relative L-infinity 1e-10
for the RHS and the state after N steps, 1e-12 for derivative operators."""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-10
TOL_DERIV = 1e-12


def _flame(n=16, seed=5):
    import cases

    return cases.make_case("flame_inout", n=n, seed=seed)


def _pair(c):
    import senga
    from oracle import Oracle

    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.set_nscbc(c["bc"])
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    ref.set_bc(c["bc"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    return box, ref


@pytest.mark.parametrize("kind", range(9))
def test_derivatives_with_bounded_x(kind):
    """All nine operators with x bounded: one-sided first/second closures
    and the mixed-derivative x-edge closures (xy, xz)."""
    import cases
    import senga
    from oracle import Oracle

    rng = np.random.default_rng(40 + kind)
    nx, ny, nz = 24, 20, 16
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f = (np.sin(0.3 * x) * np.cos(4 * np.pi * y / ny) + np.sin(2 * np.pi * z / nz) * x / nx +
         1e-3 * rng.standard_normal((nz, ny, nx)))
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    lengths = (3.1e-3, 2.3e-3, 1.7e-3)
    nend = (1, 1, 2, 2, 2, 2)
    box = senga.Box((nx, ny, nz), lengths, chem, diff, 1e-8, nend=nend)
    ref = Oracle((nx, ny, nz), lengths, cases.CHEM_1STEP, None, 1e-8, nend=nend)
    assert rel_linf(box.deriv(kind, f), ref.deriv(kind, f)) <= TOL_DERIV


def test_flame_rhs_matches_oracle():
    """RHS of the NSCBC flame box (BOUNDT, RHSCAL, RHSVEL, BOUNDS)."""
    box, ref = _pair(_flame())
    r_g, t_g, p_g = box.rhs()
    r_o, t_o, p_o = ref.rhs()
    assert rel_linf(t_g, t_o) <= TOL_STATE
    assert rel_linf(p_g, p_o) <= TOL_STATE
    for k in range(r_o.shape[0]):
        assert rel_linf(r_g[k], r_o[k]) <= TOL_STATE, f"field {k}"


def test_flame_steps_match_oracle():
    """Three RK steps incl. BOUNTT; the face planes are where the RK epilogue
    differs from the interior (correction added, inflow plane imposed)."""
    box, ref = _pair(_flame(n=16, seed=6))
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"
        assert rel_linf(g[k][..., 0], o[k][..., 0]) <= TOL_STATE, f"inflow plane field {k}"
        assert rel_linf(g[k][..., -1], o[k][..., -1]) <= TOL_STATE, f"outflow plane field {k}"
    assert rel_linf(tg, to) <= TOL_STATE


def test_flame_filter_and_graph():
    """Explicit filter with the one-sided rows on the bounded faces, then
    steps through the CUDA graph (bitwise equal to the stepped path)."""
    import senga

    c = _flame(n=16, seed=7)
    box, ref = _pair(c)
    box.step(1)
    ref.step(1)
    box.filter(1)
    ref.filter(1)
    box.step(2, graph=True)
    ref.step(2)
    g, _, _ = box.download()
    o, _, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    a = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    a.set_nscbc(c["bc"])
    a.upload(c["fields"], c["T"], c["itn"])
    b = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    b.set_nscbc(c["bc"])
    b.upload(c["fields"], c["T"], c["itn"])
    a.step(2)
    b.step(2, graph=True)
    fa, _, _ = a.download()
    fb, _, _ = b.download()
    assert np.array_equal(fa, fb)


def test_bounded_box_needs_face_conditions():
    import senga

    c = _flame()
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.upload(c["fields"], c["T"], c["itn"])
    with pytest.raises(senga.SengaError, match="status 5"):
        box.step(1)
