"""One box split along z over several contexts (senga_zgroup_*),
the stencils reading each tile's z halo from the slab that owns it, against
the same box as one context: the arithmetic per point is the same, so the
states after two steps agree to rounding (1e-13 field-normalised). Slabs
thinner than the five-plane halo (4 planes) make a tile's halo span two
other slabs. Runs all slabs on one GPU; the peer-access path between GPUs
is the same code with the slabs' pools on different devices."""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,shape,nslabs", [
    ("h2_kernels", (16, 16, 16), 2),
    ("h2_kernels", (16, 16, 16), 4),
    ("ignition32", (24, 16, 12), 3),
    ("h2_pool", (20, 12, 18), 6),
])
def test_zsplit_box_matches_one_box(name, shape, nslabs):
    import cases
    import senga

    c = cases.make_case(name, n=shape[0], seed=71) if name != "h2_pool" else cases.make_case(name, seed=71, shape=shape)
    if c["shape"] != shape:  # cubic generators: regenerate on the wanted grid by slicing a larger cube
        nx, ny, nz = shape
        c = dict(c)
        c["fields"] = np.ascontiguousarray(c["fields"][:, :nz, :ny, :nx])
        c["T"] = np.ascontiguousarray(c["T"][:nz, :ny, :nx])
        c["itn"] = np.ascontiguousarray(c["itn"][:nz, :ny, :nx])
        c["shape"] = shape
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    one = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    one.upload(c["fields"], c["T"], c["itn"])
    one.step(2)
    want, tw, _ = one.download()
    grp = senga.ZGroup(c["shape"], c["lengths"], chem, diff, c["dt"], nslabs)
    grp.upload(c["fields"], c["T"], c["itn"])
    grp.step(2)
    got, tg, _ = grp.download()
    grp.close()
    for fl in range(got.shape[0]):
        if np.max(np.abs(want[fl])) == 0.0:
            assert np.max(np.abs(got[fl])) == 0.0, fl
        else:
            assert rel_linf(got[fl], want[fl]) <= 1e-13, fl
    assert rel_linf(tg, tw) <= 1e-13


@pytest.mark.parametrize("name,shape,nslabs", [
    ("flame_inout", (24, 8, 16), 2),   # I3 inflow at x-left, O1 outflow at x-right
    ("flame_inout", (24, 8, 16), 4),
    ("wall_box", (16, 16, 16), 2),     # W1 walls on both x faces
])
def test_zsplit_nscbc_box_matches_one_box(name, shape, nslabs):
    """NSCBC x faces on a z-split box: every slab holds its part of both
    faces (BOUNDT, the face data and BOUNDS, the wall flux and wall fix per
    slab), the stencils read z halos across slabs; two steps against the
    same box as one context."""
    import cases
    import senga

    c = cases.make_case(name, seed=29, shape=shape) if name == "flame_inout" else cases.make_case(name, n=shape[0])
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    one = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    one.set_nscbc(c["bc"])
    one.upload(c["fields"], c["T"], c["itn"])
    one.step(2)
    want, tw, _ = one.download()
    assert one.status() == 0
    grp = senga.ZGroup(c["shape"], c["lengths"], chem, diff, c["dt"], nslabs, nend=c["nend"])
    grp.set_nscbc(c["bc"])
    grp.upload(c["fields"], c["T"], c["itn"])
    grp.step(2)
    got, tg, _ = grp.download()
    grp.close()
    for fl in range(got.shape[0]):
        if np.max(np.abs(want[fl])) == 0.0:
            assert np.max(np.abs(got[fl])) == 0.0, fl
        else:
            assert rel_linf(got[fl], want[fl]) <= 1e-13, fl
    assert rel_linf(tg, tw) <= 1e-13


def test_zsplit_rejects_what_it_does_not_support():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    with pytest.raises(senga.SengaError):
        senga.ZGroup((16, 16, 15), (1e-3,) * 3, chem, diff, 1e-8, 2)  # 15 planes into 2 slabs
    with pytest.raises(senga.SengaError):
        senga.ZGroup((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, 17)
    with pytest.raises(senga.SengaError):  # y bounded
        senga.ZGroup((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, 2, nend=(2, 2, 1, 1, 2, 2))
    with pytest.raises(senga.SengaError):  # x bounded on one face only
        senga.ZGroup((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, 2, nend=(1, 2, 2, 2, 2, 2))
    grp = senga.ZGroup((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, 2, nend=(1, 1, 2, 2, 2, 2))
    with pytest.raises(senga.SengaError):  # bounded x without its face conditions
        grp.step(1)
    grp.close()
