"""One periodic box split along z over several contexts (senga_zgroup_*),
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


def test_zsplit_rejects_what_it_does_not_support():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    with pytest.raises(senga.SengaError):
        senga.ZGroup((16, 16, 15), (1e-3,) * 3, chem, diff, 1e-8, 2)  # 15 planes into 2 slabs
    with pytest.raises(senga.SengaError):
        senga.ZGroup((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, 17)
