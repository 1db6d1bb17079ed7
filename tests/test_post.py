"""Post-processing record (src/output.f:240-265): DRUN, URUN/DRUN, VRUN/DRUN,
WRUN/DRUN, ERUN/DRUN, TRUN, PRUN, YRUN/DRUN (NSPEC), RRTE (NSPCMX), ETIME in
one unformatted record; RRTE is the CHRATE rate kept by RHSCAL
(src/rhscal.f:828), TRUN/PRUN those of the fifth substage's TEMPER.

CPU: writer/reader round trip and the record layout byte by byte. GPU: the
fields after two steps against the oracle (field-normalised relative
L-infinity 1e-10)."""
import struct

import numpy as np
import pytest

from conftest import rel_linf


def test_post_record_layout_and_round_trip(tmp_path):
    import senga

    rng = np.random.default_rng(3)
    nx, ny, nz, nspec, nspcmx = 5, 4, 3, 2, 9
    post = rng.standard_normal((7 + 2 * nspec, nz, ny, nx))
    p = tmp_path / senga.post_name(12, 3)
    assert p.name == "out000120003.res"
    senga.post_write(str(p), post, etime=1.25e-3, nspcmx=nspcmx)
    raw = p.read_bytes()
    n = nx * ny * nz
    body = ((7 + nspec + nspcmx) * n + 1) * 8
    assert len(raw) == body + 8
    assert struct.unpack("<i", raw[:4])[0] == body and struct.unpack("<i", raw[-4:])[0] == body
    vals = np.frombuffer(raw[4:-4], dtype="<f8")
    assert np.array_equal(vals[:(7 + 2 * nspec) * n], post.reshape(-1))
    assert np.all(vals[(7 + 2 * nspec) * n:(7 + nspec + nspcmx) * n] == 0.0)  # RRTE slots past NSPEC
    assert vals[-1] == 1.25e-3
    back, et = senga.post_read(str(p), (nx, ny, nz), nspec, nspcmx=nspcmx)
    assert np.array_equal(back, post) and et == 1.25e-3
    with pytest.raises(senga.SengaError):
        senga.post_read(str(p), (nx, ny, nz), nspec)  # wrong NSPCMX: size mismatch


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["h2_kernels", "flame_inout"])
def test_gpu_post_fields_match_oracle(case):
    import cases
    import senga
    from oracle import Oracle

    c = cases.make_case(case, n=16, seed=41)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    if "bc" in c:
        box.set_nscbc(c["bc"])
        ref.set_bc(c["bc"])
    with pytest.raises(senga.SengaError):
        box.post_fields()  # RRTE not kept
    box.keep_rates()
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(2)
    ref.step(2)
    got = box.post_fields()
    want = ref.post()
    for fl in range(got.shape[0]):
        if np.max(np.abs(want[fl])) == 0.0:
            assert np.max(np.abs(got[fl])) <= 1e-300, fl
        else:
            assert rel_linf(got[fl], want[fl]) <= 1e-10, fl
    assert np.max(np.abs(got[7 + 9])) > 0.0  # the H2 rate
