"""Restart dumps in the reference's layouts (src/output.f:296-322 writer,
src/indata.f:1405-1436 reader): round trips of both layouts, the
reference's own 1-step restart input as a parser fixture, and a record
split into sub-records."""
import os
import struct

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _state(nx=6, ny=5, nz=4, nspec=2, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((5 + nspec, nz, ny, nx)) * np.logspace(-3, 5, 5 + nspec)[:, None, None, None]


def test_unformatted_round_trip_with_nspcmx_slots(tmp_path):
    import senga

    f = _state()
    p = str(tmp_path / "dmpi.bin")
    senga.dump_write(p, f, etime=1.5e-4, tstep=2.5e-8, errold=3e-5, errldr=4e-5, nspcmx=9)
    n = f[0].size
    # one record: 4 sizes, D U V W E, YRUN(.., NSPCMX), 4 scalars, markers
    assert os.path.getsize(p) == 4 + 16 + (5 + 9) * n * 8 + 32 + 4
    with open(p, "rb") as fh:
        head = struct.unpack("<i", fh.read(4))[0]
        assert head == 16 + (5 + 9) * n * 8 + 32
        assert struct.unpack("<4i", fh.read(16)) == (6, 5, 4, 2)
    g, sc = senga.dump_read(p, nspcmx=9)
    assert np.array_equal(g, f)
    assert sc == dict(etime=1.5e-4, tstep=2.5e-8, errold=3e-5, errldr=4e-5)


def test_formatted_round_trip_is_exact(tmp_path):
    import senga

    f = _state(seed=1)
    p = str(tmp_path / "dmpi.dat")
    senga.dump_write(p, f, etime=7.0e-5, tstep=1e-9, formatted=True)
    g, sc = senga.dump_read(p, formatted=True)
    assert np.array_equal(g, f)
    assert sc["etime"] == 7.0e-5 and sc["tstep"] == 1e-9


def test_reads_the_reference_casefile_restart_input():
    """src/casefiles/1step/dmpi0000000.dat: 1001 x 1 x 1 points, 2 species;
    the species densities add up to the density."""
    import senga

    f, sc = senga.dump_read(os.path.join(GOLD, "dmpi_1step_1001.dat"), formatted=True)
    assert f.shape == (7, 1, 1, 1001)
    assert np.isfinite(f).all() and np.all(f[0] > 0)
    assert float(np.max(np.abs(f[5] + f[6] - f[0]) / f[0])) <= 1e-12
    assert np.isfinite(list(sc.values())).all()


def test_reads_a_record_split_into_subrecords(tmp_path):
    """Records beyond 2 GB come as sub-records whose leading marker is negative
    while more follow and whose trailing marker is negative when a sub-record
    precedes; built here with small pieces."""
    import senga

    f = _state(nx=3, ny=2, nz=2, nspec=1, seed=2)
    body = struct.pack("<4i", 3, 2, 2, 1) + f.tobytes() + struct.pack("<4d", 1.0, 2.0, 3.0, 4.0)
    cut = 40
    parts = [body[:cut], body[cut:]]
    p = str(tmp_path / "split.bin")
    with open(p, "wb") as fh:
        fh.write(struct.pack("<i", -len(parts[0])) + parts[0] + struct.pack("<i", len(parts[0])))
        fh.write(struct.pack("<i", len(parts[1])) + parts[1] + struct.pack("<i", -len(parts[1])))
    g, sc = senga.dump_read(p)
    assert np.array_equal(g, f)
    assert sc["errldr"] == 4.0
