"""The derivative family on the reference's own argument shapes
(src/dfbydx.f:36-37: FUNCTN with a 5-point halo on every side, FDERIV the
interior), through senga_deriv_big_host.

With the halo filled as PARFER fills it in a one-rank periodic box, every
operator equals the oracle's (which fills its own halo that way); bounded
directions never read their halo (it holds NaN here); and a periodic
direction whose halo holds other values (a neighbour rank's planes) is
differentiated with those values, as the reference does. Bound 1e-12
(field-normalised relative L-infinity), as for the other operator tests."""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-12
H = 5


def _field(shape, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return (np.sin(2 * np.pi * x / nx + 0.3) * np.cos(4 * np.pi * y / ny) + np.sin(2 * np.pi * z / nz) * (1 + x / nx) +
            1e-3 * rng.standard_normal((nz, ny, nx)))


def _pad(f, nend):
    """Halo of 5: periodic copies where the direction is periodic, NaN where
    it is bounded (those points must never be read)."""
    big = np.pad(f, H, mode="wrap")
    for axis, d in ((2, 0), (1, 1), (0, 2)):  # numpy axis of x, y, z
        if nend[2 * d] != 2:
            idx = [slice(None)] * 3
            idx[axis] = slice(0, H)
            big[tuple(idx)] = np.nan
            idx[axis] = slice(-H, None)
            big[tuple(idx)] = np.nan
    return big


@pytest.mark.parametrize("nend", [(2, 2, 2, 2, 2, 2), (1, 1, 2, 2, 2, 2), (2, 2, 1, 1, 1, 1), (1, 1, 1, 1, 1, 1)],
                         ids=["periodic", "bounded-x", "bounded-yz", "bounded-xyz"])
def test_deriv_big_matches_oracle(nend):
    import cases
    import senga
    from oracle import Oracle

    shape = (24, 20, 16)
    lengths = (3.1e-3, 2.3e-3, 1.7e-3)
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    box = senga.Box(shape, lengths, chem, diff, 1e-8, nend=nend)
    ref = Oracle(shape, lengths, cases.CHEM_1STEP, None, 1e-8, nend=nend)
    f = _field(shape, 5)
    big = _pad(f, nend)
    for kind in range(9):
        got = box.deriv_big(kind, big)
        assert np.isfinite(got).all(), f"kind {kind}: a bounded halo point was read"
        assert rel_linf(got, ref.deriv(kind, f)) <= TOL, f"kind {kind}"
        assert rel_linf(got, box.deriv(kind, f)) <= TOL, f"kind {kind} vs the folded form"


def test_deriv_big_reads_a_periodic_halo_as_given():
    """x periodic, its halo planes replaced by other data (a neighbour rank's
    planes): the first and second x derivatives use those values; compared
    with the interior schemes of src/dfbydx.f:67-105 and src/d2fdx2.f:96-111
    evaluated here in the same order."""
    import cases
    import senga

    shape = (16, 12, 10)
    lengths = (2.0e-3, 1.5e-3, 1.0e-3)
    chem = senga.Chem(cases.CHEM_1STEP)
    box = senga.Box(shape, lengths, chem, senga.Diff(None, chem), 1e-8)
    f = _field(shape, 9)
    big = np.pad(f, H, mode="wrap")
    rng = np.random.default_rng(3)
    big[:, :, :H] = rng.standard_normal(big[:, :, :H].shape)
    big[:, :, -H:] = rng.standard_normal(big[:, :, -H:].shape)
    a = 5.0 / 3.0, -2.0e1 / 2.1e1, 5.0 / 1.4e1, -5.0 / 6.3e1, 1.0 / 1.26e2
    c1 = [a[0] / 2.0, a[1] / 4.0, a[2] / 6.0, a[3] / 8.0, a[4] / 1.0e1]
    c2 = [a[0], a[1] / 4.0, a[2] / 9.0, a[3] / 1.6e1, a[4] / 2.5e1]
    ovd = 1.0 / (lengths[0] / float(np.float32(shape[0] - 1)))
    inner = big[H:-H, H:-H, :]

    def sh(m):
        return inner[:, :, H + m:H + m + shape[0]]

    d1 = c1[0] * (sh(1) - sh(-1))
    for m in range(2, 6):
        d1 = d1 + c1[m - 1] * (sh(m) - sh(-m))
    f0 = sh(0)
    d2 = c2[0] * ((sh(1) - f0) - (f0 - sh(-1)))
    for m in range(2, 6):
        d2 = d2 + c2[m - 1] * ((sh(m) - f0) - (f0 - sh(-m)))
    assert rel_linf(box.deriv_big(0, big), d1 * ovd) <= TOL
    assert rel_linf(box.deriv_big(3, big), d2 * (ovd * ovd)) <= TOL
    # and not what a folded (single-rank periodic) read would give
    assert rel_linf(box.deriv(0, f), d1 * ovd) > 1e-3
