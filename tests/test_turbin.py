"""Initial turbulence generator TURBIN (src/turbin.f:76-362 with TURBFT,
FFTSYM, ESPECT, RANINI/RANUNI).

CPU (oracle): the random stream lies in (0, 1) on single-precision values
(the reference's REAL() is single precision); the field is real, zero-mean
and solenoidal mode by mode; for odd extents (no Nyquist modes) its kinetic
energy equals the sum of E(|k|)/(2 pi k^2) over the upper half of
wavenumber space (Parseval: each upper mode and its conjugate carry that
energy). GPU: the device generator against the oracle, field-normalised
relative L-infinity 1e-10."""
import math

import numpy as np
import pytest

from conftest import rel_linf

CONST0, CK0 = 8.51064, 5.0  # input/cont.dat spectrum parameters


def test_random_stream_is_single_precision_in_unit_interval():
    import oracle

    r = oracle.ranuni(1, 30000)
    assert np.all((r > 0.0) & (r < 1.0))
    assert np.array_equal(r.astype(np.float32).astype(np.float64), r)
    assert abs(r.mean() - 0.5) < 0.01
    assert np.array_equal(r, oracle.ranuni(1, 30000))
    assert not np.array_equal(r[:100], oracle.ranuni(2, 100))


def _spectral_divergence(uvw):
    _, nz, ny, nx = uvw.shape
    F = [np.fft.fftn(c) for c in uvw]
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(nz) * nz, np.fft.fftfreq(ny) * ny, np.fft.fftfreq(nx) * nx,
                             indexing="ij")
    div = kx * F[0] + ky * F[1] + kz * F[2]
    mask = np.ones(kx.shape, bool)
    for kk, nn in ((kx, nx), (ky, ny), (kz, nz)):
        if nn % 2 == 0:
            mask &= np.abs(kk) != nn // 2
    return float(np.abs(div[mask]).max() / max(np.abs(f).max() for f in F))


@pytest.mark.parametrize("shape", [(16, 16, 16), (15, 9, 7), (16, 12, 10)])
def test_oracle_field_is_real_zero_mean_and_solenoidal(shape):
    import oracle

    uvw, im = oracle.turbin(shape, 1, CONST0, CK0)
    scale = float(np.abs(uvw).max())
    assert scale > 0.1
    assert float(np.abs(im).max()) <= 1e-13 * scale
    assert float(np.abs(uvw.mean(axis=(1, 2, 3))).max()) <= 1e-14 * scale
    assert _spectral_divergence(uvw) <= 1e-12


@pytest.mark.parametrize("shape", [(15, 9, 7), (11, 13, 9)])
def test_oracle_energy_matches_the_spectrum_for_odd_extents(shape):
    import oracle

    nx, ny, nz = shape
    uvw, _ = oracle.turbin(shape, 3, CONST0, CK0)
    tke = 0.5 * float((uvw ** 2).sum(axis=0).mean())

    def espect(k):
        w = (k / CK0) ** 2
        return CONST0 / CK0 * w * w * math.exp(-2.0 * w)

    want = 0.0
    for k in range(-(nz // 2), nz // 2 + 1):
        for j in range(-(ny // 2), ny // 2 + 1):
            for i in range(-(nx // 2), nx // 2 + 1):
                if not (k > 0 or (k == 0 and j > 0) or (k == 0 and j == 0 and i > 0)):
                    continue
                kk = math.sqrt(i * i + j * j + k * k)
                want += espect(kk) / (2.0 * math.pi * kk * kk)
    assert abs(tke - want) <= 1e-12 * want


@pytest.mark.gpu
@pytest.mark.parametrize("shape,seed", [((16, 16, 16), 1), ((15, 9, 7), 5), ((16, 12, 10), 7), ((32, 24, 20), 11)])
def test_gpu_turbin_matches_oracle(shape, seed):
    import oracle
    import senga

    got, imax = senga.turbin(shape, seed, CONST0, CK0)
    want, _ = oracle.turbin(shape, seed, CONST0, CK0)
    for c in range(3):
        assert rel_linf(got[c], want[c]) <= 1e-10, c
    assert imax <= 1e-12 * float(np.abs(want).max())
    with pytest.raises(senga.SengaError):
        senga.turbin((2048, 4, 4), seed)
