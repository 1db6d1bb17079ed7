"""FLAMIN's planar flame (src/flamin.f:44-322) and INDATA's conversion of the
start-up primitives to the conserved registers (src/indata.f:1233-1394).

CPU: the oracle's profile against its closed form (the erf of
Abramowitz-Stegun 7.1.26 within its 1.5e-7 error bound of the true erf),
the reactant and product end states as the source codes them (the product
temperature a single-precision constant, the last species the remainder),
a uniform mass flux DRIN URIN, and TEMPIN recovering T, ITNDEX and the
pressure PRIN from the conserved state. GPU: the device state, T and ITNDEX
against the oracle's for the H2 and one-step mechanisms.
"""
import math

import numpy as np
import pytest

from conftest import rel_linf

SHAPE = (64, 6, 4)
LEN = (1.0e-2, 1.0e-3, 1.0e-3)
TRIN, PRIN, DRIN, URIN = 300.0, 101325.0, 0.9, 2.5


def _mechs():
    import cases

    return {"h2": (cases.CHEM_H2, cases.DIFF_H2), "onestep": (cases.CHEM_1STEP, None)}


def _oracle(mech):
    from oracle import Oracle

    chem, diff = _mechs()[mech]
    return Oracle(SHAPE, LEN, chem, diff, 1e-9)


def _vw(seed=5):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, SHAPE[::-1]), rng.uniform(-1, 1, SHAPE[::-1])


@pytest.mark.parametrize("mech", ["h2", "onestep"])
def test_oracle_flame_profile(mech):
    import senga

    o = _oracle(mech)
    v, w = _vw()
    o.flamin(TRIN, PRIN, DRIN, URIN, v, w)
    f, T, itn = o.download()
    nspec = f.shape[0] - 5
    dx = LEN[0] / float(np.float32(SHAPE[0] - 1))
    x = np.arange(SHAPE[0]) * dx
    trinp = float(np.float32(1417.2))
    c_true = np.array([0.5 * (1 + math.erf((xx - 5e-3) / 5e-4)) for xx in x])
    assert np.max(np.abs(T[0, 0] - (TRIN + c_true * (trinp - TRIN)))) <= 1.5e-7 * (trinp - TRIN) * 1.01
    assert T[0, 0, 0] == TRIN and abs(T[0, 0, -1] - trinp) < 1e-9  # reactant and product ends
    rho = f[0]
    Y = f[5:] / rho
    assert np.max(np.abs(Y.sum(axis=0) - 1.0)) < 1e-14
    yr = {0: 1.1606960e-2, 1: 2.30295282e-1}
    for s in range(nspec - 1):
        assert abs(Y[s, 0, 0, 0] - yr.get(s, 0.0)) < 1e-15
    assert rel_linf(f[1], np.full_like(rho, DRIN * URIN)) <= 1e-14  # rho u = DRIN URIN
    assert rel_linf(f[2] / rho, v) <= 1e-14 and rel_linf(f[3] / rho, w) <= 1e-14
    chem = senga.Chem(_mechs()[mech][0])
    rg = chem.table("rgspec")[:nspec]
    p = rho * T * np.tensordot(rg, Y, axes=1)
    assert rel_linf(p, np.full_like(p, PRIN)) <= 1e-14


@pytest.mark.parametrize("mech", ["h2", "onestep"])
def test_oracle_tempin_inverts_flamin(mech):
    o = _oracle(mech)
    o.flamin(TRIN, PRIN, DRIN, URIN, *_vw())
    f, T, itn = o.download()
    T2, itn2, p2, nfail = o.tempin(TRIN)
    assert nfail == (0, 0)
    assert np.max(np.abs(T2 - T)) < 1e-5
    assert np.array_equal(itn2, itn)
    assert rel_linf(p2, np.full_like(p2, PRIN)) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("mech", ["h2", "onestep"])
@pytest.mark.parametrize("with_vw", [False, True])
def test_gpu_flamin_matches_oracle(mech, with_vw):
    import senga

    chem_path, diff_path = _mechs()[mech]
    chem = senga.Chem(chem_path)
    diff = senga.Diff(diff_path, chem)
    box = senga.Box(SHAPE, LEN, chem, diff, 1e-9)
    v, w = _vw() if with_vw else (None, None)
    box.flamin(TRIN, PRIN, DRIN, URIN, v, w)
    fg, tg, ig = box.download()
    o = _oracle(mech)
    o.flamin(TRIN, PRIN, DRIN, URIN, v, w)
    fo, to, io = o.download()
    for k in range(fo.shape[0]):
        assert rel_linf(fg[k], fo[k]) <= 1e-14, k
    assert rel_linf(tg, to) <= 1e-14
    assert np.array_equal(ig, io)
