"""Bounded y and z directions for the operator-level derivatives and the filter.

The mixed derivatives D2FDXY/D2FDXZ/D2FDYZ (src/d2fdxy.f:393-1924, and the
same sections of d2fdxz.f, d2fdyz.f) close a bounded second direction with
the mirror of the x-end rows and treat the corners where both directions are
bounded with their own one-sided/one-sided schemes (ACC1XY, ACC2XY). CPU tests
pin the oracle: the corner coefficients against the reference's DFINIT text,
exactness on polynomials for every bounded combination, the mirror images of
the corners, and a direct restatement of the low-low corner block and y-end
rows term by term. GPU tests compare the device operators with the oracle.
"""
import itertools
import json
import os

import numpy as np
import pytest

from conftest import rel_linf

HERE = os.path.dirname(os.path.abspath(__file__))
COEF = json.load(open(os.path.join(HERE, "golden", "coefficients.json")))
SHAPE = (14, 13, 12)  # nx, ny, nz: every bounded extent at least 12
LEN = (3.1e-3, 2.3e-3, 1.7e-3)
NB, NP = 1, 2  # NBOUND, NPERI
# bounded-direction sets covering each plane's four end combinations
COMBOS = [(1,), (2,), (0, 1), (0, 2), (1, 2), (0, 1, 2)]
TOL_DERIV = 1e-12


def _fd(name):
    return COEF["fd"][name]["value"]


def _nend(bounded):
    e = [NP] * 6
    for d in bounded:
        e[2 * d] = e[2 * d + 1] = NB
    return tuple(e)


def _oracle(bounded, shape=SHAPE):
    import cases
    from oracle import Oracle

    return Oracle(shape, LEN, cases.CHEM_1STEP, None, 1e-8, nend=_nend(bounded))


def _grid(shape=SHAPE):
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return (x / (nx - 1), y / (ny - 1), z / (nz - 1))  # 0..1 along each axis


PLANES = {0: (0, 1), 1: (0, 2), 2: (1, 2)}


def test_corner_coefficients_equal_reference_source():
    o = _oracle((0, 1))
    for n in ("acc1xy", "bcc1xy", "ccc1xy", "dcc1xy", "acc2xy", "bcc2xy", "ccc2xy", "dcc2xy"):
        for plane in ("XY", "XZ", "YZ"):
            want = _fd(n[:3].upper() + n[3] + plane)
            assert abs(o.scalar(n) - want) <= 1e-15 * abs(want), (n, plane)


BOTH_BOUNDED = [((0, 1), 0), ((0, 2), 1), ((1, 2), 2), ((0, 1, 2), 0), ((0, 1, 2), 1), ((0, 1, 2), 2)]


@pytest.mark.parametrize("bounded,plane", BOTH_BOUNDED, ids=lambda v: str(v))
def test_mixed_exact_on_polynomials(bounded, plane):
    """Both directions of the plane bounded: every scheme in play (one-sided
    rows on the centred difference, one-sided/one-sided corners, diagonal
    4th/6th/8th, interior) differentiates a polynomial of degree at most 4 in
    each direction and 5 in total exactly."""
    o = _oracle(bounded)
    s = _grid()
    a, b = PLANES[plane]
    c = 3 - a - b
    rng = np.random.default_rng(7 + plane)
    sa, sb, sc = s[a], s[b], s[c]
    third = 1.0 + 0.3 * np.cos(2 * np.pi * sc * (SHAPE[c] - 1) / SHAPE[c])  # any function of the third axis
    f = np.zeros_like(sa)
    d = np.zeros_like(sa)
    for p in range(5):
        for q in range(5):
            if p + q > 5:
                continue
            cpq = rng.uniform(-1, 1)
            f += cpq * sa ** p * sb ** q
            if p and q:
                d += cpq * p * q * sa ** (p - 1) * sb ** (q - 1)
    f *= third
    d *= third / (LEN[a] * LEN[b])
    assert rel_linf(o.deriv(6 + plane, f), d) <= 1e-9


# (plane, bounded direction, periodic direction)
ONE_BOUNDED = [(0, 1, 0), (1, 2, 0), (2, 2, 1), (2, 1, 2)]


@pytest.mark.parametrize("plane,bnd,per", ONE_BOUNDED, ids=lambda v: str(v))
def test_mixed_end_rows_on_linear_fields(plane, bnd, per):
    """A bounded second direction (y or z) with a periodic partner, for
    f = s sin(theta p) (s linear along the bounded direction, p the periodic
    index): the two rows at each bounded end give the 4th-order centred
    p-derivative (ACOFX1, BCOFX1; src/d2fdxy.f:422-481, 1193-1283), rows 3-5
    the diagonal 4th/6th/8th-order schemes, the rest the 10th-order interior
    one; the closed form of each row in the modified wavenumbers."""
    import math

    o = _oracle((bnd,))
    idx = np.meshgrid(np.arange(SHAPE[2]), np.arange(SHAPE[1]), np.arange(SHAPE[0]), indexing="ij")[::-1]
    nb, npr = SHAPE[bnd], SHAPE[per]
    db, dp = LEN[bnd] / (nb - 1), LEN[per] / (npr - 1)
    th = 2 * np.pi * 2 / npr
    f = idx[bnd] * db * np.sin(th * idx[per])
    got = o.deriv(6 + plane, f)
    four = (2 * _fd("ACOFX1") * math.sin(th) + 2 * _fd("BCOFX1") * math.sin(2 * th)) / dp
    rows = {2: ("ACF3XY", "BCF3XY"), 3: ("ACF4XY", "BCF4XY", "CCF4XY"), 4: ("ACF5XY", "BCF5XY", "CCF5XY", "DCF5XY")}
    inner = ("ACOFXY", "BCOFXY", "CCOFXY", "DCOFXY", "ECOFXY")

    def diag(names):
        return sum(_fd(nm) * 4 * (m + 1) * math.sin((m + 1) * th) for m, nm in enumerate(names)) / dp

    e = np.minimum(idx[bnd], nb - 1 - idx[bnd])
    fac = np.where(e <= 1, four, np.where(e == 2, diag(rows[2]), np.where(e == 3, diag(rows[3]),
                                                                        np.where(e == 4, diag(rows[4]), diag(inner)))))
    want = fac * np.cos(th * idx[per])
    assert rel_linf(got, want) <= 1e-11


@pytest.mark.parametrize("plane", [0, 1, 2])
@pytest.mark.parametrize("flip", [0, 1])
def test_mirrored_corners_change_sign(plane, flip):
    """All three directions bounded: mirroring the field along one direction
    of the plane mirrors the mixed derivative with the opposite sign, so each
    right-end and mixed-end corner is the image of the low-low one."""
    o = _oracle((0, 1, 2))
    rng = np.random.default_rng(11 + plane)
    f = rng.standard_normal(SHAPE[::-1])
    axis = 2 - PLANES[plane][flip]  # numpy axis of that direction (z, y, x order)
    d = o.deriv(6 + plane, f)
    dm = o.deriv(6 + plane, np.flip(f, axis=axis))
    assert rel_linf(np.flip(dm, axis=axis), -d) <= 1e-12


def _restated_low_corner_xy(F, i, j):
    """d2fdxy at x index i, y index j (0-based) of a 2D slice F[x, y], both
    directions bounded, i or j below 5, unscaled; term by term from
    src/d2fdxy.f: y-left end rows :422-481, the low-low corner :516-627,
    its edge rows :628-751 and inner blocks :752-835, x-left rows :151-230."""
    c = _fd
    w1 = [c("ACF1XY"), c("BCF1XY"), c("CCF1XY"), c("DCF1XY")]
    w2 = [c("ACF2XY"), c("BCF2XY"), c("CCF2XY"), c("DCF2XY")]
    if i >= 2 and j >= 2:
        m = min(i, j)

        def ring(r):
            return F[i + r, j + r] - F[i + r, j - r] - F[i - r, j + r] + F[i - r, j - r]

        if m >= 5:
            return sum(c(n) * ring(r + 1) for r, n in enumerate(("ACOFXY", "BCOFXY", "CCOFXY", "DCOFXY", "ECOFXY")))
        names = {2: ("ACF3XY", "BCF3XY"), 3: ("ACF4XY", "BCF4XY", "CCF4XY"),
                 4: ("ACF5XY", "BCF5XY", "CCF5XY", "DCF5XY")}[m]
        return sum(c(n) * ring(r + 1) for r, n in enumerate(names))
    if j <= 1 and i >= 2:  # rows 0 and 1 of the y-left end: one-sided in y, 4th-order centred in x
        def fd(jj):
            return (c("ACOFX1") * (F[i + 1, jj] - F[i - 1, jj] - F[i + 1, j] + F[i - 1, j]) +
                    c("BCOFX1") * (F[i + 2, jj] - F[i - 2, jj] - F[i + 2, j] + F[i - 2, j]))

        if j == 0:
            return sum(w * fd(jj) for w, jj in zip(w1, (1, 2, 3, 4)))
        return sum(w * fd(jj) for w, jj in zip(w2, (0, 2, 3, 4)))
    if i <= 1 and j >= 2:  # rows 0 and 1 of the x-left end: one-sided in x, 4th-order centred in y
        def fd(ii):
            return (c("ACOFY1") * (F[ii, j + 1] - F[ii, j - 1] - F[i, j + 1] + F[i, j - 1]) +
                    c("BCOFY1") * (F[ii, j + 2] - F[ii, j - 2] - F[i, j + 2] + F[i, j - 2]))

        if i == 0:
            return sum(w * fd(ii) for w, ii in zip(w1, (1, 2, 3, 4)))
        return sum(w * fd(ii) for w, ii in zip(w2, (0, 2, 3, 4)))
    if i == 0 and j == 0:
        k = [c("ACC1XY"), c("BCC1XY"), c("CCC1XY"), c("DCC1XY")]
        return sum(k[m - 1] * (F[m, m] - F[m, 0] - F[0, m] + F[0, 0]) for m in (1, 2, 3, 4))
    if i == 1 and j == 1:
        k = [c("ACC2XY"), c("BCC2XY"), c("CCC2XY"), c("DCC2XY")]
        return sum(kk * (F[m, m] - F[m, 1] - F[1, m] + F[1, 1]) for kk, m in zip(k, (0, 2, 3, 4)))
    if i == 0:  # j == 1
        return sum(w1[ii - 1] * sum(w * (F[ii, jj] - F[ii, 1] - F[0, jj] + F[0, 1]) for w, jj in zip(w2, (0, 2, 3, 4)))
                   for ii in (1, 2, 3, 4))
    # i == 1, j == 0
    return sum(w1[jj - 1] * sum(w * (F[ii, jj] - F[1, jj] - F[ii, 0] + F[1, 0]) for w, ii in zip(w2, (0, 2, 3, 4)))
               for jj in (1, 2, 3, 4))


def test_low_corner_matches_direct_restatement():
    """The oracle's low-low corner of d2fdxy with x and y bounded equals the
    reference's formulas written out term by term (coefficients read from
    its DFINIT text), point by point over the 7x7 block at the corner."""
    o = _oracle((0, 1))
    rng = np.random.default_rng(3)
    f = rng.standard_normal(SHAPE[::-1])
    d = o.deriv(6, f)
    scale = 1.0 / ((LEN[0] / (SHAPE[0] - 1)) * (LEN[1] / (SHAPE[1] - 1)))
    dmax = np.max(np.abs(d))
    for k in (0, SHAPE[2] // 2):
        F = f[k].T  # [x, y]
        for i, j in itertools.product(range(7), range(7)):
            want = _restated_low_corner_xy(F, i, j) * scale
            assert abs(d[k, j, i] - want) <= 1e-12 * dmax, (i, j, k)


# ----------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("bounded", COMBOS, ids=lambda b: "b" + "".join("xyz"[d] for d in b))
def test_gpu_derivatives_bounded_yz(bounded):
    """All nine operators on the device against the oracle with y and/or z
    bounded: first and second derivatives with their closures in any
    direction, mixed derivatives with end rows and corners."""
    import cases
    import senga

    rng = np.random.default_rng(50 + len(bounded))
    s = _grid()
    f = (np.sin(2.1 * s[0] + 0.4) * np.cos(3.3 * s[1]) + s[2] ** 3 * s[0] + 0.2 * np.sin(5.0 * s[2]) +
         1e-3 * rng.standard_normal(SHAPE[::-1]))
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    box = senga.Box(SHAPE, LEN, chem, diff, 1e-8, nend=_nend(bounded))
    ref = _oracle(bounded)
    for kind in range(9):
        assert rel_linf(box.deriv(kind, f), ref.deriv(kind, f)) <= TOL_DERIV, kind


@pytest.mark.gpu
@pytest.mark.parametrize("bounded", [(1,), (2,), (0, 1, 2)], ids=["by", "bz", "bxyz"])
def test_gpu_filter_bounded_yz(bounded):
    """The explicit filter with its one-sided rows on bounded y and z ends."""
    import cases
    import senga

    rng = np.random.default_rng(60)
    f = rng.standard_normal(SHAPE[::-1])
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    box = senga.Box(SHAPE, LEN, chem, diff, 1e-8, nend=_nend(bounded))
    ref = _oracle(bounded)
    for mode in (0, 1):
        assert rel_linf(box.filter_field(f, mode), ref.filter_field(f, mode)) <= 1e-13, mode


@pytest.mark.gpu
def test_gpu_bounded_y_box_refuses_rhs_and_stays_usable():
    """A box bounded in y runs the operators only: the step, graph step and
    RHS entry points return SENGA_ERR_UNSUPPORTED (no y face conditions are
    built), and the refusal leaves the context's stream usable."""
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    box = senga.Box(SHAPE, LEN, chem, diff, 1e-8, nend=_nend((1,)))
    for call in (lambda: box.step(1), lambda: box.step(1, graph=True), lambda: box.rhs()):
        with pytest.raises(senga.SengaError, match="status 5"):
            call()
    f = np.cos(2 * np.pi * _grid()[0])
    assert rel_linf(box.deriv(0, f), _oracle((1,)).deriv(0, f)) <= TOL_DERIV
