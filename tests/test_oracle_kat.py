"""Known-answer tests that pin the oracle (the CPU restatement) on the CPU.

The reference is Fortran and cannot be built here (no Fortran compiler), so
the oracle is pinned by
  * constants read as text from the reference's sources (tests/golden/
    coefficients.json: RK coefficients of src/dtinit.f:78-94, derivative
    coefficients of src/dfinit.f) and the order conditions they must meet;
  * closed-form answers: the modified wavenumber of each interior stencil on
    a sinusoid, polynomial exactness of the one-sided closures, the analytic
    single-step Arrhenius rate, TEMPER inverting the energy of a known T;
  * conservation laws and the RK order of accuracy;
  * the committed oracle fixtures (tests/golden/oracle_*.npz), a regression
    pin that the GPU parity tests also read.
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import rel_linf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

with open(os.path.join(GOLD, "coefficients.json")) as _f:
    COEF = json.load(_f)


def _fd(name):
    return COEF["fd"][name]["value"]


def _oracle(shape, lengths=(3.1e-3, 2.3e-3, 1.7e-3), nend=(2,) * 6, chem=None, diff=None, dt=1e-8):
    import cases
    from oracle import Oracle

    return Oracle(shape, lengths, chem or cases.CHEM_1STEP, diff, dt, nend=nend)


# ---------------------------------------------------------------- constants
def test_rk_coefficients_equal_reference_source():
    o = _oracle((12, 12, 12))
    for i in range(1, 6):
        a = COEF["rk"][f"ACOFRK({i})"]["value"]
        b = COEF["rk"][f"BCOFRK({i})"]["value"]
        bh = COEF["rk"][f"BHATRK({i})"]["value"]
        assert math.isclose(o.scalar(f"rk.rhs{i}"), a, rel_tol=1e-15, abs_tol=1e-300)
        assert math.isclose(o.scalar(f"rk.lhs{i}"), b, rel_tol=1e-15)
        assert math.isclose(o.scalar(f"rk.err{i}"), b - bh, rel_tol=1e-13)


def _butcher():
    """Butcher tableau of the 2N-storage ('2R') scheme: stage i+1 uses
    a_{i+1,i} = ACOFRK(i) and a_{j,i} = BCOFRK(i) for j > i+1."""
    from fractions import Fraction

    rk = COEF["rk"]
    a = [Fraction(rk[f"ACOFRK({i})"]["num"], rk[f"ACOFRK({i})"]["den"]) for i in range(1, 6)]
    b = [Fraction(rk[f"BCOFRK({i})"]["num"], rk[f"BCOFRK({i})"]["den"]) for i in range(1, 6)]
    bh = [Fraction(rk[f"BHATRK({i})"]["num"], rk[f"BHATRK({i})"]["den"]) for i in range(1, 6)]
    A = [[Fraction(0)] * 5 for _ in range(5)]
    for j in range(5):
        for i in range(j):
            A[j][i] = a[i] if i == j - 1 else b[i]
    c = [sum(A[j]) for j in range(5)]
    return A, b, bh, c


def test_rk_order_conditions():
    """RK4(3)5: the main weights satisfy the eight order-4 conditions, the
    embedded weights the four order-3 conditions (to the rounding of the
    13-digit rationals in the source)."""
    A, b, bh, c = _butcher()
    r = range(5)
    Ac = [sum(A[i][j] * c[j] for j in r) for i in r]
    conds4 = [
        (sum(b), 1), (sum(b[i] * c[i] for i in r), 0.5), (sum(b[i] * c[i] ** 2 for i in r), 1 / 3),
        (sum(b[i] * Ac[i] for i in r), 1 / 6), (sum(b[i] * c[i] ** 3 for i in r), 0.25),
        (sum(b[i] * c[i] * Ac[i] for i in r), 1 / 8),
        (sum(b[i] * sum(A[i][j] * c[j] ** 2 for j in r) for i in r), 1 / 12),
        (sum(b[i] * sum(A[i][j] * Ac[j] for j in r) for i in r), 1 / 24),
    ]
    for got, want in conds4:
        assert abs(float(got) - want) < 1e-11
    conds3 = [(sum(bh), 1), (sum(bh[i] * c[i] for i in r), 0.5), (sum(bh[i] * c[i] ** 2 for i in r), 1 / 3),
              (sum(bh[i] * Ac[i] for i in r), 1 / 6)]
    for got, want in conds3:
        assert abs(float(got) - want) < 1e-11


def _ref_name(n):
    u = n.upper()
    return u if u.endswith("X") or u.endswith("XY") else u + "X"


ORACLE_FD = ["acoffx", "bcoffx", "ccoffx", "dcoffx", "ecoffx", "acof1", "bcof1", "ccof1", "dcof1", "acof2",
             "bcof2", "ccof2", "dcof2", "acof3", "bcof3", "acof4", "bcof4", "ccof4", "acof5", "bcof5", "ccof5",
             "dcof5", "acofs", "bcofs", "ccofs", "dcofs", "ecofs", "acfs1", "bcfs1", "ccfs1", "dcfs1", "ecfs1",
             "acfs2", "bcfs2", "ccfs2", "dcfs2", "ecfs2", "acfs3", "bcfs3", "acfs4", "bcfs4", "ccfs4", "acfs5",
             "bcfs5", "ccfs5", "dcfs5", "acofxy", "bcofxy", "ccofxy", "dcofxy", "ecofxy"]


def test_derivative_coefficients_equal_reference_source():
    o = _oracle((12, 12, 12))
    for n in ORACLE_FD:
        assert math.isclose(o.scalar(n), _fd(_ref_name(n)), rel_tol=1e-15), n


def test_grid_spacing_convention():
    """Delta = L/(N-1) (src/dfinit.f:42-50)."""
    o = _oracle((12, 10, 8), lengths=(1.1e-3, 0.9e-3, 0.7e-3))
    assert math.isclose(o.scalar("deltax"), 1.1e-3 / 11, rel_tol=1e-15)
    assert math.isclose(o.scalar("deltay"), 0.9e-3 / 9, rel_tol=1e-15)
    assert math.isclose(o.scalar("deltaz"), 0.7e-3 / 7, rel_tol=1e-15)


# ------------------------------------------------------- interior stencils
SHAPE = (24, 20, 16)  # nx, ny, nz
LEN = (3.1e-3, 2.3e-3, 1.7e-3)


def _grid_phase(axis, mode):
    nx, ny, nz = SHAPE
    n = SHAPE[axis]
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    idx = (x, y, z)[axis]
    th = 2 * np.pi * mode / n
    return th, th * idx + 0.3


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_first_derivative_modified_wavenumber(axis):
    o = _oracle(SHAPE, LEN)
    d = LEN[axis] / (SHAPE[axis] - 1)
    c = [_fd(k) for k in ("ACOFFX", "BCOFFX", "CCOFFX", "DCOFFX", "ECOFFX")]
    for mode in (1, 3, 5):
        th, ph = _grid_phase(axis, mode)
        kmod = sum(2 * c[m - 1] * math.sin(m * th) for m in range(1, 6)) / d
        got = o.deriv(axis, np.sin(ph))
        assert rel_linf(got, kmod * np.cos(ph)) <= 1e-12


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_second_derivative_modified_wavenumber(axis):
    o = _oracle(SHAPE, LEN)
    d = LEN[axis] / (SHAPE[axis] - 1)
    c = [_fd(k) for k in ("ACOFSX", "BCOFSX", "CCOFSX", "DCOFSX", "ECOFSX")]
    for mode in (1, 4):
        th, ph = _grid_phase(axis, mode)
        k2 = sum(c[m - 1] * 2 * (math.cos(m * th) - 1) for m in range(1, 6)) / (d * d)
        got = o.deriv(3 + axis, np.sin(ph))
        assert rel_linf(got, k2 * np.sin(ph)) <= 1e-11


@pytest.mark.parametrize("plane", [0, 1, 2])
def test_mixed_derivative_modified_wavenumber(plane):
    o = _oracle(SHAPE, LEN)
    a1, a2 = [(0, 1), (0, 2), (1, 2)][plane]
    d1 = LEN[a1] / (SHAPE[a1] - 1)
    d2 = LEN[a2] / (SHAPE[a2] - 1)
    c = [_fd(k) for k in ("ACOFXY", "BCOFXY", "CCOFXY", "DCOFXY", "ECOFXY")]
    t1, p1 = _grid_phase(a1, 2)
    t2, p2 = _grid_phase(a2, 1)
    f = np.sin(p1) * np.sin(p2 + 0.2)
    k = sum(c[m - 1] * 4 * math.sin(m * t1) * math.sin(m * t2) for m in range(1, 6)) / (d1 * d2)
    got = o.deriv(6 + plane, f)
    assert rel_linf(got, k * np.cos(p1) * np.cos(p2 + 0.2)) <= 1e-12


def test_first_derivative_tenth_order_convergence():
    """Error of d/dx sin(2 pi x / P) falls as Delta^10 on refinement."""
    errs = []
    for n in (16, 32):
        shape = (n, 8, 8)
        L = 1.0e-3
        o = _oracle(shape, (L, L, L))
        d = L / (n - 1)
        P = n * d
        x = np.arange(n) * d
        f = np.broadcast_to(np.sin(2 * np.pi * x / P), (8, 8, n)).copy()
        exact = (2 * np.pi / P) * np.cos(2 * np.pi * x / P)
        errs.append(float(np.max(np.abs(o.deriv(0, f)[0, 0] - exact))) / (2 * np.pi / P))
    order = math.log(errs[0] / errs[1], 2)
    assert order > 9.5, errs


# ------------------------------------------------------ bounded closures
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_closures_exact_for_quartics(axis):
    """One-sided closures (4th-order at the wall, 4th/6th/8th inward) and the
    10th-order interior differentiate a quartic exactly (src/dfbydx.f,
    src/d2fdx2.f); both ends bounded (NBOUND=1)."""
    nend = [2] * 6
    nend[2 * axis] = nend[2 * axis + 1] = 1
    o = _oracle(SHAPE, LEN, nend=tuple(nend))
    nx, ny, nz = SHAPE
    d = LEN[axis] / (SHAPE[axis] - 1)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    s = (x, y, z)[axis] * d / LEN[axis]  # 0..1 along the bounded axis
    f = 0.3 - 1.2 * s + 0.7 * s ** 2 + 2.1 * s ** 3 - 1.4 * s ** 4
    df = (-1.2 + 1.4 * s + 6.3 * s ** 2 - 5.6 * s ** 3) / LEN[axis]
    d2f = (1.4 + 12.6 * s - 16.8 * s ** 2) / LEN[axis] ** 2
    assert rel_linf(o.deriv(axis, f), df) <= 1e-11
    assert rel_linf(o.deriv(3 + axis, f), d2f) <= 1e-9


# ------------------------------------------------------- thermochemistry
def _uniform_state(chem_path, T0, Y, shape=(12, 12, 12), p=101325.0):
    import cases
    import senga

    chem = senga.Chem(chem_path)
    nx, ny, nz = shape
    shp = (nz, ny, nx)
    T = np.full(shp, T0)
    Yf = np.array([np.full(shp, y) for y in Y])
    z = np.zeros(shp)
    fields, itn = cases.conserved(chem, np.full(shp, p), T, z, z, z, Yf)
    return chem, fields, T, itn


def test_temper_inverts_energy_from_a_perturbed_seed():
    """TEMPER (src/temper.f:58-219) recovers the temperature the energy was
    built from, starting its Newton iteration from a seed 3% off."""
    import cases

    c = cases.make_case("h2_kernels", n=10, seed=5)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], diff=c["diff"], dt=c["dt"])
    o.upload(c["fields"], c["T"] * 1.03, c["itn"])
    _, t, p = o.rhs()
    assert float(np.max(np.abs(t - c["T"]))) <= 1e-8
    # p = rho R_mix T
    import senga

    rg = senga.Chem(c["chem"]).table("rgspec")
    rmix = sum(rg[s] * c["fields"][5 + s] for s in range(9)) / c["fields"][0]
    assert rel_linf(p, c["fields"][0] * rmix * c["T"]) <= 1e-12


def test_single_step_rate_is_arrhenius():
    """1-step R->P (A=1e9, n=0, E/R_u=15000 K, first order in R):
    rate_R = -A exp(-E/(R_u T)) rho Y_R W_R / W_R, rate_P = -rate_R."""
    import cases

    c = cases.make_case("ignition32", n=12, seed=3)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], dt=c["dt"])
    o.upload(c["fields"], c["T"], c["itn"])
    r = o.chrate()
    want = -1.0e9 * np.exp(-(1.24713e8 / 8314.2) / c["T"]) * c["fields"][5]
    assert rel_linf(r[0], want) <= 1e-12
    assert rel_linf(r[1], -want) <= 1e-12


def test_h2_rates_conserve_mass():
    """sum_k rate_k = sum_steps omega * sum_k dnu_k W_k: zero to the rounding
    of the molar masses in chem.dat."""
    import cases

    c = cases.make_case("h2_kernels", n=10, seed=9)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], diff=c["diff"], dt=c["dt"])
    o.upload(c["fields"], c["T"] * 1.6, c["itn"])  # hotter: every step active
    r = o.chrate()
    tot = np.sum(r, axis=0)
    scale = np.sum(np.abs(r), axis=0)
    assert float(np.max(np.abs(tot) / scale)) <= 1e-6


# ------------------------------------------------------------ RK and RHS
def test_rk_is_fourth_order_on_a_uniform_reacting_box():
    """A uniform box reduces the PDE to the chemistry ODE; halving dt cuts
    the step-size error 16-fold (RK4(3)5[2R+]C)."""
    import cases

    # 900 K: about 1 % of the reactant burns in tend and T rises ~20 K; the
    # thermal-runaway eigenvalue k E/(R T^2) dT_ad ~ 1.6e3 /s keeps h*lambda
    # below 0.1 (a hotter start runs away within a step)
    chem, f, T, itn = _uniform_state(cases.CHEM_1STEP, 900.0, (1.0, 0.0))
    tend = 2.0e-4
    ys = []
    for nsteps in (4, 8, 16):
        o = _oracle((12, 12, 12), (1e-3, 1e-3, 1e-3), chem=cases.CHEM_1STEP, dt=tend / nsteps)
        o.upload(f, T, itn)
        o.step(nsteps)
        g, _, _ = o.download()
        ys.append(float(g[5, 0, 0, 0]))
        assert float(np.ptp(g[5])) == 0.0  # stays uniform
    e1, e2 = abs(ys[0] - ys[1]), abs(ys[1] - ys[2])
    ratio = e1 / e2
    assert 13.0 < ratio < 19.0, (ys, ratio)


def test_periodic_rhs_conserves_mass():
    """DRHS = -div(rho u): a periodic central difference sums to zero. (The
    momentum and energy convection are skew-symmetric splits, not discretely
    conservative, so only mass is checked.)"""
    import cases

    c = cases.make_case("h2_kernels", n=12, seed=4)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], diff=c["diff"], dt=c["dt"])
    o.upload(c["fields"], c["T"], c["itn"])
    r, _, _ = o.rhs()
    assert abs(float(np.sum(r[0]))) <= 1e-14 * float(np.sum(np.abs(r[0])))


# ------------------------------------------------------- golden fixtures
@pytest.mark.parametrize("key", ["h2_mavt", "onestep"])
def test_oracle_reproduces_golden_fixture(key):
    import cases
    from oracle import Oracle

    g = np.load(os.path.join(GOLD, f"oracle_{key}.npz"))
    nx, ny, nz = (int(v) for v in g["shape"])
    chem = os.path.join(cases.DATA, str(g["chem"]))
    diff = os.path.join(cases.DATA, str(g["diff"])) if str(g["diff"]) else None
    o = Oracle((nx, ny, nz), tuple(g["lengths"]), chem, diff, float(g["dt"]))
    o.upload(g["fields"], g["T"], g["itn"])
    rhs, t, p = o.rhs()
    for k in range(rhs.shape[0]):
        assert rel_linf(rhs[k], g["rhs"][k]) <= 1e-13, k
    assert rel_linf(t, g["T_rhs"]) <= 1e-14
    o.upload(g["fields"], g["T"], g["itn"])
    o.step(2)
    f2, t2, itn2 = o.download()
    for k in range(f2.shape[0]):
        assert rel_linf(f2[k], g["fields_2"][k]) <= 1e-13, k
    assert np.array_equal(itn2, g["itn_2"])


# ------------------------------------------------------------ explicit filter
def _tw():
    return math.exp(-12.0 * math.log(2.0))


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("flip", [0, 1])
def test_filter_transfer_function(axis, flip):
    """Interior 12th-order filter (src/filtrx.f:67-104, coefficients
    src/flinit.f): a mode exp(i theta j) is multiplied by
    1 + sin^12(theta/2) with the coded TWFACT = -2^-12 (grid-scale modes
    are amplified) and by 1 - sin^12(theta/2) with the sign flipped."""
    o = _oracle(SHAPE, LEN)
    for mode in (1, 3, SHAPE[axis] // 2):
        th, ph = _grid_phase(axis, mode)
        f = np.cos(ph)
        T = 1.0 + (-1.0 if flip else 1.0) * math.sin(th / 2) ** 12
        assert rel_linf(o.filter_field(f, mode=flip), T * f) <= 1e-13


def test_filter_one_sided_rows_keep_quintics():
    """The boundary rows (6th..11th order, src/flinit.f FACF1X..FLCF6X) and
    the interior leave polynomials of degree <= 5 unchanged."""
    nend = (1, 1, 1, 1, 1, 1)
    o = _oracle(SHAPE, LEN, nend=nend)
    nx, ny, nz = SHAPE
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    f = 0.4 + x - 2 * y ** 2 + 3 * z ** 3 - x ** 4 * y + 0.5 * x ** 2 * y * z ** 2 + 0.7 * x ** 5
    assert rel_linf(o.filter_field(f), f) <= 1e-12


def test_filter_rows_sum_to_one():
    """Every row of the filter conserves a constant: c0 + 2 sum c_m = 1 and
    each one-sided row sums to 1."""
    o = _oracle(SHAPE, LEN, nend=(1, 1, 2, 2, 2, 2))
    f = np.full((SHAPE[2], SHAPE[1], SHAPE[0]), 3.25)
    assert float(np.max(np.abs(o.filter_field(f) - 3.25))) <= 1e-13


# ------------------------------------------------------------ ADAPTT
def test_adaptt_pid_controller_first_steps():
    """ADAPTT (src/adaptt.f) with DTINIT's PID constants: on a cold start
    ERROLD = ERRLDR = ERRTOL = 1e-4, so the first ratio is
    0.9 (ERRTOL/ERRMAX)^(0.49/3), clipped to [0.01, 1.01]; the second uses
    ERROLD = first ERRMAX."""
    import cases

    c = cases.make_case("ignition32", n=12, seed=8)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], dt=c["dt"])
    o.upload(c["fields"], c["T"], c["itn"])
    o.set_adaptive(True)
    o.step(1)
    t1, e1, i1 = o.tstep()
    r = min(1.01, max(0.01, 0.9 * math.exp((0.49 / 3) * math.log(1e-4 / e1))))
    assert math.isclose(t1, c["dt"] * r, rel_tol=1e-14)
    assert e1 > 0 and i1 in (-4, -3, -2, -1, 0, 1, 2)
    o.step(1)
    t2, e2, _ = o.tstep()
    r2 = 0.9 * math.exp((0.49 / 3) * math.log(1e-4 / e2) + (0.34 / 3) * math.log(e1 / 1e-4)
                        + (0.1 / 3) * math.log(1e-4 / 1e-4))
    r2 = min(1.01, max(0.01, r2))
    assert math.isclose(t2, t1 * r2, rel_tol=1e-13)


# ------------------------------------------------------------ bounded x: mixed closures, NSCBC
@pytest.mark.parametrize("plane", [0, 1])
def test_mixed_closures_on_x_linear_fields(plane):
    """d2fdxy/d2fdxz with x bounded (src/d2fdxy.f:151-392): for f = x sin(theta s)
    (s = y or z, periodic) the first two rows from each x end give the
    4th-order centred s-derivative (ACOFY1, BCOFY1), rows 3-5 the diagonal
    4th/6th/8th-order schemes, the rest the 10th-order interior one."""
    nend = (1, 1, 2, 2, 2, 2)
    o = _oracle(SHAPE, LEN, nend=nend)
    nx, ny, nz = SHAPE
    a2 = 1 + plane
    ns = SHAPE[a2]
    dx = LEN[0] / (nx - 1)
    ds = LEN[a2] / (ns - 1)
    th = 2 * np.pi * 2 / ns
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    s = (y, z)[plane]
    f = x * dx * np.sin(th * s)
    got = o.deriv(6 + plane, f)
    my = (_fd("ACOFY1"), _fd("BCOFY1"))
    four = (2 * my[0] * math.sin(th) + 2 * my[1] * math.sin(2 * th)) / ds
    rows = {2: ("ACF3XY", "BCF3XY"), 3: ("ACF4XY", "BCF4XY", "CCF4XY"), 4: ("ACF5XY", "BCF5XY", "CCF5XY", "DCF5XY")}
    inner = ("ACOFXY", "BCOFXY", "CCOFXY", "DCOFXY", "ECOFXY")

    def diag(names):
        return sum(_fd(nm) * 4 * (m + 1) * math.sin((m + 1) * th) for m, nm in enumerate(names)) / ds

    for i in range(nx):
        e = min(i, nx - 1 - i)
        k = four if e < 2 else diag(rows[e]) if e < 5 else diag(inner)
        want = k * np.cos(th * s[..., i])
        assert rel_linf(got[..., i], want) <= 1e-11, (i, e)


def _uniform_inflow_state(c, p=1.0e5, n=16):
    import senga

    chem = senga.Chem(c["chem"])
    shp = (n, n, n)
    bc = c["bc"]
    T = np.full(shp, 300.0)
    Y = np.array([np.full(shp, y) for y in bc["y_in"]])
    u = np.full(shp, bc["u_in"])
    z = np.zeros(shp)
    import cases

    f, itn = cases.conserved(chem, np.full(shp, p), T, u, z, z, Y)
    return f, T, itn


def test_nscbc_uniform_inflow_state_is_steady():
    """I3 inflow + O1 outflow box holding the inflow state at p = p_inf: every
    wave amplitude vanishes and the state does not move."""
    import cases

    c = cases.make_case("flame_inout", n=16, seed=5)
    f, T, itn = _uniform_inflow_state(c)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], diff=c["diff"], dt=c["dt"], nend=c["nend"])
    o.set_bc(c["bc"])
    o.upload(f, T, itn)
    o.step(3)
    g, _, _ = o.download()
    for k in range(5):
        assert rel_linf(g[k], f[k]) <= 1e-12, k
    assert float(np.max(np.abs(g[5:] - f[5:]))) <= 1e-12


def test_nscbc_outflow_relaxes_pressure_and_inflow_is_imposed():
    """p above p_inf: the O1 plane loses mass (dRHO/dt < 0 there, sigma > 0);
    after steps the I3 plane still holds rho_in, rho_in u_in and rho_in Y_in."""
    import cases

    c = cases.make_case("flame_inout", n=16, seed=5)
    f, T, itn = _uniform_inflow_state(c, p=1.02e5)
    o = _oracle(c["shape"], c["lengths"], chem=c["chem"], diff=c["diff"], dt=c["dt"], nend=c["nend"])
    o.set_bc(c["bc"])
    o.upload(f, T, itn)
    r, _, _ = o.rhs()
    assert float(np.max(r[0][..., -1])) < 0.0
    # away from both faces (the imposed inflow density differs from the box's
    # near x = 0) the uniform state has no mass flux divergence
    assert float(np.max(np.abs(r[0][..., 6:-1]))) <= 1e-9 * float(np.max(np.abs(r[0][..., -1])))
    o.upload(f, T, itn)
    o.step(2)
    g, _, _ = o.download()
    bc = c["bc"]
    assert np.all(g[0][..., 0] == bc["rho_in"])
    assert np.all(g[1][..., 0] == bc["rho_in"] * bc["u_in"])
    for s_ in range(9):
        assert np.all(g[5 + s_][..., 0] == bc["rho_in"] * bc["y_in"][s_])
