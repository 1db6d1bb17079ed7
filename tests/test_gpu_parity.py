"""CUDA path vs the oracle (CPU restatement of the reference), through the C ABI.

Tolerance: field-normalised relative L-infinity, max|gpu-ref|/max|ref|,
<= 1e-10 for state after N steps and for the right-hand side (the FP64 sums
are reordered and contracted into FMAs on the GPU, so bit-exactness is not
expected); derivative operators <= 1e-12.
"""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-10
TOL_DERIV = 1e-12


def _pair(case):
    import senga
    from oracle import Oracle

    chem = senga.Chem(case["chem"])
    diff = senga.Diff(case["diff"], chem)
    box = senga.Box(case["shape"], case["lengths"], chem, diff, case["dt"], nend=case["nend"])
    ref = Oracle(case["shape"], case["lengths"], case["chem"], case["diff"], case["dt"], nend=case["nend"])
    box.upload(case["fields"], case["T"], case["itn"])
    ref.upload(case["fields"], case["T"], case["itn"])
    return box, ref


def _case(name, n, seed=7):
    import cases

    return cases.make_case(name, n=n, seed=seed)


@pytest.mark.parametrize("kind", range(9))
def test_derivative_family_noncubic(kind):
    """DFBYDX..D2FDYZ on a non-cubic periodic box against the oracle."""
    import senga
    from oracle import Oracle

    rng = np.random.default_rng(kind)
    nx, ny, nz = 24, 20, 16
    shape = (nz, ny, nx)
    # smooth periodic field plus a little noise (exercises every stencil weight)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f = (np.sin(2 * np.pi * x / nx) * np.cos(4 * np.pi * y / ny) + np.sin(2 * np.pi * (z / nz + x / nx))
         + 1e-3 * rng.standard_normal(shape))
    c = _case("ignition32", 16)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(None, chem)
    lengths = (3.1e-3, 2.3e-3, 1.7e-3)
    box = senga.Box((nx, ny, nz), lengths, chem, diff, 1e-8)
    ref = Oracle((nx, ny, nz), lengths, c["chem"], None, 1e-8)
    got = box.deriv(kind, f)
    want = ref.deriv(kind, f)
    assert rel_linf(got, want) <= TOL_DERIV


@pytest.mark.parametrize("name,n", [("ignition32", 16), ("h2_kernels", 16)])
def test_rhs_matches_oracle(name, n):
    c = _case(name, n)
    box, ref = _pair(c)
    r_g, t_g, p_g = box.rhs()
    r_o, t_o, p_o = ref.rhs()
    assert rel_linf(t_g, t_o) <= TOL_STATE
    assert rel_linf(p_g, p_o) <= TOL_STATE
    for k in range(r_o.shape[0]):
        assert rel_linf(r_g[k], r_o[k]) <= TOL_STATE, f"field {k}"


@pytest.mark.parametrize("name", ["ignition32", "h2_kernels"])
def test_chrate_matches_oracle(name):
    c = _case(name, 12)
    box, ref = _pair(c)
    got = box.chrate()
    want = ref.chrate()
    for k in range(want.shape[0]):
        if np.max(np.abs(want[k])) > 0:
            assert rel_linf(got[k], want[k]) <= TOL_STATE, f"species {k}"


def test_ignition32_ten_steps():
    """The 32^3 one-step ignition workload: 10 RK steps, all fields."""
    c = _case("ignition32", 32)
    box, ref = _pair(c)
    box.step(10)
    ref.step(10)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"
    assert rel_linf(tg, to) <= TOL_STATE


def test_h2_mixture_averaged_steps():
    """H2 mechanism with mixture-averaged transport, 20^3, 3 RK steps."""
    c = _case("h2_kernels", 20)
    box, ref = _pair(c)
    box.step(3)
    ref.step(3)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"
    assert rel_linf(tg, to) <= TOL_STATE


def test_noncubic_ensemble_box_steps():
    """A non-cubic box of the batched ensemble (one-step chemistry)."""
    import cases

    c = cases.make_case("ensemble", seed=11)
    c2 = dict(c)
    box, ref = _pair(c2)
    box.step(2)
    ref.step(2)
    g, _, _ = box.download()
    o, _, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"


def test_graph_replay_is_bitwise_identical():
    c = _case("ignition32", 16)
    import senga

    chem = senga.Chem(c["chem"])
    diff = senga.Diff(None, chem)
    a = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    b = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    a.upload(c["fields"], c["T"], c["itn"])
    b.upload(c["fields"], c["T"], c["itn"])
    a.step(3)
    b.step(3, graph=True)
    fa, ta, _ = a.download()
    fb, tb, _ = b.download()
    assert np.array_equal(fa, fb) and np.array_equal(ta, tb)


def test_mass_conservation_periodic():
    """Periodic box: sum of the continuity RHS vanishes to round-off."""
    c = _case("h2_kernels", 16)
    box, _ = _pair(c)
    r, _, _ = box.rhs()
    assert abs(float(np.sum(r[0]))) <= 1e-9 * float(np.sum(np.abs(r[0])))


def test_temper_failure_reports_status_without_fault():
    """An impossible energy makes the Newton inversion fail: the status word
    reports it and the context stays usable (no trap, no hang)."""
    c = _case("ignition32", 16)
    import senga

    chem = senga.Chem(c["chem"])
    diff = senga.Diff(None, chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    bad = c["fields"].copy()
    bad[4, 3, 4, 5] = -1.0e12  # rho E far below any T > 0
    box.upload(bad, c["T"], c["itn"])
    box.temper()
    assert box.status() & 1
    box.upload(c["fields"], c["T"], c["itn"])
    box.step(1)
    f, _, _ = box.download()
    assert np.isfinite(f).all()


@pytest.mark.parametrize("name", ["ignition32", "h2_kernels"])
def test_generated_and_table_driven_thermochemistry_agree(name, monkeypatch):
    """The shipped mechanisms run the generated straight-line kernel; the
    table-driven kernel (any chem.dat) gives the same right-hand side, and
    both match the oracle."""
    c = _case(name, 12)
    box, ref = _pair(c)
    assert box.info()["mech"] in (1, 2)
    r_gen, _, _ = box.rhs()
    monkeypatch.setenv("SENGA_MECH", "generic")
    box2, _ = _pair(c)
    assert box2.info()["mech"] == 0
    r_tab, _, _ = box2.rhs()
    r_o, _, _ = ref.rhs()
    for k in range(r_o.shape[0]):
        assert rel_linf(r_gen[k], r_tab[k]) <= 1e-12, f"field {k}"
        assert rel_linf(r_tab[k], r_o[k]) <= TOL_STATE, f"field {k}"


@pytest.mark.parametrize("key", ["h2_mavt", "onestep"])
def test_golden_fixture_rhs_and_two_steps(key):
    """The committed oracle fixtures (tests/golden/oracle_*.npz, non-cubic
    12x10x8): right-hand side and the state after two RK steps."""
    import os

    import cases
    import senga

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"oracle_{key}.npz"))
    shape = tuple(int(v) for v in g["shape"])
    chem = senga.Chem(os.path.join(cases.DATA, str(g["chem"])))
    diff = senga.Diff(os.path.join(cases.DATA, str(g["diff"])) if str(g["diff"]) else None, chem)
    box = senga.Box(shape, tuple(g["lengths"]), chem, diff, float(g["dt"]))
    box.upload(g["fields"], g["T"], g["itn"])
    r, t, p = box.rhs()
    for k in range(r.shape[0]):
        assert rel_linf(r[k], g["rhs"][k]) <= TOL_STATE, f"rhs field {k}"
    assert rel_linf(t, g["T_rhs"]) <= TOL_STATE
    assert rel_linf(p, g["p_rhs"]) <= TOL_STATE
    box.upload(g["fields"], g["T"], g["itn"])
    box.step(2)
    f2, t2, _ = box.download()
    for k in range(f2.shape[0]):
        assert rel_linf(f2[k], g["fields_2"][k]) <= TOL_STATE, f"field {k}"
    assert rel_linf(t2, g["T_2"]) <= TOL_STATE


@pytest.mark.parametrize("mode", [0, 1])
def test_filter_field_matches_oracle(mode):
    """Three-pass explicit filter of one field on a non-cubic periodic box."""
    import senga
    from oracle import Oracle
    import cases

    rng = np.random.default_rng(3 + mode)
    nx, ny, nz = 24, 20, 16
    f = rng.standard_normal((nz, ny, nx))
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    lengths = (3.1e-3, 2.3e-3, 1.7e-3)
    box = senga.Box((nx, ny, nz), lengths, chem, diff, 1e-8)
    ref = Oracle((nx, ny, nz), lengths, cases.CHEM_1STEP, None, 1e-8)
    assert rel_linf(box.filter_field(f, mode), ref.filter_field(f, mode)) <= 1e-13


@pytest.mark.parametrize("mode", [0, 3])
def test_filter_then_steps_match_oracle(mode):
    """FLTREM between steps (U register only as in the reference, or U and S
    with the dissipative sign), then two RK steps: all fields."""
    c = _case("h2_kernels", 16)
    box, ref = _pair(c)
    box.step(1)
    ref.step(1)
    box.filter(mode)
    ref.filter(mode)
    box.step(2)
    ref.step(2)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"
    assert rel_linf(tg, to) <= TOL_STATE


def test_adaptive_steps_match_oracle():
    """ADAPTT after every step: dt sequence, ERRMAX, INDERR and the state.
    The error register is a sum of stage right-hand sides whose weights
    (b - b_hat) nearly cancel, so its 1e-13 relative differences grow to
    ~1e-8 in ERRMAX and ~1e-9 in the new dt (ERRMAX^(0.49/3))."""
    import senga
    from oracle import Oracle

    c = _case("h2_kernels", 16)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], adaptive=True)
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    ref.set_adaptive(True)
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    for _ in range(3):
        box.step(1)
        ref.step(1)
        tg, eg, ig = box.tstep()
        to, eo, io = ref.tstep()
        assert abs(tg - to) <= 1e-7 * to
        assert abs(eg - eo) <= 1e-5 * eo
        assert ig == io
    g, _, _ = box.download()
    o, _, _ = ref.download()
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL_STATE, f"field {k}"


def test_checkpoint_resume_through_a_restart_dump(tmp_path):
    """Two steps, dump (reference unformatted layout), resume in a fresh
    context from the dump, two more steps: equal to four steps in one go.
    (A dump holds the conserved state only, as the reference's does; the
    temperature seed is re-sent with the state.)"""
    import senga

    c = _case("h2_kernels", 16)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    a = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    a.upload(c["fields"], c["T"], c["itn"])
    a.step(2)
    f2, t2, i2 = a.download()
    p = str(tmp_path / "dmpi.bin")
    senga.dump_write(p, f2, etime=2 * c["dt"], tstep=c["dt"], nspcmx=9)
    a.step(2)
    fa, _, _ = a.download()
    g, sc = senga.dump_read(p, nspcmx=9)
    assert sc["tstep"] == c["dt"]
    b = senga.Box(c["shape"], c["lengths"], chem, diff, sc["tstep"])
    b.upload(g, t2, i2)
    b.step(2)
    fb, _, _ = b.download()
    assert np.array_equal(fa, fb)
