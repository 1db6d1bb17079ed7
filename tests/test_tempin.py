"""TEMPIN, the start-up temperature (src/tempin.f:58-524).

CPU: the oracle's bracketing and bisection recover the temperature a state
was built from (to the residual tolerance 1e-4 J/m^3) and its ITNDEX, reach
the same root from guesses below and above it, agree with the host bisection
used for restart dumps on the reference's own 1-step casefile, and count the
points whose root lies outside [200, 3000] K. GPU: the device kernel returns
the oracle's T bit for bit (both round without contraction), its ITNDEX and
p, flags the failures in the status word, and a step from its T equals a step
from the exact one.
"""
import os

import numpy as np
import pytest

from conftest import rel_linf

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [("h2_kernels", dict(n=16)), ("ignition32", dict(n=16)), ("flame_inout", dict(shape=(24, 8, 8)))]


def _case(name, kw):
    import cases

    return cases.make_case(name, **kw)


def _oracle(c):
    from oracle import Oracle

    o = Oracle(c["shape"], c["lengths"], c["chem"], c.get("diff"), c["dt"], nend=c.get("nend", (2,) * 6))
    o.upload(c["fields"], np.ones_like(c["T"]), np.zeros_like(c["itn"]))
    return o


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_oracle_recovers_built_temperature(name, kw):
    c = _case(name, kw)
    o = _oracle(c)
    T, itn, p, nfail = o.tempin(300.0)
    assert nfail == (0, 0)
    assert np.max(np.abs(T - c["T"])) < 1e-5  # |R| < 1e-4 J/m^3 over rho cv ~ 1e3
    assert np.array_equal(itn, c["itn"])
    o2 = _oracle(c)
    o2.upload(c["fields"], c["T"], c["itn"])
    _, t_ref, p_ref = o2.rhs()  # TEMPER from the exact T: its pressure
    assert rel_linf(p, p_ref) <= 1e-9


def test_oracle_root_independent_of_guess():
    c = _case("h2_kernels", dict(n=16))
    t_lo = _oracle(c).tempin(250.0)[0]   # steps up
    t_hi = _oracle(c).tempin(2900.0)[0]  # steps down
    assert np.max(np.abs(t_lo - t_hi)) < 1e-5


def test_oracle_matches_host_bisection_on_reference_dump():
    """The reference's own 1-step restart dump (no temperature in the file)."""
    import cases
    import senga

    chem = senga.Chem(os.path.join(HERE, "golden", "casefile_1step_chem.dat"))
    fields, _ = senga.dump_read(os.path.join(HERE, "golden", "dmpi_1step_1001.dat"), formatted=True)
    t_host, itn_host = cases.temperature_from_state(chem, fields)
    from oracle import Oracle

    o = Oracle((1001, 1, 1), (1e-2, 1e-3, 1e-3), os.path.join(HERE, "golden", "casefile_1step_chem.dat"), None, 1e-9,
               nend=(1, 1, 2, 2, 2, 2))
    o.upload(fields, np.ones_like(t_host), np.zeros_like(itn_host))
    T, itn, p, nfail = o.tempin(300.0)
    assert nfail == (0, 0)
    assert np.max(np.abs(T - t_host)) < 1e-5
    assert np.array_equal(itn, itn_host)


def test_oracle_counts_roots_outside_limits():
    c = _case("ignition32", dict(n=16))
    f = c["fields"].copy()
    f[4, 0, 0, :4] *= 10.0  # far more energy than 3000 K holds
    o = _oracle(dict(c, fields=f))
    T, itn, p, nfail = o.tempin(300.0)
    assert nfail[0] == 4 and nfail[1] == 0
    assert np.all(T[0, 0, :4] == 3000.0)  # the last upward step


# ----------------------------------------------------------------- GPU
def _box(c):
    import senga

    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c.get("diff"), chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c.get("nend", (2,) * 6))
    if "bc" in c:
        box.set_nscbc(c["bc"])
    return box


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("trin", [300.0, 2000.0])
def test_gpu_tempin_matches_oracle_bitwise(name, kw, trin):
    c = _case(name, kw)
    box = _box(c)
    box.upload(c["fields"], np.ones_like(c["T"]), np.zeros_like(c["itn"]))
    T, itn, p = box.tempin(trin)
    To, itno, po, nfail = _oracle(c).tempin(trin)
    assert nfail == (0, 0)
    assert np.array_equal(T, To)
    assert np.array_equal(itn, itno)
    assert np.array_equal(p, po)
    assert box.status() & 6 == 0


@pytest.mark.gpu
def test_gpu_tempin_flags_roots_outside_limits():
    c = _case("ignition32", dict(n=16))
    f = c["fields"].copy()
    f[4, 0, 0, :4] *= 10.0
    box = _box(c)
    box.upload(f, np.ones_like(c["T"]), np.zeros_like(c["itn"]))
    T, itn, p = box.tempin(300.0)
    To = _oracle(dict(c, fields=f)).tempin(300.0)[0]
    assert np.array_equal(T, To)
    assert box.status() & 2


@pytest.mark.gpu
def test_gpu_step_from_tempin_equals_step_from_exact_temperature():
    c = _case("h2_kernels", dict(n=16))
    a, b = _box(c), _box(c)
    a.upload(c["fields"], np.ones_like(c["T"]), np.zeros_like(c["itn"]))
    a.tempin(800.0)
    b.upload(c["fields"], c["T"], c["itn"])
    a.step(2)
    b.step(2)
    fa, ta, _ = a.download()
    fb, tb, _ = b.download()
    for k in range(fa.shape[0]):
        assert rel_linf(fa[k], fb[k]) <= 1e-10, k
    assert rel_linf(ta, tb) <= 1e-10
