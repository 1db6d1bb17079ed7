"""CPU-only tests: the C ABI library loads and exports its declared symbols,
host-side table construction, configuration checks, INTEGF."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "senga_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(senga_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import senga

    names = _declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(senga.lib, n)]
    assert not missing, missing


def test_chem_tables_h2_match_oracle_and_identities():
    import cases
    import senga
    from oracle import Oracle

    chem = senga.Chem(cases.CHEM_H2)
    assert chem.nspec == 9 and chem.t.nstep == 21 and chem.t.nlind == 2 and chem.t.nbody == 2
    w = chem.table("wmolar")[:9]
    assert np.allclose(w * chem.table("ovwmol")[:9], 1.0, rtol=0, atol=1e-15)
    # AMASCT(1) = AMASCP(1) - R_k  (src/chemin.f:898-901)
    ct = chem.table("amasct")
    cp = chem.table("amascp")
    rg = chem.table("rgspec")
    for s in range(9):
        assert ct[s, 0, 0] == cp[s, 0, 0] - rg[s]
    ref = Oracle((12, 12, 12), (1e-3,) * 3, cases.CHEM_H2, cases.DIFF_H2, 1e-9)
    assert chem.t.alamda == ref.scalar("alamda")
    assert chem.t.prefgb == ref.scalar("prefgb")
    # Lindemann data: ln(A) and E/R conversion (src/chemin.f:841-845)
    assert chem.table("rclind")[0, 0] == math.log(6.37e14)
    diff = senga.Diff(cases.DIFF_H2, chem)
    d = np.ctypeslib.as_array(diff.t.diffco)
    assert np.array_equal(d, np.swapaxes(d, 0, 1))  # symmetric binary diffusion


def test_one_step_mechanism():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_1STEP)
    assert chem.nspec == 2 and chem.t.nstep == 1
    assert math.isclose(chem.table("rparam")[0, 2], 1.5e4, rel_tol=1e-14)  # Ea/R [K]
    # heat release 5250 K * R/W between reactant and product enthalpies
    h = chem.table("amasch")
    assert math.isclose(h[0, 0, 5] - h[1, 0, 5], 5250.0 * 8.3142e3 / 29.0, rel_tol=1e-14)


def test_bad_inputs_return_status_not_abort():
    import senga

    with pytest.raises(senga.SengaError):
        senga.Chem("/nonexistent/chem.dat")
    import cases

    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    with pytest.raises(senga.SengaError, match="status 5"):  # a bounded direction takes NBOUND on both faces
        senga.Box((16, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, nend=(2, 2, 1, 3, 2, 2))
    with pytest.raises(senga.SengaError, match="status 1"):  # bounded x needs 12 points
        senga.Box((11, 16, 16), (1e-3,) * 3, chem, diff, 1e-8, nend=(1, 1, 2, 2, 2, 2))
    # start-up entry points refuse a missing context before touching the device
    t = np.zeros(8)
    assert senga.lib.senga_tempin_host(None, 300.0, senga._dp(t), None, None) == 1
    assert senga.lib.senga_flamin(None, 300.0, 101325.0, 1.0, 1.0, None, None) == 1
    assert senga.lib.senga_deriv_host(None, 0, senga._dp(t), senga._dp(t)) == 1


def test_integf_spectrum_moment():
    """INTEGF on the Passot-Pouquet energy integrand against the closed form."""
    import senga

    CB = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
    f = CB(lambda k, u: k ** 4 * math.exp(-2.0 * k * k))
    senga.lib.senga_integf.argtypes = [CB, C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double)]
    ans = C.c_double()
    rc = senga.lib.senga_integf(f, None, 0.0, 10.0, C.byref(ans))
    assert rc == 0
    exact = 3.0 / 32.0 * math.sqrt(math.pi / 2.0)
    assert abs(ans.value - exact) <= 1e-6 * exact


def test_case_generator_state_is_consistent():
    """Conserved state rebuilds the IC temperature through the e(T) polynomial."""
    import cases

    c = cases.make_case("ignition32", n=12)
    f = c["fields"]
    assert f.shape == (7, 12, 12, 12)
    assert np.allclose(f[5] + f[6], f[0], rtol=1e-14)
    assert c["dt"] > 0 and np.isfinite(f).all()
