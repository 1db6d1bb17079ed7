"""The species kernel with its x derivatives on the FP64 tensor cores
(csrc/species_mma.cu, opt-in with SENGA_SPECIES_MMA=1) against the oracle and
against the stencil form of the same kernel (the default), on all-periodic boxes whose extents are
multiples of 8: cubic and non-cubic, the smallest (8 planes, every halo
wraps), the one-step and the H2 mechanisms, RHS and two RK steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel_linf(a, b):
    s = np.max(np.abs(b))
    return np.max(np.abs(a - b)) / (s if s > 0 else 1.0)


CASES = [("h2_pool", (16, 16, 16)), ("h2_pool", (8, 16, 24)), ("h2_pool", (40, 8, 32)),
         ("ignition32", None), ("ensemble", None)]


def _case(name, shape):
    import cases

    if name == "ensemble":
        return cases.make_case(name, seed=21)
    if shape:
        return cases.make_case(name, seed=77, shape=shape)
    return cases.make_case(name, seed=77)


@pytest.mark.parametrize("name,shape", CASES,
                         ids=[f"{n}-{'x'.join(map(str, s)) if s else 'default'}" for n, s in CASES])
def test_species_mma_matches_oracle_and_stencil_form(name, shape, monkeypatch):
    import senga
    from oracle import Oracle

    c = _case(name, shape)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    monkeypatch.setenv("SENGA_SPECIES_MMA", "1")
    monkeypatch.delenv("SENGA_FUSE", raising=False)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    assert box.species_mma()
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    r, _, _ = box.rhs()
    rr, _, _ = ref.rhs()
    for k in range(rr.shape[0]):
        assert rel_linf(r[k], rr[k]) <= TOL, f"RHS field {k}"

    # the stencil form of the same kernel, in another context
    monkeypatch.delenv("SENGA_SPECIES_MMA")
    st = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    assert not st.species_mma()
    st.upload(c["fields"], c["T"], c["itn"])
    rs, _, _ = st.rhs()
    for k in range(rs.shape[0]):
        assert rel_linf(r[k], rs[k]) <= 1e-12, f"RHS field {k}: tensor-core and stencil forms"

    box.upload(c["fields"], c["T"], c["itn"])
    ref.upload(c["fields"], c["T"], c["itn"])
    box.step(2, graph=True)
    ref.step(2)
    g, tg, _ = box.download()
    o, to, _ = ref.download()
    assert box.status() == 0
    for k in range(o.shape[0]):
        assert rel_linf(g[k], o[k]) <= TOL, f"state field {k}"
    assert rel_linf(tg, to) <= TOL


def test_species_mma_not_taken_where_it_does_not_apply(monkeypatch):
    """Extents that are not multiples of 8 keep the stencil form."""
    import cases
    import senga

    monkeypatch.setenv("SENGA_SPECIES_MMA", "1")
    c = cases.make_case("h2_pool", seed=5, shape=(20, 16, 16))
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    assert not box.species_mma()
