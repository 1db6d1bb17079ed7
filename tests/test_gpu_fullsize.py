"""The named workloads at their own sizes against the oracle.

The other parity tests run the same code on 16^3-20^3 boxes. These run it
where the bench runs it: tile edges at 128 and 256 points, the periodic fold
of a 256-plane box, the NSCBC faces and the filter over 20 steps, and the
batched engine over 50 steps. Every field after the last step must be within
the field-normalised relative L-infinity 1e-10 of the oracle (max|got - want|
/ max|want| per field; the bound of the other parity tests).

Oracle cost on 16 host threads (about 2.8e6 grid-point substage updates/s for
the H2 mechanism): the 128^3 flame 20 steps about 75 s, the 256^3 box 2
steps about 60 s (17 GB of host memory), the three ensemble boxes 50 steps
about 40 s in all.
"""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _compare(got, want, tg, tw, what):
    for k in range(want.shape[0]):
        assert rel_linf(got[k], want[k]) <= TOL, f"{what}: field {k}"
    assert rel_linf(tg, tw) <= TOL, f"{what}: T"


def test_flame_128_twenty_steps_with_filter_every_ten():
    """128^3 inflow/outflow H2 flame (I3 x-left, O1 x-right, y/z periodic),
    20 RK steps with the explicit filter (coded sign, U register) after steps
    10 and 20, as the flame workload runs it (src/senga2.f:96-194)."""
    import cases
    import senga
    from oracle import Oracle

    c = cases.make_case("flame_inout", n=128, seed=11)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"])
    box.set_nscbc(c["bc"])
    box.upload(c["fields"], c["T"], c["itn"])
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"], nend=c["nend"])
    ref.set_bc(c["bc"])
    ref.upload(c["fields"], c["T"], c["itn"])
    for _ in range(2):
        box.step(10, graph=True)
        box.filter(0)
        ref.step(10)
        ref.filter(0)
    got, tg, _ = box.download()
    want, tw, _ = ref.download()
    assert box.status() == 0
    assert np.isfinite(got).all()
    _compare(got, want, tg, tw, "flame 128^3")


def test_h2_kernels_256_two_steps():
    """The headline 256^3 periodic H2/air box, two RK steps through the graph
    path the bench times."""
    import cases
    import senga
    from oracle import Oracle

    c = cases.make_case("h2_kernels", n=256, seed=1)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    box.step(2, graph=True)
    got, tg, _ = box.download()
    assert box.status() == 0
    box.close()
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    ref.upload(c["fields"], c["T"], c["itn"])
    ref.step(2)
    want, tw, _ = ref.download()
    ref.close()
    _compare(got, want, tg, tw, "h2 256^3")


def test_ensemble_boxes_fifty_steps_through_the_batch():
    """Uneven, non-cubic ignition boxes of the ensemble workload (sizes from
    {32, 48, 64, 96}, own seed, u' and kernel peak), advanced 50 RK steps
    together through the batched engine, each against the oracle alone."""
    import cases
    import senga
    from oracle import Oracle

    specs = [((96, 32, 64), 301, 2.5, 1900.0), ((48, 48, 48), 302, 0.7, 1500.0), ((64, 96, 32), 303, 1.6, 1750.0)]
    cs = [cases.ignition_box(s, seed, up, tp) for s, seed, up, tp in specs]
    chem = senga.Chem(cs[0]["chem"])
    diff = senga.Diff(None, chem)
    b = senga.Batch([(c["shape"], c["lengths"], c["dt"]) for c in cs], chem, diff)
    for i, c in enumerate(cs):
        b.upload(i, c["fields"], c["T"], c["itn"])
    b.autotune()
    b.step(50)
    b.sync()
    assert b.status() == 0
    for i, c in enumerate(cs):
        got, tg, _ = b.download(i)
        ref = Oracle(c["shape"], c["lengths"], c["chem"], None, c["dt"])
        ref.upload(c["fields"], c["T"], c["itn"])
        ref.step(50)
        want, tw, _ = ref.download()
        ref.close()
        _compare(got, want, tg, tw, f"ensemble box {c['shape']}")
