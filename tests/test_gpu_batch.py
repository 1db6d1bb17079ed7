"""Batched ensembles and the serving loop against the single-box path.

A box's result must not depend on its batch mates: every box of a batch, and
every request of the server, is compared with the same box advanced alone
through the single-box context (same kernels, so agreement is expected to the
last bits; the bound is the field-normalised relative L-infinity 1e-12)."""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ensemble_cases():
    import cases

    # uneven, non-cubic boxes with their own seeds, u' and kernel peak T
    out = []
    for seed, n in ((21, None), (22, 16), (23, None)):
        c = cases.make_case("ensemble", n=n, seed=seed)
        out.append(c)
    # shrink the large ones to keep the oracle-free test quick
    return out


def _alone(c, chem, diff, nsteps):
    import senga

    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    box.step(nsteps)
    return box.download()


@pytest.mark.parametrize("form", ["persist", "launches", "auto"])
def test_batch_matches_boxes_run_alone(form, monkeypatch):
    """Both substage forms (one persistent launch, or four launches), and the
    one the autotuner picks."""
    import senga

    if form != "auto":
        monkeypatch.setenv("SENGA_BATCH", form)
    else:
        monkeypatch.delenv("SENGA_BATCH", raising=False)
    cs = _ensemble_cases()
    chem = senga.Chem(cs[0]["chem"])
    diff = senga.Diff(None, chem)
    b = senga.Batch([(c["shape"], c["lengths"], c["dt"]) for c in cs], chem, diff)
    for i, c in enumerate(cs):
        b.upload(i, c["fields"], c["T"], c["itn"])
    tuned = b.autotune()
    assert tuned["grid_stencil"] > 0 and tuned["grid_thermo"] > 0 and tuned["grid"] > 0
    if form != "auto":
        assert tuned["persistent"] == (form == "persist")
    b.step(2)
    b.sync()
    assert b.status() == 0
    for i, c in enumerate(cs):
        got, tg, _ = b.download(i)
        want, tw, _ = _alone(c, chem, diff, 2)
        for k in range(want.shape[0]):
            assert rel_linf(got[k], want[k]) <= TOL, f"box {i} field {k}"
        assert rel_linf(tg, tw) <= TOL


@pytest.mark.parametrize("form", ["persist", "launches"])
def test_server_results_equal_alone_and_in_the_mix(form, monkeypatch):
    """Requests of different sizes and lengths, an arena that holds only a
    few boxes at a time: requests wait for room, are batched while running,
    and each result equals the same request run alone (either substage
    form)."""
    import senga
    import cases

    monkeypatch.setenv("SENGA_BATCH", form)

    reqs = []
    for k, (seed, n, nsteps) in enumerate(((31, 16, 3), (32, 24, 1), (33, 16, 2), (34, 20, 4), (35, 16, 2))):
        c = cases.make_case("ensemble", n=n, seed=seed)
        reqs.append((c, nsteps))
    chem = senga.Chem(reqs[0][0]["chem"])
    diff = senga.Diff(None, chem)
    per_box = max(c["fields"].size for c, _ in reqs) * 8 * 4  # ~ fields + scratch of the largest box
    srv = senga.Server(int(per_box * 2.2), chem, diff)
    ids = [srv.submit(c["shape"], c["lengths"], c["dt"], c["fields"], c["T"], c["itn"], ns) for c, ns in reqs]
    saw_pending = False
    done = 0
    for _ in range(100):
        st = srv.stats()
        saw_pending = saw_pending or st["pending"] > 0 and st["active"] > 0
        done += srv.tick()
        if done == len(reqs):
            break
    assert done == len(reqs)
    assert saw_pending, "the arena should have forced some requests to wait"
    for rid, (c, ns) in zip(ids, reqs):
        got, tg, _, times = srv.result(rid)
        assert times[0] <= times[1] <= times[2]
        want, tw, _ = _alone(c, chem, diff, ns)
        for k in range(want.shape[0]):
            assert rel_linf(got[k], want[k]) <= TOL, f"request {rid} field {k}"
        assert rel_linf(tg, tw) <= TOL


def test_server_point_cap_admits_in_order_and_results_match():
    """With a per-tick point cap of two small boxes, later requests wait for
    earlier ones to finish (not for arena room); results equal runs alone."""
    import senga
    import cases

    reqs = []
    for seed, nsteps in ((41, 2), (42, 1), (43, 3), (44, 1)):
        c = cases.make_case("ensemble", n=16, seed=seed)
        reqs.append((c, nsteps))
    chem = senga.Chem(reqs[0][0]["chem"])
    diff = senga.Diff(None, chem)
    srv = senga.Server(256 * 1024 * 1024, chem, diff)
    srv.set_max_points(2 * 16 ** 3)
    ids = [srv.submit(c["shape"], c["lengths"], c["dt"], c["fields"], c["T"], c["itn"], ns) for c, ns in reqs]
    done = 0
    for _ in range(100):
        done += srv.tick()
        if done == len(reqs):
            break
    assert done == len(reqs)
    times = [srv.result(rid)[3] for rid in ids]  # [submit, admit, done] each
    # the third request was admitted only once the second had finished
    assert times[2][1] >= times[1][2]
    assert times[3][1] >= times[0][2]
    for rid, (c, ns) in zip(ids, reqs):
        got, tg, _, _ = srv.result(rid)
        want, tw, _ = _alone(c, chem, diff, ns)
        for k in range(want.shape[0]):
            assert rel_linf(got[k], want[k]) <= TOL, f"request {rid} field {k}"
