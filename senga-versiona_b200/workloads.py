"""Ensemble and serving workloads (benchmark drivers built on the public API).

ensemble: 64 independent periodic boxes, each axis drawn from {32,48,64,96},
    one-step chemistry, per-box seed, u' ~ U[0.5, 3] m/s, kernel peak
    T ~ U[1400, 2000] K, each box at its own CFL-0.5 dt; K RK steps advanced
    (a) together by the batched engine and (b) one box at a time through the
    single-box path; aggregate GPSU/s of both.
serve: a seeded Poisson stream of requests (mean rate 20/s) drawn from the
    ensemble distribution plus 128^3 boxes with probability 0.1, each asking
    for N ~ U[20, 200] RK steps, submitted in real time to the serving loop;
    p50/p99 time-to-completion and aggregate GPSU/s, against plain
    sequential solves of the same requests (per-shape single-box step time
    x steps, measured on the same GPU).
flame: the 128^3 inflow/outflow H2/air flame box (NSCBC I3 inflow at
    x-left, O1 outflow at x-right, y/z periodic, mixture-averaged), K RK
    steps with the explicit filter every 10 steps (coded TWFACT sign, U
    register only, as the reference's FLTREM would run).
Initial states of the served requests come from a cache of two generated
boxes per shape; each request rescales the velocity of its template to its
own u' (kinetic energy updated in rho E). Inputs are synthetic.
"""
import math
import time

import numpy as np

import cases
import senga

SIZES = (32, 48, 64, 96)


def ensemble_cases(nbox=64, seed=1000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nbox):
        shape = tuple(int(rng.choice(SIZES)) for _ in range(3))
        up = float(rng.uniform(0.5, 3.0))
        tpk = float(rng.uniform(1400.0, 2000.0))
        out.append(cases.ignition_box(shape, seed + 17 * i + 1, up, tpk))
    return out


def _events(stream, device=0):
    import torch

    s = torch.cuda.ExternalStream(stream, device=device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    return s, a, b


def run_ensemble(steps=50, warmup=3, nbox=64, device=0, seed=1000):
    cs = ensemble_cases(nbox, seed)
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    gpsu = sum(5 * c["fields"][0].size for c in cs) * steps
    # batched
    b = senga.Batch([(c["shape"], c["lengths"], c["dt"]) for c in cs], chem, diff, device=device)
    for i, c in enumerate(cs):
        b.upload(i, c["fields"], c["T"], c["itn"])
    tuned = b.autotune()
    b.step(warmup)
    b.sync()
    s, e0, e1 = _events(b.stream, device)
    e0.record(s)
    b.step(steps)
    e1.record(s)
    b.sync()
    t_batch = e0.elapsed_time(e1) / 1e3
    status = b.status()
    b.close()
    # one box at a time through the single-box path
    t_seq = 0.0
    for c in cs:
        box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], device=device)
        box.upload(c["fields"], c["T"], c["itn"])
        box.step(1, graph=True)
        box.sync()
        s, e0, e1 = _events(box.stream, device)
        e0.record(s)
        box.step(steps, graph=True)
        e1.record(s)
        box.sync()
        t_seq += e0.elapsed_time(e1) / 1e3
        box.close()
    return {"gpsu": gpsu, "t_batched_s": t_batch, "t_sequential_s": t_seq, "batched_gpsu_s": gpsu / t_batch,
            "sequential_gpsu_s": gpsu / t_seq, "speedup": t_seq / t_batch, "autotune": tuned,
            "boxes": nbox, "points": int(sum(c["fields"][0].size for c in cs)), "status_word": status}


def run_flame(steps=20, warmup=3, n=128, device=0, seed=11, filter_every=10, filter_mode=0):
    chem = senga.Chem(cases.CHEM_H2)
    c = cases.make_case("flame_inout", n=n, seed=seed)
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], nend=c["nend"], device=device)
    box.set_nscbc(c["bc"])
    box.upload(c["fields"], c["T"], c["itn"])
    box.step(warmup, graph=True)
    box.sync()
    s, e0, e1 = _events(box.stream, device)
    e0.record(s)
    done = 0
    while done < steps:
        k = min(filter_every, steps - done)
        box.step(k, graph=True)
        done += k
        if done % filter_every == 0:
            box.filter(filter_mode)
    e1.record(s)
    box.sync()
    t = e0.elapsed_time(e1) / 1e3
    f, T, _ = box.download()
    status = box.status()
    box.close()
    npts = n ** 3
    return {"gpsu": npts * 5 * steps, "seconds": t, "gpsu_s": npts * 5 * steps / t, "points": npts,
            "finite": bool(np.isfinite(f).all()), "t_min": float(T.min()), "t_max": float(T.max()),
            "status_word": status, "dt": c["dt"]}


def serve_requests(nreq=2000, rate=20.0, seed=2024, p_big=0.1):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
    reqs = []
    for i in range(nreq):
        big = rng.uniform() < p_big
        shape = (128, 128, 128) if big else tuple(int(rng.choice(SIZES)) for _ in range(3))
        reqs.append(dict(t=float(t[i]), shape=shape, nsteps=int(rng.integers(20, 201)),
                         uprime=float(rng.uniform(0.5, 3.0)), tpeak=float(rng.uniform(1400.0, 2000.0)),
                         template=int(rng.integers(0, 2))))
    return reqs


def _template(cache, shape, k):
    key = (shape, k)
    if key not in cache:
        c = cases.ignition_box(shape, 7000 + 31 * k + sum(shape), 1.0, 1700.0)
        rho = c["fields"][0]
        ke = 0.5 * (c["fields"][1] ** 2 + c["fields"][2] ** 2 + c["fields"][3] ** 2) / rho
        cache[key] = (c, ke)
    return cache[key]


def _instance(cache, r):
    """The request's state: its template with velocity rescaled to u'."""
    c, ke = _template(cache, r["shape"], r["template"])
    f = c["fields"].copy()
    s = r["uprime"] / 1.0
    f[1:4] *= s
    f[4] += (s * s - 1.0) * ke
    return c, f


def run_serve(nreq=2000, rate=20.0, seed=2024, device=0, arena_frac=0.6, max_points=32 * 1024 * 1024):
    import torch

    reqs = serve_requests(nreq, rate, seed)
    cache = {}
    for r in reqs:  # build every template before the clock starts
        _template(cache, r["shape"], r["template"])
    chem = senga.Chem(cases.CHEM_1STEP)
    diff = senga.Diff(None, chem)
    free, _ = torch.cuda.mem_get_info(device)
    arena = int(min(arena_frac * free, 120e9))
    srv = senga.Server(arena, chem, diff, device=device)
    # about 32 M points per tick (~0.1 s): requests run close to arrival
    # order instead of all sharing one long tick
    srv.set_max_points(max_points)
    t0 = time.perf_counter()
    ids = {}
    i = 0
    done = 0
    while done < nreq:
        now = time.perf_counter() - t0
        while i < nreq and reqs[i]["t"] <= now:
            r = reqs[i]
            c, f = _instance(cache, r)
            # the CFL bound is set by the sound speed (~350-850 m/s) plus |u|
            # (< 10 m/s): the template's dt with a 3 % margin covers u' <= 3 m/s
            dt = 0.97 * c["dt"]
            ids[srv.submit(r["shape"], c["lengths"], dt, f, c["T"], c["itn"], r["nsteps"])] = i
            i += 1
        st = srv.stats()
        if st["active"] == 0 and st["pending"] == 0:
            if i < nreq:
                time.sleep(max(0.0, min(0.01, reqs[i]["t"] - (time.perf_counter() - t0))))
            continue
        done += srv.tick()
    wall = time.perf_counter() - t0
    st = srv.stats()
    lat = []
    for rid, k in ids.items():
        _, _, _, tm = srv.result(rid)
        lat.append(tm[2] - reqs[k]["t"])
    srv.close()
    lat = np.array(lat)
    gpsu = st["gpsu"]
    # plain sequential solves: per-shape single-box RK step time x steps
    t_seq = 0.0
    step_time = {}
    for shape in sorted(set(r["shape"] for r in reqs)):
        c, _ = _template(cache, shape, 0)
        box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], device=device)
        box.upload(c["fields"], c["T"], c["itn"])
        box.step(2, graph=True)
        box.sync()
        s, e0, e1 = _events(box.stream, device)
        e0.record(s)
        box.step(3, graph=True)
        e1.record(s)
        box.sync()
        step_time[shape] = e0.elapsed_time(e1) / 3e3
        box.close()
    for r in reqs:
        t_seq += r["nsteps"] * step_time[r["shape"]]
    return {"requests": nreq, "rate_per_s": rate, "wall_s": wall, "gpsu": int(gpsu), "served_gpsu_s": gpsu / wall,
            "busy_gpsu_s": gpsu / max(1e-9, wall - reqs[0]["t"]), "sequential_gpsu_s": gpsu / t_seq,
            "sequential_s": t_seq, "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()), "arena_bytes": arena, "max_points_per_tick": max_points}


if __name__ == "__main__":
    # python senga-versiona_b200/workloads.py ensemble [steps] [persist|launches|auto]
    import json
    import os
    import sys

    what = sys.argv[1] if len(sys.argv) > 1 else "ensemble"
    if what != "ensemble":
        raise SystemExit("usage: workloads.py ensemble [steps] [persist|launches|auto]")
    nsteps = int(sys.argv[2]) if len(sys.argv) > 2 else 20
    form = sys.argv[3] if len(sys.argv) > 3 else "auto"
    if form == "auto":
        os.environ.pop("SENGA_BATCH", None)
    else:
        os.environ["SENGA_BATCH"] = form
    r = run_ensemble(steps=nsteps, warmup=3)
    print(json.dumps({"form": form, **{k: r[k] for k in ("batched_gpsu_s", "sequential_gpsu_s", "speedup",
                                                          "autotune", "status_word", "boxes", "points")}}))
