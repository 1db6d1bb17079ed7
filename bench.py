"""Benchmark: grid-point substage updates per second (GPSU/s) of the plain
RHS + RK path on the 256^3 periodic H2/air ignition-kernel workload
(mixture-averaged transport, 21-step mechanism, FP64).

A "step" is one RK4(3)5 time step = 5 substages over the whole box, so
GPSU per step = 5 * nx*ny*nz. Inputs are synthetic (seeded turbulence and
hot kernels, see cases.py). The state (1.9 GB for 256^3 H2) is far larger
than L2, so no cache flush is needed between timed steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 runs N independent replicas (one box per GPU, no inter-GPU exchange:
the path does not shard in this build), value = sum over ranks.
--impl reference times the CPU restatement of the reference (the oracle:
the Fortran reference cannot be compiled here) with all host threads on the
same 256^3 state, one RK substage per timed step; the device library is not
loaded on that path.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "senga-versiona_b200"))

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def peaks():
    try:
        with open(PEAKS) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def dram_traffic_per_point():
    """DRAM bytes per point of each kernel from the committed ncu summary
    (dram__bytes_read.sum + dram__bytes_write.sum of one capture, per point;
    the traffic grows in proportion to the point count)."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic_h2_kernels.json")) as fh:
            return json.load(fh)["dram_bytes_per_point"]
    except Exception:
        return {}


def compulsory_bytes_per_gpsu(nspec):
    # read+write of the S and U registers and of T (Newton seed): 8*(4*Nc+2)
    return 8 * (4 * (5 + nspec) + 2)


def kernel_bytes_per_point(nspec, adaptive=False):
    """Algorithmic bytes per interior point of each kernel family: distinct
    fields read + written, 8 B each (the interval index 4 B); stencil halo
    re-reads count zero."""
    S, nc = nspec, 5 + nspec
    # reads U (nc), T, ITNDEX; writes T, ITNDEX, p, lambda, lambda/cp, mu,
    # rho*D_k, h_k, h_mix, wdot_k, u, v, w, E, Y_k
    thermo = 8 * (nc + 1) + 4 + 8 * (10 + 4 * S) + 4
    flow = 8 * (4 + 3 + 1 + 1 + 1 + 1 + 1) + 8 * (5 + 1)
    species_a = 8 * (3 + 1 + 1 + 4 * S) + 8 * (S + 3 + 1 + 1)
    species_b = 8 * (3 + 1 + 5 + 1 + 2 * S + nc) + 8 * (2 * nc) + (16 * nc if adaptive else 0)
    # the two species kernels as one: reads rho u, rho v, rho w, the flow RHS
    # (5), DIVM, Y_k, rho D_k, h_k, the CHRATE rate, h_mix, S; writes S and U
    species = 8 * (3 + 5 + 1 + 4 * S + 1 + nc) + 8 * (2 * nc) + (16 * nc if adaptive else 0)
    return {"thermo": thermo, "flow": flow, "species_a": species_a, "species_b_rk": species_b, "species": species}


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.fh.flush()
        self.fh.seek(0)
        rows = [r.split(",") for r in self.fh.read().strip().splitlines() if r.strip()]
        os.unlink(self.fh.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def oracle_box(n, case="h2_kernels"):
    """The workload's state on an n^3 grid, built and held by the oracle
    alone: chem.dat is read by the oracle's own table reader, so the device
    library is never loaded on this path."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    from oracle import Oracle, OracleChem

    c = cases.make_case(case, n=n, seed=1, chem_reader=OracleChem)
    o = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    o.upload(c["fields"], c["T"], c["itn"])
    return o, c


def time_substages(o, count, threads, irk0=0):
    """Wall time of `count` consecutive RK substages of the oracle on
    `threads` OpenMP threads; returns (seconds, next substage index)."""
    o.set_threads(threads)
    irk = irk0
    t0 = time.perf_counter()
    for _ in range(count):
        o.substage(irk % 5 + 1)
        irk += 1
    return time.perf_counter() - t0, irk


def cpu_baseline_sample(n=128):
    """Reported CPU baseline: the oracle (C++ restatement of the reference's
    path, reference loop order, -O2 without contraction) on an n^3 sample of
    the headline state, one RK substage on 1 thread and one on all host
    threads (OpenMP over k-planes). Returns the cpu_baseline object."""
    threads = os.cpu_count() or 1
    o, _ = oracle_box(n)
    pts = n ** 3
    t1, irk = time_substages(o, 1, 1)
    tall, _ = time_substages(o, 1, threads, irk)
    o.close()
    return {"value": pts / tall, "unit": "GPSU/s", "cores": threads, "kind": "port",
            "sample": f"{n}^3 periodic H2/air state of the headline workload, one RK substage per timing",
            "one_core_value": pts / t1, "cpu_model": cpu_model(),
            "seconds": {"one_core": t1, "all_cores": tall}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="grid extent (cubic); 256 is the named workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the 128^3 flame and the batched ensemble measured beside the headline")
    ap.add_argument("--workload", default="h2_kernels", choices=["h2_kernels", "ensemble", "serve", "flame"],
                    help="h2_kernels: the 256^3 headline; ensemble: 64 batched boxes vs one at a time; "
                         "serve: Poisson request stream through the serving loop; "
                         "flame: 128^3 NSCBC inflow/outflow flame, filter every 10 steps")
    ap.add_argument("--requests", type=int, default=2000, help="serve: number of requests")
    ap.add_argument("--boxes", type=int, default=64, help="ensemble: number of boxes")
    args = ap.parse_args()
    if args.workload != "h2_kernels":
        return workload_main(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric, unit = "grid-point substage updates/s", "GPSU/s"
    workload = {"workload": f"h2_kernels_{args.n}^3", "grid": [args.n] * 3, "mechanism": "H2/air 9 sp 21 steps",
                "transport": "mixture-averaged", "boundaries": "triply periodic", "substages_per_step": 5,
                "parallelism": f"replicas x{args.gpus}", "l2": "inputs larger than L2 (no flush needed)"}

    if args.impl == "reference":
        if rank != 0:
            return
        # The reference's path on the host cores: the oracle on the same
        # n^3 state, all host threads. One timed step = one RK substage of
        # the whole box (a bounded sample: a full 5-substage step of 256^3
        # takes about half a minute on 16 cores); the metric is per
        # grid-point substage update, so the sample's rate is the workload's.
        threads = os.cpu_count() or 1
        o, c = oracle_box(args.n)
        pts = args.n ** 3
        _, irk = time_substages(o, args.warmup, threads)
        dt, _ = time_substages(o, args.steps, threads, irk)
        o.close()
        v = pts * args.steps / dt
        workload["sample"] = f"{args.n}^3 state, one RK substage per timed step"
        line = {"impl": "reference", "metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(args.steps, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": workload,
                "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": f"{args.n}^3 periodic H2/air state, {args.steps} timed RK substage(s) "
                                           f"after {args.warmup} warm-up substage(s), oracle (C++ restatement)",
                                 "cpu_model": cpu_model()},
                "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import cases
    import senga

    c = cases.make_case("h2_kernels", n=args.n, seed=1 + rank)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], device=local)
    box.upload(c["fields"], c["T"], c["itn"])
    npts = c["shape"][0] * c["shape"][1] * c["shape"][2]
    workload["thermochemistry_kernel"] = {0: "table-driven", 1: "generated 1-step", 2: "generated H2"}[box.info()["mech"]]
    workload["species_kernels"] = "fused: one launch per substage" if box.species_fused() else "separate"

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # warm-up (graph capture happens here)
    box.step(max(args.warmup, 3), graph=True)
    box.sync()
    # per-kernel profile of one step (device events, after warm-up)
    prof, launches_per_step = box.profile_step()
    box.sync()

    stream = torch.cuda.ExternalStream(box.stream, device=local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    time.sleep(0.4)
    ev0.record(stream)
    box.step(args.steps, graph=True)
    ev1.record(stream)
    box.sync()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    import replicas

    ms = replicas.max_over_ranks(ev0.elapsed_time(ev1), device="cuda")
    status = box.status()
    gpsu = replicas.job_rate(npts, 5 * args.steps, world, ms / 1e3)

    # end-to-end through the host C ABI: per step, upload the state from pinned
    # host memory, advance one RK step, download the state.
    nc = 5 + chem.nspec
    pin_f = torch.empty((nc,) + box.shape, dtype=torch.float64, pin_memory=True).numpy()
    pin_t = torch.empty(box.shape, dtype=torch.float64, pin_memory=True).numpy()
    pin_i = torch.empty(box.shape, dtype=torch.int32, pin_memory=True).numpy()
    f0, t0_, i0 = box.download()
    pin_f[...] = f0
    pin_t[...] = t0_
    pin_i[...] = i0
    # results land in page-locked buffers too (pageable copies run at a
    # fraction of the link speed)
    out_f = torch.empty((nc,) + box.shape, dtype=torch.float64, pin_memory=True).numpy()
    out_t = torch.empty(box.shape, dtype=torch.float64, pin_memory=True).numpy()
    out_i = torch.empty(box.shape, dtype=torch.int32, pin_memory=True).numpy()
    e2e_steps = max(1, min(args.steps, 3))
    barrier()
    t_e0 = time.perf_counter()
    for _ in range(e2e_steps):
        box.upload(pin_f, pin_t, pin_i)
        box.step(1, graph=True)
        box.download(out=(out_f, out_t, out_i))
    t_e = replicas.max_over_ranks(time.perf_counter() - t_e0, device="cuda")
    state_bytes = nc * npts * 8 + npts * 8 + npts * 4
    e2e_serial = replicas.job_rate(npts, 5 * e2e_steps, world, t_e)

    # the same per-step work for a queue of independent boxes (ensembles,
    # serving): two contexts on their own streams, each job = page-locked
    # upload + one graph-launched RK step + download. One step runs at a
    # time; the next job's upload and the previous job's download run on the
    # copy engines while it computes.
    box2 = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"], device=local)
    box2.upload(pin_f, pin_t, pin_i)
    box2.step(1, graph=True)  # graph capture outside the timed region
    box2.sync()
    outs = [(out_f, out_t, out_i),
            tuple(torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32,
                              pin_memory=True).numpy() for a in (out_f, out_t, out_i))]
    pair = (box, box2)
    jobs = 2 * max(args.steps, 2)
    barrier()
    t_p0 = time.perf_counter()
    for j in range(jobs):
        b, prev = pair[j % 2], pair[(j + 1) % 2]
        b.upload_async(pin_f, pin_t, pin_i)
        if j > 0:
            prev.sync()  # job j-1's step is done: fetch its result
            prev.download_async(*outs[(j - 1) % 2])
        b.step(1, graph=True)
    last = pair[(jobs - 1) % 2]
    last.sync()
    last.download_async(*outs[(jobs - 1) % 2])
    box.sync()
    box2.sync()
    t_p = replicas.max_over_ranks(time.perf_counter() - t_p0, device="cuda")
    del box2
    e2e = {"value": replicas.job_rate(npts, 5 * jobs, world, t_p), "unit": unit, "h2d_bytes_per_step": state_bytes,
           "d2h_bytes_per_step": state_bytes,
           "call": "two contexts alternating senga_upload_state_async + senga_step_graph(1) + "
                   "senga_download_state_async from/to page-locked host buffers, one job per step, "
                   "copies overlapping the other context's step",
           "serial": {"value": e2e_serial,
                      "call": "senga_upload_state_host + senga_step_graph(1) + senga_download_state_host per step"}}

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    hbm, peak_kind = peaks()
    fp64 = senga.fp64_peak(local)  # FP64 FMA probe: denominator of the thermochemistry kernel's FP64 figure
    kb = kernel_bytes_per_point(chem.nspec)
    kern = {}
    tot = sum(prof.values())
    for k, t_ms in prof.items():
        launch_ms = t_ms / 5.0
        ach = kb[k] * npts / (launch_ms / 1e3) / 1e9
        kern[k] = {"ms_per_launch": launch_ms, "share": t_ms / tot, "alg_bytes_per_point": kb[k],
                   "achieved_gbs": ach, "frac_hbm": ach / hbm}
    stencil = max((k for k in ("flow", "species_a", "species_b_rk", "species") if k in prof), key=lambda k: prof[k])
    dom = max(prof, key=prof.get)
    rk = kern[stencil]
    tpp = dram_traffic_per_point().get(stencil)
    traffic = tpp * npts if tpp else None
    step_ms = ms / args.steps
    whole = gpsu / world * compulsory_bytes_per_gpsu(chem.nspec) / 1e9
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_baseline_sample(min(args.n, 128))
    extras = None
    if not args.no_extras and world == 1:
        # the other named single-GPU workloads, device-timed on the same
        # GPU: the 128^3 NSCBC flame (20 steps, filter every 10) and the
        # 64-box ensemble (50 steps) batched against one box at a time
        box.close()
        import workloads

        fl = workloads.run_flame(steps=20, warmup=3, device=local)
        en = workloads.run_ensemble(steps=50, warmup=3, nbox=64, device=local)
        # the serving workload's request stream cut to its first 300 requests
        # (Poisson 20/s, the ensemble's box distribution plus 10% 128^3
        # cases, 20-200 steps each), so that the default run stays short
        sv = workloads.run_serve(nreq=300, device=local)
        extras = {
            "flame_128": {"workload": "flame_inout_128^3_H2_nscbc_I3_O1, filter every 10 steps", "steps": 20,
                          "value": fl["gpsu_s"], "unit": unit, "ms_per_step": 1e3 * fl["seconds"] / 20,
                          "finite": fl["finite"], "status_word": fl["status_word"]},
            "ensemble_64": {"workload": "64 boxes, axes from {32,48,64,96}, 1-step chemistry", "steps": 50,
                            "points": en["points"], "batched_value": en["batched_gpsu_s"],
                            "sequential_value": en["sequential_gpsu_s"], "unit": unit,
                            "batched_vs_sequential": en["speedup"], "status_word": en["status_word"]},
            "serve_300": {"workload": "first 300 requests of the serving stream (Poisson 20/s, 1-step chemistry, "
                                      "boxes from {32,48,64,96}^3 plus 10% 128^3, 20-200 steps)",
                          "requests": sv["requests"], "wall_s": sv["wall_s"], "served_value": sv["served_gpsu_s"],
                          "sequential_value": sv["sequential_gpsu_s"], "unit": unit, "p50_s": sv["p50_s"],
                          "p99_s": sv["p99_s"], "mean_latency_s": sv["mean_latency_s"]}}
    line = {
        "metric": metric, "value": gpsu, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload,
        "roofline": {"bound": "hbm", "kernel": stencil, "achieved": rk["achieved_gbs"], "peak": hbm,
                     "unit": "GB/s", "frac": rk["frac_hbm"], "traffic": traffic, "peak_kind": peak_kind,
                     "traffic_source": "profiles/dram_traffic_h2_kernels.json (128^3 capture, per point x points)"},
        "dominant_kernel": dom,
        "kernels": kern,
        "whole_step_hbm_frac": whole / hbm,
        "fp64_peak_tflops_measured": fp64,
        "compulsory_bytes_per_gpsu": compulsory_bytes_per_gpsu(chem.nspec),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "workloads": extras,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "status_word": status,
    }
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def workload_main(args):
    """Ensemble and serving workloads (single GPU)."""
    import torch

    import workloads

    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            cb = cpu_baseline_sample(48)
            print(json.dumps({"impl": "reference", "metric": "grid-point substage updates/s", "value": cb["value"],
                              "unit": "GPSU/s", "n_gpus": 1, "higher_is_better": True,
                              "config": {"workload": args.workload, "sample": "48^3 periodic H2/air state"},
                              "cpu_baseline": cb,
                              "e2e": {"value": cb["value"], "unit": "GPSU/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if args.workload == "ensemble":
        steps = args.steps if args.steps != 5 else 50
        r = workloads.run_ensemble(steps=steps, warmup=max(3, args.warmup), nbox=args.boxes)
        line = {"metric": "grid-point substage updates/s", "value": r["batched_gpsu_s"], "unit": "GPSU/s",
                "n_gpus": 1, "steps": steps, "warmup": max(3, args.warmup),
                "ms_per_step": 1e3 * r["t_batched_s"] / steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "ensemble_64_boxes_{32,48,64,96}^3_1step", "boxes": r["boxes"],
                           "points": r["points"], "autotune": r["autotune"]},
                "sequential_value": r["sequential_gpsu_s"], "batched_vs_sequential": r["speedup"],
                "status_word": r["status_word"]}
    elif args.workload == "flame":
        steps = args.steps if args.steps != 5 else 20
        r = workloads.run_flame(steps=steps, warmup=max(3, args.warmup))
        line = {"metric": "grid-point substage updates/s", "value": r["gpsu_s"], "unit": "GPSU/s", "n_gpus": 1,
                "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": 1e3 * r["seconds"] / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": "flame_inout_128^3_H2_nscbc_I3_O1", "filter": "every 10 steps, coded TWFACT "
                           "sign, U register only", "points": r["points"]},
                "finite": r["finite"], "T_range": [r["t_min"], r["t_max"]], "status_word": r["status_word"]}
    else:
        r = workloads.run_serve(nreq=args.requests)
        line = {"metric": "grid-point substage updates/s", "value": r["served_gpsu_s"], "unit": "GPSU/s",
                "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"serve_poisson_{r['requests']}req_20per_s", "arena_bytes": r["arena_bytes"],
                           "max_points_per_tick": r["max_points_per_tick"]},
                "p50_s": r["p50_s"], "p99_s": r["p99_s"], "mean_latency_s": r["mean_latency_s"], "wall_s": r["wall_s"],
                "gpsu": r["gpsu"], "sequential_value": r["sequential_gpsu_s"],
                "served_vs_sequential": r["served_gpsu_s"] / r["sequential_gpsu_s"],
                "busy_value": r["busy_gpsu_s"]}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
