"""Benchmark of the Ndyn MD timestep path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c4]
                    [--impl ours|reference] [--precision mixed|fp64]

A step is one MD timestep (the dynamics loop body, src/nd.f90:138-178) of
every system of the workload.  Default workload (c4): 512 independent
replicas (half Cu Morse crystals, half LJ argon liquids, 500-20,000 atoms
each, own Berendsen thermostats) stepped together in mixed precision, with
the plain single-system FP64 path timed on a sample of the same replicas
one after another, and the mixed path's force error against FP64 on the
thermalised replicas.  Other workloads: c1 (Cu Morse crystal 4000 atoms,
FP64, NVE), c2 (LJ argon liquid 256,000 atoms, NVT, mixed), c3 (rocksalt
Buckingham 1,048,576 atoms, NPT).

Multi-GPU: the workload does not shard (one system per GPU, no exchange),
so N ranks run N independent replicas ("replicas only"): value is the
aggregate atom-steps/s, time is the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--config", default="c4", choices=["c1", "c2", "c3", "c4", "c5", "c5batch"])
    ap.add_argument("--requests", type=int, default=128, help="c5: requests in the stream")
    ap.add_argument("--rate", type=float, default=200.0, help="c5: Poisson arrivals per s")
    ap.add_argument("--steps-scale", type=float, default=0.05,
                    help="c5: factor on every request's step count")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tpa", type=int, default=0, help="threads per atom (0 = library choice)")
    ap.add_argument("--bare", action="store_true",
                    help="only the warm-up and timed steps (for profiler launch lists): no "
                         "force error, plain baseline, e2e, CPU baseline or kernel timing")
    ap.add_argument("--graph-steps", type=int, default=100,
                    help="steps per CUDA graph (1 = eager launches, as ncu needs)")
    ap.add_argument("--replica-stride", type=int, default=1,
                    help="c4: every S-th replica only (a smaller case of the same "
                         "ensemble, for profiler captures)")
    ap.add_argument("--gather-depth", type=int, default=0,
                    help="neighbour gathers in flight per thread (0 = library choice)")
    return ap.parse_args()


def workload(cfg, scale_cells=None):
    from ndyn_omp_b200 import workloads as W
    if cfg == "c5":
        return [], "mixed"
    if cfg == "c5batch":
        # the first 64 requests of the c5 stream, resident together as one batch
        reqs = W.serving_requests(64, 200.0, seed=5)
        return [W.build_request(r) for r in reqs], "mixed"
    if cfg == "c1":
        return [W.cu_crystal(scale_cells or 10, 300.0, seed=1, quirk="ref")], "fp64"
    if cfg == "c2":
        return [W.ar_liquid(scale_cells or 40, 120.0, seed=2, quirk="fixed")], "mixed"
    if cfg == "c3":
        c = scale_cells or (64, 64, 32)
        return [W.nacl_solid(c, 600.0, seed=3, quirk="fixed")], "mixed"
    return W.replica_ensemble(512, seed=4, quirk="fixed"), "mixed"


WORKLOAD_TEXT = {
    "c1": "Cu FCC 10^3 cells (4000 atoms) Morse D=0.3429 a=1.3588 r0=2.866 rc=6.0 skin 0.5, "
          "NVE, FP64, reference list semantics",
    "c2": "LJ argon liquid 256000 atoms (FCC 40^3, rho*=0.8442, +-0.05 sigma jitter), "
          "eps=0.0104 sigma=3.405 rc=2.5 sigma skin=0.3 sigma, Berendsen 120 K tau=100 steps",
    "c3": "rocksalt Buckingham 1048576 atoms (64x64x32 cells, a=5.64, +-0.02 A), rc=8 "
          "skin 1.6, thermostat 600 K + barostat P=0 (Pparm 10)",
    "c4": "512 replicas (half Cu Morse crystals, half LJ Ar liquids), N log-uniform "
          "[500,20000] in whole FCC cells, T uniform [100,1500] K, own thermostats",
    "c5batch": "the first 64 requests of the c5 stream (Morse/LJ/Buckingham, 1e3-2e5 atoms, "
               "NVE/NVT/NPT, 2.35 M atoms) resident together as one batch",
    "c5": "serving: Poisson stream of MD requests (Morse/LJ/Buckingham, N log-uniform "
          "[1e3,2e5], steps log-uniform [1e3,5e4] x steps-scale, T uniform [100,1500] K, "
          "NVE/NVT/NPT), 150 GB HBM budget, graph blocks of 100 steps",
}


# ---------------------------------------------------------------------------
class ClockSampler:
    """NVML sampling of SM clock and throttle reasons while timing."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index):
        self.samples, self.reasons, self.ok = [], 0, False
        self.max_mhz = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self.nv = pynvml
            # NVML numbers all GPUs of the node; find ours by PCI bus id
            p = torch.cuda.get_device_properties(index)
            bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False
        self._stop = threading.Event()

    def _loop(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    "samples": 0}
        rs = [n for b, n in self.REASONS.items() if self.reasons & b and n != "gpu_idle"]
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": rs, "samples": len(self.samples)}


def hbm_peak():
    try:
        return float(json.load(open(MEASURED))["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_atom(cfg):
    """DRAM bytes per atom of one pair-kernel launch from the committed ncu
    summary (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", f"k_pair_{cfg}_traffic.txt")
    try:
        for ln in open(p):
            if ln.startswith("dram_bytes_per_atom:"):
                return float(ln.split(":")[1])
    except OSError:
        return None
    return None


# ---------------------------------------------------------------------------
# the CPU legs time the oracle's reference-flags build (libndyn_oracle_fast:
# -Ofast -march=x86-64-v4 -funsafe-math-optimizations -fopenmp, the release
# flags of the reference's src/Makefile with a portable -march)
CPU_BUILD = "oracle restatement of the reference OpenMP FP64 loop, built with the reference's " \
            "release flags (-Ofast -funsafe-math-optimizations -fopenmp, -march=x86-64-v4)"


def cpu_rate(spec, target_s, threads=None, fixed_steps=None):
    """Oracle (the reference's FP64 OpenMP path restated) on the host cores:
    setup untimed, then the step loop timed.  Returns (atom-steps/s, steps,
    seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py
    from helpers import oracle_from_spec
    threads = threads or os.cpu_count()
    o = oracle_from_spec(spec, threads=threads, fast=True)
    assert o.setup_lists() == 0
    dt = spec["control"]["dt"]
    if fixed_steps is None:
        t0 = time.perf_counter()
        rc, _ = o.run(1, dt, loop_only=True)
        t1 = time.perf_counter() - t0
        steps = int(max(2, min(1000000, target_s / max(t1, 1e-6))))
    else:
        steps = fixed_steps
    t0 = time.perf_counter()
    rc, _ = o.run(steps, dt, loop_only=True)
    el = time.perf_counter() - t0
    assert rc == 0, rc
    n = len(spec["typ"])
    return n * steps / el, steps, el, threads


def spread_sample(specs, atom_budget):
    """Systems spread evenly over the list (sizes and materials as they
    come), as many as the atom budget allows (at least one)."""
    n = len(specs)
    for k in range(n, 0, -1):
        pick = [specs[(j * n) // k] for j in range(k)]
        if sum(len(s["typ"]) for s in pick) <= atom_budget or k == 1:
            return pick, [(j * n) // k for j in range(k)]
    return specs[:1], [0]


def cpu_rate_systems(specs, steps, warmup, threads):
    """The oracle on each system in turn (the reference runs one system at
    a time): warm-up and timed steps per system; returns (atom-steps/s,
    seconds of timed work)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_from_spec
    work = el = 0.0
    for sp in specs:
        o = oracle_from_spec(sp, threads=threads, fast=True)
        assert o.setup_lists() == 0
        dt = sp["control"]["dt"]
        if warmup:
            o.run(warmup, dt, loop_only=True)
        t0 = time.perf_counter()
        rc, _ = o.run(steps, dt, loop_only=True)
        el += time.perf_counter() - t0
        assert rc == 0, rc
        work += len(sp["typ"]) * steps
    return work / el, el


def n_atoms(specs):
    return sum(len(s["typ"]) for s in specs)


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def force_error(specs, states, local, warm=0):
    """Relative L2 force error of the mixed path against the FP64 path on the
    given configurations: over all atoms of all systems, and the largest
    per-system value.  warm > 0: the configurations are first thermalised
    by that many FP64 steps (a perfect lattice has zero net forces, against
    which no relative error is meaningful)."""
    import ndyn_omp_b200 as nd
    from ndyn_omp_b200 import workloads as W
    if warm:
        with nd.Context(local, "fp64") as cx:
            ids = [W.add_to_context(cx, sp) for sp in specs]
            cx.run(warm)
            states = [cx.state(i) for i in ids]
    fs = {}
    for p in ("fp64", "mixed"):
        with nd.Context(local, p) as cx:
            ids = []
            for sp, st in zip(specs, states):
                q = dict(sp)
                if st is not None:
                    q.update(pos=st[0], vel=st[1], box=st[3])
                ids.append(W.add_to_context(cx, q))
            cx.setup_lists()
            cx.compute0(True, True)
            fs[p] = [cx.forces(i)[0] for i in ids]
    per = [rel_l2(m, f) for m, f in zip(fs["mixed"], fs["fp64"])]
    allv = rel_l2(np.concatenate([f.ravel() for f in fs["mixed"]]),
                  np.concatenate([f.ravel() for f in fs["fp64"]]))
    return allv, max(per)


def plain_fp64_rate(specs, local, steps, stride):
    """The plain path: each sampled replica alone in an FP64 context (its own
    list build and graphs, untimed), `steps` steps timed with CUDA events on
    the library's stream; returns summed atom-steps / summed time, the
    number of systems, and the FP64 force kernel's algorithmic bytes and
    mean launch time summed over them (eager launches with events)."""
    import torch

    import ndyn_omp_b200 as nd
    from ndyn_omp_b200 import workloads as W
    tot_as, tot_s, n, alg_bytes, pair_s = 0.0, 0.0, 0, 0.0, 0.0
    for sp in specs[::stride]:
        with nd.Context(local, "fp64") as cx:
            sid = W.add_to_context(cx, sp)
            cx.run(100)  # list build and the 100-step graph capture
            st = torch.cuda.ExternalStream(cx.stream_ptr)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            cx.run(steps, cont=True)
            e1.record(st)
            torch.cuda.synchronize()
            tot_s += e0.elapsed_time(e1) / 1e3
            na = len(sp["typ"])
            tot_as += na * steps
            n += 1
            nb_half = cx.neighbor_count(sid) / (2.0 * na)
            prof = cx.profile_run(20)
            alg_bytes += na * (4.0 * nb_half + 148.0)
            pair_s += prof["pair_ms"] / 1e3
    return tot_as / tot_s, n, alg_bytes, pair_s


# ---------------------------------------------------------------------------
def dist_init():
    from ndyn_omp_b200 import replicas as R
    return R.init()


def barrier(ws):
    from ndyn_omp_b200 import replicas as R
    R.barrier(ws)


def allmax(x, ws):
    """the slowest rank's value (times are max over ranks)"""
    from ndyn_omp_b200 import replicas as R
    return R.reduce_max(x, ws)


def finish(ws):
    from ndyn_omp_b200 import replicas as R
    R.finish(ws)


def run_reference(args, ws, rank):
    """--impl reference: the reference's CPU path (the oracle port; the
    Fortran reference cannot be compiled in this image) on all host threads,
    same workload, metric and unit.  Each step is one MD step of a bounded
    sample of the workload."""
    if rank != 0:
        return
    specs, _ = workload(args.config)
    threads = os.cpu_count()
    budget = 60.0
    # calibrate on a small sample of the same material, then size the sample
    # so the K+W steps fit the budget
    if args.config in ("c2", "c1"):
        base = 40 if args.config == "c2" else 10
        probe_cells = 12 if args.config == "c2" else 6
        probe = workload(args.config, probe_cells)[0][0]
        r, _, _, _ = cpu_rate(probe, 2.0, threads)
        want_atoms = r * budget / max(args.steps + args.warmup, 1)
        cells = int(min(base, max(6, round((want_atoms / 4) ** (1 / 3)))))
        sample = workload(args.config, cells)[0][0]
        sample_txt = f"{len(sample['typ'])} atoms ({cells}^3 FCC cells) of the same liquid"
    elif args.config == "c3":
        probe = workload("c3", (8, 8, 8))[0][0]
        r, _, _, _ = cpu_rate(probe, 2.0, threads)
        want_atoms = r * budget / max(args.steps + args.warmup, 1)
        n = int(min(64, max(6, round((want_atoms / 8) ** (1 / 3)))))
        sample = workload("c3", (n, n, n))[0][0]
        sample_txt = f"{len(sample['typ'])} atoms ({n}^3 rocksalt cells)"
    elif args.config in ("c4", "c5batch"):
        # the systems run one after another (the reference runs one system at
        # a time): a spread of them, as many as fit the budget at K+W steps
        r, _, _, _ = cpu_rate(specs[1], 1.0, threads)
        pick, idx = spread_sample(specs, r * budget / max(args.steps + args.warmup, 1))
        v, el = cpu_rate_systems(pick, args.steps, args.warmup, threads)
        sample_txt = (f"{len(pick)} of {len(specs)} systems spread evenly over the list "
                      f"({n_atoms(pick)} atoms), one after another")
        line = {
            "impl": "reference", "metric": "atom-steps/s", "value": v, "unit": "atom-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_TEXT[args.config], "sample": sample_txt},
            "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": threads, "kind": "port",
                             "sample": sample_txt + f", {args.steps} steps each; " + CPU_BUILD},
            "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    else:
        # c5: the stream's first request system
        from ndyn_omp_b200 import workloads as W
        sample = W.build_request(W.serving_requests(1, args.rate, seed=5)[0])
        sample_txt = f"request 0 of the stream ({len(sample['typ'])} atoms)"
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_from_spec
    o = oracle_from_spec(sample, threads=threads, fast=True)
    assert o.setup_lists() == 0
    dt = sample["control"]["dt"]
    if args.warmup:
        o.run(args.warmup, dt, loop_only=True)
    t0 = time.perf_counter()
    rc, _ = o.run(args.steps, dt, loop_only=True)
    el = time.perf_counter() - t0
    assert rc == 0
    n = len(sample["typ"])
    v = n * args.steps / el
    line = {
        "impl": "reference", "metric": "atom-steps/s", "value": v, "unit": "atom-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_TEXT[args.config], "sample": sample_txt},
        "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": threads, "kind": "port",
                         "sample": sample_txt + f", {args.steps} steps; " + CPU_BUILD},
        "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def serve_stream(local, ws, rank, nreq, rate, steps_scale, seed=5):
    """The request loop over one seeded Poisson stream: requests arrive on a
    wall clock; between blocks every arrived request is submitted, and each
    server step admits what fits the HBM budget and advances every resident
    run by one block.  Latency = completion - arrival (wall clock).  Returns
    the stream's specs, latencies (s), makespan (s, max over ranks),
    failures and the server's stats."""
    import torch

    import ndyn_omp_b200 as nd
    from ndyn_omp_b200 import workloads as W
    reqs = W.serving_requests(nreq, rate, seed=seed + rank)
    specs = []
    for r in reqs:
        sp = W.build_request(r)
        sp["steps"] = max(1, int(round(sp["steps"] * steps_scale)))
        specs.append(sp)
    srv = nd.Server(local, "mixed", hbm_budget=150e9, block_steps=100)
    arrival, lat, which, failed = {}, {}, {}, []
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    k = 0
    while len(lat) < len(specs):
        now = time.perf_counter() - t0
        while k < len(specs) and reqs[k]["arrival"] <= now:
            t = W.submit_to_server(srv, specs[k])
            arrival[t] = reqs[k]["arrival"]
            which[t] = k
            k += 1
        st = srv.stats()
        if st["resident"] + st["queued"] == 0:
            if k < len(specs):
                time.sleep(max(0.0, min(0.01, reqs[k]["arrival"] - now)))
            continue
        srv.step()
        tn = time.perf_counter() - t0
        for t in srv.poll():
            lat[t] = tn - arrival[t]
            if srv.status(t) == 2:
                srv.result(t)
            else:
                r = reqs[which[t]]
                failed.append({"request": which[t], "status": srv.status(t),
                               "pot": r["pot"], "atoms": len(specs[which[t]]["typ"]),
                               "ensemble": r["ensemble"], "T": round(r["T"], 1),
                               "steps": specs[which[t]]["steps"]})
    t_end = max(arrival[t] + lat[t] for t in lat)
    makespan = allmax(t_end - reqs[0]["arrival"], ws)
    st = srv.stats()
    srv.close()
    return specs, np.array(sorted(lat.values())), makespan, failed, st


def serving_summary(local, ws, rank, nreq=64, steps_scale=0.02, rates=(50.0, 200.0, 800.0)):
    """p50/p99 completion latency and aggregate atom-steps/s of a scaled
    serving stream at each arrival rate (the default bench line's serving
    record)."""
    out = {"requests": nreq, "steps_scale": steps_scale, "hbm_budget_gb": 150,
           "block_steps": 100, "rates": []}
    for rate in rates:
        specs, lat, makespan, failed, st = serve_stream(local, ws, rank, nreq, rate, steps_scale)
        total = float(sum(len(sp["typ"]) * sp["steps"] for sp in specs))
        lv = lat * 1e3
        out["rates"].append({"rate_per_s": rate, "p50_ms": float(np.percentile(lv, 50)),
                             "p99_ms": float(np.percentile(lv, 99)),
                             "atom_steps_per_s": total * ws / makespan, "failed": len(failed)})
    return out


def run_serving(args, ws, rank, local):
    """c5: the request loop (serve_stream) on the configured stream."""
    import torch
    torch.cuda.set_device(local)
    from ndyn_omp_b200 import workloads as W
    reqs = W.serving_requests(args.requests, args.rate, seed=5 + rank)
    probe_specs = []
    for r in reqs[:8]:
        sp = W.build_request(r)
        if len(sp["typ"]) <= 60000:
            probe_specs.append(sp)
    probe = probe_specs[:4] or [W.build_request(reqs[0])]
    # the stated force error: mixed vs FP64 on the first requests' systems
    ea, em = force_error(probe, [None] * len(probe), local, warm=100)
    with ClockSampler(local) as clk:
        specs, lat, makespan, failed, st = serve_stream(local, ws, rank, args.requests, args.rate,
                                                        args.steps_scale)
    total = float(sum(len(sp["typ"]) * sp["steps"] for sp in specs))
    lv = lat * 1e3
    # each rank serves its own stream: aggregate work over the slowest rank
    value_all = total * ws / makespan
    line = {
        "metric": "atom-steps/s", "value": value_all, "unit": "atom-steps/s", "n_gpus": ws,
        "steps": len(specs), "warmup": 0, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair math + i64 fixed-point sums + f64 integrator",
        "data": "synthetic (seeded Poisson request stream, seeded lattices and velocities)",
        "config": {"workload": WORKLOAD_TEXT["c5"], "requests": len(specs),
                   "rate_per_s": args.rate, "steps_scale": args.steps_scale,
                   "atom_steps": total, "hbm_budget_gb": 150, "block_steps": 100,
                   "parallelism": f"replicas x{ws} (one server per GPU)" if ws > 1 else "1 GPU"},
        "latency_ms": {"p50": float(np.percentile(lv, 50)), "p99": float(np.percentile(lv, 99)),
                       "max": float(lv[-1])},
        "makespan_s": makespan, "failed": st["failed"], "failed_requests": failed[:20],
        "server": {k: st[k] for k in ("t_admit", "t_setup", "t_block", "t_retire",
                                      "graph_captures", "blocks")},
        "force_rel_err_vs_fp64": ea, "force_rel_err_max_system": em,
        "clocks": clk.summary(),
        "e2e": {"value": value_all, "unit": "atom-steps/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "what": "wall clock from the first arrival to the last completion: submit "
                        "(host copies), admission, list builds, blocks, result copies"},
        "roofline": None, "cpu_baseline": None, "gpu_launches": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.config == "c5" and args.impl != "reference":
        run_serving(args, ws, rank, local)
        finish(ws)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        finish(ws)
        return
    import torch

    import ndyn_omp_b200 as nd
    from ndyn_omp_b200 import workloads as W
    torch.cuda.set_device(local)
    specs, prec = workload(args.config)
    if args.config == "c4" and args.replica_stride > 1:
        specs = specs[::args.replica_stride]
    prec = args.precision or prec
    N = n_atoms(specs)

    # stated force error of this precision against the FP64 path (the FP64
    # path itself matches the CPU oracle to 1e-12, tests/test_gpu_parity.py)
    force_err = None
    batch = args.config in ("c4", "c5batch")
    if prec == "mixed" and not batch and not args.bare:
        force_err, _ = force_error(specs[:1], [None], local)

    ctx = nd.Context(local, prec)
    ids = [W.add_to_context(ctx, s) for s in specs]
    ctx.set_tuning(args.tpa, args.graph_steps)
    if args.gather_depth:
        ctx.set_gather_depth(args.gather_depth)
    skin_changed = None
    if batch and not args.bare:
        # launch shape (threads per atom, gathers in flight), then the
        # rebuild interval: a per-system list skin kept only where a second
        # timed trial confirms it
        ctx.autotune(30)
        skin_changed = ctx.autotune_skin(40)
    # warm-up (includes the dynamics prologue: cell + Verlet list build), then
    # one block of the timed region's size so that its CUDA graph is captured
    # before the clock starts
    ctx.run(max(args.warmup, 3))
    ctx.run(min(args.graph_steps, args.steps), cont=True)
    # half the full-list entries per atom (each pair once)
    nb_half = sum(ctx.neighbor_count(i) for i in ids) / (2.0 * N)
    nup0 = sum(ctx.list_updates(i) for i in ids)
    s = torch.cuda.ExternalStream(ctx.stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(s)
        ctx.run(args.steps, cont=True)
        e1.record(s)
        torch.cuda.synchronize()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    rebuilds = sum(ctx.list_updates(i) for i in ids) - nup0
    ms = allmax(ms, ws)
    steady = None
    if batch and not args.bare:
        # the same run further on, once the replicas' rebuilds no longer all
        # date from the run's first list build: 300 more steps untimed, then
        # 100 timed (a long run's steady state)
        ctx.run(300, cont=True)
        torch.cuda.synchronize()
        e0.record(s)
        ctx.run(100, cont=True)
        e1.record(s)
        torch.cuda.synchronize()
        ms_ss = allmax(e0.elapsed_time(e1), ws) / 100
        steady = {"ms_per_step": ms_ss, "value": N * ws / (ms_ss / 1e3),
                  "after_steps": max(args.warmup, 3) + min(args.graph_steps, args.steps) +
                  args.steps + 300, "steps": 100}
    value = N * args.steps * ws / (ms / 1e3)
    clocks = clk.summary()
    if args.bare:
        if rank == 0:
            print(json.dumps({"metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
                              "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": ms / args.steps, "bare": True,
                              "config": {"workload": WORKLOAD_TEXT[args.config], "atoms": N,
                                         "graph_steps": args.graph_steps},
                              "list_rebuilds_in_timed_region": rebuilds, "clocks": clocks}),
                  flush=True)
        ctx.close()
        finish(ws)
        return

    extra = {}
    if batch:
        # the mixed path's force error on the thermalised systems, and the
        # plain single-system FP64 path on every 8th system in sequence
        states = [ctx.state(i) for i in ids]
        if prec == "mixed":
            ea, em = force_error(specs, states, local)
            force_err = ea
            extra["force_rel_err_max_replica"] = em
        prate, pn, palg, ppair = plain_fp64_rate(specs, local, 200, 8)
        peak0, _ = hbm_peak()
        extra["plain_fp64"] = {
            "value": prate, "unit": "atom-steps/s",
            "sample": f"{pn} of {len(specs)} systems (every 8th), each alone in an FP64 context, "
                      f"200 steps, CUDA-graph blocks of 100",
            "batched_over_plain": (value / ws) / prate,
            # the FP64 force kernel on the same systems: algorithmic bytes
            # (4 n_half + 148 per atom, each system's own n_half) over its
            # mean launch time, summed over the systems
            "roofline": {"bound": "hbm", "achieved": palg / ppair / 1e9, "peak": peak0,
                         "unit": "GB/s", "frac": palg / ppair / 1e9 / peak0,
                         "pair_ms_summed": ppair * 1e3}}

    # per-kernel mean launch time over the same kind of steps (eager launches
    # with CUDA events on the library's stream)
    prof = ctx.profile_run(min(200, max(20, args.steps // 10)))
    tpa, gsteps = ctx.tuning()
    peak, peak_kind = hbm_peak()
    roof = None
    if nb_half:
        # algorithmic bytes of the fused pair kernel per atom: half-list
        # indices 4*n_half + own position/type 28 + neighbour positions 24
        # (each read once) + integrate2 state (read vel, acc; write vel, acc) 96
        alg_atom = 4.0 * nb_half + 148.0
        achieved = N * alg_atom / (prof["pair_ms"] / 1e3) / 1e9
        tr = traffic_per_atom(args.config)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": (tr * N if tr else None),
                "peak_kind": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                              else "fallback: no MEASURED_PEAKS.json; 6.65 TB/s B200 copy "
                                   "bandwidth"),
                "alg_bytes_per_atom": alg_atom, "n_half": nb_half,
                "pair_ms": prof["pair_ms"], "integrate_ms": prof["integrate_ms"],
                "rebuild_ms_per_step": prof["rebuild_ms"]}

    # end to end through the C ABI with host buffers: every system's state
    # loaded from pinned host memory in one call (ndg_load_state, sys = -1),
    # K steps (the prologue list build included), every state read back into
    # pinned host memory in one call (ndg_get_state, sys = -1)
    p0, v0, a0, b0 = ctx.states()

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    hp, hv, ha = pinned(p0), pinned(v0), pinned(a0)
    out = (pinned(np.zeros_like(p0)), pinned(np.zeros_like(v0)), pinned(np.zeros_like(a0)),
           np.zeros_like(b0))
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.load_states(hp, hv, ha, b0)
    rows = ctx.run(args.steps)
    ctx.states(out=out)
    torch.cuda.synchronize()
    el = allmax(time.perf_counter() - t0, ws)
    h2d = N * 3 * 8 * 3 + b0.size * 8                 # pos, vel, acc (3,np) each, boxes
    d2h = N * 3 * 8 * 3 + b0.size * 8 + 120 * len(rows)  # the same back, thermo records
    e2e = {"value": N * args.steps * ws / el, "unit": "atom-steps/s",
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "what": "ndg_load_state(all systems) + ndg_run(K) (incl. list build) + "
                   "ndg_get_state(all systems), host buffers page-locked"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        if batch:
            # the systems one after another, as the reference runs them: a
            # spread of them sized for ~15 s at 100 steps each
            r0, _, _, th = cpu_rate(specs[1], 1.0)
            pick, _ = spread_sample(specs, r0 * 15.0 / 100)
            r, el = cpu_rate_systems(pick, 100, 10, th)
            cpu = {"value": r, "unit": "atom-steps/s", "cores": th, "kind": "port",
                   "sample": f"{len(pick)} of {len(specs)} systems spread over the list "
                             f"({n_atoms(pick)} atoms) x 100 steps each ({el:.1f} s), one after "
                             f"another; " + CPU_BUILD}
        else:
            sample = specs[0]
            if args.config == "c3":
                sample = workload("c3", (24, 24, 24))[0][0]
            r, st, el, th = cpu_rate(sample, 15.0)
            cpu = {"value": r, "unit": "atom-steps/s", "cores": th, "kind": "port",
                   "sample": f"{len(sample['typ'])} atoms x {st} steps ({el:.1f} s), "
                             + CPU_BUILD}

    serving = None
    if batch and not args.bare and args.config == "c4":
        # the serving loop on a scaled c5 stream at the three arrival rates
        serving = serving_summary(local, ws, rank)

    touched = N * (4.0 * 2 * (nb_half or 40) + 200.0)
    line = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair math + i64 fixed-point sums + f64 integrator" if prec == "mixed"
        else "f64",
        "data": "synthetic (seeded lattice + Maxwell-Boltzmann velocities)",
        "config": {"workload": WORKLOAD_TEXT[args.config], "atoms": N, "precision": prec,
                   "list_semantics": specs[0]["control"].get("quirk", "ref"),
                   "parallelism": f"replicas x{ws} (one system per GPU)" if ws > 1 else "1 GPU",
                   "l2": f"inputs larger than L2: ~{touched / 1e6:.0f} MB touched per step "
                         f"vs 126 MB L2" if touched > L2_BYTES else "L2-resident workload",
                   "threads_per_atom": tpa, "gather_depth": ctx.gather_depth(),
                   "graph_steps": gsteps, "replica_stride": args.replica_stride,
                   "skin_retuned_systems": skin_changed,
                   "list_split": dict(zip(("rows", "threads_per_atom"), ctx.list_split())),
                   "baseline_metric": "atom-steps/s at 1 GPU, batched mixed vs plain FP64 at "
                                      "stated force error; p50/p99"},
        "force_rel_err_vs_fp64": force_err,
        **extra,
        "steady_state": steady,
        "serving": serving,
        "list_rebuilds_in_timed_region": rebuilds,
        # per step integrate1 (with the work plan) and the two pair kernels; per
        # graph block k_begin_block and k_decide; the 8 rebuild kernels (the
        # six of the counting sort and both forms of the list build) on steps
        # whose conditional node fires (at most one per step, at most one per
        # list update)
        "gpu_launches": 3 * args.steps + 2 * -(-args.steps // gsteps) + 8 * min(args.steps, rebuilds),
        "clocks": clocks,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    finish(ws)


if __name__ == "__main__":
    main()
