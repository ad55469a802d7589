#!/usr/bin/env python
"""Benchmark of the delta-SPH single-GPU step on the 3-D dam break at scale:
dx = 0.005 m, 3,456,000 fluid + 765,468 wall particles (4,221,468), one step =
predictor + corrector sub-step (single_gpu_sph_src/deltasph/main.cu:58-90).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  `value` is whole-job particle-steps/s with
the state resident in HBM (CUDA-event time of K steps replayed from a CUDA
graph, max over ranks); `e2e` is the same metric through the C ABI from
pinned host buffers (upload, K steps with a per-step status read, download).
With N > 1 (torchrun) every rank runs an independent replica of the case:
the path does not shard (replicas only), so there is no collective on the
data path; only the barrier and the max-over-ranks timing reduction.

Two more keys time the other forms of the step on the same GPU: `learned`
(learned corrector, trained first on dam-break snapshots at dx = 0.02, then
run on this case with and without the judging plain corrector) and
`batched` (256 uneven dam-break scenes in one batched handle vs the same
scenes looped through single-scene handles).

--impl reference times the reference solver's equations on the host cores
(the CPU oracle, an OpenMP restatement of the reference's CUDA kernels; the
reference has no CPU path of its own) and, beside it, the reference's own
CUDA kernels compiled for sm_100a (key `reference_cuda`).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("dam break dx=0.005 m: water 0.6x0.6x1.2 m in a 1.6x0.6x1.2 m tank, 3,456,000 fluid + 765,468 "
            "dummy-wall particles (3 layers), 500-step case, 1 step = predictor + corrector")
BYTES_PER_PARTICLE_SEARCH = 188  # hash 20 + sort 16 + cell bounds 4 + reorder 148
BYTES_PER_CELL_SEARCH = 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["config1", "config0", "medium"], default="config1",
                    help="config1: the measured case; config0: dx=0.02 (105,048 particles); medium: dx=0.0075 "
                         "(about 1.3 M particles, for profiling captures that must stay small)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="target CPU-baseline sample duration")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-corrector leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form leg")
    ap.add_argument("--learn-epochs", type=int, default=20)
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes instead of zsph_autotune's")
    ap.add_argument("--ref-cuda-child", choices=["plain", "profiled"], default=None,
                    help=argparse.SUPPRESS)  # one reference-CUDA run in a fresh process (reference arm)
    ap.add_argument("--shapes", default=None, metavar="CW,MINB,SPG[,SEGS]",
                    help="apply these launch shapes (zsph_set_launch_shapes) instead of running zsph_autotune")
    return ap.parse_args()


def workload_config(args, case, grid_num, dt, world) -> dict:
    """The `config` object of both arms' JSON lines (same keys and values)."""
    return {"workload": WORKLOAD if args.workload == "config1" else f"{args.workload}: {case.name}",
            "ptc_num": case.n, "fluid": case.n_fluid, "wall": case.n_wall, "grid_num": int(grid_num),
            "dt": float(dt), "parallelism": f"replicas x{world}",
            "l2": (f"inputs larger than L2 (particle state {case.n * 72 / 1e9:.2f} GB + scratch per step)"
                   if case.n * 72 > 126e6 else "inputs smaller than L2 (profiling and parity-size case)")}


def make_case(name):
    from zsph_b200 import cases
    if name == "medium":
        return cases.dam_break(0.0075, end_step=500)
    return cases.config1() if name == "config1" else cases.config0()


# ---------------------------------------------------------------- distributed
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
            tmo = float(os.environ.get("ZSPH_PG_TIMEOUT", "300"))
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=tmo))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        sm, smmax = [], []
        for r in rows:
            try:
                sm.append(float(r[1]))
                smmax.append(float(r[2]))
            except ValueError:
                pass
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        load = [s for s in sm if smmax and s > 0.5 * max(smmax)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(smmax) if smmax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def ncu_traffic(kernel_group: str):
    """Per-launch DRAM bytes of a kernel group from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(kernel_group)


# ---------------------------------------------------------------- pair kernels
# FP32 operations per interacting pair, counted from the pair arithmetic of
# k_boundary (L matrix, div v, the folded gradient sums) and k_governing
# (continuity, delta diffusion with its recurrence, pressure, viscosity) for a
# fluid-fluid pair; an FMA counts 2, a MUFU reciprocal or square root 1.
FLOP_PER_PAIR = {"boundary": 54, "governing": 68}


def stencil_candidates(sol, n):
    """Candidates per particle in the governing stencil (3x3 rows of 3 cells,
    delta_ns.cu:200-212) of the sorted state, from the search's cell bounds."""
    import numpy as np
    t = sol.download_tmp()
    gs, ge, h = t["grid_start"].astype(np.int64), t["grid_end"].astype(np.int64), t["hash"].astype(np.int64)
    gp = sol.gp
    X, XY = gp.grid_xdim, gp.grid_xdim * gp.grid_ydim
    tot = np.zeros(n, np.int64)
    for z in (-1, 0, 1):
        for y in (-1, 0, 1):
            c = h + z * XY + y * X
            cs, ce = c - 1, c + 1
            ok = (cs >= gp.grid_hash_min) & (ce <= gp.grid_hash_max)
            s = gs[np.clip(cs, 0, len(gs) - 1)]
            e = ge[np.clip(ce, 0, len(ge) - 1)]
            tot += np.where(ok, np.maximum(e - s, 0), 0)
    return float(tot.mean())


def pair_kernel_rates(sol, kern, nb_b, nb_g, n, clocks, full_size=True):
    """Rates of the pair kernels: candidate tests/s of the list build,
    interacting pair evaluations/s and FP32 FLOP/s of boundary and governing
    against the nominal FP32 peak (148 SMs x 128 lanes x 2 x max SM clock),
    and DRAM GB/s from the committed ncu traffic."""
    import numpy as np
    mhz = (clocks or {}).get("sm_max_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    cand = stencil_candidates(sol, n)
    out = {"fp32_peak_tflops_nominal": fp32_peak}
    per_launch = lambda k: (kern[k]["ms_per_step"] / max(kern[k]["launches_per_step"], 1) / 1e3) if k in kern else 0
    t_nb = per_launch("nblist")
    if t_nb:
        tr = ncu_traffic("nblist") if full_size else None
        out["nblist"] = {"ms_per_substep": t_nb * 1e3, "stencil_candidates_per_particle": cand,
                              "candidate_tests_per_s": cand * n / t_nb,
                              "dram_gbs": tr / t_nb / 1e9 if tr else None}
    for name in ("walls", "xfer_classify", "xfer_search", "nblist_xfer", "nblist_fallback"):
        if per_launch(name):
            out[name] = {"ms_per_substep": per_launch(name) * 1e3}
    for name, nb in (("boundary", nb_b), ("governing", nb_g)):
        t = per_launch(name)
        if not t:
            continue
        pairs = float(np.mean(nb[nb >= 0]))
        evals = pairs * n / t
        tr = ncu_traffic(name) if full_size else None
        out[name] = {"ms_per_substep": t * 1e3, "interacting_pairs_per_particle": pairs, "pair_evals_per_s": evals,
                     "fp32_tflops": evals * FLOP_PER_PAIR[name] / 1e12,
                     "fp32_frac_of_nominal_peak": evals * FLOP_PER_PAIR[name] / 1e12 / fp32_peak,
                     "dram_gbs": tr / t / 1e9 if tr else None}
    return out


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(case, target_s: float) -> dict:
    """The FP32 CPU oracle (OpenMP restatement of the reference's kernels) on
    a bounded sample of the same workload: whole steps of the full case,
    as many as fit in about target_s seconds (at least one)."""
    import numpy as np
    from oracle import pyoracle as po
    threads = os.cpu_count() or 1
    po.set_threads(threads)
    o = po.Oracle(case.json, case.state, np.float32)
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter()
    steps, dt = 1, t1 - t0
    while dt < target_s and steps < 3:
        s0 = time.perf_counter()
        o.step(1)
        dt += time.perf_counter() - s0
        steps += 1
    return {"value": case.n * steps / dt, "unit": "particle-steps/s", "cores": po.max_threads(), "kind": "port",
            "sample": f"{steps} full step(s) of the {case.n:,}-particle case (FP32 CPU oracle, OpenMP, "
                      f"{dt:.1f} s)"}


def guarded_leg(name, fn):
    """Runs one secondary leg; an exception becomes {"error": ...} in its
    key (and a note on stderr) instead of ending the run."""
    try:
        return fn()
    except Exception as e:  # noqa: BLE001 - the headline line must still be printed
        msg = f"{type(e).__name__}: {e}"[:400]
        print(f"bench: the {name} leg failed: {msg}", file=sys.stderr, flush=True)
        return {"error": msg}


# ---------------------------------------------------------------- learned form
GROWTH_STEPS = 2000


def learned_leg(args, dist, sol, stream, sptr, n, ms_plain):
    """Learned-corrector form on the bench's case and its speed/error
    frontier.  The network is trained on the GPU (own tensor-core kernels)
    on 200 snapshots of plain dam-break steps at dx = 0.02 (every 10th of
    2000 steps after 100 settling steps).  Three correctors then run from the
    same state of the bench's case (zsph_run_learned_ex): the network
    corrector, and two correctors that skip the second search and list build
    by walking the predictor's neighbour lists at the predicted positions,
    one with the predictor's boundary data (lagged) and one with a fresh
    boundary pass.  Each is timed over K steps with the plain corrector
    judging every 10th step (tolerance 1e-2, fallback above it) and over K
    steps unjudged, and runs 2000 judged steps (every 10th) for its error
    growth."""
    import torch
    import zsph_b200 as z
    from zsph_b200 import cases
    t0 = time.perf_counter()
    c0 = cases.config0()
    s0 = z.Solver.from_case(c0)
    s0.run(100)
    snaps = s0.collect(2000, 10, 200)
    net = z.Mlp(seed=1)
    train = s0.train(net, epochs=args.learn_epochs, batch_tiles=148, lr=2e-3, seed=3, val_frac=0.1)
    s0.close()
    prep_s = time.perf_counter() - t0
    K = args.steps

    def timed(fn):
        torch.cuda.synchronize()
        dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return dist.max(a.elapsed_time(b)), r

    start = sol.download("old")
    forms = {}
    for name, corr, nt in (("network", z.CORR_NETWORK, net), ("reuse_lagged", z.CORR_REUSE_LAGGED, None),
                           ("reuse_fresh", z.CORR_REUSE_FRESH, None)):
        sol.upload(start)
        ms_j, rj = timed(lambda: sol.run_learned(nt, K, judge_every=10, tol=1e-2, stream=sptr, corrector=corr))
        sol.upload(start)
        ms_u, ru = timed(lambda: sol.run_learned(nt, K, judge_every=0, tol=1e-2, stream=sptr, corrector=corr))
        sol.upload(start)
        ms_g, rg = timed(lambda: sol.run_learned(nt, GROWTH_STEPS, judge_every=10, tol=1e-2, stream=sptr,
                                                 corrector=corr, series=GROWTH_STEPS // 10))
        errs = rg.pop("err_series")
        forms[name] = {
            "ms_per_step": ms_j / K, "speedup_vs_plain": ms_plain / (ms_j / K), "run": rj,
            "unjudged": {"ms_per_step": ms_u / K, "speedup_vs_plain": ms_plain / (ms_u / K), "run": ru},
            "growth": {"steps": GROWTH_STEPS, "judge_every": 10, "ms_per_step": ms_g / GROWTH_STEPS,
                       "speedup_vs_plain": ms_plain / (ms_g / GROWTH_STEPS), "run": rg,
                       "err_at_step": {str(10 * (k + 1)): errs[k] for k in (0, 9, 49, 99, 149, 199) if k < len(errs)},
                       "err_series_every_100_steps": errs[9::10]}}
    sol.upload(start)
    net.close()
    ok = [k for k, f in forms.items() if f["growth"]["run"]["fallbacks"] == 0 and f["growth"]["run"]["err_max"] <= 1e-2]
    best = max(ok, key=lambda k: forms[k]["speedup_vs_plain"]) if ok else None
    fn = forms["network"]
    return {"value": dist.world * n / (fn["ms_per_step"] / 1e3), "unit": "particle-steps/s",
            "ms_per_step": fn["ms_per_step"], "speedup_vs_plain": fn["speedup_vs_plain"], "judge_every": 10,
            "tol": 1e-2, "run": fn["run"], "unjudged": fn["unjudged"],
            "frontier": forms, "fastest_within_tol": best,
            "train": dict(train, snapshots=snaps, data="dam break dx=0.02 (105,048 particles), plain steps 100-2100, "
                                                       "every 10th step", prep_seconds=prep_s),
            "what": "network: corrector stage = predictor-stage value + (value - previous corrector value) + network "
                    "residual; reuse_lagged / reuse_fresh: governing walk on the predictor's neighbour lists at the "
                    "predicted positions with lagged / fresh boundary data (no second search or list build). Judged "
                    "steps run the plain corrector, compare accelerations (relative L2, fluid) and keep the plain "
                    "result; above tol the plain corrector runs until a judged step passes"}


# ---------------------------------------------------------------- batched form
def batched_leg(args, dist, stream, sptr):
    """256 seeded dam-break scenes of uneven sizes (cases.batch_scenes, seed
    2026) advanced together: one batched handle whose every kernel launch
    covers all scenes, K steps replayed from its CUDA graph after the
    autotuner picked the launch shapes; beside it the same scenes stepped
    one after another with 256 single-scene handles (one graph replay per
    scene and step).  Both timed with CUDA events on the same stream."""
    import torch
    import zsph_b200 as z
    from zsph_b200 import cases
    scenes, _ = cases.batch_scenes(256, seed=2026)
    n = sum(c.n for c in scenes)
    K, W = args.steps, args.warmup

    def timed(fn):
        torch.cuda.synchronize()
        dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return dist.max(a.elapsed_time(b))

    bt = z.Solver.from_batch(scenes)
    tune = bt.autotune(3, stream=sptr)
    bt.run(W, sptr)
    ms_b = timed(lambda: bt.run(K, sptr))
    flags_b = bt.status()
    bt.close()
    # the same scenes in one persistent launch per step (grid barriers between the stages)
    bp = z.Solver.from_batch(scenes)
    bp.set_persistent(True)
    bp.run(W, sptr)
    ms_p = timed(lambda: bp.run(K, sptr))
    flags_p = bp.status()
    pinfo = bp.persistent_info()
    bp.close()
    solo = [z.Solver.from_case(c) for c in scenes]
    for s in solo:
        s.run(W, sptr)

    def loop():
        for _ in range(K):
            for s in solo:
                s.run(1, sptr)

    ms_l = timed(loop)
    for s in solo:
        s.close()
    nf = [c.n_fluid for c in scenes]
    return {"value": dist.world * n * K / (ms_b / 1e3), "unit": "particle-steps/s", "ms_per_step": ms_b / K,
            "loop_value": dist.world * n * K / (ms_l / 1e3), "loop_ms_per_step": ms_l / K,
            "speedup_vs_loop": ms_l / ms_b, "scenes": len(scenes), "particles": n,
            "persistent": {"value": dist.world * n * K / (ms_p / 1e3), "ms_per_step": ms_p / K,
                           "vs_graph_of_launches": ms_b / ms_p, "ctas": pinfo["ctas"],
                           "graph": {1: "replayed from a CUDA graph", -1: "one direct launch per zsph_run",
                                     0: "not run"}[pinfo["graph"]], "status_flags": flags_p,
                           "what": "every scene's whole step in one cooperative launch: the stages of the "
                                   "graph-of-launches step behind bounded grid barriers"},
            "fluid_per_scene": {"min": min(nf), "max": max(nf), "sum": sum(nf)}, "tune": tune,
            "status_flags": flags_b,
            "what": "aggregate particle-steps/s of 256 scenes (widths U[0.2,0.6] m, aspect U[0.5,2], dx U[0.01,0.02] m, "
                    "seed 2026) in one batched handle, vs the same scenes looped through single-scene handles"}


# ---------------------------------------------------------------- our arm
def run_ours(args, dist: Dist):
    import ctypes
    import numpy as np
    import torch
    import zsph_b200 as z

    dev = dist.local if torch.cuda.device_count() > 1 else 0
    torch.cuda.set_device(dev)
    case = make_case(args.workload)
    cp, gp = z.params_from_json(case.json)
    n, G = case.n, cp.grid_num
    sol = z.Solver(gp, G)
    sol.upload(case.state)
    stream = torch.cuda.Stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    K, W = args.steps, args.warmup

    # launch shapes from the project's autotuner (untimed; it restores the state after every trial)
    if args.shapes:
        vals = [int(v) for v in args.shapes.split(",")]
        cw, mb, spg = vals[:3]
        sg = vals[3] if len(vals) > 3 else 0
        sol.set_launch_shapes(cw, mb, spg, sg)
        tune = {"list_cells_per_cta": cw, "governing_min_ctas": mb, "steps_per_graph": spg, "list_segments": sg,
                "applied": True}
    else:
        tune = None if args.no_tune else sol.autotune(3, sptr)

    # warm-up (captures the CUDA graph), then K steps timed with CUDA events
    with torch.cuda.stream(stream):
        sol.run(W, sptr)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    xf0 = sol.list_transfer_info()
    e0.record(stream)
    sol.run(K, sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    xf1 = sol.list_transfer_info()
    xfer = {k: xf1[k] - xf0[k] for k in xf1}
    dist.barrier()
    ms_local = e0.elapsed_time(e1)
    ms = dist.max(ms_local)
    flags = sol.status()
    if flags & z.FLAG_NAN:
        raise SystemExit("non-finite state during the timed steps")
    value = dist.world * n * K / (ms / 1e3)

    # per-launch durations (3 profiled steps, events on the launching stream)
    prof = [sol.step_profiled(sptr) for _ in range(3)]
    per = {}
    for step in prof:
        for name, t in step:
            per.setdefault(name, []).append(t)
    launches = len(prof[0])
    step_ms_prof = sum(t for _, t in prof[-1])
    kern = {k: {"launches_per_step": len(v) // 3, "ms_per_step": sum(v) / 3,
                "share": (sum(v) / 3) / step_ms_prof} for k, v in per.items()}
    search_names = ("hash_count", "scan", "scatter", "rank_gather")
    # the search group's duration from events at group boundaries only (an event node costs a few us, which
    # per-launch events would charge to each of the group's four kernels)
    grp = [sol.step_profiled(sptr, groups=True) for _ in range(3)]
    search_ms_sub = statistics.mean(t for step in grp for name, t in step if name == "search")
    pair_ms_sub = statistics.mean(t for step in grp for name, t in step if name == "pair")
    search_bytes = BYTES_PER_PARTICLE_SEARCH * n + BYTES_PER_CELL_SEARCH * G
    peaks = measured_peaks()
    ach = search_bytes / (search_ms_sub / 1e3) / 1e9
    dom = max(kern.items(), key=lambda kv: kv[1]["ms_per_step"])
    nb_b, nb_g = sol.neighbor_counts("new")
    pairs_gov = float(np.mean(nb_g[nb_g >= 0]))
    roofline = {"bound": "hbm", "kernel": "search+sort group: " + ", ".join(search_names),
                "algorithmic_bytes": search_bytes, "group_us_per_substep": search_ms_sub * 1e3,
                "pair_group_us_per_substep": pair_ms_sub * 1e3,
                "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"] if peaks["hbm_gbs"] else None,
                "peak_source": f"{peaks['source']} hbm_gbs (copy test)",
                # the committed ncu traffic is scaled to the dx = 0.005 case
                "traffic": ncu_traffic("search_group") if args.workload == "config1" else None}
    gov_ms = kern.get("governing", {}).get("ms_per_step", 0) / 2
    pair = pair_kernel_rates(sol, kern, nb_b, nb_g, n, ck, full_size=args.workload == "config1")
    dominant = {"kernel": dom[0], "ms_per_step": dom[1]["ms_per_step"], "share": dom[1]["share"],
                "bound": {"nblist": "instruction issue (candidate tests and per-lane hit emission)",
                          "boundary": "L1 data pipe (scattered neighbour records)",
                          "governing": "L1 data pipe (scattered neighbour records)"}.get(
                              dom[0], "see profiles/kernels_medium.md") +
                         "; not HBM-bound, no tensor-core work on the pair path",
                "interacting_pairs_per_particle": pairs_gov,
                "governing_pair_evals_per_s": pairs_gov * n / (gov_ms / 1e3) if gov_ms else None,
                "traffic": ncu_traffic(dom[0]) if args.workload == "config1" else None}

    # end to end through the C ABI from pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hp = {k: pin(getattr(case.state, k)) for k in ("pos", "vel", "rhop", "type", "table")}
    hout = {k: torch.empty_like(v).pin_memory() for k, v in hp.items()}
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    z.check(z.lib.zsph_cpu_to_gpu(ctypes.byref(sol.old), ctypes.byref(sol.tmp), ptr(hp["pos"]), ptr(hp["vel"]),
                                  ptr(hp["rhop"]), ptr(hp["type"]), ptr(hp["table"]), None, n, sptr))
    flag = ctypes.c_int(0)
    for _ in range(K):
        sol.run(1, sptr)
        z.check(z.lib.zsph_status(sol.h, ctypes.byref(flag), 0), sol.h)
    z.check(z.lib.zsph_gpu_to_cpu(ctypes.byref(sol.old), ctypes.byref(sol.tmp), ptr(hout["pos"]), ptr(hout["vel"]),
                                  ptr(hout["rhop"]), ptr(hout["type"]), ptr(hout["table"]), None, None, n, sptr))
    t_e2e = dist.max(time.perf_counter() - t0)
    h2d = 40 * n  # pos 12, vel 12, rhop 8, type 4, table 4 (acc_drhodt is zero-filled on the device)
    d2h = 40 * n + 4 * K
    e2e = {"value": dist.world * n * K / t_e2e, "unit": "particle-steps/s",
           "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
           "what": "zsph_cpu_to_gpu of the case from pinned host memory, K x (zsph_run 1 step + zsph_status "
                   "read of the 4-byte device status word), zsph_gpu_to_cpu of pos/vel/rhop/type/table; "
                   "host wall clock, max over ranks"}

    # the other forms' legs and the CPU baseline come after the headline measurement: a failure in one of
    # them is reported in its key and the line is still printed
    learned = None if args.no_learned else guarded_leg(
        "learned", lambda: learned_leg(args, dist, sol, stream, sptr, n, ms / K))
    batched = None if args.no_batched else guarded_leg("batched", lambda: batched_leg(args, dist, stream, sptr))

    cpu = None
    if dist.rank == 0 and not args.no_cpu_baseline:
        cpu = guarded_leg("cpu_baseline", lambda: cpu_baseline(case, args.cpu_seconds))

    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": dist.world,
        "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (lattice dam break, no randomness)",
        "config": workload_config(args, case, G, cp.dt, dist.world),
        "fluid_particle_steps_per_s": dist.world * case.n_fluid * K / (ms / 1e3),
        "clocks": ck, "e2e": e2e, "gpu_launches": sol.launches_per_step() * K, "launches_per_step": launches,
        "tune": tune, "list_transfer": xfer,
        "roofline": roofline, "dominant_kernel": dominant, "pair_kernels": pair, "kernels": kern, "cpu_baseline": cpu,
        "learned": learned, "batched": batched, "status_flags": flags,
    }
    sol.close()
    return line


# ---------------------------------------------------------------- reference arm
REF_CUDA_RUNS = 3


def ref_cuda_child(args):
    """One reference-CUDA measurement in this (fresh) process: `plain` is the
    step loop timed first event to last (oracle/ref_driver.cu ref_run);
    `profiled` adds an event after each launch slot and the host time of the
    Thrust sort calls (ref_run_profiled).  Prints one JSON line."""
    from oracle import pyoracle as po
    case = make_case(args.workload)
    t0 = time.perf_counter()
    if args.ref_cuda_child == "plain":
        ms = po.ref_run(case.json, case.state, args.steps, warmup=args.warmup)[2]
        out = {"ms_per_step": ms}
    else:
        out = po.ref_run_profiled(case.json, case.state, args.steps, warmup=args.warmup)
    out["process_seconds"] = time.perf_counter() - t0
    print(json.dumps(out), flush=True)


def reference_cuda_leg(args, case) -> dict:
    """The reference's own CUDA kernels (oracle/_ref, built from its sources):
    REF_CUDA_RUNS plain runs and one profiled run, each in a fresh process
    started one after another, before any CPU work of this arm.  Reports the
    median of the plain runs with their spread, and the per-slot split."""
    from oracle import pyoracle as po
    if not po.ref_available():
        return {"unavailable": "oracle/_ref/libzsph_ref.so not built"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"torch: {e}"[:200]}

    def child(mode):
        cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--ref-cuda-child", mode,
               "--workload", args.workload, "--steps", str(args.steps), "--warmup", str(args.warmup)]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
        if r.returncode != 0:
            raise RuntimeError(f"reference CUDA run failed (rc {r.returncode}): {r.stderr[-300:]}")
        return json.loads(r.stdout.strip().splitlines()[-1])

    try:
        plain = [child("plain") for _ in range(REF_CUDA_RUNS)]
        prof = child("profiled")
    except Exception as e:  # noqa: BLE001 - keep the CPU line even if the GPU leg fails
        return {"unavailable": str(e)[:300]}
    runs = [p["ms_per_step"] for p in plain]
    ms = statistics.median(runs)
    slots = prof["slot_ms"]
    sort_slots = slots["sort_index"] + slots["sort_index_2"]
    return {"value": case.n / (ms / 1e3), "unit": "particle-steps/s", "ms_per_step": ms,
            "ms_per_step_runs": runs, "spread": (max(runs) - min(runs)) / ms, "steps": args.steps,
            "warmup": args.warmup,
            "profiled": {"ms_per_step": prof["ms_per_step"], "slot_ms": slots, "host_sort_ms": prof["host_sort_ms"],
                         "sort_share": sort_slots / prof["ms_per_step"]},
            "what": "the reference's own hash/sort/boundary/governing/time integration kernels (unmodified sources, "
                    "-maxrregcount 64, sm_100a), Thrust sort, launch order of main.cu:63-88, CUDA events; median "
                    f"of {REF_CUDA_RUNS} runs, each in a fresh process, run before the CPU leg; `profiled` is one "
                    "more run with an event after each launch slot and the host time of each Thrust sort call"}


def run_reference(args, dist: Dist):
    """Reference arm.  `value`: the reference solver's equations on the host
    cores; the reference has no CPU implementation of its own (its kernels
    exist only as CUDA), so this is the CPU oracle, an OpenMP restatement of
    those kernels (kind "port"), W untimed and K timed full steps of the
    same case.  `reference_cuda`: the reference's own CUDA build on the GPU,
    measured first, in separate processes."""
    if dist.rank != 0:
        return None
    import numpy as np
    from oracle import pyoracle as po
    case = make_case(args.workload)
    rc, op = po.params(case.json)
    if rc:
        raise SystemExit(f"case constants rejected by the oracle (rc {rc})")
    ref_cuda = reference_cuda_leg(args, case)

    K, W = args.steps, args.warmup
    threads = os.cpu_count() or 1
    po.set_threads(threads)
    o = po.Oracle(case.json, case.state, np.float32)
    if W:
        o.step(W)
    t0 = time.perf_counter()
    o.step(K)
    dt = time.perf_counter() - t0
    value = case.n * K / dt
    cpu = {"value": value, "unit": "particle-steps/s", "cores": po.max_threads(), "kind": "port",
           "sample": f"{K} full steps (after {W} untimed) of the {case.n:,}-particle case: FP32 CPU oracle, OpenMP, "
                     f"{dt:.1f} s"}
    line = {"impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": dt / K * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (lattice dam break, no randomness)",
            "config": workload_config(args, case, op.grid_num, op.dt, dist.world),
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_cuda": ref_cuda}
    return line


def main():
    args = parse()
    if args.ref_cuda_child:
        ref_cuda_child(args)
        return
    dist = Dist()
    try:
        line = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
        if dist.rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
