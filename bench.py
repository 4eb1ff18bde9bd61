#!/usr/bin/env python
"""Benchmark of the sm_100a Shatterforge physics path.

Headline: body-steps/s of the batched rigid step on the 256-scene debris mix (256 independent scenes, body counts
log-uniform in 500-20,000, compound bodies of Geometric(0.3) bricks, 4-16 static box obstacles each; dt = 1/60 s,
8 impulse iterations, 2 substeps), every scene stepped in the same launches. Beside it, in the same JSON line:
  * the plain path (one scene per launch sequence) timed on the same simulated state, and the batched/plain ratio;
  * the load path: all 37 structures of the structures-in-one-lattice configuration solved in one persistent launch
    to residual 1e-6 (omega 1.7), as brick-sweeps/s;
  * e2e: the same metric through the public C ABI with the body state written from and read back to pinned host
    buffers every step;
  * roofline of the dominant kernel (CUDA events around each launch, algorithmic bytes per unit as documented);
  * cpu_baseline: the CPU restatement of the reference (the oracle) on a bounded sample of the same workload.

`--impl reference` times only the CPU restatement (the reference itself is a wasm32 Rust crate that cannot be
built here) with every host thread, and prints its own line.

Multi-GPU (torchrun): each rank runs its own 256-scene mix (seeded by rank), no collective on the data path;
value = all ranks' body-steps / the slowest rank's device time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "body-steps/s & SOR brick-sweeps/s; served p50/p99 ms vs plain GPU path"
UNIT = "body-steps/s"
DT = 1.0 / 60.0
ITERS = 8
SOLVE_BYTES_PER_CONTACT_ITER = 184     # contact 64 + impulse r/w 24 + both bodies' v, w r/w 96
# DRAM bytes (read + write) per contact-iteration of k_solve, from one ncu capture at the peak of contacts on the
# half-size mix: 722.7 MB for that launch / (≈847,700 contacts, from the same substep's k_prep grid, x 8 iterations);
# the roofline's `traffic` scales it to this run's average launch
SOLVE_DRAM_BYTES_PER_CONTACT_ITER = 106.6
GEN_BYTES_PER_BRICK = 40               # local offset 12 + body id 4 read, world position 12 written and re-read
GEN_BYTES_PER_CONTACT = 64             # one contact's setup written
# DRAM bytes (read + write) of k_contacts_gen per algorithmic byte, from the ncu capture in free fall on the half-size
# mix (the benchmark window's regime): 77.2 MB against 40 B x 1.11M bricks + 64 B x ~4,000 contacts
GEN_DRAM_PER_ALGORITHMIC_BYTE = 1.73
SOR_BYTES_PER_BRICK_SWEEP = 24         # grid path: f64 potential r/w 16 + rhs 4 + link word 4
SOR_CLUSTER_BYTES_PER_BRICK = 52       # cluster path, once per solve: staging reads (phi 8, rhs 4, code 4, sid 4,
                                       # place 4, neighbours 12) + the potential written back 8 + gather 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--scale", type=float, default=1.0, help="body-count scale of the debris mix (1.0 = as specified)")
    ap.add_argument("--plain-steps", type=int, default=5, help="steps of the plain/batched comparison at the contact peak")
    ap.add_argument("--plain-steps-window", type=int, default=20, help="at most this many steps of the headline window")
    ap.add_argument("--peak-step", type=int, default=110, help="the step at which the mix has its peak of contacts")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = as --steps")
    ap.add_argument("--no-sor", action="store_true")
    ap.add_argument("--sor-max-sweeps", type=int, default=200000, help="sweep limit of the timed load-path solve")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-collapse", action="store_true")
    ap.add_argument("--no-sat", action="store_true")
    ap.add_argument("--no-boxes", action="store_true")
    ap.add_argument("--box-steps", type=int, default=20, help="timed steps of the box world's pile")
    ap.add_argument("--box-warmup", type=int, default=60, help="steps before the timed ones (the pile lands)")
    ap.add_argument("--collapse-frames", type=int, default=600, help="frames of the collapse run (frame order, damage on)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="length of the served arrival stream")
    ap.add_argument("--serve-plain-seconds", type=float, default=1.0, help="length of the stream the plain path serves")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-worlds", type=int, default=96)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-age-steps", type=int, default=300,
                    help="steps the population has run before the aged stream (0 = skip the aged runs)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        except OSError:
            return out
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1])); mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons), samples=len(sm))
        return out


# ---------------------------------------------------------------- distributed plumbing
def dist_setup(args):
    rank, world, local = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def barrier(pg, args):
    if pg is None:
        return
    import torch
    if args.impl == "ours":
        pg.barrier(device_ids=[torch.cuda.current_device()])
    else:
        pg.barrier()


def _reduce_device(pg) -> str:
    """NCCL reduces device tensors, gloo host tensors."""
    return "cuda" if pg.get_backend() == "nccl" else "cpu"


def allreduce_max(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def combine(pg, ms: float, body_steps: float) -> tuple[float, float, float]:
    """Whole-job figures of a weak-scaling run: (slowest rank's ms, all ranks' body-steps, body-steps / s of the job)."""
    ms_max = allreduce_max(pg, ms)
    total = allreduce_sum(pg, body_steps)
    return ms_max, total, total / (ms_max * 1e-3)


def rank_seed(rank: int) -> int:
    """Each rank steps its own 256-scene mix (independent units, no data-path collective)."""
    return 3 + 7919 * rank


# ---------------------------------------------------------------- CPU restatement (oracle) timing
def cpu_body_steps(scenes, warmup: int, steps: int, budget_s: float, threads: int, order=None):
    """The oracle (the reference's CPU path, restated; built -march=native on this host) steps each scene from rest in
    the reference's own list order: `warmup` untimed steps, then up to `steps` timed steps or until `budget_s` per
    scene. Scenes are taken largest first by `threads` worker threads (the oracle releases the GIL). Returns
    (body-steps/s, timed steps in all, scenes that ran every step): body-steps over the slowest thread's summed
    timed seconds."""
    import queue

    from oracle import binding as orc
    order = orc.ORDER_LIST if order is None else order
    work = queue.Queue()
    for sc in sorted(scenes, key=lambda x: -x.n_bodies):
        work.put(sc)
    per_thread = [0.0] * threads
    results = []
    lock = threading.Lock()

    def worker(t):
        while True:
            try:
                sc = work.get_nowait()
            except queue.Empty:
                return
            ow = orc.OracleWorld(sc)
            for _ in range(warmup):
                ow.step(DT, iterations=ITERS, order=order, pinch_kill=0)
            _, _, fl = ow.bodies()
            alive = int((fl & 1).sum())
            t0 = time.perf_counter()
            n = 0
            while n < steps and time.perf_counter() - t0 < budget_s:
                ow.step(DT, iterations=ITERS, order=order, pinch_kill=0)
                n += 1
            el = time.perf_counter() - t0
            _, _, fl = ow.bodies()
            ow.close()
            # bodies only leave by falling out of the world (pinch removal is off): the mean of start and end counts
            bsteps = n * (alive + int((fl & 1).sum())) / 2.0
            with lock:
                per_thread[t] += el
                results.append((bsteps, n, n == steps))

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    bsteps = sum(r[0] for r in results)
    el = max(per_thread) if results else 1.0
    return bsteps / max(el, 1e-9), sum(r[1] for r in results), sum(1 for r in results if r[2])


def median_scene(scenes):
    order = np.argsort([s.n_bodies for s in scenes])
    return scenes[int(order[len(order) // 2])]


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_name() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_arm(args, rank, world, pg):
    """The reference's CPU path, restated (the Rust/wasm reference cannot be built here), on every host thread: the
    whole 256-scene mix, each scene stepped from rest over the same window as our arm (warm-up untimed)."""
    if rank != 0:
        return
    from oracle import binding as orc
    from shatterforge_b200 import scenes as S
    orc.use_native()
    scenes = S.debris_mix(n_scenes=args.scenes, scale=args.scale)
    threads = host_threads()
    per = max(1.0, args.cpu_seconds)
    rate, steps, complete = cpu_body_steps(scenes, args.warmup, args.steps, per, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"debris mix: {args.scenes} scenes, 1/60 s, {ITERS} iterations, 2 substeps",
                   "sample": f"all {len(scenes)} scenes ({sum(s.n_bodies for s in scenes)} bodies), steps {args.warmup}.."
                             f"{args.warmup + args.steps} from rest; {complete} scenes ran every step (at most "
                             f"{per:.0f} s of timed stepping each)"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_name(),
                         "order": "reference list order (src/lib.rs:1579-1601)", "build": "-O2 -march=native -ffp-contract=off",
                         "sample": f"{len(scenes)} scenes over {threads} threads, largest first; {steps} timed scene-steps"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_steps(w, k: int, awake_out: list | None = None):
    """k world steps, one call each; returns (summed alive bodies, device ms from the library's events). The summed
    awake bodies (after each step) go to awake_out[0] when given."""
    alive = 0
    awake = 0
    ms = 0.0
    for _ in range(k):
        st = w.step(DT, 1)
        alive += st.alive
        awake += st.awake
        ms += st.ms_last_step
    if awake_out is not None:
        awake_out.append(awake)
    return alive, ms


# ---------------------------------------------------------------- serving
def _latency(res, kind=None):
    lat = np.array([(r["t_done"] - r["t_arrival"]) * 1e3 for r in res if kind is None or r["kind"] == kind])
    if len(lat) == 0:
        return None
    return {"n": int(len(lat)), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p999_ms": float(np.percentile(lat, 99.9)), "mean_ms": float(lat.mean())}


def colour_comparison(scenes, params):
    """The GPU colouring's colour count beside the reference's round-based colouring (gpu/gpu_world.js:922-1038,
    restated in the CPU oracle) on the same manifolds, 100 steps into 16 scenes of the mix (near their contact peak)."""
    import shatterforge_b200 as sf
    from oracle import binding as orc
    w = sf.World(scenes, **params)
    w.step(DT, nsteps=100)
    ref_max, ovf, n = 0, 0, 0
    for k, sc in enumerate(scenes):
        m = w.manifolds(k)
        if len(m) == 0:
            continue
        b = m[:, 1]
        _, used, o = orc.ref_colouring(m[:, 0], b, np.ones(len(m), np.uint8), (b != 0xFFFFFFFF).astype(np.uint8), sc.n_bodies)
        ref_max, ovf, n = max(ref_max, used), ovf + o, n + len(m)
    out = {"gpu": int(w.stats().colors), "gpu_overflow": 0, "reference_algorithm": ref_max, "reference_overflow": ovf,
           "manifolds": n, "note": "greedy colouring by priority (Jones-Plassmann rounds) vs the reference's 16 colours "
                                   "in 2 + 4 claim rounds with an overflow pass, on the same manifolds"}
    w.close()
    return out


def serve_run(args, worlds, structs, slots, batching: bool, seconds: float, seed: int, states=None):
    """One server on the population, fed a Poisson stream of `seconds` at --serve-rate; returns the summary."""
    import shatterforge_b200 as sf
    from shatterforge_b200 import serving as SV

    srv = SV.Server(slots=slots, structures=structs, budget_bytes=int(args.serve_budget_gb * 2**30), batching=batching,
                    sweeps_per_tick=128, iterations=ITERS, pinch_kill=0)
    ids = [srv.add_scene(w) for w in worlds]
    if states is not None:
        for i, st in zip(ids, states):
            srv.set_scene_state(i, *st)
    sids = structs.structure_ids()
    srv.start()
    # resident structures start solved (their potentials are part of the resident state)
    for q in sids:
        srv.submit_solve(q, omega=1.7, tol=1e-6, max_sweeps=200000)
    srv.drain(600000)
    srv.poll(cap=len(sids) + 8)
    rng = np.random.default_rng(seed)
    n = int(args.serve_rate * seconds)
    t0 = srv.stats()["now_s"] + 0.05
    t = t0 + np.cumsum(rng.exponential(1.0 / args.serve_rate, n))
    steps_of = {}
    bricks_of = {q: np.nonzero(structs.static_sid == q)[0] for q in sids}
    for k in range(n):
        if rng.random() < 0.7:
            wid = int(rng.integers(len(ids)))
            ns = int(rng.integers(1, 9))
            steps_of[srv.submit_step(ids[wid], ns, t_arrival=float(t[k]))] = ns * worlds[wid].n_bodies
        else:
            q = int(sids[int(rng.integers(len(sids)))])
            lb = rng.choice(bricks_of[q], 3)
            lv = rng.uniform(50.0, 400.0, 3).astype(np.float32)
            srv.submit_solve(q, omega=1.7, tol=1e-6, max_sweeps=20000, loads=(lb, lv), t_arrival=float(t[k]))
    unfinished = 0
    try:
        srv.drain(int(max(60.0, 20 * seconds) * 1000))
    except sf.SfError:
        unfinished = srv.stats()["pending"]
    res = srv.poll(cap=n + 16)
    st = srv.stats()
    srv.close()
    done = [r for r in res if r["status"] == 0]
    span = max(r["t_done"] for r in done) - t0 if done else float("nan")
    body_steps = sum(steps_of.get(r["ticket"], 0) for r in done)
    return {"requests": n, "completed": len(done), "unfinished": int(unfinished), "seconds_of_arrivals": seconds,
            "throughput_req_s": len(done) / span, "served_body_steps_per_s": body_steps / span,
            "all": _latency(done), "step": _latency(done, 1), "solve": _latency(done, 2),
            "ticks": {"step": int(st["step_ticks"]), "solve": int(st["solve_ticks"])},
            "loads": int(st["loads"]), "restores": int(st["restores"]), "evictions": int(st["evictions"]),
            "resident_gb": st["pool_bytes"] / 2**30}


def serve_section(args):
    from shatterforge_b200 import scenes as S
    from shatterforge_b200 import serving as SV

    rng = np.random.default_rng(17)
    sizes = np.exp(rng.uniform(math.log(1000), math.log(100000), args.serve_worlds)).astype(np.int64)
    lib = S.ClusterLibrary(0x51ED)
    worlds = [S.debris_scene(int(nb), seed=5000 + k, lib=lib, name=f"served{k}") for k, nb in enumerate(sizes)]
    structs = S.structure_lattice(seed=7)
    # one slot per world while the budget holds them all; otherwise fewer slots of the largest size (LRU eviction)
    slots = [SV.slot_for(w_) for w_ in worlds]
    budget = int(args.serve_budget_gb * 2**30) - 4 * 2**30      # headroom for the structures world and scratch
    if SV.pool_bytes(slots) > budget:
        big = tuple(max(c[i] for c in slots) for i in range(4))
        k = max(1, budget // SV.pool_bytes([big]))
        slots = [big] * int(min(k, len(worlds)))
    batched = serve_run(args, worlds, structs, slots, True, args.serve_seconds, seed=23)
    plain = serve_run(args, worlds, structs, slots, False, args.serve_plain_seconds, seed=23)
    aged = None
    if args.serve_age_steps > 0:
        # the same population after it has run a while (most debris settled): the worlds a server keeps resident
        import shatterforge_b200 as sf
        wa = sf.World(worlds, iterations=ITERS, pinch_kill=0)
        wa.step(DT, nsteps=args.serve_age_steps)
        st, sl, fl = wa.bodies()
        awake = int(wa.stats().awake)
        off = wa.body_off
        states = [(st[off[k]:off[k + 1]], sl[off[k]:off[k + 1]], fl[off[k]:off[k + 1]]) for k in range(len(worlds))]
        wa.close()
        aged = {"age_steps": args.serve_age_steps, "awake_bodies": awake,
                "batched": serve_run(args, worlds, structs, slots, True, args.serve_seconds, seed=29, states=states),
                "plain": serve_run(args, worlds, structs, slots, False, args.serve_plain_seconds, seed=29, states=states)}
    return {"rate_req_s": args.serve_rate, "worlds": len(worlds), "world_bodies": int(sizes.sum()),
            "structures": len(structs.structure_ids()), "structure_bricks": structs.n_static,
            "slots": len(slots), "budget_gb": args.serve_budget_gb, "mix": "70% scene steps (1-8 steps), 30% structure "
            "solves (3 random loads of 50-400 kg, omega 1.7 to 1e-6, from resident potentials)",
            "batched": batched, "plain": plain, "aged": aged,
            "note": "latency = completion - arrival on the server clock; plain = one request at a time with its own "
                    "launches, on the same population and the first seconds of the same stream"}


def plain_compare(sf, scenes, params, stream, args):
    """The plain path (every scene its own world, stepped one scene per launch sequence) against the batched path over
    the same steps from the same state: (a) the headline's window, steps warmup..warmup+K from rest (K at most
    --plain-steps-window); (b) --plain-steps steps at the mix's contact peak (after --peak-step steps)."""
    import torch

    def timed(fn):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        out = fn()
        t1.record(stream); torch.cuda.synchronize()
        return out, t0.elapsed_time(t1)

    def window(wb, worlds, k):
        acc = []
        b_alive, _ = run_steps(wb, k, acc)
        return b_alive, acc[0]

    def plain_steps(worlds, k):
        alive = awake = 0
        for _ in range(k):
            for pw in worlds:
                st = pw.step(DT, 1)
                alive += st.alive
                awake += st.awake
        return alive, awake

    out = {}
    wb = sf.World(scenes, **params)
    wb.set_stream(stream.cuda_stream)
    worlds = []
    for sc in scenes:
        pw = sf.World(sc, **params)
        pw.set_stream(stream.cuda_stream)
        worlds.append(pw)
    # (a) from rest, the headline's window
    run_steps(wb, args.warmup)
    for pw in worlds:
        run_steps(pw, args.warmup)
    k = min(args.steps, args.plain_steps_window)
    (b_alive, b_awake), b_ms = timed(lambda: window(wb, worlds, k))
    (p_alive, p_awake), p_ms = timed(lambda: plain_steps(worlds, k))
    out["window"] = {"steps": f"{args.warmup}..{args.warmup + k} from rest", "plain": p_alive / (p_ms * 1e-3),
                     "batched": b_alive / (b_ms * 1e-3), "batched_over_plain": (b_alive / b_ms) / max(p_alive / p_ms, 1e-30),
                     "awake_fraction": b_awake / max(b_alive, 1)}
    # (b) at the contact peak, from the batched world's state
    run_steps(wb, max(0, args.peak_step - args.warmup - k))
    st, sl, fl = wb.bodies()
    for j, pw in enumerate(worlds):
        a, b = wb.body_off[j], wb.body_off[j + 1]
        pw.set_bodies(st[a:b], sl[a:b], fl[a:b])
    (b_alive, b_awake), b_ms = timed(lambda: window(wb, worlds, args.plain_steps))
    (p_alive, p_awake), p_ms = timed(lambda: plain_steps(worlds, args.plain_steps))
    out["peak"] = {"steps": f"{args.peak_step}..{args.peak_step + args.plain_steps}", "plain": p_alive / (p_ms * 1e-3),
                   "batched": b_alive / (b_ms * 1e-3), "batched_over_plain": (b_alive / b_ms) / max(p_alive / p_ms, 1e-30),
                   "awake_fraction": b_awake / max(b_alive, 1), "contacts": int(wb.stats().contacts)}
    out["value"] = out["window"]["plain"]
    out["unit"] = UNIT
    out["note"] = "plain = each scene its own world and launches; batched = all scenes in one world, same steps, same state"
    for pw in worlds:
        pw.close()
    wb.close()
    return out


def collapse_section(sf, S, args, stream):
    """The 16-storey tower (47,760 bricks) with eight ground columns removed, run frame by frame in the reference's
    order (substeps with damage on contact, rebuild of the marked bodies, connectivity, the resting loads, the
    structures' load-path frame and the debris pieces' load fields and joints, connectivity again;
    src/lib.rs:3650-3659): wall time per frame with its parts, and the oracle running the same frames in the
    reference's list order on one host thread."""
    import torch
    tw, rm = S.tower16_structure()
    sc = tw.without_static(rm)
    ids = sc.structure_ids()
    frames = args.collapse_frames
    w = sf.World(sc, iterations=ITERS, detach_bodies=8000, detach_bricks=60000, damage=1, max_colors=1024)
    w.set_stream(stream.cuda_stream)
    for s in ids:
        w.structure_warm(s)
    parts = {"step": 0.0, "rebuild": 0.0, "connectivity": 0.0, "load_path": 0.0, "piece_fields": 0.0}
    tally = {"crushed": 0, "pieces_split": 0, "pieces_detached": 0, "joints_failed": 0, "piece_joints_failed": 0,
             "piece_bricks_crushed": 0, "piece_brick_updates": 0}
    torch.cuda.synchronize()
    t_all = time.perf_counter()
    ft = []
    for f in range(1, frames + 1):
        tf = time.perf_counter()
        t = time.perf_counter(); w.step(DT); torch.cuda.synchronize(); parts["step"] += time.perf_counter() - t
        t = time.perf_counter(); rb = w.rebuild_bodies(); parts["rebuild"] += time.perf_counter() - t
        t = time.perf_counter(); c1, _, _ = w.connectivity(); parts["connectivity"] += time.perf_counter() - t
        t = time.perf_counter()
        w.structure_loads(ids)
        fr = w.structure_frame(f, ids, dt=DT)
        parts["load_path"] += time.perf_counter() - t
        t = time.perf_counter(); bf = w.bodies_frame(DT, fr.crushed); parts["piece_fields"] += time.perf_counter() - t
        t = time.perf_counter(); c2, _, _ = w.connectivity(); parts["connectivity"] += time.perf_counter() - t
        tally["piece_joints_failed"] += int(bf.failed)
        tally["piece_bricks_crushed"] += int(bf.crushed)
        tally["piece_brick_updates"] += int(bf.brick_updates)
        tally["pieces_split"] += rb.pieces
        tally["pieces_detached"] += c1.pieces + c2.pieces
        tally["joints_failed"] += int(fr.failed)
        tally["crushed"] += int(w.damage()[0].crushed)
        ft.append(time.perf_counter() - tf)
    wall = time.perf_counter() - t_all
    st = w.stats()
    out = {"workload": f"16-storey tower, 47,760 bricks, 8 ground columns removed, {frames} frames, damage on",
           "ms_per_frame": wall * 1e3 / frames, "parts_ms_per_frame": {k: v * 1e3 / frames for k, v in parts.items()},
           "bodies_alive_at_end": int(st.alive), **tally}
    w.close()
    if not args.no_cpu:
        from oracle import binding as orc
        orc.use_native()
        ow = orc.OracleWorld(sc)
        ow.set_capacity(8000, 60000)
        for s in ids:
            ow.structure_warm(s)
        t0 = time.perf_counter()
        n = 0
        for f in range(1, frames + 1):
            ow.step(DT, iterations=ITERS, order=orc.ORDER_LIST, damage=1)
            ow.rebuild_bodies()
            ow.connectivity()
            ow.structure_loads(ids)
            o = ow.structure_frame(f, DT, ids)
            ow.body_frame(DT, o[6])
            ow.connectivity()
            n = f
            if time.perf_counter() - t0 > args.cpu_seconds:
                break
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"ms_per_frame": cpu_s * 1e3 / n, "frames": f"1..{n}", "cores": 1, "kind": "port",
                               "order": "reference list order",
                               "gpu_ms_per_frame_same_frames": sum(ft[:n]) * 1e3 / n}
    return out


def sat_section(sf, args):
    """The batched narrow-phase calls: box-box SAT (engine/src/phys.rs:502-628) on 1M random overlapping pairs and
    convex-cell SAT (gpu/gpu_world.js:421-530) on 200k pairs of the hull library, timed through the C ABI with host
    arrays (device allocation, copies both ways and the kernel inside the timed call), best of three; the oracle's
    restatement on one host thread on a sample of the same pairs."""
    from shatterforge_b200 import hulls
    rng = np.random.default_rng(7)

    def quats(n):
        q = rng.normal(size=(n, 4))
        return q / np.linalg.norm(q, axis=1, keepdims=True)

    nb = 1 << 20
    ba = np.zeros((nb, 10), np.float32); bb = np.zeros((nb, 10), np.float32)
    for x in (ba, bb):
        x[:, :3] = rng.uniform(-0.6, 0.6, (nb, 3)); x[:, 3:7] = quats(nb); x[:, 7:] = rng.uniform(0.1, 0.6, (nb, 3))
    data = hulls.library().packed()
    nh = 200000
    ha = np.zeros((nh, 11), np.float32); hb = np.zeros((nh, 11), np.float32)
    for x in (ha, hb):
        x[:, :3] = rng.uniform(-0.45, 0.45, (nh, 3)); x[:, 3:7] = quats(nh); x[:, 7:10] = rng.uniform(0.15, 0.5, (nh, 3))
        x[:, 10] = rng.integers(0, len(data), nh)

    def best(f):
        t = []
        for _ in range(3):
            t0 = time.perf_counter(); r = f(); t.append(time.perf_counter() - t0)
        return min(t), r
    tb, (cb, _, _) = best(lambda: sf.collide_boxes(ba, bb, margin=0.02))
    th, (ch, _, _) = best(lambda: sf.collide_hulls(data, ha, hb, margin=0.02))
    out = {"boxes": {"pairs": nb, "pairs_per_s": nb / tb, "ms": tb * 1e3, "touching": int((cb > 0).sum()),
                     "bytes_per_pair": 10 * 4 * 2 + 20 * 4 + 4},
           "hulls": {"pairs": nh, "pairs_per_s": nh / th, "ms": th * 1e3, "touching": int((ch > 0).sum()),
                     "bytes_per_pair": 11 * 4 * 2 + 36 * 4 + 4},
           "note": "end to end through the C ABI with host arrays: allocation, host-device copies and the kernel"}
    if not args.no_cpu:
        from oracle import binding as orc
        orc.use_native()
        ns, nsh = 200000, 50000
        t0 = time.perf_counter()
        hits_b = orc.collide_batch_hits(ba[:ns], bb[:ns])
        tcb = time.perf_counter() - t0
        t0 = time.perf_counter()
        hits_h = orc.collide_batch_hits(ha[:nsh], hb[:nsh], hull_data=data)
        tch = time.perf_counter() - t0
        out["cpu_baseline"] = {"boxes_pairs_per_s": ns / tcb, "hulls_pairs_per_s": nsh / tch, "cores": 1,
                               "kind": "port", "sample": f"the first {ns} box pairs and {nsh} hull pairs in one call "
                               f"each ({hits_b} and {hits_h} touching)"}
    return out


def boxes_section(args):
    """The engine crate's box world (engine/src/phys.rs World::step) on the GPU: the reference's throughput pile of
    20,000 boxes at 12 sub-steps without sleep (its published CPU figure: 226 ms a 60 Hz step on one core of a
    2.8 GHz Xeon, docs/PHASE0.md:12), timed on the device after it has landed; a batch of 148 piles of 2,000 (one
    scene a block); end to end through the C ABI (the boxes uploaded, the steps, the state read back); and the
    oracle's list-order restatement of the same step on one host thread."""
    from shatterforge_b200 import boxes as X
    dt = np.float32(1.0 / 60.0)
    p = X.box_params(allow_sleep=0)
    big = X.pile(20000)
    out = {"workload": "pile(20000) (engine/src/phys.rs:631-646), 12 sub-steps, no sleep, dt 1/60 s"}
    w = X.BoxWorld(big, p)
    w.step(dt, args.box_warmup)
    w.step(dt, args.box_steps)
    st = w.stats()
    ms = st.ms / args.box_steps
    out.update({"ms_per_step": ms, "box_steps_per_s": 20000 / (ms * 1e-3), "warmup_steps": args.box_warmup,
                "timed_steps": args.box_steps, "pairs": int(st.pairs), "manifolds": int(st.manifolds),
                "points": int(st.points), "colours": int(st.colours), "colour_rounds": int(st.rounds),
                "reference_cpu_ms_per_step": 226.0,
                "reference_note": "docs/PHASE0.md:12, native, 1 thread, 2.8 GHz Xeon VM (not rerunnable here)"})
    w.close()
    # the reference's other published figure: the same pile at 4 sub-steps, 118 ms natively (docs/PHASE0.md:12)
    w = X.BoxWorld(big, X.box_params(allow_sleep=0, substeps=4))
    w.step(dt, args.box_warmup)
    w.step(dt, args.box_steps)
    st4 = w.stats()
    out["substeps4"] = {"ms_per_step": st4.ms / args.box_steps, "box_steps_per_s": 20000 / (st4.ms / args.box_steps * 1e-3),
                        "reference_cpu_ms_per_step": 118.0}
    w.close()
    t0 = time.perf_counter()
    w = X.BoxWorld(big, p)
    w.step(dt, args.box_warmup + args.box_steps)
    _ = w.state()
    e2e_s = time.perf_counter() - t0
    w.close()
    out["e2e"] = {"ms_per_step": e2e_s * 1e3 / (args.box_warmup + args.box_steps),
                  "note": "wall clock: create (host boxes uploaded), every step, state read back",
                  "h2d_bytes": int(big.nbytes), "d2h_bytes": 20000 * 22 * 4}
    # the same pile with convex cells of the hull library in place of four boxes in five (the WebGPU world's hull
    # shapes, their pairs through the convex-cell SAT)
    from shatterforge_b200 import hulls
    lib = hulls.library().packed()
    ids = np.random.default_rng(3).integers(1, len(lib), 20000).astype(np.uint32)
    ids[::5] = 0
    w = X.BoxWorld(big, p)
    w.set_hulls(lib, ids)
    w.step(dt, args.box_warmup)
    w.step(dt, args.box_steps)
    st = w.stats()
    out["cells"] = {"workload": "pile(20000), four boxes in five replaced by convex cells, 12 sub-steps, no sleep",
                    "ms_per_step": st.ms / args.box_steps, "box_steps_per_s": 20000 / (st.ms / args.box_steps * 1e-3),
                    "pairs": int(st.pairs), "manifolds": int(st.manifolds), "colours": int(st.colours)}
    w.close()
    batch = [X.pile(2000)] * 148
    w = X.BoxWorld(batch, p)
    w.step(dt, args.box_warmup)
    w.step(dt, args.box_steps)
    st = w.stats()
    bms = st.ms / args.box_steps
    out["batch"] = {"scenes": 148, "boxes": 148 * 2000, "ms_per_step": bms,
                    "box_steps_per_s": 148 * 2000 / (bms * 1e-3)}
    w.close()
    if not args.no_cpu:
        from oracle import binding as orc
        orc.use_native()
        ow = orc.OracleBoxWorld(big, p, orc.ORDER_LIST)
        ow.step(dt, 2)
        n, t0 = 0, time.perf_counter()
        while n < args.box_steps and time.perf_counter() - t0 < args.cpu_seconds:
            ow.step(dt)
            n += 1
        cms = (time.perf_counter() - t0) * 1e3 / n
        out["cpu_baseline"] = {"ms_per_step": cms, "cores": 1, "kind": "port",
                               "sample": f"steps 3..{2 + n} of the same pile in the reference's list order"}
    return out


def our_arm(args, rank, world, local, pg):
    import torch

    import shatterforge_b200 as sf
    from shatterforge_b200 import scenes as S

    dev = torch.cuda.current_device()
    seed = rank_seed(rank)
    scenes = S.debris_mix(seed=seed, n_scenes=args.scenes, scale=args.scale)
    n_bodies = sum(s.n_bodies for s in scenes)
    n_bricks = sum(s.n_body_bricks for s in scenes)
    # a stream of its own (not the legacy default stream), so the library may capture its launch sequences in graphs
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    params = dict(iterations=ITERS, pinch_kill=0, verify=1)

    # ---- device-resident timed run
    w = sf.World(scenes, **params)
    w.set_stream(stream.cuda_stream)
    run_steps(w, args.warmup)
    w.set_profiling(True)
    w.reset_profile()
    barrier(pg, args)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    awake_acc = []
    with Clocks(dev) as clk:
        e0.record(stream)
        alive_sum, _ = run_steps(w, args.steps, awake_acc)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(pg, args)
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    prof = w.profile()
    tuning = w.tuning()
    stats = w.stats()
    ms_max, alive_total, _ = combine(pg, ms, alive_sum)
    awake_total = allreduce_sum(pg, float(awake_acc[0]))
    value = alive_total / (ms_max * 1e-3)

    # roofline of the dominant phase's kernel: contact generation or the solve, whichever phase took longer;
    # both are printed
    phase_ms = prof["ms"]
    top = max(phase_ms, key=phase_ms.get)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_source = "measured" if "hbm_gbs" in peaks else "fallback"
    launches = max(int(prof["substeps"]), 1)
    solve_ms = phase_ms["solve"]
    solve_bytes = SOLVE_BYTES_PER_CONTACT_ITER * prof["solve_contact_iters"]
    nsl = max(prof["solve_launches"], 1)
    roof_solve = {"kernel": "k_solve (coloured sequential-impulse solve)", "bound": "hbm",
                  "achieved": solve_bytes / max(solve_ms * 1e-3, 1e-12) / 1e9, "peak": hbm, "peak_source": peak_source,
                  "unit": "GB/s", "traffic": SOLVE_DRAM_BYTES_PER_CONTACT_ITER * prof["solve_contact_iters"] / nsl,
                  "bytes_per_launch": solve_bytes / nsl, "ms_per_launch": solve_ms / nsl, "launches": int(prof["solve_launches"]),
                  "unit_bytes": f"{SOLVE_BYTES_PER_CONTACT_ITER} B per contact-iteration"}
    roof_solve["frac"] = roof_solve["achieved"] / hbm
    gen_bytes = GEN_BYTES_PER_BRICK * prof["gen_bricks"] + GEN_BYTES_PER_CONTACT * prof["contacts_sum"]
    roof_gen = {"kernel": "k_contacts_gen (broad and narrow phase, one thread per awake brick)", "bound": "hbm",
                "achieved": gen_bytes / max(prof["gen_ms"] * 1e-3, 1e-12) / 1e9, "peak": hbm, "peak_source": peak_source,
                "unit": "GB/s", "traffic": GEN_DRAM_PER_ALGORITHMIC_BYTE * gen_bytes / launches,
                "bytes_per_launch": gen_bytes / launches, "ms_per_launch": prof["gen_ms"] / launches, "launches": launches,
                "unit_bytes": f"{GEN_BYTES_PER_BRICK} B per awake brick + {GEN_BYTES_PER_CONTACT} B per contact"}
    roof_gen["frac"] = roof_gen["achieved"] / hbm
    roofline = dict(roof_gen if phase_ms["contacts"] >= phase_ms["solve"] else roof_solve)
    roofline["phase_share"] = max(phase_ms["contacts"], phase_ms["solve"]) / max(sum(phase_ms.values()), 1e-12)
    rooflines = {"k_contacts_gen": roof_gen, "k_solve": roof_solve}
    w.close()

    # ---- plain path: each scene alone, stepped by its own launches; over the headline's step window from rest, and
    # for a few steps at the mix's contact peak, against the batched path over the same steps from the same state
    plain = None
    if not args.no_plain and rank == 0 and args.plain_steps > 0:
        plain = plain_compare(sf, scenes, params, stream, args)

    # ---- end to end through the C ABI with pinned host buffers
    e2e_steps = args.e2e_steps or args.steps
    we = sf.World(scenes, **params)
    we.set_stream(stream.cuda_stream)
    run_steps(we, args.warmup)
    nb = we.info.n_bodies
    h_state = torch.empty((nb, 13), dtype=torch.float32, pin_memory=True).numpy()
    h_sleep = torch.empty((nb,), dtype=torch.float32, pin_memory=True).numpy()
    h_flags = torch.empty((nb,), dtype=torch.uint8, pin_memory=True).numpy()
    s0, s1, s2 = we.bodies()
    h_state[:] = s0; h_sleep[:] = s1; h_flags[:] = s2
    barrier(pg, args)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_alive = 0
    for _ in range(e2e_steps):
        we.set_bodies(h_state, h_sleep, h_flags)
        e_alive += we.step(DT, 1).alive
        we.bodies(out=(h_state, h_sleep, h_flags))
    torch.cuda.synchronize()
    e_s = time.perf_counter() - t0
    barrier(pg, args)
    e_s = allreduce_max(pg, e_s)
    e_alive = allreduce_sum(pg, e_alive)
    bytes_io = nb * (13 * 4 + 4 + 1)
    e2e = {"value": e_alive / e_s, "unit": UNIT, "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
           "steps": e2e_steps, "note": "host-owned state: write bodies, step, read bodies, every step (pinned buffers)"}
    we.close()

    # ---- load path: 37 structures in one lattice, one persistent launch to residual 1e-6
    sor = None
    if not args.no_sor:
        c3 = S.structure_lattice(seed=2 + rank)
        ws = sf.World(c3)
        ws.set_stream(stream.cuda_stream)
        # warm-up: two full solves from zero. The first teaches the launch split each structure's sweep count (the
        # structures that take longest get the large blocks); the second captures the graph the timed solve replays
        for _ in range(2):
            ws.set_phi(np.zeros(c3.n_static, np.float32))
            ws.structure_solve(-1, omega=1.7, tol=1e-6, max_sweeps=args.sor_max_sweeps)
        ws.set_phi(np.zeros(c3.n_static, np.float32))
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        rep = ws.structure_solve(-1, omega=1.7, tol=1e-6, max_sweeps=args.sor_max_sweeps)
        t1.record(stream); torch.cuda.synchronize()
        s_ms = t0.elapsed_time(t1)
        bs = rep.brick_sweeps
        graphs = int(ws.stats().graph_launches)
        cluster = int(ws.stats().cluster_solves) > 0
        if cluster:
            # cells stay in shared memory for the whole solve: HBM is read and written once per solve, and a sweep
            # costs two cluster barriers and two dependent f64 cell updates, so the solve takes the critical
            # structure's sweep count times its time per sweep
            roof = {"bound": "sync", "unit": "us per sweep of the critical structure",
                    "achieved": s_ms * 1e3 / max(rep.max_sweeps_done, 1),
                    "hbm_bytes_per_solve": SOR_CLUSTER_BYTES_PER_BRICK * c3.n_static,
                    "hbm_gbs_per_solve": SOR_CLUSTER_BYTES_PER_BRICK * c3.n_static / (s_ms * 1e-3) / 1e9, "peak_hbm": hbm}
        else:
            roof = {"bound": "hbm", "unit": "GB/s", "achieved": SOR_BYTES_PER_BRICK_SWEEP * bs / (s_ms * 1e-3) / 1e9,
                    "peak": hbm, "frac": SOR_BYTES_PER_BRICK_SWEEP * bs / (s_ms * 1e-3) / 1e9 / hbm,
                    "unit_bytes": f"{SOR_BYTES_PER_BRICK_SWEEP} B per brick-sweep"}
        sw, _ = ws.solve_detail()
        counts = np.bincount(c3.static_sid, minlength=len(sw))
        slow = np.argsort(-sw.astype(np.int64))[:5]
        sor_slowest = [{"structure": int(q), "bricks": int(counts[q]), "sweeps": int(sw[q])} for q in slow]
        sor = {"brick_sweeps_per_s": bs / (s_ms * 1e-3), "bricks": c3.n_static, "structures": rep.structures,
               "slowest": sor_slowest,
               "path": "one thread-block cluster per structure" if cluster else "grid-wide persistent kernel",
               "cuda_graph_replays": graphs, "autotune_blocks_per_sm": ws.tuning()["sor"],
               "max_sweeps": rep.max_sweeps_done, "brick_sweeps": bs, "ms": s_ms, "max_residual": rep.max_residual,
               "roofline": roof}
        ws.close()

    collapse = None
    if not args.no_collapse and rank == 0:
        collapse = collapse_section(sf, S, args, stream)
    sat = None
    if not args.no_sat and rank == 0:
        sat = sat_section(sf, args)
    boxes = None
    if not args.no_boxes and rank == 0:
        boxes = boxes_section(args)

    # ---- CPU baseline: the oracle on a bounded sample of the same workload and step window
    cpu = None
    serve = None
    if not args.no_serve and rank == 0:
        serve = serve_section(args)

    if not args.no_cpu and rank == 0:
        from oracle import binding as orc
        cpu_colours = colour_comparison(scenes[:16], params)
        orc.use_native()
        med = median_scene(scenes)
        rate1, n1, _ = cpu_body_steps([med], args.warmup, args.steps, args.cpu_seconds, 1)
        threads = host_threads()
        rate_n, n_n, complete = cpu_body_steps(scenes, args.warmup, args.steps, args.cpu_seconds, threads)
        cpu = {"value": rate1, "unit": UNIT, "cores": 1, "kind": "port", "cpu": cpu_name(),
               "order": "reference list order (src/lib.rs:1579-1601)", "build": "-O2 -march=native -ffp-contract=off",
               "sample": f"the median scene ({med.n_bodies} bodies), steps {args.warmup}..{args.warmup + n1} from rest",
               "all_cores": {"value": rate_n, "cores": threads,
                             "sample": f"all {len(scenes)} scenes, largest first over {threads} threads, steps "
                                       f"{args.warmup}..{args.warmup + args.steps} from rest ({complete} scenes ran "
                                       f"every step; {n_n} timed scene-steps)"},
               "colours": cpu_colours}

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generators of the configured shapes)",
        "config": {"workload": f"debris mix: {args.scenes} scenes in one batch, {n_bodies} bodies, {n_bricks} brick spheres"
                               f" per GPU, dt 1/60 s, {ITERS} iterations, 2 substeps",
                   "scenes": args.scenes, "bodies_per_gpu": n_bodies, "bricks_per_gpu": n_bricks, "iterations": ITERS,
                   "substeps": 2, "pinch_kill": 0, "l2": "inputs larger than L2 (world state several hundred MB)",
                   "parallelism": f"{world} independent replica(s)"},
        "clocks": clocks,
        "e2e": e2e,
        "gpu_launches": int(prof["launches"]),
        "awake_fraction": awake_total / max(alive_total, 1),
        "awake_body_steps_per_s": awake_total / (ms_max * 1e-3),
        "roofline": roofline,
        "rooflines": rooflines,
        "phases_ms": {k: round(v, 3) for k, v in phase_ms.items()},
        "top_phase": top,
        "autotune": {"blocks_per_sm_by_log2_size": tuning, "note": "launch shapes picked online per size bucket; "
                     "they do not change results"},
        "last_step": {"contacts": int(stats.contacts), "manifolds": int(stats.manifolds), "colors": int(stats.colors),
                      "color_rounds": int(stats.color_rounds), "islands": int(stats.islands), "alive": int(stats.alive),
                      "awake": int(stats.awake)},
        "plain": plain,
        "sor": sor,
        "collapse": collapse,
        "sat": sat,
        "boxes": boxes,
        "cpu_baseline": cpu,
        "serve": serve,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world, pg)
        else:
            our_arm(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
