#!/usr/bin/env python
"""Benchmark of ysim's per-substep cloth hot path on B200.

Workload: the plain TriangularCloth 512x512 self-colliding cloth (262,144
vertices, 522,242 triangles) over a static displaced level-7 icosphere
(327,680 triangles), subh = 1/1200, 20 substeps per frame.  A step is one
substep: swept LBVH refit, broad phase (hash-semantics self rows + BVH rows
against the obstacle), narrow phase, per-vertex contacts, spring forces and
integration; every 10th frame also rebuilds the cloth's LBVH (Morton, radix
sort, Karras), amortised into the timed steps as it comes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  value = substeps/s over all ranks, timed on the
device with CUDA events on the scene's stream around each substep (one CUDA
graph launch: refit and fused kernel), the L2 flushed (a 256 MiB write)
between timed substeps and excluded from the timed intervals; the roofline's
per-kernel durations come from bursts of further substeps interleaved with
the timed ones, with events around each kernel.  e2e =
the same metric through the public API with host buffers, from the state the
timed substeps started from (so the same stretch of the drape): every frame uploads
the external-force buffer from pinned host memory (applyEnvironmentForces'
output) and reads the positions back into pinned host memory.
Multi-GPU: replicas only (one independent cloth per rank, no collective on the
data path); value sums the ranks' substeps over the slowest rank's time.

The line also carries, measured in the same run: batched vs plain (C4, 256
instances), the adjoint (C5), the tree builders on the C2 cloth, C1 over
analytic colliders, C2 with BVH self rows, and the collision microbenchmark
(C3: LBVH and spatial hash at 1M / 4M / 16M triangles, face-face hash on the
C2 geometry).  --no-batched / --no-adjoint / --no-collide leave those out.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "substeps/s at 262k-vert self-colliding cloth; batched vs plain; adjoint ms/step"
UNIT = "substeps/s"
# Untimed substeps before the warm-up of the headline workload.  The 512x512
# cloth starts 0.046 above the obstacle's top and falls at 1 m/s^2: its first
# contacts come near substep 370, and at substep 500 it has about 11k contacts
# per substep (18k at 540, 54k at 800), so every timed substep is in the
# contact regime whatever --steps is.
PREROLL = 500


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--preroll", type=int, default=PREROLL,
                    help="untimed substeps before warm-up; the default puts the timed substeps in the contact "
                         "regime of the drape (first contacts near substep 370, about 11k per substep at 500)")
    ap.add_argument("--allow-free-fall", action="store_true",
                    help="report a run whose timed substeps saw no contacts instead of failing it")
    ap.add_argument("--e2e-frames", type=int, default=None,
                    help="end-to-end frames (default: the frames the timed substeps make up)")
    ap.add_argument("--cpu-substeps", type=int, default=3, help="substeps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--P", type=int, default=512)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-vs-plain (C4) object")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (C5) object")
    ap.add_argument("--no-collide", action="store_true",
                    help="skip the collision microbenchmark (C3: 1M / 4M / 16M triangles) object")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--workload", choices=["cloth", "collide", "batched", "adjoint", "c2-kernels"], default="cloth",
                    help="cloth: the headline substep benchmark; collide: the LBVH / spatial-hash microbenchmark; "
                         "batched / adjoint: that object of the headline line alone; c2-kernels: the headline "
                         "workload's kernels launched one by one for a profiler (pre-roll, --steps substeps "
                         "without graphs, then one build of the cloth's tree with each builder)")
    ap.add_argument("--sizes", default="1000000,4000000,16000000")
    ap.add_argument("--fused-variant", type=int, choices=[8, 7, 4], default=None,
                    help="use this fused-kernel variant (CTAs per SM) instead of the autotuner's choice")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def spec_for(args):
    from ysim_b200 import generators as G
    return G.config_c2(seed=args.seed, P=args.P)


def workload_config(args, spec, extra=None):
    cloth = spec.meshes[0]
    ob = spec.meshes[1]
    cfg = {
        "workload": f"TriangularCloth {args.P}x{args.P} ({cloth.nV} v, {cloth.nF} tris) self-colliding + static "
                    f"displaced icosphere L7 ({ob.nF} tris); subh 1/1200, 20 substeps/frame; rebuild every 10 frames",
        "vertices": cloth.nV, "triangles": cloth.nF, "obstacle_triangles": ob.nF,
        "self_collision": "cpu-spatial-hash semantics (reference default)",
        "margin": spec.params.margin, "radius": spec.params.radius,
        "l2": "flushed between timed substeps (256 MiB write), excluded from timing",
        "seed": args.seed,
    }
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------------------ ranks
def max_over_ranks(ms: float, world: int, device=None) -> float:
    """Slowest rank's time (the timed region is bracketed by barriers on every
    rank; replicas do no data-path collective)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(ms: float, steps: int, world: int, device=None):
    """Whole-job substeps/s: every rank ran `steps` substeps of its own replica."""
    slow = max_over_ranks(ms, world, device)
    return world * steps / (slow / 1000.0), slow


# ------------------------------------------------------------------ clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def count(self) -> int:
        return len(self.lines)

    def wait_samples(self, n: int, busy, timeout_s: float):
        """Keep the GPU busy (busy()) until n samples have arrived or the
        timeout passes: nvidia-smi takes a few hundred ms to start and then
        samples every 200 ms, longer than a short timed region."""
        t0 = time.time()
        while self.proc and self.count() < n and time.time() - t0 < timeout_s:
            busy()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ roofline
def algorithmic_bytes(spec, rows_per_substep: float, contacts_per_substep: float):
    """Compulsory bytes per substep of the reference dataflow (each buffer
    element counted once per stage): refit kernel, and the stages the fused
    kernel covers (query, narrow, bucket, forces, integrate, snapshot)."""
    cloth, ob = spec.meshes[0], spec.meshes[1]
    V, M = cloth.nV, cloth.nF
    P = int(round(V ** 0.5))
    E = 3 * (P - 1) ** 2 + 2 * (P - 1)
    E_int = E - 4 * (P - 1)
    C, K = rows_per_substep, contacts_per_substep
    nodes = (2 * M - 1) + (2 * ob.nF - 1)
    refit = M * (8 + 12 + 32) + V * 24 + (2 * M - 1) * 32 * 1.5 + (2 * M - 1) * 8
    query = V * 12 + nodes * 32 + C * 8
    narrow = C * 8 + K * 48 + V * 24
    bucket = K * 48 * 2 + (V + 1) * 4 * 2
    forces = V * 48 + 2 * E * 4 + E * 12 + 2 * E_int * 8
    integ = V * (36 + 4 + 4 + 8 + 24) + K * 48
    snap = V * 24
    return {"refit": refit, "fused": query + narrow + bucket + forces + integ + snap}


def measured_traffic(args):
    """DRAM bytes per launch (read + write) of the dominant kernels from the
    committed ncu capture of this workload (profiles/), when it is the one
    captured (the 512x512 C2 cloth)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "traffic_c2_tricloth512.json")
    if args.P != 512 or not os.path.exists(path):
        return {}
    with open(path) as fh:
        d = json.load(fh)
    return {"k_fused": d.get("k_fused"), "refit": d.get("refit"),
            "k_fused_warp_instructions": d.get("k_fused_warp_instructions"),
            "k_fused_threads_per_instruction": d.get("k_fused_threads_per_instruction"),
            "source": "ncu captures of this workload in the contact phase: profiles/traffic_c2_tricloth512.json ("
                      + d.get("source", "") + ")"}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU baseline
def cpu_baseline(spec, state, nsub, threads=None):
    """Time the CPU oracle (all host threads) on `nsub` substeps of the same
    workload, started from the GPU run's state."""
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    cores = O.max_threads()
    o, kind = reference_scene(spec)
    if kind == "reference":
        o.x, o.v, o.xp = state["x"].copy(), state["v"].copy(), state["xprev"].copy()
    else:
        o.set("x", state["x"]); o.set("v", state["v"]); o.set("xprev", state["xprev"])
    o.step(1)  # frame-0 preamble rebuild, untimed
    t0 = time.perf_counter()
    o.step(nsub)
    dt = time.perf_counter() - t0
    # one more substep on a single host thread (the reference's CPU style)
    O.set_threads(1)
    t1 = time.perf_counter()
    o.step(1)
    dt1 = time.perf_counter() - t1
    O.set_threads(cores)
    return nsub / dt, cores, dt, kind, 1.0 / dt1


def reference_scene(spec):
    """The reference's own kernels on the host (oracle/_ref) when they were
    built from the reference checkout, else the pinned CPU restatement."""
    from oracle import oracle as O
    try:
        from oracle import refkernels
        if refkernels.available():
            refkernels.lib()
            from oracle.refdriver import RefScene
            return RefScene(spec), "reference"
    except (OSError, FileNotFoundError, RuntimeError):
        pass
    return O.OracleScene(spec), "port"


def run_reference(args, rank, world):
    """Reference arm: the path's CPU implementation on the host cores, all
    threads (OpenMP), on this arm's config and the same stretch of the drape.
    The pinned CPU restatement (bit-identical to the CUDA path's trajectory)
    pre-rolls the scene to the substep the CUDA arm's timed substeps start
    from (pre-roll + warm-up), untimed; the reference kernels then take that
    state, rebuild their trees in an untimed frame-0 substep, and time
    `steps` substeps (at most --cpu-substeps).  Rank 0 alone works."""
    if rank != 0:
        return
    from oracle import oracle as O
    spec = spec_for(args)
    cores = O.max_threads()
    start = args.preroll + max(args.warmup, 6)
    t0 = time.perf_counter()
    port = O.OracleScene(spec)
    port.step(max(start - 1, 0))
    preroll_s = time.perf_counter() - t0
    state = {"x": port.get("x"), "v": port.get("v"), "xprev": port.get("xprev")}
    scene, kind = reference_scene(spec)
    if kind == "reference":
        del port
        scene.x, scene.v, scene.xp = state["x"].copy(), state["v"].copy(), state["xprev"].copy()
    else:
        scene = port
    scene.step(1)  # frame-0 preamble of the reference kernels (tree build), untimed
    nsteps = max(1, min(args.steps, args.cpu_substeps))
    t0 = time.perf_counter()
    scene.step(nsteps)
    dt = time.perf_counter() - t0
    contacts = getattr(scene, "ncontacts", None)
    if contacts is None:
        contacts = scene.stats()["contacts"]
    v = nsteps / dt
    sample = (f"{nsteps} substeps of the full workload from substep {start} of the drape (the CUDA arm's first timed "
              f"substep; pre-rolled by the pinned CPU restatement in {preroll_s:.0f} s, untimed), after an untimed "
              "frame-0 tree build; ")
    sample += ("the reference's Metal kernels compiled for the host (oracle/_ref) with the pinned CPU-hash "
               "restatement for self rows" if kind == "reference" else "CPU restatement, OpenMP")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": nsteps,
        "warmup": start, "ms_per_step": 1000.0 * dt / nsteps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": workload_config(args, spec, {"parallelism": "host cores, OpenMP over kernel thread ids",
                                               "first_timed_substep": start,
                                               "contacts_last_substep": int(contacts)}),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from ysim_b200.scene import Scene

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    spec = spec_for(args)
    scene = Scene(spec, device=local)
    lib = scene.lib
    stream = torch.cuda.ExternalStream(scene.stream(), device=local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    # pre-roll frame by frame so a scene that goes unstable stops the run early
    done = 0
    while done < args.preroll:
        n = min(spec.params.substeps, args.preroll - done)
        scene.step(n)
        done += n
        st0 = scene.stats()
        if st0["flags"] & 1:
            if rank == 0:
                print(json.dumps({"metric": METRIC, "error": f"scene went non-finite during pre-roll at substep {done}",
                                  "stats": st0}), flush=True)
            sys.exit(3)
    tuned, tune_ms = scene.autotune()
    classes = scene.autotune_classes()
    if classes:
        tuned = classes[-1]["ctas_per_sm"]
    if args.fused_variant:  # a fixed variant (profiling: ncu perturbs the autotuner's timings)
        scene.set_fused_variant(args.fused_variant)
        scene.set_thread_order(True)
        tuned = args.fused_variant
    scene.step(max(args.warmup, 6))  # also re-captures the graphs the autotuner dropped
    scene.sync()
    scene.clear_flags()
    before = scene.totals()
    # the state the timed substeps start from; the end-to-end frames start
    # from it too, so both cover the same stretch of the drape
    snap = {k: scene.get(k) for k in ("x", "v", "xprev")}

    # ---- device-timed substeps (value)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    def gpu_busy():  # L2-flush fills: load on the GPU without advancing the scene
        with torch.cuda.stream(stream):
            for _ in range(16):
                flush.fill_(0.5)
        torch.cuda.synchronize()

    sampler.start()
    sampler.wait_samples(1, gpu_busy, 10.0)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    _lib_check = __import__("ysim_b200._lib", fromlist=["check"]).check
    # The substeps as the library runs them: one CUDA-graph launch each (the
    # flush before it keeps the GPU busy while the host enqueues, so no host
    # launch gap falls inside an interval).  Interleaved with them, in ten
    # bursts through the same stretch of the drape, a tenth as many further
    # substeps run with CUDA events around each kernel (direct launches):
    # their refit / fused durations and candidate / contact counts give the
    # roofline.  The bursts are not part of `value`.
    import ctypes as C
    chunks = min(10, args.steps)
    per = [args.steps // chunks + (1 if c < args.steps % chunks else 0) for c in range(chunks)]
    kper = max(1, args.steps // (10 * chunks))
    kt = [0.0, 0.0, 0.0, 0.0]
    k_rows = k_cont = 0
    ksteps = 0
    i = 0
    for c in range(chunks):
        for _ in range(per[c]):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
            starts[i].record(stream)
            scene.step(1)
            ends[i].record(stream)
            i += 1
        k_before = scene.totals()
        _lib_check(lib.ys_scene_set_timing(scene.h, 1), "set_timing")
        for _ in range(kper):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
            scene.step(1)
        scene.sync()
        burst = (C.c_double * 4)()
        _lib_check(lib.ys_scene_kernel_times(scene.h, burst), "kernel_times")
        _lib_check(lib.ys_scene_set_timing(scene.h, 0), "set_timing")
        kt = [kt[j] + burst[j] for j in range(4)]
        k_after = scene.totals()
        k_rows += k_after[0] - k_before[0]
        k_cont += k_after[1] - k_before[1]
        ksteps += kper
    torch.cuda.synchronize()
    scene.sync()
    sampler.wait_samples(sampler.count() + 2, gpu_busy, 3.0)
    clocks = sampler.stop()
    clocks["window"] = ("nvidia-smi every 200 ms from its first sample before the timed substeps to two samples "
                        "after them, the GPU kept busy by L2-flush fills outside the timed substeps")
    ms = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))
    after = scene.totals()
    st = scene.stats()
    value, ms = aggregate(ms, args.steps, world, device=f"cuda:{local}")
    # candidate rows and contacts per substep over the timed and the burst substeps
    rows_ps = (after[0] - before[0] - k_rows) / args.steps
    cont_ps = (after[1] - before[1] - k_cont) / args.steps
    k_rows_ps = k_rows / ksteps
    k_cont_ps = k_cont / ksteps
    if cont_ps == 0 and k_cont_ps == 0 and not args.allow_free_fall:
        # a window with no contacts times the free fall, where the narrow
        # phase's response and the contact lists never fire
        if rank == 0:
            print(json.dumps({"metric": METRIC, "error": "no contacts in the timed substeps (free fall); "
                              "lengthen --preroll or pass --allow-free-fall",
                              "preroll_substeps": args.preroll, "candidate_rows_per_substep": rows_ps}), flush=True)
        sys.exit(4)

    # ---- e2e through the public API with host buffers
    nsub = spec.params.substeps
    nV = scene.nV
    ext = torch.empty((nV, 3), dtype=torch.float32).pin_memory()
    mass = np.concatenate([m.mass if m.mass is not None else np.zeros(m.nV, np.float32) for m in spec.meshes])
    cloth_mask = np.concatenate([np.full(m.nV, 1.0 if m.behavior in (0, 1) else 0.0, np.float32)
                                 for m in spec.meshes])
    g = np.asarray(spec.params.gravity, np.float32)
    ext.numpy()[:] = (g[None, :] * (mass * cloth_mask)[:, None]).astype(np.float32)
    xout = torch.empty((nV, 3), dtype=torch.float32).pin_memory()
    for k in ("x", "v", "xprev"):
        scene.set(k, snap[k])
    # one untimed frame: the first external-force upload switches the force
    # source from g * m to the buffer, which drops and re-captures the
    # substep graphs
    _lib_check(lib.ys_scene_set_external_forces(scene.h, C.c_void_p(ext.data_ptr())), "ext")
    scene.step(nsub)
    _lib_check(lib.ys_scene_read_positions_async(scene.h, C.c_void_p(xout.data_ptr())), "read")
    scene.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    e2e_frames = args.e2e_frames if args.e2e_frames else max(1, -(-args.steps // nsub))
    for _ in range(e2e_frames):
        _lib_check(lib.ys_scene_set_external_forces(scene.h, C.c_void_p(ext.data_ptr())), "ext")
        scene.step(nsub)
        _lib_check(lib.ys_scene_read_positions_async(scene.h, C.c_void_p(xout.data_ptr())), "read")
    e1.record(stream)
    scene.sync()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_val, e2e_ms = aggregate(e2e_ms, e2e_frames * nsub, world, device=f"cuda:{local}")
    assert np.isfinite(xout.numpy()).all()

    # ---- roofline of the dominant kernel
    ab = algorithmic_bytes(spec, k_rows_ps, k_cont_ps)
    fused_ms = kt[2] / max(kt[3], 1)
    refit_ms = kt[0] / max(kt[1], 1)
    peak, peak_kind = measured_peak()
    ach = ab["fused"] / (fused_ms / 1000.0) / 1e9
    traffic = measured_traffic(args)
    roof = {"bound": "hbm", "kernel": "k_fused (query+narrow+contacts+forces+integrate)", "achieved": ach,
            "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": ach / peak,
            "traffic": traffic.get("k_fused"), "algorithmic_bytes": ab["fused"], "avg_launch_ms": fused_ms,
            "refit_kernel": {"achieved": ab["refit"] / (refit_ms / 1000.0) / 1e9, "algorithmic_bytes": ab["refit"],
                             "avg_launch_ms": refit_ms, "traffic": traffic.get("refit"),
                             "launches_per_substep": "range refit: leaf pass (sorted-leaf order, block boxes) + one pass for the nodes whose range crosses a 256-leaf block and the root"},
            "traffic_source": traffic.get("source")}
    # The kernel is issue- and latency-bound, not bandwidth-bound: the same
    # launch against the SMs' instruction-issue peak (148 SMs x 4 schedulers x
    # 1 warp instruction per cycle at the sampled SM clock), with the warp
    # instructions of the committed ncu capture of this workload.
    ninst = traffic.get("k_fused_warp_instructions")
    if ninst and clocks.get("sm_mhz"):
        peak_ginst = 148 * 4 * clocks["sm_mhz"] / 1000.0
        got = ninst / (fused_ms / 1000.0) / 1e9
        roof["issue"] = {"bound": "instruction issue", "warp_instructions": ninst, "achieved": got,
                         "peak": peak_ginst, "unit": "G warp inst/s", "frac": got / peak_ginst,
                         "threads_per_instruction": traffic.get("k_fused_threads_per_instruction"),
                         "source": "warp instructions per launch from the ncu capture; duration and clock live"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        state = {"x": scene.get("x"), "v": scene.get("v"), "xprev": scene.get("xprev")}
        v_cpu, cores, dt, kind, v_one = cpu_baseline(spec, state, args.cpu_substeps)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": cores, "kind": kind, "single_thread_value": v_one,
               "sample": f"{args.cpu_substeps} substeps of the full workload from the GPU run's state "
                         f"({dt:.1f} s on {cores} threads; "
                         + ("reference Metal kernels compiled for the host + pinned CPU-hash restatement)"
                            if kind == "reference" else "CPU restatement)")
                         + "; single_thread_value: one more substep on one host thread"}

    build = analytic = bvh_self = None
    collide = []
    if rank == 0:
        m0 = spec.meshes[0]
        build = measure_build(scene.get("x")[: m0.nV], m0.facets, local)
        analytic = measure_analytic(local)
        bvh_self = measure_bvh_self(args, spec, snap, local)
    batched = None if args.no_batched else measure_batched(args, rank, world, local)
    adjoint = None if (args.no_adjoint or rank != 0) else measure_adjoint(args, local)
    if rank == 0 and not args.no_collide:
        scene.close()  # room for the 16M-triangle microbenchmark
        run_collide(args, collide.append)

    # launches in the timed loop: per substep the refit's leaf kernel, its
    # level kernels and its top-level kernel, and k_fused (one CUDA graph);
    # kt counts the refit as one timed stage, so the level launches are taken
    # from the kernel list of the recorded substeps: 6 refit launches on C2
    refit_launches = 6 if spec.meshes[0].behavior == 0 and spec.params.self_mode else 1
    launches = int(round((kt[1] * refit_launches + kt[3]) / ksteps * args.steps))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 6), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": workload_config(args, spec, {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                                                   "candidate_rows_per_substep": rows_ps,
                                                   "contacts_per_substep": cont_ps, "preroll_substeps": args.preroll,
                                                   "first_timed_substep": args.preroll + max(args.warmup, 6),
                                                   "fused_variant": {"ctas_per_sm": tuned,
                                                                     "autotune_ms": dict(zip(("8", "7", "4"), tune_ms)),
                                                                     "per_size_class": classes},
                                                   "flags": st["flags"]}),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nV * 12 / nsub,
                    "d2h_bytes_per_step": nV * 12 / nsub,
                    "note": f"{e2e_frames} frames of {nsub} substeps from the state the timed substeps started "
                            "from (the same stretch of the drape), each with one external-force upload and one "
                            "position read-back (bytes shown per substep); no L2 flush between substeps, unlike "
                            "value"},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "batched": batched,
            "adjoint": adjoint,
            "tree_build": build,
            "analytic_colliders": analytic,
            "c2_bvh_self": bvh_self,
            "collide_c3": collide,
        }
        print(json.dumps(line), flush=True)
    scene.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ BVH self rows
def measure_bvh_self(args, spec, snap, local, steps=20):
    """C2 with BVH self rows (checkSelfCollisions, the reference's
    YSIM_CPUSH_SELF=0 path) instead of the CPU-hash semantics, from the state
    the headline's timed substeps started from: device-timed substeps/s of the
    library's CUDA-graph substep (its own per-class autotune first)."""
    import dataclasses
    import torch
    from ysim_b200 import _lib
    from ysim_b200.scene import Scene
    sp = dataclasses.replace(spec, params=dataclasses.replace(spec.params, self_mode=_lib.SELF_BVH))
    s = Scene(sp, device=local)
    try:
        for k in ("x", "v", "xprev"):
            s.set(k, snap[k])
        s.step(1)  # frame-0 rebuild from the draped state
        s.autotune_classes()
        s.step(6)
        stream = torch.cuda.ExternalStream(s.stream(), device=local)
        s.sync()
        before = s.totals()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        after = s.totals()
        return {"workload": "C2 with BVH self rows, from the headline's first timed state", "steps": steps,
                "substeps_per_s": 1000.0 / ms, "ms_per_substep": ms,
                "candidate_rows_per_substep": (after[0] - before[0]) / steps,
                "contacts_per_substep": (after[1] - before[1]) / steps, "flags": s.stats()["flags"],
                "timing": "CUDA events around the substeps (graph replays, no L2 flush)"}
    finally:
        s.close()


# ------------------------------------------------------------------ tree build
def measure_build(x, F, local, reps=10, warm=3):
    """One full rebuild of a tree (scene box, Morton codes, radix sort, then
    Karras topology + bottom-up boxes, or the Apetrei one-pass build) through
    the standalone LBVH, on the cloth's positions at the end of the run;
    median of `reps` CUDA-event-timed builds after 3 warm-up builds."""
    import ctypes as C
    import torch
    from ysim_b200 import _lib
    lib = _lib.load()
    dx = torch.from_numpy(np.ascontiguousarray(x, np.float32).reshape(-1)).to(f"cuda:{local}")
    df = torch.from_numpy(np.ascontiguousarray(F, np.uint32).view(np.int32).reshape(-1)).to(f"cuda:{local}")
    out = {"mesh": f"C2 cloth, {len(F):,} triangles", "reps": reps}
    for name, builder in (("karras", _lib.BUILD_KARRAS), ("apetrei", _lib.BUILD_APETREI)):
        h = C.c_void_p()
        _lib.check(lib.ys_lbvh_create(C.byref(h), len(F), local, None), "ys_lbvh_create")
        try:
            _lib.check(lib.ys_lbvh_set_builder(h, builder), "ys_lbvh_set_builder")
            times = []
            for i in range(warm + reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                _lib.check(lib.ys_lbvh_build(h, C.c_void_p(dx.data_ptr()), len(x), C.c_void_p(df.data_ptr()),
                                             len(F)), "ys_lbvh_build")
                e1.record()
                torch.cuda.synchronize()
                if i >= warm:
                    times.append(e0.elapsed_time(e1))
            out[f"{name}_ms"] = float(np.median(times))
        finally:
            lib.ys_lbvh_destroy(h)
    out["apetrei_over_karras"] = out["apetrei_ms"] / out["karras_ms"]
    return out


def measure_analytic(local, steps=200):
    """C1's FastGridCloth 64 x 64 draped over obstacles, fused substeps per
    second: over the triangle icosphere (level 4, BVH queries), and over
    analytic colliders (sphere, box, cylinder, floor plane; markers + shape
    tests, no obstacle tree).  Pre-rolled to contact, device-timed."""
    import torch
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    out = {"workload": "C1 cloth 64x64 (4,096 v), 200 fused substeps after a 2-frame pre-roll from height 0.32"}
    for name, spec in (("triangle_icosphere", G.config_c1(height=0.32)),
                       ("analytic_shapes", G.config_c1_analytic(height=0.32))):
        sc = Scene(spec, device=local)
        try:
            sc.step(2 * spec.params.substeps)
            stream = torch.cuda.ExternalStream(sc.stream(), device=local)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            sc.sync()
            e0.record(stream)
            sc.step(steps)
            e1.record(stream)
            sc.sync()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            st = sc.stats()
            out[name] = {"substeps_per_s": steps / (ms / 1000.0), "ms_per_substep": ms / steps,
                         "contacts_last_substep": st["contacts"], "flags": st["flags"]}
        finally:
            sc.close()
    return out


# ------------------------------------------------------------------ batched
def measure_batched(args, rank, world, local, steps=100):
    """Batched vs plain (C4): the instances of this rank's shard (balanced by
    vertex count, generators.shard_instances) as ONE scene -- one refit and one fused launch per
    substep for all of them, replayed as a CUDA graph -- against the same
    instances as one scene each, in two ways: (1) every instance stepped
    before the next substep, each scene on its own stream, so that their
    kernels overlap on the GPU (host clock between full synchronisations);
    (2) as the workload states it, each instance run through the plain path
    on its own, one after another (each run device-timed on its stream, the
    times summed).  Batched is device-timed (CUDA events on its stream).  All
    are the max over ranks; the whole batch advancing one substep is one
    batch substep."""
    import time
    import torch
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    full = G.config_c4(instances=args.instances)
    spec = G.shard_instances(full, rank, world)
    parts = G.split_instances(spec)
    scene = Scene(spec, device=local)
    stream = torch.cuda.ExternalStream(scene.stream(), device=local)
    scene.step(20)
    tuned, _ = scene.autotune()
    classes = scene.autotune_classes()
    scene.step(6)  # re-capture the substep graphs of all six buffer-rotation states, untimed
    scene.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    scene.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    b_ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, device=f"cuda:{local}")
    flags = scene.stats()["flags"]
    scene.close()
    plain = [Scene(p, device=local) for p in parts]
    for q, p in zip(plain, parts):
        # each instance is one size class of its own: the batched scene's
        # choice for that class, before the warm-up, which captures the graphs
        nv = max(m.nV for m in p.meshes if m.grid_n)
        ch = next((c for c in classes if nv <= c["max_mesh_vertices"]), None)
        q.set_fused_variant(ch["ctas_per_sm"] if ch else tuned)
        if ch:
            q.set_thread_order(ch["thread_order"])
        q.step(20)
    for q in plain:
        q.sync()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        for q in plain:
            q.step(1)
    for q in plain:
        q.sync()
    torch.cuda.synchronize()
    p_ms = max_over_ranks((time.perf_counter() - t) * 1e3 / steps, world, device=f"cuda:{local}")
    # the comparison as the workload states it: each instance run through the
    # plain path on its own, one after another; each run device-timed on its
    # scene's stream, the times summed
    seq = 0.0
    for q in plain:
        qs = torch.cuda.ExternalStream(q.stream(), device=local)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(qs)
        q.step(steps)
        b.record(qs)
        b.synchronize()
        seq += a.elapsed_time(b)
    s_ms = max_over_ranks(seq / steps, world, device=f"cuda:{local}")
    for q in plain:
        flags |= q.stats()["flags"]
        q.close()
    nverts = sum(m.nV for m in full.meshes)
    return {"workload": f"{args.instances} FastGridCloth instances, side U{{16..256}} (seeded), each over its own "
                        f"level-4 icosphere; subh 1/6000; instances sharded over {world} GPU(s), balanced by "
                        f"vertex count",
            "instances": args.instances, "vertices": nverts,
            "cloth_vertices": sum(m.nV for m in full.meshes if m.grid_n), "value": 1000.0 / b_ms,
            "unit": "batch substeps/s", "ms_per_substep": b_ms,
            "vertex_substeps_per_s": nverts * 1000.0 / b_ms,
            "plain": {"value": 1000.0 / p_ms, "ms_per_substep": p_ms,
                      "timing": "host clock between synchronisations (one scene per instance, own stream, "
                                "all instances stepped before the next substep: their kernels overlap)"},
            "batched_over_plain": p_ms / b_ms,
            "plain_sequential": {"value": 1000.0 / s_ms, "ms_per_substep": s_ms,
                                 "timing": "each instance alone through the plain path, one after another, "
                                           "device-timed (CUDA events on its stream) and summed"},
            "batched_over_plain_sequential": s_ms / b_ms, "steps": steps, "flags": flags,
            "fused_variant": {"per_size_class": classes,
                              "note": "one fused launch per size class of the instances, each with the register-cap "
                                      "variant and thread order ys_scene_autotune_classes chose on the batched "
                                      "scene's live state; each plain instance uses its class's choice"},
            "note": "the ~4.3M vertices quoted for this config differ from the drawn total (vertices above)"}


def measure_adjoint(args, local, steps=200, every=20, reps=4):
    """Adjoint (C5): FastGridCloth 128x128 over a level-4 icosphere, 200
    steps, checkpoints every 20; loss = mean |x_T - x*|^2 with x* the final
    state of a rollout whose per-spring stiffness is k exp(N(0, 0.3^2));
    forward (with checkpoints), backward (segment replays + reverse kernels)
    and the plain forward of the same scene, all device-timed on the scene's
    stream."""
    import torch
    from ysim_b200 import generators as G
    from ysim_b200.adjoint import ClothRollout
    from ysim_b200.scene import Scene
    spec = G.config_c5()
    c = spec.meshes[0]
    k, L = G.grid_spring_params(c.grid_n, c.grid_rest, (c.kstretch, c.kshear, c.kbend))
    roll = ClothRollout(spec, steps=steps, checkpoint_every=every, device=local)
    stream = torch.cuda.ExternalStream(roll.scene.stream(), device=local)
    dev = torch.device("cuda", local)
    kt = torch.tensor(k, device=dev, requires_grad=True)
    Lt = torch.tensor(L, device=dev, requires_grad=True)
    vt = torch.zeros((c.nV, 3), device=dev, requires_grad=True)
    rng = np.random.default_rng(5)
    kstar_np = (k * np.exp(rng.normal(0.0, 0.3, k.shape))).astype(np.float32)
    kstar = torch.tensor(kstar_np, device=dev)
    with torch.no_grad():
        target = roll(kstar, Lt, vt).clone()
    fw, bw = [], []
    for it in range(reps + 1):
        kt.grad = Lt.grad = vt.grad = None
        a, b, d = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        a.record(stream)
        xT = roll(kt, Lt, vt)
        b.record(stream)
        loss = ((xT - target) ** 2).sum(1).mean()
        loss.backward()
        d.record(stream)
        torch.cuda.synchronize()
        if it:
            fw.append(a.elapsed_time(b))
            bw.append(b.elapsed_time(d))
    g32 = [t.grad.double().cpu().numpy() for t in (kt, Lt, vt)]
    roll.close()
    s = Scene(spec, device=local)
    st = torch.cuda.ExternalStream(s.stream(), device=local)
    s.step(10)
    s.sync()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(st)
    s.step(steps)
    b.record(st)
    torch.cuda.synchronize()
    plain = a.elapsed_time(b) / steps
    s.close()
    f = float(np.median(fw)) / steps
    g = float(np.median(bw)) / steps
    f64 = measure_adjoint_fp64(spec, k, L, target, local, steps, every, reps)
    g64 = f64.pop("_grads")
    full = {n_: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            for n_, a, b in zip(("k", "L", "v0"), g32, g64)}
    prefix = fp32_vs_fp64_prefix(spec, k, L, kstar_np, local, every)
    return {"workload": "FastGridCloth 128x128 over a level-4 icosphere, 200 steps, checkpoint every 20",
            "forward_ms_per_step": f, "backward_ms_per_step": g, "backward_over_forward": g / f,
            "plain_forward_ms_per_step": plain, "unit": "ms/step",
            "gradients": "w.r.t. per-spring k, L and v0; checked against FP64 finite differences and an FP64 "
                         "reference adjoint in the GPU tests",
            "fp32_vs_fp64": {"full_200_steps": full, "branch_stable_prefix": prefix,
                             "measure": "norm-relative difference per parameter group between the FP32 adjoint "
                                        "and the 64-bit mode on the same loss; over the full rollout the two "
                                        "forwards take different branches at contact pushes (a pushed vertex is "
                                        "re-tested exactly at the thickness), so only the prefix before the first "
                                        "push compares derivatives of one function"},
            "fp64": f64}


def fp32_vs_fp64_prefix(spec, k, L, kstar, local, every):
    """FP32 adjoint against the 64-bit mode on the C5 problem's steps before
    its first contact push (found from the recorded contacts of the FP32
    forward: a contact with d below the thickness), seeded with the gradient
    of the MSE loss against the perturbed-stiffness rollout at the same step,
    taken at the binary64 state."""
    import torch
    from ysim_b200.adjoint import ClothRollout
    from ysim_b200.scene import Scene
    c = spec.meshes[0]
    s = Scene(spec, device=local)
    s.set_record(True)
    T = None
    for t in range(1, 201):
        s.step(1)
        off, cc = s.contacts()
        if (cc["d"][: int(off[c.nV])] < c.thickness).any():
            T = t - 1
            break
    s.close()
    if not T:
        return None
    dev = torch.device("cuda", local)
    roll = ClothRollout(spec, steps=T, checkpoint_every=every, device=local)
    with torch.no_grad():
        target = roll(torch.tensor(kstar, device=dev), torch.tensor(L, device=dev),
                      torch.zeros((c.nV, 3), device=dev)).double()
    roll.close()
    # both reverse passes take the loss gradient of the binary64 rollout (a
    # seed formed from the FP32 state would be mostly its rounding: x_T - x*
    # is a few binary32 ulps of x_T in the first steps)
    out, seed = {}, None
    for prec, dt in ((64, torch.float64), (32, torch.float32)):
        roll = ClothRollout(spec, steps=T, checkpoint_every=every, device=local, precision=prec)
        p = [torch.tensor(np.asarray(a), dtype=dt, device=dev, requires_grad=True)
             for a in (k, L, np.zeros((c.nV, 3), np.float32))]
        xT = roll(*p)
        if seed is None:
            seed = (2.0 * (xT.detach() - target) / c.nV).double()
        xT.backward(seed.to(dt))
        out[prec] = [t.grad.double().cpu().numpy() for t in p]
        roll.close()
    rel = {n_: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
           for n_, a, b in zip(("k", "L", "v0"), out[32], out[64])}
    return {"steps": T, **rel}


def measure_adjoint_fp64(spec, k, L, target, local, steps, every, reps, window=40):
    """The adjoint's 64-bit mode on the same workload: forward and backward
    ms/step (same loss), and the gradient against FP64 central differences of
    the same rollout on the workload's first `window` steps, a branch-stable
    window (contacts detected, none pushing: the contact response makes the
    rollout piecewise once vertices are pushed to the thickness and re-tested
    there, and differences across those branches measure no derivative).
    The check problem takes a random initial velocity and the linear loss
    sum(w x_T); per parameter group the three largest components, and 64
    random ones over the three groups, each step balancing truncation against round-off (k: 1e-3
    relative, L: 1e-6, v0: 1e-5); relative error = |g - fd| / max(|fd|, 1% of
    the group's largest gradient)."""
    import torch
    from ysim_b200.adjoint import ClothRollout
    c = spec.meshes[0]
    dev = torch.device("cuda", local)
    roll = ClothRollout(spec, steps=steps, checkpoint_every=every, device=local, precision=64)
    stream = torch.cuda.ExternalStream(roll.scene.stream(), device=local)
    kt = torch.tensor(k, dtype=torch.float64, device=dev, requires_grad=True)
    Lt = torch.tensor(L, dtype=torch.float64, device=dev, requires_grad=True)
    vt = torch.zeros((c.nV, 3), dtype=torch.float64, device=dev, requires_grad=True)
    tgt = target.double()
    fw, bw = [], []
    for it in range(reps + 1):
        kt.grad = Lt.grad = vt.grad = None
        a, b, d = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        a.record(stream)
        xT = roll(kt, Lt, vt)
        b.record(stream)
        ((xT - tgt) ** 2).sum(1).mean().backward()
        d.record(stream)
        torch.cuda.synchronize()
        if it:
            fw.append(a.elapsed_time(b) / steps)
            bw.append(b.elapsed_time(d) / steps)
    g64 = [t.grad.double().cpu().numpy() for t in (kt, Lt, vt)]
    roll.close()
    # finite-difference check on the branch-stable window
    rng = np.random.default_rng(11)
    v0 = torch.tensor(rng.normal(0, 0.02, (c.nV, 3)), device=dev)
    w = torch.tensor(rng.normal(0, 1, (c.nV, 3)) / c.nV, device=dev)
    roll = ClothRollout(spec, steps=window, checkpoint_every=every, device=local, precision=64)
    params = [t.detach().clone().requires_grad_(True) for t in (kt, Lt, v0)]
    (roll(*params) * w).sum().backward()
    grads = [p.grad.cpu().numpy().reshape(-1) for p in params]
    base = [p.detach().clone().reshape(-1) for p in params]

    def loss(group, i, delta):
        p = [b_.clone() for b_ in base]
        p[group][i] += delta
        with torch.no_grad():
            return float((roll(p[0], p[1], p[2].reshape(-1, 3)) * w).sum())

    worst, n = 0.0, 0
    for group, g in enumerate(grads):
        for i in list(np.argsort(-np.abs(g))[:3]) + list(rng.integers(len(g), size=22 if group < 2 else 20)):
            i = int(i)
            eps = 1e-3 * abs(float(base[0][i])) if group == 0 else (1e-6 if group == 1 else 1e-5)
            fd = (loss(group, i, eps) - loss(group, i, -eps)) / (2 * eps)
            worst = max(worst, abs(g[i] - fd) / max(abs(fd), 1e-2 * float(np.abs(g).max())))
            n += 1
    roll.close()
    f, b = float(np.median(fw)), float(np.median(bw))
    return {"forward_ms_per_step": f, "backward_ms_per_step": b, "backward_over_forward": b / f,
            "fd_check": {"window_steps": window, "components": n, "worst_rel_err": worst,
                         "loss": "sum(w x_T), random v0"},
            "arithmetic": "binary64 throughout; bit-identical to the FP64 reference rollout in the GPU tests",
            "_grads": g64}


def run_batched(args, rank, world, local):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    b = measure_batched(args, rank, world, local)
    if rank == 0:
        line = {"metric": "batched vs plain substeps/s (C4)", "value": b["value"], "unit": b["unit"],
                "n_gpus": world, "higher_is_better": True, "scaling": "strong", "dtype": "f32",
                "data": "synthetic (seeded)", "batched": b}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ collide
def run_collide(args, emit=None):
    """Collision microbenchmark: N triangles (centroids U[0,1]^3, vertex
    offsets N(0, sigma^2), sigma log-normal around 1e-3) and N query points;
    LBVH build + refit + point query within h = 1e-3 against the spatial-hash
    broad phase (cell 2h).  Device-timed with CUDA events; the two candidate
    sets are checked for equality on the device.  One record per N (and one
    for the face-face hash on the C2 geometry) to emit (printed as a JSON
    line each by default)."""
    if emit is None:
        emit = lambda rec: print(json.dumps(rec), flush=True)  # noqa: E731
    import ctypes as C
    import torch
    from ysim_b200 import _lib, generators as G
    lib = _lib.load()
    torch.cuda.set_device(0)
    h = np.float32(1e-3)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def P(t):
        return C.c_void_p(t.data_ptr())

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    for n in [int(v) for v in args.sizes.split(",")]:
        x, f, q = G.soup(n, seed=3)
        dx, df, dq = dev(x.reshape(-1)), dev(f.reshape(-1).astype(np.int32)), dev(q.reshape(-1))
        v = dev(np.random.default_rng(4).normal(0, 0.1, x.shape).astype(np.float32).reshape(-1))
        cap = 8 * n
        pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")

        def keys(m):
            k = (pairs[0:2 * min(m, cap):2].long() << 32) | pairs[1:2 * min(m, cap):2].long()
            return torch.sort(k).values

        t = C.c_void_p()
        _lib.check(lib.ys_lbvh_create(C.byref(t), n, 0, None), "lbvh_create")
        reps = max(3, min(args.steps, 10))
        # the reference's tree (midpoint split of equal-code runs), timed
        build_ms = timed(lambda: _lib.check(lib.ys_lbvh_build(t, P(dx), len(x), P(df), n)), reps)
        refit_ms = timed(lambda: _lib.check(lib.ys_lbvh_refit(t, P(dx), P(v), np.float32(1e-3), 1)), reps)
        _lib.check(lib.ys_lbvh_build(t, P(dx), len(x), P(df), n))
        query_ms = timed(lambda: _lib.check(lib.ys_lbvh_query(t, P(dq), len(q), h, 0, P(pairs), cap, P(cnt))), reps)
        nb = int(cnt.item())
        key_ref = keys(nb)
        # the same tree with the (code, index) split: one parent per node,
        # every internal box the union of a sorted-leaf range (range refit)
        _lib.check(lib.ys_lbvh_set_split(t, 1))
        cbuild_ms = timed(lambda: _lib.check(lib.ys_lbvh_build(t, P(dx), len(x), P(df), n)), reps)
        crefit_ms = timed(lambda: _lib.check(lib.ys_lbvh_refit(t, P(dx), P(v), np.float32(1e-3), 1)), reps)
        _lib.check(lib.ys_lbvh_build(t, P(dx), len(x), P(df), n))
        cquery_ms = timed(lambda: _lib.check(lib.ys_lbvh_query(t, P(dq), len(q), h, 0, P(pairs), cap, P(cnt))),
                          reps)
        nc = int(cnt.item())
        key_b = keys(nc)
        _lib.check(lib.ys_lbvh_destroy(t), "lbvh_destroy")
        sh = C.c_void_p()
        _lib.check(lib.ys_shash_create(C.byref(sh), n, 40 * n, 0, None), "shash_create")
        sh_build_ms = timed(lambda: _lib.check(lib.ys_shash_build(sh, P(dx), P(df), n, np.float32(2 * h))), reps)
        sh_query_ms = timed(lambda: _lib.check(lib.ys_shash_query(sh, P(dq), len(q), h, P(pairs), cap, P(cnt))), reps)
        ns = int(cnt.item())
        ent, big = C.c_uint32(), C.c_uint32()
        _lib.check(lib.ys_shash_entries(sh, C.byref(ent), C.byref(big)))
        key_s = keys(ns)
        same = bool(nc == ns and nc <= cap and torch.equal(key_b, key_s))
        ref_unique = torch.unique_consecutive(key_ref)
        ref_missing = int((~torch.isin(key_s, ref_unique)).sum().item())
        _lib.check(lib.ys_shash_destroy(sh))
        line = {"workload": "collision microbenchmark", "triangles": n, "queries": n, "h": float(h),
                "lbvh_build_ms": build_ms, "lbvh_refit_swept_ms": refit_ms, "lbvh_query_ms": query_ms,
                "shash_build_ms": sh_build_ms, "shash_query_ms": sh_query_ms, "candidates": ns,
                "shash_entries": ent.value, "shash_oversized": big.value, "candidate_sets_equal": same,
                "equality": "spatial hash vs LBVH with the (code, index) split, as sets and counts",
                "consistent_split": {"lbvh_build_ms": cbuild_ms, "lbvh_refit_swept_ms": crefit_ms,
                                     "lbvh_query_ms": cquery_ms,
                                     "refit": "sorted-leaf ranges: a leaf pass with block boxes, then the nodes "
                                              "whose range crosses a 256-leaf block (no climb)"},
                "reference_split": {"candidates": nb, "duplicates": nb - int(ref_unique.numel()),
                                    "missing": ref_missing,
                                    "note": "the reference's midpoint split of runs of >= 3 equal Morton codes "
                                            "leaves some leaves unreached and others reached twice"},
                "timing": f"CUDA events, median of {reps}; calls include their host-side synchronisation; "
                          "LBVH times are for the reference split"}
        emit(line)
        del dx, df, dq, v, pairs
    torch.cuda.empty_cache()
    run_face_face(args, lib, timed, dev, P, emit)


def run_face_face(args, lib, timed, dev, P, emit):
    """The face-face spatial hash (the reference's SpatialHashing<METAL>
    broad phase) on the C2 geometry: the 512x512 cloth and the level-7
    icosphere as one packed scene, self rows on."""
    import ctypes as C
    import torch
    from ysim_b200 import _lib
    spec = spec_for(args)
    # the packed scene arrays (Scene::pack): positions, per-mesh vertex and
    # face offsets, facets with mesh-local ids, behaviours, shapes (meshes)
    ms = spec.meshes
    x = np.concatenate([np.asarray(m.x, np.float32) for m in ms])
    so = np.concatenate([[0], np.cumsum([m.nV for m in ms])]).astype(np.uint32)
    fo = np.concatenate([[0], np.cumsum([m.nF for m in ms])]).astype(np.uint32)
    F = np.concatenate([np.asarray(m.facets, np.uint32) for m in ms])
    beh = np.array([m.behavior for m in ms], np.uint32)
    shape = np.zeros(len(ms), np.uint32)
    nF = len(F)
    cap = 64 * nF
    dx, dso, dF, dfo = dev(x.reshape(-1)), dev(so.view(np.int32)), dev(F.reshape(-1).view(np.int32)), dev(fo.view(np.int32))
    db, ds = dev(beh.view(np.int32)), dev(shape.view(np.int32))
    rows = torch.empty(cap * 8, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    h = C.c_void_p()
    _lib.check(lib.ys_shff_create(C.byref(h), nF, 0, None))
    margin = np.float32(spec.params.margin)
    ms = timed(lambda: _lib.check(lib.ys_shff_detect(h, P(dx), len(x), P(dso), P(dF), P(dfo), nF, P(db), P(ds),
                                                      len(beh), margin, 1, P(rows), cap, P(cnt))), 10)
    st = (C.c_uint32 * 6)()
    _lib.check(lib.ys_shff_stats(h, st))
    _lib.check(lib.ys_shff_destroy(h))
    line = {"workload": "face-face spatial hash (SpatialHashing broad phase), C2 geometry", "faces": nF,
            "vertices": len(x), "margin": float(margin), "detect_ms": ms, "rows": int(cnt.item()),
            "entries": st[0], "cells": st[1], "candidate_pairs": st[2], "grid": [st[3], st[4], st[5]],
            "timing": "CUDA events around the whole detect (no host synchronisation inside), median of 10"}
    emit(line)


def run_c2_kernels(args):
    """The headline workload's kernels as separate launches, for a profiler's
    launch list or a capture of one kernel: --preroll substeps (CUDA graphs),
    then --steps substeps launched directly with CUDA events around the refit
    and fused stages, then one standalone build of the cloth's tree with the
    Karras and with the Apetrei builder.  Prints one JSON line."""
    import ctypes as C
    import torch
    from ysim_b200 import _lib
    from ysim_b200.scene import Scene
    torch.cuda.set_device(0)
    spec = spec_for(args)
    scene = Scene(spec, device=0)
    scene.step(args.preroll)
    scene.autotune_classes()
    if args.fused_variant:
        scene.set_fused_variant(args.fused_variant)
    scene.set_graphs(False)
    _lib.check(scene.lib.ys_scene_set_timing(scene.h, 1), "set_timing")
    t0 = scene.totals()
    scene.step(args.steps)
    scene.sync()
    kt = (C.c_double * 4)()
    _lib.check(scene.lib.ys_scene_kernel_times(scene.h, kt), "kernel_times")
    t1 = scene.totals()
    m0 = spec.meshes[0]
    x = scene.get("x")[: m0.nV]
    scene.close()  # the builds run with the scene's memory released
    build = measure_build(x, m0.facets, 0, reps=1, warm=0)
    print(json.dumps({"workload": "C2 kernels, one by one", "preroll": args.preroll, "steps": args.steps,
                      "refit_ms": kt[0] / max(kt[1], 1), "fused_ms": kt[2] / max(kt[3], 1),
                      "rows_per_substep": (t1[0] - t0[0]) / max(args.steps, 1),
                      "contacts_per_substep": (t1[1] - t0[1]) / max(args.steps, 1), "tree_build": build}), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.workload == "c2-kernels":
        if rank == 0:
            run_c2_kernels(args)
        return
    if args.workload == "collide":
        if rank == 0:
            run_collide(args)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    if args.workload == "adjoint":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            a = measure_adjoint(args, local)
            print(json.dumps({"metric": "adjoint ms/step (C5)", "value": a["backward_ms_per_step"],
                              "unit": "ms/step", "higher_is_better": False, "dtype": "f32", "adjoint": a}),
                  flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
