"""Headless run of a scene file or run config on the CUDA path, with a profile.

    python -m ysim_b200.run SCENE.json [--frames N] [--csv PATH] [--level none|per_frame|in_frame]
                                       [--staged] [--device D]

The `--scene` automation of the reference (include/sim_config.hpp): the run
config's "profile" block gives the frame count, the CSV path (default
profiles/<scene stem>-<N>f.csv, defaultProfilePath) and the detail level;
command-line flags override it.  Each frame is one Simulator::update (the
frame preamble and `substeps` substeps); the CSV has the FrameProfiler schema
with the frame's wall time (host clock around the frame, synchronised) and,
per level, the sections "physics_total" (CUDA events around the frame's
substeps) and, for in_frame, "broad_refit" and "substep_kernel" (the kernels'
CUDA-event times).  The run config is written beside the CSV
(sidecarScenePath).  Prints one JSON line with the run's summary.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

from . import _lib
from . import loader as LD
from . import profiler as PF
from . import scene_format as SF


def run(path: str, frames=None, csv_path=None, level=None, staged=False, device=0, quiet=False) -> dict:
    import torch
    ls = LD.load(path)
    cfg = ls.config
    nframes = int(frames if frames is not None else cfg.profile.frames)
    lvl = level or cfg.profile.level
    if lvl not in SF.PROFILE_LEVELS:
        raise SF.SceneFormatError(f"unknown profile level '{lvl}'")
    out = csv_path or cfg.profile.output_path or SF.default_profile_path("", SF.path_stem(path), nframes)
    from .scene import Scene
    torch.cuda.set_device(device)
    scene = Scene(ls.spec, device=device)
    try:
        if ls.ext is not None:
            ext = np.ascontiguousarray(ls.ext, np.float32)
            _lib.check(scene.lib.ys_scene_set_external_forces(scene.h, ext.ctypes.data_as(C.c_void_p)), "ext")
        stream = torch.cuda.ExternalStream(scene.stream(), device=device)
        prof = PF.FrameProfiler(max(nframes, 1))
        if lvl == "in_frame":
            _lib.check(scene.lib.ys_scene_set_timing(scene.h, 1), "timing")
        kt_prev = (C.c_double * 4)()
        nsub = ls.spec.params.substeps
        t0 = time.perf_counter()
        totals_prev = scene.totals()
        for f in range(nframes):
            scene.sync()
            w0 = time.perf_counter()
            if lvl != "none":
                prof.begin_frame(f, w0 - t0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            broad = narrow = 0
            if staged:
                for _ in range(nsub):
                    scene.step_staged(1)
                    st = scene.stats()
                    broad += st["broad_rows"]
                    narrow += st["contacts"]
            else:
                scene.step(nsub)
            e1.record(stream)
            scene.sync()
            torch.cuda.synchronize()
            w1 = time.perf_counter()
            if not staged:
                tot = scene.totals()
                broad, narrow = tot[0] - totals_prev[0], tot[1] - totals_prev[1]
                totals_prev = tot
            if lvl != "none":
                prof.add_collision_counts(broad, narrow)
                prof.add_sample("physics_total", e0.elapsed_time(e1))
                if lvl == "in_frame":
                    kt = (C.c_double * 4)()
                    _lib.check(scene.lib.ys_scene_kernel_times(scene.h, kt), "kernel_times")
                    prof.add_sample("broad_refit", kt[0] - kt_prev[0])
                    prof.add_sample("substep_kernel", kt[2] - kt_prev[2])
                    kt_prev = kt
                prof.end_frame((w1 - w0) * 1000.0)
        st = scene.stats()
        x = scene.get("x")
    finally:
        scene.close()
    summary = {"scene": path, "frames": nframes, "substeps_per_frame": int(ls.spec.params.substeps),
               "vertices": int(ls.spec.nV), "meshes": len(ls.spec.meshes), "level": lvl,
               "path": "staged" if staged else "fused", "flags": st["flags"],
               "finite": bool(np.isfinite(x).all()), "warnings": ls.warnings}
    if lvl != "none":
        if not prof.export_csv(out):
            raise OSError(f"cannot write '{out}'")
        with open(SF.sidecar_scene_path(out), "w") as fh:
            fh.write(SF.run_config_to_string(cfg))
        fm = [fr.frame_ms for fr in prof.frames]
        summary.update({"csv": out, "mean_frame_ms": float(np.mean(fm)) if fm else 0.0,
                        "substeps_per_s": (nframes * nsub) / (sum(fm) / 1000.0) if fm and sum(fm) > 0 else None})
    if not quiet:
        print(json.dumps(summary), flush=True)
    return summary


def main(argv=None):
    ap = argparse.ArgumentParser(description="Headless run of a ysim scene file on the CUDA path")
    ap.add_argument("scene")
    ap.add_argument("--frames", type=int)
    ap.add_argument("--csv")
    ap.add_argument("--level", choices=SF.PROFILE_LEVELS)
    ap.add_argument("--staged", action="store_true", help="one kernel group per reference stage")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    try:
        run(a.scene, a.frames, a.csv, a.level, a.staged, a.device)
    except SF.SceneFormatError as e:
        print(f"scene load failed: {e}", file=sys.stderr)
        return 2
    return 0


if __name__ == "__main__":
    sys.exit(main())
