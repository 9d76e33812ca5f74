"""Host build of the reference's own Metal compute kernels: oracle/_ref/libysref.so.

TEST INFRASTRUCTURE ONLY.  Compiles oracle/ref_harness.cpp once per shader,
each time including one shader of the reference checkout in place
(src/metal/bvh.metal, bruteforce.metal, physics.metal, spatialhashing.metal)
with oracle/ref_shim
standing in for <metal_stdlib>, plus oracle/ref_sceneio.cpp over the
reference's scene-file, run-config and primitive-geometry headers
(include/scene_format.hpp, sim_config.hpp, primitive_geometry.hpp); nothing of
the reference is copied into this repository.  Skipped (returns None) when the reference checkout is absent;
the built library is git-ignored but travels with the working tree.

The reference checkout is the directory given by --reference, else by the
YSIM_REFERENCE environment variable, else a checkout named `reference` beside
this repository's directory.

    python -m oracle.build_ref [--reference DIR] [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("YSIM_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libysref.so")
SHADERS = {"BVH": "bvh.metal", "NARROW": "bruteforce.metal", "PHYSICS": "physics.metal",
           "SH": "spatialhashing.metal"}


def available() -> bool:
    return all(os.path.exists(os.path.join(REF, "src", "metal", f)) for f in SHADERS.values()) and \
        os.path.exists(os.path.join(REF, "include", "scene_format.hpp"))


def build(force: bool = False):
    if not available():
        return OUT if os.path.exists(OUT) else None
    deps = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "ref_shim", "metal_shim.h"),
            os.path.join(HERE, "ref_sceneio.cpp")]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for key, shader in SHADERS.items():
        obj = os.path.join(OUT_DIR, f"{key.lower()}.o")
        cmd = ["g++", "-std=c++17", "-O3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-w",
               "-I", os.path.join(HERE, "ref_shim"), f"-DYS_REF_{key}",
               f"-DYS_REF_SRC={os.path.join(REF, 'src', 'metal', shader)}", "-c",
               os.path.join(HERE, "ref_harness.cpp"), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference build failed for {shader}:\n{r.stdout}{r.stderr}")
        objs.append(obj)
    # the scene-file, run-config and primitive-geometry headers (plain C++ with
    # the bundled nlohmann/json)
    obj = os.path.join(OUT_DIR, "sceneio.o")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-w",
           "-I", os.path.join(REF, "include"), "-c", os.path.join(HERE, "ref_sceneio.cpp"), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed for the scene-file headers:\n" + r.stdout + r.stderr)
    objs.append(obj)
    r = subprocess.run(["g++", "-shared", "-fopenmp", "-o", OUT + ".tmp", *objs], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference link failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    for o in objs:
        os.remove(o)
    return OUT


if __name__ == "__main__":
    if "--reference" in sys.argv:
        REF = os.path.abspath(sys.argv[sys.argv.index("--reference") + 1])
    print(build(force="--force" in sys.argv))
