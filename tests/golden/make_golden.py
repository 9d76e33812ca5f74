"""Generate the golden vectors in tests/golden/ from the reference's own kernels.

    python tests/golden/make_golden.py

Needs the reference checkout (oracle/_ref is built from it by
oracle/build_ref.py); the fixtures it writes are committed so that the tests
can check the CUDA path and the oracle against reference outputs on machines
without the reference.  Inputs are seeded synthetic data of this repository's
generators; outputs are the reference kernels' results:
  morton_tree.npz -- fillMortons_Tri codes, stable sort, buildTree_Tri topology,
                     bottomUpBoxes boxes, buildSweptLeaf_Tri refit, queryPoints
                     pairs (inclusive AABB test, h = 1e-3 and a self query),
                     and the agglomerativeBuild_Tri + agglomerativeSwapRoot
                     tree (agg_*);
  substep_*.npz   -- one mid-drape substep of a small scene: broad rows (the
                     oracle's), narrow_pt_tri contacts, the cloth's spring
                     forces and integrate_cloth(_grid) positions / velocities;
  scene_io.json   -- the scene-file / run-config round trips and load errors
                     (scene_format.hpp, sim_config.hpp) of tests/golden/scenes
                     and tests/scene_cases.py, libstdc++'s mt19937 +
                     uniform_real_distribution<float> draws, and a
                     FrameProfiler CSV export;
  scene_io_geom.npz -- primitive::sphere / cube / cylinder meshes;
  analytic.npz    -- narrow_pt_analytic contacts of vertex clouds around every
                     collider kind (static, rotated, moving, ellipsoid,
                     disabled; tests/analytic_cases.py), with the rotation
                     margins passed to the kernel.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import refkernels as R  # noqa: E402
from ysim_b200 import generators as G  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
import analytic_cases as AC  # noqa: E402
import scene_cases as SCN  # noqa: E402


def canon(p):
    p = np.asarray(p, np.uint32).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p


def morton_tree():
    out = {}
    for name, (x, f, q) in {"soup": G.soup(2000, seed=41),
                            "grid": G.grid_cloth(24, 1.0, (0.0, 0.2, 0.0)) + (None,)}.items():
        if q is None:
            rng = np.random.default_rng(42)
            x = (x + rng.uniform(-1e-3, 1e-3, x.shape)).astype(np.float32)
            q = x.copy()
        box = np.zeros(6, np.float32)
        O.lib().yso_scene_box(O.P(x), len(x), O.P(box))
        codes, idx = R.fill_mortons(x, f, box)
        o = np.argsort(codes, kind="stable")
        codes, idx = codes[o], idx[o]
        nodes, parent = R.build_tree(x, f, codes, idx)
        v = np.random.default_rng(43).normal(0, 0.5, x.shape).astype(np.float32)
        swept = R.refit(nodes, parent, x, v, f, codes, idx, np.float32(1.0 / 1200.0), True)
        self_q = name == "grid"
        margin = np.float32(0.03 if self_q else 0.02)
        rows, n, _ = R.query_points(q, f, swept, margin, 0, 0 if self_q else 1)
        an, ap, _ = R.agglomerative(x, f, codes, idx)
        out.update({f"{name}_agg_a": an["a"], f"{name}_agg_b": an["b"], f"{name}_agg_mn": an["mn"],
                    f"{name}_agg_mx": an["mx"], f"{name}_agg_parent": ap})
        out.update({f"{name}_x": x, f"{name}_f": f, f"{name}_q": q, f"{name}_v": v, f"{name}_box": box,
                    f"{name}_codes": codes, f"{name}_idx": idx, f"{name}_a": nodes["a"], f"{name}_b": nodes["b"],
                    f"{name}_mn": nodes["mn"], f"{name}_mx": nodes["mx"], f"{name}_parent": parent,
                    f"{name}_swept_mn": swept["mn"], f"{name}_swept_mx": swept["mx"], f"{name}_margin": margin,
                    f"{name}_self": np.int32(self_q),
                    f"{name}_pairs": canon(np.stack([rows["point"], rows["tri"]], 1))})
    np.savez_compressed(os.path.join(HERE, "morton_tree.npz"), **out)


SPECS = {
    "c1": lambda: G.config_c1(P=24, level=2, height=0.2999),
    "c2hash": lambda: G.config_c2(P=32, level=3, height=0.315, gravity=-9.81),
}


def substep(name):
    spec = SPECS[name]()
    o = O.OracleScene(spec)
    o.step(3 * spec.params.substeps + 1)
    o.stage(0); o.stage(1); o.stage(2)
    x, xp, v = o.get("x"), o.get("xprev"), o.get("v")
    rows = o.rows()
    p = spec.params
    voff, foff, F, vaf, vaf_off = [0], [0], [], [], [0]
    for m in spec.meshes:
        a = O.adjacency(m.x, m.facets)
        vaf_off += list(vaf_off[-1] + a["vaf_off"][1:])
        vaf.append(a["vaf"])
        F.append(m.facets.reshape(-1))
        voff.append(voff[-1] + m.nV)
        foff.append(foff[-1] + m.nF)
    voff = np.array(voff, np.uint32)
    rc = R.narrow(rows, x, voff, np.concatenate(F).astype(np.uint32), np.array(foff, np.uint32),
                  np.concatenate(vaf).astype(np.uint32), np.array(vaf_off, np.uint32), np.float32(p.radius),
                  np.float32(p.margin), xp)
    rc = rc[np.lexsort((rc["tri"], rc["tobj"], rc["point"], rc["qobj"]))]
    # canonical per-vertex CSR of the reference contacts
    nV = spec.nV
    g = voff[rc["qobj"]] + rc["point"]
    off = np.zeros(nV + 1, np.uint32)
    np.add.at(off, g + 1, 1)
    off = np.cumsum(off).astype(np.uint32)
    m = spec.meshes[0]
    n0 = m.nV
    mass3 = np.repeat(m.mass, 3).astype(np.float32)
    ext = (np.asarray(p.gravity, np.float32)[None, :] * m.mass[:, None]).astype(np.float32)
    if m.behavior == 0:
        adj = O.adjacency(m.x, m.facets)
        prm = np.array([m.kstretch, m.kshear, m.kbend, m.thickness], np.float32)
        f = R.tri_forces(x[:n0], v[:n0], ext, mass3, m.mask, np.float32(p.subh), np.float32(p.kair),
                         np.float32(p.kd), prm, adj, m.facets.reshape(-1))
        kind = "tri"
    else:
        prm = R.grid_params(m.grid_n, m.grid_rest, (m.kstretch, m.kshear, m.kbend), m.thickness)
        f = R.grid_forces(x[:n0], v[:n0], ext, mass3, np.float32(p.subh), np.float32(p.kair), np.float32(p.kd), prm)
        kind = "grid"
    xn, vn, anomaly = R.integrate(kind, x[:n0], v[:n0], f, mass3, m.mask, rc, off, voff, 0, np.float32(p.subh), prm)
    rws = np.stack([rows["qobj"], rows["point"], rows["tobj"], rows["tri"]], 1).astype(np.uint32)
    rws = rws[np.lexsort((rws[:, 3], rws[:, 2], rws[:, 1], rws[:, 0]))]
    np.savez_compressed(os.path.join(HERE, f"substep_{name}.npz"), x=x, xprev=xp, v=v, rows=rws,
                        c_point=rc["point"], c_tri=rc["tri"], c_qobj=rc["qobj"], c_tobj=rc["tobj"], c_n=rc["n"],
                        c_d=rc["d"], csr_off=off, f=f, x_next=xn, v_next=vn, anomaly=np.int32(anomaly))


def analytic():
    shapes, x, xp, so, beh, pairs = AC.cases(seed=11, per_shape=600)
    rms, out = [], []
    for k, (cloth, obj) in enumerate(pairs):
        rm = O.rot_margin(shapes[k], AC.RADIUS, AC.THICKNESS)
        rms.append(rm)
        if not shapes[k]["flags"] & 1:
            continue  # narrowAnalytic skips a collider that is not collidable
        out.append(R.narrow_analytic(x, xp, so, shapes, int(cloth), k, int(beh[cloth]), AC.RADIUS, AC.THICKNESS,
                                     np.float32(rm)))
    c = AC.canon_contacts(np.concatenate(out))
    np.savez_compressed(os.path.join(HERE, "analytic.npz"), shapes=shapes.view(np.uint8), x=x, xprev=xp,
                        state_off=so, beh=beh, pairs=pairs, radius=AC.RADIUS, thickness=AC.THICKNESS,
                        rot_margin=np.array(rms, np.float32), contacts=c.view(np.uint8))


def profiler_frames():
    """A fixed set of frames for the FrameProfiler CSV check."""
    rng = np.random.default_rng(9)
    n = 250
    fms = rng.uniform(0.0, 40.0, n)
    fms[3], fms[7], fms[9] = 0.0, 1e-7, 123456789.0
    sec = rng.uniform(0, 5, (n, 4))
    sec[0, 0], sec[1, 1] = 1e300, -2.5e-20
    return dict(seq=(np.arange(n) + 5).tolist(), wall=np.cumsum(rng.uniform(0.001, 0.05, n)).tolist(),
                frame_ms=fms.tolist(), broad=rng.integers(0, 10**9, n).tolist(),
                narrow=rng.integers(0, 10**6, n).tolist(), names=["physics total", "refit", "substep-kernel", "x.y"],
                sec_ms=sec.tolist(), max_frames=240)


def scene_io():
    import json
    import tempfile
    out = {"roundtrip": {}, "runconfig": {}, "errors": [], "jiggle": {}}
    for name in SCN.fixture_names():
        t = SCN.fixture_text(name)
        out["roundtrip"][name] = R.scene_roundtrip(t)[1]
        out["runconfig"][name] = R.scene_roundtrip(t, runconfig=True)[1]
    for name, t in SCN.error_cases():
        ok1, m1, _ = R.scene_roundtrip(t)
        ok2, m2, _ = R.scene_roundtrip(t, runconfig=True)
        out["errors"].append({"name": name, "scene": [ok1, m1], "runconfig": [ok2, m2]})
    for seed in SCN.JIGGLE_SEEDS:
        out["jiggle"][str(seed)] = R.uniform_float(seed, 0.0, 1.0 / 10000.0, 700).view(np.uint32).tolist()
    pf = profiler_frames()
    with tempfile.TemporaryDirectory() as d:
        out["profiler_csv"] = R.profiler_csv(os.path.join(d, "p.csv"), pf["seq"], pf["wall"], pf["frame_ms"],
                                             pf["broad"], pf["narrow"], pf["names"], pf["sec_ms"], pf["max_frames"])
    out["profiler_frames"] = pf
    out["paths"] = [list(R.profile_paths(r, sp, f)) + [r, sp, f]
                    for r, sp, f in (("", "/a/b/flag.ysim.json", 30), ("/x/y", "scene", 5), ("", "noext", 1))]
    with open(os.path.join(HERE, "scene_io.json"), "w") as f:
        json.dump(out, f)
    geom = {}
    for k, s, t in SCN.PRIMITIVE_CASES:
        p, fc = R.primitive(k, s, t)
        geom[f"{k}_{s}_{t}_x"] = p
        geom[f"{k}_{s}_{t}_f"] = fc
    np.savez_compressed(os.path.join(HERE, "scene_io_geom.npz"), **geom)


if __name__ == "__main__":
    if not R.available():
        sys.exit("reference checkout absent: cannot regenerate golden vectors")
    morton_tree()
    for k in SPECS:
        substep(k)
    analytic()
    scene_io()
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith(".npz"):
            print(fn, os.path.getsize(os.path.join(HERE, fn)))
