"""One substep of the reference implementation on the host cores.

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY (bench.py --impl reference).  The stages
are the reference's own kernels compiled for the host (oracle/_ref, OpenMP
over thread ids, the way dispatchThreads spreads them over the GPU):
buildSweptLeaf_Tri + bottomUpBoxes (refit), queryPoints (inter-object rows),
narrow_pt_tri, narrow_bucket_*, compute_tri_spring_forces /
compute_cloth_grid_forces_fast and integrate_cloth(_grid), called in the order
of Simulator::update (simulator.hpp:3512-3815).  Two pieces have no
host-runnable reference form and come from the pinned oracle: the CPU-hash
self rows (CpuSpatialHash lives in an uncompilable header fragment) and the
per-frame LBVH rebuild's sort (the Metal radix sort needs threadgroup
barriers; its result is the stable sort numpy computes).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O
from . import refkernels as R
from .oracle import ROW_DTYPE


class RefScene:
    def __init__(self, spec):
        self.spec = spec
        p = spec.params
        self.p = p
        self.meshes = spec.meshes
        self.voff = np.cumsum([0] + [m.nV for m in spec.meshes]).astype(np.uint32)
        self.foff = np.cumsum([0] + [m.nF for m in spec.meshes]).astype(np.uint32)
        self.F = np.concatenate([m.facets.reshape(-1) for m in spec.meshes]).astype(np.uint32)
        self.x = np.concatenate([m.x for m in spec.meshes]).astype(np.float32)
        self.v = np.concatenate([m.v if m.v is not None else np.zeros_like(m.x) for m in spec.meshes]).astype(np.float32)
        self.xp = self.x.copy()
        vaf, vaf_off = [], [0]
        self.adj = []
        for m in spec.meshes:
            a = O.adjacency(m.x, m.facets)
            self.adj.append(a)
            vaf_off += list(vaf_off[-1] + a["vaf_off"][1:])
            vaf.append(a["vaf"])
        self.vaf = np.concatenate(vaf).astype(np.uint32)
        self.vaf_off = np.array(vaf_off, np.uint32)
        self.trees = [None] * len(spec.meshes)
        self.frame = 0
        self.cursor = 0
        self.cap = p.cols_per_point * int(self.voff[-1])

    def _mx(self, i):
        return self.x[self.voff[i]:self.voff[i + 1]]

    def build(self, i):
        m = self.meshes[i]
        x = self._mx(i)
        box = np.zeros(6, np.float32)
        O.lib().yso_scene_box(O.P(np.ascontiguousarray(x)), len(x), O.P(box))
        codes, idx = R.fill_mortons(x, m.facets, box)
        o = np.argsort(codes, kind="stable")
        codes, idx = codes[o], idx[o]
        nodes, parent = R.build_tree(x, m.facets, codes, idx)
        self.trees[i] = [nodes, parent, codes, idx]

    def substep(self):
        p = self.p
        cloth = lambda m: m.behavior in (0, 1)
        if self.cursor == 0:
            if p.rebuild_frames and self.frame % p.rebuild_frames == 0:
                for i, m in enumerate(self.meshes):
                    if self.trees[i] is not None and m.behavior == 4:
                        continue
                    self.build(i)
        # refit (non-static)
        for i, m in enumerate(self.meshes):
            if m.flags & 1:
                continue
            nodes, parent, codes, idx = self.trees[i]
            self.trees[i][0] = R.refit(nodes, parent, self._mx(i), self.v[self.voff[i]:self.voff[i + 1]], m.facets,
                                       codes, idx, np.float32(p.subh), True)
        # detect: hybrid CPU-hash self rows, then BVH rows
        rows = []
        for q, m in enumerate(self.meshes):
            if p.self_mode == 1 and cloth(m) and (m.flags & 2) and (m.flags & 4):
                pr = O.self_hash(self._mx(q), self.xp[self.voff[q]:self.voff[q + 1]], m.facets, np.float32(p.margin))
                r = np.zeros(len(pr), ROW_DTYPE)
                r["point"], r["tri"], r["qobj"], r["tobj"] = pr[:, 0], pr[:, 1], q, q
                rows.append(r)
        for q, mq in enumerate(self.meshes):
            if mq.behavior in (4, 7) or not (mq.flags & 2):
                continue
            for t, mt in enumerate(self.meshes):
                if q == t:
                    if p.self_mode != 2:
                        continue
                elif not (mt.flags & 2):
                    continue
                else:
                    a, b = self.trees[q][0][0], self.trees[t][0][0]
                    if (a["mx"] < b["mn"]).any() or (a["mn"] > b["mx"]).any():
                        continue
                r, n, _ = R.query_points(self._mx(q), mt.facets, self.trees[t][0], np.float32(p.margin), q, t,
                                         cap=max(64, 64 * mq.nV))
                rows.append(r)
        rows = np.concatenate(rows) if rows else np.zeros(0, ROW_DTYPE)
        rows = rows[: self.cap]
        self.nrows = len(rows)
        # narrow + per-vertex CSR (reference bucket kernels), canonical order
        c = R.narrow(rows, self.x, self.voff, self.F, self.foff, self.vaf, self.vaf_off, np.float32(p.radius),
                     np.float32(p.margin), self.xp)
        nV = int(self.voff[-1])
        offsets = np.zeros(nV + 1, np.uint32)
        counter = np.zeros(nV, np.uint32)
        csr = np.zeros_like(c)
        R.lib().yref_bucket(R.P(np.ascontiguousarray(c)), len(c), R.P(self.voff), nV + 1, R.P(offsets),
                            R.P(counter), R.P(csr))
        g = self.voff[csr["qobj"]] + csr["point"]
        csr = csr[np.lexsort((csr["tri"], csr["tobj"], g))]
        self.ncontacts = len(csr)
        # snapshot, forces, integrate
        self.xp_next = self.x.copy()
        for i, m in enumerate(self.meshes):
            if m.behavior not in (4, 7):
                self.xp[self.voff[i]:self.voff[i + 1]] = self.x[self.voff[i]:self.voff[i + 1]]
        newx, newv = self.x.copy(), self.v.copy()
        for i, m in enumerate(self.meshes):
            if not cloth(m):
                continue
            s, e = self.voff[i], self.voff[i + 1]
            x, v = self.x[s:e], self.v[s:e]
            mass3 = np.repeat(m.mass, 3).astype(np.float32)
            ext = (np.asarray(p.gravity, np.float32)[None, :] * m.mass[:, None]).astype(np.float32)
            if m.behavior == 0:
                prm = np.array([m.kstretch, m.kshear, m.kbend, m.thickness], np.float32)
                f = R.tri_forces(x, v, ext, mass3, m.mask, np.float32(p.subh), np.float32(p.kair), np.float32(p.kd),
                                 prm, self.adj[i], m.facets.reshape(-1))
                kind = "tri"
            else:
                prm = R.grid_params(m.grid_n, m.grid_rest, (m.kstretch, m.kshear, m.kbend), m.thickness)
                f = R.grid_forces(x, v, ext, mass3, np.float32(p.subh), np.float32(p.kair), np.float32(p.kd), prm)
                kind = "grid"
            xn, vn, _ = R.integrate(kind, x, v, f, mass3, m.mask, csr, offsets, self.voff, i, np.float32(p.subh), prm)
            newx[s:e], newv[s:e] = xn, vn
        self.x, self.v = newx, newv
        self.cursor += 1
        if self.cursor >= p.substeps:
            self.cursor = 0
            self.frame += 1

    def step(self, n=1):
        for _ in range(n):
            self.substep()
