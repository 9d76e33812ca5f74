"""Shared helpers for the parity tests."""
import numpy as np


def canon_pairs(pairs: np.ndarray) -> np.ndarray:
    """(point, tri) pairs sorted lexicographically."""
    p = np.asarray(pairs, np.uint32).reshape(-1, 2)
    if len(p) == 0:
        return p
    o = np.lexsort((p[:, 1], p[:, 0]))
    return p[o]


def canon_rows(rows) -> np.ndarray:
    """Broad rows as a sorted (qobj, point, tobj, tri) uint32 table."""
    t = np.stack([rows["qobj"], rows["point"], rows["tobj"], rows["tri"]], 1).astype(np.uint32)
    if len(t) == 0:
        return t
    o = np.lexsort((t[:, 3], t[:, 2], t[:, 1], t[:, 0]))
    return t[o]


def rel_err(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale) if a.size else 0.0


def reachable(nodes) -> np.ndarray:
    """Mask of the nodes a traversal from the root can reach (runs of three or
    more equal Morton codes leave unclaimed subtrees in the reference's
    topology; their boxes are never read)."""
    n = (len(nodes) + 1) // 2
    seen = np.zeros(len(nodes), bool)
    stack = [0]
    while stack:
        i = stack.pop()
        if seen[i]:
            continue
        seen[i] = True
        if nodes["a"][i] >= 0 and i < n - 1:
            stack += [int(nodes["a"][i]), int(nodes["b"][i])]
    return seen


def canon_rows_full(rows) -> np.ndarray:
    """BroadCollision rows (any structured dtype with the 8 row fields) as a
    lexicographically sorted (n, 8) uint64 array."""
    names = ("point", "tri", "qobj", "tobj", "qbeh", "tbeh", "qshape", "tshape")
    if len(rows) == 0:
        return np.zeros((0, 8), np.uint64)
    a = np.stack([np.asarray(rows[k]).astype(np.uint64) for k in names], 1)
    return a[np.lexsort(a.T[::-1])]
