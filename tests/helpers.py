"""Shared helpers of the test suite: golden fixtures, error metrics and a
small pure-Python plan builder used to exercise the oracle's replay and plan
checks on the CPU."""
import os

import numpy as np

from cuda_fot_b200 import meshgen as mg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name))
    loop = int(z["loop"])
    n_maps = sum(1 for k in z.files if k.startswith("map"))
    n_pd = sum(1 for k in z.files if k.startswith("point_in"))
    n_cd = sum(1 for k in z.files if k.startswith("cell_in"))
    md = mg.MeshData(loop, int(z["n_cells"]), [int(v) for v in z["n_points"]],
                     [z[f"map{k}"] for k in range(n_maps)],
                     [z[f"point_in{k}"] for k in range(n_pd)],
                     [z[f"cell_in{j}"] for j in range(n_cd)], str(z["layout"]))
    out_pd = [z[f"point_out{k}"] for k in range(n_pd)]
    out_cd = [z[f"cell_out{j}"] for j in range(n_cd)]
    return md, out_pd, out_cd, int(z["iters"])


def golden_names():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def rel_err(a, b):
    """Normwise relative error max|a-b| / max|b| (b the reference)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    if den == 0:
        return float(np.abs(a - b).max())
    return float(np.abs(a - b).max() / den)


def bitwise_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def py_plan(md, block_size):
    """A valid hierarchical plan built in Python: contiguous blocks, greedy
    block colouring against written points, greedy thread colouring inside
    each block, cells sorted by thread colour.  Returns the export dict the
    oracle replay and checks take."""
    m0 = np.asarray(md.maps[0])
    n, dim = m0.shape
    nb = (n + block_size - 1) // block_size
    point_cols = {}
    bcol = []
    for b in range(nb):
        pts = set(m0[b * block_size:(b + 1) * block_size].ravel().tolist())
        used = set()
        for p in pts:
            used |= point_cols.get(p, set())
        c = 0
        while c in used:
            c += 1
        bcol.append(c)
        for p in pts:
            point_cols.setdefault(p, set()).add(c)
    n_col = max(bcol) + 1
    order = sorted(range(nb), key=lambda b: (bcol[b], b))
    colour_offsets = np.zeros(n_col + 1, dtype=np.uint32)
    for b in range(nb):
        colour_offsets[bcol[b] + 1] += 1
    colour_offsets = np.cumsum(colour_offsets).astype(np.uint32)
    block_start, cell_id, tcol, ntcol, pts_off, pts_all = [0], [], [], [], [0], []
    lidx = [[] for _ in range(dim)]
    for b in order:
        cells = list(range(b * block_size, min(n, (b + 1) * block_size)))
        pts = sorted(set(m0[cells].ravel().tolist()))
        local = {p: i for i, p in enumerate(pts)}
        masks = {}
        cc = []
        for c in cells:
            forb = set()
            for s in range(dim):
                forb |= masks.get(m0[c, s], set())
            k = 0
            while k in forb:
                k += 1
            cc.append(k)
            for s in range(dim):
                masks.setdefault(m0[c, s], set()).add(k)
        srt = sorted(range(len(cells)), key=lambda i: (cc[i], i))
        for i in srt:
            c = cells[i]
            cell_id.append(c)
            tcol.append(cc[i])
            for s in range(dim):
                lidx[s].append(local[m0[c, s]])
        ntcol.append(max(cc) + 1)
        block_start.append(len(cell_id))
        pts_all.extend(pts)
        pts_off.append(len(pts_all))
    return {"n_cells": n, "n_blocks": nb, "n_colours": n_col, "mesh_dim": dim,
            "colour_offsets": colour_offsets,
            "block_start": np.array(block_start, dtype=np.uint32),
            "cell_id": np.array(cell_id, dtype=np.uint32),
            "tcol": np.array(tcol, dtype=np.uint8),
            "block_ntcol": np.array(ntcol, dtype=np.uint8),
            "pts_off": np.array(pts_off, dtype=np.uint32),
            "pts": np.array(pts_all, dtype=np.uint32),
            "lidx": np.array(lidx, dtype=np.uint16).reshape(dim, n)}
