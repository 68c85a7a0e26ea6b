"""Seeded synthetic meshes and data for the five indirect-increment loops.

The application meshes the reference measured on (Airfoil, miniAero, LULESH,
Volna, BookLeaf inputs read from external paths, e.g. ``res_calc.cu:13-16``)
are not available, so these generators stand in for them with the shapes,
sizes and value distributions of the benchmark configurations.  Every array
comes from ``numpy.random.Generator(Philox(seed))``; the default seed 1
mirrors the reference test harness's ``srand(1)`` (``tests.hpp:44``).

A generated problem is a :class:`MeshData`:

* ``maps[k]``: uint32 array (n_cells, mesh_dim[k]), AOS, the k-th mapping;
* ``n_points[k]``: size of mapping k's target set;
* ``point_data[k]``: array (n_points[k], dim) in AOS (``layout="aos"``) or
  (dim, n_points[k]) in SOA, the reference's ``point_weights[k]``;
* ``cell_data[j]``: array (dim, n_cells), always SOA like the reference's
  ``cell_weights[j]``.

Data bindings follow each reference driver's ``initProblem``:
res_calc.cu:10-28, mini_aero.cu:10-24, lulesh.cu:10-24, volna.cu:11-27,
getacc.cu:11-26.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List

import numpy as np

RES_CALC, MINI_AERO, LULESH, VOLNA, GETACC = range(5)
LOOP_NAMES = ["res_calc", "mini_aero", "lulesh", "volna", "getacc"]


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


@dataclass
class MeshData:
    loop: int
    n_cells: int
    n_points: List[int]
    maps: List[np.ndarray]
    point_data: List[np.ndarray]
    cell_data: List[np.ndarray]
    layout: str = "aos"
    meta: dict = field(default_factory=dict)

    def copy(self) -> "MeshData":
        return MeshData(self.loop, self.n_cells, list(self.n_points),
                        [m.copy() for m in self.maps],
                        [d.copy() for d in self.point_data],
                        [d.copy() for d in self.cell_data], self.layout,
                        dict(self.meta))

    def to_layout(self, layout: str) -> "MeshData":
        """Point data in AOS (n, dim) or SOA (dim, n); cell data stays SOA."""
        out = self.copy()
        if layout != self.layout:
            out.point_data = [np.ascontiguousarray(d.T) for d in self.point_data]
            out.layout = layout
        return out

    def unique_bytes(self) -> int:
        """Algorithmic bytes of one loop iteration: every indirectly read point
        dataset once, the incremented dataset twice (read and write), every
        direct dataset once, every distinct mapping once (4 B per entry)."""
        nbytes = 2 * self.point_data[0].nbytes
        for k in range(1, len(self.point_data)):
            nbytes += self.point_data[k].nbytes
        for d in self.cell_data:
            nbytes += d.nbytes
        seen = []
        for m in self.maps:
            if not any(m.shape == s.shape and np.array_equal(m, s) for s in seen):
                seen.append(m)
                nbytes += m.nbytes
        return nbytes


# --------------------------------------------------------------------------
# permutations of a point set
# --------------------------------------------------------------------------

def permute_points(md: MeshData, point_sets, perm: np.ndarray) -> None:
    """Renumber the points of the given mappings: old point i becomes perm[i].
    The point datasets bound to those mappings move with them."""
    perm = perm.astype(np.uint32)
    for k in point_sets:
        md.maps[k] = perm[md.maps[k]]
        d = md.point_data[k]
        if md.layout == "aos":
            new = np.empty_like(d)
            new[perm] = d
        else:
            new = np.empty_like(d)
            new[:, perm] = d
        md.point_data[k] = new


def permute_cells(md: MeshData, order: np.ndarray) -> None:
    """Reorder the cells: new cell i is old cell order[i]."""
    for k in range(len(md.maps)):
        md.maps[k] = np.ascontiguousarray(md.maps[k][order])
    md.cell_data = [np.ascontiguousarray(d[:, order]) for d in md.cell_data]


# --------------------------------------------------------------------------
# res_calc: Airfoil-style edge flux on a 2D quad grid
# --------------------------------------------------------------------------

def res_calc(nx: int = 1000, ny: int = 1000, seed: int = 1,
             layout: str = "aos") -> MeshData:
    """nx x ny quad cells, (nx+1) x (ny+1) nodes with unit spacing plus
    U(-0.1, 0.1) jitter; the interior edges each map to their 2 end nodes and
    their 2 cells (cell 1 = left / bottom).  q = (1, 0.5, 0, 2.5) times
    (1 + U(-0.01, 0.01)) per component, adt = U(0.5, 1.5), res = 0.
    Mappings (res_calc.cu:13-21): 0 edge->cell (res), 1 edge->node (x),
    2 and 3 edge->cell (q, adt)."""
    g = rng(seed)
    nnode_x = nx + 1
    cells = np.arange(nx * ny, dtype=np.int64).reshape(ny, nx)  # [j, i]
    node = lambda i, j: j * nnode_x + i  # noqa: E731
    # edges in natural order: for each cell (row-major) its right, then top edge
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    ii = ii.ravel()
    jj = jj.ravel()
    has_r = ii < nx - 1
    has_t = jj < ny - 1
    n_r = has_r.astype(np.int64)
    n_t = has_t.astype(np.int64)
    per = n_r + n_t
    start = np.concatenate([[0], np.cumsum(per)[:-1]])
    n_edges = int(per.sum())
    e2c = np.empty((n_edges, 2), dtype=np.uint32)
    e2n = np.empty((n_edges, 2), dtype=np.uint32)
    # right edges: between cell (i,j) and (i+1,j); normal +x so node1 is the
    # upper end (dy = y1 - y2 > 0)
    r_idx = start[has_r]
    i_r, j_r = ii[has_r], jj[has_r]
    e2c[r_idx, 0] = cells[j_r, i_r]
    e2c[r_idx, 1] = cells[j_r, i_r + 1]
    e2n[r_idx, 0] = node(i_r + 1, j_r + 1)
    e2n[r_idx, 1] = node(i_r + 1, j_r)
    # top edges: between cell (i,j) and (i,j+1); normal +y so node1 is the
    # left end (x1 - x2 < 0)
    t_idx = start[has_t] + n_r[has_t]
    i_t, j_t = ii[has_t], jj[has_t]
    e2c[t_idx, 0] = cells[j_t, i_t]
    e2c[t_idx, 1] = cells[j_t + 1, i_t]
    e2n[t_idx, 0] = node(i_t, j_t + 1)
    e2n[t_idx, 1] = node(i_t + 1, j_t + 1)
    n_nodes = (nx + 1) * (ny + 1)
    n_cells = nx * ny
    gx, gy = np.meshgrid(np.arange(nx + 1, dtype=np.float64),
                         np.arange(ny + 1, dtype=np.float64))
    x = np.stack([gx.ravel(), gy.ravel()], axis=1)
    x += g.uniform(-0.1, 0.1, size=x.shape)
    q = np.array([1.0, 0.5, 0.0, 2.5]) * (1.0 + g.uniform(-0.01, 0.01, size=(n_cells, 4)))
    adt = g.uniform(0.5, 1.5, size=(n_cells, 1))
    res = np.zeros((n_cells, 4))
    md = MeshData(RES_CALC, n_edges, [n_cells, n_nodes, n_cells, n_cells],
                  [e2c, e2n, e2c.copy(), e2c.copy()], [res, x, q, adt], [],
                  "aos", {"nx": nx, "ny": ny, "seed": seed})
    return md.to_layout(layout)


def airfoil_extras(md: MeshData) -> dict:
    """The data an Airfoil solver iteration needs beyond res_calc's, for a
    mesh made by res_calc(nx, ny): each cell's 4 nodes counter-clockwise, the
    4 (nx + ny) boundary edges (bottom, right, top, left) oriented like the
    interior edges (with dx = x1 - x2, dy = y1 - y2 the normal (dy, -dx)
    points out of the cell), solid walls at the bottom and top (bound 1),
    far field left and right (bound 0), and the free stream
    qinf = (1, 0.5, 0, 2.5) the generator's q perturbs."""
    nx, ny = md.meta["nx"], md.meta["ny"]
    node = lambda i, j: j * (nx + 1) + i  # noqa: E731
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    ii, jj = ii.ravel(), jj.ravel()
    c2n = np.stack([node(ii, jj), node(ii + 1, jj), node(ii + 1, jj + 1), node(ii, jj + 1)],
                   axis=1).astype(np.uint32)
    i = np.arange(nx)
    j = np.arange(ny)
    cell = lambda i, j: j * nx + i  # noqa: E731
    bottom = (np.stack([node(i + 1, 0), node(i, 0)], 1), cell(i, 0), np.ones(nx))
    right = (np.stack([node(nx, j + 1), node(nx, j)], 1), cell(nx - 1, j), np.zeros(ny))
    top = (np.stack([node(i, ny), node(i + 1, ny)], 1), cell(i, ny - 1), np.ones(nx))
    left = (np.stack([node(0, j), node(0, j + 1)], 1), cell(0, j), np.zeros(ny))
    parts = (bottom, right, top, left)
    return {"cell_to_node": c2n,
            "bedge_to_node": np.concatenate([p[0] for p in parts]).astype(np.uint32),
            "bedge_to_cell": np.concatenate([p[1] for p in parts]).astype(np.uint32),
            "bound": np.concatenate([p[2] for p in parts]).astype(np.int32),
            "qinf": np.array([1.0, 0.5, 0.0, 2.5]), "cfl": 0.9}


# --------------------------------------------------------------------------
# mini_aero: 3D face flux on a structured hex mesh
# --------------------------------------------------------------------------

def mini_aero(n: int = 128, seed: int = 1, layout: str = "aos",
              permute: bool = True) -> MeshData:
    """n^3 hex cells, 3 (n-1) n^2 interior faces each giving (left, right)
    cells.  Face record (12, SOA): centre, unit normal (area 1), tangent,
    binormal (the two other unit axes).  Cell record (28): conserved values
    (1, 0.3, 0.1, 0, 2.5) (1 + U(-0.01, 0.01)), centre (3), gradients
    U(-1e-3, 1e-3) (15), limiters U(0, 1) (5) at offsets 0, 5, 8, 23
    (mini_aero.hpp:57-88).  flux = 0.  With permute, cell numbering is a
    seeded random permutation (worst locality).  Mappings
    (mini_aero.cu:13-19): 0 and 1 are the same face->cell mapping."""
    g = rng(seed)
    n_cells = n ** 3
    cid = np.arange(n_cells, dtype=np.int64).reshape(n, n, n)  # [z, y, x]
    faces_l, faces_r, centres, axes = [], [], [], []
    for axis in range(3):
        if axis == 0:
            l, r = cid[:, :, :-1], cid[:, :, 1:]
        elif axis == 1:
            l, r = cid[:, :-1, :], cid[:, 1:, :]
        else:
            l, r = cid[:-1, :, :], cid[1:, :, :]
        l = l.ravel()
        r = r.ravel()
        lz, ly, lx = np.unravel_index(l, (n, n, n))
        c = np.stack([lx + 0.5, ly + 0.5, lz + 0.5], axis=1).astype(np.float64)
        c[:, axis] += 0.5
        faces_l.append(l)
        faces_r.append(r)
        centres.append(c)
        axes.append(np.full(l.shape, axis))
    l = np.concatenate(faces_l)
    r = np.concatenate(faces_r)
    centre = np.concatenate(centres)
    axis = np.concatenate(axes)
    n_faces = l.size
    eye = np.eye(3)
    face = np.empty((12, n_faces))
    face[0:3] = centre.T
    face[3:6] = eye[axis].T
    face[6:9] = eye[(axis + 1) % 3].T
    face[9:12] = eye[(axis + 2) % 3].T
    f2c = np.stack([l, r], axis=1).astype(np.uint32)
    cz, cy, cx = np.unravel_index(np.arange(n_cells), (n, n, n))
    rec = np.empty((n_cells, 28))
    rec[:, 0:5] = np.array([1.0, 0.3, 0.1, 0.0, 2.5]) * (
        1.0 + g.uniform(-0.01, 0.01, size=(n_cells, 5)))
    rec[:, 5:8] = np.stack([cx + 0.5, cy + 0.5, cz + 0.5], axis=1)
    rec[:, 8:23] = g.uniform(-1e-3, 1e-3, size=(n_cells, 15))
    rec[:, 23:28] = g.uniform(0.0, 1.0, size=(n_cells, 5))
    flux = np.zeros((n_cells, 5))
    md = MeshData(MINI_AERO, n_faces, [n_cells, n_cells], [f2c, f2c.copy()],
                  [flux, rec], [face], "aos",
                  {"n": n, "seed": seed, "permuted": permute})
    if permute:
        perm = g.permutation(n_cells)
        permute_points(md, [0], perm)
        md.maps[1] = md.maps[0].copy()
        rec_new = np.empty_like(rec)
        rec_new[perm] = rec
        md.point_data[1] = rec_new
    return md.to_layout(layout)


# --------------------------------------------------------------------------
# LULESH: hex element -> node force scatter
# --------------------------------------------------------------------------

def lulesh(n: int = 96, seed: int = 1, layout: str = "aos",
           permute: bool = True) -> MeshData:
    """n^3 hex elements, (n+1)^3 nodes in the node order of grid.hpp:427-442
    (bottom face 0-3 counter-clockwise, then the top face), unit spacing plus
    U(-0.05, 0.05) jitter; sigma_xx/yy/zz = U(-1, 0) (cell data 0, SOA),
    determ = 0 (cell data 1), f = 0.  With permute, node numbering is a seeded
    random permutation (worst locality).  Mappings (lulesh.cu:13-19): 0 and 1
    are the same element->node mapping."""
    g = rng(seed)
    N = n + 1
    l, rr, c = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    l, rr, c = l.ravel(), rr.ravel(), c.ravel()
    bot = l * N * N
    top = (l + 1) * N * N
    inner = rr * N + c
    outer = (rr + 1) * N + c
    e2n = np.stack([bot + inner, bot + inner + 1, bot + outer + 1, bot + outer,
                    top + inner, top + inner + 1, top + outer + 1, top + outer],
                   axis=1).astype(np.uint32)
    n_nodes = N ** 3
    nl, nr, nc = np.unravel_index(np.arange(n_nodes), (N, N, N))
    xyz = np.stack([nc, nr, nl], axis=1).astype(np.float64)
    xyz += g.uniform(-0.05, 0.05, size=xyz.shape)
    n_el = n ** 3
    sig = g.uniform(-1.0, 0.0, size=(3, n_el))
    determ = np.zeros((1, n_el))
    f = np.zeros((n_nodes, 3))
    md = MeshData(LULESH, n_el, [n_nodes, n_nodes], [e2n, e2n.copy()],
                  [f, xyz], [sig, determ], "aos",
                  {"n": n, "seed": seed, "permuted": permute})
    if permute:
        perm = g.permutation(n_nodes)
        permute_points(md, [0], perm)
        md.maps[1] = md.maps[0].copy()
        new = np.empty_like(xyz)
        new[perm] = xyz
        md.point_data[1] = new
    return md.to_layout(layout)


# --------------------------------------------------------------------------
# volna: shallow-water edge flux on triangles (FP32)
# --------------------------------------------------------------------------

def volna(nx: int = 256, ny: int = 256, seed: int = 1,
          layout: str = "aos") -> MeshData:
    """nx x ny unit quads, each split along its (i,j)-(i+1,j+1) diagonal
    into a lower triangle T0 and an upper triangle T1; the interior edges
    (diagonals and shared quad sides) each map to 2 triangles.  Per triangle
    (h, hu, hv, zb) = (1 + U(0, 0.1), 0, 0, U(-0.1, 0)) (FP32, the
    incremented dataset) and the triangle area 0.5 (cellVolumes).  Per edge:
    fluxes U(-1e-3, 1e-3) (3), bathySource U(-1e-4, 1e-4) (2), the unit normal
    from the geometry (2), isBoundary = 0 (int).  Mappings (volna.cu:14-18):
    0 and 1 are the same edge->cell mapping."""
    g = rng(seed)
    t0 = lambda i, j: 2 * (j * nx + i)      # noqa: E731
    t1 = lambda i, j: 2 * (j * nx + i) + 1  # noqa: E731
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    ii, jj = ii.ravel(), jj.ravel()
    s2 = 1.0 / np.sqrt(2.0)
    # diagonal (T0 -> T1): normal (-1, 1)/sqrt2
    ed = [np.stack([t0(ii, jj), t1(ii, jj)], axis=1)]
    nd = [np.tile([-s2, s2], (ii.size, 1))]
    m = ii < nx - 1  # right side: T0(i,j) -> T1(i+1,j), normal +x
    ed.append(np.stack([t0(ii[m], jj[m]), t1(ii[m] + 1, jj[m])], axis=1))
    nd.append(np.tile([1.0, 0.0], (m.sum(), 1)))
    m = jj < ny - 1  # top side: T1(i,j) -> T0(i,j+1), normal +y
    ed.append(np.stack([t1(ii[m], jj[m]), t0(ii[m], jj[m] + 1)], axis=1))
    nd.append(np.tile([0.0, 1.0], (m.sum(), 1)))
    e2c = np.concatenate(ed).astype(np.uint32)
    normals = np.concatenate(nd)
    # interleave so that neighbouring edges are adjacent in the natural order
    order = np.argsort(np.minimum(e2c[:, 0], e2c[:, 1]), kind="stable")
    e2c = np.ascontiguousarray(e2c[order])
    normals = normals[order]
    n_edges = e2c.shape[0]
    n_tri = 2 * nx * ny
    out = np.empty((n_tri, 4), dtype=np.float32)
    out[:, 0] = 1.0 + g.uniform(0.0, 0.1, size=n_tri)
    out[:, 1] = 0.0
    out[:, 2] = 0.0
    out[:, 3] = g.uniform(-0.1, 0.0, size=n_tri)
    vol = np.full((n_tri, 1), 0.5, dtype=np.float32)
    flux = g.uniform(-1e-3, 1e-3, size=(3, n_edges)).astype(np.float32)
    bathy = g.uniform(-1e-4, 1e-4, size=(2, n_edges)).astype(np.float32)
    norms = np.ascontiguousarray(normals.T.astype(np.float32))
    isb = np.zeros((1, n_edges), dtype=np.int32)
    md = MeshData(VOLNA, n_edges, [n_tri, n_tri], [e2c, e2c.copy()],
                  [out, vol], [flux, bathy, norms, isb], "aos",
                  {"nx": nx, "ny": ny, "seed": seed})
    return md.to_layout(layout)


# --------------------------------------------------------------------------
# getacc: BookLeaf-style quad element -> node scatter (FP64)
# --------------------------------------------------------------------------

def getacc(nx: int = 512, ny: int = 512, seed: int = 1,
           layout: str = "aos") -> MeshData:
    """nx x ny quad elements, (nx+1)(ny+1) nodes, element nodes counter-
    clockwise.  Per element: cnmass U(0, 1) with about 1/8 of the corners set
    to 0 (so the functor's fallback branches run), rho U(0.5, 1.5), cnwt
    U(0, 1), cnfx and cnfy U(-1, 1).  The node accumulator (4) starts at 0.
    Mapping (getacc.cu:14-17): 0 element->node."""
    g = rng(seed)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    ii, jj = ii.ravel(), jj.ravel()
    N = nx + 1
    e2n = np.stack([jj * N + ii, jj * N + ii + 1, (jj + 1) * N + ii + 1,
                    (jj + 1) * N + ii], axis=1).astype(np.uint32)
    n_el = nx * ny
    n_nodes = (nx + 1) * (ny + 1)
    cnmass = g.uniform(0.0, 1.0, size=(4, n_el))
    cnmass[g.uniform(size=(4, n_el)) < 0.125] = 0.0
    rho = g.uniform(0.5, 1.5, size=(1, n_el))
    cnwt = g.uniform(0.0, 1.0, size=(4, n_el))
    cnfx = g.uniform(-1.0, 1.0, size=(4, n_el))
    cnfy = g.uniform(-1.0, 1.0, size=(4, n_el))
    out = np.zeros((n_nodes, 4))
    md = MeshData(GETACC, n_el, [n_nodes], [e2n], [out],
                  [cnmass, rho, cnwt, cnfx, cnfy], "aos",
                  {"nx": nx, "ny": ny, "seed": seed})
    return md.to_layout(layout)


GENERATORS = {RES_CALC: res_calc, MINI_AERO: mini_aero, LULESH: lulesh,
              VOLNA: volna, GETACC: getacc}


def small(loop: int, seed: int = 1, layout: str = "aos") -> MeshData:
    """A small instance of each loop (a few hundred to a few thousand cells),
    sized for the oracle and the golden fixtures."""
    if loop == RES_CALC:
        return res_calc(12, 10, seed, layout)
    if loop == MINI_AERO:
        return mini_aero(6, seed, layout)
    if loop == LULESH:
        return lulesh(5, seed, layout)
    if loop == VOLNA:
        return volna(9, 7, seed, layout)
    if loop == GETACC:
        return getacc(9, 7, seed, layout)
    raise ValueError(loop)
