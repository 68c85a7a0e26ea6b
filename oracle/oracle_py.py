"""ctypes access to the CPU checker libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline / reference arm of bench.py, never by the product package.

* ``oracle/_build/liboracle.so``: the C restatement of the reference's serial
  loop (fot_oracle.c), the coloured-plan replay and the plan checks.
* ``oracle/_ref/libref.so``: the reference's own serial / OpenMP loop drivers
  and host plan builder, compiled from the reference sources by
  ``make -C oracle ref`` (present only where it was built).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

u32p = C.POINTER(C.c_uint32)


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def build_ref() -> bool:
    """Compile the reference's serial path where its sources exist (REF_DIR
    in the environment, else oracle/Makefile's default)."""
    subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)
    return os.path.exists(os.path.join(HERE, "_ref", "libref.so"))


_orc = None
_ref = None


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        lib = C.CDLL(ORACLE_SO)
        lib.orc_loop_serial.restype = C.c_int
        lib.orc_replay_hier.restype = C.c_int
        lib.orc_check_plan.restype = C.c_int
        lib.orc_is_permutation.restype = C.c_int
        lib.orc_point_graph.restype = C.c_uint32
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref)")
        lib = C.CDLL(REF_SO)
        lib.ref_loop_serial.restype = C.c_int
        lib.ref_loop_omp.restype = C.c_int
        lib.ref_hier_plan.restype = C.c_int
        lib.ref_count_cache_lines.restype = C.c_uint64
        _ref = lib
    return _ref


class _Args:
    """Keeps the ctypes argument arrays (and the numpy buffers they point to)
    alive for one call."""

    def __init__(self, md, point_data: List[np.ndarray], cell_data: List[np.ndarray]):
        self.maps = [np.ascontiguousarray(m, dtype=np.uint32) for m in md.maps]
        self.n_points = (C.c_uint32 * len(md.n_points))(*md.n_points)
        self.map_ptrs = (u32p * len(self.maps))(*[m.ctypes.data_as(u32p) for m in self.maps])
        self.pd = point_data
        self.cd = cell_data
        self.pd_ptrs = (C.c_void_p * max(1, len(point_data)))(*[d.ctypes.data for d in point_data])
        self.cd_ptrs = (C.c_void_p * max(1, len(cell_data)))(*[d.ctypes.data for d in cell_data])


def _copies(md):
    pd = [np.ascontiguousarray(d).copy() for d in md.point_data]
    cd = [np.ascontiguousarray(d).copy() for d in md.cell_data]
    return pd, cd


def serial(md, iters: int = 1):
    """Oracle serial loop; returns (point_data, cell_data) after `iters`."""
    pd, cd = _copies(md)
    a = _Args(md, pd, cd)
    rc = orc().orc_loop_serial(md.loop, int(md.layout == "soa"), md.n_cells,
                               a.n_points, a.map_ptrs, a.pd_ptrs, a.cd_ptrs, iters)
    if rc:
        raise RuntimeError(f"orc_loop_serial failed: {rc}")
    return pd, cd


class OrcPlan(C.Structure):
    _fields_ = [("n_cells", C.c_uint32), ("n_blocks", C.c_uint32),
                ("n_colours", C.c_uint32), ("mesh_dim", C.c_uint32),
                ("colour_offsets", u32p), ("block_start", u32p),
                ("cell_id", u32p), ("tcol", C.POINTER(C.c_uint8)),
                ("block_ntcol", C.POINTER(C.c_uint8)), ("pts_off", u32p),
                ("pts", u32p), ("lidx", C.POINTER(C.c_uint16))]


def _orc_plan(plan: dict):
    keep = {k: np.ascontiguousarray(v) for k, v in plan.items() if isinstance(v, np.ndarray)}
    p = OrcPlan(plan["n_cells"], plan["n_blocks"], plan["n_colours"], plan["mesh_dim"],
                keep["colour_offsets"].ctypes.data_as(u32p),
                keep["block_start"].ctypes.data_as(u32p),
                keep["cell_id"].ctypes.data_as(u32p),
                keep["tcol"].ctypes.data_as(C.POINTER(C.c_uint8)),
                keep["block_ntcol"].ctypes.data_as(C.POINTER(C.c_uint8)),
                keep["pts_off"].ctypes.data_as(u32p),
                keep["pts"].ctypes.data_as(u32p),
                keep["lidx"].ctypes.data_as(C.POINTER(C.c_uint16)))
    return p, keep


def replay_hier(md, plan: dict, iters: int = 1):
    """CPU replay of a coloured plan (block colours in order, zeroed block
    cache summed in thread-colour order, then out += cache)."""
    pd, cd = _copies(md)
    a = _Args(md, pd, cd)
    p, keep = _orc_plan(plan)
    rc = orc().orc_replay_hier(md.loop, int(md.layout == "soa"), md.n_cells,
                               a.n_points, a.map_ptrs, a.pd_ptrs, a.cd_ptrs,
                               iters, C.byref(p))
    if rc:
        raise RuntimeError(f"orc_replay_hier failed: {rc}")
    return pd, cd


class OrcAirfoil(C.Structure):
    _fields_ = [("cell_to_node", u32p), ("n_bedges", C.c_uint32), ("bedge_to_node", u32p),
                ("bedge_to_cell", u32p), ("bound", C.POINTER(C.c_int32)),
                ("qinf", C.c_double * 4), ("cfl", C.c_double)]


def airfoil(md, extras: dict, iters: int = 1, plan: Optional[dict] = None):
    """The Airfoil iteration around res_calc (orc_airfoil_run): returns
    (point_data after `iters` iterations, rms of the last one).  res_calc
    runs in serial edge order, or replays `plan` (an exported plan, cell_id
    relative to md's cells)."""
    pd, cd = _copies(md)
    a = _Args(md, pd, cd)
    keep = [np.ascontiguousarray(extras["cell_to_node"], dtype=np.uint32),
            np.ascontiguousarray(extras["bedge_to_node"], dtype=np.uint32),
            np.ascontiguousarray(extras["bedge_to_cell"], dtype=np.uint32),
            np.ascontiguousarray(extras["bound"], dtype=np.int32)]
    A = OrcAirfoil(keep[0].ctypes.data_as(u32p), len(keep[2]), keep[1].ctypes.data_as(u32p),
                   keep[2].ctypes.data_as(u32p), keep[3].ctypes.data_as(C.POINTER(C.c_int32)),
                   (C.c_double * 4)(*[float(v) for v in extras["qinf"]]), float(extras["cfl"]))
    P = None
    if plan is not None:
        p, pkeep = _orc_plan(plan)
        P = C.byref(p)
    rms = C.c_double()
    rc = orc().orc_airfoil_run(int(md.layout == "soa"), md.n_cells, a.n_points, a.map_ptrs,
                               a.pd_ptrs, C.byref(A), iters, P, C.byref(rms))
    if rc:
        raise RuntimeError(f"orc_airfoil_run failed: {rc}")
    return pd, rms.value


def check_plan(plan: dict, map0: np.ndarray, n_points0: int, block_size: int):
    """Returns (code, message); code 0 means the plan is valid."""
    p, keep = _orc_plan(plan)
    m = np.ascontiguousarray(map0, dtype=np.uint32)
    err = C.create_string_buffer(512)
    rc = orc().orc_check_plan(C.byref(p), m.ctypes.data_as(u32p), n_points0,
                              block_size, err, 512)
    return rc, err.value.decode()


def is_permutation(perm: np.ndarray) -> bool:
    p = np.ascontiguousarray(perm, dtype=np.uint32)
    return bool(orc().orc_is_permutation(p.ctypes.data_as(u32p), p.size))


def point_graph(n_points: int, mapping: np.ndarray):
    m = np.ascontiguousarray(mapping, dtype=np.uint32)
    n_cells, dim = m.shape
    ind = np.zeros(n_points + 1, dtype=np.uint32)
    ends = np.zeros(max(1, n_cells * dim * (dim - 1)), dtype=np.uint32)
    n = orc().orc_point_graph(n_points, n_cells, dim, m.ctypes.data_as(u32p),
                              ind.ctypes.data_as(u32p), ends.ctypes.data_as(u32p))
    return ind, ends[:n].copy()


def bandwidth_profile(n_points: int, mapping: np.ndarray):
    m = np.ascontiguousarray(mapping, dtype=np.uint32)
    bw = C.c_uint64()
    prof = C.c_uint64()
    orc().orc_bandwidth_profile(n_points, m.shape[0], m.shape[1],
                                m.ctypes.data_as(u32p), C.byref(bw), C.byref(prof))
    return bw.value, prof.value


# ---------------------------------------------------------------------------
# the reference's own compiled loop drivers
# ---------------------------------------------------------------------------

def ref_serial(md, iters: int = 1):
    """The reference's loopCPUCellCentred<StepSeq>; returns (point_data,
    cell_data, seconds)."""
    pd, cd = _copies(md)
    a = _Args(md, pd, cd)
    secs = C.c_double()
    rc = ref().ref_loop_serial(md.loop, int(md.layout == "soa"), md.n_cells,
                               a.n_points, a.map_ptrs, a.pd_ptrs, a.cd_ptrs,
                               iters, C.byref(secs))
    if rc:
        raise RuntimeError(f"ref_loop_serial failed: {rc}")
    return pd, cd, secs.value


def ref_omp(md, iters: int = 1):
    """The reference's loopCPUCellCentredOMP<StepOMP> (AOS only); returns
    (point_data, cell_data, loop_seconds, colouring_seconds)."""
    pd, cd = _copies(md)
    a = _Args(md, pd, cd)
    t_loop = C.c_double()
    t_col = C.c_double()
    rc = ref().ref_loop_omp(md.loop, int(md.layout == "soa"), md.n_cells,
                            a.n_points, a.map_ptrs, a.pd_ptrs, a.cd_ptrs, iters,
                            C.byref(t_loop), C.byref(t_col))
    if rc:
        raise RuntimeError(f"ref_loop_omp failed: {rc}")
    return pd, cd, t_loop.value, t_col.value


def ref_hier_plan(md, block_size: int):
    """The reference's host plan builder (HierarchicalColourMemory)."""
    pd, cd = _copies(md)
    a = _Args(md, pd, cd)
    secs = C.c_double()
    nc = C.c_uint32()
    nb = C.c_uint32()
    tc = C.c_double()
    rc = ref().ref_hier_plan(md.loop, md.n_cells, a.n_points, a.map_ptrs,
                             a.pd_ptrs, a.cd_ptrs, block_size, C.byref(secs),
                             C.byref(nc), C.byref(nb), C.byref(tc))
    if rc:
        raise RuntimeError(f"ref_hier_plan failed: {rc}")
    return {"seconds": secs.value, "n_colours": nc.value, "n_blocks": nb.value,
            "avg_thread_colours": tc.value}


def sector_count(map0: np.ndarray, cells_per_block: int, dim: int, type_size: int, soa: bool) -> int:
    """The reference's sector model (countCacheLinesForBlock,
    problem.hpp:654-672) summed over blocks of consecutive cells, restated
    with numpy: per block, the distinct 32-byte sectors of point dataset 0
    touched -- AOS: element p * dim + d lies in sector (p * dim + d) //
    (32 // type_size); SOA: distinct p // (32 // type_size), times dim."""
    m = np.asarray(map0, dtype=np.int64)
    per = 32 // type_size
    total = 0
    for c0 in range(0, m.shape[0], cells_per_block):
        pts = m[c0:c0 + cells_per_block].ravel()
        if soa:
            total += dim * len(np.unique(pts // per))
        else:
            el = (pts[:, None] * dim + np.arange(dim)[None, :]).ravel()
            total += len(np.unique(el // per))
    return int(total)


def ref_sector_count(map0: np.ndarray, cells_per_block: int, dim: int, type_size: int,
                     soa: bool) -> int:
    """The same through the reference's own countCacheLinesForBlock."""
    m = np.ascontiguousarray(map0, dtype=np.uint32)
    return int(ref().ref_count_cache_lines(m.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           C.c_uint32(m.shape[0]), C.c_uint32(m.shape[1]),
                                           C.c_uint32(cells_per_block), C.c_uint32(dim),
                                           C.c_uint32(type_size), C.c_int(int(soa))))
