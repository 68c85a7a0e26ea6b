"""Python host binding of libfot's C ABI (include/fot.h).

It mirrors the reference's host interface (``Problem<SOA>`` in problem.hpp):
a :class:`Problem` owns a mesh and its datasets on the GPU; ``reorder``,
``partition``, ``reorder_to_partition`` and ``renumber_points`` are the
reference's ordering calls; ``loop_gpu_cell_centred(num)`` and
``loop_gpu_hierarchical(num)`` its loop drivers (with the camel-case names as
aliases); ``point_weights(k)`` / ``cell_weights(j)`` read datasets back and
``applied_permutation`` maps original point numbers to current ones.

Every call goes through libfot.so; there is no CPU fallback.  Importing this
module raises if the library has not been built
(``python -m cuda_fot_b200.build``).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional

import numpy as np

from . import meshgen as mg

_HERE = os.path.dirname(os.path.abspath(__file__))
# FOT_LIBRARY selects another build of the library (e.g. one compiled with
# `python -m cuda_fot_b200.build --functor-dir DIR --out PATH`)
LIB_PATH = os.environ.get("FOT_LIBRARY") or os.path.join(_HERE, "libfot.so")

FOT_OK = 0
AOS, SOA = 0, 1
EXEC_ATOMIC, EXEC_HIER, EXEC_HIER_LAUNCH = 0, 1, 2
ORDER_NATURAL, ORDER_RANDOM, ORDER_RCM, ORDER_GPS = 0, 1, 2, 3
PLAN_NO_AGGREGATE, PLAN_USE_PARTITION, PLAN_DIRECT_READS, PLAN_SIMPLE_TILES = 1, 2, 4, 8
PLAN_BLOCK_FLAGS = 16
PARTITION_BISECT, PARTITION_GROW = 0, 1

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cuda_fot_b200.build`")
_lib = C.CDLL(LIB_PATH)
_lib.fot_last_error.restype = C.c_char_p
_lib.fot_version.restype = C.c_char_p

u32p = C.POINTER(C.c_uint32)


class FotError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libfot error {code}: {msg}")
        self.code = code


def _check(rc: int) -> None:
    if rc != FOT_OK:
        raise FotError(rc, _lib.fot_last_error().decode())


class LoopInfo(C.Structure):
    _fields_ = [("n_mappings", C.c_uint32), ("mesh_dim", C.c_uint32 * 4),
                ("n_point_sets", C.c_uint32), ("point_dim", C.c_uint32 * 4),
                ("point_type_size", C.c_uint32 * 4), ("n_cell_sets", C.c_uint32),
                ("cell_dim", C.c_uint32 * 8), ("cell_type_size", C.c_uint32 * 8),
                ("cell_written_mask", C.c_uint32)]


class PlanDesc(C.Structure):
    _fields_ = [("exec", C.c_int), ("block_size", C.c_uint32), ("flags", C.c_uint32),
                ("reserved", C.c_uint32)]


class PlanStats(C.Structure):
    _fields_ = [("exec", C.c_int), ("block_size", C.c_uint32), ("n_blocks", C.c_uint32),
                ("n_colours", C.c_uint32), ("max_block_points", C.c_uint32),
                ("max_block_points1", C.c_uint32), ("max_thread_colours", C.c_uint32),
                ("avg_thread_colours", C.c_double), ("avg_block_points", C.c_double),
                ("plan_bytes", C.c_uint64), ("smem_bytes", C.c_uint32), ("grid", C.c_uint32),
                ("build_ms", C.c_double), ("shared_points", C.c_uint32),
                ("partial_slots", C.c_uint32), ("kernel", C.c_char * 32)]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["kernel"] = d["kernel"].decode()
        return d


def version() -> str:
    return _lib.fot_version().decode()


def loop_info(loop: int) -> LoopInfo:
    info = LoopInfo()
    _check(_lib.fot_loop_describe(loop, C.byref(info)))
    return info


def _dtype(type_size: int, loop: int, cell_set: Optional[int] = None):
    if type_size == 8:
        return np.float64
    if loop == mg.VOLNA and cell_set == 3:
        return np.int32
    return np.float32


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)  # torch.cuda.Stream


class Plan:
    """An execution plan (fot_plan): atomic, or hierarchical-colour."""

    def __init__(self, problem: "Problem", exec: int, block_size: int = 256, flags: int = 0):
        self.problem = problem
        self._h = C.c_void_p()
        desc = PlanDesc(exec, block_size, flags, 0)
        _check(_lib.fot_plan_build(problem._h, C.byref(desc), C.byref(self._h)))
        self.exec = exec
        self.block_size = block_size

    def stats(self) -> dict:
        s = PlanStats()
        _check(_lib.fot_plan_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def export(self) -> dict:
        """Plan arrays for the oracle's checks and replay.  cell_id maps each
        position to the cell's index before this plan was built."""
        nb, nc, npts = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(_lib.fot_plan_export(self._h, C.byref(nb), C.byref(nc), C.byref(npts),
                                    *([None] * 9)))
        p = self.problem
        n, D = p.n_cells, p.info.mesh_dim[0]
        arrs = {"colour_offsets": np.zeros(nc.value + 1, np.uint32),
                "block_start": np.zeros(nb.value + 1, np.uint32),
                "cell_id": np.zeros(n, np.uint32), "tcol": np.zeros(n, np.uint8),
                "block_ntcol": np.zeros(nb.value, np.uint8),
                "pts_off": np.zeros(nb.value + 1, np.uint32),
                "pts": np.zeros(max(1, npts.value), np.uint32),
                "lidx": np.zeros((D, n), np.uint16)}
        _check(_lib.fot_plan_export(
            self._h, None, None, None,
            *[arrs[k].ctypes.data_as(C.c_void_p) for k in
              ["colour_offsets", "block_start", "cell_id", "tcol", "block_ntcol", "pts_off",
               "pts", "lidx"]]))
        arrs.update({"n_cells": n, "n_blocks": nb.value, "n_colours": nc.value, "mesh_dim": D})
        return arrs

    def run(self, iterations: int = 1, stream=None) -> None:
        _check(_lib.fot_run(self.problem._h, self._h, iterations, _stream_ptr(stream)))

    def graph(self, iterations: int, stream=None) -> "Graph":
        return Graph(self, iterations, stream)

    def sector_count(self, layout: Optional[str] = None):
        """The reference's sector model over this plan's blocks and their
        written points (fot_plan_sector_count): (sectors, blocks)."""
        lay = -1 if layout is None else (SOA if layout == "soa" else AOS)
        sec, nb = C.c_uint64(), C.c_uint64()
        _check(_lib.fot_plan_sector_count(self._h, C.c_int(lay), C.byref(sec), C.byref(nb)))
        return sec.value, nb.value

    def inject_lost_flag(self, block: int) -> None:
        """Test hook (fot_plan_inject_lost_flag): lose one block's completion
        flag so that the next run's dependency waits hit their time limit."""
        _check(_lib.fot_plan_inject_lost_flag(self._h, C.c_uint32(block)))

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_plan_destroy(self._h)
            self._h = None


class Graph:
    """`iterations` iterations of a plan captured as one CUDA graph."""

    def __init__(self, plan: Plan, iterations: int, stream=None):
        self.plan = plan
        self._h = C.c_void_p()
        _check(_lib.fot_graph_create(plan.problem._h, plan._h, iterations, _stream_ptr(stream),
                                     C.byref(self._h)))

    def launch(self, stream=None) -> None:
        _check(_lib.fot_graph_launch(self._h, _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_graph_destroy(self._h)
            self._h = None


class Batch:
    """Hierarchical plans of many problems run by ONE persistent launch over a
    (mesh, block colour) tile queue (fot_batch)."""

    def __init__(self, plans: List[Plan]):
        self.plans = list(plans)  # keeps the problems and plans alive
        n = len(self.plans)
        probs = (C.c_void_p * n)(*[pl.problem._h.value for pl in self.plans])
        hs = (C.c_void_p * n)(*[pl._h.value for pl in self.plans])
        self._h = C.c_void_p()
        _check(_lib.fot_batch_create(probs, hs, C.c_uint32(n), C.byref(self._h)))

    def run(self, iterations: int = 1, stream=None) -> None:
        _check(_lib.fot_batch_run(self._h, C.c_uint32(iterations), _stream_ptr(stream)))

    def sync(self, stream=None) -> None:
        _check(_lib.fot_batch_sync(self._h, _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_batch_destroy(self._h)
            self._h = None


class RowList:
    """Distinct rows of point dataset k kept on the device (fot_rowlist):
    gather packs them into a device buffer, scatter_add adds one in."""

    def __init__(self, problem: "Problem", k: int, rows: np.ndarray):
        self.problem = problem
        r = np.ascontiguousarray(rows, dtype=np.uint32)
        self.n = len(r)
        self._h = C.c_void_p()
        _check(_lib.fot_rowlist_create(problem._h, C.c_uint32(k), r.ctypes.data_as(u32p),
                                       C.c_uint32(self.n), C.byref(self._h)))

    def gather(self, dst_ptr: int, stream=None) -> None:
        _check(_lib.fot_rowlist_gather(self._h, C.c_void_p(dst_ptr), _stream_ptr(stream)))

    def scatter_add(self, src_ptr: int, stream=None) -> None:
        _check(_lib.fot_rowlist_scatter_add(self._h, C.c_void_p(src_ptr), _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_rowlist_destroy(self._h)
            self._h = None


class AirfoilDesc(C.Structure):
    _fields_ = [("cell_to_node", u32p), ("n_bedges", C.c_uint32), ("bedge_to_node", u32p),
                ("bedge_to_cell", u32p), ("bound", C.POINTER(C.c_int32)),
                ("qinf", C.c_double * 4), ("cfl", C.c_double)]


class Airfoil:
    """The Airfoil solver iteration around a res_calc problem (fot_airfoil):
    save_soln, then twice adt_calc, res_calc (through a plan), bres_calc and
    update.  Maps are given in the problem's original numbering."""

    def __init__(self, problem: "Problem", cell_to_node: np.ndarray, bedge_to_node: np.ndarray,
                 bedge_to_cell: np.ndarray, bound: np.ndarray, qinf, cfl: float = 0.9):
        self.problem = problem
        self._keep = [np.ascontiguousarray(cell_to_node, dtype=np.uint32),
                      np.ascontiguousarray(bedge_to_node, dtype=np.uint32),
                      np.ascontiguousarray(bedge_to_cell, dtype=np.uint32),
                      np.ascontiguousarray(bound, dtype=np.int32)]
        c2n, b2n, b2c, bnd = self._keep
        desc = AirfoilDesc(c2n.ctypes.data_as(u32p), C.c_uint32(len(b2c)), b2n.ctypes.data_as(u32p),
                           b2c.ctypes.data_as(u32p), bnd.ctypes.data_as(C.POINTER(C.c_int32)),
                           (C.c_double * 4)(*[float(v) for v in qinf]), C.c_double(cfl))
        self._h = C.c_void_p()
        _check(_lib.fot_airfoil_create(problem._h, C.byref(desc), C.byref(self._h)))

    def run(self, plan: Plan, iterations: int = 1, stream=None, rms: bool = True):
        """Runs `iterations` solver iterations with `plan` for res_calc;
        returns the last iteration's rms (synchronising) or None."""
        out = C.c_double()
        _check(_lib.fot_airfoil_run(self._h, plan._h, C.c_uint32(iterations),
                                    C.byref(out) if rms else None, _stream_ptr(stream)))
        return out.value if rms else None

    def graph(self, plan: Plan, iterations: int, stream=None) -> "AirfoilGraph":
        """`iterations` solver iterations captured as one CUDA graph."""
        return AirfoilGraph(self, plan, iterations, stream)

    def rms(self, stream=None) -> float:
        """The last iteration's rms (synchronises the stream)."""
        out = C.c_double()
        _check(_lib.fot_airfoil_get_rms(self._h, C.byref(out), _stream_ptr(stream)))
        return out.value

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_airfoil_destroy(self._h)
            self._h = None


class AirfoilGraph:
    """Airfoil solver iterations captured as one CUDA graph
    (fot_airfoil_graph_create); launch() replays them."""

    def __init__(self, airfoil: Airfoil, plan: Plan, iterations: int, stream=None):
        self.airfoil, self.plan = airfoil, plan
        self._h = C.c_void_p()
        _check(_lib.fot_airfoil_graph_create(airfoil._h, plan._h, C.c_uint32(iterations),
                                             _stream_ptr(stream), C.byref(self._h)))

    def launch(self, stream=None) -> None:
        _check(_lib.fot_graph_launch(self._h, _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_graph_destroy(self._h)
            self._h = None


class Problem:
    """A loop's mesh and datasets on the GPU (the reference's Problem<SOA>)."""

    def __init__(self, loop: int, n_cells: int, n_points: List[int], maps: List[np.ndarray],
                 layout: str = "aos"):
        self.loop = loop
        self.layout = layout
        self.info = loop_info(loop)
        self.n_cells = int(n_cells)
        self.n_points = [int(v) for v in n_points]
        maps = [np.ascontiguousarray(m, dtype=np.uint32) for m in maps]
        np_arr = (C.c_uint32 * len(self.n_points))(*self.n_points)
        ptrs = (u32p * len(maps))(*[m.ctypes.data_as(u32p) for m in maps])
        self._h = C.c_void_p()
        _check(_lib.fot_problem_create(loop, SOA if layout == "soa" else AOS, self.n_cells,
                                       np_arr, ptrs, C.byref(self._h)))

    @classmethod
    def from_mesh(cls, md: "mg.MeshData") -> "Problem":
        p = cls(md.loop, md.n_cells, md.n_points, md.maps, md.layout)
        for k, d in enumerate(md.point_data):
            p.set_point_data(k, d)
        for j, d in enumerate(md.cell_data):
            p.set_cell_data(j, d)
        return p

    # ---- datasets -------------------------------------------------------------
    def point_shape(self, k):
        dim = self.info.point_dim[k]
        return (self.n_points[k], dim) if self.layout == "aos" else (dim, self.n_points[k])

    def point_dtype(self, k):
        return _dtype(self.info.point_type_size[k], self.loop)

    def cell_dtype(self, j):
        return _dtype(self.info.cell_type_size[j], self.loop, j)

    def set_point_data(self, k: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=self.point_dtype(k))
        _check(_lib.fot_set_point_data(self._h, k, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)))

    def set_cell_data(self, j: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=self.cell_dtype(j))
        _check(_lib.fot_set_cell_data(self._h, j, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)))

    def point_weights(self, k: int = 0) -> np.ndarray:
        out = np.empty(self.point_shape(k), dtype=self.point_dtype(k))
        _check(_lib.fot_get_point_data(self._h, k, out.ctypes.data_as(C.c_void_p), C.c_size_t(out.nbytes)))
        return out

    def cell_weights(self, j: int) -> np.ndarray:
        out = np.empty((self.info.cell_dim[j], self.n_cells), dtype=self.cell_dtype(j))
        _check(_lib.fot_get_cell_data(self._h, j, out.ctypes.data_as(C.c_void_p), C.c_size_t(out.nbytes)))
        return out

    def set_layout(self, layout: str) -> None:
        """Convert the point datasets to "aos" or "soa" on the GPU
        (fot_set_layout; the reference's AOStoSOA runs on the host)."""
        _check(_lib.fot_set_layout(self._h, SOA if layout == "soa" else AOS))
        self.layout = layout

    read_point_data = set_point_data
    read_cell_data = set_cell_data

    def point_data_device(self, k: int) -> int:
        p = C.c_void_p()
        _check(_lib.fot_point_data_device(self._h, k, C.byref(p)))
        return p.value

    def cell_data_device(self, j: int) -> int:
        p = C.c_void_p()
        _check(_lib.fot_cell_data_device(self._h, j, C.byref(p)))
        return p.value

    def mapping(self, k: int) -> np.ndarray:
        out = np.empty((self.n_cells, self.info.mesh_dim[k]), dtype=np.uint32)
        _check(_lib.fot_get_mapping(self._h, k, out.ctypes.data_as(u32p)))
        return out

    def point_permutation(self, k: int = 0) -> np.ndarray:
        out = np.empty(self.n_points[k], dtype=np.uint32)
        _check(_lib.fot_get_point_permutation(self._h, k, out.ctypes.data_as(u32p)))
        return out

    @property
    def applied_permutation(self) -> np.ndarray:
        return self.point_permutation(0)

    def cell_order(self) -> np.ndarray:
        out = np.empty(self.n_cells, dtype=np.uint32)
        _check(_lib.fot_get_cell_order(self._h, out.ctypes.data_as(u32p)))
        return out

    def mesh_data(self) -> "mg.MeshData":
        """The problem's current state (mappings and datasets) as MeshData."""
        return mg.MeshData(self.loop, self.n_cells, list(self.n_points),
                           [self.mapping(k) for k in range(self.info.n_mappings)],
                           [self.point_weights(k) for k in range(self.info.n_point_sets)],
                           [self.cell_weights(j) for j in range(self.info.n_cell_sets)],
                           self.layout)

    # ---- statistics (GPU) ----------------------------------------------------------
    def mesh_features(self) -> dict:
        """fot_mesh_features: spread of mapping 0's rows and point degrees."""
        out = (C.c_double * 6)()
        _check(_lib.fot_mesh_features(self._h, out, C.c_int(6)))
        return {"span_max": out[0], "span_mean": out[1],
                "deg_hist": [out[2], out[3], out[4], out[5]]}

    def sector_count(self, cells_per_block: int = 256, layout: Optional[str] = None):
        """The reference's sector model over runs of cells_per_block cells
        (fot_sector_count): (sectors, blocks)."""
        lay = -1 if layout is None else (SOA if layout == "soa" else AOS)
        sec, nb = C.c_uint64(), C.c_uint64()
        _check(_lib.fot_sector_count(self._h, C.c_uint32(cells_per_block), C.c_int(lay),
                                     C.byref(sec), C.byref(nb)))
        return sec.value, nb.value

    # ---- orderings (problem.hpp:439-551) ----------------------------------------
    def reorder(self, order: int = ORDER_GPS, seed: int = 1) -> None:
        _check(_lib.fot_reorder(self._h, order, C.c_uint64(seed)))

    def partition(self, part_size: int, seed: int = 1, tolerance: float = 1.001,
                  method: str = "bisect") -> None:
        """fot_partition_tol: ceil(n_cells / part_size) parts by recursive
        graph bisection ("bisect") or region growing ("grow")."""
        m = {"bisect": PARTITION_BISECT, "grow": PARTITION_GROW}[method]
        _check(_lib.fot_partition_tol(self._h, C.c_uint32(part_size), C.c_float(tolerance), C.c_int(m)))

    def partition_quality(self) -> dict:
        """fot_partition_quality: parts, balance, (part, point) pairs per point
        and the fraction of points shared by parts."""
        out = (C.c_double * 4)()
        _check(_lib.fot_partition_quality(self._h, out, C.c_int(4)))
        return {"parts": int(out[0]), "max_over_mean": out[1], "pairs_per_point": out[2],
                "shared_points": out[3]}

    def reorder_to_partition(self) -> None:
        _check(_lib.fot_reorder_to_partition(self._h))

    def renumber_points(self) -> None:
        _check(_lib.fot_renumber_points(self._h))

    def partition_vector(self) -> np.ndarray:
        out = np.empty(self.n_cells, dtype=np.uint32)
        _check(_lib.fot_get_partition(self._h, out.ctypes.data_as(u32p)))
        return out

    def set_partition(self, part: np.ndarray) -> None:
        a = np.ascontiguousarray(part, dtype=np.uint32)
        _check(_lib.fot_set_partition(self._h, a.ctypes.data_as(u32p)))

    # ---- plans and loop drivers -------------------------------------------------
    def plan(self, exec: int = EXEC_HIER, block_size: int = 256, flags: int = 0) -> Plan:
        return Plan(self, exec, block_size, flags)

    def sync(self, stream=None) -> None:
        _check(_lib.fot_sync(self._h, _stream_ptr(stream)))

    def loop_gpu_cell_centred(self, num: int, aggregate: bool = True) -> Plan:
        """The atomic executor, `num` iterations (problem.hpp:90-194)."""
        plan = self.plan(EXEC_ATOMIC, 256, 0 if aggregate else PLAN_NO_AGGREGATE)
        plan.run(num)
        self.sync()
        return plan

    def loop_gpu_hierarchical(self, num: int, block_size: int = 256,
                              use_partition: bool = False, persistent: bool = True) -> Plan:
        """The hierarchical-colour executor, `num` iterations (problem.hpp:198-339)."""
        plan = self.plan(EXEC_HIER if persistent else EXEC_HIER_LAUNCH, block_size,
                         PLAN_USE_PARTITION if use_partition else 0)
        plan.run(num)
        self.sync()
        return plan

    loopGPUCellCentred = loop_gpu_cell_centred
    loopGPUHierarchical = loop_gpu_hierarchical
    reorderToPartition = reorder_to_partition
    renumberPoints = renumber_points

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.fot_problem_destroy(self._h)
            self._h = None
