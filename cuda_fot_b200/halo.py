"""Partitioned runs of one mesh over several GPUs (one process per GPU).

The reference runs a mesh on one GPU.  Here the cells of a mesh are split
into parts, one per rank (a partition from ``Problem.partition`` or any
vector of part ids); each rank's problem holds its cells and every point
they touch, in a local numbering.  A point of the incremented set (point
dataset 0) is owned by the lowest rank touching it; the other ranks' copies
are halo rows that start from zero.  After a rank's loop iterations its
halo rows travel to their owners in one all-to-all (``torch.distributed``:
NCCL between GPUs, gloo on the CPU) and are added there in rank order, so
each owner ends with the whole mesh's result for its points.  The loops
never write the datasets they read (only point dataset 0 changes; LULESH's
element volumes belong to the rank holding the element), so no halo data
flows the other way.

* ``split_mesh(md, part, n_ranks)`` -> one ``LocalMesh`` per rank (host,
  deterministic: every rank can compute the whole split itself);
* ``exchange(lm, gather, scatter_add, new_buffer, group)`` -> the halo
  all-to-all of one rank, with the row movement supplied by the caller;
* ``PartitionedLoop`` -> a rank's engine problem, plan and device row lists
  (``fot_rowlist_*``) with ``run(iterations)`` = loop + exchange;
* ``assemble(md, locals, results)`` -> the owners' rows back in the global
  numbering (for checks).
"""
from __future__ import annotations

from contextlib import nullcontext
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import meshgen as mg


@dataclass
class LocalMesh:
    """One rank's part of a mesh.  ``md`` holds the rank's cells (in global
    order) and the points they touch, renumbered per point set in global
    order; its point dataset 0 keeps the global values on owned rows and is
    zero on halo rows.  ``send[o]`` lists the local rows of set 0 owned by
    rank o, ``recv[s]`` the local rows the matching rows of rank s add to
    (both in ascending global id)."""
    rank: int
    md: mg.MeshData
    cells: np.ndarray
    points: List[np.ndarray]
    owned: np.ndarray
    send: Dict[int, np.ndarray] = field(default_factory=dict)
    recv: Dict[int, np.ndarray] = field(default_factory=dict)

    def row_elems(self) -> int:
        d = self.md.point_data[0]
        return d.shape[1] if self.md.layout == "aos" else d.shape[0]


def _rows(arr: np.ndarray, idx: np.ndarray, layout: str) -> np.ndarray:
    return arr[idx] if layout == "aos" else arr[:, idx]


def split_mesh(md: mg.MeshData, part: np.ndarray, n_ranks: int) -> List[LocalMesh]:
    """Split md by the cell -> rank vector `part` (values < n_ranks)."""
    part = np.asarray(part)
    if part.shape != (md.n_cells,) or (part.size and part.max() >= n_ranks):
        raise ValueError("part must give a rank < n_ranks for every cell")
    cells = [np.nonzero(part == r)[0] for r in range(n_ranks)]
    pts = [[np.unique(m[c]) for m in md.maps] for c in cells]
    # owner of each point of set 0: the lowest rank touching it
    owner = np.full(md.n_points[0], -1, dtype=np.int64)
    for r in range(n_ranks):
        p0 = pts[r][0]
        fresh = p0[owner[p0] < 0]
        owner[fresh] = r
    out = []
    for r in range(n_ranks):
        c = cells[r]
        maps = [np.searchsorted(pts[r][k], m[c]).astype(np.uint32) for k, m in enumerate(md.maps)]
        pdata = [np.ascontiguousarray(_rows(d, pts[r][k], md.layout))
                 for k, d in enumerate(md.point_data)]
        owned = owner[pts[r][0]] == r
        halo = np.nonzero(~owned)[0]
        if md.layout == "aos":
            pdata[0][halo] = 0
        else:
            pdata[0][:, halo] = 0
        cdata = [np.ascontiguousarray(d[:, c]) if d.ndim == 2 else np.ascontiguousarray(d[c])
                 for d in md.cell_data]
        lmd = mg.MeshData(md.loop, len(c), [len(p) for p in pts[r]], maps, pdata, cdata,
                          md.layout, dict(md.meta, rank=r, n_ranks=n_ranks))
        lm = LocalMesh(r, lmd, c, pts[r], owned)
        for o in np.unique(owner[pts[r][0][halo]]):
            lm.send[int(o)] = halo[owner[pts[r][0][halo]] == o].astype(np.uint32)
        out.append(lm)
    # the owner's rows for each sender, in the sender's (ascending global) order
    for s, lm in enumerate(out):
        for o, rows in lm.send.items():
            gids = lm.points[0][rows]
            out[o].recv[s] = np.searchsorted(out[o].points[0], gids).astype(np.uint32)
    return out


def exchange(lm: LocalMesh, gather: Callable[[int], "object"], scatter_add: Callable[[int, "object"], None],
             new_buffer: Callable[[int], "object"], group=None) -> None:
    """The halo all-to-all of rank lm.rank: gather(o) returns the packed rows
    this rank sends to owner o (a flat tensor, rows in lm.send[o] order),
    scatter_add(s, t) adds the rows received from rank s (lm.recv[s] order),
    new_buffer(n) makes an empty flat tensor of n elements.  Every rank of
    the group calls it once, in the same step."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    re = lm.row_elems()
    send_counts = [len(lm.send.get(o, ())) * re for o in range(world)]
    recv_counts = [len(lm.recv.get(s, ())) * re for s in range(world)]
    parts = [gather(o) for o in range(world) if send_counts[o]]
    send_buf = torch.cat(parts) if parts else new_buffer(0)
    recv_buf = new_buffer(sum(recv_counts))
    dist.all_to_all_single(recv_buf, send_buf, recv_counts, send_counts, group=group)
    off = 0
    for s in range(world):
        n = recv_counts[s]
        if n:
            scatter_add(s, recv_buf[off:off + n])
        off += n


def assemble(md: mg.MeshData, locals_: List[LocalMesh], results: List[np.ndarray]) -> np.ndarray:
    """Point dataset 0 in the global numbering from each rank's final local
    dataset 0 (owned rows only)."""
    out = np.empty_like(md.point_data[0])
    for lm, res in zip(locals_, results):
        rows = np.nonzero(lm.owned)[0]
        g = lm.points[0][rows]
        if md.layout == "aos":
            out[g] = res[rows]
        else:
            out[:, g] = res[:, rows]
    return out


class PartitionedLoop:
    """A rank's part on its GPU: the engine problem of lm.md, its plan, and
    device row lists of the halo rows it sends and the owned rows it
    receives.  run(k) = k loop iterations, then the halo exchange; `stream`
    is a torch.cuda.Stream or None (torch's current stream)."""

    def __init__(self, lm: LocalMesh, exec: int, block_size: int = 256, flags: int = 0,
                 order: Optional[int] = None, group=None):
        from . import fot as F
        self.F, self.lm, self.group = F, lm, group
        self.p = F.Problem.from_mesh(lm.md)
        if order is not None:
            self.p.reorder(order, seed=1)
        perm = self.p.point_permutation(0)  # local row -> current row
        self.plan = self.p.plan(exec, block_size, flags)
        self.send = {o: F.RowList(self.p, 0, perm[r]) for o, r in lm.send.items()}
        self.recv = {s: F.RowList(self.p, 0, perm[r]) for s, r in lm.recv.items()}
        self.perm = perm

    def run(self, iterations: int, stream=None) -> None:
        import torch
        dt = torch.float64 if self.p.point_dtype(0) == np.float64 else torch.float32
        re = self.lm.row_elems()
        self.plan.run(iterations, stream)

        def gather(o):
            buf = torch.empty(len(self.lm.send[o]) * re, dtype=dt, device="cuda")
            self.send[o].gather(buf.data_ptr(), stream)
            return buf

        def scatter_add(s, t):
            self.recv[s].scatter_add(t.data_ptr(), stream)

        # the collective is ordered after torch's current stream: issue it
        # under the stream the loop and the row kernels run on
        ctx = torch.cuda.stream(stream) if isinstance(stream, torch.cuda.Stream) else nullcontext()
        with ctx:
            exchange(self.lm, gather, scatter_add,
                     lambda n: torch.empty(n, dtype=dt, device="cuda"), self.group)

    def result(self) -> np.ndarray:
        """Point dataset 0 in the local numbering (host)."""
        w = self.p.point_weights(0)
        return w[self.perm] if self.lm.md.layout == "aos" else w[:, self.perm]


def exchange_in_process(loops: List[PartitionedLoop], stream=None) -> None:
    """The halo exchange of parts held by one process (one GPU): for each
    owner, the senders' rows are added in rank order, as ``exchange`` does
    across processes."""
    import torch
    for o, lo in enumerate(loops):
        for s, ls in enumerate(loops):
            if o in ls.lm.send:
                dt = torch.float64 if ls.p.point_dtype(0) == np.float64 else torch.float32
                buf = torch.empty(len(ls.lm.send[o]) * ls.lm.row_elems(), dtype=dt, device="cuda")
                ls.send[o].gather(buf.data_ptr(), stream)
                lo.recv[s].scatter_add(buf.data_ptr(), stream)
