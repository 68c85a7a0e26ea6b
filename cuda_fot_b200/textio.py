"""The reference's text formats for meshes, datasets, partitions and
permutations, so that meshes prepared for the reference's drivers load into
the engine and results can be compared with the reference's tools.

* mesh file (one per mapping; Mesh(istreams, mesh_dim), mesh.hpp:56-98): a
  first line "num_points num_cells", then one line per cell with its
  mesh_dim point numbers;
* point data (Problem::readPointData / writePointData, problem.hpp:583-616):
  one line per point with its dim values, point-major in the file whatever
  the in-memory layout;
* cell data (Problem::readCellData, problem.hpp:618-632): one line per cell
  with its dim values (held component-major, SOA, in memory);
* partition (Problem::readPartition / writePartition, problem.hpp:553-582): a
  first line with the block size, then one part number per cell;
* permutation (writePermutation, problem.hpp:675-681): one number per line.

Readers take whitespace-separated values, as the reference's operator>>
readers do, and raise InputFileError naming the file and the first row that
is short or malformed (the reference throws InvalidInputFile with the same
information).  Writers print floating-point values with 17 significant
digits, so that a round trip is exact.
"""
from __future__ import annotations

import os
from typing import List, Optional, Sequence, TextIO, Tuple, Union

import numpy as np

from . import meshgen as mg

PathOrFile = Union[str, os.PathLike, TextIO]


class InputFileError(ValueError):
    """A file ended early or held something that is not a number.  `row`
    counts the values' rows from 1 (the header, where there is one, is row
    0), as the reference's InvalidInputFile does."""

    def __init__(self, what: str, name: str, row: int):
        super().__init__(f"invalid {what} file {name!r}: row {row} is missing or malformed")
        self.what, self.name, self.row = what, name, row


def _open(f: PathOrFile, mode: str):
    if hasattr(f, "read") or hasattr(f, "write"):
        return f, False
    return open(f, mode), True


def _name(f: PathOrFile) -> str:
    return str(getattr(f, "name", f))


def _read_tokens(f: PathOrFile) -> List[str]:
    """Whitespace-separated tokens: the reference's readers take values with
    operator>>, so line breaks carry no meaning."""
    fh, own = _open(f, "r")
    try:
        return fh.read().split()
    finally:
        if own:
            fh.close()


def _take(tok: List[str], first: int, n: int, dim: int, dtype, what: str, name: str,
          row0: int) -> np.ndarray:
    """n rows of dim values from tokens[first:]; row numbers start at row0."""
    need = n * dim
    have = max(0, min(len(tok) - first, need))
    try:
        vals = np.array(tok[first:first + have], dtype=dtype)
    except ValueError:
        # locate the first value that does not parse
        for i in range(have):
            try:
                np.array([tok[first + i]], dtype=dtype)
            except ValueError:
                raise InputFileError(what, name, row0 + i // dim) from None
        raise
    if have < need:
        raise InputFileError(what, name, row0 + have // dim)
    return vals.reshape(n, dim)


# ---- meshes --------------------------------------------------------------------
def read_mesh(f: PathOrFile, mesh_dim: int) -> Tuple[int, np.ndarray]:
    """(num_points, mapping of shape (num_cells, mesh_dim), uint32)."""
    tok = _read_tokens(f)
    if len(tok) < 2:
        raise InputFileError("mesh", _name(f), 0)
    try:
        n_points, n_cells = int(tok[0]), int(tok[1])
    except ValueError:
        raise InputFileError("mesh", _name(f), 0) from None
    m = _take(tok, 2, n_cells, mesh_dim, np.int64, "mesh", _name(f), 1)
    if m.size and (m.min() < 0 or m.max() >= n_points):
        raise ValueError(f"mesh file {_name(f)!r}: point number out of range (0..{n_points - 1})")
    return n_points, m.astype(np.uint32)


def write_mesh(f: PathOrFile, mapping: np.ndarray, n_points: int) -> None:
    m = np.asarray(mapping)
    fh, own = _open(f, "w")
    try:
        fh.write(f"{n_points} {m.shape[0]}\n")
        np.savetxt(fh, m, fmt="%d")
    finally:
        if own:
            fh.close()


# ---- datasets ------------------------------------------------------------------
def read_point_data(f: PathOrFile, n_points: int, dim: int, dtype=np.float64) -> np.ndarray:
    """Point-major (n_points, dim) array.  Stricter than the reference, whose
    reader leaves the rest of the dataset untouched when the file ends early:
    a short file is an error here."""
    return _take(_read_tokens(f), 0, n_points, dim, dtype, "point data", _name(f), 1)


def read_cell_data(f: PathOrFile, n_cells: int, dim: int, dtype=np.float64) -> np.ndarray:
    """Component-major (dim, n_cells) array, the engine's cell-data layout."""
    rows = _take(_read_tokens(f), 0, n_cells, dim, dtype, "cell data", _name(f), 1)
    return np.ascontiguousarray(rows.T)


def _fmt(dtype) -> str:
    if np.issubdtype(dtype, np.integer):
        return "%d"
    return "%.17g" if np.dtype(dtype).itemsize == 8 else "%.9g"


def write_point_data(f: PathOrFile, data: np.ndarray, layout: str = "aos") -> None:
    """Rows of point values; `data` is (n, dim) for AOS or (dim, n) for SOA."""
    d = np.asarray(data)
    rows = d.T if layout == "soa" else d
    fh, own = _open(f, "w")
    try:
        np.savetxt(fh, rows.reshape(rows.shape[0], -1), fmt=_fmt(d.dtype))
    finally:
        if own:
            fh.close()


def write_cell_data(f: PathOrFile, data: np.ndarray) -> None:
    """Rows of cell values from a component-major (dim, n_cells) array."""
    d = np.asarray(data)
    fh, own = _open(f, "w")
    try:
        np.savetxt(fh, d.T.reshape(d.shape[1], -1), fmt=_fmt(d.dtype))
    finally:
        if own:
            fh.close()


# ---- partitions and permutations ----------------------------------------------------
def read_partition(f: PathOrFile, n_cells: int) -> Tuple[int, np.ndarray]:
    """(block size recorded in the file, part number of each cell)."""
    tok = _read_tokens(f)
    if not tok:
        raise InputFileError("partition", _name(f), 0)
    try:
        block = int(tok[0])
    except ValueError:
        raise InputFileError("partition", _name(f), 0) from None
    parts = _take(tok, 1, n_cells, 1, np.int64, "partition", _name(f), 1)[:, 0]
    return block, parts.astype(np.uint32)


def write_partition(f: PathOrFile, block_size: int, parts: np.ndarray) -> None:
    fh, own = _open(f, "w")
    try:
        fh.write(f"{block_size}\n")
        np.savetxt(fh, np.asarray(parts).reshape(-1, 1), fmt="%d")
    finally:
        if own:
            fh.close()


def read_permutation(f: PathOrFile, n: Optional[int] = None) -> np.ndarray:
    tok = _read_tokens(f)
    n = len(tok) if n is None else n
    return _take(tok, 0, n, 1, np.int64, "permutation", _name(f), 1)[:, 0].astype(np.uint32)


def write_permutation(f: PathOrFile, perm: np.ndarray) -> None:
    fh, own = _open(f, "w")
    try:
        np.savetxt(fh, np.asarray(perm).reshape(-1, 1), fmt="%d")
    finally:
        if own:
            fh.close()


# ---- whole problems -----------------------------------------------------------------
def load_mesh_data(loop: int, mesh_files: Sequence[PathOrFile], point_files: Sequence[PathOrFile],
                   cell_files: Sequence[PathOrFile] = (), layout: str = "aos") -> mg.MeshData:
    """A MeshData (cuda_fot_b200.meshgen) from the reference's input files of
    one loop, in the order of its driver's initProblem: one mesh file and one
    point-data file per mapping, one file per cell dataset."""
    from . import fot as F
    info = F.loop_info(loop)
    if len(mesh_files) != info.n_mappings or len(point_files) != info.n_point_sets:
        raise ValueError(f"{mg.LOOP_NAMES[loop]} needs {info.n_mappings} mesh and point-data files")
    if len(cell_files) != info.n_cell_sets:
        raise ValueError(f"{mg.LOOP_NAMES[loop]} needs {info.n_cell_sets} cell-data files")
    n_points, maps = [], []
    for k, f in enumerate(mesh_files):
        npk, m = read_mesh(f, info.mesh_dim[k])
        if maps and m.shape[0] != maps[0].shape[0]:
            raise ValueError(f"mesh file {_name(f)!r}: {m.shape[0]} cells, the first mesh has {maps[0].shape[0]}")
        n_points.append(npk)
        maps.append(m)
    n_cells = maps[0].shape[0]
    pd = []
    for k, f in enumerate(point_files):
        dt = F._dtype(info.point_type_size[k], loop)
        d = read_point_data(f, n_points[k], info.point_dim[k], dt)
        pd.append(np.ascontiguousarray(d.T) if layout == "soa" else d)
    cd = []
    for j, f in enumerate(cell_files):
        dt = F._dtype(info.cell_type_size[j], loop, j)
        cd.append(read_cell_data(f, n_cells, info.cell_dim[j], dt))
    return mg.MeshData(loop, n_cells, n_points, maps, pd, cd, layout)


def save_mesh_data(md: mg.MeshData, directory: str, names: Optional[Sequence[str]] = None) -> dict:
    """Write a MeshData as the reference's input files: mesh_<name> and
    data_<name> per mapping, cell_data_<j> per cell dataset.  Returns the
    paths by kind."""
    os.makedirs(directory, exist_ok=True)
    names = list(names) if names else [str(k) for k in range(len(md.maps))]
    out = {"mesh": [], "point": [], "cell": []}
    for k, m in enumerate(md.maps):
        p = os.path.join(directory, f"mesh_{names[k]}")
        write_mesh(p, m, md.n_points[k])
        out["mesh"].append(p)
        p = os.path.join(directory, f"data_{names[k]}")
        write_point_data(p, md.point_data[k], md.layout)
        out["point"].append(p)
    for j, d in enumerate(md.cell_data):
        p = os.path.join(directory, f"cell_data_{j}")
        write_cell_data(p, d)
        out["cell"].append(p)
    return out
