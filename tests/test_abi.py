"""CPU checks of the C ABI boundary: the library exports every function that
include/fot.h declares, and the Python binding refuses to run without it."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cuda_fot_b200", "libfot.so")


def declared_functions():
    names = []
    for hdr in ("fot.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:int|const char \*)\s*(fot_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_core_entry_points():
    names = declared_functions()
    for n in ["fot_problem_create", "fot_plan_build", "fot_run", "fot_sync", "fot_reorder",
              "fot_partition", "fot_batch_run", "fot_graph_create", "fot_last_error"]:
        assert n in names


def test_library_exports_every_declared_function():
    if not os.path.exists(LIB):
        subprocess.run(["python", "-m", "cuda_fot_b200.build"], cwd=ROOT, check=True)
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_describe_matches_reference_bindings():
    from cuda_fot_b200 import fot
    info = fot.loop_info(0)
    assert info.n_mappings == 4 and list(info.point_dim)[:4] == [4, 2, 4, 1]
    info = fot.loop_info(1)
    assert list(info.point_dim)[:2] == [5, 28] and info.cell_dim[0] == 12
    info = fot.loop_info(2)
    assert info.mesh_dim[0] == 8 and info.cell_written_mask == 2
    info = fot.loop_info(3)
    assert info.point_type_size[0] == 4 and info.n_cell_sets == 4
    info = fot.loop_info(4)
    assert info.n_mappings == 1 and list(info.cell_dim)[:5] == [4, 1, 4, 4, 4]
    with pytest.raises(fot.FotError):
        fot.loop_info(7)
