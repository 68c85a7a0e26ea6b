"""The reference's text formats (cuda_fot_b200.textio): every loop's inputs
round-trip exactly in both layouts, values are read as whitespace-separated
tokens like the reference's operator>> readers, and short or malformed files
name the failing row."""
import io

import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from cuda_fot_b200 import textio as tio


def small(loop, layout):
    if loop == mg.RES_CALC:
        return mg.res_calc(7, 5, 3, layout)
    if loop == mg.MINI_AERO:
        return mg.mini_aero(3, 3, layout)
    if loop == mg.LULESH:
        return mg.lulesh(3, 3, layout)
    if loop == mg.VOLNA:
        return mg.volna(6, 4, 3, layout)
    return mg.getacc(6, 4, 3, layout)


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("loop", range(5))
def test_problem_files_round_trip(tmp_path, loop, layout):
    md = small(loop, layout)
    paths = tio.save_mesh_data(md, str(tmp_path))
    back = tio.load_mesh_data(loop, paths["mesh"], paths["point"], paths["cell"], layout)
    assert back.n_cells == md.n_cells and list(back.n_points) == list(md.n_points)
    for a, b in zip(back.maps, md.maps):
        assert np.array_equal(a, b)
    for a, b in zip(back.point_data, md.point_data):
        assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b)
    for a, b in zip(back.cell_data, md.cell_data):
        assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b)


def test_values_are_tokens_not_lines():
    f = io.StringIO("5 3  0 1 1 2\n 2\n3\n")
    n_points, m = tio.read_mesh(f, 2)
    assert n_points == 5 and m.tolist() == [[0, 1], [1, 2], [2, 3]]


def test_short_and_malformed_files_name_the_row():
    with pytest.raises(tio.InputFileError) as e:
        tio.read_point_data(io.StringIO("1 2\n3 4\n5\n"), 3, 2)
    assert e.value.row == 3
    with pytest.raises(tio.InputFileError) as e:
        tio.read_mesh(io.StringIO("4 2\n0 1\n1 x\n"), 2)
    assert e.value.row == 2
    with pytest.raises(tio.InputFileError) as e:
        tio.read_mesh(io.StringIO("4"), 2)
    assert e.value.row == 0
    with pytest.raises(ValueError):
        tio.read_mesh(io.StringIO("2 1\n0 2\n"), 2)  # point 2 of 2 points


def test_partition_and_permutation_round_trip():
    parts = np.array([0, 0, 1, 2, 1, 2, 2], np.uint32)
    f = io.StringIO()
    tio.write_partition(f, 64, parts)
    f.seek(0)
    block, back = tio.read_partition(f, len(parts))
    assert block == 64 and np.array_equal(back, parts)
    perm = np.random.default_rng(1).permutation(11).astype(np.uint32)
    f = io.StringIO()
    tio.write_permutation(f, perm)
    f.seek(0)
    assert np.array_equal(tio.read_permutation(f), perm)
