"""The C++ drop-in (include/fot_problem.hpp): a res_calc driver written
against the reference's Problem API reads the reference's text inputs,
optionally reorders and partitions, runs the engine's loops and writes the
un-permuted result, which must match the oracle's serial loop."""
import os
import subprocess

import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from cuda_fot_b200 import textio
from oracle import oracle_py as O
from tests.helpers import rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_inputs(md, d):
    # the reference's res_calc input files: mesh_<name> and data_<name>
    textio.save_mesh_data(md, d, ["res", "x", "q", "adt"])


@pytest.fixture(scope="module", params=["aos", "soa"])
def driver(request, tmp_path_factory):
    out = tmp_path_factory.mktemp("shim") / f"shim_res_calc_{request.param}"
    lib = os.path.join(ROOT, "cuda_fot_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    "-DSHIM_SOA=%d" % (request.param == "soa"),
                    os.path.join(ROOT, "tests", "cpp", "shim_res_calc.cpp"), "-o", str(out),
                    "-L" + lib, "-lfot", "-Wl,-rpath," + lib], check=True)
    return str(out)


@pytest.mark.gpu
@pytest.mark.parametrize("exec_,reorder", [("hier", "0"), ("global", "0"), ("hier", "1"),
                                           ("global", "1")])
def test_reference_style_driver(driver, tmp_path, exec_, reorder):
    md = mg.res_calc(40, 30, seed=2)
    write_inputs(md, str(tmp_path))
    out = tmp_path / "result"
    r = subprocess.run([driver, str(tmp_path), "3", exec_, reorder, str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(out)
    ser, _ = O.serial(md, 3)
    # the text round trip keeps 17 significant digits
    assert rel_err(got, ser[0]) <= 1e-12
