"""GPU tests of the partitioned path's device side: row lists
(fot_rowlist_*) against numpy, and a mesh split into parts whose engine
problems run on one GPU with the halo exchange done in process
(halo.exchange_in_process, the same rank-ordered sums as the all-to-all):
the owners' assembled rows equal the serial loop over the whole mesh."""
import datetime
import socket

import numpy as np
import pytest

from cuda_fot_b200 import halo as H
from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal, rel_err

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("loop", ["res_calc", "volna"])
def test_rowlist_gather_scatter(loop, layout):
    import torch
    md = (mg.res_calc(20, 16, 1) if loop == "res_calc" else mg.volna(16, 12, 1)).to_layout(layout)
    p = F().Problem.from_mesh(md)
    d0 = md.point_data[0].copy()
    dim = d0.shape[1] if layout == "aos" else d0.shape[0]
    rng = np.random.default_rng(1)
    rows = rng.choice(md.n_points[0], 37, replace=False).astype(np.uint32)
    vals = rng.standard_normal(d0.shape).astype(d0.dtype)
    p.set_point_data(0, vals)
    rl = F().RowList(p, 0, rows)
    dt = torch.float64 if d0.dtype == np.float64 else torch.float32
    buf = torch.empty(len(rows) * dim, dtype=dt, device="cuda")
    rl.gather(buf.data_ptr())
    torch.cuda.synchronize()
    want = vals[rows] if layout == "aos" else vals[:, rows].T
    assert bitwise_equal(buf.cpu().numpy().reshape(len(rows), dim), want)
    add = rng.standard_normal((len(rows), dim)).astype(d0.dtype)
    src = torch.from_numpy(add.ravel()).cuda()
    rl.scatter_add(src.data_ptr())
    p.sync()
    ref = vals.copy()
    if layout == "aos":
        ref[rows] = ref[rows] + add
    else:
        ref[:, rows] = ref[:, rows] + add.T
    assert bitwise_equal(p.point_weights(0), ref)


def test_rowlist_checks():
    md = mg.res_calc(10, 8, 1)
    p = F().Problem.from_mesh(md)
    with pytest.raises(F().FotError):
        F().RowList(p, 0, np.array([1, 2, 2], np.uint32))
    with pytest.raises(F().FotError):
        F().RowList(p, 0, np.array([md.n_points[0]], np.uint32))
    rl = F().RowList(p, 0, np.array([3, 1], np.uint32))
    p.reorder(F().ORDER_RCM)
    import torch
    buf = torch.empty(8, dtype=torch.float64, device="cuda")
    with pytest.raises(F().FotError) as e:
        rl.gather(buf.data_ptr())
    assert e.value.code == -3  # stale after renumbering


def _partitioned(md, n_parts, exec_, block, flags, order, iters):
    part = np.random.default_rng(5).integers(0, n_parts, md.n_cells)
    lms = H.split_mesh(md, part, n_parts)
    loops = [H.PartitionedLoop(lm, exec_, block, flags, order) for lm in lms]
    for lp in loops:
        lp.plan.run(iters)
    H.exchange_in_process(loops)
    for lp in loops:
        lp.p.sync()
    return H.assemble(md, lms, [lp.result() for lp in loops])


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("loop", ["res_calc", "mini_aero", "lulesh", "volna", "getacc"])
def test_parts_on_one_gpu_equal_the_whole(loop, layout):
    md = {"res_calc": lambda: mg.res_calc(48, 40, 2), "mini_aero": lambda: mg.mini_aero(10, 2, permute=True),
          "lulesh": lambda: mg.lulesh(8, 2, permute=True), "volna": lambda: mg.volna(30, 24, 2),
          "getacc": lambda: mg.getacc(30, 24, 2)}[loop]().to_layout(layout)
    ser = O.serial(md, 3)[0][0]
    tol = 1e-5 if loop == "volna" else 1e-12
    got = _partitioned(md, 3, F().EXEC_ATOMIC, 256, F().PLAN_NO_AGGREGATE, F().ORDER_RCM, 3)
    assert rel_err(got, ser) <= tol
    got = _partitioned(md, 3, F().EXEC_HIER, 128, 0, F().ORDER_GPS, 3)
    assert rel_err(got, ser) <= tol


def test_partitioned_loop_through_a_process_group():
    """One rank (NCCL, world size 1): run() = the loop and an (empty)
    all-to-all; the result is the whole mesh's."""
    import torch.distributed as dist
    md = mg.res_calc(32, 24, 3)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        lms = H.split_mesh(md, np.zeros(md.n_cells, dtype=np.int64), 1)
        lp = H.PartitionedLoop(lms[0], F().EXEC_ATOMIC, 256, 0, F().ORDER_RCM)
        lp.run(2)
        lp.p.sync()
        got = H.assemble(md, lms, [lp.result()])
    finally:
        dist.destroy_process_group()
    assert rel_err(got, O.serial(md, 2)[0][0]) <= 1e-12
