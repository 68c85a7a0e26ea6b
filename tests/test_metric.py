"""The benchmark metric's definition and the cost model's pure host helpers.

Unique (algorithmic) bytes per iteration of the three benchmark meshes:
every indirectly read dataset once, the incremented dataset read and written,
every direct dataset once, every distinct mapping once -- res_calc 1000^2
152.0 MB, mini_aero 128^3 1,286.7 MB, LULESH 96^3 122.3 MB.  Group-centred
training targets and corpus merging are checked on small arrays."""
import json

import numpy as np

from cuda_fot_b200 import meshgen as mg


def test_unique_bytes_of_the_benchmark_meshes():
    assert mg.res_calc(1000, 1000, 1).unique_bytes() == 152_000_016
    assert round(mg.lulesh(96, 1, permute=True).unique_bytes() / 1e6, 1) == 122.3
    assert round(mg.mini_aero(128, 1, permute=True).unique_bytes() / 1e6, 1) == 1286.7


def test_centred_targets_remove_each_groups_mean():
    from cuda_fot_b200 import costmodel as CM
    y = np.array([1.0, 3.0, 10.0, 11.0, 12.0], np.float32)
    g = np.array([0, 0, 1, 1, 1])
    t = CM.centred_targets(y, g)
    assert np.allclose(t, [-1, 1, -1, 0, 1])


def test_merge_renumbers_groups(tmp_path):
    from cuda_fot_b200 import costmodel as CM
    paths = []
    for s in range(2):
        info = [{"gid": 0, "seed": s + 1}, {"gid": 1, "seed": s + 1}]
        d = {"X": np.full((3, CM.N_FEATURES), s, np.float32), "y": np.arange(3, dtype=np.float32),
             "seconds": np.ones(3), "group": np.array([0, 1, 1], np.int32),
             "label": np.array(["a", "b", "c"]), "info": json.dumps(info)}
        p = tmp_path / f"s{s}.npz"
        np.savez_compressed(p, **d)
        paths.append(str(p))
    m = CM.merge(paths, str(tmp_path / "all.npz"))
    assert m["group"].tolist() == [0, 1, 1, 2, 3, 3]
    info = json.loads(str(m["info"]))
    assert [e["gid"] for e in info] == [0, 1, 2, 3] and [e["seed"] for e in info] == [1, 1, 2, 2]
