"""CPU tests of the Airfoil iteration's oracle (orc_airfoil_run).

The loops around res_calc (save_soln, adt_calc, bres_calc, update) are not
part of the reference, so no reference output pins them; the C restatement is
checked here against an independent pure-Python statement of the same
scheme on small meshes (bit for bit: Python floats are IEEE doubles and
neither side fuses multiply-adds), and for the properties of the scheme:
the layout does not matter, the residual falls as the iteration converges,
and a uniform free stream on a regular mesh is a fixed point."""
import math

import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal

GAM, GM1, EPS = 1.4, 0.4, 0.05


def _flux(x1, x2, q1, q2, adt1, adt2):
    """res_calc's edge flux (res_calc_func.hpp:9-60), increments of cell 1."""
    dx, dy = x1[0] - x2[0], x1[1] - x2[1]
    ri = 1.0 / q1[0]
    p1 = GM1 * (q1[3] - 0.5 * ri * (q1[1] * q1[1] + q1[2] * q1[2]))
    vol1 = ri * (q1[1] * dy - q1[2] * dx)
    ri = 1.0 / q2[0]
    p2 = GM1 * (q2[3] - 0.5 * ri * (q2[1] * q2[1] + q2[2] * q2[2]))
    vol2 = ri * (q2[1] * dy - q2[2] * dx)
    mu = 0.5 * (adt1 + adt2) * EPS
    return [0.5 * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]),
            0.5 * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) + mu * (q1[1] - q2[1]),
            0.5 * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) + mu * (q1[2] - q2[2]),
            0.5 * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) + mu * (q1[3] - q2[3])]


def py_airfoil(md, ex, iters):
    """Pure-Python Airfoil iterations (AOS data), res_calc in edge order."""
    x = [list(r) for r in md.point_data[1]]
    q = [list(r) for r in md.point_data[2]]
    adt = [float(r[0]) for r in md.point_data[3]]
    res = [list(r) for r in md.point_data[0]]
    e2c, e2n = md.maps[0], md.maps[1]
    c2n = ex["cell_to_node"]
    qinf, cfl = [float(v) for v in ex["qinf"]], float(ex["cfl"])
    total = 0.0
    for _ in range(iters):
        qold = [list(r) for r in q]
        for _stage in range(2):
            for c in range(len(q)):
                px = [x[n][0] for n in c2n[c]]
                py = [x[n][1] for n in c2n[c]]
                ri = 1.0 / q[c][0]
                u, v = ri * q[c][1], ri * q[c][2]
                snd = math.sqrt(GAM * GM1 * (ri * q[c][3] - 0.5 * (u * u + v * v)))
                s = 0.0
                for j in range(4):
                    dx = px[(j + 1) & 3] - px[j]
                    dy = py[(j + 1) & 3] - py[j]
                    s += abs(u * dy - v * dx) + snd * math.sqrt(dx * dx + dy * dy)
                adt[c] = s / cfl
            for e in range(len(e2c)):
                a, b = int(e2c[e][0]), int(e2c[e][1])
                f = _flux(x[e2n[e][0]], x[e2n[e][1]], q[a], q[b], adt[a], adt[b])
                for k in range(4):
                    res[a][k] += f[k]
                for k in range(4):
                    res[b][k] += -f[k]
            for e in range(len(ex["bedge_to_cell"])):
                c = int(ex["bedge_to_cell"][e])
                n1, n2 = ex["bedge_to_node"][e]
                dx, dy = x[n1][0] - x[n2][0], x[n1][1] - x[n2][1]
                q1 = q[c]
                ri = 1.0 / q1[0]
                p1 = GM1 * (q1[3] - 0.5 * ri * (q1[1] * q1[1] + q1[2] * q1[2]))
                if ex["bound"][e] == 1:
                    res[c][1] += p1 * dy
                    res[c][2] += -p1 * dx
                else:
                    vol1 = ri * (q1[1] * dy - q1[2] * dx)
                    ri2 = 1.0 / qinf[0]
                    p2 = GM1 * (qinf[3] - 0.5 * ri2 * (qinf[1] * qinf[1] + qinf[2] * qinf[2]))
                    vol2 = ri2 * (qinf[1] * dy - qinf[2] * dx)
                    mu = adt[c] * EPS
                    res[c][0] += 0.5 * (vol1 * q1[0] + vol2 * qinf[0]) + mu * (q1[0] - qinf[0])
                    res[c][1] += 0.5 * (vol1 * q1[1] + p1 * dy + vol2 * qinf[1] + p2 * dy) + mu * (q1[1] - qinf[1])
                    res[c][2] += 0.5 * (vol1 * q1[2] - p1 * dx + vol2 * qinf[2] - p2 * dx) + mu * (q1[2] - qinf[2])
                    res[c][3] += 0.5 * (vol1 * (q1[3] + p1) + vol2 * (qinf[3] + p2)) + mu * (q1[3] - qinf[3])
            total = 0.0
            for c in range(len(q)):
                adti = 1.0 / adt[c]
                for k in range(4):
                    d = adti * res[c][k]
                    q[c][k] = qold[c][k] - d
                    res[c][k] = 0.0
                    total += d * d
    return np.array(q), np.array(adt), math.sqrt(total / len(q))


@pytest.mark.parametrize("shape,iters", [((4, 3), 1), ((6, 5), 3), ((1, 1), 2)])
def test_oracle_matches_python_statement(shape, iters):
    md = mg.res_calc(*shape, 1)
    ex = mg.airfoil_extras(md)
    pd, rms = O.airfoil(md, ex, iters)
    q, adt, prms = py_airfoil(md, ex, iters)
    assert bitwise_equal(pd[2], q)
    assert bitwise_equal(pd[3][:, 0], adt)
    assert rms == prms
    assert not np.any(pd[0])  # update leaves res zeroed


def test_oracle_layouts_agree():
    md = mg.res_calc(20, 16, 2)
    ex = mg.airfoil_extras(md)
    pa, ra = O.airfoil(md, ex, 4)
    ps, rs = O.airfoil(md.to_layout("soa"), ex, 4)
    assert ra == rs
    assert bitwise_equal(pa[2], ps[2].reshape(4, -1).T)


def test_residual_falls():
    md = mg.res_calc(30, 20, 1)
    ex = mg.airfoil_extras(md)
    rms = [O.airfoil(md, ex, n)[1] for n in (1, 10, 60)]
    assert rms[0] > rms[1] > rms[2] > 0


def test_uniform_stream_is_a_fixed_point():
    """On an unjittered grid with q = qinf everywhere and walls parallel to
    the flow, every flux balances: the update is zero to rounding."""
    md = mg.res_calc(8, 6, 1)
    md.point_data[1] = np.round(md.point_data[1])  # node coordinates back on the grid
    ex = mg.airfoil_extras(md)
    md.point_data[2][:] = ex["qinf"]
    pd, rms = O.airfoil(md, ex, 3)
    assert rms < 1e-14
    assert np.abs(pd[2] - ex["qinf"]).max() < 1e-14
