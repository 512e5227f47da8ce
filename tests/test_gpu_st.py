"""GPU parity of the space-time path (krige_st_* C-ABI) against the CPU oracle.

Same bar as the spatial parity tests: identical neighbour sets, estimates and
variances within 1e-9 relative (FP64) and 1e-6 relative (FP32 factorisation
with FP64 refinement), floors 1e-3 * std(z) and 1e-3 * sill.
"""
import numpy as np
import pytest

import bench_workloads as bw
from oracle.oracle import OracleSpaceTime

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "fp32_refine": 1e-6}
PRECISIONS = ["fp64", "fp32_refine"]


def _gpu(**kw):
    from krigekit_b200 import SpaceTimeKriging
    return SpaceTimeKriging(**kw)


def _compare(g, o, zstd, sill, tol):
    nn, inear = g.get_neighbours(1)
    onn = o.nnear[:, 0]
    np.testing.assert_array_equal(nn, onn)
    for ib in range(len(nn)):
        assert np.array_equal(inear[ib, :nn[ib]], o.inear[ib, 0, :nn[ib]]), f"block {ib}"
    e, v = g.get_results()
    oe, ov = o.get_results()
    ee = bw.rel_err(e, oe, 1e-3 * zstd)
    ve = bw.rel_err(v, ov, 1e-3 * sill)
    assert ee.max() <= tol, f"estimate rel err {ee.max():.3e}"
    assert ve.max() <= tol, f"variance rel err {ve.max():.3e}"


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("pad3d", [False, True])
def test_product_sum_blocks(precision, pad3d):
    """Config-5 shape at reduced size: product-sum model, 4 x 4 block support on
    10 % of the targets; 2-D stations, and the same stations written as 3-D with
    z = 0 (the reference engine's form, which the grid search must not grid on z)."""
    w = bw.config5(grid_n=14, ntimes=4, nstations=150, ndays=60)
    nd = 3 if pad3d else 2
    g = bw.apply_st(_gpu(precision=precision, nmin=4), w, pad3d=pad3d)
    g.solve()
    o = bw.apply_st(OracleSpaceTime(ndim=nd, nmin=4), w, pad3d=pad3d)
    o.solve()
    _compare(g, o, w["zstd"], w["sill"], TOL[precision])


def _sum_metric_case(seed=3, nst=120, nday=50):
    rng = np.random.default_rng(seed)
    st = rng.uniform(0, 1, (nst, 2))
    days = np.arange(nday, dtype=np.float64)
    obs = np.column_stack([np.repeat(st, nday, axis=0), np.tile(days, nst)])
    f = bw.cosine_field(rng, 3, 0.3)
    z = f(obs * np.array([1.0, 1.0, 0.02])) + rng.normal(0, 0.05, len(obs))
    g2 = np.column_stack([rng.uniform(0, 1, 300), rng.uniform(0, 1, 300)])
    tt = rng.uniform(0, nday - 1, 300)
    return obs, z, g2, tt


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("sector", [False, True])
def test_sum_metric_joint(precision, sector):
    """Sum-metric model with a bounded transform, temporal structure and joint sills,
    plain and sector search."""
    obs, z, g2, tt = _sum_metric_case()

    def setup(k):
        k.set_st_model(model="sum_metric", transform="exp", at=5.0, time_nugget=0.0, time_sill=1.0)
        k.set_obs(1, obs, z, nmax=12 if sector else 40)
        k.set_vgm(1, 1, "sph", nugget=0.02, sill=0.5, a_major=0.4)
        k.set_vgm(1, 1, "exp", sill=0.3, a_major=0.2)
        k.set_vgm_temporal(1, 1, "exp", nugget=0.0, sill=0.3, at_k=10.0)
        if isinstance(k, OracleSpaceTime):
            k.set_vgm_joint_sills(1, 1, [0.1, 0.05])
        else:
            k.set_vgm_joint_sills(1, 1, 0.1, 0.05)
        k.set_grid(g2, time=tt)
        k.set_search(1, time_at=0.05, sector_search=sector)
        return k

    g = setup(_gpu(precision=precision))
    g.solve()
    o = setup(OracleSpaceTime(ndim=2))
    o.solve()
    _compare(g, o, float(np.std(z)), 1.2, TOL[precision])


def test_st_errors():
    from krigekit_b200 import _lib
    g = _gpu()
    with pytest.raises(RuntimeError, match="sum_metric"):
        g.set_st_model(model="product_sum", transform="lin")
        _lib.call("krige_st_set_st_model", g._h(), b"other", b"lin", 1.0, 0.0, 1.0, 0.0)
    with pytest.raises(RuntimeError, match="time_at"):
        g.set_obs(1, np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]), np.array([1.0, 2.0]))
        g.set_search(1, time_at=0.0)
    g.close()
