"""CTA-per-target solve (65..128 equations) and the kernel tuner, against the oracle.

Systems of 65..128 neighbours go to k_solve_block: the warp kernel's register
Cholesky spread over four warps, FP64 in both precision settings.  The
reference solves them like any other system (solver.f90:224-300), so the bar
is the FP64 one: identical neighbour sets, estimates and variances within
1e-9 relative.  The cases cover every covariance path of the assembly kernel
(general, one-variable table, cokriging table pair, space-time), drift
columns, cokriging, the edges 65 and 128, ragged sizes that fill all four
neighbour-count lists, and a global neighbourhood (nmax >= nobs, the
reference's tests/test_ordinary_kriging.py style).  The tuner's runs on a
sample must leave no trace: counters, status bits and results are those of
the chosen kernel alone.
"""
import numpy as np
import pytest

import bench_workloads as bw
from oracle.oracle import OracleKriging

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _gpu(precision="fp64", autotune=0, **kw):
    from krigekit_b200 import Kriging
    k = Kriging(precision=precision, **kw)
    k.set_autotune(autotune)
    return k


def _compare(g, o, w, nvar=1):
    for iv in range(1, nvar + 1):
        nn, inear = g.get_neighbours(iv)
        np.testing.assert_array_equal(nn, o.nnear[:, iv - 1])
        for ib in range(len(nn)):
            assert np.array_equal(inear[ib, :nn[ib]], o.inear[ib, iv - 1, :nn[ib]]), f"block {ib}"
    e, v = g.get_results(squeeze=False)
    oe, ov = o.get_results(squeeze=False)
    e = np.asarray(e).reshape(oe.shape)
    v = np.asarray(v).reshape(ov.shape)
    ee = bw.rel_err(e, oe, 1e-3 * w["zstd"])
    ve = bw.rel_err(v, ov, 1e-3 * w["sill"])
    assert np.nanmax(ee) <= TOL, f"estimate rel err {np.nanmax(ee):.3e}"
    assert np.nanmax(ve) <= TOL, f"variance rel err {np.nanmax(ve):.3e}"
    np.testing.assert_array_equal(np.isnan(e), np.isnan(oe))


def _run(w, precision="fp64", autotune=0, **extra):
    kw = dict(ndim=w["ndim"], nvar=w["nvar"], **w["kw"], **extra)
    g = bw.apply(_gpu(precision, autotune, **kw), w)
    g.solve()
    o = bw.apply(OracleKriging(**kw), w)
    o.solve()
    return g, o


def _npp(g, nvar):
    return sum(g.get_neighbours(iv)[0] for iv in range(1, nvar + 1))


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_block_ordinary_global_neighbourhood(precision):
    """nmax >= nobs: every target uses all 100 observations (global kriging)."""
    w = bw.config1(grid_n=24, nobs=100)
    w["obs"][0].update(nmax=100, maxdist=None)
    g, o = _run(w, precision)
    _compare(g, o, w)
    assert (_npp(g, 1) == 100).all()
    c = g.gpu_counters()
    assert c["bucket_le128"] == 24 * 24 and c["general_list"] == 0, c
    assert c["chol"] == 24 * 24 and c["fp64_resolve"] == 0
    assert g.kernel_plan()["npp<=128"]["kernel"] == "block128"


@pytest.mark.parametrize("nmax", [65, 128])
def test_block_size_edges(nmax):
    w = bw.config1(grid_n=16, nobs=3000)
    w["obs"][0].update(nmax=nmax, maxdist=None)
    g, o = _run(w)
    _compare(g, o, w)
    assert (_npp(g, 1) == nmax).all()
    assert g.gpu_counters()["bucket_le128"] == 16 * 16


def test_block_anisotropic_sector_search():
    """Four sectors of 30 on the table covariance path (up to 120 equations)."""
    w = bw.config2(grid_n=20, nobs=6000, nclusters=8)
    w["obs"][0]["nmax"] = 30
    g, o = _run(w)
    _compare(g, o, w)
    npp = _npp(g, 1)
    assert npp.max() > 64 and npp.max() <= 120


def test_block_external_drift_3d():
    """Kriging with two external drifts in 3-D (five right-hand-side columns)."""
    w = bw.config3(grid_n=(10, 10, 4), nobs=6000)
    w["obs"][0]["nmax"] = 90
    g, o = _run(w)
    _compare(g, o, w)
    assert (_npp(g, 1) == 90).all()


@pytest.mark.parametrize("std_ck", [True, False])
def test_block_cokriging(std_ck):
    """Two variables of 60 neighbours each (120 equations), standardised and
    Isaaks & Srivastava forms, on the two-variable table path."""
    w = bw.config4(grid_n=14, nobs=(800, 3000))
    w["kw"] = dict(std_ck=std_ck)
    for ob in w["obs"]:
        ob["nmax"] = 60
    g, o = _run(w)
    _compare(g, o, w, nvar=2)
    assert (_npp(g, 2) == 120).all()


def test_block_space_time():
    """Space-time product-sum model of 100 neighbours (space-time table path)."""
    w = bw.config5(grid_n=6, ntimes=3, nstations=60, ndays=40)
    w["obs"][0]["nmax"] = 100
    from krigekit_b200 import SpaceTimeKriging
    from oracle.oracle import OracleSpaceTime
    g = SpaceTimeKriging(precision="fp64")
    g.set_autotune(0)
    g = bw.apply_st(g, w, blocks=False)
    g.solve()
    o = bw.apply_st(OracleSpaceTime(ndim=2), w, blocks=False)
    o.solve()
    _compare(g, o, w)
    assert (g.get_neighbours(1)[0] == 100).all()


def test_ragged_sizes_fill_every_list():
    """maxdist leaves 2..200 neighbours: all four lists and both register
    kernel families in one solve."""
    rng = np.random.default_rng(21)
    x = rng.uniform(0, 1, (2500, 2))
    z = bw.cosine_field(rng, 2, 0.2)(x) + rng.normal(0, 0.05, len(x))
    w = dict(ndim=2, nvar=1, kw={}, obs=[dict(coord=x, value=z, nmax=200, maxdist=0.16)],
             vgm=[(1, 1, dict(vtype="exp", nugget=0.03, sill=1.0, a_major=0.3))], search=[dict()],
             grid=rng.uniform(-0.15, 1.15, (900, 2)), zstd=float(np.std(z)), sill=1.03)
    for precision in ("fp64", "fp32_refine"):
        g, o = _run(w, precision)
        if precision == "fp64":
            _compare(g, o, w)
        else:  # the register kernels of at most 64 equations take the FP32 form
            e, _ = g.get_results()
            oe, _ = o.get_results()
            assert np.nanmax(bw.rel_err(e, oe, 1e-3 * w["zstd"])) <= 1e-6
        c = g.gpu_counters()
        npp = _npp(g, 1)
        assert c["bucket_le32"] == ((npp >= 2) & (npp <= 32)).sum() > 0
        assert c["bucket_le64"] == ((npp > 32) & (npp <= 64)).sum() > 0
        assert c["bucket_le128"] == ((npp > 64) & (npp <= 128)).sum() > 0
        assert c["bucket_gt128"] == (npp > 128).sum() > 0
        plan = g.kernel_plan()
        sfx = "" if precision == "fp64" else "_fp32r"
        assert [plan[k]["kernel"] for k in ("npp<=32", "npp<=64", "npp<=128", "npp>128")] == \
            ["warp32" + sfx, "warp64" + sfx, "block128", "general"]


def test_autotune_times_candidates_and_leaves_no_trace():
    """autotune=2 times the candidates of each list long enough to tune on a
    sample (both forms of each warp kernel under precision "auto") and keeps
    the fastest; the sample runs must not show in the
    counters, the status bits or the results (the chosen kernel solves the
    whole list afterwards)."""
    rng = np.random.default_rng(33)
    x = rng.uniform(0, 1, (6000, 2))
    z = bw.cosine_field(rng, 2, 0.2)(x) + rng.normal(0, 0.05, len(x))
    grid = rng.uniform(0, 1, (2600, 2))
    cands = {("npp<=32", "fp64"): {"warp32", "warp64"},
             ("npp<=32", "fp32_refine"): {"warp32_fp32r", "warp64_fp32r"},
             ("npp<=32", "auto"): {"warp32", "warp32_fp32r", "warp64", "warp64_fp32r"},
             ("npp<=64", "fp64"): {"warp64", "block128"},
             ("npp<=64", "fp32_refine"): {"warp64_fp32r", "block128"},
             ("npp<=64", "auto"): {"warp64", "warp64_fp32r", "block128"}}
    for nmax, lst in ((24, "npp<=32"), (48, "npp<=64"), (80, "npp<=128")):
        w = dict(ndim=2, nvar=1, kw={}, obs=[dict(coord=x, value=z, nmax=nmax)],
                 vgm=[(1, 1, dict(vtype="sph", nugget=0.02, sill=1.0, a_major=0.25))], search=[dict()],
                 grid=grid, zstd=float(np.std(z)), sill=1.02)
        for precision in ("fp64", "fp32_refine", "auto"):
            g, o = _run(w, precision, autotune=2)
            plan = g.kernel_plan()[lst]
            assert set(plan["us_per_target"]) == cands.get((lst, precision), {"block128", "general"}), plan
            assert plan["kernel"] == min(plan["us_per_target"], key=plan["us_per_target"].get)
            c = g.gpu_counters()
            assert c["chol"] == len(grid) and c["fail"] == 0 and c["ldlt"] == 0, c
            st = g.get_status()
            assert int(((st & 4) != 0).sum()) == c["fp64_resolve"]
            assert not (st & 8).any()
            if not plan["kernel"].endswith("_fp32r"):
                _compare(g, o, w)
            else:
                e, _ = g.get_results()
                oe, _ = o.get_results()
                assert np.nanmax(bw.rel_err(e, oe, 1e-3 * w["zstd"])) <= 1e-6
            # the next solve of the same signature takes the cached plan
            g2 = bw.apply(_gpu(precision, 1, ndim=2, nvar=1), w)
            g2.solve()
            assert g2.kernel_plan()[lst] == plan
            assert g2.phases()["launches"] < g.phases()["launches"]


def test_block_kernel_beats_general_on_large_systems():
    """The tuner's own timings: a CTA per target is faster than a thread per
    target at 100 equations."""
    rng = np.random.default_rng(34)
    x = rng.uniform(0, 1, (8000, 2))
    z = bw.cosine_field(rng, 2, 0.2)(x)
    w = dict(ndim=2, nvar=1, kw={}, obs=[dict(coord=x, value=z, nmax=100)],
             vgm=[(1, 1, dict(vtype="exp", nugget=0.02, sill=1.0, a_major=0.3))], search=[dict()],
             grid=rng.uniform(0, 1, (4096, 2)), zstd=float(np.std(z)), sill=1.02)
    g = bw.apply(_gpu("fp64", 2, ndim=2, nvar=1), w)
    g.solve()
    us = g.kernel_plan()["npp<=128"]["us_per_target"]
    assert us["block128"] < us["general"], us
