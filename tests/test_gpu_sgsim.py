"""Sequential Gaussian simulation on the GPU against the oracle.

The reference simulates the targets one by one along a random path
(set_sim_base, kriging_base.F90:1226-1320; search_neighbors' simulation
branch, kriging.F90:524-612; estimate_block_base + sim_draw_base,
kriging_base.F90:3473-3495).  Given the same path and the same N(0, 1)
draws the result is deterministic, which the reference's own regression
test relies on (tests/test_sgsim.py with test_data/path4800.csv and
sample4800.csv, committed here as tests/golden fixtures).  The GPU solves
every target's system at once and draws level by level; the oracle
(oracle/kk_oracle.c, orc_sgsim) restates the sequential algorithm.  The
values carry rounding from every earlier draw they depend on, so they are
compared at 1e-9 of the field's spread; the conditional variances at the
FP64 bar.
"""
import numpy as np
import pandas as pd
import pytest

import bench_workloads as bw
from conftest import golden
from oracle.oracle import OracleKriging

pytestmark = pytest.mark.gpu

VGM_PC2D = dict(vtype="sph", nugget=0.0, sill=0.12, a_major=5000.0)


def _pc2d():
    pc = pd.read_csv(golden("pc2d.csv"))
    gr = pd.read_csv(golden("grid2d.csv"))
    return pc[["x", "y"]].values, pc["pc"].values, gr[["x", "y"]].values


def _pair(obs, z, grid, vgm, nsim, path, sample, nmax=20, search=None, obs_kw=None, **kw):
    from krigekit_b200 import Kriging
    g = Kriging(ndim=obs.shape[1], nvar=1, nsim=nsim, seed=11, **kw)
    o = OracleKriging(ndim=obs.shape[1], nvar=1, nsim=nsim, **kw)
    for k in (g, o):
        k.set_obs(1, obs, z, nmax=nmax, **(obs_kw or {}))
        k.set_vgm(1, 1, **vgm)
        k.set_grid(grid)
        k.set_search(1, **(search or {}))
    g.set_sim(path, sample)
    o.set_sim(path, sample)
    g.solve()
    o.solve()
    return g, o


def _check(g, o, zspread, nsim):
    nn, inear = g.get_sim_neighbours(o.sim_inear.shape[1])
    np.testing.assert_array_equal(nn, o.sim_nnear)  # observation and simulated members per target
    for t in range(len(nn)):
        k = int(nn[t].sum())
        assert np.array_equal(inear[t, :k], o.sim_inear[t, :k]), f"target {t}"  # system order too
    e, v = g.get_results(squeeze=False)
    oe, ov = o.get_results(squeeze=False)
    e = np.asarray(e).reshape(len(ov), nsim)
    np.testing.assert_allclose(np.asarray(v).ravel(), ov, rtol=1e-9, atol=1e-12)
    err = np.abs(e - oe).max() / zspread
    assert err <= 1e-9, f"realisations differ by {err:.3e} of the spread"
    assert np.isfinite(e).all()
    return e


def test_sgsim_reference_path_and_sample():
    """The reference's deterministic case: pc2d, 4800 targets, nmax 20, the
    stored path and draws."""
    obs, z, grid = _pc2d()
    path = pd.read_csv(golden("path4800.csv"))["randpath"].values
    sample = pd.read_csv(golden("sample4800.csv"))["sample"].values
    g, o = _pair(obs, z, grid, VGM_PC2D, 1, path, sample)
    e = _check(g, o, float(np.ptp(z)), 1)
    cnt = g.gpu_counters()
    assert cnt["sim_one_launch"] == 1 and cnt["sim_levels"] > 1  # every level in one launch
    sims, _ = g.get_results()
    assert sims.shape == (len(grid),)
    sims_m, _ = g.get_results(squeeze=False)
    assert sims_m.shape == (len(grid), 1, 1)
    assert sims.min() >= -5.0 and sims.max() <= 5.0  # the reference test's bound
    np.testing.assert_array_equal(sims, e[:, 0])


@pytest.mark.parametrize("nsim", [3])
def test_sgsim_several_realisations(nsim):
    rng = np.random.default_rng(5)
    obs = rng.uniform(0, 1, (300, 2))
    z = np.sin(6 * obs[:, 0]) + np.cos(4 * obs[:, 1]) + rng.normal(0, 0.1, 300)
    grid = np.column_stack([g.ravel() for g in np.meshgrid((np.arange(40) + 0.5) / 40, (np.arange(30) + 0.5) / 30)])
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, (len(grid), nsim))
    vgm = dict(vtype="exp", nugget=0.02, sill=1.0, a_major=0.3)
    g, o = _pair(obs, z, grid, vgm, nsim, path, sample, nmax=24)
    e = _check(g, o, float(np.ptp(z)), nsim)
    sims, _ = g.get_results()
    assert sims.shape == (len(grid), nsim)
    assert not np.allclose(e[:, 0], e[:, 1])


def test_sgsim_anisotropic_maxdist_and_simple_kriging():
    """Anisotropic search (rotated kd-tree), maxdist on the simulated members,
    simple kriging with a mean (the mean term on the observation weights)."""
    rng = np.random.default_rng(6)
    obs = rng.uniform(0, 10, (200, 2))
    z = np.sin(obs[:, 0]) * np.cos(0.5 * obs[:, 1]) + 2.0
    grid = rng.uniform(0, 10, (900, 2))
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, len(grid))
    vgm = dict(vtype="sph", nugget=0.01, sill=0.5, a_major=4.0, a_minor1=2.0, azimuth=30.0)
    g, o = _pair(obs, z, grid, vgm, 1, path, sample, nmax=16, search=dict(anis1=0.5, azimuth=30.0),
                 obs_kw=dict(maxdist=3.0, sk_mean=2.0), anisotropic_search=True, unbias=0)
    _check(g, o, float(np.ptp(z)), 1)


def test_sgsim_grid_on_observations():
    """The reference's co-location case (test_sgsim.py): a simulated target at
    a datum is dropped from later neighbourhoods, so nothing is singular and
    the data are reproduced."""
    from krigekit_b200 import Kriging
    rng = np.random.default_rng(3)
    coord = rng.uniform(0.0, 100.0, size=(12, 2))
    value = np.exp(rng.normal(0.0, 1.0, size=12))
    k = Kriging(nsim=1, seed=5)
    k.set_obs(ivar=1, coord=coord, value=value, nmax=12)
    k.set_grid(coord=coord.copy())
    k.set_vgm(ivar=1, jvar=1, vtype="sph", nugget=0.0, sill=1.0, a_major=40.0)
    k.set_sim()
    k.set_search()
    k.solve()
    est, _ = k.get_results()
    est = np.asarray(est).reshape(coord.shape[0], -1)[:, 0]
    assert np.isnan(est).sum() == 0
    np.testing.assert_allclose(est, value, rtol=1e-2, atol=1e-2)


def test_sgsim_seed_reproducibility_and_ensemble():
    from krigekit_b200 import ordinary_kriging, sequential_gaussian_simulation
    obs, z, grid = _pc2d()
    a = sequential_gaussian_simulation(obs, z, grid, VGM_PC2D, nsim=1, nmax=20, seed=7)
    b = sequential_gaussian_simulation(obs, z, grid, VGM_PC2D, nsim=1, nmax=20, seed=7)
    c = sequential_gaussian_simulation(obs, z, grid, VGM_PC2D, nsim=1, nmax=20, seed=701)
    np.testing.assert_array_equal(a, b)
    assert not np.allclose(a, c)
    sims = sequential_gaussian_simulation(obs, z, grid, VGM_PC2D, nsim=50, nmax=20, seed=1001)
    assert sims.shape == (len(grid), 50)
    est, _ = ordinary_kriging(obs, z, grid, VGM_PC2D, nmax=20)
    corr = np.corrcoef(sims.mean(axis=1), est)[0, 1]
    assert corr > 0.90, corr


def test_sgsim_errors():
    from krigekit_b200 import Kriging
    obs, z, grid = _pc2d()
    k = Kriging(ndim=2, nvar=2, nsim=1)
    for iv in (1, 2):
        k.set_obs(iv, obs, z, nmax=10)
    for iv, jv in ((1, 1), (1, 2), (2, 2)):
        k.set_vgm(iv, jv, **VGM_PC2D)
    k.set_grid(grid)
    with pytest.raises(RuntimeError, match="co-simulation"):
        k.solve()
    k2 = Kriging(ndim=2, nvar=1, nsim=1)
    k2.set_obs(1, obs, z)
    k2.set_grid(grid)
    with pytest.raises(RuntimeError, match="nmax"):
        k2.set_sim()
    with pytest.raises(RuntimeError, match="mutually exclusive"):
        Kriging(ndim=2, nvar=1, nsim=1, cross_validation=True)


def test_sgsim_lattice_at_table_zone_edges():
    """A 200 x 200 lattice of targets with a spherical range of 50 cells:
    targets 5 cells apart sit at 0.1 of the range, the end of the first
    table zone, where the reference's lookup reads one cell early (the
    fraction of an unclamped index); the GPU's fast covariance must take the
    reference's arithmetic there."""
    w1 = bw.config1(grid_n=200)
    ob = w1["obs"][0]
    rng = np.random.default_rng(9)
    grid = w1["grid"]
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, (len(grid), 2))
    vgm = w1["vgm"][0][2]
    g, o = _pair(ob["coord"], ob["value"], grid, vgm, 2, path, sample, nmax=24)
    _check(g, o, float(np.ptp(ob["value"])), 2)


@pytest.mark.parametrize("ndim", [2, 3])
def test_sgsim_sector_search(ndim):
    """Sector search in the simulation (kriging.F90:533-553): the sorted
    candidates among the observations and earlier targets through the
    sector filter, with maxdist on observations and targets."""
    rng = np.random.default_rng(30 + ndim)
    nobs, nt = (400, 1600) if ndim == 2 else (500, 1200)
    obs = rng.uniform(0, 10, (nobs, ndim))
    z = np.sin(obs[:, 0]) + np.cos(0.7 * obs[:, 1]) + (0.3 * obs[:, 2] if ndim == 3 else 0.0)
    grid = rng.uniform(0, 10, (nt, ndim))
    path = rng.permutation(nt) + 1
    sample = rng.normal(0, 1, nt)
    vgm = dict(vtype="sph", nugget=0.02, sill=1.0, a_major=4.0, a_minor1=2.0, azimuth=35.0)
    search = dict(anis1=0.5, azimuth=35.0, sector_search=True)
    g, o = _pair(obs, z, grid, vgm, 1, path, sample, nmax=6, search=search, obs_kw=dict(maxdist=3.5),
                 anisotropic_search=True)
    _check(g, o, float(np.ptp(z)), 1)
    assert o.sim_nnear[:, 1].max() > 0 and o.sim_nnear.sum(axis=1).max() <= (2 ** ndim) * 6


def test_sgsim_maxdist_on_observations():
    """maxdist cuts observation members as well as simulated ones
    (kriging.F90:660-661), in the kd-tree branch and in the branch where
    every observation and earlier target fits within nmax."""
    rng = np.random.default_rng(12)
    obs = rng.uniform(0, 10, (60, 2))
    z = np.cos(obs[:, 0]) * np.sin(0.5 * obs[:, 1])
    grid = rng.uniform(0, 10, (500, 2))
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, len(grid))
    vgm = dict(vtype="exp", nugget=0.05, sill=1.0, a_major=3.0)
    g, o = _pair(obs, z, grid, vgm, 1, path, sample, nmax=70, obs_kw=dict(maxdist=2.5))
    _check(g, o, float(np.ptp(z)), 1)
    assert (o.sim_nnear[:, 0] < 60).all() and o.sim_nnear[:, 0].min() > 0


def test_sgsim_external_drift():
    """Kriging with two external drifts in the simulation: the simulated
    members carry the target drift at their nodes."""
    rng = np.random.default_rng(43)
    obs = rng.uniform(0, 10, (500, 2))
    grid = rng.uniform(0, 10, (2000, 2))
    dfun = lambda x: np.column_stack([np.sin(0.4 * x[:, 0]), 0.1 * x[:, 1]])
    z = 0.8 * dfun(obs)[:, 0] - 0.5 * dfun(obs)[:, 1] + 0.2 * np.cos(obs[:, 1])
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, (len(grid), 2))
    from krigekit_b200 import Kriging
    g = Kriging(ndim=2, nvar=1, ndrift=2, nsim=2, seed=3)
    o = OracleKriging(ndim=2, nvar=1, ndrift=2, nsim=2)
    for k in (g, o):
        k.set_obs(1, obs, z, nmax=20)
        k.set_obs_drift(1, dfun(obs))
        k.set_vgm(1, 1, vtype="sph", nugget=0.02, sill=0.5, a_major=4.0)
        k.set_grid(grid)
        k.set_grid_drift(dfun(grid))
        k.set_search(1)
        k.set_sim(path, sample)
    g.solve()
    o.solve()
    _check(g, o, float(np.ptp(z)), 2)


def test_sgsim_3d_rangescale_and_local_nugget():
    """3-D simulation with a per-target range scale and local nugget (the
    lags of a target's system scaled by its range scale, its nugget on the
    diagonal of observation and simulated members alike)."""
    from krigekit_b200 import Kriging
    rng = np.random.default_rng(51)
    obs = rng.uniform(0, 5, (400, 3))
    z = np.sin(obs[:, 0]) + np.cos(obs[:, 1]) * 0.5 + 0.2 * obs[:, 2]
    grid = rng.uniform(0, 5, (1500, 3))
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, len(grid))
    rs = rng.uniform(0.7, 1.4, len(grid))
    ln = rng.uniform(0.0, 0.05, len(grid))
    g = Kriging(ndim=3, nvar=1, nsim=1, seed=2)
    o = OracleKriging(ndim=3, nvar=1, nsim=1)
    for k in (g, o):
        k.set_obs(1, obs, z, nmax=18)
        k.set_vgm(1, 1, vtype="exp", nugget=0.05, sill=1.0, a_major=2.0, a_minor1=1.5, a_minor2=1.0, azimuth=15.0)
        k.set_grid(grid, rangescale=rs, localnugget=ln)
        k.set_search(1)
        k.set_sim(path, sample)
    g.solve()
    o.solve()
    _check(g, o, float(np.ptp(z)), 1)


def test_sgsim_one_launch_equals_level_by_level():
    """The one-launch draw (k_sgsim_flow) and the level-by-level launches
    (k_sgsim_level) give the same realisations bit for bit."""
    from krigekit_b200 import Kriging
    obs, z, grid = _pc2d()
    rng = np.random.default_rng(17)
    path = rng.permutation(len(grid)) + 1
    sample = rng.normal(0, 1, (len(grid), 3))
    out = []
    for by_level in (False, True):
        k = Kriging(ndim=2, nvar=1, nsim=3)
        k.set_obs(1, obs, z, nmax=16)
        k.set_vgm(1, 1, **VGM_PC2D)
        k.set_grid(grid)
        k.set_search(1)
        k.set_sim(path, sample)
        k.set_sim_draw(by_level)
        k.solve()
        cnt = k.gpu_counters()
        assert cnt["sim_one_launch"] == (0 if by_level else 1)
        out.append(np.asarray(k.get_results(squeeze=False)[0]).copy())
        k.close()
    np.testing.assert_array_equal(out[0], out[1])
    assert np.isfinite(out[0]).all()
