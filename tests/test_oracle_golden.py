"""Pin the CPU oracle to the reference's golden vectors and known answers.

Every expected value below comes from the reference test-suite or its
committed fixtures (ougx/krigekit tests/*.py, test_data/*.csv); each test
cites the reference test it restates.
"""
import numpy as np
import pandas as pd
import pytest

from conftest import golden
from oracle.oracle import OracleKriging, OracleSpaceTime, calc_rotmat, kdtree_nn

VGM_PC2D = dict(vtype="sph", nugget=0.0, sill=0.12, a_major=5000.0)


def _ok1d(x, z, target, spec, nmax=50):
    k = OracleKriging(ndim=1, nvar=1)
    k.set_obs(1, np.asarray(x, float)[:, None], np.asarray(z, float), nmax=nmax)
    k.set_vgm(1, 1, **spec)
    k.set_grid(np.array([[float(target)]]))
    k.set_search(1)
    k.solve(keep_weights=True)
    e, v = k.get_results()
    return float(e[0]), float(v[0]), k


def test_assembled_system_1d():
    # tests/test_api.py:39-66: matA = [[4,0,1],[0,4,1],[1,1,0]], rhsB = [1.25,1.25,1]
    e, v, k = _ok1d([0.0, 2.0], [1.0, 3.0], 1.0,
                    dict(vtype="sph", nugget=0.0, sill=4.0, a_major=2.0))
    np.testing.assert_allclose(k.weight[0, 0, 0, :2], [0.5, 0.5], rtol=1e-12)
    # tests/test_cokriging.py spherical symmetric case: estimate 2.0, variance 3.5
    assert e == pytest.approx(2.0, rel=1e-12)
    assert v == pytest.approx(3.5, rel=1e-12)


def test_pure_nugget_ok():
    # tests/test_cokriging.py TestAnalyticalBenchmarks: estimate = mean, var = C0(1+1/n)
    spec = dict(vtype="sph", nugget=2.0, sill=0.0, a_major=1.0)
    e, v, _ = _ok1d([0.0, 1.0, 2.0], [1.0, 3.0, 5.0], 10.0, spec)
    assert e == pytest.approx(3.0, rel=1e-12)
    assert v == pytest.approx(2.0 * (1 + 1 / 3), rel=1e-12)


def test_exact_interpolation():
    # tests/test_cokriging.py test_exact_interpolation_no_nugget
    x, z = [0.0, 1.5, 4.0], [2.0, 7.0, 4.0]
    spec = dict(vtype="sph", nugget=0.0, sill=1.0, a_major=6.0)
    for xi, zi in zip(x, z):
        e, v, _ = _ok1d(x, z, xi, spec)
        assert e == pytest.approx(zi, rel=1e-5)
        assert abs(v) < 1e-5


def test_nugget_cokriging():
    # tests/test_cokriging.py test_nugget_cok_*: V estimate 3.0, variance 16/3
    for uvals in ([10.0, 20.0], [1000.0, 2000.0]):
        k = OracleKriging(ndim=1, nvar=2, std_ck=True)
        k.set_obs(1, np.array([[0.0], [1.0], [2.0]]), np.array([1.0, 3.0, 5.0]), nmax=50)
        k.set_obs(2, np.array([[4.0], [5.0]]), np.array(uvals), nmax=50)
        k.set_vgm(1, 1, "sph", nugget=4.0, sill=0.0, a_major=1.0)
        k.set_vgm(2, 2, "sph", nugget=1.0, sill=0.0, a_major=1.0)
        k.set_vgm(1, 2, "sph", nugget=1.5, sill=0.0, a_major=1.0)
        k.set_grid(np.array([[100.0]]))
        k.set_search(1)
        k.set_search(2)
        k.solve()
        e, v = k.get_results()
        assert e[0, 0] == pytest.approx(3.0, rel=1e-9)
        assert v[0, 0, 0] == pytest.approx(16.0 / 3.0, rel=1e-9)


def test_sector_neighbours_2d():
    # tests/test_sector_search.py:20-58 -> neighbours [1, 3, 4, 5]
    obs = np.array([[0.1, 0.1], [0.2, 0.2], [-5.0, 5.0], [-5.0, -5.0], [5.0, -5.0]])
    k = OracleKriging(ndim=2, nvar=1)
    k.set_obs(1, obs, np.array([10.0, 10.0, 20.0, 20.0, 20.0]), nmax=1)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=1.0, a_major=100.0)
    k.set_grid(np.array([[0.0, 0.0]]))
    k.set_search(1, sector_search=True)
    k.solve()
    assert list(k.neighbours(0)) == [1, 3, 4, 5]


def test_sector_neighbours_3d():
    # tests/test_sector_search.py:65-110 -> neighbours [1, 3, 4, 5, 6, 7, 8, 9]
    obs = np.array([[0.1, 0.1, 0.1], [0.2, 0.2, 0.2], [-5, 5, 5], [5, -5, 5], [-5, -5, 5],
                    [5, 5, -5], [-5, 5, -5], [5, -5, -5], [-5, -5, -5]], dtype=float)
    k = OracleKriging(ndim=3, nvar=1)
    k.set_obs(1, obs, np.ones(9) * 10.0, nmax=1)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=1.0, a_major=100.0)
    k.set_grid(np.array([[0.0, 0.0, 0.0]]))
    k.set_search(1, sector_search=True)
    k.solve()
    assert list(k.neighbours(0)) == [1, 3, 4, 5, 6, 7, 8, 9]


def test_spacetime_sector_neighbours():
    # tests/test_sector_search.py:117-160 -> neighbours [1, 3, 4, 5]
    obs = np.array([[0.1, 0.1, 0.0, 0.0], [0.2, 0.2, 0.0, 0.0], [-5.0, 5.0, 0.0, 0.0],
                    [-5.0, -5.0, 0.0, 0.0], [5.0, -5.0, 0.0, 0.0]])
    k = OracleSpaceTime(ndim=3, nvar=1)
    k.set_st_model("sum_metric", "linear", at=10.0)
    k.set_obs(1, obs, np.array([10.0, 10.0, 20.0, 20.0, 20.0]), nmax=1)
    k.set_vgm(1, 1, "sph", nugget=0, sill=0.8, a_major=500, a_minor1=300, a_minor2=100)
    k.set_vgm_temporal(1, 1, vtype="exp", nugget=0, sill=0.5, at_k=10.0)
    k.set_vgm_joint_sills(1, 1, [0.3])
    k.set_grid(np.array([[0.0, 0.0, 0.0]]), np.array([0.0]))
    k.set_search(1, sector_search=True)
    k.solve()
    assert list(k.neighbours(0)) == [1, 3, 4, 5]


def test_grid2d_golden():
    # test_data/grid2d.csv: 4800 OK estimates/variances for pc2d (sph sill 0.12,
    # range 5000, nmax 62).  The fixture was produced with analytic covariance and
    # clipped estimates; with the analytic path the variance matches to print precision.
    pc = pd.read_csv(golden("pc2d.csv"))
    g = pd.read_csv(golden("grid2d.csv"))
    for analytic, vtol in ((True, 1e-9), (False, 1e-7)):
        k = OracleKriging(ndim=2, nvar=1)
        k.analytic = analytic
        k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values, nmax=62)
        k.set_vgm(1, 1, **VGM_PC2D)
        k.set_grid(g[["x", "y"]].values)
        k.set_search(1)
        k.solve()
        e, v = k.get_results()
        assert np.abs(v - g["variance"].values).max() < vtol
        assert np.abs(np.clip(e, 0, 1) - g["estimate"].values).max() < 5e-5


def test_loo_cv_golden():
    # tests/test_variogram.py:148-196: corr > 0.999 and RMSE < 0.01 against pc2d.csv loo-cv
    pc = pd.read_csv(golden("pc2d.csv"))
    k = OracleKriging(ndim=2, nvar=1)
    k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values)
    k.set_vgm(1, 1, **VGM_PC2D)
    k.set_grid_cv()
    k.set_search(1)
    k.solve()
    e, v = k.get_results()
    ref = pc["loo-cv"].values
    assert np.corrcoef(e, ref)[0, 1] > 0.999
    assert np.sqrt(np.mean((e - ref) ** 2)) < 0.01
    assert np.all(v > 0)


def test_block_gq_vs_explicit_nodes():
    # tests/test_bk.py:185-212: GQ blocks equal explicit-node blocks at rtol 1e-5
    pc = pd.read_csv(golden("pc2d.csv"))
    pnt = pd.read_csv(golden("gridblockpnt2d.csv"))
    blk = pd.read_csv(golden("gridblock2d.csv"))
    res = []
    for mode in ("nodes", "gq"):
        k = OracleKriging(ndim=2, nvar=1)
        k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values, nmax=62)
        k.set_vgm(1, 1, **VGM_PC2D)
        if mode == "nodes":
            k.set_grid_block(pnt[["x", "y"]].values, 1, blk["pnts"].values,
                             pointweight=pnt["weight"].values)
        else:
            size = 2.0 * (pnt["x"].max() - blk["x"].iloc[0]) / (2 * 0.4305681558)
            k.set_grid_block(blk[["x", "y"]].values, -4, None, blocksize=np.array([size, size]))
        k.set_search(1)
        k.solve()
        res.append(k.get_results())
    np.testing.assert_allclose(res[0][0], res[1][0], rtol=1e-5)
    np.testing.assert_allclose(res[0][1], res[1][1], rtol=1e-5)


def test_table_matches_analytic():
    # variogram.f90 header: table error < 5e-7 against the analytic model
    rng = np.random.default_rng(7)
    obs = rng.uniform(0, 1, (300, 2))
    z = rng.normal(size=300)
    grid = rng.uniform(0, 1, (50, 2))
    out = []
    for analytic in (False, True):
        k = OracleKriging(ndim=2, nvar=1)
        k.analytic = analytic
        k.set_obs(1, obs, z, nmax=16)
        k.set_vgm(1, 1, "exp", nugget=0.05, sill=1.0, a_major=0.3)
        k.set_grid(grid)
        k.set_search(1)
        k.solve()
        out.append(k.get_results())
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-5


def test_rotmat_azimuth():
    # rotation.f90:51-95: azimuth-only 2-D rotation with anisotropy
    m = calc_rotmat(30.0, 0.0, 0.0, 0.5, 1.0)
    a = np.deg2rad(30.0)
    np.testing.assert_allclose(m[:2, :2], [[np.cos(a) / 0.5, -np.sin(a) / 0.5],
                                          [np.sin(a), np.cos(a)]], rtol=1e-15)


def test_kdtree_exact_knn():
    rng = np.random.default_rng(3)
    data = rng.uniform(0, 1, (2000, 2))
    q = np.array([0.4, 0.6])
    dis, idx = kdtree_nn(data, q, 25, sort=True)
    d2 = ((data - q) ** 2).sum(1)
    assert set(idx - 1) == set(np.argsort(d2)[:25])
    assert np.all(np.diff(dis) >= 0)


# --------------------------------------------------------------------------
# sequential Gaussian simulation (orc_sgsim): the reference's behaviours
# --------------------------------------------------------------------------
_VGM_PC2D = dict(vtype="sph", nugget=0.0, sill=0.12, a_major=5000.0)


def _sgsim_pc2d(path, sample, nsim=1, nmax=20):
    pc = pd.read_csv(golden("pc2d.csv"))
    gr = pd.read_csv(golden("grid2d.csv"))
    o = OracleKriging(ndim=2, nvar=1, nsim=nsim)
    o.set_obs(1, pc[["x", "y"]].values, pc["pc"].values, nmax=nmax)
    o.set_vgm(1, 1, **_VGM_PC2D)
    o.set_grid(gr[["x", "y"]].values)
    o.set_search(1)
    o.set_sim(path, sample)
    return o.solve(), pc, gr


def test_sgsim_reference_regression_case():
    """tests/test_sgsim.py::test_class_interface_with_precomputed_path_sample:
    the stored path and draws give finite realisations within [-5, 5]."""
    path = pd.read_csv(golden("path4800.csv"))["randpath"].values
    sample = pd.read_csv(golden("sample4800.csv"))["sample"].values
    o, _, gr = _sgsim_pc2d(path, sample)
    sims, var = o.get_results()
    assert sims.shape == (len(gr),) and np.isfinite(sims).all()
    assert sims.min() >= -5.0 and sims.max() <= 5.0
    assert (var >= 0.0).all()
    # later targets condition mostly on earlier simulated ones
    assert o.sim_nnear[:, 1].mean() > 15


def test_sgsim_first_target_is_ordinary_kriging():
    """The first visited target sees only the observations: with a zero draw
    its value and variance are the ordinary-kriging estimate and variance."""
    path = pd.read_csv(golden("path4800.csv"))["randpath"].values
    o, pc, gr = _sgsim_pc2d(path, np.zeros(len(path)))
    first = path[0] - 1
    k = OracleKriging(ndim=2, nvar=1)
    k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values, nmax=20)
    k.set_vgm(1, 1, **_VGM_PC2D)
    k.set_grid(gr[["x", "y"]].values[first:first + 1])
    k.set_search(1)
    e, v = k.solve().get_results()
    sims, var = o.get_results()
    assert abs(sims[first] - e[0]) <= 1e-12 * max(1.0, abs(e[0]))
    assert abs(var[first] - v[0]) <= 1e-12
    assert o.sim_nnear[first, 1] == 0


def test_sgsim_grid_on_observations():
    """tests/test_sgsim.py::test_grid_on_observations_no_nan: targets at the
    data reproduce them (co-located simulated targets are dropped)."""
    rng = np.random.default_rng(3)
    coord = rng.uniform(0.0, 100.0, size=(12, 2))
    value = np.exp(rng.normal(0.0, 1.0, size=12))
    o = OracleKriging(ndim=2, nvar=1, nsim=1)
    o.set_obs(1, coord, value, nmax=12)
    o.set_grid(coord.copy())
    o.set_vgm(1, 1, "sph", nugget=0.0, sill=1.0, a_major=40.0)
    o.set_search(1)
    o.set_sim(np.arange(1, 13), rng.normal(0, 1, 12))
    est, _ = o.solve().get_results()
    assert np.isnan(est).sum() == 0
    np.testing.assert_allclose(est, value, rtol=1e-2, atol=1e-2)


def _first_target_vs_kriging(search, obs_kw, nmax=12):
    """SGSIM's first visited target sees only the observations: with a zero
    draw its value and variance equal ordinary kriging under the same search
    (sectors, maxdist)."""
    rng = np.random.default_rng(21)
    obs = rng.uniform(0, 10, (150, 2))
    z = np.sin(obs[:, 0]) + 0.5 * np.cos(obs[:, 1])
    grid = rng.uniform(0, 10, (60, 2))
    path = rng.permutation(len(grid)) + 1
    vgm = dict(vtype="exp", nugget=0.05, sill=1.0, a_major=3.0, a_minor1=1.5, azimuth=20.0)
    o = OracleKriging(ndim=2, nvar=1, nsim=1, anisotropic_search=True)
    o.set_obs(1, obs, z, nmax=nmax, **obs_kw)
    o.set_vgm(1, 1, **vgm)
    o.set_grid(grid)
    o.set_search(1, **search)
    o.set_sim(path, np.zeros(len(grid)))
    sims, var = o.solve().get_results()
    first = path[0] - 1
    k = OracleKriging(ndim=2, nvar=1, anisotropic_search=True)
    k.set_obs(1, obs, z, nmax=nmax, **obs_kw)
    k.set_vgm(1, 1, **vgm)
    k.set_grid(grid[first:first + 1])
    k.set_search(1, **search)
    e, v = k.solve().get_results()
    assert o.sim_nnear[first, 1] == 0
    assert o.sim_nnear[first, 0] == k.nnear[0, 0]
    np.testing.assert_array_equal(o.sim_inear[first, :k.nnear[0, 0]], k.neighbours(0) - 1)
    assert abs(sims[first] - e[0]) <= 1e-12 * max(1.0, abs(e[0]))
    assert abs(var[first] - v[0]) <= 1e-12
    return o, obs, grid


def test_sgsim_sector_search_first_target_and_sector_caps():
    """Sector search in the simulation (kriging.F90:533-553): the first
    target's set is the kriging sector set; every later set holds at most
    four sectors of nmax members, observations and earlier targets together."""
    o, obs, grid = _first_target_vs_kriging(dict(anis1=0.5, azimuth=20.0, sector_search=True), {}, nmax=5)
    path = o.sim_path
    pos = np.empty(len(grid), dtype=int)
    pos[path - 1] = np.arange(len(grid))
    for t in range(len(grid)):
        n = int(o.sim_nnear[t].sum())
        idx = o.sim_inear[t, :n]
        assert n <= 4 * 5
        assert (idx[o.sim_nnear[t, 0]:] >= len(obs)).all() and (idx[:o.sim_nnear[t, 0]] < len(obs)).all()
        assert (idx[o.sim_nnear[t, 0]:] - len(obs) < pos[t]).all()  # only targets visited before
    assert o.sim_nnear[:, 1].max() > 0


def test_sgsim_maxdist_applies_to_observations():
    """maxdist cuts the observation members too (filter_by_maxlag after the
    simulation branch, kriging.F90:660-661): the first target equals
    kriging with the same maxdist, and no member lies beyond it."""
    o, obs, grid = _first_target_vs_kriging(dict(anis1=0.5, azimuth=20.0), dict(maxdist=1.5), nmax=16)
    assert (o.sim_nnear[:, 0] < 16).any()


def test_sgsim_external_drift_first_target_is_ked():
    """External drift in the simulation (kriging.F90:789-794, 936-937): the
    first visited target is kriging with external drift; later systems carry
    the target drift of their simulated members."""
    rng = np.random.default_rng(41)
    obs = rng.uniform(0, 10, (200, 2))
    grid = rng.uniform(0, 10, (120, 2))
    dfun = lambda x: np.column_stack([np.sin(0.4 * x[:, 0]), 0.1 * x[:, 1]])
    z = 0.8 * dfun(obs)[:, 0] - 0.5 * dfun(obs)[:, 1] + 0.2 * np.cos(obs[:, 1])
    path = rng.permutation(len(grid)) + 1
    vgm = dict(vtype="sph", nugget=0.02, sill=0.5, a_major=4.0)

    def setup(k, g):
        k.set_obs(1, obs, z, nmax=14)
        k.set_obs_drift(1, dfun(obs))
        k.set_vgm(1, 1, **vgm)
        k.set_grid(g)
        k.set_grid_drift(dfun(g))
        k.set_search(1)
        return k

    o = setup(OracleKriging(ndim=2, nvar=1, ndrift=2, nsim=1), grid)
    o.set_sim(path, np.zeros(len(grid)))
    sims, var = o.solve().get_results()
    first = path[0] - 1
    k = setup(OracleKriging(ndim=2, nvar=1, ndrift=2), grid[first:first + 1])
    e, v = k.solve().get_results()
    assert abs(sims[first] - e[0]) <= 1e-12 * max(1.0, abs(e[0]))
    assert abs(var[first] - v[0]) <= 1e-12
    assert np.isfinite(sims).all() and o.sim_nnear[:, 1].max() > 0
