"""GPU parity: the CUDA path through the C-ABI against the CPU oracle.

Neighbour sets must be identical to the oracle's (which restates the
reference kd-tree, its heap tie-breaking and the sector filter); estimates
and variances must agree to 1e-9 relative in FP64 and to 1e-6 relative with
FP32 factorisation + FP64 refinement, using the relative error
|e - e_ref| / max(|e_ref|, floor) with floor = 1e-3 * std(z) for estimates
and 1e-3 * sill for variances.
"""
import numpy as np
import pandas as pd
import pytest

import bench_workloads as bw
from conftest import golden
from oracle.oracle import OracleKriging

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "fp32_refine": 1e-6}
PRECISIONS = ["fp64", "fp32_refine"]


def _gpu(**kw):
    from krigekit_b200 import Kriging
    return Kriging(**kw)


def _run_pair(w, precision, nmin=0, **extra):
    kw = dict(ndim=w["ndim"], nvar=w["nvar"], **w["kw"], **extra)
    g = bw.apply(_gpu(precision=precision, nmin=nmin, **kw), w)
    g.solve()
    o = bw.apply(OracleKriging(nmin=nmin, **kw), w)
    o.solve()
    return g, o


def _check_neighbours(g, o, nvar=1):
    for iv in range(1, nvar + 1):
        nn, inear = g.get_neighbours(iv)
        onn = o.nnear[:, iv - 1]
        np.testing.assert_array_equal(nn, onn)
        for ib in range(len(nn)):
            n = nn[ib]
            assert np.array_equal(inear[ib, :n], o.inear[ib, iv - 1, :n]), f"block {ib} var {iv}"


def _check_values(g, o, w, tol):
    e, v = g.get_results(squeeze=False)
    oe, ov = o.get_results(squeeze=False)
    e = np.asarray(e).reshape(oe.shape)
    v = np.asarray(v).reshape(ov.shape)
    ee = bw.rel_err(e, oe, 1e-3 * w["zstd"])
    ve = bw.rel_err(v, ov, 1e-3 * w["sill"])
    assert ee.max() <= tol, f"estimate rel err {ee.max():.3e}"
    assert ve.max() <= tol, f"variance rel err {ve.max():.3e}"


# ---------------------------------------------------------------- known answers
@pytest.mark.parametrize("precision", PRECISIONS)
def test_symmetric_1d(precision):
    k = _gpu(ndim=1, nvar=1, precision=precision)
    k.set_obs(1, np.array([[0.0], [2.0]]), np.array([1.0, 3.0]), nmax=2)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=4.0, a_major=2.0)
    k.set_grid(np.array([[1.0]]))
    k.set_search(1)
    k.solve()
    e, v = k.get_results()
    assert e[0] == pytest.approx(2.0, rel=1e-12)
    assert v[0] == pytest.approx(3.5, rel=1e-12)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_nugget_cokriging(precision):
    k = _gpu(ndim=1, nvar=2, std_ck=True, precision=precision)
    k.set_obs(1, np.array([[0.0], [1.0], [2.0]]), np.array([1.0, 3.0, 5.0]), nmax=50)
    k.set_obs(2, np.array([[4.0], [5.0]]), np.array([10.0, 20.0]), nmax=50)
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


def test_sector_neighbours_reference_kat():
    # reference tests/test_sector_search.py:20-58
    obs = np.array([[0.1, 0.1], [0.2, 0.2], [-5.0, 5.0], [-5.0, -5.0], [5.0, -5.0]])
    k = _gpu(ndim=2, nvar=1)
    k.set_obs(1, obs, np.array([10.0, 10.0, 20.0, 20.0, 20.0]), nmax=1)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=1.0, a_major=100.0)
    k.set_grid(np.array([[0.0, 0.0]]))
    k.set_search(1, sector_search=True)
    k.solve()
    nn, inear = k.get_neighbours(1)
    assert list(inear[0, :nn[0]]) == [1, 3, 4, 5]


# ---------------------------------------------------------------- golden CSVs
@pytest.mark.parametrize("precision", PRECISIONS)
def test_grid2d_golden(precision):
    pc = pd.read_csv(golden("pc2d.csv"))
    gr = pd.read_csv(golden("grid2d.csv"))
    k = _gpu(ndim=2, nvar=1, precision=precision)
    k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values, nmax=62)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=0.12, a_major=5000.0)
    k.set_grid(gr[["x", "y"]].values)
    k.set_search(1)
    k.solve()
    e, v = k.get_results()
    assert np.abs(v - gr["variance"].values).max() < 1e-7
    assert np.abs(np.clip(e, 0, 1) - gr["estimate"].values).max() < 5e-5


def test_loo_cv_golden():
    pc = pd.read_csv(golden("pc2d.csv"))
    k = _gpu(ndim=2, nvar=1, cross_validation=True)
    k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=0.12, a_major=5000.0)
    k.set_grid_cv()
    k.set_search(1)
    k.solve()
    e, v = k.get_results()
    ref = pc["loo-cv"].values
    assert np.corrcoef(e, ref)[0, 1] > 0.999
    assert np.sqrt(np.mean((e - ref) ** 2)) < 0.01


# ---------------------------------------------------------------- synthetic configs (small)
@pytest.mark.parametrize("precision", PRECISIONS)
def test_config1_small(precision):
    w = bw.config1(grid_n=60)
    g, o = _run_pair(w, precision, nmin=4)
    _check_neighbours(g, o)
    _check_values(g, o, w, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_config2_small_sector(precision):
    w = bw.config2(grid_n=80, nobs=20_000, nclusters=10)
    g, o = _run_pair(w, precision, nmin=4)
    _check_neighbours(g, o)
    _check_values(g, o, w, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_config3_small_ked(precision):
    w = bw.config3(grid_n=(16, 16, 6), nobs=20_000)
    g, o = _run_pair(w, precision, nmin=4)
    _check_neighbours(g, o)
    _check_values(g, o, w, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_config4_small_cokriging(precision):
    w = bw.config4(grid_n=30, nobs=(2_000, 20_000))
    g, o = _run_pair(w, precision, nmin=4)
    _check_neighbours(g, o, nvar=2)
    _check_values(g, o, w, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_cokriging_shared_anisotropy(precision):
    """Linear model of coregionalisation whose structures share one range and
    anisotropy (Level-B tables for vgm(i, j), i <= j; the reference evaluates
    the other orientation analytically, and so does this library)."""
    w = bw.config4(grid_n=30, nobs=(2_000, 20_000))
    vgm = []
    for (i, j), (bn, be) in {(1, 1): (0.05, 0.95), (1, 2): (0.0, 0.665), (2, 2): (0.05, 0.95)}.items():
        vgm.append((i, j, dict(vtype="nug", nugget=bn, sill=0.0, a_major=1.0)))
        vgm.append((i, j, dict(vtype="exp", nugget=0.0, sill=be, a_major=0.3, a_minor1=0.15, azimuth=40.0)))
    w["vgm"] = vgm
    g, o = _run_pair(w, precision, nmin=4)
    _check_neighbours(g, o, nvar=2)
    _check_values(g, o, w, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_nested_ranges_one_variable(precision):
    """Nested structures that differ only in range (Level-A tables whose
    transforms are multiples of one matrix), anisotropic, one variable."""
    w = bw.config1(grid_n=24, nobs=3000)
    w["vgm"] = [(1, 1, dict(vtype="sph", nugget=0.03, sill=0.6, a_major=0.12, a_minor1=0.06, azimuth=25.0)),
                (1, 1, dict(vtype="exp", nugget=0.0, sill=0.4, a_major=0.5, a_minor1=0.25, azimuth=25.0))]
    w["sill"] = 1.03
    g, o = _run_pair(w, precision, nmin=4)
    _check_neighbours(g, o)
    _check_values(g, o, w, TOL[precision])


def test_ties_use_exact_kdtree_order():
    # obs on an integer lattice, targets at lattice-symmetric points: many equal
    # distances at the selection boundary exercise the exact kd-tree replica
    xs, ys = np.meshgrid(np.arange(12.0), np.arange(12.0))
    obs = np.column_stack([xs.ravel(), ys.ravel()])
    z = np.sin(obs[:, 0]) + np.cos(obs[:, 1])
    tg = np.array([[5.5, 5.5], [3.0, 4.0], [6.5, 2.0], [0.0, 0.0], [11.0, 5.5]])
    for sector in (False, True):
        w = dict(ndim=2, nvar=1, kw={}, obs=[dict(coord=obs, value=z, nmax=7 if not sector else 3)],
                 vgm=[(1, 1, dict(vtype="exp", nugget=0.1, sill=1.0, a_major=6.0))],
                 search=[dict(sector_search=sector)], grid=tg, zstd=float(np.std(z)), sill=1.1)
        g, o = _run_pair(w, "fp64")
        _check_neighbours(g, o)
        _check_values(g, o, w, 1e-9)


@pytest.mark.parametrize("sector", [False, True])
def test_ties_lattice_grid(sector):
    """A 60 x 60 lattice of observations and 7 081 targets on the lattice
    points and the cell centres: every target has equal distances at its
    selection boundary, so most of them go through the kd-tree replica."""
    xs, ys = np.meshgrid(np.arange(60.0), np.arange(60.0))
    obs = np.column_stack([xs.ravel(), ys.ravel()])
    z = np.sin(0.3 * obs[:, 0]) + np.cos(0.2 * obs[:, 1])
    cx, cy = np.meshgrid(np.arange(59.0) + 0.5, np.arange(59.0) + 0.5)
    tg = np.vstack([obs, np.column_stack([cx.ravel(), cy.ravel()])])
    w = dict(ndim=2, nvar=1, kw={}, obs=[dict(coord=obs, value=z, nmax=7 if not sector else 3)],
             vgm=[(1, 1, dict(vtype="exp", nugget=0.1, sill=1.0, a_major=6.0))],
             search=[dict(sector_search=sector)], grid=tg, zstd=float(np.std(z)), sill=1.1)
    g, o = _run_pair(w, "fp64")
    _check_neighbours(g, o)
    _check_values(g, o, w, 1e-9)
    assert g.gpu_counters()["search_redo"][0] > len(tg) // 4
