"""GPU parity on edge cases of the solve path, against the CPU oracle.

Sparse neighbourhoods (maxdist leaves targets with 0, 1 or a few neighbours,
with and without nmin), neighbourhoods above 64 (the CTA-per-target and the
general kernel), simple
kriging, Gauss-quadrature blocks, 3-D sector search, per-target range scale
and local nugget, 1-D kriging, and the error raised for duplicate
observations.  Same bar as the other parity tests: identical neighbour sets,
estimates and variances within 1e-9 relative (FP64) and 1e-6 (FP32
factorisation with FP64 refinement), floors 1e-3 * std(z) and 1e-3 * sill.
"""
import numpy as np
import pytest

import bench_workloads as bw
from oracle.oracle import OracleKriging

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "fp32_refine": 1e-6}
PRECISIONS = ["fp64", "fp32_refine"]


def _pair(precision, setup, **kw):
    from krigekit_b200 import Kriging
    g = setup(Kriging(precision=precision, **kw))
    g.solve()
    o = setup(OracleKriging(**kw))
    o.solve()
    return g, o


def _check(g, o, zstd, sill, tol, nvar=1):
    for iv in range(1, nvar + 1):
        nn, inear = g.get_neighbours(iv)
        np.testing.assert_array_equal(nn, o.nnear[:, iv - 1])
        for ib in range(len(nn)):
            assert np.array_equal(inear[ib, :nn[ib]], o.inear[ib, iv - 1, :nn[ib]]), f"block {ib}"
    e, v = g.get_results()
    oe, ov = o.get_results()
    ee = bw.rel_err(e, oe, 1e-3 * zstd)
    ve = bw.rel_err(v, ov, 1e-3 * sill)
    assert ee.max() <= tol, f"estimate rel err {ee.max():.3e}"
    assert ve.max() <= tol, f"variance rel err {ve.max():.3e}"
    return e


def _field(seed, n, ndim=2):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, ndim))
    f = bw.cosine_field(rng, ndim, 0.2)
    return x, f(x) + rng.normal(0, 0.05, n)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("nmin", [0, 3])
def test_sparse_neighbourhoods(precision, nmin):
    x, z = _field(11, 300)
    grid = np.column_stack([g.ravel() for g in np.meshgrid(np.linspace(0, 1, 25), np.linspace(0, 1, 25))])

    def setup(k):
        k.set_obs(1, x, z, nmax=16, maxdist=0.06)
        k.set_vgm(1, 1, "sph", nugget=0.05, sill=1.0, a_major=0.3)
        k.set_grid(grid)
        k.set_search(1)
        return k

    g, o = _pair(precision, setup, ndim=2, nvar=1, nmin=nmin)
    e = _check(g, o, float(np.std(z)), 1.05, TOL[precision])
    nn, _ = g.get_neighbours(1)
    assert (nn == 0).any() and (nn == 1).any() and (nn >= 4).any()
    # fewer than max(2, nmin) neighbours: NaN
    assert np.isnan(e[nn < max(2, nmin)]).all()
    assert np.isfinite(e[nn >= max(2, nmin)]).all()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("nmax", [100, 150])
def test_large_neighbourhood(precision, nmax):
    """100 neighbours: the CTA-per-target kernel; 150: the general kernel."""
    x, z = _field(12, 4000)
    grid = np.random.default_rng(5).uniform(0.1, 0.9, (300, 2))

    def setup(k):
        k.set_obs(1, x, z, nmax=nmax)
        k.set_vgm(1, 1, "exp", nugget=0.02, sill=1.0, a_major=0.2)
        k.set_grid(grid)
        k.set_search(1)
        return k

    g, o = _pair(precision, setup, ndim=2, nvar=1)
    _check(g, o, float(np.std(z)), 1.02, TOL[precision])
    assert (g.get_neighbours(1)[0] == nmax).all()
    c = g.gpu_counters()
    assert c["bucket_le128" if nmax <= 128 else "bucket_gt128"] == len(grid), c


@pytest.mark.parametrize("precision", PRECISIONS)
def test_simple_kriging(precision):
    x, z = _field(13, 2000)
    grid = np.random.default_rng(6).uniform(0, 1, (400, 2))

    def setup(k):
        k.set_obs(1, x, z, nmax=24, sk_mean=0.1)
        k.set_vgm(1, 1, "gau", nugget=0.01, sill=0.9, a_major=0.15)
        k.set_grid(grid)
        k.set_search(1)
        return k

    g, o = _pair(precision, setup, ndim=2, nvar=1, unbias=0)
    _check(g, o, float(np.std(z)), 0.91, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_gauss_quadrature_blocks(precision):
    x, z = _field(14, 2000)
    centres = np.random.default_rng(7).uniform(0.05, 0.95, (200, 2))

    def setup(k):
        k.set_obs(1, x, z, nmax=20)
        k.set_vgm(1, 1, "sph", nugget=0.05, sill=1.0, a_major=0.25)
        k.set_grid_block(centres, -4, None, blocksize=[0.04, 0.02])
        k.set_search(1)
        return k

    g, o = _pair(precision, setup, ndim=2, nvar=1)
    _check(g, o, float(np.std(z)), 1.05, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_sector_search_3d(precision):
    x, z = _field(15, 6000, ndim=3)
    grid = np.random.default_rng(8).uniform(0.1, 0.9, (300, 3))

    def setup(k):
        k.set_obs(1, x, z, nmax=6)
        k.set_vgm(1, 1, "exp", nugget=0.02, sill=1.0, a_major=0.3, a_minor1=0.2, a_minor2=0.1, azimuth=20.0)
        k.set_grid(grid)
        k.set_search(1, anis1=0.7, anis2=0.4, azimuth=20.0, sector_search=True)
        return k

    g, o = _pair(precision, setup, ndim=3, nvar=1, anisotropic_search=True)
    _check(g, o, float(np.std(z)), 1.02, TOL[precision])


def test_sector_total_beyond_warp_buffers():
    """3-D sector search with 8 x 48 neighbours: more than the warp search
    keeps, so every target takes the exact kd-tree path (and the general
    kernel, 384 > 64 rows)."""
    x, z = _field(18, 5000, ndim=3)
    grid = np.random.default_rng(10).uniform(0.2, 0.8, (40, 3))

    def setup(k):
        k.set_obs(1, x, z, nmax=48)
        k.set_vgm(1, 1, "exp", nugget=0.05, sill=1.0, a_major=0.4)
        k.set_grid(grid)
        k.set_search(1, sector_search=True)
        return k

    g, o = _pair("fp64", setup, ndim=3, nvar=1)
    _check(g, o, float(np.std(z)), 1.05, TOL["fp64"])
    assert g.gpu_stats()["search_redo"] == len(grid)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rangescale_and_local_nugget(precision):
    x, z = _field(16, 2000)
    rng = np.random.default_rng(9)
    grid = rng.uniform(0, 1, (300, 2))
    rs = rng.uniform(0.5, 2.0, 300)
    ln = rng.uniform(0.0, 0.1, 300)

    def setup(k):
        k.set_obs(1, x, z, nmax=20)
        k.set_vgm(1, 1, "exp", nugget=0.02, sill=1.0, a_major=0.2)
        k.set_grid(grid, rangescale=rs, localnugget=ln)
        k.set_search(1)
        return k

    g, o = _pair(precision, setup, ndim=2, nvar=1)
    _check(g, o, float(np.std(z)), 1.12, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_one_dimension(precision):
    x, z = _field(17, 500, ndim=1)
    grid = np.linspace(0, 1, 301).reshape(-1, 1)

    def setup(k):
        k.set_obs(1, x, z, nmax=12)
        k.set_vgm(1, 1, "sph", nugget=0.01, sill=1.0, a_major=0.1)
        k.set_grid(grid)
        k.set_search(1)
        return k

    g, o = _pair(precision, setup, ndim=1, nvar=1)
    _check(g, o, float(np.std(z)), 1.01, TOL[precision])


def test_duplicate_observations_raise():
    from krigekit_b200 import Kriging
    x = np.array([[0.1, 0.2], [0.3, 0.4], [0.1, 0.2]])
    k = Kriging(ndim=2, nvar=1)
    with pytest.raises(RuntimeError):
        k.set_obs(1, x, np.array([1.0, 2.0, 3.0]))
    k.close()


def test_duplicate_observations_large_set_reports_first_pair():
    """The duplicate check of a large observation set (hash partitions over
    threads) reports the pair the reference's sequential scan finds first:
    the smallest index that repeats an earlier point, and that point."""
    from krigekit_b200 import Kriging
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, (100_000, 2))
    x[90_000] = x[5]
    x[70_000] = x[12_345]
    x[80_000] = -0.0 * x[80_000] + x[3]  # equal coordinates again, later index
    k = Kriging(ndim=2, nvar=1)
    with pytest.raises(RuntimeError, match="points 12346 and 70001"):
        k.set_obs(1, x, np.zeros(len(x)))
    x[70_000] += 1e-9
    with pytest.raises(RuntimeError, match="points 4 and 80001"):
        k.set_obs(1, x, np.zeros(len(x)))
    x[[80_000, 90_000]] += 1e-9
    k.set_obs(1, x, np.zeros(len(x)))  # no duplicates left
    k.close()
