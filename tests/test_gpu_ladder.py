"""GPU parity of the rare branches of the solve, through the C-ABI, against the oracle.

Each case builds host inputs that force one branch of the reference's solve
(solve_linear_system_base, kriging_base.F90:3244-3398; estimate_block_base,
kriging_base.F90:3407-3503) and checks both that the branch ran on the GPU
(krige_gpu_counters) and that the results agree with the oracle:

* FP32 factorisations of ill-conditioned systems re-solved in FP64;
* Cholesky failure -> Bunch-Kaufman LDL^T of the augmented matrix;
* LDL^T failure -> 1e-6 * mean-diagonal jitter -> LDL^T again;
* LDL^T failure with nothing to jitter -> NaN (neglect_error) or an error;
* Isaaks & Srivastava cokriging (std_ck=False), bounds clipping,
  leave-one-out cross-validation, update_obs_value + solve.

Nothing here faults a GPU: singular and indefinite systems come from the
host inputs (observation variances and per-target local nuggets).
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


def _compare(g, o, zstd, sill, tol, nvar=1):
    for iv in range(1, nvar + 1):
        nn, inear = g.get_neighbours(iv)
        np.testing.assert_array_equal(nn, o.nnear[:, iv - 1])
        for ib in range(len(nn)):
            assert np.array_equal(inear[ib, :nn[ib]], o.inear[ib, iv - 1, :nn[ib]]), f"block {ib} var {iv}"
    e, v = g.get_results(squeeze=False)
    oe, ov = o.get_results(squeeze=False)
    e = np.asarray(e).reshape(oe.shape)
    v = np.asarray(v).reshape(ov.shape)
    assert np.array_equal(np.isnan(e), np.isnan(oe))
    ok = ~np.isnan(oe)
    ee = bw.rel_err(e[ok], oe[ok], 1e-3 * zstd)
    ve = bw.rel_err(v[~np.isnan(ov)], ov[~np.isnan(ov)], 1e-3 * sill)
    assert ee.size == 0 or ee.max() <= tol, f"estimate rel err {ee.max():.3e}"
    assert ve.size == 0 or ve.max() <= tol, f"variance rel err {ve.max():.3e}"
    return e, v


# ------------------------------------------------------------ failure ladder
def _ladder_case(all_zero_variance):
    """36 observations on a jittered 0.1 lattice, spherical range 0.05 (every
    observation pair is farther apart than the range, so K is diagonal:
    cov0 + observation variance + local nugget).  With variances alternating
    0 / 2 a local nugget of -1 zeroes half the diagonal (the augmented matrix
    has equal rows: singular, so LDL^T fails and the jitter retry succeeds),
    -1.5 makes K indefinite but regular (Cholesky fails, LDL^T succeeds).
    With every variance 0, a local nugget of -1 zeroes K altogether: the mean
    diagonal is 0, nothing is jittered and the target fails."""
    rng = np.random.default_rng(11)
    g = np.arange(6) * 0.1 + 0.05
    gx, gy = np.meshgrid(g, g, indexing="xy")
    obs = np.column_stack([gx.ravel(), gy.ravel()]) + rng.uniform(-0.015, 0.015, (36, 2))
    z = np.sin(7 * obs[:, 0]) + np.cos(5 * obs[:, 1])
    var = np.zeros(36) if all_zero_variance else np.where(np.arange(36) % 2 == 0, 0.0, 2.0)
    tgt = np.array([[0.21, 0.32], [0.33, 0.27], [0.28, 0.41], [0.4, 0.22], [0.12, 0.17]])
    ln = np.array([0.0, -1.0, -1.5, -0.5, 0.0])
    return obs, z, var, tgt, ln


def _ladder_setup(k, case):
    obs, z, var, tgt, ln = case
    k.set_obs(1, obs, z, variance=var, nmax=9)
    k.set_vgm(1, 1, "sph", nugget=0.0, sill=1.0, a_major=0.05)
    k.set_grid(tgt, localnugget=ln)
    k.set_search(1)
    return k


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ldlt_and_jitter_retry(precision):
    case = _ladder_case(False)
    g = _ladder_setup(_gpu(ndim=2, nvar=1, precision=precision), case)
    g.solve()
    o = _ladder_setup(OracleKriging(ndim=2, nvar=1), case)
    o.solve()
    assert o.solver_stats["ssytrf_fact"] == 2
    _compare(g, o, float(np.std(case[1])), 1.0, TOL[precision])
    c = g.gpu_counters()
    assert c["ldlt"] == 2, c
    assert c["jitter"] == 1, c
    assert c["fail"] == 0, c
    assert g.solver_stats["ssytrf_fact"] == 2
    st = g.get_status()
    assert (st[[1, 2]] & 8).all() and not (st[[0, 3, 4]] & 8).any()  # KK_ST_LDLT on the two targets
    if precision == "fp32_refine":
        # the FP32 factorisations of both fail first and go through the FP64 form
        assert c["fp64_resolve"] >= 2, c
        assert (st[[1, 2]] & 4).all()  # KK_ST_FP64


@pytest.mark.parametrize("precision", PRECISIONS)
def test_singular_target_nan_when_neglect_error(precision):
    case = _ladder_case(True)
    g = _ladder_setup(_gpu(ndim=2, nvar=1, precision=precision, neglect_error=True), case)
    g.solve()
    o = _ladder_setup(OracleKriging(ndim=2, nvar=1, neglect_error=True), case)
    o.solve()
    e, v = _compare(g, o, float(np.std(case[1])), 1.0, TOL[precision])
    assert np.isnan(e[1]).all() and np.isnan(v[1]).all()
    assert np.isfinite(e[[0, 2, 3, 4]]).all()
    c = g.gpu_counters()
    assert c["fail"] == 1 and c["jitter"] == 0, c
    assert g.solver_stats["fail"] == 1
    assert g.get_status()[1] & 16  # KK_ST_FAIL


@pytest.mark.parametrize("precision", PRECISIONS)
def test_singular_target_error_without_neglect_error(precision):
    case = _ladder_case(True)
    g = _ladder_setup(_gpu(ndim=2, nvar=1, precision=precision, neglect_error=False), case)
    with pytest.raises(RuntimeError, match="[Ss]ingular"):
        g.solve()
    o = _ladder_setup(OracleKriging(ndim=2, nvar=1, neglect_error=False), case)
    with pytest.raises(Exception, match="[Ss]ingular"):
        o.solve()


def test_fp64_resolve_of_ill_conditioned_systems():
    """Nugget-free-like Gaussian model (nugget 1e-5 of the sill) on clustered
    observations: covariance matrices with condition numbers about 2e6, which
    the FP32 factorisation cannot refine to 1e-10; those targets are solved
    again in FP64.  The condition number multiplies the few-ulp differences of
    the covariance entries (fused multiply-adds) by about 2e6, so both forms
    are held to 1e-7 here."""
    rng = np.random.default_rng(21)
    cent = rng.uniform(0.2, 0.8, (6, 2))
    obs = np.vstack([cent[rng.integers(0, 6, 300)] + rng.normal(0, 0.02, (300, 2)), rng.uniform(0, 1, (60, 2))])
    z = np.sin(6 * obs[:, 0]) * np.cos(4 * obs[:, 1])
    gg = (np.arange(12) + 0.5) / 12
    gx, gy = np.meshgrid(gg, gg)
    tgt = np.column_stack([gx.ravel(), gy.ravel()])

    def setup(k):
        k.set_obs(1, obs, z, nmax=24)
        k.set_vgm(1, 1, "gau", nugget=1e-5, sill=1.0, a_major=0.3)
        k.set_grid(tgt)
        k.set_search(1)
        return k

    o = setup(OracleKriging(ndim=2, nvar=1))
    o.solve()
    out = {}
    for precision in PRECISIONS:
        g = setup(_gpu(ndim=2, nvar=1, precision=precision))
        g.solve()
        out[precision] = _compare(g, o, float(np.std(z)), 1.0, 1e-7)
        c = g.gpu_counters()
        assert c["fail"] == 0 and c["ldlt"] == 0, c
        if precision == "fp32_refine":
            assert c["fp64_resolve"] > 0, c
            st = g.get_status()
            assert int(((st & 4) != 0).sum()) == c["fp64_resolve"]
    e64, v64 = out["fp64"]
    e32, v32 = out["fp32_refine"]
    assert bw.rel_err(e32, e64, 1e-3 * float(np.std(z))).max() <= 1e-7


# ------------------------------------------------------------ estimate variants
@pytest.mark.parametrize("precision", PRECISIONS)
def test_isaaks_srivastava_cokriging(precision):
    """std_ck=False (the reference wrapper's default for nvar > 1): one
    unbiasedness row and the secondary weights shifted by the local mean
    difference (kriging_base.F90:3433-3455)."""
    w = bw.config4(grid_n=30, nobs=(500, 3000))
    kw = dict(ndim=2, nvar=2, std_ck=False)
    g = bw.apply(_gpu(precision=precision, nmin=4, **kw), w)
    g.solve()
    o = bw.apply(OracleKriging(nmin=4, **kw), w)
    o.solve()
    _compare(g, o, w["zstd"], w["sill"], TOL[precision], nvar=2)
    c = g.gpu_counters()
    assert c["fail"] == 0 and c["chol"] > 0, c


@pytest.mark.parametrize("precision", PRECISIONS)
def test_bounds_clipping(precision):
    """Estimates clipped to bounds inside the solve (kriging_base.F90:3497-3498)."""
    w = bw.config1(grid_n=40)
    kw = dict(ndim=2, nvar=1, bounds=(-0.4, 0.5))
    g = bw.apply(_gpu(precision=precision, nmin=4, **kw), w)
    g.solve()
    o = bw.apply(OracleKriging(nmin=4, **kw), w)
    o.solve()
    e, _ = _compare(g, o, w["zstd"], w["sill"], TOL[precision])
    ok = np.isfinite(e)
    assert (e[ok] == -0.4).sum() > 50 and (e[ok] == 0.5).sum() > 50
    assert e[ok].min() == -0.4 and e[ok].max() == 0.5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_leave_one_out_vs_oracle(precision):
    """Leave-one-out at the observations of variable 1 (set_grid_cv_base,
    kriging_base.F90:1120-1135; the target's own observation is skipped by
    the search, kriging.F90:647-657), compared with the oracle at the solve
    tolerance."""
    w = bw.config1(grid_n=10, nobs=1500)
    o1 = w["obs"][0]

    def setup(k):
        k.set_obs(1, o1["coord"], o1["value"], nmax=32, maxdist=0.3)
        k.set_vgm(1, 1, "sph", nugget=0.05, sill=1.0, a_major=0.25)
        k.set_grid_cv()
        k.set_search(1)
        return k

    g = setup(_gpu(ndim=2, nvar=1, precision=precision, cross_validation=True))
    g.solve()
    o = setup(OracleKriging(ndim=2, nvar=1))
    o.solve()
    _compare(g, o, w["zstd"], w["sill"], TOL[precision])
    nn, inear = g.get_neighbours(1)
    own = np.arange(1, len(nn) + 1)
    assert not any(own[i] in inear[i, :nn[i]] for i in range(len(nn)))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_leave_one_out_golden_vs_oracle(precision):
    """The reference fixture's leave-one-out setup (pc2d, all 62 observations)
    against the oracle at the solve tolerance."""
    pc = pd.read_csv(golden("pc2d.csv"))

    def setup(k):
        k.set_obs(1, pc[["x", "y"]].values, pc["pc"].values)
        k.set_vgm(1, 1, "sph", nugget=0.0, sill=0.12, a_major=5000.0)
        k.set_grid_cv()
        k.set_search(1)
        return k

    g = setup(_gpu(ndim=2, nvar=1, precision=precision, cross_validation=True))
    g.solve()
    o = setup(OracleKriging(ndim=2, nvar=1))
    o.solve()
    _compare(g, o, float(pc["pc"].std()), 0.12, TOL[precision])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_update_obs_value_then_solve(precision):
    """update_obs_value (kriging_base.F90:649-680) followed by solve gives the
    oracle's result for the new values, twice in a row."""
    w = bw.config2(grid_n=40, nobs=5000, nclusters=10)
    kw = dict(ndim=2, nvar=1, **w["kw"])
    g = bw.apply(_gpu(precision=precision, nmin=4, **kw), w)
    g.solve()
    z0 = np.asarray(w["obs"][0]["value"])
    rng = np.random.default_rng(3)
    for step in range(2):
        znew = z0 * (0.5 + step) + rng.normal(0, 0.2, z0.size)
        g.update_obs_value(1, znew)
        g.solve()
        w2 = dict(w, obs=[dict(w["obs"][0], value=znew)])
        o = bw.apply(OracleKriging(nmin=4, **kw), w2)
        o.solve()
        _compare(g, o, float(np.std(znew)), w["sill"], TOL[precision])
