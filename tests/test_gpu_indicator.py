"""Multiple indicator kriging on the GPU (IndicatorKriging, krige_ind_create) against the oracle.

The reference solves K indicator variables as one cokriging system and then
clips each category probability to [0, 1] and normalises the K of them to sum
to one (post_solve_indicator, kriging_indicator.F90:170-185).  The oracle
solves the same cokriging system; the post-processing is restated here in
numpy.  K = 3 runs on the register kernels, K = 4 (ten right-hand-side columns
with the Isaaks & Srivastava form) on the general kernel.
"""
import numpy as np
import pytest

import bench_workloads as bw
from oracle.oracle import OracleKriging

pytestmark = pytest.mark.gpu


def _categories(ncat, nobs=360, seed=4):
    rng = np.random.default_rng(seed)
    obs = rng.uniform(0, 1, (nobs, 2))
    f = bw.cosine_field(rng, 2, 0.25)(obs)
    edges = np.quantile(f, np.linspace(0, 1, ncat + 1)[1:-1])
    cats = np.digitize(f, edges) + 1
    g = (np.arange(18) + 0.5) / 18
    gx, gy = np.meshgrid(g, g)
    return obs, cats, np.column_stack([gx.ravel(), gy.ravel()])


def _indicator_vgm(k, ncat, cross="same", proportions=None):
    """The reference's set_indicator_vgm loop (kriging_indicator.py:378-412) on any object."""
    if proportions is not None and cross != "same":
        auto = np.asarray(proportions) * (1.0 - np.asarray(proportions))
    else:
        auto = np.full(ncat, 0.2)
    for iv in range(1, ncat + 1):
        for jv in range(1, ncat + 1):
            if iv == jv:
                ps, pn = float(auto[iv - 1]), 0.02
            elif cross == "independent":
                ps, pn = 0.0, 0.0
            elif cross == "proportional":
                ps, pn = float(np.sqrt(auto[iv - 1] * auto[jv - 1])), 0.02
            else:
                ps, pn = 0.2, 0.02
            k.set_vgm(iv, jv, "sph", nugget=pn, sill=ps, a_major=0.4, a_minor1=0.4, a_minor2=0.4)


def _post(est, kcat):
    p = np.clip(est[:, :kcat], 0.0, 1.0)
    s = p.sum(axis=1, keepdims=True)
    p = np.where(s > 0, p / np.where(s > 0, s, 1.0), p)
    out = est.copy()
    out[:, :kcat] = p
    return out


@pytest.mark.parametrize("ncat,cross,precision", [(3, "same", "fp64"), (3, "proportional", "fp32_refine"),
                                                  (4, "same", "fp64"), (4, "independent", "fp32_refine")])
def test_indicator_probabilities_vs_oracle(ncat, cross, precision):
    from krigekit_b200 import IndicatorKriging
    obs, cats, grid = _categories(ncat)
    props = np.array([(cats == c).mean() for c in range(1, ncat + 1)])
    ik = IndicatorKriging(ncat=ncat, ndim=2, precision=precision)
    ik.set_categorical_obs(obs, cats, nmax=12)
    ik.set_indicator_vgm(vtype="sph", nugget=0.02, sill=0.2, a_major=0.4, cross=cross,
                         proportions=props if cross != "same" else None)
    ik.set_grid(grid)
    for k in range(1, ncat + 1):
        ik.set_search(ivar=k)
    ik.solve()
    probs, _ = ik.get_results()
    o = OracleKriging(ndim=2, nvar=ncat)
    for k in range(1, ncat + 1):
        o.set_obs(k, obs, (cats == k).astype(float), nmax=12)
    _indicator_vgm(o, ncat, cross, props)
    o.set_grid(grid)
    for k in range(1, ncat + 1):
        o.set_search(k)
    o.solve()
    oe, _ = o.get_results(squeeze=False)
    ref = _post(oe.reshape(len(grid), ncat), ncat)
    probs = np.asarray(probs).reshape(len(grid), ncat)
    np.testing.assert_allclose(probs, ref, rtol=0, atol=1e-9 if precision == "fp64" else 1e-6)
    np.testing.assert_allclose(probs.sum(axis=1), 1.0, atol=1e-12)
    assert probs.min() >= 0.0 and probs.max() <= 1.0
    if ncat == 4:
        assert ik.gpu_counters()["chol"] == len(grid)  # every system on the general kernel


def test_indicator_with_secondary_variable():
    """ncat < nvar: the secondary co-variate is kriged with the categories but
    left out of the normalisation (krige_ind_set_ncat)."""
    from krigekit_b200 import IndicatorKriging
    obs, cats, grid = _categories(2)
    sec = np.sin(5 * obs[:, 0]) + obs[:, 1]
    ik = IndicatorKriging(ncat=2, nvar=3, ndim=2, std_ck=True, precision="fp64")
    ik.set_categorical_obs(obs, cats, nmax=10)
    ik.set_obs(3, obs, sec, nmax=10)
    o = OracleKriging(ndim=2, nvar=3, std_ck=True)
    for k in (1, 2):
        o.set_obs(k, obs, (cats == k).astype(float), nmax=10)
    o.set_obs(3, obs, sec, nmax=10)
    for k in (ik, o):
        for iv in range(1, 4):
            for jv in range(iv, 4):
                k.set_vgm(iv, jv, "sph", nugget=0.02 if iv == jv else 0.0, sill=0.2 if iv == jv else 0.05,
                          a_major=0.4)
        k.set_grid(grid)
        for iv in range(1, 4):
            k.set_search(iv)
        k.solve()
    est, _ = ik.get_results()
    oe, _ = o.get_results(squeeze=False)
    ref = _post(oe.reshape(len(grid), 3), 2)
    np.testing.assert_allclose(np.asarray(est).reshape(len(grid), 3), ref, rtol=0, atol=1e-9)
