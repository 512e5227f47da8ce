"""GPU weight store through the C-ABI, against the oracle (kriging_base.F90:2703-2990).

store_weight=True keeps the kriging weights and neighbour lists of a solve;
update_obs_value then makes the next solve a re-estimate from them (one
gather-dot kernel, no search and no solve); use_old_weight=True with
set_weights() loads a store from the caller.  Weights come from the FP64 form,
so they are compared with the oracle's at the FP64 tolerance, and so are the
re-estimated values against an oracle solve with the new observation values.
The layouts and error messages follow the reference's tests
(tests/test_weight_store.py).
"""
import numpy as np
import pytest

import bench_workloads as bw
from oracle.oracle import OracleKriging

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _gpu(**kw):
    from krigekit_b200 import Kriging
    return Kriging(**kw)


def _rel(x, ref, floor):
    return np.abs(np.asarray(x) - np.asarray(ref)) / np.maximum(np.abs(ref), floor)


def _oracle_weights(w_cfg, kw, values=None):
    w2 = w_cfg if values is None else dict(w_cfg, obs=[dict(o, value=v) for o, v in zip(w_cfg["obs"], values)])
    o = bw.apply(OracleKriging(**kw), w2)
    o.solve(keep_weights=True)
    return o


def _check_store(g, o, nvar):
    st = g.get_weights()
    nn, inear, wt = st["nnear"], st["inear"], st["weight"]
    nb = nn.shape[0]
    assert nn.shape == (nb, nvar) and inear.ndim == 3
    np.testing.assert_array_equal(nn, o.nnear)
    nm = inear.shape[2]
    assert nm == o.inear.shape[2]
    w4 = wt if nvar > 1 else wt[:, None, :, :]
    assert w4.shape == (nb, nvar, nvar, nm)
    for ib in range(nb):
        for v in range(nvar):
            k = nn[ib, v]
            np.testing.assert_array_equal(inear[ib, v, :k], o.inear[ib, v, :k])
            assert not inear[ib, v, k:].any() and not w4[ib, :, v, k:].any()  # zero padding
    scale = np.abs(o.weight).max()
    err = np.abs(w4 - o.weight).max() / scale
    assert err <= TOL, f"weights rel err {err:.3e}"
    _, var = g.get_results(squeeze=False)
    sv = st["variance"] if nvar > 1 else st["variance"][:, None, None]
    np.testing.assert_array_equal(sv, np.asarray(var).reshape(sv.shape))
    return st


@pytest.mark.parametrize("case", ["ok_plain", "ok_sector", "cokriging_std", "cokriging_isaaks"])
def test_store_replay_vs_oracle(case):
    if case == "ok_plain":
        w = bw.config1(grid_n=25, nobs=800)
        kw = dict(ndim=2, nvar=1)
    elif case == "ok_sector":
        w = bw.config2(grid_n=25, nobs=4000, nclusters=8)
        kw = dict(ndim=2, nvar=1, **w["kw"])
    else:
        w = bw.config4(grid_n=20, nobs=(400, 2500))
        kw = dict(ndim=2, nvar=2, std_ck=(case == "cokriging_std"))
    nvar = kw["nvar"]
    g = bw.apply(_gpu(precision="fp32_refine", store_weight=True, **kw), w)
    g.solve()
    o = _oracle_weights(w, kw)
    st = _check_store(g, o, nvar)
    if nvar == 1:  # ordinary kriging: weights sum to one
        sums = np.array([st["weight"][ib, 0, :st["nnear"][ib, 0]].sum() for ib in range(len(st["nnear"]))])
        np.testing.assert_allclose(sums, 1.0, atol=1e-12)
    e0, v0 = g.get_results(squeeze=False)
    oe0, _ = o.get_results(squeeze=False)
    assert _rel(np.asarray(e0).reshape(oe0.shape), oe0, 1e-3 * w["zstd"]).max() <= TOL
    # re-estimates from the store with new values, twice in a row
    rng = np.random.default_rng(8)
    base = [np.asarray(ob["value"]) for ob in w["obs"]]
    for step in range(2):
        vals = [b * (1.0 + 0.5 * step) + rng.normal(0, 0.3, b.size) for b in base]
        for iv, v in enumerate(vals, start=1):
            g.update_obs_value(iv, v)
        g.solve()
        assert g.phases()["launches"] == 1  # one gather-dot kernel, no search or solve
        e, var = g.get_results(squeeze=False)
        o2 = _oracle_weights(w, kw, vals)
        oe, ov = o2.get_results(squeeze=False)
        zstd = float(np.std(vals[0]))
        assert _rel(np.asarray(e).reshape(oe.shape), oe, 1e-3 * zstd).max() <= TOL, f"step {step}"
        np.testing.assert_array_equal(np.asarray(var), np.asarray(v0))  # variances do not move
    g.close()


def test_set_weights_loads_a_store():
    """The reference's in-memory round trip (test_weight_store.py:504-589):
    weights of one object, loaded into another with new values."""
    w = bw.config1(grid_n=20, nobs=600)
    kw = dict(ndim=2, nvar=1)
    g1 = bw.apply(_gpu(store_weight=True, **kw), w)
    g1.solve()
    st = g1.get_weights()
    e1, v1 = g1.get_results()
    z = np.asarray(w["obs"][0]["value"])
    g2 = bw.apply(_gpu(use_old_weight=True, **kw), dict(w, obs=[dict(w["obs"][0], value=2.0 * z)]))
    g2.set_weights(st)
    g2.solve()
    e2, v2 = g2.get_results()
    np.testing.assert_allclose(e2, 2.0 * e1, rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(v2, v1)
    # without the variance key the variance is zero
    g3 = bw.apply(_gpu(use_old_weight=True, **kw), w)
    g3.set_weights({k: v for k, v in st.items() if k != "variance"})
    g3.solve()
    e3, v3 = g3.get_results()
    np.testing.assert_allclose(e3, e1, rtol=1e-12, atol=1e-12)
    assert np.all(v3 == 0.0)
    st2 = g3.get_weights()  # the staged store reads back unchanged
    np.testing.assert_array_equal(st2["inear"], st["inear"])
    np.testing.assert_array_equal(st2["weight"], st["weight"])


def test_weight_store_errors():
    w = bw.config1(grid_n=8, nobs=300)
    kw = dict(ndim=2, nvar=1)
    g = bw.apply(_gpu(**kw), w)
    g.solve()
    with pytest.raises(RuntimeError, match="Weight store not allocated"):
        g.get_weights()
    g2 = bw.apply(_gpu(store_weight=True, **kw), w)
    g2.solve()
    st = g2.get_weights()
    with pytest.raises(ValueError, match="store_weight=True"):
        g2.set_weights(st)
    g2.free_weight_store()
    with pytest.raises(RuntimeError, match="Weight store not allocated"):
        g2.get_weights()
    with pytest.raises(ValueError, match="mutually exclusive"):
        _gpu(store_weight=True, use_old_weight=True, **kw)
    g3 = bw.apply(_gpu(use_old_weight=True, **kw), w)
    with pytest.raises(RuntimeError, match="set_weights"):
        g3.solve()


def test_variance_all_and_info():
    w = bw.config4(grid_n=10, nobs=(300, 1500))
    kw = dict(ndim=2, nvar=2, std_ck=True)
    g = bw.apply(_gpu(**kw), w)
    g.solve()
    _, v = g.get_results(squeeze=False)
    va = g.get_variance_all(copy=True)
    np.testing.assert_array_equal(va, np.asarray(v))
    info = g.get_info()
    assert "Number of Variables" in info and "Variable 2:" in info
    assert str(g) == g.get_info()
