"""krige_resolve_static: the allocation-free FP64 re-solve, through the C-ABI.

It re-solves the neighbour sets of the last krige_solve with the generic
one-thread-per-target kernel whose workspace, work list and counters live in
a fixed static device array.  Each case calls it twice in a row with new
observation values and compares both results with the existing entry points
(krige_update_obs_value + krige_solve in FP64) on a second handle and with
the oracle's solve of the same values, and checks that the torch caching
allocator saw no allocation during the calls.
This file is collected last so that it also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

import bench_workloads as bw

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _handle_pair(w):
    if w.get("st"):
        from krigekit_b200 import SpaceTimeKriging
        a = bw.apply_st(SpaceTimeKriging(precision="fp64"), w)
        b = bw.apply_st(SpaceTimeKriging(precision="fp64"), w)
        return a, b
    from krigekit_b200 import Kriging
    kw = dict(ndim=w["ndim"], nvar=w["nvar"], **w["kw"])
    a = bw.apply(Kriging(precision="fp64", **kw), w)
    b = bw.apply(Kriging(precision="fp64", **kw), w)
    return a, b


def _compare(a, b, zstd, sill, what):
    e_s, v_s = _results(a)
    e_r, v_r = _results(b)
    assert np.array_equal(np.isnan(e_s), np.isnan(e_r))
    ok = ~np.isnan(e_r)
    ee = bw.rel_err(e_s[ok], e_r[ok], 1e-3 * zstd)
    ve = bw.rel_err(v_s, v_r, 1e-3 * sill)
    assert np.nanmax(ee) <= TOL, f"{what}: estimate rel err {np.nanmax(ee):.3e}"
    assert np.nanmax(ve) <= TOL, f"{what}: variance rel err {np.nanmax(ve):.3e}"


def _results(k):
    e, v = k.get_results(squeeze=False)
    return np.array(e), np.array(v)


def _resolve_static(k, ivar, value):
    from krigekit_b200 import _lib
    lib = _lib.load()
    if value is None:
        ierr = lib.krige_resolve_static(ctypes.c_int64(k._handle), 0, 0, None)
    else:
        v = np.ascontiguousarray(value, dtype=np.float64)
        ierr = lib.krige_resolve_static(ctypes.c_int64(k._handle), ivar, v.size,
                                        v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return int(ierr)


def _allocations():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.memory_stats().get("allocation.all.allocated", 0)


def _vs_oracle(a, w, zstd, sill, what):
    """The re-solve's results against the oracle's solve of workload w."""
    from oracle.oracle import OracleKriging, OracleSpaceTime
    if w.get("st"):
        o = bw.apply_st(OracleSpaceTime(ndim=2), w)
    else:
        o = bw.apply(OracleKriging(ndim=w["ndim"], nvar=w["nvar"], **w["kw"]), w)
    o.solve()
    oe, ov = (np.array(x) for x in o.get_results(squeeze=False))
    e_s, v_s = _results(a)
    e_s = e_s.reshape(oe.shape)
    v_s = v_s.reshape(ov.shape)
    ok = ~np.isnan(oe)
    assert np.array_equal(np.isnan(e_s), np.isnan(oe)), what
    ee = np.nanmax(bw.rel_err(e_s[ok], oe[ok], 1e-3 * zstd))
    ve = np.nanmax(bw.rel_err(v_s, ov, 1e-3 * sill))
    assert ee <= TOL, f"{what}: estimate rel err {ee:.3e} against the oracle"
    assert ve <= TOL, f"{what}: variance rel err {ve:.3e} against the oracle"


def _with_values(w, ivar, znew):
    obs = [dict(o) for o in w["obs"]]
    obs[ivar - 1]["value"] = znew
    return dict(w, obs=obs)


def _check_two_calls(w, ivar):
    from krigekit_b200 import _lib
    a, b = _handle_pair(w)
    a.solve()
    b.solve()
    z0 = np.asarray(w["obs"][ivar - 1]["value"], dtype=np.float64)
    rng = np.random.default_rng(77)
    for call in range(2):
        znew = z0 * (1.0 + 0.5 * call) + rng.normal(0.0, 0.1, z0.size)
        before = _allocations()
        ierr = _resolve_static(a, ivar, znew)
        after = _allocations()
        assert ierr == 0, _lib.last_error()
        assert after == before, f"call {call}: {after - before} device allocations"
        b.update_obs_value(ivar, znew)
        b.solve()
        _compare(a, b, float(np.std(znew)), w["sill"], f"call {call}")
        assert a.gpu_counters()["fail"] == 0
        _vs_oracle(a, _with_values(w, ivar, znew), float(np.std(znew)), w["sill"], f"call {call}")
    # null values: the same neighbour sets and values give the same results again
    e1, v1 = _results(a)
    assert _resolve_static(a, 0, None) == 0, _lib.last_error()
    e2, v2 = _results(a)
    np.testing.assert_array_equal(e1, e2)
    np.testing.assert_array_equal(v1, v2)
    a.close()
    b.close()


def test_resolve_static_sector_search():
    w = bw.config2(grid_n=70, nobs=6000, nclusters=12)
    _check_two_calls(w, 1)


def test_resolve_static_cokriging():
    w = bw.config4(grid_n=40, nobs=(600, 4000))
    _check_two_calls(w, 2)


def test_resolve_static_external_drift_changed_between_calls():
    """KED (two external drifts): krige_set_grid_drift between the calls must
    reach the re-solve, like it reaches the next krige_solve."""
    from krigekit_b200 import _lib
    w = bw.config3(grid_n=(12, 12, 4), nobs=3000)
    a, b = _handle_pair(w)
    a.solve()
    b.solve()
    gd0 = np.asarray(w["grid_drift"])
    for call in range(2):
        gd = gd0 * (1.0 + 0.3 * (call + 1)) + 0.05 * (call + 1)
        a.set_grid_drift(gd)
        b.set_grid_drift(gd)
        assert _resolve_static(a, 0, None) == 0, _lib.last_error()
        b.solve()
        _compare(a, b, w["zstd"], w["sill"], f"drift call {call}")
        _vs_oracle(a, dict(w, grid_drift=gd), w["zstd"], w["sill"], f"drift call {call}")
    a.close()
    b.close()


def test_resolve_static_space_time():
    """Space-time product-sum model with block targets (krige_st_* handle)."""
    w = bw.config5(grid_n=10, ntimes=3, nstations=120, ndays=40)
    _check_two_calls(w, 1)


def test_resolve_static_after_set_vgm():
    """A variogram replaced between krige_solve and the re-solve (new sill and
    range, same model shape): the re-solve rebuilds the tables in place."""
    from krigekit_b200 import _lib
    w = bw.config1(grid_n=20, nobs=600)
    a, b = _handle_pair(w)
    a.solve()
    b.solve()
    for call, (sill, rng_) in enumerate(((1.4, 0.18), (0.7, 0.33))):
        for k in (a, b):
            k.set_vgm(1, 1, "sph", nugget=0.05, sill=sill, a_major=rng_, append=False)
        assert _resolve_static(a, 0, None) == 0, _lib.last_error()
        b.solve()
        _compare(a, b, w["zstd"], sill + 0.05, f"vgm call {call}")
        vgm = [(1, 1, dict(vtype="sph", nugget=0.05, sill=sill, a_major=rng_))]
        _vs_oracle(a, dict(w, vgm=vgm), w["zstd"], sill + 0.05, f"vgm call {call}")
    a.close()
    b.close()


def test_resolve_static_rejects_oversized_systems():
    from krigekit_b200 import Kriging, _lib
    rng = np.random.default_rng(5)
    n = 1500  # one system of 1501 equations needs ~36 MB of workspace, above the 32 MiB array
    obs = rng.uniform(0, 1, (n, 2))
    k = Kriging(precision="fp64")
    k.set_obs(1, obs, np.sin(6 * obs[:, 0]), nmax=n)
    k.set_vgm(1, 1, "exp", nugget=0.1, sill=1.0, a_major=0.3)
    k.set_grid(np.array([[0.5, 0.5]]))
    k.set_search(1)
    k.solve()
    e0, v0 = _results(k)
    z_new = np.cos(5 * obs[:, 1])
    assert _resolve_static(k, 1, z_new) == 1
    assert "static scratch" in _lib.last_error()
    # the rejected call changed nothing: the last solve's results stay readable
    e1, v1 = _results(k)
    np.testing.assert_array_equal(e0, e1)
    np.testing.assert_array_equal(v0, v1)
    k.close()


def test_resolve_static_needs_a_solve():
    from krigekit_b200 import Kriging, _lib
    w = bw.config1(grid_n=10, nobs=200)
    k = bw.apply(Kriging(precision="fp64", ndim=2, nvar=1), w)
    assert _resolve_static(k, 0, None) == 1
    assert "krige_solve" in _lib.last_error()
    k.solve()
    k.set_obs(1, w["obs"][0]["coord"], w["obs"][0]["value"], nmax=32)
    assert _resolve_static(k, 0, None) == 1
    assert "krige_solve" in _lib.last_error()
    k.close()
