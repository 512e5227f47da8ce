"""CPU oracle for the kriging solve path -- TEST INFRASTRUCTURE ONLY.

This module drives ``kk_oracle.c`` (a plain-C restatement of the reference
engine, ougx/krigekit src/libkriging) through ctypes.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import it, as
the checker or the timed CPU port.  The product package ``krigekit_b200``
never imports it.

``OracleKriging`` mirrors the reference ``Kriging`` class setters
(src/krigekit/kriging.py:403-1579: set_obs, set_obs_drift, set_vgm,
set_grid, set_grid_block, set_grid_drift, set_search, solve, get_results,
get_result_df) so that parity tests read like the reference's own tests.
``OracleSpaceTime`` mirrors ``SpaceTimeKriging`` (src/krigekit/kriging_st.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")
MAXVAR = 4
MAXSTRUCT = 16

VTYPES = {"nug": 0, "sph": 1, "exp": 2, "gau": 3, "hol": 4, "pow": 5,
          "bsq": 6, "cir": 7, "lin": 8, "cyc": 9, "dco": 10}


def build(force: bool = False) -> str:
    """Compile kk_oracle.c into oracle/liborc.so (gcc, OpenMP, no FMA contraction)."""
    src = os.path.join(HERE, "kk_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(os.path.join(HERE, "kk_oracle.h"))):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
           "-shared", "-o", LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


class _Spec(ctypes.Structure):
    _fields_ = [("vtype", ctypes.c_int), ("nugget", ctypes.c_double), ("sill", ctypes.c_double),
                ("a_major", ctypes.c_double), ("a_minor1", ctypes.c_double),
                ("a_minor2", ctypes.c_double), ("azimuth", ctypes.c_double),
                ("dip", ctypes.c_double), ("plunge", ctypes.c_double),
                ("is_product", ctypes.c_int)]


_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)


class _Problem(ctypes.Structure):
    _fields_ = [
        ("ndim", _I), ("nlag", _I), ("nvar", _I), ("ndrift", _I), ("unbias", _I),
        ("std_ck", _I), ("neglect_error", _I), ("anisotropic_search", _I), ("nmin", _I),
        ("bounds", _D * 2),
        ("nobs", _I * MAXVAR), ("obs_coord", _PD * MAXVAR), ("obs_value", _PD * MAXVAR),
        ("obs_var", _PD * MAXVAR), ("obs_drift", _PD * MAXVAR), ("nmax", _I * MAXVAR),
        ("maxdist", _D * MAXVAR), ("sk_mean", _D * MAXVAR),
        ("s_anis1", _D * MAXVAR), ("s_anis2", _D * MAXVAR), ("s_az", _D * MAXVAR),
        ("s_dip", _D * MAXVAR), ("s_plunge", _D * MAXVAR), ("sector", _I * MAXVAR),
        ("time_at", _D * MAXVAR),
        ("nstruct", (_I * MAXVAR) * MAXVAR),
        ("vgm", ((_Spec * MAXSTRUCT) * MAXVAR) * MAXVAR),
        ("st", _I), ("st_model", _I), ("st_transform", _I),
        ("st_at", _D), ("st_k_ps", _D), ("st_time_nugget", _D), ("st_time_sill", _D),
        ("nstruct_t", (_I * MAXVAR) * MAXVAR),
        ("vgm_t", ((_Spec * MAXSTRUCT) * MAXVAR) * MAXVAR),
        ("st_joint", ((_D * MAXSTRUCT) * MAXVAR) * MAXVAR),
        ("st_has_joint", (_I * MAXVAR) * MAXVAR),
        ("nblock", _I), ("block_coord", _PD), ("nblockpnt", _PI), ("grid_coord", _PD),
        ("grid_weight", _PD), ("rangescale", _PD), ("localnugget", _PD), ("block_drift", _PD),
        ("nthread", _I), ("ncache", _I), ("cross_validation", _I), ("analytic", _I),
    ]


class _Result(ctypes.Structure):
    _fields_ = [("value", _PD), ("variance", _PD), ("nnear", _PI), ("inear", _PI),
                ("mmax", _I), ("weight", _PD), ("stats", _I * 5), ("err", _I),
                ("errmsg", ctypes.c_char * 256)]


class _SimResult(ctypes.Structure):
    _fields_ = [("value", _PD), ("variance", _PD), ("nnear", _PI), ("inear", _PI), ("mmax", _I),
                ("err", _I), ("errmsg", ctypes.c_char * 256)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_solve.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(_Result)]
        _lib.orc_solve.restype = _I
        _lib.orc_calc_rotmat.argtypes = [_D, _D, _D, _D, _D, _PD]
        _lib.orc_corefunc.argtypes = [_I, _D]
        _lib.orc_corefunc.restype = _D
        _lib.orc_kdtree_nn.argtypes = [_PD, _I, _I, _PD, _I, _I, _PD, _PI]
        _lib.orc_sysv.argtypes = [_I, _PD, _I, _PD]
        _lib.orc_sysv.restype = _I
        _lib.orc_sgsim.argtypes = [ctypes.POINTER(_Problem), _PI, _PD, _I, ctypes.POINTER(_SimResult)]
        _lib.orc_sgsim.restype = _I
    return _lib


def _dp(a):
    return a.ctypes.data_as(_PD) if a is not None else None


class OracleKriging:
    """Oracle twin of the reference ``Kriging`` class (spatial)."""

    st = False

    def __init__(self, ndim: int = 2, nvar: int = 1, ndrift: int = 0, unbias: int = 1,
                 nsim: int = 0, anisotropic_search: bool = False, neglect_error: bool = True,
                 std_ck: bool = False, bounds: Optional[tuple] = None, nmin: int = 0, **_ignored):
        self.nsim = int(nsim)
        self.sim_path = None
        self.sim_sample = None
        self.ndim, self.nvar, self.ndrift, self.unbias = ndim, nvar, ndrift, unbias
        self.nlag = ndim
        self.anisotropic_search = anisotropic_search
        self.neglect_error = neglect_error
        self.std_ck = std_ck
        self.nmin = nmin
        huge = sys.float_info.max
        self.bounds = (-huge, huge) if bounds is None else tuple(bounds)
        self.obs = [None] * nvar
        self.vgm = {}
        self.vgm_t = {}
        self.search = [None] * nvar
        self.grid = None
        self.grid_drift = None
        self.result = None

    # -- setters mirroring kriging.py --------------------------------------
    def set_obs(self, ivar, coord, value, variance=None, nmax=None, maxdist=None, sk_mean=0.0):
        coord = np.ascontiguousarray(np.asarray(coord, dtype=np.float64).reshape(len(value), -1))
        n = coord.shape[0]
        self.obs[ivar - 1] = dict(
            coord=coord, value=np.ascontiguousarray(value, dtype=np.float64),
            variance=(np.ascontiguousarray(variance, dtype=np.float64)
                      if variance is not None else np.zeros(n)),
            nmax=int(nmax) if nmax is not None else np.iinfo(np.int32).max,
            maxdist=float(maxdist) if maxdist is not None else sys.float_info.max,
            sk_mean=float(sk_mean), drift=None)

    def set_obs_drift(self, ivar, drift):
        d = np.ascontiguousarray(np.asarray(drift, dtype=np.float64).reshape(-1, self.ndrift))
        self.obs[ivar - 1]["drift"] = d

    def set_vgm(self, ivar, jvar, vtype, nugget=0.0, sill=1.0, a_major=1.0, a_minor1=None,
                a_minor2=None, azimuth=0.0, dip=0.0, plunge=0.0, append=True, product=False):
        if a_minor1 is None:
            a_minor1 = a_major
        if a_minor2 is None:
            a_minor2 = a_minor1
        if jvar < ivar:  # the reference wrapper's swap collapses to (ivar, ivar), kriging.py:884-887
            jvar = ivar
        a, b = ivar - 1, jvar - 1
        spec = (VTYPES[vtype.lower()[:3]], nugget, sill, a_major, a_minor1, a_minor2,
                azimuth, dip, plunge, int(bool(product)))
        if not append:
            self.vgm[(a, b)] = []
        self.vgm.setdefault((a, b), []).append(spec)

    def set_grid_cv(self):
        """Leave-one-out targets at obs(1) (set_grid_cv_base, kriging_base.F90:1120-1135)."""
        self.cross_validation = True
        self.grid = dict(coord=self.obs[0]["coord"].copy(), nblockpnt=None, gcoord=None,
                         gweight=None, rangescale=None, localnugget=None)
        if self.ndrift > 0:
            d = self.obs[0]["drift"]
            self.grid_drift = np.repeat(d[:, None, :], self.nvar, axis=1)

    def set_grid(self, coord=None, rangescale=None, localnugget=None):
        if coord is None:
            return self.set_grid_cv()
        coord = np.ascontiguousarray(np.asarray(coord, dtype=np.float64).reshape(-1, self.nlag))
        self.grid = dict(coord=coord, nblockpnt=None, gcoord=None, gweight=None,
                         rangescale=rangescale, localnugget=localnugget)

    def set_grid_block(self, coord, block_type, nblockpnt, pointweight=None, blocksize=None,
                       rangescale=None, localnugget=None):
        coord = np.asarray(coord, dtype=np.float64).reshape(-1, self.nlag)
        if block_type == -4:
            # set_grid_gq_base, kriging_base.F90:1010-1068 (gaussian_quadrature.f90)
            frac = np.array([0.4305681558, 0.1699905218, -0.1699905218, -0.4305681558])
            wgq4 = np.array([0.1739274226, 0.3260725774, 0.3260725774, 0.1739274226])
            nb = coord.shape[0]
            bs = np.asarray(blocksize, dtype=np.float64)
            if bs.ndim == 1:
                bs = np.tile(bs, (nb, 1))
            ngq = 4 ** self.ndim
            ii = np.array([[i, j, k] for k in range(4) for j in range(4) for i in range(4)])[:ngq]
            if self.ndim == 2:
                ii = np.array([[i, j] for j in range(4) for i in range(4)])
            elif self.ndim == 1:
                ii = np.arange(4).reshape(-1, 1)
            gcoord = np.empty((nb * ngq, self.ndim))
            gw = np.empty(nb * ngq)
            for ib in range(nb):
                w = np.ones(ngq)
                for d in range(self.ndim):
                    w = w * wgq4[ii[:, d]]
                for d in range(self.ndim):
                    gcoord[ib * ngq:(ib + 1) * ngq, d] = coord[ib, d] + frac[ii[:, d]] * bs[ib, d]
                gw[ib * ngq:(ib + 1) * ngq] = w
            nbp = np.full(nb, ngq, dtype=np.int32)
            bcoord = coord
        else:
            nbp = np.asarray(nblockpnt, dtype=np.int32)
            gcoord = coord
            if pointweight is None:
                gw = np.repeat(1.0 / nbp, nbp)
            else:
                gw = np.asarray(pointweight, dtype=np.float64)
            # set_grid_centroid_common, kriging_base.F90:1500-1560
            starts = np.concatenate([[0], np.cumsum(nbp)[:-1]])
            bcoord = np.empty((len(nbp), self.nlag))
            for ib, (s, n) in enumerate(zip(starts, nbp)):
                wsum = 0.0
                for k in range(n):
                    wsum += gw[s + k]
                for d in range(self.nlag):
                    acc = 0.0
                    for k in range(n):
                        acc += gcoord[s + k, d] * gw[s + k]
                    bcoord[ib, d] = acc / wsum
        self.grid = dict(coord=np.ascontiguousarray(bcoord), nblockpnt=np.ascontiguousarray(nbp),
                         gcoord=np.ascontiguousarray(gcoord), gweight=np.ascontiguousarray(gw),
                         rangescale=rangescale, localnugget=localnugget)

    def set_grid_drift(self, drift, ivar=None):
        nb = self.grid["coord"].shape[0]
        d = np.asarray(drift, dtype=np.float64).reshape(nb, self.ndrift)
        if self.grid_drift is None:
            self.grid_drift = np.zeros((nb, self.nvar, self.ndrift))
        if ivar is None or ivar < 0:
            for v in range(self.nvar):
                self.grid_drift[:, v, :] = d
        else:
            self.grid_drift[:, ivar - 1, :] = d

    def set_search(self, ivar=1, anis1=1.0, anis2=1.0, azimuth=0.0, dip=0.0, plunge=0.0,
                   sector_search=False, time_at=1.0):
        self.search[ivar - 1] = (anis1, anis2, azimuth, dip, plunge, int(bool(sector_search)),
                                 time_at)

    # -- solve --------------------------------------------------------------
    analytic = False
    cross_validation = False

    def _problem(self, nthread=0, ncache=64):
        P = _Problem()
        keep = []
        P.ndim, P.nlag, P.nvar, P.ndrift, P.unbias = self.ndim, self.nlag, self.nvar, self.ndrift, self.unbias
        P.std_ck = int(self.std_ck)
        P.neglect_error = int(self.neglect_error)
        P.anisotropic_search = int(self.anisotropic_search)
        P.nmin = int(self.nmin)
        P.bounds[0], P.bounds[1] = self.bounds
        for v in range(self.nvar):
            o = self.obs[v]
            if o is None:
                raise RuntimeError("Call set_obs() for every variable before solve().")
            if self.search[v] is None:
                raise RuntimeError("set_search() needs to be called before solve().")
            P.nobs[v] = o["coord"].shape[0]
            P.obs_coord[v] = _dp(o["coord"])
            P.obs_value[v] = _dp(o["value"])
            P.obs_var[v] = _dp(o["variance"])
            if self.ndrift > 0:
                if o["drift"] is None:
                    raise RuntimeError("Observation drift is not set while ndrift > 0.")
                P.obs_drift[v] = _dp(o["drift"])
            P.nmax[v] = min(o["nmax"], np.iinfo(np.int32).max)
            P.maxdist[v] = o["maxdist"]
            P.sk_mean[v] = o["sk_mean"]
            a1, a2, az, dp_, pl, sec, ta = self.search[v]
            P.s_anis1[v], P.s_anis2[v], P.s_az[v], P.s_dip[v], P.s_plunge[v] = a1, a2, az, dp_, pl
            P.sector[v] = sec
            P.time_at[v] = ta
        for (a, b), specs in self.vgm.items():
            for (x, y) in ((a, b), (b, a)):
                P.nstruct[x][y] = len(specs)
                for k, s in enumerate(specs):
                    P.vgm[x][y][k] = _Spec(*s)
        self._fill_st(P)
        g = self.grid
        if g is None:
            raise RuntimeError("Call set_grid() before solve().")
        nb = g["coord"].shape[0]
        P.nblock = nb
        P.block_coord = _dp(g["coord"])
        if g["nblockpnt"] is not None:
            P.nblockpnt = g["nblockpnt"].ctypes.data_as(_PI)
            P.grid_coord = _dp(g["gcoord"])
            P.grid_weight = _dp(g["gweight"])
        for key in ("rangescale", "localnugget"):
            if g[key] is not None:
                arr = np.ascontiguousarray(np.broadcast_to(np.asarray(g[key], dtype=np.float64), (nb,)))
                keep.append(arr)
                setattr(P, key, _dp(arr))
        if self.ndrift > 0:
            if self.grid_drift is None:
                raise RuntimeError("Grid drift is not set while ndrift > 0.")
            gd = np.ascontiguousarray(self.grid_drift)
            keep.append(gd)
            P.block_drift = _dp(gd)
        P.nthread = nthread
        P.ncache = ncache
        P.analytic = int(self.analytic)
        P.cross_validation = int(self.cross_validation)
        return P, keep

    def _fill_st(self, P):
        P.st = 0

    def set_sim(self, randpath, sample):
        """SGSIM visiting order (1-based, nblock) and N(0, 1) draws: (nblock,),
        (nblock, nsim) or (nblock, 1, nsim) like the reference's set_sim
        (kriging.py:1134-1203); the p-th visited target takes row p."""
        self.sim_path = np.ascontiguousarray(np.asarray(randpath, dtype=np.int32).ravel())
        smp = np.asarray(sample, dtype=np.float64)
        smp = smp.reshape(smp.shape[0], -1)
        if smp.shape[1] != self.nsim:
            raise ValueError("sample needs nsim columns")
        self.sim_sample = np.ascontiguousarray(smp)
        return self

    def _solve_sim(self):
        P, keep = self._problem(nthread=1, ncache=0)
        nb = P.nblock
        nmax = int(self.obs[0]["nmax"])
        ntot = self.obs[0]["coord"].shape[0] + nb
        if nmax <= 0 or nmax > ntot:
            nmax = ntot
        mm = min((2 ** self.ndim) * nmax if P.sector[0] else nmax, ntot)
        self.value = np.full((nb, self.nsim), np.nan)
        self.variance = np.full(nb, np.nan)
        self.sim_nnear = np.zeros((nb, 2), dtype=np.int32)
        self.sim_inear = np.zeros((nb, mm), dtype=np.int32)
        R = _SimResult()
        R.value = _dp(self.value)
        R.variance = _dp(self.variance)
        R.nnear = self.sim_nnear.ctypes.data_as(_PI)
        R.inear = self.sim_inear.ctypes.data_as(_PI)
        R.mmax = mm
        ierr = lib().orc_sgsim(ctypes.byref(P), self.sim_path.ctypes.data_as(_PI), _dp(self.sim_sample),
                               self.nsim, ctypes.byref(R))
        if ierr:
            raise RuntimeError(R.errmsg.decode())
        self._keep = keep
        return self

    def solve(self, nthread: int = 0, ncache: Optional[int] = 64, keep_neighbours: bool = True,
              keep_weights: bool = False):
        if self.nsim > 0:
            return self._solve_sim()
        P, keep = self._problem(nthread=nthread, ncache=64 if ncache is None else ncache)
        nb, nv = P.nblock, self.nvar
        mmax = 1
        for v in range(nv):
            o = self.obs[v]
            sec = self.search[v][5]
            nm = min(o["nmax"], o["coord"].shape[0])
            need = o["coord"].shape[0] > nm
            m = (2 ** self.ndim) * nm if (sec and need) else (nm if need else o["coord"].shape[0])
            mmax = max(mmax, m)
        self.value = np.full((nb, nv), np.nan)
        self.variance = np.full((nb, nv, nv), np.nan)
        self.nnear = np.zeros((nb, nv), dtype=np.int32) if keep_neighbours else None
        self.inear = np.zeros((nb, nv, mmax), dtype=np.int32) if keep_neighbours else None
        self.weight = np.zeros((nb, nv, nv, mmax)) if keep_weights else None
        R = _Result()
        R.value = _dp(self.value)
        R.variance = _dp(self.variance)
        if keep_neighbours:
            R.nnear = self.nnear.ctypes.data_as(_PI)
            R.inear = self.inear.ctypes.data_as(_PI)
        if keep_weights:
            R.weight = _dp(self.weight)
        R.mmax = mmax
        ierr = lib().orc_solve(ctypes.byref(P), ctypes.byref(R))
        self.stats = dict(zip(["fail", "chol_fact", "chol_reuse", "ssytrf_fact", "ssytrf_reuse"],
                              list(R.stats)))
        if ierr:
            raise RuntimeError(R.errmsg.decode())
        self._keep = keep
        return self

    @property
    def solver_stats(self):
        return self.stats

    def get_results(self, squeeze: bool = True):
        est = self.value.copy()
        var = self.variance.copy()
        if self.nsim > 0:  # (nblock, nsim) realisations, (nblock,) conditional variance
            return (est[:, 0] if squeeze and self.nsim == 1 else est), var
        if squeeze and self.nvar == 1:
            return est[:, 0], var[:, 0, 0]
        return est, var

    def neighbours(self, ib, ivar=1):
        """1-based sorted neighbour indices of block ib (0-based) for variable ivar."""
        n = self.nnear[ib, ivar - 1]
        return self.inear[ib, ivar - 1, :n].copy()


class OracleSpaceTime(OracleKriging):
    """Oracle twin of the reference ``SpaceTimeKriging`` class."""

    st = True

    def __init__(self, ndim: int = 2, nvar: int = 1, ndrift: int = 0, unbias: int = 1,
                 anisotropic_search: bool = False, neglect_error: bool = True, **kw):
        super().__init__(ndim=ndim, nvar=nvar, ndrift=ndrift, unbias=unbias,
                         anisotropic_search=anisotropic_search, neglect_error=neglect_error,
                         std_ck=True, **kw)
        self.nlag = ndim + 1
        self.st_params = dict(model=1, transform=VTYPES["lin"], at=1.0, k_ps=0.0,
                              time_nugget=0.0, time_sill=1.0)
        self.joint = {}

    def set_st_model(self, model="product_sum", transform="linear", at=1.0, k_ps=0.0,
                     time_nugget=0.0, time_sill=1.0):
        m = {"sum_metric": 0, "product_sum": 1}[model] if isinstance(model, str) else int(model)
        tmap = {"linear": "lin", "bounded": "exp", "power": "pow"}
        t = VTYPES[tmap.get(transform, transform)[:3]] if isinstance(transform, str) else int(transform)
        self.st_params = dict(model=m, transform=t, at=at, k_ps=k_ps, time_nugget=time_nugget,
                              time_sill=time_sill)

    def set_vgm_temporal(self, ivar, jvar, vtype="sph", nugget=0.0, sill=1.0, at_k=1.0):
        a, b = min(ivar, jvar) - 1, max(ivar, jvar) - 1
        self.vgm_t.setdefault((a, b), []).append(
            (VTYPES[vtype.lower()[:3]], nugget, sill, at_k, at_k, at_k, 0.0, 0.0, 0.0, 0))

    def set_vgm_joint_sills(self, ivar, jvar, sills):
        a, b = min(ivar, jvar) - 1, max(ivar, jvar) - 1
        self.joint[(a, b)] = list(np.atleast_1d(sills).astype(float))

    def set_obs(self, ivar, coord, value, variance=None, nmax=None, maxdist=None, sk_mean=0.0):
        super().set_obs(ivar, np.asarray(coord, dtype=np.float64).reshape(len(value), self.nlag),
                        value, variance, nmax, maxdist, sk_mean)

    def set_grid(self, coord=None, time=None, rangescale=None, localnugget=None):
        c = np.asarray(coord, dtype=np.float64).reshape(-1, self.ndim)
        full = np.column_stack([c, np.asarray(time, dtype=np.float64).reshape(-1)])
        super().set_grid(full, rangescale=rangescale, localnugget=localnugget)

    def set_grid_nodes(self, coord, time, nblockpnt, node_coord, node_time, pointweight):
        """Block targets with explicit integration nodes (krige_st_set_grid_block)."""
        c = np.column_stack([np.asarray(coord, dtype=np.float64).reshape(-1, self.ndim),
                             np.asarray(time, dtype=np.float64).reshape(-1)])
        g = np.column_stack([np.asarray(node_coord, dtype=np.float64).reshape(-1, self.ndim),
                             np.asarray(node_time, dtype=np.float64).reshape(-1)])
        self.grid = dict(coord=np.ascontiguousarray(c),
                         nblockpnt=np.ascontiguousarray(nblockpnt, dtype=np.int32),
                         gcoord=np.ascontiguousarray(g),
                         gweight=np.ascontiguousarray(pointweight, dtype=np.float64),
                         rangescale=None, localnugget=None)

    def set_search(self, ivar=1, anis1=1.0, anis2=1.0, azimuth=0.0, dip=0.0, plunge=0.0,
                   time_at=1.0, sector_search=False):
        self.search[ivar - 1] = (anis1, anis2, azimuth, dip, plunge, int(bool(sector_search)),
                                 time_at)

    def _fill_st(self, P):
        P.st = 1
        sp = self.st_params
        P.st_model, P.st_transform = sp["model"], sp["transform"]
        P.st_at, P.st_k_ps = sp["at"], sp["k_ps"]
        P.st_time_nugget, P.st_time_sill = sp["time_nugget"], sp["time_sill"]
        for (a, b), specs in self.vgm_t.items():
            for (x, y) in ((a, b), (b, a)):
                P.nstruct_t[x][y] = len(specs)
                for k, s in enumerate(specs):
                    P.vgm_t[x][y][k] = _Spec(*s)
        for (a, b), sills in self.joint.items():
            for (x, y) in ((a, b), (b, a)):
                P.st_has_joint[x][y] = 1
                for k, s in enumerate(sills):
                    P.st_joint[x][y][k] = s


def calc_rotmat(az, dip, plunge, anis1, anis2):
    out = np.zeros(9)
    lib().orc_calc_rotmat(az, dip, plunge, anis1, anis2, _dp(out))
    return out.reshape(3, 3, order="F")


def kdtree_nn(data, qv, nn, sort=False):
    """kd-tree n-nearest over data (n, dim); returns (dis, 1-based idx)."""
    data = np.ascontiguousarray(data, dtype=np.float64)
    n, dim = data.shape
    qv = np.ascontiguousarray(qv, dtype=np.float64)
    dis = np.zeros(nn)
    idx = np.zeros(nn, dtype=np.int32)
    lib().orc_kdtree_nn(_dp(data), dim, n, _dp(qv), nn, int(sort), _dp(dis),
                        idx.ctypes.data_as(_PI))
    return dis, idx
