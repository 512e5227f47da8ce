"""Drop-in ``Kriging`` class over the B200 kriging library.

Mirrors the reference wrapper ougx/krigekit src/krigekit/kriging.py
(class ``Kriging`` :403-1985, helpers ``ordinary_kriging`` / ``cokriging``
:1992-2205): same constructor flags and defaults, same setters, the same
``(nobs, ndim)`` array convention transposed to column-major before each
C call, and the same result arrays / DataFrame columns.  Every call goes to
``libkrigecuda.so`` (sm_100a); there is no CPU path.

GPU-specific keyword extensions: ``precision`` ("auto" = per neighbour-count
list the faster of the two forms as timed by the kernel tuner, FP64 when not
tuned; "fp32_refine" = FP32 factorisation with an FP64 residual correction;
"fp64"), ``nmin`` (targets with fewer neighbours give NaN), ``device``.
"""
from __future__ import annotations

import ctypes
import random
import sys
from typing import Optional

import numpy as np

from . import _lib

_c_int = ctypes.c_int
_c_double = ctypes.c_double
_PRECISION = {"fp64": 0, "fp32_refine": 1, "auto": 2}


def _farray(a, dtype=np.float64):
    return np.asfortranarray(a, dtype=dtype)


def _fempty(shape, dtype=np.float64):
    return np.empty(shape, dtype=dtype, order="F")


def _coord_to_fortran(coord) -> np.ndarray:
    """(n, ndim) -> column-major (ndim, n), like kriging.py:342-360."""
    a = np.asarray(coord, dtype=np.float64)
    if a.ndim == 1:
        return np.asfortranarray(a.reshape(-1, 1))
    return np.asfortranarray(a.T)


def _drift_to_fortran(drift) -> np.ndarray:
    return np.asfortranarray(np.asarray(drift, dtype=np.float64).T)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))



KERNELS = ("warp32", "warp64", "block128", "general", "warp32_fp32r", "warp64_fp32r")
PLAN_LISTS = ("npp<=32", "npp<=64", "npp>128", "npp<=128")


def kernel_plan(handle) -> dict:
    """{list: {"kernel": name, "us_per_target": {candidate: us}}} of the last
    solve of a handle (krige_get_kernel_plan); empty lists are left out."""
    nk = len(KERNELS)
    ker = (ctypes.c_int * 4)()
    us = (ctypes.c_double * (4 * nk))()
    _lib.call("krige_get_kernel_plan", handle, ker, us)
    out = {}
    for li, name in enumerate(PLAN_LISTS):
        if ker[li] < 0:
            continue
        timed = {KERNELS[k]: us[li * nk + k] for k in range(nk) if us[li * nk + k] == us[li * nk + k]}
        out[name] = {"kernel": KERNELS[ker[li]], "us_per_target": timed}
    return out


class Kriging:
    """Spatial kriging / cokriging on one B200 (drop-in for krigekit.Kriging)."""

    _CREATE = "krige_create"  # C-ABI constructor of the handle

    def __init__(
        self,
        ndim: int = 2,
        nvar: int = 1,
        ndrift: int = 0,
        unbias: int = 1,
        nsim: int = 0,
        anisotropic_search: bool = False,
        weight_correction: bool = False,
        use_old_weight: bool = False,
        store_weight: bool = False,
        cross_validation: bool = False,
        write_mat: bool = False,
        neglect_error: bool = True,
        varying_vgm: bool = False,
        std_ck: bool = False,
        verbose: bool = False,
        pf_cache: bool = False,
        weight_file: str = "",
        bounds: Optional[tuple] = None,
        seed: Optional[int] = None,
        precision: str = "auto",
        nmin: int = 0,
        device: Optional[int] = None,
    ):
        if store_weight and use_old_weight:
            raise ValueError("store_weight and use_old_weight are mutually exclusive")
        lib = _lib.load()
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("krigekit_b200 needs a CUDA device (B200); none is visible")
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        dev = torch.cuda.current_device() if device is None else int(device)
        _lib.use_torch_allocator()
        h = ctypes.c_int64(0)
        _lib.check(getattr(lib, self._CREATE)(ctypes.byref(h)), self._CREATE)
        self._handle = h.value
        self._lib = lib
        _lib.register(self)
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.call("krige_set_device", self._h(), dev, ctypes.c_void_p(stream))
        _lib.call("krige_set_precision", self._h(), _PRECISION[precision])
        _lib.call("krige_set_nmin", self._h(), int(nmin))
        huge = sys.float_info.max
        c_bounds = _farray(bounds if bounds is not None else [-huge, huge])
        seed = seed or random.randint(0, 2 ** 31 - 1)
        _lib.call("krige_initialize", self._h(), ndim, nvar, ndrift, unbias, nsim,
                  int(anisotropic_search), int(weight_correction), int(use_old_weight),
                  int(store_weight), int(cross_validation), int(write_mat), int(neglect_error),
                  int(varying_vgm), int(std_ck), int(verbose), int(pf_cache),
                  weight_file.encode("utf-8") if weight_file else b"", _dptr(c_bounds), int(seed))
        self.ndim, self.nvar, self.ndrift, self.nsim = ndim, nvar, ndrift, nsim
        self.unbias = unbias
        self.anisotropic_search = anisotropic_search
        self.cross_validation = cross_validation
        self.std_ck = std_ck
        self.verbose = verbose
        self.bounds = c_bounds
        self.seed = seed
        self.precision = precision
        self.device = dev
        self.store_weight = store_weight
        self.use_old_weight = use_old_weight
        self._nblock = 0
        self._nobs = np.zeros(nvar, dtype=np.int64)
        self._nvgm_struct = np.zeros((nvar, nvar), dtype=np.int64)

    def _h(self):
        return ctypes.c_int64(self._handle)

    def close(self):
        """Release the handle and its device buffers (krige_destroy)."""
        if getattr(self, "_handle", 0):
            h = ctypes.c_int64(self._handle)
            self._handle = 0
            self._lib.krige_destroy(ctypes.byref(h))

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ setters
    def set_obs(self, ivar: int, coord, value, variance=None, nmax: Optional[int] = None,
                maxdist: Optional[float] = None, sk_mean: float = 0.0):
        """Observations of variable ivar (kriging.py:592-662)."""
        coord_f = _coord_to_fortran(coord)
        value_f = _farray(np.asarray(value, dtype=np.float64).ravel())
        nobs, ndim_c = coord_f.shape[1], coord_f.shape[0]
        if value_f.size != nobs:
            raise ValueError(f"value length ({value_f.size}) must match nobs ({nobs})")
        if variance is not None:
            var_f = _farray(np.asarray(variance, dtype=np.float64).ravel())
            if var_f.size != nobs:
                raise ValueError(f"variance length ({var_f.size}) must match nobs ({nobs})")
        else:
            var_f = None  # zero measurement variance
        c_nmax = int(nmax) if nmax is not None else np.iinfo(np.int32).max
        c_maxdist = float(maxdist) if maxdist is not None else sys.float_info.max
        _lib.call("krige_set_obs", self._h(), ivar, nobs, ndim_c, _dptr(coord_f), _dptr(value_f),
                  None if var_f is None else _dptr(var_f), c_nmax, c_maxdist, float(sk_mean))
        self._nobs[ivar - 1] = nobs

    def set_obs_drift(self, ivar: int, drift):
        drift_f = _drift_to_fortran(drift)
        _lib.call("krige_set_obs_drift", self._h(), ivar, drift_f.shape[0], drift_f.shape[1], _dptr(drift_f))

    def update_obs_value(self, ivar: int, value):
        value_f = _farray(np.asarray(value, dtype=np.float64).ravel())
        if value_f.size != self._nobs[ivar - 1]:
            raise ValueError(f"value length ({value_f.size}) must match nobs ({self._nobs[ivar - 1]})")
        _lib.call("krige_update_obs_value", self._h(), ivar, value_f.size, _dptr(value_f))

    def set_vgm(self, ivar: int, jvar: int, vtype: str, nugget: float = 0.0, sill: float = 1.0,
                a_major: float = 1.0, a_minor1: Optional[float] = None, a_minor2: Optional[float] = None,
                azimuth: float = 0.0, dip: float = 0.0, plunge: float = 0.0, append: bool = True,
                product: bool = False):
        """One nested structure for the (ivar, jvar) pair (kriging.py:806-891)."""
        if a_minor1 is None:
            a_minor1 = a_major
        if a_minor2 is None:
            a_minor2 = a_minor1
        if not append and self._nvgm_struct[ivar - 1, jvar - 1] > 0:
            _lib.call("krige_reset_vgm", self._h(), ivar, jvar)
            self._nvgm_struct[ivar - 1, jvar - 1] = 0
            self._nvgm_struct[jvar - 1, ivar - 1] = 0
        if jvar < ivar:
            # the reference wrapper's swap (kriging.py:884-887) ends as (ivar, ivar)
            jvar = ivar
        _lib.call("krige_set_vgm", self._h(), ivar, jvar, vtype.lower()[:3].encode("utf-8"),
                  float(nugget), float(sill), float(a_major), float(a_minor1), float(a_minor2),
                  float(azimuth), float(dip), float(plunge), 1 if product else 0)
        self._nvgm_struct[ivar - 1, jvar - 1] += 1
        if ivar != jvar:
            self._nvgm_struct[jvar - 1, ivar - 1] += 1

    def set_grid(self, coord=None, rangescale=None, localnugget=None):
        """Point-kriging targets (kriging.py:947-989)."""
        if coord is None:
            self.set_grid_cv()
            return
        coord_f = _coord_to_fortran(coord)
        ngrid = coord_f.shape[1]
        # absent rangescale / localnugget: null (all ones / zeros in the library)
        rs_f = _farray(rangescale) if rangescale is not None else None
        ln_f = _farray(localnugget) if localnugget is not None else None
        _lib.call("krige_set_grid", self._h(), ngrid, coord_f.shape[0], _dptr(coord_f),
                  None if rs_f is None else _dptr(rs_f), None if ln_f is None else _dptr(ln_f))
        self._nblock = ngrid

    def set_grid_block(self, coord, block_type: int, nblockpnt=None, pointweight=None, blocksize=None,
                       rangescale=None, localnugget=None):
        """Block-kriging targets (kriging.py:992-1081)."""
        coord_f = _coord_to_fortran(coord)
        ngrid, ndim_c = coord_f.shape[1], coord_f.shape[0]
        if block_type == -4:
            nblock = ngrid
            if blocksize is None:
                raise ValueError("blocksize must be specified for Gaussian quadrature blocks.")
            blocksize = np.asarray(blocksize, dtype=np.float64)
            if blocksize.ndim == 1:
                blocksize = np.tile(blocksize, (nblock, 1))
            blocksize_f = _coord_to_fortran(blocksize)
            nbp_f = np.ascontiguousarray(np.ones(nblock, dtype=np.int32))
            pw_f = _farray(np.ones(nblock))
        else:
            nbp_f = np.ascontiguousarray(nblockpnt, dtype=np.int32)
            nblock = len(nbp_f)
            npoint = int(np.sum(nbp_f))
            if np.any(nbp_f <= 0):
                raise ValueError("nblockpnt must contain positive counts")
            if npoint != ngrid:
                raise ValueError(f"sum(nblockpnt) ({npoint}) must match coord rows ({ngrid})")
            blocksize_f = _coord_to_fortran(np.zeros((nblock, self.ndim)))
            if pointweight is not None:
                if len(pointweight) != npoint:
                    raise ValueError(f"pointweight length ({len(pointweight)}) must match sum(nblockpnt) ({npoint})")
                pw_f = _farray(pointweight)
            else:
                pw_f = _farray(np.repeat(1.0 / nbp_f, nbp_f))
        rs_f = _farray(rangescale) if rangescale is not None else _farray(np.ones(nblock))
        ln_f = _farray(localnugget) if localnugget is not None else _farray(np.zeros(nblock))
        _lib.call("krige_set_grid_block", self._h(), int(block_type), ngrid, ndim_c, _dptr(coord_f), nblock,
                  _iptr(nbp_f), _dptr(pw_f), _dptr(blocksize_f), _dptr(rs_f), _dptr(ln_f))
        self._nblock = nblock

    def set_grid_cv(self):
        """Leave-one-out targets at the observations of variable 1."""
        _lib.call("krige_set_grid_cv", self._h())
        self._nblock = int(self._nobs[0])

    def set_grid_drift(self, drift, ivar: Optional[int] = None):
        drift_f = _drift_to_fortran(drift)
        _lib.call("krige_set_grid_drift", self._h(), ivar if ivar is not None else -1,
                  drift_f.shape[0], drift_f.shape[1], _dptr(drift_f))

    def set_search(self, ivar: int = 1, anis1: float = 1.0, anis2: float = 1.0, azimuth: float = 0.0,
                   dip: float = 0.0, plunge: float = 0.0, sector_search: bool = False):
        """Search configuration of variable ivar (kriging.py:1206-1251)."""
        _lib.call("krige_set_search", self._h(), ivar, float(anis1), float(anis2), float(azimuth),
                  float(dip), float(plunge), int(bool(sector_search)))

    # -------------------------------------------------------------------- solve
    def set_sim_draw(self, by_level: bool = False):
        """How the simulation draws its values (extension): every dependency
        level in one launch (default) or one launch per level; the values are
        the same bit for bit."""
        _lib.call("krige_set_sim_draw", self._h(), int(bool(by_level)))

    def set_sim(self, randpath: Optional[np.ndarray] = None, sample: Optional[np.ndarray] = None):
        """Sequential Gaussian simulation: visiting order and N(0, 1) draws
        (kriging.py:1134-1203).  randpath is a 1-based permutation of the
        targets; sample is (nblocks,), (nblocks, nsim) or (nblocks, nvar,
        nsim), row p taken by the p-th visited target.  Either may be None:
        the library then draws them from the constructor's seed (its own
        generator, not the reference's)."""
        if self.nsim <= 0:
            raise AssertionError("nsim must be > 0 when setting SGSIM parameters.")
        nb = self._nb()
        rp_ptr = ctypes.c_void_p(0)
        s_ptr = ctypes.c_void_p(0)
        nsim_c = nvar_c = 0
        nblocks = nb
        keep = []
        if randpath is not None:
            rp = np.ascontiguousarray(np.asarray(randpath, dtype=np.int32).ravel())
            if rp.size != nb:
                raise ValueError(f"randpath length ({rp.size}) must match nblocks ({nb})")
            if not np.array_equal(np.sort(rp), np.arange(1, nb + 1, dtype=np.int32)):
                raise ValueError("randpath must be a 1-based permutation of 1..nblocks")
            rp_ptr = ctypes.c_void_p(rp.ctypes.data)
            keep.append(rp)
        if sample is not None:
            sa = np.asarray(sample, dtype=np.float64)
            if sa.ndim == 1:
                sa = sa[:, np.newaxis, np.newaxis]
            elif sa.ndim == 2:
                sa = sa[:, np.newaxis, :]
            elif sa.ndim != 3:
                raise ValueError(f"sample must be 2-D (nblocks, nsim) or 3-D (nblocks, nvar, nsim), got shape {sa.shape}")
            sf = _drift_to_fortran(sa)  # (nsim, nvar, nblocks) column-major
            nsim_c, nvar_c, n_s = sf.shape
            if nsim_c != self.nsim or nvar_c != self.nvar or n_s != nb:
                raise ValueError(f"sample shape ({nsim_c}, {nvar_c}, {n_s}) must be ({self.nsim}, {self.nvar}, {nb})")
            s_ptr = ctypes.c_void_p(sf.ctypes.data)
            keep.append(sf)
        _lib.call("krige_set_sim", self._h(), nblocks, rp_ptr, nsim_c, nvar_c, s_ptr)
        self._set_sim = True

    def get_sim_neighbours(self, mmax: int):
        """Neighbour sets of the last sequential simulation (extension;
        krige_get_sim_neighbours): (nnear (nblocks, 2) observation and
        simulated members, inear (nblocks, mmax) 0-based in system order:
        observations < nobs, then nobs + visiting position)."""
        nb = self._nb()
        nn = np.zeros((nb, 2), dtype=np.int32)
        inear = np.zeros((nb, mmax), dtype=np.int32)
        _lib.call("krige_get_sim_neighbours", self._h(), nb, int(mmax), _iptr(nn), _iptr(inear))
        return nn, inear

    def solve(self, nthread: int = 0, ncache: Optional[int] = None):
        """Run the kriging solve on the GPU (kriging.py:1321-1344)."""
        _lib.call("krige_solve", self._h(), int(nthread), -1 if ncache is None else int(ncache))

    @property
    def solver_stats(self) -> dict:
        buf = (ctypes.c_int * 5)()
        self._lib.krige_solver_stats(self._h(), buf)
        return {"fail": buf[0], "chol_fact": buf[1], "chol_reuse": buf[2],
                "ssytrf_fact": buf[3], "ssytrf_reuse": buf[4]}

    def gpu_stats(self) -> dict:
        """GPU counters of the last solve (extension)."""
        buf = (ctypes.c_int * 8)()
        ms = ctypes.c_double(0.0)
        _lib.call("krige_gpu_stats", self._h(), buf, ctypes.byref(ms))
        return {"fail": buf[0], "chol": buf[1], "ldlt": buf[3], "search_redo": buf[5],
                "fp64_resolve": buf[6], "refine_iterations": buf[7], "solve_ms": ms.value}

    def gpu_counters(self) -> dict:
        """Raw device counters of the last solve (extension; krige_gpu_counters)."""
        buf = (ctypes.c_int * 32)()
        _lib.call("krige_gpu_counters", self._h(), 32, buf)
        return {"bucket_le32": buf[0], "bucket_le64": buf[1], "bucket_gt128": buf[2], "bucket_le128": buf[22],
                "general_list": buf[3],
                "fp64_resolve": buf[4], "fail": buf[5], "chol": buf[6], "ldlt": buf[7],
                "search_redo": [buf[16 + v] for v in range(4)], "refine_passes": buf[20], "jitter": buf[21],
                "sim_one_launch": buf[24], "sim_levels": buf[25]}

    def set_autotune(self, mode: int = 1):
        """Kernel choice per neighbour-count list (extension; krige_set_autotune):
        0 fixed, 1 timed once per system signature (default), 2 timed again on
        the next solve."""
        _lib.call("krige_set_autotune", self._h(), int(mode))

    def kernel_plan(self) -> dict:
        """Kernel that solved each non-empty neighbour-count list in the last
        solve, with the tuner's microseconds per target of every timed
        candidate (extension; krige_get_kernel_plan)."""
        return kernel_plan(self._h())

    @staticmethod
    def autotune_clear():
        """Forget every cached kernel plan (extension; krige_autotune_clear)."""
        _lib.call("krige_autotune_clear")

    def profile(self, enable: bool = True):
        """Record per-phase device time of each solve (extension)."""
        _lib.call("krige_gpu_profile", self._h(), int(bool(enable)))

    def phases(self) -> dict:
        """Device ms per phase of the last solve and its kernel launches (extension)."""
        out = (ctypes.c_double * 4)()
        nl = ctypes.c_int(0)
        _lib.call("krige_gpu_phases", self._h(), out, ctypes.byref(nl))
        km = (ctypes.c_double * 2)()
        _lib.call("krige_gpu_kernel_ms", self._h(), km)
        return {"search_ms": out[0], "bucket_ms": out[1], "solve_ms": out[2], "fallback_ms": out[3],
                "assemble_ms": km[0], "factor_ms": km[1], "launches": nl.value}

    # ------------------------------------------------------------------ results
    def _nb(self):
        nb = ctypes.c_int(0)
        _lib.call("krige_get_nblocks", self._h(), ctypes.byref(nb))
        return nb.value

    def get_results(self, copy: bool = False, squeeze: bool = True):
        """(estimate, variance) as in kriging.py:1382-1440."""
        nb, nv, ns = self._nb(), self.nvar, max(1, self.nsim)
        estimate = _fempty((nb, nv, ns))
        variance = _fempty((nb, nv, nv))
        _lib.call("krige_get_estimate_all", self._h(), nb, nv, ns, _dptr(estimate))
        _lib.call("krige_get_variance_all", self._h(), nb, nv, _dptr(variance))
        if squeeze:
            if self.nvar == 1:
                estimate = estimate[:, 0]
                variance = variance[:, 0, 0]
            if ns <= 1:
                estimate = estimate[..., 0]
        if copy:
            estimate = np.array(estimate, order="C", copy=True)
            variance = np.array(variance, order="C", copy=True)
        return estimate, variance

    def get_estimate_all(self, copy: bool = False):
        if self.nvar <= 1:
            raise RuntimeError("get_estimate_all is only available for multivariable kriging/simulation (nvar > 1)")
        nb = self._nb()
        out = _fempty((nb, self.nvar, 1))
        _lib.call("krige_get_estimate_all", self._h(), nb, self.nvar, 1, _dptr(out))
        return np.array(out, order="C", copy=True) if copy else out

    def get_result_array(self) -> np.ndarray:
        """Structured array with columns x, y[, z], estimate|est_v*, variance|var_v* (kriging.py:1442-1557)."""
        nblocks, nv, nd = self._nb(), self.nvar, self.ndim
        coord_f = _fempty((nd, nblocks))
        _lib.call("krige_get_block_coord", self._h(), nd, nblocks, _dptr(coord_f))
        coord = np.ascontiguousarray(coord_f.T)
        est_f = _fempty((nblocks, nv, 1))
        _lib.call("krige_get_estimate_all", self._h(), nblocks, nv, 1, _dptr(est_f))
        var_f = _fempty((nblocks, nv, nv))
        _lib.call("krige_get_variance_all", self._h(), nblocks, nv, _dptr(var_f))
        coord_names = ["x", "y", "z"][:nd]
        sim_fields = ["estimate"] if nv == 1 else [f"est_v{iv + 1}" for iv in range(nv)]
        var_fields = ["variance"] if nv == 1 else [f"var_v{iv + 1}" for iv in range(nv)]
        out = np.empty(nblocks, dtype=[(n, np.float64) for n in coord_names + sim_fields + var_fields])
        for i, name in enumerate(coord_names):
            out[name] = coord[:, i]
        for iv, name in enumerate(sim_fields):
            out[name] = est_f[:, iv, 0]
        for iv, name in enumerate(var_fields):
            out[name] = var_f[:, iv, iv]
        return out

    def get_result_df(self):
        import pandas as pd
        return pd.DataFrame(self.get_result_array())

    def get_variance_all(self, copy: bool = False):
        """Conditional covariance matrix of all variables, (nblock, nvar, nvar) (kriging.py:1714-1735)."""
        nb, nv = self._nb(), self.nvar
        out = _fempty((nb, nv, nv))
        _lib.call("krige_get_variance_all", self._h(), nb, nv, _dptr(out))
        return np.array(out, order="C", copy=True) if copy else out

    # ------------------------------------------------------------ weight store
    def free_weight_store(self):
        """Release the in-memory weight store (kriging.py:1746-1749)."""
        _lib.call("krige_free_weight_store", self._h())

    def get_weights(self) -> dict:
        """Stored kriging weights and neighbours (kriging.py:1875-1971).

        Keys ``nnear`` (nblock, ngroups), ``inear`` (nblock, ngroups, nmax,
        1-based, zero-padded), ``weight`` (nblock, nvar, ngroups, nmax) --
        (nblock, ngroups, nmax) for one variable -- and ``variance`` ((nblock,)
        or (nblock, nvar, nvar)).  Needs ``store_weight=True`` and a solve.
        """
        nm, ng, nb = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _lib.call("krige_get_weight_dims", self._h(), ctypes.byref(nm), ctypes.byref(ng), ctypes.byref(nb))
        nm, ng, nb, nv = nm.value, ng.value, nb.value, self.nvar
        nnear_f = np.zeros((ng, nb), dtype=np.int32, order="F")
        inear_f = np.zeros((nm, ng, nb), dtype=np.int32, order="F")
        weight_f = np.zeros((nm, ng, nv, nb), dtype=np.float64, order="F")
        var_f = np.zeros((nv, nv, nb), dtype=np.float64, order="F")
        _lib.call("krige_get_weight_nnear", self._h(), ng, nb, _iptr(nnear_f))
        _lib.call("krige_get_weight_inear", self._h(), nm, ng, nb, _iptr(inear_f))
        _lib.call("krige_get_weight_data", self._h(), nm, ng, nv, nb, _dptr(weight_f))
        _lib.call("krige_get_weight_var", self._h(), nv, nb, _dptr(var_f))
        weight = np.ascontiguousarray(weight_f.T)  # (nb, nv, ng, nm)
        var = np.ascontiguousarray(var_f.T)        # (nb, nv, nv)
        if nv == 1:
            weight = weight[:, 0, :, :]
            var = var[:, 0, 0]
        return {"nnear": np.ascontiguousarray(nnear_f.T), "inear": np.ascontiguousarray(inear_f.T),
                "weight": weight, "variance": var}

    def set_weights(self, weights: dict) -> None:
        """Load a weight store so that solve() re-estimates from it (kriging.py:1752-1873)."""
        if self.store_weight:
            raise ValueError("set_weights() is incompatible with store_weight=True. "
                             "Construct Kriging without store_weight=True when reusing weights.")
        nnear = np.ascontiguousarray(weights["nnear"], dtype=np.int32)
        inear = np.ascontiguousarray(weights["inear"], dtype=np.int32)
        weight = np.asarray(weights["weight"], dtype=np.float64)
        if nnear.ndim != 2:
            raise ValueError("nnear must be 2-D (nblock, ngroups)")
        if inear.ndim != 3:
            raise ValueError("inear must be 3-D (nblock, ngroups, nmax)")
        nb, ng = nnear.shape
        nm = inear.shape[2]
        nv = self.nvar
        if weight.ndim == 3:
            weight_f = np.asfortranarray(weight.T[:, :, np.newaxis, :])
        elif weight.ndim == 4:
            weight_f = np.asfortranarray(np.transpose(weight, (3, 2, 1, 0)))
        else:
            raise ValueError("weight must be 3-D (nblock, ngroups, nmax) or 4-D (nblock, nvar, ngroups, nmax)")
        var = weights.get("variance")
        if var is not None:
            var = np.asarray(var, dtype=np.float64)
            if var.ndim == 1:
                var = var[:, np.newaxis, np.newaxis]
            var_f = np.asfortranarray(np.transpose(var, (1, 2, 0)))
        else:
            var_f = np.zeros((nv, nv, nb), dtype=np.float64, order="F")
        order = np.ascontiguousarray(np.arange(1, nb + 1, dtype=np.int32))
        nnear_f = np.asfortranarray(nnear.T)
        inear_f = np.asfortranarray(inear.T)
        _lib.call("krige_set_weights", self._h(), nm, ng, nv, nb, _iptr(nnear_f), _iptr(inear_f),
                  _dptr(weight_f), _iptr(order), _dptr(var_f))
        self.use_old_weight = True

    def get_info(self) -> str:
        """Configuration summary (kriging.py:1973-1977)."""
        ptr = self._lib.krige_to_str(self._h())
        if not ptr:
            return ""
        return ctypes.cast(ptr, ctypes.c_char_p).value.decode("utf-8", errors="ignore")

    def __str__(self):
        return self.get_info()

    # ------------------------------------------------------------ extensions
    def get_neighbours(self, ivar: int = 1):
        """(nnear[nblock], inear[nblock, mmax]) -- 1-based ascending neighbour indices."""
        nb = self._nb()
        mm = ctypes.c_int(0)
        _lib.call("krige_get_mmax", self._h(), ivar, ctypes.byref(mm))
        nnear = np.zeros(nb, dtype=np.int32)
        inear = np.zeros((nb, mm.value), dtype=np.int32)
        _lib.call("krige_get_neighbours", self._h(), ivar, nb, mm.value, _iptr(nnear), _iptr(inear))
        return nnear, inear

    def get_status(self):
        nb = self._nb()
        st = np.zeros(nb, dtype=np.int32)
        _lib.call("krige_get_status", self._h(), nb, _iptr(st))
        return st

    def __repr__(self):
        return f"Kriging(ndim={self.ndim}, nvar={self.nvar}, precision={self.precision!r}, device={self.device})"


def sequential_gaussian_simulation(obs_coord, obs_value, grid_coord, vgm_spec, nsim: int, nmax=None,
                                   randpath=None, sample=None, seed=None, rangescale=None, localnugget=None,
                                   nthread: int = 0, ncache=None) -> np.ndarray:
    """Sequential Gaussian simulation of one variable (kriging.py:2144-2205):
    (ngrid,) for one realisation, (ngrid, nsim) for several, in target order."""
    obs_coord = np.asarray(obs_coord, dtype=np.float64)
    ndim = obs_coord.shape[1]
    if nmax is None:
        nmax = len(obs_coord) + len(grid_coord)
    k = Kriging(ndim=ndim, nvar=1, nsim=nsim, seed=seed)
    k.set_obs(ivar=1, coord=obs_coord, value=obs_value, nmax=nmax)
    k.set_grid(coord=grid_coord, rangescale=rangescale, localnugget=localnugget)
    for spec in ([vgm_spec] if isinstance(vgm_spec, dict) else list(vgm_spec)):
        k.set_vgm(ivar=1, jvar=1, **spec)
    k.set_sim(randpath, sample)
    k.set_search(ivar=1)
    k.solve(nthread=nthread, ncache=ncache)
    sims, _ = k.get_results()
    return sims


def ordinary_kriging(obs_coord, obs_value, grid_coord, vgm_spec, nmax=None, maxdist=None, search_anis1=1.0,
                     search_anis2=1.0, search_azimuth=0.0, rangescale=None, localnugget=None, nthread=0,
                     ncache=None, **kw):
    """One-shot ordinary kriging (kriging.py:1992-2070)."""
    assert obs_coord.shape[0] == obs_value.shape[0], (
        f"obs_coord has {obs_coord.shape[0]} rows but obs_value has {obs_value.shape[0]} elements.")
    if nmax is None:
        nmax = len(obs_coord) + len(grid_coord)
    ndim = obs_coord.shape[1]
    k = Kriging(ndim=ndim, nvar=1, **kw)
    k.set_obs(ivar=1, coord=obs_coord, value=obs_value, nmax=nmax, maxdist=maxdist)
    k.set_grid(coord=grid_coord, rangescale=rangescale, localnugget=localnugget)
    for spec in ([vgm_spec] if isinstance(vgm_spec, dict) else list(vgm_spec)):
        k.set_vgm(ivar=1, jvar=1, **spec)
    k.set_search(ivar=1, anis1=search_anis1, anis2=search_anis2, azimuth=search_azimuth)
    k.solve(nthread=nthread, ncache=ncache)
    return k.get_results()


def cokriging(obs_coords, obs_values, grid_coord, vgm_spec, nmax=None, rangescale=None, localnugget=None,
              nthread=0, ncache=None, std_ck=False, **kw):
    """One-shot ordinary cokriging (kriging.py:2073-2160).

    ``vgm_spec`` maps (ivar, jvar) pairs (1-based, jvar >= ivar) to a structure
    dict or a list of structure dicts.
    """
    nvar = len(obs_coords)
    ndim = np.asarray(obs_coords[0]).shape[1]
    k = Kriging(ndim=ndim, nvar=nvar, std_ck=std_ck, **kw)
    for iv in range(nvar):
        k.set_obs(ivar=iv + 1, coord=obs_coords[iv], value=obs_values[iv],
                  nmax=nmax if nmax is not None else len(obs_coords[iv]))
    k.set_grid(coord=grid_coord, rangescale=rangescale, localnugget=localnugget)
    for (iv, jv), spec in vgm_spec.items():
        for s in ([spec] if isinstance(spec, dict) else list(spec)):
            k.set_vgm(iv, jv, **s)
    for iv in range(nvar):
        k.set_search(ivar=iv + 1)
    k.solve(nthread=nthread, ncache=ncache)
    return k.get_results()
