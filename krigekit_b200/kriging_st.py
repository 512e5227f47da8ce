"""Drop-in ``SpaceTimeKriging`` class over the B200 kriging library.

Mirrors the reference wrapper ougx/krigekit src/krigekit/kriging_st.py
(class ``SpaceTimeKriging`` :275-1000, helpers ``spacetime_kriging`` /
``spacetime_cokriging`` :1003-1140): the same constructor flags, setters and
coordinate conventions -- observation coordinates ``(nobs, ndim+1)`` with time
in the last column, or spatial ``(n, ndim)`` plus a separate ``time`` array.
Every call goes to ``libkrigecuda.so`` through its ``krige_st_*`` entry points
(kriging_st_capi.f90); there is no CPU path.

Extensions: ``precision``, ``nmin`` and ``device`` as in :class:`Kriging`, and
:meth:`set_grid_block` for block support (the reference binds
``krige_st_set_grid_block`` but has no Python method for it).
"""
from __future__ import annotations

import ctypes
import random
import sys
from typing import Optional

import numpy as np

from . import _lib
from .kriging import _PRECISION, _dptr, _farray, _fempty, _iptr

_VTYPE_ALIASES = {"linear": "lin", "bounded": "exp", "power": "pow"}


def _normalize_vtype(s: str) -> str:
    s = str(s).lower()
    return _VTYPE_ALIASES.get(s, s)


def _split_coords(coord, time, n_expected=None):
    """Combined (n, ndim+1) or split (n, ndim) + time -> (spatial (n, ndim), time (n,))."""
    a = np.asarray(coord, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError(f"coord must be 2-D, got shape {a.shape}")
    if time is None:
        if a.shape[1] not in (2, 3, 4):
            raise ValueError(f"Combined coord must be (n, ndim+1) with ndim=1,2,3, got {a.shape}")
        spatial, t = a[:, :-1], a[:, -1]
    else:
        if a.shape[1] not in (1, 2, 3):
            raise ValueError(f"Split coord must be (n, ndim) with ndim=1,2,3, got {a.shape}")
        spatial, t = a, np.asarray(time, dtype=np.float64).ravel()
        if len(t) != len(spatial):
            raise ValueError(f"time length ({len(t)}) != n ({len(spatial)})")
    return spatial, t


class SpaceTimeKriging:
    """Space-time kriging on one B200 (drop-in for krigekit.SpaceTimeKriging)."""

    def __init__(
        self,
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
        verbose: bool = False,
        weight_file: str = "",
        bounds: Optional[tuple] = None,
        seed: Optional[int] = None,
        precision: str = "auto",
        nmin: int = 0,
        device: Optional[int] = None,
    ):
        lib = _lib.load()
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("krigekit_b200 needs a CUDA device (B200); none is visible")
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        dev = torch.cuda.current_device() if device is None else int(device)
        _lib.use_torch_allocator()
        h = ctypes.c_int64(0)
        _lib.check(lib.krige_st_create(ctypes.byref(h)), "krige_st_create")
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
        _lib.call("krige_st_initialize", self._h(), nvar, ndrift, unbias, nsim, int(anisotropic_search),
                  int(weight_correction), int(use_old_weight), int(store_weight), int(cross_validation),
                  int(write_mat), int(neglect_error), int(verbose),
                  weight_file.encode("utf-8") if weight_file else b"", _dptr(c_bounds), int(seed))
        self.nvar, self.ndrift, self.nsim = nvar, ndrift, nsim
        self.verbose = verbose
        self.precision = precision
        self.device = dev
        self.ndim = None  # set by the first set_obs (spatial dimension)
        self._nobs = [0] * nvar

    def _h(self):
        return ctypes.c_int64(self._handle)

    def close(self):
        """Release the handle and its device buffers (krige_st_destroy)."""
        if getattr(self, "_handle", 0):
            h = ctypes.c_int64(self._handle)
            self._handle = 0
            self._lib.krige_st_destroy(ctypes.byref(h))

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ setters
    def set_st_model(self, model: str = "sum_metric", transform: str = "linear", at: float = 1.0,
                     time_nugget: float = 0.0, time_sill: float = 1.0, k_ps: float = 0.0):
        """Global space-time model (kriging_st.py:356-392)."""
        model = model.lower()
        if model not in ("sum_metric", "product_sum"):
            raise ValueError("model must be 'sum_metric' or 'product_sum'")
        _lib.call("krige_st_set_st_model", self._h(), model.encode(), _normalize_vtype(transform).encode(),
                  float(at), float(time_nugget), float(time_sill), float(k_ps))

    def set_obs(self, ivar: int, coord, value, time=None, variance=None, nmax: Optional[int] = None,
                maxdist: Optional[float] = None, sk_mean: float = 0.0):
        """Observations of variable ivar (kriging_st.py:394-489)."""
        spatial, t = _split_coords(coord, time)
        ndim = spatial.shape[1]
        if self.ndim is None:
            self.ndim = ndim
        elif self.ndim != ndim:
            raise ValueError(f"ndim mismatch: object was initialised with ndim={self.ndim} "
                             f"but this coord implies ndim={ndim}")
        nobs = len(spatial)
        coord_f = np.empty((ndim + 1, nobs), dtype=np.float64, order="F")
        coord_f[:ndim, :] = spatial.T
        coord_f[ndim, :] = t
        value_f = _farray(np.asarray(value, dtype=np.float64).ravel())
        if value_f.size != nobs:
            raise ValueError(f"value length ({value_f.size}) != nobs ({nobs})")
        var_f = _farray(variance) if variance is not None else _farray(np.zeros(nobs))
        c_nmax = int(nmax) if nmax is not None else np.iinfo(np.int32).max
        c_maxdist = float(maxdist) if maxdist is not None else sys.float_info.max
        _lib.call("krige_st_set_obs", self._h(), ivar, nobs, ndim, _dptr(coord_f), _dptr(value_f), _dptr(var_f),
                  c_nmax, c_maxdist, float(sk_mean))
        self._nobs[ivar - 1] = nobs

    def update_obs_value(self, ivar: int, value):
        if ivar < 1 or ivar > self.nvar:
            raise ValueError(f"ivar must be in [1, {self.nvar}], got {ivar}")
        value_f = _farray(np.asarray(value, dtype=np.float64).ravel())
        _lib.call("krige_update_obs_value", self._h(), ivar, value_f.size, _dptr(value_f))

    def set_obs_drift(self, ivar: int, drift):
        drift_f = _farray(np.asarray(drift, dtype=np.float64).T)
        _lib.call("krige_set_obs_drift", self._h(), ivar, drift_f.shape[0], drift_f.shape[1], _dptr(drift_f))

    def set_vgm(self, ivar: int, jvar: int, vtype: str, nugget: float = 0.0, sill: float = 1.0,
                a_major: float = 1.0, a_minor1: Optional[float] = None, a_minor2: Optional[float] = None,
                azimuth: float = 0.0, dip: float = 0.0, plunge: float = 0.0):
        """One spatial nested structure of vgm(ivar, jvar) (kriging_st.py:595-618)."""
        if a_minor1 is None:
            a_minor1 = a_major
        if a_minor2 is None:
            a_minor2 = a_minor1
        _lib.call("krige_st_set_vgm", self._h(), ivar, jvar, str(vtype).encode(), float(nugget), float(sill),
                  float(a_major), float(a_minor1), float(a_minor2), float(azimuth), float(dip), float(plunge))

    def set_vgm_temporal(self, ivar: int, jvar: int, vtype: str, nugget: float = 0.0, sill: float = 1.0,
                         at_k: float = 1.0):
        """One temporal nested structure of vgm(ivar, jvar) (kriging_st.py:620-636)."""
        _lib.call("krige_st_set_vgm_temporal", self._h(), ivar, jvar, str(vtype).encode(), float(nugget),
                  float(sill), float(at_k))

    def set_vgm_joint_sills(self, ivar: int, jvar: int, *sills: float):
        """Joint sills of the sum-metric model, one per spatial structure (kriging_st.py:638-651)."""
        if len(sills) == 1 and np.ndim(sills[0]) == 1:
            sills = tuple(sills[0])
        arr = _farray(np.asarray(sills, dtype=np.float64))
        _lib.call("krige_st_set_vgm_joint_sills", self._h(), ivar, jvar, len(sills), _dptr(arr))

    def set_grid(self, coord, time=None, rangescale=None, localnugget=None):
        """Point targets (kriging_st.py:653-714)."""
        spatial, t = _split_coords(coord, time)
        coord_f = np.asfortranarray(spatial.T)
        ngrid = coord_f.shape[1]
        # absent rangescale / localnugget: null (all ones / zeros in the library)
        rs_f = _farray(rangescale) if rangescale is not None else None
        ln_f = _farray(localnugget) if localnugget is not None else None
        _lib.call("krige_st_set_grid", self._h(), ngrid, _dptr(coord_f), _dptr(_farray(t)),
                  None if rs_f is None else _dptr(rs_f), None if ln_f is None else _dptr(ln_f))

    def set_grid_block(self, coord, time, nblockpnt, block_coord, block_time, pointweight=None,
                       rangescale=None, localnugget=None):
        """Block targets with explicit integration nodes (krige_st_set_grid_block).

        coord (nblocks, ndim) + time (nblocks) are the block centres (the search
        centres); block_coord (npnts, ndim) + block_time (npnts) the nodes,
        nblockpnt (nblocks) nodes per block, pointweight (npnts) their weights
        (default: equal weights within a block).
        """
        c = np.asfortranarray(np.asarray(coord, dtype=np.float64).T)
        nb = c.shape[1]
        nbp = np.ascontiguousarray(nblockpnt, dtype=np.int32)
        g = np.asfortranarray(np.asarray(block_coord, dtype=np.float64).T)
        npnt = g.shape[1]
        if pointweight is None:
            pointweight = np.repeat(1.0 / nbp, nbp)
        # absent rangescale / localnugget: null (all ones / zeros in the library)
        rs_f = _farray(rangescale) if rangescale is not None else None
        ln_f = _farray(localnugget) if localnugget is not None else None
        _lib.call("krige_st_set_grid_block", self._h(), nb, _dptr(c), _dptr(_farray(np.ravel(time))),
                  _iptr(nbp), npnt, _dptr(g), _dptr(_farray(np.ravel(block_time))),
                  _dptr(_farray(np.ravel(pointweight))), None if rs_f is None else _dptr(rs_f),
                  None if ln_f is None else _dptr(ln_f))

    def set_grid_cv(self):
        """Cross-validation targets at the observations."""
        _lib.call("krige_set_grid_cv", self._h())

    def set_grid_drift(self, drift):
        drift_f = _farray(np.asarray(drift, dtype=np.float64).T)
        _lib.call("krige_st_set_grid_drift", self._h(), drift_f.shape[0], drift_f.shape[1], _dptr(drift_f))

    def set_search(self, ivar: int, time_at: float = 1.0, anis1: float = 1.0, anis2: float = 1.0,
                   azimuth: float = 0.0, dip: float = 0.0, plunge: float = 0.0, sector_search: bool = False):
        """Search of variable ivar; search-space time = t * time_at (kriging_st.py:776-828)."""
        _lib.call("krige_st_set_search", self._h(), ivar, float(time_at), float(anis1), float(anis2),
                  float(azimuth), float(dip), float(plunge), int(bool(sector_search)))

    # -------------------------------------------------------------------- solve
    def solve(self, nthread: int = 0, ncache: Optional[int] = None):
        _lib.call("krige_solve", self._h(), int(nthread), -1 if ncache is None else int(ncache))

    @property
    def solver_stats(self) -> dict:
        """chol_ok, ssytrf_fact, ssytrf_reuse of the last solve (kriging_st.py:897-930)."""
        buf = (ctypes.c_int * 5)()
        self._lib.krige_solver_stats(self._h(), buf)
        return {"chol_ok": buf[1], "ssytrf_fact": buf[3], "ssytrf_reuse": buf[4]}

    def gpu_stats(self) -> dict:
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
                "search_redo": [buf[16 + v] for v in range(4)], "refine_passes": buf[20], "jitter": buf[21]}

    def set_autotune(self, mode: int = 1):
        """Kernel choice per neighbour-count list (extension; krige_set_autotune)."""
        _lib.call("krige_set_autotune", self._h(), int(mode))

    def kernel_plan(self) -> dict:
        """Kernel per neighbour-count list of the last solve (extension)."""
        from .kriging import kernel_plan
        return kernel_plan(self._h())

    def profile(self, enable: bool = True):
        _lib.call("krige_gpu_profile", self._h(), int(bool(enable)))

    def phases(self) -> dict:
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
        """(estimate, variance) of variable 1 as in kriging_st.py:932-975."""
        nb, ns = self._nb(), 1
        estimate = _fempty((nb, ns))
        variance = _fempty(nb)
        _lib.call("krige_get_estimate", self._h(), ns, nb, _dptr(estimate))
        _lib.call("krige_get_variance", self._h(), nb, _dptr(variance))
        est = estimate[:, 0] if squeeze else estimate
        if copy:
            est = np.array(est, order="C", copy=True)
            variance = np.array(variance, order="C", copy=True)
        return est, variance

    def get_neighbours(self, ivar: int = 1):
        """(nnear[nblock], inear[nblock, mmax]) -- 1-based ascending neighbour indices."""
        nb = self._nb()
        mm = ctypes.c_int(0)
        _lib.call("krige_get_mmax", self._h(), ivar, ctypes.byref(mm))
        nnear = np.zeros(nb, dtype=np.int32)
        inear = np.zeros((nb, mm.value), dtype=np.int32)
        _lib.call("krige_get_neighbours", self._h(), ivar, nb, mm.value, _iptr(nnear), _iptr(inear))
        return nnear, inear

    def __repr__(self):
        return f"SpaceTimeKriging(nvar={self.nvar}, ndim={self.ndim}, precision={self.precision!r})"


def spacetime_kriging(obs_coord, obs_value, grid_coord, grid_time, spatial_spec, temporal_spec, joint_sills=(),
                      model: str = "sum_metric", transform: str = "linear", at: float = 1.0,
                      time_nugget: float = 0.0, time_sill: float = 1.0, nmax: int = 20,
                      maxdist: Optional[float] = None, search_anis1: float = 1.0, search_anis2: float = 1.0,
                      search_azimuth: float = 0.0, k_ps: float = 0.0, nthread: int = 0,
                      ncache: Optional[int] = None, **kw):
    """One-shot ordinary space-time kriging (kriging_st.py:1003-1066)."""
    k = SpaceTimeKriging(nvar=1, **kw)
    k.set_st_model(model=model, transform=transform, at=at, time_nugget=time_nugget, time_sill=time_sill,
                   k_ps=k_ps)
    k.set_obs(ivar=1, coord=obs_coord, value=obs_value, nmax=nmax, maxdist=maxdist)
    for spec in ([spatial_spec] if isinstance(spatial_spec, dict) else list(spatial_spec)):
        k.set_vgm(1, 1, **spec)
    for spec in ([temporal_spec] if isinstance(temporal_spec, dict) else list(temporal_spec)):
        k.set_vgm_temporal(1, 1, **spec)
    if model == "sum_metric":
        k.set_vgm_joint_sills(1, 1, *joint_sills)
    k.set_grid(coord=grid_coord, time=grid_time)
    k.set_search(ivar=1, time_at=at, anis1=search_anis1, anis2=search_anis2, azimuth=search_azimuth)
    k.solve(nthread=nthread, ncache=ncache)
    return k.get_results()


def spacetime_cokriging(obs_coords, obs_values, grid_coord, grid_time, spatial_specs: dict, temporal_specs: dict,
                        joint_sills: dict, model: str = "sum_metric", transform: str = "linear", at: float = 1.0,
                        time_nugget: float = 0.0, time_sill: float = 1.0, nmax: int = 20,
                        maxdist: Optional[float] = None, nthread: int = 0, ncache: Optional[int] = None, **kw):
    """One-shot ordinary space-time cokriging (kriging_st.py:1069-1130).

    ``obs_coords`` / ``obs_values``: one array per variable, coordinates
    ``(nobs_i, ndim + 1)`` with time last; ``spatial_specs`` /
    ``temporal_specs``: (ivar, jvar) -> structure dict or list of dicts;
    ``joint_sills``: (ivar, jvar) -> sills of the sum-metric model.
    """
    nvar = len(obs_coords)
    k = SpaceTimeKriging(nvar=nvar, **kw)
    k.set_st_model(model=model, transform=transform, at=at, time_nugget=time_nugget, time_sill=time_sill)
    for i, (coord, value) in enumerate(zip(obs_coords, obs_values), start=1):
        k.set_obs(ivar=i, coord=coord, value=value, nmax=nmax, maxdist=maxdist)
    for (iv, jv), spec in spatial_specs.items():
        for s in ([spec] if isinstance(spec, dict) else list(spec)):
            k.set_vgm(iv, jv, **s)
    for (iv, jv), spec in temporal_specs.items():
        for s in ([spec] if isinstance(spec, dict) else list(spec)):
            k.set_vgm_temporal(iv, jv, **s)
    if model == "sum_metric":
        for (iv, jv), sills in joint_sills.items():
            k.set_vgm_joint_sills(iv, jv, *sills)
    k.set_grid(coord=grid_coord, time=grid_time)
    for i in range(1, nvar + 1):
        k.set_search(ivar=i, time_at=at)
    k.solve(nthread=nthread, ncache=ncache)
    return k.get_results()
