"""Drop-in ``IndicatorKriging`` (multiple indicator kriging) over the B200 library.

Mirrors the reference wrapper ougx/krigekit src/krigekit/kriging_indicator.py
(class ``IndicatorKriging`` :54-412): the K categories are K indicator
variables of a cokriging system on a ``krige_ind_create`` handle, whose solve
ends with the category probabilities of every target clipped to [0, 1] and
normalised to sum to one (post_solve_indicator,
src/libkriging/kriging_indicator.F90:170-185), on the GPU like the rest of the
solve.  Variables past ``ncat`` are secondary continuous co-variates.
Sequential indicator simulation (``nsim > 0``) is not part of this library.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import _lib
from .kriging import Kriging


class IndicatorKriging(Kriging):
    """Multiple indicator kriging of ``ncat`` categories (drop-in for krigekit.IndicatorKriging)."""

    _CREATE = "krige_ind_create"

    def __init__(self, ncat: int, nvar: Optional[int] = None, ndim: int = 2, ndrift: int = 0, unbias: int = 1,
                 nsim: int = 0, **kw):
        nvar = nvar if nvar is not None else ncat
        if nvar < ncat:
            raise ValueError(f"nvar ({nvar}) must be >= ncat ({ncat})")
        if nsim:
            raise ValueError("sequential indicator simulation (nsim > 0) is not part of the GPU kriging path")
        super().__init__(ndim=ndim, nvar=nvar, ndrift=ndrift, unbias=unbias, nsim=nsim, **kw)
        if ncat < nvar:
            _lib.call("krige_ind_set_ncat", self._h(), int(ncat))
        self.ncat = ncat

    def set_categorical_obs(self, coord, categories, category_labels=None, nmax: int = 32,
                            maxdist: Optional[float] = None, variance=None):
        """K binary indicator datasets from category labels (kriging_indicator.py:239-292)."""
        cats = np.asarray(categories)
        if category_labels is None:
            category_labels = sorted(np.unique(cats).tolist())
        if len(category_labels) != self.ncat:
            raise ValueError(f"len(category_labels)={len(category_labels)} must equal ncat={self.ncat}")
        var_arr = np.zeros(len(cats)) if variance is None else np.asarray(variance, dtype=np.float64)
        for k, label in enumerate(category_labels, start=1):
            self.set_obs(ivar=k, coord=coord, value=(cats == label).astype(np.float64), variance=var_arr,
                         nmax=nmax, maxdist=maxdist)

    def set_indicator_vgm(self, vtype: str = "sph", nugget: float = 0.0, sill: float = 1.0, a_major: float = 1.0,
                          a_minor1: Optional[float] = None, a_minor2: Optional[float] = None, azimuth: float = 0.0,
                          dip: float = 0.0, plunge: float = 0.0, cross: str = "same", proportions=None):
        """Variograms of all K x K indicator pairs (kriging_indicator.py:294-412).

        ``cross``: "same" (one sill for every pair), "independent" (no cross
        covariance) or "proportional" (auto sills p (1 - p), cross sills
        sqrt(s_k s_l); needs ``proportions``).  Every (ivar, jvar) pair goes
        through ``set_vgm`` in the reference's loop order.
        """
        valid = {"same", "independent", "proportional"}
        if cross not in valid:
            raise ValueError(f"cross must be one of {valid!r}, got {cross!r}")
        if cross == "proportional" and proportions is None:
            raise ValueError("cross='proportional' requires proportions to be supplied")
        if proportions is not None and cross != "same":
            p = np.asarray(proportions, dtype=float)
            if len(p) != self.ncat:
                raise ValueError(f"len(proportions)={len(p)} must equal ncat={self.ncat}")
            auto = p * (1.0 - p)
        else:
            auto = np.full(self.ncat, sill)
        for iv in range(1, self.ncat + 1):
            for jv in range(1, self.ncat + 1):
                if iv == jv:
                    ps, pn = float(auto[iv - 1]), nugget
                elif cross == "independent":
                    ps, pn = 0.0, 0.0
                elif cross == "proportional":
                    ps, pn = float(np.sqrt(auto[iv - 1] * auto[jv - 1])), nugget
                else:
                    ps, pn = sill, nugget
                self.set_vgm(ivar=iv, jvar=jv, vtype=vtype, nugget=pn, sill=ps, a_major=a_major,
                             a_minor1=a_minor1, a_minor2=a_minor2, azimuth=azimuth, dip=dip, plunge=plunge)

    def __repr__(self):
        return f"IndicatorKriging(ncat={self.ncat}, nvar={self.nvar}, ndim={self.ndim}, device={self.device})"
