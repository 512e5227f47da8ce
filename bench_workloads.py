"""Seeded synthetic workloads with the shapes of the five benchmark configurations.

No public dataset is involved: each configuration is generated from
``numpy.random.default_rng(1000 * c + k)`` (k = 1 locations, 2 field, 3 noise,
4+ extras) with the sizes, variograms and search parameters of the kriging
benchmark configurations:

  1. 2-D ordinary kriging, 2 000 obs, 100 x 100 targets, spherical, maxdist 0.3, nmax 32
  2. 2-D anisotropic ordinary kriging, 200 000 clustered obs, 2000 x 2000 targets,
     exponential, 4-sector search with 16 per sector
  3. 3-D kriging with 2 external drifts, 500 000 obs, 256 x 256 x 64 targets,
     Gaussian with nugget 1e-3, vertical anisotropy 0.1, nmax 48
  4. 2-variable LMC cokriging (std_ck), 50 000 + 500 000 obs, 2048 x 2048 targets
  5. space-time product-sum, 1 000 stations x 365 days, 512 x 512 x 24 targets,
     4 x 4 block support on 10 % of the targets

``scale`` shrinks the target grid (and optionally the observations) for
parity tests that the CPU oracle finishes in seconds.
"""
from __future__ import annotations

import numpy as np


def cosine_field(rng, ndim, ell, nterm=256):
    """sqrt(2/n) * sum cos(k_m . x + phi_m), k_m ~ N(0, ell^-2 I)."""
    k = rng.normal(0.0, 1.0 / ell, size=(nterm, ndim))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=nterm)
    amp = np.sqrt(2.0 / nterm)

    def f(x):
        x = np.atleast_2d(x)
        out = np.empty(x.shape[0])
        for s in range(0, x.shape[0], 65536):
            out[s:s + 65536] = amp * np.cos(x[s:s + 65536] @ k.T + phi).sum(axis=1)
        return out
    return f


def _centres(n, lo=0.0, hi=1.0):
    return lo + (np.arange(n) + 0.5) * (hi - lo) / n


def _grid2(nx, ny):
    gx, gy = np.meshgrid(_centres(nx), _centres(ny), indexing="xy")
    return np.column_stack([gx.ravel(), gy.ravel()])


def config1(grid_n=100, nobs=2000):
    c = 1
    r1, r2, r3 = (np.random.default_rng(1000 * c + k) for k in (1, 2, 3))
    obs = r1.uniform(0, 1, (nobs, 2))
    z = cosine_field(r2, 2, 0.2)(obs) + r3.normal(0, 0.05, nobs)
    return dict(name="cfg1_ok2d", ndim=2, nvar=1, kw={}, obs=[dict(coord=obs, value=z, nmax=32, maxdist=0.3)],
                vgm=[(1, 1, dict(vtype="sph", nugget=0.05, sill=1.0, a_major=0.25))],
                search=[dict()], grid=_grid2(grid_n, grid_n), nmin=4, zstd=float(np.std(z)), sill=1.05)


def config2(grid_n=2000, nobs=200_000, nclusters=50):
    c = 2
    r1, r2 = (np.random.default_rng(1000 * c + k) for k in (1, 2))
    centres = r1.uniform(0, 1, (nclusters, 2))
    ncl = int(round(0.8 * nobs))
    which = r1.integers(0, nclusters, ncl)
    obs = np.vstack([centres[which] + r1.normal(0, 0.01, (ncl, 2)), r1.uniform(0, 1, (nobs - ncl, 2))])
    z = cosine_field(r2, 2, 0.2)(obs)
    return dict(name="cfg2_ok2d_aniso_sector", ndim=2, nvar=1, kw=dict(anisotropic_search=True),
                obs=[dict(coord=obs, value=z, nmax=16)],
                vgm=[(1, 1, dict(vtype="exp", nugget=0.02, sill=1.0, a_major=0.1, a_minor1=0.05, azimuth=30.0))],
                search=[dict(anis1=0.5, azimuth=30.0, sector_search=True)], grid=_grid2(grid_n, grid_n),
                nmin=4, zstd=float(np.std(z)), sill=1.02)


def config3(grid_n=(256, 256, 64), nobs=500_000):
    c = 3
    r1, r2, r3, r4 = (np.random.default_rng(1000 * c + k) for k in (1, 2, 3, 4))
    obs = np.column_stack([r1.uniform(0, 1, nobs), r1.uniform(0, 1, nobs), r1.uniform(0, 0.25, nobs)])
    f1, f2 = cosine_field(r2, 3, 0.3), cosine_field(r4, 3, 0.3)
    res = cosine_field(r3, 3, 0.08)
    d1, d2 = f1(obs), f2(obs)
    z = 0.7 * d1 - 0.3 * d2 + res(obs)
    nx, ny, nz = grid_n
    gx, gy, gz = np.meshgrid(_centres(nx), _centres(ny), _centres(nz, 0.0, 0.25), indexing="ij")
    grid = np.column_stack([gx.ravel(), gy.ravel(), gz.ravel()])
    gd = np.column_stack([f1(grid), f2(grid)])
    return dict(name="cfg3_ked3d", ndim=3, nvar=1, kw=dict(ndrift=2, anisotropic_search=True),
                obs=[dict(coord=obs, value=z, nmax=48, drift=np.column_stack([d1, d2]))],
                vgm=[(1, 1, dict(vtype="gau", nugget=1e-3, sill=1.0, a_major=0.08, a_minor2=0.008))],
                search=[dict(anis2=0.1)], grid=grid, grid_drift=gd, nmin=4, zstd=float(np.std(z)), sill=1.001)


def config4(grid_n=2048, nobs=(50_000, 500_000)):
    c = 4
    r1, r2, r3 = (np.random.default_rng(1000 * c + k) for k in (1, 2, 3))
    o1 = r1.uniform(0, 1, (nobs[0], 2))
    o2 = r1.uniform(0, 1, (nobs[1], 2))
    fa, fb = cosine_field(r2, 2, 0.15), cosine_field(r3, 2, 0.15)
    rho = 0.7
    z1 = fa(o1)
    z2 = rho * fa(o2) + np.sqrt(1 - rho ** 2) * fb(o2)
    nug = dict(vtype="nug", a_major=1.0)
    vgm = []
    for (i, j), (bn, bs, be) in {(1, 1): (0.05, 0.5, 0.45), (1, 2): (0.035, 0.35, 0.315),
                                 (2, 2): (0.05, 0.5, 0.45)}.items():
        vgm.append((i, j, dict(nug, nugget=bn, sill=0.0)))
        vgm.append((i, j, dict(vtype="sph", nugget=0.0, sill=bs, a_major=0.15)))
        vgm.append((i, j, dict(vtype="exp", nugget=0.0, sill=be, a_major=0.4)))
    return dict(name="cfg4_lmc_cokriging", ndim=2, nvar=2, kw=dict(std_ck=True),
                obs=[dict(coord=o1, value=z1, nmax=32), dict(coord=o2, value=z2, nmax=32)],
                vgm=vgm, search=[dict(), dict()], grid=_grid2(grid_n, grid_n), nmin=4,
                zstd=float(np.std(z1)), sill=1.0)


def config5(grid_n=512, ntimes=24, nstations=1000, ndays=365, block_every=10):
    c = 5
    r1, r2, r3 = (np.random.default_rng(1000 * c + k) for k in (1, 2, 3))
    st = r1.uniform(0, 1, (nstations, 2))
    days = np.arange(ndays, dtype=np.float64)
    obs = np.column_stack([np.repeat(st, ndays, axis=0), np.tile(days, nstations)])
    fs = cosine_field(r2, 2, 0.2)
    ft = cosine_field(r2, 1, 10.0)
    z = fs(obs[:, :2]) * (1.0 + 0.5 * ft(obs[:, 2:3])) + r3.normal(0, 0.05, obs.shape[0])
    g2 = _grid2(grid_n, grid_n)
    tt = (np.arange(ntimes) + 0.5) * 365.0 / ntimes
    grid = np.column_stack([np.tile(g2, (ntimes, 1)), np.repeat(tt, g2.shape[0])])
    return dict(name="cfg5_st_productsum", ndim=2, nvar=1, st=True, kw={},
                obs=[dict(coord=obs, value=z, nmax=64)],
                st_model=dict(model="product_sum", transform="linear", at=1.0, k_ps=0.5),
                vgm=[(1, 1, dict(vtype="exp", nugget=0.05, sill=0.6, a_major=0.2))],
                vgm_t=[(1, 1, dict(vtype="sph", nugget=0.0, sill=0.4, at_k=10.0))],
                search=[dict(time_at=0.02)], grid=grid, cell=1.0 / grid_n, block_every=block_every,
                nmin=4, zstd=float(np.std(z)), sill=0.65 + 0.4 + 0.5 * 0.65 * 0.4)


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}


def apply(k, w, set_grid=True):
    """Configure a Kriging-like object (product or oracle) from a workload dict."""
    for iv, o in enumerate(w["obs"], start=1):
        k.set_obs(iv, o["coord"], o["value"], nmax=o.get("nmax"), maxdist=o.get("maxdist"))
        if "drift" in o:
            k.set_obs_drift(iv, o["drift"])
    for (i, j, spec) in w["vgm"]:
        k.set_vgm(i, j, **spec)
    if set_grid:
        k.set_grid(w["grid"])
        if "grid_drift" in w:
            k.set_grid_drift(w["grid_drift"])
    for iv, s in enumerate(w["search"], start=1):
        k.set_search(iv, **s)
    return k


GQ4_FRAC = np.array([0.4305681558, 0.1699905218, -0.1699905218, -0.4305681558])  # gaussian_quadrature.f90
GQ4_W = np.array([0.1739274226, 0.3260725774, 0.3260725774, 0.1739274226])


def st_blocks(w, pad3d=False):
    """Space-time targets of a config-5 workload as blocks: every block_every-th
    target carries 4 x 4 Gauss-quadrature nodes over its grid cell at the
    target time, the others one node at the target."""
    g = w["grid"]
    nd = g.shape[1] - 1
    cell = w["cell"]
    blk = (np.arange(len(g)) % w["block_every"]) == 0
    nbp = np.where(blk, 16, 1).astype(np.int32)
    ox, oy = np.meshgrid(GQ4_FRAC * cell, GQ4_FRAC * cell, indexing="ij")
    wq = np.outer(GQ4_W, GQ4_W).ravel()
    owner = np.repeat(np.arange(len(g)), nbp)          # target of each node, in target order
    within = np.arange(len(owner)) - np.repeat(np.cumsum(nbp) - nbp, nbp)
    isb = blk[owner]
    nodes = g[owner, :2].copy()
    nodes[isb, 0] += ox.ravel()[within[isb]]
    nodes[isb, 1] += oy.ravel()[within[isb]]
    ntime = g[owner, nd]
    wts = np.where(isb, wq[np.where(isb, within, 0)], 1.0)
    coord = g[:, :nd]
    if pad3d:
        coord = np.column_stack([coord, np.zeros(len(coord))])
        nodes = np.column_stack([nodes, np.zeros(len(nodes))])
    return dict(coord=coord, time=g[:, nd], nblockpnt=nbp, node_coord=nodes, node_time=ntime, weight=wts)


def apply_st(k, w, blocks=True, pad3d=False, set_grid=True):
    """Configure a space-time kriging object (product or oracle) from a config-5 workload."""
    m = w["st_model"]
    k.set_st_model(model=m["model"], transform=m["transform"], at=m["at"], k_ps=m["k_ps"])
    o = w["obs"][0]
    c = o["coord"]
    if pad3d:  # 2-D stations written as 3-D with z = 0, as the reference engine takes them
        c = np.column_stack([c[:, :2], np.zeros(len(c)), c[:, 2]])
    k.set_obs(1, c, o["value"], nmax=o.get("nmax"), maxdist=o.get("maxdist"))
    for (i, j, spec) in w["vgm"]:
        k.set_vgm(i, j, **spec)
    for (i, j, spec) in w["vgm_t"]:
        k.set_vgm_temporal(i, j, **spec)
    if set_grid:
        b = st_blocks(w, pad3d)
        if blocks:
            set_st_blocks(k, b)
        else:
            k.set_grid(b["coord"], time=b["time"])
    for iv, s in enumerate(w["search"], start=1):
        k.set_search(iv, **s)
    return k


def set_st_blocks(k, b):
    """Block targets on a product (set_grid_block) or oracle (set_grid_nodes) object."""
    if hasattr(k, "set_grid_nodes"):
        k.set_grid_nodes(b["coord"], b["time"], b["nblockpnt"], b["node_coord"], b["node_time"], b["weight"])
    else:
        k.set_grid_block(b["coord"], b["time"], b["nblockpnt"], b["node_coord"], b["node_time"], b["weight"])


def st_block_subset(b, idx):
    """The blocks idx (and their nodes) of a st_blocks() dict."""
    idx = np.asarray(idx)
    nbp = b["nblockpnt"]
    start = np.concatenate([[0], np.cumsum(nbp)[:-1]])
    cnt = nbp[idx]
    first = np.repeat(start[idx], cnt)
    within = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    nodes = first + within
    return dict(coord=b["coord"][idx], time=b["time"][idx], nblockpnt=cnt.astype(np.int32),
                node_coord=b["node_coord"][nodes], node_time=b["node_time"][nodes], weight=b["weight"][nodes])


class Workload:
    """One configuration at a given size, configured onto the product classes
    or the CPU oracle for any subset of its targets."""

    def __init__(self, c, grid=None, nmax=None):
        self.c = c
        if c == 1:
            self.w = config1(grid_n=grid or 100)
        elif c == 2:
            self.w = config2(grid_n=grid or 2000)
        elif c == 3:
            g = grid or 256
            self.w = config3(grid_n=(g, g, max(1, g // 4)))
        elif c == 4:
            self.w = config4(grid_n=grid or 2048)
        elif c == 5:
            self.w = config5(grid_n=grid or 512)
        else:
            raise ValueError(f"unknown configuration {c}")
        if nmax is not None:  # neighbours per variable (per sector in sector search)
            for o in self.w["obs"]:
                o["nmax"] = int(nmax)
            self.w["name"] += f"_nmax{int(nmax)}"
        self.st = bool(self.w.get("st", False))
        self.blocks = st_blocks(self.w) if self.st else None
        self.ntarget = len(self.w["grid"])
        self.nobs = int(sum(len(o["coord"]) for o in self.w["obs"]))

    @property
    def name(self):
        return self.w["name"]

    def pq(self):
        """(drift + unbiasedness rows, variables) of one system."""
        kw = self.w["kw"]
        q = self.w["nvar"]
        aug = q if kw.get("std_ck", False) or self.st else 1
        return kw.get("ndrift", 0) + aug, q

    def ndim(self):
        return self.w["ndim"]

    autotune = None  # kernel plan of the product objects (None: the library default)

    def product(self, precision, nmin=None, idx=None, **extra):
        from krigekit_b200 import Kriging, SpaceTimeKriging
        nmin = self.w["nmin"] if nmin is None else nmin
        if self.st:
            k = SpaceTimeKriging(nvar=1, precision=precision, nmin=nmin, **extra)
        else:
            k = Kriging(ndim=self.w["ndim"], nvar=self.w["nvar"], precision=precision, nmin=nmin, **self.w["kw"],
                        **extra)
        if self.autotune is not None:
            k.set_autotune(self.autotune)
        return self.configure(k, idx)

    def oracle(self, nmin=None, idx=None):
        from oracle.oracle import OracleKriging, OracleSpaceTime
        nmin = self.w["nmin"] if nmin is None else nmin
        if self.st:
            k = OracleSpaceTime(ndim=2, nmin=nmin)
        else:
            k = OracleKriging(ndim=self.w["ndim"], nvar=self.w["nvar"], nmin=nmin, **self.w["kw"])
        return self.configure(k, idx)

    def configure(self, k, idx=None):
        """Observations, variograms, targets and search of this workload on k."""
        w = self.w
        if self.st:
            apply_st(k, w, set_grid=False)
        else:
            apply(k, w, set_grid=False)
        self.set_targets(k, idx)
        return k

    def targets(self, idx=None):
        """Host arrays of the targets idx (all by default), built once per idx:
        a caller holds its targets already, so building them is not part of a
        solve."""
        key = None if idx is None else (len(idx), int(idx[0]) if len(idx) else 0, int(idx[-1]) if len(idx) else 0)
        cache = self.__dict__.setdefault("_tcache", {})
        if key in cache:
            return cache[key]
        w = self.w
        sel = np.arange(self.ntarget) if idx is None else np.asarray(idx)
        if self.st:
            t = dict(blocks=st_block_subset(self.blocks, sel))
        else:
            t = dict(grid=np.ascontiguousarray(w["grid"][sel]))
            if "grid_drift" in w:
                t["grid_drift"] = np.ascontiguousarray(w["grid_drift"][sel])
        cache.clear()
        cache[key] = t
        return t

    def set_targets(self, k, idx=None):
        """Targets idx (all by default) on k; returns the host bytes passed."""
        t = self.targets(idx)
        if self.st:
            set_st_blocks(k, t["blocks"])
            return sum(a.nbytes for a in t["blocks"].values())
        k.set_grid(t["grid"])
        nbytes = t["grid"].nbytes
        if "grid_drift" in t:
            k.set_grid_drift(t["grid_drift"])
            nbytes += t["grid_drift"].nbytes
        return nbytes

    def set_data(self, k, idx=None):
        """What a caller passes for every solve: observations, targets, search.
        Variograms stay on k.  Returns the host bytes passed."""
        w = self.w
        nbytes = 0
        for iv, o in enumerate(w["obs"], start=1):
            k.set_obs(iv, o["coord"], o["value"], nmax=o.get("nmax"), maxdist=o.get("maxdist"))
            nbytes += o["coord"].nbytes + o["value"].nbytes
            if "drift" in o:
                k.set_obs_drift(iv, o["drift"])
                nbytes += o["drift"].nbytes
        nbytes += self.set_targets(k, idx)
        for iv, s in enumerate(w["search"], start=1):
            k.set_search(iv, **s)
        return nbytes

    def describe(self):
        o = self.w["obs"][0]
        s = self.w["search"][0]
        parts = [f"nmax {o.get('nmax')}"]
        if s.get("sector_search"):
            parts.append(f"{2 ** self.w['ndim']} sectors x {o.get('nmax')}")
        if self.w["kw"].get("anisotropic_search"):
            parts.append(f"anisotropic search {s}")
        if self.st:
            parts.append(f"time_at {s.get('time_at')}, block support on 1/{self.w['block_every']} of the targets")
        return ", ".join(parts)


def rel_err(x, ref, floor):
    """|x - ref| / max(|ref|, floor), NaN-aware (NaN in both counts as equal)."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    both_nan = np.isnan(x) & np.isnan(ref)
    e = np.abs(x - ref) / np.maximum(np.abs(ref), floor)
    e[both_nan] = 0.0
    e[np.isnan(e)] = np.inf
    return e
