"""Seeded synthetic inputs for the benchmark and parity configurations.

The reference publishes no dataset for this path, so every workload is built
from a seed: a blob land mask (thresholded Gaussian-smoothed noise), a depth
field (Gaussian random field mapped to a depth range), 10 m wind fields and a
JONSWAP start spectrum with cos^2 spreading about the wind
(wam_jonswap_module.f90:136-211 for the spectral shape).

Workloads (names used by bench.py and the tests):
  c0  1 deg 60x40 (20-60N, 40W-20E), ~10% land, 4000 m, KL=24 ML=25 FR1=0.04177,
      ST4, constant wind 5-20 m/s, 900 s / 900 s
  c1  0.1 deg 1200x900 (45S-45N), ~30% land, depth 10-5000 m (correlation 50
      cells), KL=36 ML=30 FR1=0.0345, ST6, depth refraction, hourly wind
      12+-5 m/s, 120 s propagation / 600 s source
  c2  c1 recipe at 400x300 (0.3 deg), ST4, 24 x 600 s (adjoint window)
  c4  0.25 deg 1440x680 (85S-85N), ~35% land, 10-6000 m, KL=36 ML=35 ST4,
      zonal wind profile + eddies, 300 s / 900 s
  c3  ensemble of 32 members (make_ensemble): regional 0.25-1 deg grids of
      2k-150k sea points (log-uniform), KL x ML 24x25 or 36x30, ST4 and ST6
      alternating, each with its own c0-recipe wind (own seed, speed scaled by
      a factor in 0.85-1.15), 4000 m, 900 s / 900 s
Grids can be scaled down (`scale`) for parity tests.
"""
import math

import numpy as np

from .grid import regular_grid
from .model import make_config

G = 9.806
ZPI = 2.0 * 3.1415927


def _smooth(field, sigma):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(field, sigma=sigma, mode="wrap")


def blob_mask(rng, nx, ny, land_frac, sigma):
    """Sea mask (True = sea) with ~land_frac land made of contiguous blobs."""
    n = _smooth(rng.standard_normal((nx, ny)), sigma)
    thr = np.quantile(n, 1.0 - land_frac)
    return n < thr


def grf(rng, nx, ny, corr):
    f = _smooth(rng.standard_normal((nx, ny)), corr)
    f = (f - f.mean()) / (f.std() + 1e-30)
    return f


def jonswap_factors(fr, th, fp, alpha, gamma, sa, sb, udir):
    """Frequency part E(IJ,M) and directional part D(IJ,K) of the start spectrum."""
    fr = np.asarray(fr, np.float64)[None, :]
    fp = np.asarray(fp, np.float64)[:, None]
    alpha = np.broadcast_to(np.asarray(alpha, np.float64), (fp.shape[0],))[:, None]
    arg = 1.25 * (fp / fr) ** 4
    et = np.where(arg < 50.0, alpha * G ** 2 / ZPI ** 4 * fr ** -5 * np.exp(-np.minimum(arg, 50.0)), 0.0)
    sig = np.where(fr > fp, sb, sa)
    a2 = 0.5 * ((fr / fp - 1.0) / sig) ** 2
    et = et * np.where(a2 < 99.0, np.exp(np.log(gamma) * np.exp(-np.minimum(a2, 99.0))), 1.0)
    spr = np.maximum(0.0, np.cos(np.asarray(th)[None, :] - np.asarray(udir)[:, None])) ** 2 * (2.0 / math.pi)
    return et.astype(np.float32), spr.astype(np.float32)


def jonswap_spectrum(fr, th, fp, alpha, gamma, sa, sb, udir):
    """Start spectrum F(IJ,K,M) [NSEA, KL, ML] float32: JONSWAP x cos^2 spreading."""
    et, spr = jonswap_factors(fr, th, fp, alpha, gamma, sa, sb, udir)
    return et[:, None, :] * spr[:, :, None]


def wind_from_uv(u, v):
    """Speed >= 2 m/s and direction ATAN2(U,V) in [0,2pi) (wam_wind_module.f90:1157-1200)."""
    s = np.maximum(np.hypot(u, v), 2.0)
    d = np.mod(np.arctan2(u, v), 2 * math.pi)
    return s.astype(np.float32), d.astype(np.float32)


class Workload:
    """Grid, configuration, fields and start state of one configuration."""

    def __init__(self, name, cfg, grid, depth, u10, udir, e_fm, d_fk, wind_fn=None, n_src_steps=1, sub_steps=1):
        self.name, self.cfg, self.grid = name, cfg, grid
        self.depth, self.u10, self.udir = depth, u10, udir
        self.e_fm, self.d_fk = e_fm, d_fk  # start spectrum = E(IJ,M) * D(IJ,K)
        self.wind_fn = wind_fn
        self.nsea = grid["nsea"]
        self.n_src_steps = n_src_steps
        self.sub_steps = sub_steps  # propagation steps per source step (IDELT/IDELPRO)
        self.tauw = np.zeros(self.nsea, np.float32)
        self.ustar = np.zeros(self.nsea, np.float32)
        self.z0 = np.zeros(self.nsea, np.float32)
        self.roairn = np.full(self.nsea, 1.225, np.float32)
        self.wstar = np.zeros(self.nsea, np.float32)

    def spectrum_f(self):
        """Start FL3 as a Fortran-ordered (NSEA, KL, ML) float32 array."""
        return np.asfortranarray(self.e_fm[:, None, :] * self.d_fk[:, :, None])

    def spectrum_device(self, torch, device, ld=None, dtype=None):
        """Start FL3 on the device as a (ML, KL, ld) tensor (sea point fastest)."""
        ld = self.nsea if ld is None else ld
        dtype = torch.float32 if dtype is None else dtype
        e = torch.tensor(self.e_fm.T, device=device, dtype=dtype)   # (ML, NSEA)
        d = torch.tensor(self.d_fk.T, device=device, dtype=dtype)   # (KL, NSEA)
        f = torch.zeros((self.cfg["ml"], self.cfg["kl"], ld), device=device, dtype=dtype)
        f[:, :, :self.nsea] = e[:, None, :] * d[None, :, :]
        return f


def _finish(name, cfg, g, depth_grid, u_grid, v_grid, rng, seed_fn=None, **kw):
    sea = g["_mask"]
    order = sea.T.ravel()
    depth = depth_grid.T.ravel()[order].astype(np.float32)
    u = u_grid.T.ravel()[order]
    v = v_grid.T.ravel()[order]
    u10, udir = wind_from_uv(u, v)
    fr = cfg["fr1"] * 1.1 ** np.arange(cfg["ml"])
    th = (np.arange(cfg["kl"]) + 0.5) * (2 * math.pi / cfg["kl"])
    e_fm, d_fk = jonswap_factors(fr, th, np.full(g["nsea"], 0.2), 0.018, 3.3, 0.07, 0.09, udir)
    return Workload(name, cfg, g, depth, u10, udir, e_fm, d_fk, **kw)


def vary_sea_state(w, seed=99, fp_range=(0.07, 0.25), wstar_range=(0.0, 1.5)):
    """Start spectra with a per-point peak frequency drawn from fp_range and
    a per-point convective velocity scale WSTAR from wstar_range (the gust
    branch of WSIGSTAR, wam_source_module.f90:4250-4339), so that the
    cut-off index, the wind-sea mask and the gustiness vary over the grid.
    Modifies w in place and returns it."""
    rng = np.random.default_rng(seed)
    cfg = w.cfg
    fr = cfg["fr1"] * 1.1 ** np.arange(cfg["ml"])
    th = (np.arange(cfg["kl"]) + 0.5) * (2 * math.pi / cfg["kl"])
    fp = rng.uniform(fp_range[0], fp_range[1], w.nsea)
    w.e_fm, w.d_fk = jonswap_factors(fr, th, fp, 0.018, 3.3, 0.07, 0.09, w.udir)
    w.wstar = rng.uniform(wstar_range[0], wstar_range[1], w.nsea).astype(np.float32)
    return w


def make_direction_variant(kl, iphys, seed=1234, scale=0.25, precision=4, device=0):
    """The small open-ocean grid of "c0" with KL directions and ST4 (iphys=1)
    or ST6 (iphys=2) source terms.  The direction count decides how the source
    kernels split the directions of a sea point over a warp's 32 lanes (the
    DIA and SDISSIP_ARD take the directions beyond the first 32 in batches
    over frequencies), so the parity tests run KL = 33, 48 and 64 besides the
    configurations' 24 and 36."""
    rng = np.random.default_rng(seed)
    nx, ny = max(8, int(60 * scale)), max(6, int(40 * scale))
    sea = blob_mask(rng, nx, ny, 0.10, 3)
    g = regular_grid(sea, 20.0, -40.0, 40.0 / ny, 60.0 / nx)
    cfg = make_config(kl, 25, 0.04177, iphys, 900, 900, g["delphi"], shallow_run=False, spherical_run=True,
                      betamax=1.42 if iphys == 1 else 1.20, precision=precision, device=device)
    depth = np.full((nx, ny), 4000.0)
    spd = 5 + 15 * _unit(_smooth(rng.random((nx, ny)), 3))
    drc = 2 * math.pi * _unit(_smooth(rng.random((nx, ny)), 3))
    u, v = spd * np.sin(drc), spd * np.cos(drc)
    g["_mask"] = sea
    return _finish(f"c0/kl{kl}/st{4 if iphys == 1 else 6}", cfg, g, depth, u, v, rng, n_src_steps=48, sub_steps=1)


def make_workload(name, seed=1234, scale=1.0, precision=4, device=0):
    rng = np.random.default_rng(seed)
    if name == "c0":
        nx, ny = max(8, int(60 * scale)), max(6, int(40 * scale))
        dlat = dlon = 1.0 * 60 / nx
        sea = blob_mask(rng, nx, ny, 0.10, 3)
        g = regular_grid(sea, 20.0, -40.0, 40.0 / ny, 60.0 / nx)
        cfg = make_config(24, 25, 0.04177, 1, 900, 900, g["delphi"], shallow_run=False, spherical_run=True,
                          betamax=1.42, precision=precision, device=device)
        depth = np.full((nx, ny), 4000.0)
        spd = 5 + 15 * _unit(_smooth(rng.random((nx, ny)), 3))
        drc = 2 * math.pi * _unit(_smooth(rng.random((nx, ny)), 3))
        u, v = spd * np.sin(drc), spd * np.cos(drc)
        g["_mask"] = sea
        return _finish(name, cfg, g, depth, u, v, rng, n_src_steps=48, sub_steps=1)
    if name in ("c1", "c2"):
        if name == "c1":
            nx, ny, south, span_lat, span_lon, iphys = int(1200 * scale), int(900 * scale), -45.0, 90.0, 120.0, 2
        else:
            nx, ny, south, span_lat, span_lon, iphys = int(400 * scale), int(300 * scale), -45.0, 90.0, 120.0, 1
        nx, ny = max(nx, 8), max(ny, 6)
        sea = blob_mask(rng, nx, ny, 0.30, max(2.0, 20 * scale))
        g = regular_grid(sea, south, -60.0, span_lat / ny, span_lon / nx)
        cfg = make_config(36, 30, 0.0345, iphys, 600, 120, g["delphi"], shallow_run=True, spherical_run=True,
                          refraction_d_run=True, betamax=1.42 if iphys == 1 else 1.20,
                          precision=precision, device=device)
        d01 = _unit(grf(rng, nx, ny, max(2.0, 50 * scale)))
        depth = 10.0 * (5000.0 / 10.0) ** d01
        u = 12 + 5 * grf(rng, nx, ny, max(2.0, 20 * scale))
        v = 5 * grf(rng, nx, ny, max(2.0, 20 * scale))
        g["_mask"] = sea
        return _finish(name, cfg, g, depth, u, v, rng, n_src_steps=36 if name == "c1" else 24, sub_steps=5)
    if name == "c4":
        nx, ny = max(16, int(1440 * scale)), max(8, int(680 * scale))
        sea = blob_mask(rng, nx, ny, 0.35, max(2.0, 15 * scale))
        g = regular_grid(sea, -85.0, 0.0, 170.0 / (ny - 1), 360.0 / nx)
        cfg = make_config(36, 35, 0.0345, 1, 900, 300, g["delphi"], shallow_run=True, spherical_run=True,
                          refraction_d_run=True, betamax=1.42, precision=precision, device=device)
        d01 = _unit(grf(rng, nx, ny, max(2.0, 30 * scale)))
        depth = 10.0 * (6000.0 / 10.0) ** d01
        lat = np.asarray(g["lat"])[None, :]
        zon = 10 * np.exp(-((np.abs(lat) - 50) / 12) ** 2) - 7 * np.exp(-((np.abs(lat) - 15) / 8) ** 2)
        u = zon + 4 * grf(rng, nx, ny, max(2.0, 10 * scale))
        v = 4 * grf(rng, nx, ny, max(2.0, 10 * scale))
        g["_mask"] = sea
        return _finish(name, cfg, g, depth, u, v, rng, n_src_steps=96, sub_steps=3)
    raise KeyError(name)


def make_ensemble(n_members=32, seed=777, size_range=(2000, 150000), precision=4, device=0):
    """Members of the batched-ensemble configuration (list of Workload)."""
    rng = np.random.default_rng(seed)
    out = []
    for g in range(n_members):
        target = float(np.exp(rng.uniform(math.log(size_range[0]), math.log(size_range[1]))))
        if rng.random() < 0.5:
            kl, ml, fr1 = 24, 25, 0.04177
        else:
            kl, ml, fr1 = 36, 30, 0.0345
        iphys = 1 if g % 2 == 0 else 2
        ncell = target / 0.9
        nx = max(8, int(math.sqrt(1.5 * ncell)))
        ny = max(6, int(ncell / nx))
        res = min(float(rng.uniform(0.25, 1.0)), 100.0 / ny)
        south = -0.5 * ny * res
        west = float(rng.uniform(-180.0, 180.0 - nx * res))
        sea = blob_mask(rng, nx, ny, 0.10, 3)
        grid = regular_grid(sea, south, west, res, res)
        cfg = make_config(kl, ml, fr1, iphys, 900, 900, grid["delphi"], shallow_run=False, spherical_run=True,
                          betamax=1.42 if iphys == 1 else 1.20, precision=precision, device=device)
        depth = np.full((nx, ny), 4000.0)
        fac = float(rng.uniform(0.85, 1.15))
        spd = fac * (5 + 15 * _unit(_smooth(rng.random((nx, ny)), 3)))
        drc = 2 * math.pi * _unit(_smooth(rng.random((nx, ny)), 3))
        u, v = spd * np.sin(drc), spd * np.cos(drc)
        grid["_mask"] = sea
        out.append(_finish(f"c3/{g}", cfg, grid, depth, u, v, rng, n_src_steps=96, sub_steps=1))
    return out


def _unit(x):
    return (x - x.min()) / (x.max() - x.min() + 1e-30)
