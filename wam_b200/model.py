"""Host-side mirror of the reference module interface for the hot path.

The reference's "operator API" is a set of Fortran module procedures
(wam_source_module.f90 / wam_propagation_module.f90).  `WamModel` exposes the
same procedures with the same argument meaning on top of libwamgpu's C ABI:

    PREPARE_PROPAGATION          -> WamModel.prepare_propagation()
    PREPARE_SOURCE(DEPTH)        -> WamModel.prepare_source()
    IMPLSCH(FL3, U10, UDIR, TAUW, USTAR, Z0, ROAIRN, WSTAR, DEPTH, INDEP)
                                 -> WamModel.implsch(...)        (host arrays)
    PROPAGS(F3)                  -> WamModel.propags(F3)         (host array)

plus device-resident forms (`implsch_dev`, `propags_dev`) that take torch CUDA
tensors.  Errors raise WamgpuError where the reference calls ABORT1.
Spectra use the reference layout FL3(IJ,K,M) (sea point fastest): as a numpy
array that is shape (NSEA, KL, ML) in Fortran order, or equivalently a
C-contiguous (ML, KL, NSEA) array.
"""
import ctypes

import numpy as np

from ._lib import RestartDates, WamgpuConfig, WamgpuError, load

_PF = ctypes.POINTER(ctypes.c_float)
OUT_NPARAM = 40  # WAMGPU_OUT_NPARAM
_PI = ctypes.POINTER(ctypes.c_int)


def effective_parameters(iphys, ml, betamax=1.20, cdfac=1.13):
    """Module parameters after INITMDL (initmdl.f90:153-160, wam_general_module.f90:63-74)."""
    if iphys == 1:
        zalp, alpha, tauwshelter = 0.0080, 0.0062, 0.25
    else:
        zalp, alpha, tauwshelter = 0.0080, 0.0060, 0.0
    if ml <= 30:
        alpha = 0.0075
    return dict(betamax=betamax, zalp=zalp, alpha=alpha, tauwshelter=tauwshelter, cdfac=cdfac)


def make_config(kl, ml, fr1, iphys, idelt, idelpro, delphi, shallow_run=True, spherical_run=True,
                refraction_d_run=False, refraction_c_run=False, reduced_grid=False, isnonlin=0, lcflx=False,
                betamax=1.20, cdfac=1.13, iref=1, ndepth=69, deptha=1.0, depthd=1.1, precision=4, device=0):
    """Configuration dict (field names of struct wamgpu_config)."""
    cfg = dict(kl=kl, ml=ml, fr1=fr1, iref=iref, iphys=iphys, shallow_run=int(shallow_run),
               spherical_run=int(spherical_run), refraction_d_run=int(refraction_d_run),
               refraction_c_run=int(refraction_c_run), reduced_grid=int(reduced_grid), isnonlin=isnonlin,
               lcflx=int(lcflx), idelt=idelt, idelpro=idelpro, ndepth=ndepth, deptha=deptha, depthd=depthd,
               delphi=float(delphi), precision=precision, device=device)
    cfg.update(effective_parameters(iphys, ml, betamax, cdfac))
    return cfg


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a):
    return a.ctypes.data_as(_PF)


def _ip(a):
    return a.ctypes.data_as(_PI)


class WamModel:
    """One rank's slab of sea points on one GPU (one context, one stream)."""

    def __init__(self, cfg: dict):
        self.L = load()
        fields = {f for f, _ in WamgpuConfig._fields_}
        c = WamgpuConfig(**{k: v for k, v in cfg.items() if k in fields})
        self.cfg = dict(cfg)
        self.kl, self.ml = cfg["kl"], cfg["ml"]
        self.dtype = np.float64 if cfg.get("precision", 4) == 8 else np.float32
        h = ctypes.c_void_p()
        rc = self.L.wamgpu_create(ctypes.byref(c), ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.wamgpu_last_error(h).decode() if h else "wamgpu_create failed"
            if h:
                self.L.wamgpu_destroy(h)
            self.h = None
            raise WamgpuError(f"wamgpu_create: {msg} ({rc})")
        self.nsea = 0
        self.counter = 1
        self.total_cfl = 0.0

    def close(self):
        if getattr(self, "h", None):
            self.L.wamgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise WamgpuError(f"{what}: {self.L.wamgpu_last_error(self.h).decode()} ({rc})")

    # ---- tables and grid -------------------------------------------------
    def table(self, name):
        n = self.L.wamgpu_get_table(self.h, name.encode(), None, None)
        if n < 0:
            raise KeyError(name)
        f = np.zeros(n, np.float32)
        i = np.zeros(n, np.int32)
        self.L.wamgpu_get_table(self.h, name.encode(), _fp(f), _ip(i))
        return i if name in ("IKP", "IKP1", "IKM", "IKM1", "K1W", "K2W", "K11W", "K21W", "INLCOEF", "INDICESSAT",
                             "DIA_SCALARS", "INDEP") else f

    def set_grid(self, g):
        """Grid-module arrays (dict from wam_b200.grid.regular_grid or equivalent)."""
        n = int(g["nsea"])
        self._g = {k: np.ascontiguousarray(g[k], np.int32) for k in ("klat", "klon", "kfromij")}
        self._g.update({k: _f32(g[k]) for k in ("wlat", "sinph", "cosph", "dellam")})
        G = self._g
        self._check(self.L.wamgpu_set_grid(self.h, n, _ip(G["klat"]), _ip(G["klon"]), _fp(G["wlat"]),
                                           _ip(G["kfromij"]), len(G["sinph"]), _fp(G["sinph"]), _fp(G["cosph"]),
                                           _fp(G["dellam"])), "set_grid")
        self.nsea = n

    def set_depth(self, depth):
        self._check(self.L.wamgpu_set_depth(self.h, _fp(_f32(depth))), "set_depth")

    def set_current(self, u=None, v=None):
        uu = None if u is None else _f32(u)
        vv = None if v is None else _f32(v)
        self._check(self.L.wamgpu_set_current(self.h, _fp(uu) if uu is not None else None,
                                              _fp(vv) if vv is not None else None), "set_current")

    def prepare_propagation(self):
        """PREPARE_PROPAGATION incl. CHECK_CFL; returns (total_cfl, COUNTER)."""
        cfl = ctypes.c_float()
        cnt = ctypes.c_int()
        self._check(self.L.wamgpu_prepare_propagation(self.h, ctypes.byref(cfl), ctypes.byref(cnt)),
                    "prepare_propagation")
        self.total_cfl, self.counter = cfl.value, cnt.value
        return self.total_cfl, self.counter

    def prepare_source(self):
        self._check(self.L.wamgpu_prepare_source(self.h), "prepare_source")

    def indep(self):
        out = np.zeros(self.nsea, np.int32)
        self._check(self.L.wamgpu_get_indep(self.h, _ip(out)), "get_indep")
        return out

    # ---- reference-facing procedures on host arrays ------------------------
    def implsch(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth=None, indep=None):
        """IMPLSCH in place on float32 host arrays (fl3 Fortran-ordered (NSEA,KL,ML))."""
        for a in (fl3, tauw, ustar, z0):
            if not (a.dtype == np.float32 and (a.flags.f_contiguous or a.ndim == 1)):
                raise WamgpuError("IMPLSCH in/out arrays must be float32 and Fortran-contiguous")
        args = [_fp(fl3), _fp(_keep(self, u10)), _fp(_keep(self, udir)), _fp(tauw), _fp(ustar), _fp(z0),
                _fp(_keep(self, roairn)), _fp(_keep(self, wstar)),
                _fp(_keep(self, depth)) if depth is not None else None,
                _ip(np.ascontiguousarray(indep, np.int32)) if indep is not None else None]
        self._check(self.L.wamgpu_implsch_host(self.h, *args), "implsch")
        self._kept = []

    def set_diagnostics(self, decisions=None, llws=None, ld=None):
        """Test diagnostics of IMPLSCH's integer decisions (wamgpu_set_diagnostics):
        decisions an int32 CUDA tensor (4, ld), llws None or a uint8 CUDA
        tensor (2, ML, KL, ld); decisions=None switches them off."""
        if decisions is None:
            self._check(self.L.wamgpu_set_diagnostics(self.h, None, None, 0), "set_diagnostics")
            return
        ld = decisions.shape[-1] if ld is None else ld
        self._check(self.L.wamgpu_set_diagnostics(self.h, decisions.data_ptr(),
                                                  None if llws is None else llws.data_ptr(), int(ld)),
                    "set_diagnostics")

    def implsch_decisions(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar):
        """implsch() that also returns the step's integer decisions: JU, MIJ1,
        MIJ2 (first and last FRCUTINDEX), LFIT (LFACTOR iterations, -1 for
        ST4) as int arrays of NSEA, and the LLWS masks of the first and the
        last SINPUT call (LLWS1, LLWS2, uint8 shaped like FL3)."""
        import torch
        dev = torch.device("cuda", int(self.cfg.get("device", 0)))
        n = self.nsea
        dg = torch.full((4, n), -99, dtype=torch.int32, device=dev)
        ll = torch.full((2, self.ml, self.kl, n), 7, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize(dev)
        self.set_diagnostics(dg, ll, n)
        try:
            self.implsch(fl3, u10, udir, tauw, ustar, z0, roairn, wstar)
        finally:
            self.set_diagnostics(None)
        d, m = dg.cpu().numpy(), ll.cpu().numpy()
        return dict(JU=d[0], MIJ1=d[1], MIJ2=d[2], LFIT=d[3], LLWS1=np.asfortranarray(m[0].transpose(2, 1, 0)),
                    LLWS2=np.asfortranarray(m[1].transpose(2, 1, 0)))

    def propags(self, f3):
        if not (f3.dtype == np.float32 and f3.flags.f_contiguous):
            raise WamgpuError("PROPAGS array must be float32 and Fortran-contiguous")
        self._check(self.L.wamgpu_propags_host(self.h, _fp(f3)), "propags")

    def fluxes(self):
        out = np.zeros(7 * self.nsea, np.float32)
        self._check(self.L.wamgpu_get_fluxes(self.h, _fp(out)), "get_fluxes")
        return out.reshape(7, self.nsea)

    # ---- device-resident forms (torch CUDA tensors) ------------------------
    def implsch_dev(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, ld=None, stream=None):
        """fl3: tensor of shape (ML, KL, ld) (contiguous, sea point fastest)."""
        ld = fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_implsch_dev(self.h, fl3.data_ptr(), ld, u10.data_ptr(), udir.data_ptr(),
                                              tauw.data_ptr(), ustar.data_ptr(), z0.data_ptr(), roairn.data_ptr(),
                                              wstar.data_ptr(), s), "implsch_dev")

    def propags_dev(self, f3, ld=None, scratch=None, stream=None):
        ld = f3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        sc = None if scratch is None else ctypes.c_void_p(scratch.data_ptr())
        self._check(self.L.wamgpu_propags_dev(self.h, f3.data_ptr(), ld, sc, s), "propags_dev")

    def output_parameters_dev(self, fl3, u10, udir, tauw, ustar, z0, block=None, from_=True, ld=None, stream=None):
        """COMPUTE_OUTPUT_PARAMETER on the device: returns block, a tensor
        (WAMGPU_OUT_NPARAM, ld) whose row IP-1 holds the reference's output
        parameter IP (9 Hs, 11 mean period, 12 TM1, 13 TM2, 10 peak period,
        14 mean direction, ...); USTAR and Z0 are set by AIRSEA when USTAR is
        zero everywhere."""
        import torch
        ld = fl3.shape[-1] if ld is None else ld
        if block is None:
            block = torch.empty((OUT_NPARAM, ld), dtype=fl3.dtype, device=fl3.device)
        s = None if stream is None else ctypes.c_void_p(stream)
        p = lambda t: t.data_ptr()
        self._check(self.L.wamgpu_output_parameters_dev(self.h, p(fl3), ld, p(u10), p(udir), p(tauw), p(ustar), p(z0),
                                                        int(bool(from_)), p(block), block.shape[-1], s),
                    "output_parameters_dev")
        return block

    def output_swell_dev(self, fl3, udir, ustar, block, from_=True, ld=None, stream=None):
        """SWELL_SEPARATION on the device: rows 16..22 and 24..30 of block
        (wind-sea and swell parameters 17-23, 25-31); returns block."""
        ld = fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_output_swell_dev(self.h, fl3.data_ptr(), ld, udir.data_ptr(), ustar.data_ptr(),
                                                   int(bool(from_)), block.data_ptr(), block.shape[-1], s),
                    "output_swell_dev")
        return block

    def restart_write(self, path, fl3, u10, udir, tauw, dates, depth=None, u=None, v=None, ij2newij=None, ld=None):
        """SAVE_RESTART_FILE from device tensors; dates: dict of CDTPRO, CDTSOU,
        CDA, CDTA, CDCA strings (blank = not stored)."""
        d = RestartDates(**{k.lower(): str(dates.get(k, "")).ljust(14)[:14].encode() for k in
                            ("CDTPRO", "CDTSOU", "CDA", "CDTA", "CDCA")})
        ld = fl3.shape[-1] if ld is None else ld
        p = lambda t: None if t is None else t.data_ptr()
        perm = None if ij2newij is None else np.ascontiguousarray(ij2newij, np.int32)
        self._check(self.L.wamgpu_restart_write(self.h, str(path).encode(), p(fl3), ld, p(u10), p(udir), p(tauw),
                                                p(depth), p(u), p(v), ctypes.byref(d),
                                                None if perm is None else _ip(perm)), "restart_write")

    def restart_read(self, path, fl3, u10, udir, tauw, depth=None, u=None, v=None, ij2newij=None, ld=None):
        """CONNECT_RESTART into device tensors; returns the dates."""
        d = RestartDates()
        ld = fl3.shape[-1] if ld is None else ld
        p = lambda t: None if t is None else t.data_ptr()
        perm = None if ij2newij is None else np.ascontiguousarray(ij2newij, np.int32)
        self._check(self.L.wamgpu_restart_read(self.h, str(path).encode(), p(fl3), ld, p(u10), p(udir), p(tauw),
                                               p(depth), p(u), p(v), ctypes.byref(d),
                                               None if perm is None else _ip(perm)), "restart_read")
        return {k.upper(): getattr(d, k).decode() for k in ("cdtpro", "cdtsou", "cda", "cdta", "cdca")}

    def set_wind_grid(self, grid, nx_in, ny_in, west_in, south_in, dx_in, dy_in, periodic=False, equal_grid=False):
        """Interpolation tables from a wind input grid (integer 1/100 arc-second
        units) to the sea points of `grid` (wamgpu_set_wind_grid)."""
        ny = int(grid["ny"])
        zdello = np.ascontiguousarray(np.broadcast_to(np.asarray(grid.get("zdello", grid["xdello"])), (ny,)), np.int32)
        ifromij = np.ascontiguousarray(grid["ixlg"], np.int32)
        self._check(self.L.wamgpu_set_wind_grid(self.h, int(nx_in), int(ny_in), int(west_in), int(south_in), int(dx_in),
                                                int(dy_in), int(bool(periodic)), int(bool(equal_grid)),
                                                int(grid["amowep"]), int(grid["amosop"]), int(grid["xdella"]),
                                                _ip(zdello), _ip(ifromij)), "set_wind_grid")

    def wind_dev(self, u_in, v_in, u10, udir, code_in=3, stream=None):
        """WAM_WIND on the device: input components (tensors (ny_in, nx_in),
        longitude fastest) to U10 and UDIR of every sea point."""
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_wind_dev(self.h, u_in.data_ptr(), v_in.data_ptr(), int(code_in), u10.data_ptr(),
                                           udir.data_ptr(), s), "wind_dev")

    def put_points_dev(self, data, points, value=0.0, ld=None, stream=None):
        """PUT_ICE / PUT_DRY on a device tensor shaped (..., ld) with the sea
        point fastest (a spectrum (ML, KL, ld) or a parameter block): every
        row at the 1-based sea points `points` (an int32 CUDA tensor) becomes
        `value`; points outside the owned range are skipped."""
        ld = data.shape[-1] if ld is None else ld
        nrows = data.numel() // data.shape[-1]
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_put_points_dev(self.h, data.data_ptr(), ld, nrows, points.data_ptr(),
                                                 int(points.numel()), float(value), s), "put_points_dev")

    def propags_dev_static(self, f3, ld=None, stream=None):
        """PROPAGS through the fixed per-device scratch (no allocation; calls
        overlapping on one device race, spectra above WAMGPU_STATIC_SCRATCH_BYTES
        are rejected)."""
        ld = f3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_propags_dev_static(self.h, f3.data_ptr(), ld, s), "propags_dev_static")

    def step(self, fl3, nprop, u10, udir, tauw, ustar, z0, roairn, wstar):
        """nprop x PROPAGS then IMPLSCH on host arrays (one H2D and one D2H of FL3)."""
        for a in (fl3, tauw, ustar, z0):
            if a.dtype != np.float32:
                raise WamgpuError("step arrays must be float32")
        self._check(self.L.wamgpu_step_host(self.h, _fp(fl3), int(nprop), _fp(_keep(self, u10)), _fp(_keep(self, udir)),
                                            _fp(tauw), _fp(ustar), _fp(z0), _fp(_keep(self, roairn)),
                                            _fp(_keep(self, wstar))), "step")
        self._kept = []

    def step_dev(self, fl3, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, scratch=None, ld=None, stream=None):
        """nprop x PROPAGS then IMPLSCH on device tensors; fl3 shape (ML, KL, ld)."""
        ld = fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        sc = None if scratch is None else ctypes.c_void_p(scratch.data_ptr())
        self._check(self.L.wamgpu_step_dev(self.h, fl3.data_ptr(), ld, sc, int(nprop), u10.data_ptr(), udir.data_ptr(),
                                           tauw.data_ptr(), ustar.data_ptr(), z0.data_ptr(), roairn.data_ptr(),
                                           wstar.data_ptr(), s), "step_dev")

    # ---- latitude bands (one grid over several ranks) -----------------------
    def set_owned(self, i0, i1):
        """Only sea points i0..i1-1 are updated; the others are halo points."""
        self._check(self.L.wamgpu_set_owned(self.h, int(i0), int(i1)), "set_owned")

    def set_counter(self, counter):
        """Install the COUNTER agreed over all ranks (not below this grid's own)."""
        self._check(self.L.wamgpu_set_counter(self.h, int(counter)), "set_counter")
        self.counter = int(counter)

    def propags_substep_dev(self, src, dst, ld=None, stream=None):
        """One PROPAGS sub-step src -> dst (device tensors shaped (ML, KL, ld))."""
        ld = src.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_propags_substep_dev(self.h, src.data_ptr(), dst.data_ptr(), ld, s), "propags_substep")

    def propags_substep_range_dev(self, src, dst, i0, i1, ld=None, stream=None):
        """One PROPAGS sub-step over the points i0..i1-1 of the owned range."""
        ld = src.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_propags_substep_range_dev(self.h, src.data_ptr(), dst.data_ptr(), ld, int(i0), int(i1),
                                                            s), "propags_substep_range")

    def halo_width(self):
        """Largest |neighbour - point| over KLAT/KLON, in sea points."""
        w = self.L.wamgpu_get_halo_width(self.h)
        self._check(0 if w >= 0 else w, "get_halo_width")
        return w

    # ---- derivatives (ST4) ---------------------------------------------------
    def implsch_tl_dev(self, fl3, dfl3, tauw, dtauw, u10, du10, udir, roairn, wstar,
                       fl3_out, dfl3_out, tauw_out, dtauw_out, ld=None, stream=None):
        """IMPLSCH and its tangent-linear: (FL3, TAUW, U10) + perturbations ->
        new (FL3, TAUW) + perturbations. Spectra shaped (ML, KL, ld)."""
        ld = fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        p = lambda t: t.data_ptr()
        self._check(self.L.wamgpu_implsch_tl_dev(self.h, p(fl3), p(dfl3), ld, p(tauw), p(dtauw), p(u10), p(du10),
                                                 p(udir), p(roairn), p(wstar), p(fl3_out), p(dfl3_out), p(tauw_out),
                                                 p(dtauw_out), s), "implsch_tl_dev")

    def implsch_adj_dev(self, fl3, tauw, u10, udir, roairn, wstar, lam_fl3, lam_tauw, lam_u10, ld=None, stream=None):
        """Adjoint of IMPLSCH at the checkpoint (FL3, TAUW, U10): lam_fl3 and
        lam_tauw map in place from the new state's adjoints to the old
        state's; lam_u10 is overwritten with the adjoint of U10."""
        ld = fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        p = lambda t: t.data_ptr()
        self._check(self.L.wamgpu_implsch_adj_dev(self.h, p(fl3), ld, p(tauw), p(u10), p(udir), p(roairn), p(wstar),
                                                  p(lam_fl3), p(lam_tauw), p(lam_u10), s), "implsch_adj_dev")

    def propags_adj_dev(self, lam, ld=None, scratch=None, stream=None):
        """Transpose of propags_dev (all COUNTER sub-steps), in place on lam."""
        ld = lam.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        sc = None if scratch is None else ctypes.c_void_p(scratch.data_ptr())
        self._check(self.L.wamgpu_propags_adj_dev(self.h, lam.data_ptr(), ld, sc, s), "propags_adj_dev")

    # ---- checkpointed assimilation windows --------------------------------------
    def checkpoint_reserve(self, n, ld):
        """Room for n checkpoints of spectra with leading dimension ld (0 releases)."""
        self._check(self.L.wamgpu_checkpoint_reserve(self.h, int(n), int(ld)), "checkpoint_reserve")

    def step_ckpt_dev(self, slot, fl3, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, scratch=None, ld=None,
                      stream=None):
        """step_dev that also stores checkpoint `slot` (IMPLSCH's input spectrum, TAUW, U10)."""
        ld = fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        sc = None if scratch is None else ctypes.c_void_p(scratch.data_ptr())
        p = lambda t: t.data_ptr()
        self._check(self.L.wamgpu_step_ckpt_dev(self.h, int(slot), p(fl3), ld, sc, int(nprop), p(u10), p(udir), p(tauw),
                                                p(ustar), p(z0), p(roairn), p(wstar), s), "step_ckpt_dev")

    def step_adj_dev(self, slot, nprop, lam_fl3, lam_tauw, lam_u10, udir, roairn, wstar, scratch=None, ld=None,
                     stream=None):
        """Adjoint of the step stored in `slot`: lam_fl3, lam_tauw in place; lam_u10 written."""
        ld = lam_fl3.shape[-1] if ld is None else ld
        s = None if stream is None else ctypes.c_void_p(stream)
        sc = None if scratch is None else ctypes.c_void_p(scratch.data_ptr())
        p = lambda t: t.data_ptr()
        self._check(self.L.wamgpu_step_adj_dev(self.h, int(slot), int(nprop), p(lam_fl3), ld, p(lam_tauw), p(lam_u10),
                                               p(udir), p(roairn), p(wstar), sc, s), "step_adj_dev")

    def set_timing(self, enable=True):
        self._check(self.L.wamgpu_set_timing(self.h, int(enable)), "set_timing")

    def timing(self):
        """{'propags': (ms, launches), 'implsch': (ms, launches)} since the last call."""
        ms = np.zeros(2, np.float32)
        cnt = np.zeros(2, np.int32)
        self._check(self.L.wamgpu_get_timing(self.h, _fp(ms), _ip(cnt)), "get_timing")
        return {"propags": (float(ms[0]), int(cnt[0])), "implsch": (float(ms[1]), int(cnt[1]))}

    def sync(self):
        self._check(self.L.wamgpu_sync(self.h), "sync")


def _keep(model, a):
    arr = _f32(a)
    if not hasattr(model, "_kept"):
        model._kept = []
    model._kept.append(arr)
    return arr
