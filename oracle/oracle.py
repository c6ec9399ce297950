"""ctypes wrapper around the CPU oracle (oracle/liboracle.so).

ORACLE — test infrastructure only.  Imported by tests/ and by bench.py's
CPU-baseline leg; never by the wam_b200 package.  The oracle is a
statement-order C++ restatement of WAM Cycle 7's IMPLSCH/PROPAGS path and its
table builders (wam_source_module.f90, wam_propagation_module.f90,
wam_fre_dir_module.f90, wam_tables_module.f90, preproc_module.f90).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OracleConfig(ctypes.Structure):
    _fields_ = [("kl", ctypes.c_int), ("ml", ctypes.c_int), ("fr1", ctypes.c_double), ("iref", ctypes.c_int),
                ("iphys", ctypes.c_int), ("shallow_run", ctypes.c_int), ("spherical_run", ctypes.c_int),
                ("refraction_d_run", ctypes.c_int), ("refraction_c_run", ctypes.c_int), ("reduced_grid", ctypes.c_int),
                ("isnonlin", ctypes.c_int), ("lcflx", ctypes.c_int), ("idelt", ctypes.c_int), ("idelpro", ctypes.c_int),
                ("betamax", ctypes.c_double), ("zalp", ctypes.c_double), ("alpha", ctypes.c_double),
                ("tauwshelter", ctypes.c_double), ("cdfac", ctypes.c_double), ("ndepth", ctypes.c_int),
                ("deptha", ctypes.c_double), ("depthd", ctypes.c_double), ("delphi", ctypes.c_double)]


class GridDef(ctypes.Structure):
    _fields_ = [("NX", ctypes.c_int), ("NY", ctypes.c_int), ("AMOSOP", ctypes.c_int), ("AMOWEP", ctypes.c_int),
                ("AMOEAP", ctypes.c_int), ("XDELLA", ctypes.c_int), ("XDELLO", ctypes.c_int),
                ("reduced_grid", ctypes.c_int)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.POINTER(OracleConfig), ctypes.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_get_table.argtypes = [vp, ctypes.c_char_p, dp]
        L.oracle_get_itable.argtypes = [vp, ctypes.c_char_p, ip]
        L.oracle_set_grid.argtypes = [vp, ctypes.c_int, ip, ip, dp, ip, ctypes.c_int, dp, dp, dp, ctypes.c_double]
        L.oracle_set_fields.argtypes = [vp, dp, dp, dp]
        L.oracle_prepare_propagation.argtypes = [vp, dp, ip]
        L.oracle_prepare_source.argtypes = [vp]
        L.oracle_get_indep.argtypes = [vp, ip]
        L.oracle_get_coef.argtypes = [vp, ctypes.c_char_p, dp]
        L.oracle_implsch.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp, ip, dp,
                                     ctypes.c_int]
        L.oracle_implsch_diag.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp, ip, dp,
                                          ctypes.c_int, ip, dp, ctypes.POINTER(ctypes.c_ubyte)]
        L.oracle_propags.argtypes = [vp, dp]
        L.oracle_resident_set.argtypes = [vp] + [dp] * 9
        L.oracle_count_implsch.argtypes = [ctypes.POINTER(OracleConfig), ctypes.c_int] + [dp] * 9 + [ip, dp]
        L.oracle_output_params.argtypes = [vp, ctypes.c_int] + [dp] * 9 + [ip, ctypes.c_int, dp]
        L.oracle_output_swell.argtypes = [vp, ctypes.c_int, dp, dp, dp, ctypes.c_int, dp]
        L.oracle_resident_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.oracle_resident_get.argtypes = [vp, dp, dp, dp, dp]
        L.oracle_grid_create.restype = vp
        L.oracle_grid_create.argtypes = [ctypes.POINTER(GridDef), ctypes.c_char_p]
        L.oracle_grid_destroy.argtypes = [vp]
        L.oracle_grid_nsea.argtypes = [vp]
        L.oracle_grid_get.argtypes = [vp, ip, ip, dp, ip, dp, dp, dp, dp, ip, ip, ip]
        assert L.oracle_sizeof_config() == ctypes.sizeof(OracleConfig)
        assert L.oracle_sizeof_griddef() == ctypes.sizeof(GridDef)
        _LIB = L
    return _LIB


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if a is not None else None


def build_grid(nx, ny, amosop, amowep, amoeap, xdella, xdello, mask, reduced=False):
    """Reference neighbour tables for a land-sea mask[nx, ny] (True = sea)."""
    L = lib()
    g = GridDef(nx, ny, amosop, amowep, amoeap, xdella, xdello, int(reduced))
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).T)  # (ny, nx) rows -> i fastest
    h = L.oracle_grid_create(ctypes.byref(g), m.tobytes())
    try:
        n = L.oracle_grid_nsea(h)
        out = dict(klat=np.zeros(4 * n, np.int32), klon=np.zeros(2 * n, np.int32), wlat=np.zeros(2 * n),
                   kfromij=np.zeros(n, np.int32), sinph=np.zeros(ny), cosph=np.zeros(ny), dellam=np.zeros(ny),
                   ixlg=np.zeros(n, np.int32), kxlt=np.zeros(n, np.int32))
        delphi = ctypes.c_double()
        iper = ctypes.c_int()
        L.oracle_grid_get(h, _i(out["klat"]), _i(out["klon"]), _d(out["wlat"]), _i(out["kfromij"]), _d(out["sinph"]),
                          _d(out["cosph"]), _d(out["dellam"]), ctypes.byref(delphi), _i(out["ixlg"]), _i(out["kxlt"]),
                          ctypes.byref(iper))
        out["delphi"] = delphi.value
        out["iper"] = iper.value
        out["nsea"] = n
        return out
    finally:
        L.oracle_grid_destroy(h)


class Oracle:
    """One model configuration of the CPU oracle, FP32 (precision=4) or FP64 (8)."""

    def __init__(self, cfg: dict, precision=4):
        self.L = lib()
        fields = {f for f, _ in OracleConfig._fields_}
        c = OracleConfig(**{k: v for k, v in cfg.items() if k in fields})
        self.cfg = dict(cfg)
        self.h = self.L.oracle_create(ctypes.byref(c), precision)
        if not self.h:
            raise RuntimeError("oracle_create failed")
        self.kl, self.ml = cfg["kl"], cfg["ml"]
        self.nsea = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def table(self, name):
        n = self.L.oracle_get_table(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        self.L.oracle_get_table(self.h, name.encode(), _d(out))
        return out

    def itable(self, name):
        n = self.L.oracle_get_itable(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, np.int32)
        self.L.oracle_get_itable(self.h, name.encode(), _i(out))
        return out

    def set_grid(self, g):
        self.nsea = g["nsea"]
        self.L.oracle_set_grid(self.h, g["nsea"], _i(np.ascontiguousarray(g["klat"], np.int32)),
                               _i(np.ascontiguousarray(g["klon"], np.int32)), _d(np.ascontiguousarray(g["wlat"], float)),
                               _i(np.ascontiguousarray(g["kfromij"], np.int32)), len(g["sinph"]),
                               _d(np.ascontiguousarray(g["sinph"], float)), _d(np.ascontiguousarray(g["cosph"], float)),
                               _d(np.ascontiguousarray(g["dellam"], float)), float(g["delphi"]))

    def set_fields(self, depth, u=None, v=None):
        d = np.ascontiguousarray(depth, float)
        uu = None if u is None else np.ascontiguousarray(u, float)
        vv = None if v is None else np.ascontiguousarray(v, float)
        self.L.oracle_set_fields(self.h, _d(d), _d(uu), _d(vv))

    def prepare_propagation(self):
        cfl = ctypes.c_double()
        cnt = ctypes.c_int()
        rc = self.L.oracle_prepare_propagation(self.h, ctypes.byref(cfl), ctypes.byref(cnt))
        return rc, cfl.value, cnt.value

    def prepare_source(self):
        self.L.oracle_prepare_source(self.h)

    def indep(self):
        out = np.zeros(self.nsea, np.int32)
        self.L.oracle_get_indep(self.h, _i(out))
        return out

    def coef(self, name):
        n = self.L.oracle_get_coef(self.h, name.encode(), None)
        out = np.zeros(n)
        self.L.oracle_get_coef(self.h, name.encode(), _d(out))
        return out

    def implsch(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep, lcflx=False, nthreads=0):
        """One IMPLSCH step in place on float64 copies; returns (fl3, tauw, ustar, z0, fluxes)."""
        nsea = fl3.shape[0]
        f = np.array(fl3, dtype=float, order="F")
        tw, us, zz = (np.array(a, dtype=float) for a in (tauw, ustar, z0))
        fl = np.zeros(7 * nsea) if lcflx else None
        self.L.oracle_implsch(self.h, nsea, nsea, _d(f), _d(np.ascontiguousarray(u10, float)),
                              _d(np.ascontiguousarray(udir, float)), _d(tw), _d(us), _d(zz),
                              _d(np.ascontiguousarray(roairn, float)), _d(np.ascontiguousarray(wstar, float)),
                              _d(np.ascontiguousarray(depth, float)), _i(np.ascontiguousarray(indep, np.int32)), _d(fl),
                              nthreads)
        return f, tw, us, zz, (fl.reshape(7, nsea) if fl is not None else None)

    def implsch_diag(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep, lcflx=False, nthreads=0):
        """implsch() plus the step's integer decisions: returns (fl3, tauw, ustar, z0, fluxes, diag) where diag
        holds JU, MIJ1, MIJ2 (first and last FRCUTINDEX), LFIT (LFACTOR iterations, -1 for ST4), the REAL values
        they were rounded from (JU_ARG, MIJ1_ARG, MIJ2_ARG), the smallest relative distance of the LFACTOR |ERR|
        from its exit threshold over the iterations (LF_MARGIN) and the LLWS masks of the first and the last
        SINPUT call (LLWS1, LLWS2: uint8 arrays shaped like FL3)."""
        nsea = fl3.shape[0]
        f = np.array(fl3, dtype=float, order="F")
        tw, us, zz = (np.array(a, dtype=float) for a in (tauw, ustar, z0))
        fl = np.zeros(7 * nsea) if lcflx else None
        idg = np.zeros(4 * nsea, np.int32)
        fdg = np.zeros(4 * nsea)
        ll = np.zeros(2 * nsea * self.kl * self.ml, np.uint8)
        self.L.oracle_implsch_diag(self.h, nsea, nsea, _d(f), _d(np.ascontiguousarray(u10, float)),
                                   _d(np.ascontiguousarray(udir, float)), _d(tw), _d(us), _d(zz),
                                   _d(np.ascontiguousarray(roairn, float)), _d(np.ascontiguousarray(wstar, float)),
                                   _d(np.ascontiguousarray(depth, float)), _i(np.ascontiguousarray(indep, np.int32)),
                                   _d(fl), nthreads, _i(idg), _d(fdg), ll.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        idg, fdg = idg.reshape(4, nsea), fdg.reshape(4, nsea)
        ll = ll.reshape(2, self.ml, self.kl, nsea)
        diag = dict(JU=idg[0], MIJ1=idg[1], MIJ2=idg[2], LFIT=idg[3], JU_ARG=fdg[0], MIJ1_ARG=fdg[1], MIJ2_ARG=fdg[2],
                    LF_MARGIN=fdg[3], LLWS1=np.asfortranarray(ll[0].transpose(2, 1, 0)),
                    LLWS2=np.asfortranarray(ll[1].transpose(2, 1, 0)))
        return f, tw, us, zz, (fl.reshape(7, nsea) if fl is not None else None), diag

    def count_implsch(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep):
        """Floating-point operation counts of IMPLSCH on these points (the
        restatement run with a counting number type): dict of additions,
        multiplications, divisions, square roots, transcendental functions and
        comparisons, summed over the points."""
        fields = {f for f, _ in OracleConfig._fields_}
        c = OracleConfig(**{k: v for k, v in self.cfg.items() if k in fields})
        nsea = fl3.shape[0]
        cnt = np.zeros(6)
        a = lambda x: np.ascontiguousarray(x, float)
        self.L.oracle_count_implsch(ctypes.byref(c), nsea, _d(np.asfortranarray(fl3, float)), _d(a(u10)), _d(a(udir)),
                                    _d(a(tauw)), _d(a(ustar)), _d(a(z0)), _d(a(roairn)), _d(a(wstar)), _d(a(depth)),
                                    _i(np.ascontiguousarray(indep, np.int32)), _d(cnt))
        return dict(zip(("add", "mul", "div", "sqrt", "trans", "cmp"), cnt.astype(np.int64).tolist()))

    def output_params(self, fl3, u10, udir, ustar, tauw, z0, depth, u=None, v=None, indep=None, from_=True):
        """COMPUTE_OUTPUT_PARAMETER: returns (block[40, nsea] with row IP-1 = parameter IP, ustar, z0)."""
        nsea = fl3.shape[0]
        f = np.asfortranarray(fl3, float)
        us, zz = np.array(ustar, float), np.array(z0, float)
        c = lambda a: None if a is None else np.ascontiguousarray(a, float)
        out = np.zeros(40 * nsea)
        ind = np.ascontiguousarray(indep if indep is not None else self.indep(), np.int32)
        self.L.oracle_output_params(self.h, nsea, _d(f), _d(c(u10)), _d(c(udir)), _d(us), _d(c(tauw)), _d(zz),
                                    _d(c(depth)), _d(c(u)), _d(c(v)), _i(ind), int(bool(from_)), _d(out))
        return out.reshape(40, nsea), us, zz

    def output_swell(self, fl3, udir, ustar, from_=True, block=None):
        """SWELL_SEPARATION: rows 16..22 and 24..30 (parameters 17-23, 25-31)
        of block[40, nsea] (zeros when not given) filled."""
        nsea = fl3.shape[0]
        f = np.asfortranarray(fl3, float)
        out = np.zeros((40, nsea)) if block is None else np.array(block, float)
        c = lambda a: np.ascontiguousarray(a, float)
        o = np.ascontiguousarray(out).ravel()
        self.L.oracle_output_swell(self.h, nsea, _d(f), _d(c(udir)), _d(c(ustar)), int(bool(from_)), _d(o))
        return o.reshape(40, nsea)

    def resident_set(self, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth):
        """Keep a model state inside the oracle in its own precision (the timed CPU baseline)."""
        c = lambda a: np.ascontiguousarray(a, float)
        self._res = [np.asfortranarray(fl3, float)] + [c(a) for a in (u10, udir, tauw, ustar, z0, roairn, wstar, depth)]
        self.L.oracle_resident_set(self.h, *[_d(a) for a in self._res])

    def resident_step(self, nprop, nthreads=0):
        """One WAMODEL pass on the resident state: nprop PROPAGS, then IMPLSCH (all host threads when 0)."""
        rc = self.L.oracle_resident_step(self.h, int(nprop), int(nthreads or os.cpu_count() or 1))
        if rc != 0:
            raise RuntimeError("oracle_resident_step: no resident state")

    def resident_get(self):
        """(fl3, tauw, ustar, z0) of the resident state."""
        n = self.nsea
        f = np.zeros((n, self.kl, self.ml), order="F")
        tw, us, zz = np.zeros(n), np.zeros(n), np.zeros(n)
        self.L.oracle_resident_get(self.h, _d(f), _d(tw), _d(us), _d(zz))
        return f, tw, us, zz

    def propags(self, fl3):
        f = np.array(fl3, dtype=float, order="F")
        self.L.oracle_propags(self.h, _d(f))
        return f


def put_points(data, points, value, nijs=1, nijl=None):
    """PUT_ICE_SPEC / PUT_DRY_SPEC (wam_ice_module.f90:312-324,
    wam_topo_module.f90:557-569) and the PUT_*_PAR forms: for every 1-based
    sea point of the list (IJ_ICE / IJ_DRY) inside NIJS..NIJL, all values of
    that point (data[ij-1, ...], sea point first) become `value`.  Returns a
    modified copy."""
    out = np.array(data, copy=True, order="F")
    nijl = out.shape[0] if nijl is None else nijl
    for ij in np.asarray(points).reshape(-1):
        if nijs <= ij <= nijl:
            out[ij - 1, ...] = value
    return out


M_S_PER = 360 * 360000


def wind_tables(grid, nx_in, ny_in, west_in, south_in, dx_in, dy_in, periodic=False, equal_grid=False):
    """INITIALIZE of INTERPOLATION_TO_GRID (wam_wind_module.f90:1296-1375):
    per sea point the input cell I1, I2, K1, K2 (1-based) and the weights DI,
    DK, in the reference's integer units and REAL (float32) arithmetic.
    Raises where the reference calls ABORT1 (a point outside the input grid)."""
    f32 = np.float32
    ifr = np.asarray(grid["ixlg"], np.int64)
    kfr = np.asarray(grid["kfromij"], np.int64)
    if equal_grid:
        z = np.zeros(ifr.size, f32)
        return ifr, ifr.copy(), kfr, kfr.copy(), z, z.copy()
    zdello = np.broadcast_to(np.asarray(grid.get("zdello", grid["xdello"]), np.int64), (int(grid["ny"]),))
    i1 = grid["amowep"] + (ifr - 1) * zdello[kfr - 1] - west_in
    i1 = np.mod(i1 + 2 * M_S_PER, M_S_PER)
    di = i1.astype(f32) / f32(dx_in)
    k1 = grid["amosop"] + (kfr - 1) * grid["xdella"] - south_in
    dk = k1.astype(f32) / f32(dy_in)
    i1 = di.astype(np.int64) + 1
    k1 = dk.astype(np.int64) + 1
    k2 = np.minimum(ny_in, k1 + 1)
    i2 = i1 + 1
    di = (di - i1.astype(f32)) + f32(1.)
    dk = (dk - k1.astype(f32)) + f32(1.)
    if periodic:
        i2 = np.where(i1 == nx_in, 1, i2)
        i1 = np.where(i1 == 0, nx_in, i1)
    else:
        i2 = np.where(i1 == nx_in, nx_in, i2)
    if i1.min() < 1 or i1.max() > nx_in or k1.min() < 1 or k1.max() > ny_in:
        raise ValueError("point is outside of input grid")
    return i1, i2, k1, k2, di.astype(f32), dk.astype(f32)


def wam_wind(u_in, v_in, tables, code_in=3, equal_grid=False):
    """WAM_WIND (wam_wind_module.f90:1063-1216) in float32: the input
    components u_in, v_in [ny_in, nx_in] at the sea points (bilinear, or a
    copy on the model's own grid), speed, direction ATAN2(U,V) in [0, 2 pi),
    the friction-velocity (1) or stress (2) input turned into U10, U10 >= 2."""
    f32 = np.float32
    i1, i2, k1, k2, di, dk = tables
    U = np.asarray(u_in, f32)
    V = np.asarray(v_in, f32)
    at = lambda F, i, k: F[k - 1, i - 1]
    if equal_grid:
        uu, vv = at(U, i1, k1), at(V, i1, k1)
    else:
        one = f32(1.)
        uu = (at(U, i1, k1) * (one - di) + at(U, i2, k1) * di) * (one - dk) + \
             (at(U, i1, k2) * (one - di) + at(U, i2, k2) * di) * dk
        vv = (at(V, i1, k1) * (one - di) + at(V, i2, k1) * di) * (one - dk) + \
             (at(V, i1, k2) * (one - di) + at(V, i2, k2) * di) * dk
    us = np.sqrt(uu * uu + vv * vv).astype(f32)
    ds = np.where(us != 0, np.arctan2(uu, vv), f32(0.)).astype(f32)
    ds = np.where(ds < 0, ds + f32(2.) * f32(3.1415927), ds).astype(f32)
    if code_in in (1, 2):
        ust = np.maximum(f32(0.01), us) if code_in == 1 else np.maximum(f32(0.01), np.sqrt(us / f32(1.225)))
        z0 = f32(0.0185) / f32(9.806) * (ust * ust)
        cd = f32(0.40) / np.log(f32(10.) / z0)
        us = (ust / cd).astype(f32)
    return np.maximum(us, f32(2.0)).astype(f32), ds


def write_restart(path, nsea, dates, u10, udir, tauw, fl3, depth=None, u=None, v=None, ij2newij=None):
    """SAVE_RESTART_FILE's records (wam_restart_module.f90:414-591) as a
    Fortran sequential unformatted file: record lengths around every record,
    REAL as float32.  fl3 is (NSEA, KL, ML); with ij2newij file position p
    holds model point ij2newij[p-1]."""
    perm = np.arange(nsea) if ij2newij is None else np.asarray(ij2newij) - 1

    def rec(fh, payload):
        m = np.int32(len(payload)).tobytes()
        fh.write(m + payload + m)

    with open(path, "wb") as fh:
        head = np.int32(nsea).tobytes() + b"".join(str(dates.get(k, "")).ljust(14)[:14].encode()
                                                     for k in ("CDTPRO", "CDTSOU", "CDA", "CDTA", "CDCA"))
        rec(fh, head)
        for a in (u10, udir, tauw):
            rec(fh, np.asarray(a, np.float32)[perm].tobytes())
        rec(fh, np.asarray(fl3, np.float32)[perm].tobytes(order="F"))
        if str(dates.get("CDTA", "")).strip():
            rec(fh, np.asarray(depth, np.float32)[perm].tobytes())
        if str(dates.get("CDCA", "")).strip():
            rec(fh, np.asarray(u, np.float32)[perm].tobytes() + np.asarray(v, np.float32)[perm].tobytes())


def read_restart(path, kl, ml, ij2newij=None):
    """CONNECT_RESTART's records (wam_restart_module.f90:109-327): returns a
    dict of NSEA, the dates, U10, UDIR, TAUW, FL3 (NSEA, KL, ML) in model
    order, and DEPTH / U / V when their dates are not blank."""
    with open(path, "rb") as fh:
        data = fh.read()
    recs, pos = [], 0
    while pos < len(data):
        n = int(np.frombuffer(data, np.int32, 1, pos)[0])
        recs.append(data[pos + 4:pos + 4 + n])
        assert int(np.frombuffer(data, np.int32, 1, pos + 4 + n)[0]) == n, "record length markers differ"
        pos += n + 8
    head = recs[0]
    nsea = int(np.frombuffer(head, np.int32, 1, 0)[0])
    out = {"NSEA": nsea}
    for i, k in enumerate(("CDTPRO", "CDTSOU", "CDA", "CDTA", "CDCA")):
        out[k] = head[4 + 14 * i:18 + 14 * i].decode()
    perm = np.arange(nsea) if ij2newij is None else np.asarray(ij2newij) - 1

    def model(x):
        y = np.empty_like(x)
        y[perm] = x
        return y
    f = lambda r: np.frombuffer(r, np.float32)
    out["U10"], out["UDIR"], out["TAUW"] = (model(f(recs[i])) for i in (1, 2, 3))
    spec = f(recs[4]).reshape((nsea, kl, ml), order="F")
    out["FL3"] = np.asfortranarray(model(spec))
    i = 5
    if out["CDTA"].strip():
        out["DEPTH"] = model(f(recs[i])); i += 1
    if out["CDCA"].strip():
        uv = f(recs[i])
        out["U"], out["V"] = model(uv[:nsea]), model(uv[nsea:])
    return out
