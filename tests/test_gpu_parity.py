"""GPU parity: libwamgpu's IMPLSCH and PROPAGS against the CPU oracle.

Every comparison goes through the C ABI (host-buffer entry points for FP32,
device-pointer entry points for the FP64 run of the same kernels) on seeded
synthetic inputs at sizes the oracle finishes in seconds.  The "mixed" cases
start from spectra with per-point peak frequencies between 0.07 and 0.25 Hz
and convective velocities WSTAR up to 1.5 m/s (the gust branch of
WSIGSTAR), so the cut-off index and the wind-sea mask vary over the grid.

Bars:
  * PROPAGS, FP32: bit-exact (coefficients recomputed in reference order).
  * The integer decisions of IMPLSCH (wamgpu_set_diagnostics): JU, the
    cut-off index MIJ of both FRCUTINDEX calls, the LFACTOR iteration count
    (ST6) and both LLWS masks are compared element by element with the
    oracle's.  A point where one differs is counted and must be a genuine
    rounding-boundary case: for MIJ the oracle's operand within 1e-4 of the
    rounding boundary, for the LFACTOR count the oracle's |ERR| within 1e-3
    (relative) of its exit threshold 1.54E-4 at some iteration.  At most 0.5%
    of the points may hold such a flip (none has been seen).
  * IMPLSCH, FP32, every point whose decisions agree: 1e-5 relative to the
    point's largest bin, per step, with no outlier allowance (observed
    <= 7e-7, ST6 included).
  * USTAR 1e-5, Z0 1e-4 relative; TAUW 1e-5 of its scale.
  * LCFLX surface fluxes (WNFLUXES) 1e-5 of each component's scale.
  * FP64 GPU vs FP64 oracle: 1e-12 (1e-9 on the ST6 grid).
  * Hs and Tm after 12 simulated hours (6 h on the regional ST6 grid) on
    the full 60x40 1-degree grid and sampled larger grids: 1e-4 relative at
    the maximum against the FP32 oracle; against the FP64 GPU run the FP32
    error stays within twice that of the FP32 oracle itself, and the FP64 GPU
    run stays within 1e-8 of the FP64 oracle at the median and 1e-5 at the
    maximum (an FP64 threshold decision can flip at a point).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-5


def _spinup(o, w, steps=3):
    indep = o.indep()
    f = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    for _ in range(steps):
        f, tw, us, zz, _ = o.implsch(f, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
        for _ in range(w.sub_steps):
            f = o.propags(f)
    return (np.asfortranarray(f.astype(np.float32)), tw.astype(np.float32), us.astype(np.float32),
            zz.astype(np.float32), indep)


def _setup(oracle_mod, w, precision=4, **cfgx):
    from wam_b200 import WamModel
    cfg = dict(w.cfg, precision=precision, **cfgx)
    o = oracle_mod.Oracle(cfg, precision=precision)
    o.set_grid(w.grid)
    o.set_fields(w.depth, getattr(w, "u", None), getattr(w, "v", None))
    rc, cfl, cnt = o.prepare_propagation()
    assert rc == 0
    o.prepare_source()
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    if getattr(w, "u", None) is not None:
        m.set_current(w.u, w.v)
    gcfl, gcnt = m.prepare_propagation()
    m.prepare_source()
    assert gcnt == cnt and np.float32(gcfl) == np.float32(cfl), (cfl, cnt, gcfl, gcnt)
    return o, m


def _point_rel(a, ref):
    ref = np.asarray(ref)
    pmax = np.abs(ref).max(axis=(1, 2))
    return (np.abs(np.asarray(a) - ref).max(axis=(1, 2))) / np.maximum(pmax, 1e-30)


def _decision_flips(gd, od, iphys):
    """Points whose integer decisions differ, each checked to be a rounding-
    boundary case; returns (mask of flipped points, report lines)."""
    n = gd["JU"].size
    flipped = np.zeros(n, bool)
    report = []
    assert np.array_equal(gd["JU"], od["JU"]), "JU differs (NINT of U10/DELU on identical inputs)"
    for k in ("MIJ1", "MIJ2"):
        for i in np.nonzero(gd[k] != od[k])[0]:
            arg = od[k + "_ARG"][i]
            dist = abs(arg - (np.floor(arg) + 0.5)) if iphys == 1 else abs(arg - np.round(arg))
            report.append(f"{k} point {i}: gpu {gd[k][i]} oracle {od[k][i]}, oracle operand {arg!r}")
            assert dist < 1e-4, report[-1] + " is not a rounding-boundary case"
            flipped[i] = True
    for i in np.nonzero(gd["LFIT"] != od["LFIT"])[0]:
        report.append(f"LFIT point {i}: gpu {gd['LFIT'][i]} oracle {od['LFIT'][i]}, margin {od['LF_MARGIN'][i]:.2e}")
        assert od["LF_MARGIN"][i] < 1e-3, report[-1] + " is not a threshold case"
        flipped[i] = True
    for k in ("LLWS1", "LLWS2"):
        d = (gd[k] != od[k]).any(axis=(1, 2))
        for i in np.nonzero(d)[0]:
            report.append(f"{k} point {i}: {int((gd[k][i] != od[k][i]).sum())} bins")
        flipped |= d
    assert flipped.mean() <= 0.005, f"{flipped.sum()} of {n} points with flipped decisions:\n" + "\n".join(report)
    return flipped, report


WORKLOADS = [("c0", 0.25, False), ("c0", 1.0, True), ("c1", 0.02, False), ("c1", 0.03, True), ("c2", 0.05, False),
             ("c2", 0.05, True), ("c4", 0.02, False)]


@pytest.fixture(scope="module", params=WORKLOADS, ids=[f"{w[0]}@{w[1]}{'-mixed' if w[2] else ''}" for w in WORKLOADS])
def case(request, oracle_mod):
    from wam_b200.synth import make_workload, vary_sea_state
    name, scale, mixed = request.param
    w = make_workload(name, scale=scale)
    if mixed:
        vary_sea_state(w)
    o, m = _setup(oracle_mod, w)
    S = _spinup(o, w)
    return name, w, o, m, S


def test_indep_bit_exact(case):
    name, w, o, m, S = case
    assert np.array_equal(m.indep(), o.indep())


def test_propags_bit_exact(case):
    name, w, o, m, S = case
    ref = o.propags(S[0].astype(float)).astype(np.float32)
    got = np.asfortranarray(S[0].copy())
    m.propags(got)
    assert np.array_equal(got, ref), f"{name}: max diff {np.abs(got - ref).max()}"


def test_implsch_fp32_one_step(case):
    name, w, o, m, S = case
    f, tw, us, zz, indep = S
    fo, two, uso, zo, _, od = o.implsch_diag(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth,
                                             indep)
    fg = np.asfortranarray(f.copy())
    tg, ug, zg = tw.copy(), us.copy(), zz.copy()
    gd = m.implsch_decisions(fg, w.u10, w.udir, tg, ug, zg, w.roairn, w.wstar)
    flipped, report = _decision_flips(gd, od, w.cfg["iphys"])
    err = _point_rel(fg, fo)
    ok = ~flipped
    assert err[ok].max() <= TOL_STEP, f"{name}: max point error {err[ok].max():.3e} (decisions equal)"
    assert np.max(np.abs(ug - uso)[ok] / uso[ok]) <= 1e-5
    assert np.max(np.abs(zg - zo)[ok] / zo[ok]) <= 1e-4
    tscale = np.maximum(np.abs(two), 1e-3 * np.abs(two).max())
    assert np.max((np.abs(tg - two) / tscale)[ok]) <= 1e-5
    lf = gd["LFIT"][gd["LFIT"] >= 0]
    print(f"\n{name}@{w.nsea}: max point error {err.max():.2e}, decision flips {int(flipped.sum())} of {w.nsea}, "
          f"MIJ1 range {gd['MIJ1'].min()}-{gd['MIJ1'].max()}, LFACTOR iterations "
          f"{'-' if lf.size == 0 else f'{lf.min()}-{lf.max()} (mean {lf.mean():.1f})'}")


def test_implsch_fp64_matches_fp64_oracle(case, oracle_mod):
    import torch
    name, w, o, m, S = case
    f, tw, us, zz, indep = S
    o64, m64 = _setup(oracle_mod, w, precision=8)
    fo, two, uso, zo, _ = o64.implsch(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
    dev = torch.device("cuda")
    ten = lambda a: torch.tensor(np.asarray(a), dtype=torch.float64, device=dev)
    F = ten(np.ascontiguousarray(np.asarray(f).transpose(2, 1, 0)))
    T, U, Z = ten(tw), ten(us), ten(zz)
    m64.implsch_dev(F, ten(w.u10), ten(w.udir), T, U, Z, ten(w.roairn), ten(w.wstar))
    m64.sync()
    fg = F.cpu().numpy().transpose(2, 1, 0)
    err = _point_rel(fg, fo)
    assert err.max() <= (1e-12 if name != "c1" else 1e-9), f"{name} FP64: {err.max():.3e}"
    assert np.allclose(U.cpu().numpy(), uso, rtol=1e-12)


def test_fp32_error_against_fp64(case, oracle_mod):
    """The FP32 GPU step stays as close to the FP64 oracle as the FP32 oracle does."""
    name, w, o, m, S = case
    f, tw, us, zz, indep = S
    o64 = oracle_mod.Oracle(dict(w.cfg, precision=8), precision=8)
    o64.set_grid(w.grid); o64.set_fields(w.depth); o64.prepare_propagation(); o64.prepare_source()
    f64, *_ = o64.implsch(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
    f32o, *_ = o.implsch(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
    fg = np.asfortranarray(f.copy())
    m.implsch(fg, w.u10, w.udir, tw.copy(), us.copy(), zz.copy(), w.roairn, w.wstar)
    e_gpu = _point_rel(fg, f64)
    e_orc = _point_rel(f32o, f64)
    assert e_gpu.max() <= max(2 * e_orc.max(), 1e-6), (e_gpu.max(), e_orc.max())


@pytest.mark.parametrize("name,scale,mixed", [("c0", 0.5, True), ("c2", 0.05, True), ("c1", 0.02, True)])
def test_lcflx_surface_fluxes(oracle_mod, name, scale, mixed):
    """WNFLUXES (wam_source_module.f90:3970-4054) with LCFLX: PHIOC, TAUOC,
    PHIBOT, TAUBOT and PHIAW of the step from wamgpu_get_fluxes against the
    oracle's, per component relative to its largest magnitude."""
    from wam_b200.synth import make_workload, vary_sea_state
    w = make_workload(name, scale=scale)
    if mixed:
        vary_sea_state(w)
    o, m = _setup(oracle_mod, w, lcflx=1)
    f, tw, us, zz, indep = _spinup(o, w)
    fo, two, uso, zo, fx, od = o.implsch_diag(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth,
                                              indep, lcflx=True)
    fg = np.asfortranarray(f.copy())
    gd = m.implsch_decisions(fg, w.u10, w.udir, tw.copy(), us.copy(), zz.copy(), w.roairn, w.wstar)
    flipped, _ = _decision_flips(gd, od, w.cfg["iphys"])
    gx = m.fluxes()
    names = ["PHIOC", "TAUOC_X", "TAUOC_Y", "PHIBOT", "TAUBOT_X", "TAUBOT_Y", "PHIAW"]
    for q, nm in enumerate(names):
        scale_q = np.abs(fx[q]).max()
        if scale_q == 0:
            assert np.all(gx[q] == 0), nm
            continue
        err = np.abs(gx[q] - fx[q])[~flipped] / scale_q
        assert err.max() <= 1e-5, f"{name} {nm}: {err.max():.3e}"


def _run_hours(o, m, w, hours, m64=None):
    import torch
    steps = int(round(hours * 3600 / w.cfg["idelt"]))
    indep = o.indep()
    fo = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    fg = np.asfortranarray(w.spectrum_f().copy())
    tg, ug, zg = w.tauw.copy(), w.ustar.copy(), w.z0.copy()
    if m64 is not None:
        dev = torch.device("cuda")
        ten = lambda a: torch.tensor(np.asarray(a), dtype=torch.float64, device=dev)
        F6 = w.spectrum_device(torch, dev, dtype=torch.float64)
        S6 = torch.empty_like(F6)
        fl6 = [ten(a) for a in (w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar)]
    for _ in range(steps):
        for _ in range(w.sub_steps):
            fo = o.propags(fo)
            m.propags(fg)
        fo, tw, us, zz, _ = o.implsch(fo, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
        m.implsch(fg, w.u10, w.udir, tg, ug, zg, w.roairn, w.wstar)
        if m64 is not None:
            m64.step_dev(F6, w.sub_steps, *fl6, scratch=S6)
    g64 = None
    if m64 is not None:
        m64.sync()
        g64 = F6.cpu().numpy().transpose(2, 1, 0)
    return fo, fg, g64


def _hs_tm(o, f):
    dfim, fr = o.table("DFIM"), o.table("FR")
    e = (f.sum(axis=1) * dfim).sum(axis=1)
    m1 = (f.sum(axis=1) * dfim / fr).sum(axis=1)
    return 4 * np.sqrt(e), m1 / e


@pytest.mark.parametrize("name,scale,hours,mixed", [("c0", 1.0, 12, False), ("c0", 1.0, 12, True),
                                                    ("c1", 0.02, 6, False), ("c4", 0.02, 12, False)])
def test_hs_tm_after_simulated_hours(oracle_mod, name, scale, hours, mixed):
    from wam_b200.synth import make_workload, vary_sea_state
    w = make_workload(name, scale=scale)
    if mixed:
        vary_sea_state(w)
    o, m = _setup(oracle_mod, w)
    o64, m64 = _setup(oracle_mod, w, precision=8)
    fo, fg, g64 = _run_hours(o, m, w, hours, m64=m64)
    steps = int(round(hours * 3600 / w.cfg["idelt"]))
    indep = o64.indep()
    f64 = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    for _ in range(steps):
        for _ in range(w.sub_steps):
            f64 = o64.propags(f64)
        f64, tw, us, zz, _ = o64.implsch(f64, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
    rel = lambda a, b: np.abs(a - b) / b
    (hs_o, tm_o), (hs_g, tm_g), (hs_6, tm_6), (hs_g6, tm_g6) = (_hs_tm(o, x) for x in (fo, fg.astype(float), f64, g64))
    # FP32 GPU against the FP32 oracle: 1e-4 at the maximum
    assert rel(hs_g, hs_o).max() <= 1e-4 and rel(tm_g, tm_o).max() <= 1e-4, (rel(hs_g, hs_o).max(), rel(tm_g, tm_o).max())
    # the FP64 GPU run of the same kernels against the FP64 oracle: their
    # summation orders and FMA contraction differ (~1e-9 after 48 steps), and
    # CUDA's FP64 exp/log are not the host's, so in FP64 an LFACTOR exit or
    # a MIJ rounding can flip at a point that sits on its threshold; one such
    # point moves by a few 1e-6 (3.2e-6 seen on the regional grid after 6 h)
    e6 = np.concatenate([rel(hs_g6, hs_6), rel(tm_g6, tm_6)])
    assert np.median(e6) <= 1e-8 and e6.max() <= 1e-5, (np.median(e6), e6.max())
    # against FP64 the FP32 GPU run is as close as the FP32 oracle
    for g, ref, orc in ((hs_g, hs_g6, hs_o), (tm_g, tm_g6, tm_o)):
        assert rel(g, ref).max() <= 2 * rel(orc, ref).max() + 1e-6, (rel(g, ref).max(), rel(orc, ref).max())
    print(f"\n{name}@{scale} {hours} h: Hs max rel err vs FP32 oracle {rel(hs_g, hs_o).max():.2e}, vs FP64 GPU "
          f"{rel(hs_g, hs_g6).max():.2e} (FP32 oracle vs FP64 {rel(hs_o, hs_g6).max():.2e}); Tm "
          f"{rel(tm_g, tm_o).max():.2e} / {rel(tm_g, tm_g6).max():.2e} ({rel(tm_o, tm_g6).max():.2e})")


@pytest.mark.parametrize("iphys", [1, 2])
def test_implsch_isnonlin_table(oracle_mod, iphys):
    """SNONLIN with the MAKE_SHALLOW_SNL depth factors (ISNONLIN = 1,
    wam_source_module.f90:975-1048) instead of the AKMEAN scaling: the shallow
    regional grid, one FP32 step against the oracle."""
    from wam_b200.synth import make_workload
    w = make_workload("c2" if iphys == 1 else "c1", scale=0.02)
    w.cfg = dict(w.cfg, isnonlin=1)
    o, m = _setup(oracle_mod, w)
    f, tw, us, zz, indep = _spinup(o, w)
    fo, two, uso, zo, _, od = o.implsch_diag(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth,
                                             indep)
    fg = np.asfortranarray(f.copy())
    tg, ug, zg = tw.copy(), us.copy(), zz.copy()
    gd = m.implsch_decisions(fg, w.u10, w.udir, tg, ug, zg, w.roairn, w.wstar)
    flipped, _ = _decision_flips(gd, od, iphys)
    err = _point_rel(fg, fo)
    assert err[~flipped].max() <= TOL_STEP
    assert np.max(np.abs(ug - uso) / uso) <= 1e-5
