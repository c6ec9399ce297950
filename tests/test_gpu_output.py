"""Integrated output parameters on the device (wamgpu_output_parameters_dev,
COMPUTE_OUTPUT_PARAMETER wam_output_module.f90:481-640) against the oracle's
restatement, on spectra with a spread of sea states (per-point peak
frequencies) after a few model steps, in deep (1-degree ST4 grid) and
shallow water (regional grid, currents included).

The output unit rounds every operation separately, in the reference's
order, so the FP32 parameters equal the FP32 oracle's bit for bit, except
the two ATAN2 directions (current direction 8 and mean direction 14), which
use the device library's arctangent: within 2e-6 relative.  FP64 against the
FP64 oracle: 1e-12 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 40]
ANGLES = {8, 14}


def _case(oracle_mod, name, scale, precision, currents):
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload, vary_sea_state
    w = vary_sea_state(make_workload(name, scale=scale))
    cfg = dict(w.cfg, precision=precision)
    rng = np.random.default_rng(5)
    u = v = None
    if currents:
        u = (0.5 * rng.standard_normal(w.nsea)).astype(np.float32)
        v = (0.5 * rng.standard_normal(w.nsea)).astype(np.float32)
    o = oracle_mod.Oracle(cfg, precision=precision)
    o.set_grid(w.grid)
    o.set_fields(w.depth, u, v)
    o.prepare_propagation()
    o.prepare_source()
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    if currents:
        m.set_current(u, v)
    m.prepare_propagation()
    m.prepare_source()
    # a few oracle steps give USTAR, TAUW, Z0 and developed spectra
    f = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    for _ in range(2):
        f, tw, us, zz, _ = o.implsch(f, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, o.indep())
    return w, o, m, f, tw, us, zz, u, v


def _gpu(m, w, f, tw, us, zz, precision, from_=True):
    import torch
    dt = torch.float64 if precision == 8 else torch.float32
    t = lambda a: torch.tensor(np.asarray(a), dtype=dt, device="cuda")
    F = t(np.ascontiguousarray(np.asarray(f).transpose(2, 1, 0)))
    U, D, T, S, Z = t(w.u10), t(w.udir), t(tw), t(us), t(zz)
    blk = m.output_parameters_dev(F, U, D, T, S, Z, from_=from_)
    m.sync()
    return blk.cpu().numpy(), S.cpu().numpy(), Z.cpu().numpy()


def _compare(got, ref, precision, label, angle_tol=2e-6):
    for p in PARAMS:
        g, r = got[p - 1], ref[p - 1]
        if precision == 8:
            err = np.max(np.abs(g - r) / np.maximum(np.abs(r), 1e-30))
            assert err <= 1e-12, f"{label} parameter {p}: {err:.2e}"
        elif p in ANGLES:
            d = np.abs(g - r)
            d = np.minimum(d, 360.0 - d)  # 0 and 360 deg are the same direction
            assert np.max(d / 360.0) <= angle_tol, f"{label} parameter {p}: {np.max(d):.3e} deg"
        else:
            bad = np.nonzero(g.astype(np.float32) != r.astype(np.float32))[0]
            assert bad.size == 0, (f"{label} parameter {p}: {bad.size} points differ, e.g. point {bad[0]}: "
                                   f"{g[bad[0]]!r} vs {r[bad[0]]!r}")
    untouched = [p for p in range(1, 41) if p not in PARAMS]
    assert np.all(got[[p - 1 for p in untouched]] == 0)


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("name,scale,currents", [("c0", 0.5, False), ("c2", 0.05, True)])
def test_output_parameters_match_oracle(oracle_mod, name, scale, currents, precision):
    w, o, m, f, tw, us, zz, u, v = _case(oracle_mod, name, scale, precision, currents)
    ref, _, _ = o.output_params(f, w.u10, w.udir, us, tw, zz, w.depth, u, v)
    got, _, _ = _gpu(m, w, f, tw, us, zz, precision)
    _compare(got, ref, precision, f"{name} {'fp64' if precision == 8 else 'fp32'}")
    # Hs is the square root of the integrated energy: independent check
    dfim = o.table("DFIM")
    e = (np.asarray(f).sum(axis=1) * dfim).sum(axis=1) + o.table("SCALARS")[3] * np.asarray(f)[:, :, -1].sum(axis=1)
    assert np.allclose(got[8], 4 * np.sqrt(np.maximum(e, 1e-12)), rtol=1e-5)
    m.close()


def test_output_parameters_going_to_and_airsea(oracle_mod):
    """The "going to" direction convention, and USTAR zero everywhere: AIRSEA
    first sets USTAR and Z0 (written back), as the reference does before its
    first output."""
    w, o, m, f, tw, us, zz, u, v = _case(oracle_mod, "c0", 0.5, 4, False)
    us0, z00 = np.zeros_like(us), np.zeros_like(zz)
    ref, us_o, z0_o = o.output_params(f, w.u10, w.udir, us0, tw, z00, w.depth, from_=False)
    got, us_g, z0_g = _gpu(m, w, f, tw, us0, z00, 4, from_=False)
    # AIRSEA's logarithms are the device library's: u* and z0 within a few ulp
    assert np.max(np.abs(us_g - us_o) / us_o) <= 2e-6
    assert np.max(np.abs(z0_g - z0_o) / z0_o) <= 2e-5
    for p in PARAMS:
        tol = 2e-5 if p in (3, 4, 5, 16, 32) else (2e-6 if p in ANGLES else 0.0)
        g, r = got[p - 1], ref[p - 1]
        if p in ANGLES:
            d = np.abs(g - r)
            d = np.minimum(d, 360.0 - d) / 360.0
        else:
            d = np.abs(g - r) / np.maximum(np.abs(r), 1e-30)
        assert np.max(d) <= tol, f"parameter {p}: {np.max(d):.3e}"
    m.close()


SWELL = [17, 18, 19, 20, 21, 22, 23, 25, 26, 27, 28, 29, 30, 31]
SWELL_ANGLES = {22, 30}


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("name,scale,from_", [("c0", 0.5, True), ("c2", 0.05, False)])
def test_swell_separation_matches_oracle(oracle_mod, name, scale, from_, precision):
    """SWELL_SEPARATION (wam_swell_module.f90:106-350) through
    wamgpu_output_swell_dev: wind-sea parameters 17-23 and swell parameters
    25-31 against the oracle.  The split of every bin uses the correctly
    rounded cosine on both sides, so FP32 values are bit-identical except
    the two mean directions (ATAN2 of the device library); FP64 to 1e-12.
    The other rows of the block are left as they were."""
    import torch
    w, o, m, f, tw, us, zz, u, v = _case(oracle_mod, name, scale, precision, False)
    ref = o.output_swell(f, w.udir, us, from_=from_)
    dt = torch.float64 if precision == 8 else torch.float32
    t = lambda a: torch.tensor(np.asarray(a), dtype=dt, device="cuda")
    F = t(np.ascontiguousarray(np.asarray(f).transpose(2, 1, 0)))
    blk = torch.full((40, w.nsea), 7.0, dtype=dt, device="cuda")
    m.output_swell_dev(F, t(w.udir), t(us), blk, from_=from_)
    m.sync()
    got = blk.cpu().numpy()
    for p in SWELL:
        g, r = got[p - 1], ref[p - 1]
        if precision == 8:
            err = np.max(np.abs(g - r) / np.maximum(np.abs(r), 1e-30))
            assert err <= 1e-12, f"{name} fp64 parameter {p}: {err:.2e}"
        elif p in SWELL_ANGLES:
            d = np.abs(g - r)
            d = np.minimum(d, 360.0 - d)
            assert np.max(d / 360.0) <= 2e-6, f"{name} parameter {p}: {np.max(d):.3e} deg"
        else:
            bad = np.nonzero(g.astype(np.float32) != r.astype(np.float32))[0]
            assert bad.size == 0, f"{name} parameter {p}: {bad.size} points differ, e.g. {g[bad[0]]!r} vs {r[bad[0]]!r}"
    others = [p for p in range(1, 41) if p not in SWELL]
    assert np.all(got[[p - 1 for p in others]] == 7.0)
    # both parts present on these sea states, and the wind-sea and swell
    # energies add up to the total (the bins below EPSMIN aside)
    hs_ws, hs_sw = got[16].astype(float), got[24].astype(float)
    assert (hs_sw > 0).any() and (hs_ws > 0.01).any()
    tot = o.output_params(f, w.u10, w.udir, us, tw, zz, w.depth)[0][8].astype(float)
    assert np.allclose((hs_ws ** 2 + hs_sw ** 2) / 16.0, tot ** 2 / 16.0, rtol=1e-4, atol=1e-10)
    m.close()
