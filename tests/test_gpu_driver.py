"""The device-resident WAMODEL pass (wamodel.f90:286-451) with ice and dry
points: PUT_ICE / PUT_DRY (wamgpu_put_points_dev, wam_ice_module.f90:312-324,
wam_topo_module.f90:557-569) on the device spectrum and the integrated output
parameters of the resident state (wamgpu_output_parameters_dev), against the
oracle running the same sequence on the host."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(oracle_mod, name="c2", scale=0.05, precision=4):
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload, vary_sea_state
    w = vary_sea_state(make_workload(name, scale=scale))
    cfg = dict(w.cfg, precision=precision)
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    o = oracle_mod.Oracle(cfg, precision=precision)
    o.set_grid(w.grid)
    o.set_fields(w.depth)
    o.prepare_propagation()
    o.prepare_source()
    return w, m, o


@pytest.mark.parametrize("owned", [False, True])
def test_put_points_matches_oracle(oracle_mod, owned):
    """Every bin of the listed points, duplicates and all, and nothing else;
    with an owned range only the listed points inside it."""
    import torch
    w, m, o = _model(oracle_mod)
    n = w.nsea
    lo, hi = (n // 4, 3 * n // 4) if owned else (0, n)
    if owned:
        m.set_owned(lo, hi)
        m.prepare_propagation()
    rng = np.random.default_rng(3)
    pts = rng.integers(1, n + 1, size=max(3, n // 7)).astype(np.int32)
    pts = np.concatenate([pts, pts[:2]])  # repeated points, as an ice list may hold
    f = (rng.random((n, w.cfg["kl"], w.cfg["ml"])) + 0.5).astype(np.float32, order="F")
    ref = oracle_mod.put_points(f, pts, 0.0, nijs=lo + 1, nijl=hi)
    F = torch.tensor(np.ascontiguousarray(f.transpose(2, 1, 0)), device="cuda")
    m.put_points_dev(F, torch.tensor(pts, device="cuda"), 0.0)
    m.sync()
    got = np.asfortranarray(F.cpu().numpy().transpose(2, 1, 0))
    assert np.array_equal(got, ref)
    # the parameter-block form (PUT_ICE_PAR): one row per parameter
    blk = rng.random((40, n)).astype(np.float32)
    B = torch.tensor(blk, device="cuda")
    m.put_points_dev(B, torch.tensor(pts, device="cuda"), -999.0)
    m.sync()
    refb = oracle_mod.put_points(blk.T, pts, -999.0, nijs=lo + 1, nijl=hi).T
    assert np.array_equal(B.cpu().numpy(), refb)
    m.close()


def test_resident_pass_with_ice_and_dry(oracle_mod):
    """Three passes of [IDELT/IDELPRO x PROPAGS, IMPLSCH, PUT_ICE, PUT_DRY]
    with the spectrum resident on the device, then the output parameters,
    against the oracle's host sequence.  Ice and dry points hold exact zeros
    and the same output values as the oracle's; the other points' Hs and
    mean period agree within the per-step tolerance accumulated over three
    passes."""
    import torch
    w, m, o = _model(oracle_mod)
    n = w.nsea
    rng = np.random.default_rng(8)
    ice = rng.choice(np.arange(1, n + 1), size=n // 10, replace=False).astype(np.int32)
    dry = rng.choice(np.setdiff1d(np.arange(1, n + 1), ice), size=n // 20, replace=False).astype(np.int32)
    nprop = w.cfg["idelt"] // w.cfg["idelpro"]
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    F = w.spectrum_device(torch, dev)
    S = torch.empty_like(F)
    u10, udir, tauw, ustar, z0, roairn, wstar = (t(a) for a in (w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn,
                                                               w.wstar))
    ice_d, dry_d = torch.tensor(ice, device=dev), torch.tensor(dry, device=dev)
    fo = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    indep = o.indep()
    for _ in range(3):
        m.step_dev(F, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, scratch=S)
        m.put_points_dev(F, ice_d, 0.0)
        m.put_points_dev(F, dry_d, 0.0)
        for _ in range(nprop):
            fo = o.propags(fo)
        fo, tw, us, zz, _ = o.implsch(fo, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
        fo = oracle_mod.put_points(fo, ice, 0.0)
        fo = oracle_mod.put_points(fo, dry, 0.0)
    blk = m.output_parameters_dev(F, u10, udir, tauw, ustar, z0)
    m.sync()
    got = blk.cpu().numpy()
    fg = np.asfortranarray(F.cpu().numpy().transpose(2, 1, 0))
    ref, _, _ = o.output_params(fo, w.u10, w.udir, us, tw, zz, w.depth)
    frozen = np.concatenate([ice, dry]) - 1
    assert np.all(fg[frozen] == 0)
    assert np.array_equal(got[8][frozen], ref[8][frozen].astype(np.float32))
    live = np.setdiff1d(np.arange(n), frozen)
    for p in (9, 11, 12, 13):
        err = np.abs(got[p - 1][live] - ref[p - 1][live]) / ref[p - 1][live]
        assert err.max() <= 1e-4, (p, err.max())
    m.close()
