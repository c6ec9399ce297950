"""Direction counts beyond one warp's 32 lanes, against the CPU oracle.

The source kernels give each lane of a warp one direction.  The directions
beyond the first 32 (KL - 32 of them) are done in batches over frequencies
(DIA, SDISSIP_ARD and their adjoints), with batch sizes that depend on KL:

  * KL = 33: one extra direction, up to 31 MCs per DIA batch;
  * KL = 48: 16 extra directions, one MC per batch, 64 slot entries (two per
    lane);
  * KL = 64: 32 extra directions, where the host enlarges the scratch rows.

The configurations themselves use KL = 24 and 36.  Each variant runs the
small open-ocean grid for ST4 and ST6:
  * the FP32 step through the host-buffer entry point, within the tolerances
    of tests/test_gpu_parity.py (2e-6 ST4, 1e-4 ST6 per sea point);
  * the FP64 step against the FP64 oracle (1e-12 ST4, 1e-9 ST6);
  * for ST4, the FP64 tangent-linear/adjoint dot product at every sea point.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = [(33, 1), (48, 1), (64, 1), (33, 2), (48, 2), (64, 2)]


def _setup(oracle_mod, w, precision):
    from wam_b200 import WamModel
    cfg = dict(w.cfg, precision=precision)
    o = oracle_mod.Oracle(cfg, precision=precision)
    o.set_grid(w.grid)
    o.set_fields(w.depth, None, None)
    rc, cfl, cnt = o.prepare_propagation()
    assert rc == 0
    o.prepare_source()
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    return o, m


def _spinup(o, w, steps=3):
    indep = o.indep()
    f = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    for _ in range(steps):
        f, tw, us, zz, _ = o.implsch(f, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
        f = o.propags(f)
    return (np.asfortranarray(f.astype(np.float32)), tw.astype(np.float32), us.astype(np.float32),
            zz.astype(np.float32), indep)


def _point_rel(a, ref):
    ref = np.asarray(ref)
    pmax = np.abs(ref).max(axis=(1, 2))
    return (np.abs(np.asarray(a) - ref).max(axis=(1, 2))) / np.maximum(pmax, 1e-30)


def _check_points(err, tol, label):
    bad = err > tol
    assert bad.mean() <= 0.01, f"{label}: {bad.sum()} of {err.size} points above {tol} (max {err.max():.3e})"
    assert err.max() <= 1e-2, f"{label}: max point error {err.max():.3e}"


@pytest.mark.parametrize("kl,iphys", VARIANTS, ids=[f"kl{k}-st{4 if p == 1 else 6}" for k, p in VARIANTS])
def test_implsch_direction_counts(oracle_mod, kl, iphys):
    import torch
    from wam_b200.synth import make_direction_variant
    w = make_direction_variant(kl, iphys)
    o, m = _setup(oracle_mod, w, 4)
    f, tw, us, zz, indep = _spinup(o, w)
    # FP32 through the host-buffer entry point
    fo, two, uso, zo, _ = o.implsch(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
    fg = np.asfortranarray(f.copy())
    tg, ug, zg = tw.copy(), us.copy(), zz.copy()
    m.implsch(fg, w.u10, w.udir, tg, ug, zg, w.roairn, w.wstar)
    _check_points(_point_rel(fg, fo), 2e-6 if iphys == 1 else 1e-4, f"KL={kl} FP32")
    assert np.max(np.abs(ug - uso) / uso) <= 1e-5
    m.close()
    # FP64 on the device against the FP64 oracle
    o64, m64 = _setup(oracle_mod, w, 8)
    fo, two, uso, zo, _ = o64.implsch(f.astype(float), w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
    dev = torch.device("cuda")
    ten = lambda a: torch.tensor(np.asarray(a), dtype=torch.float64, device=dev)
    F = ten(np.ascontiguousarray(np.asarray(f).transpose(2, 1, 0)))
    T, U, Z = ten(tw), ten(us), ten(zz)
    m64.implsch_dev(F, ten(w.u10), ten(w.udir), T, U, Z, ten(w.roairn), ten(w.wstar))
    m64.sync()
    err = _point_rel(F.cpu().numpy().transpose(2, 1, 0), fo)
    _check_points(err, 1e-12 if iphys == 1 else 1e-9, f"KL={kl} FP64")
    assert np.allclose(U.cpu().numpy(), uso, rtol=1e-12)
    m64.close()


@pytest.mark.parametrize("kl", [33, 48, 64])
def test_implsch_adjoint_dot_product_direction_counts(kl):
    """<TL dx, ly> = <dx, ADJ ly> per sea point, FP64, ST4."""
    import torch
    from wam_b200 import WamModel
    from wam_b200.adjoint import _stream
    from wam_b200.synth import make_direction_variant
    dev = torch.device("cuda", 0)
    w = make_direction_variant(kl, 1, precision=8)
    m = WamModel(w.cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    t = lambda a: torch.tensor(np.asarray(a, np.float64), dtype=torch.float64, device=dev)
    st = dict(f=w.spectrum_device(torch, dev, dtype=torch.float64), u10=t(w.u10), udir=t(w.udir), tauw=t(w.tauw),
              ustar=t(w.ustar), z0=t(w.z0), roairn=t(w.roairn), wstar=t(w.wstar))
    s = _stream()
    for _ in range(3):
        m.step_dev(st["f"], 1, st["u10"], st["udir"], st["tauw"], st["ustar"], st["z0"], st["roairn"], st["wstar"],
                   scratch=torch.empty_like(st["f"]), stream=s)
    g = torch.Generator(device=dev).manual_seed(11)
    rn = lambda x: torch.randn(x.shape, generator=g, device=dev, dtype=x.dtype)
    dF, dT, dU = 0.1 * st["f"] * rn(st["f"]), 0.1 * st["tauw"] * rn(st["tauw"]), 0.3 * rn(st["u10"])
    fo, dfo = torch.empty_like(st["f"]), torch.empty_like(st["f"])
    to, dto = torch.empty_like(st["tauw"]), torch.empty_like(st["tauw"])
    m.implsch_tl_dev(st["f"], dF, st["tauw"], dT, st["u10"], dU, st["udir"], st["roairn"], st["wstar"], fo, dfo, to,
                     dto, stream=s)
    lF, lT = rn(st["f"]), rn(st["tauw"])
    aF, aT, aU = lF.clone(), lT.clone(), torch.empty_like(st["u10"])
    m.implsch_adj_dev(st["f"], st["tauw"], st["u10"], st["udir"], st["roairn"], st["wstar"], aF, aT, aU, stream=s)
    torch.cuda.synchronize()
    lhs = (dfo * lF).sum(dim=(0, 1)) + dto * lT
    rhs = (dF * aF).sum(dim=(0, 1)) + dT * aT + dU * aU
    rel = ((lhs - rhs).abs() / torch.maximum(lhs.abs(), rhs.abs())).cpu().numpy()
    assert np.isfinite(rel).all()
    assert np.median(rel) < 1e-13 and rel.max() < 1e-10, (np.median(rel), rel.max())
    m.close()
