"""Derivatives of one WAMODEL pass through the C ABI (ST4 physics).

The reference has no tangent-linear or adjoint code, so these are pinned by
the forward path itself:
  - IMPLSCH tangent-linear (wamgpu_implsch_tl_dev) against its adjoint
    (wamgpu_implsch_adj_dev): <TL dx, ly> = <dx, ADJ ly> at every sea point;
  - the tangent-linear against central finite differences of the production
    forward kernel (wamgpu_implsch_dev), both in FP64, and the
    tangent-linear's base state against that kernel's output;
  - the PROPAGS transpose (wamgpu_propags_adj_dev) against PROPAGS:
    <P d, l> = <d, P^T l> for the coefficient families;
  - the gradient of an Hs misfit over a window of passes through
    torch.autograd (wam_b200.adjoint) against central differences of the
    cost.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch, torch.device("cuda", 0)


def _s():
    """Library calls run on torch's current stream, ordered with the tensor
    work around them."""
    from wam_b200.adjoint import _stream
    return _stream()


def _spun_up(name, scale, precision, wstar=None, passes=3, isnonlin=None):
    """A prepared model and its state after a few forward passes."""
    torch, dev = _torch()
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale, precision=precision)
    if isnonlin is not None:
        w.cfg["isnonlin"] = isnonlin
    m = WamModel(w.cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    dt = torch.float64 if precision == 8 else torch.float32
    t = lambda a: torch.tensor(np.asarray(a, np.float64), dtype=dt, device=dev)
    st = dict(f=w.spectrum_device(torch, dev, dtype=dt), u10=t(w.u10), udir=t(w.udir), tauw=t(w.tauw),
              ustar=t(w.ustar), z0=t(w.z0), roairn=t(w.roairn),
              wstar=t(w.wstar) if wstar is None else torch.full((w.nsea,), wstar, dtype=dt, device=dev))
    nprop = w.cfg["idelt"] // w.cfg["idelpro"]
    for _ in range(passes):
        m.step_dev(st["f"], nprop, st["u10"], st["udir"], st["tauw"], st["ustar"], st["z0"], st["roairn"],
                   st["wstar"], scratch=torch.empty_like(st["f"]), stream=_s())
    torch.cuda.synchronize()
    return w, m, st, nprop


def _tl(m, st, dF, dT, dU):
    torch, _ = _torch()
    fo, dfo = torch.empty_like(st["f"]), torch.empty_like(st["f"])
    to, dto = torch.empty_like(st["tauw"]), torch.empty_like(st["tauw"])
    m.implsch_tl_dev(st["f"], dF, st["tauw"], dT, st["u10"], dU, st["udir"], st["roairn"], st["wstar"], fo, dfo, to, dto,
                     stream=_s())
    return fo, dfo, to, dto


def _perturbation(torch, st, seed):
    g = torch.Generator(device=st["f"].device).manual_seed(seed)
    rn = lambda x: torch.randn(x.shape, generator=g, device=x.device, dtype=x.dtype)
    return 0.1 * st["f"] * rn(st["f"]), 0.1 * st["tauw"] * rn(st["tauw"]), 0.3 * rn(st["u10"]), rn


@pytest.mark.parametrize("name,scale,wstar,isnonlin", [("c0", 0.2, None, None), ("c2", 0.04, None, None),
                                                        ("c2", 0.04, 0.8, None), ("c2", 0.04, None, 1)])
def test_implsch_tl_adjoint_dot_product_fp64(name, scale, wstar, isnonlin):
    torch, _ = _torch()
    w, m, st, _ = _spun_up(name, scale, 8, wstar, isnonlin=isnonlin)
    dF, dT, dU, rn = _perturbation(torch, st, 11)
    _, dfo, _, dto = _tl(m, st, dF, dT, dU)
    lF, lT = rn(st["f"]), rn(st["tauw"])
    aF, aT, aU = lF.clone(), lT.clone(), torch.empty_like(st["u10"])
    m.implsch_adj_dev(st["f"], st["tauw"], st["u10"], st["udir"], st["roairn"], st["wstar"], aF, aT, aU, stream=_s())
    lhs = (dfo * lF).sum(dim=(0, 1)) + dto * lT
    rhs = (dF * aF).sum(dim=(0, 1)) + dT * aT + dU * aU
    rel = ((lhs - rhs).abs() / torch.maximum(lhs.abs(), rhs.abs())).cpu().numpy()
    assert np.isfinite(rel).all()
    assert np.median(rel) < 1e-13 and rel.max() < 1e-10, (np.median(rel), rel.max())
    m.close()


@pytest.mark.parametrize("name,scale,isnonlin", [("c0", 0.2, None), ("c2", 0.04, None), ("c2", 0.04, 1)])
def test_implsch_tl_matches_forward_and_finite_differences(name, scale, isnonlin):
    torch, _ = _torch()
    w, m, st, _ = _spun_up(name, scale, 8, isnonlin=isnonlin)
    n = w.nsea
    dF, dT, dU, rn = _perturbation(torch, st, 5)
    fo, dfo, to, dto = _tl(m, st, dF, dT, dU)

    def forward(eps):
        f, tw = (st["f"] + eps * dF).contiguous(), st["tauw"] + eps * dT
        us, z0 = torch.empty_like(tw), torch.empty_like(tw)
        m.implsch_dev(f, st["u10"] + eps * dU, st["udir"], tw, us, z0, st["roairn"], st["wstar"], stream=_s())
        return f, tw

    # base state of the tangent-linear pass == the production kernel
    f0, t0 = forward(0.0)
    scale_f = f0.abs().amax(dim=(0, 1))
    assert float(((fo - f0).abs().amax(dim=(0, 1)) / scale_f).max()) < 1e-10
    assert float(((to - t0).abs() / t0.abs().clamp_min(1e-30)).max()) < 1e-10
    # central differences projected on random weights, per sea point
    lF, lT = rn(st["f"]), rn(st["tauw"])
    eps = 1e-4
    fp, tp = forward(eps)
    fm, tm = forward(-eps)
    j_fd = (((fp - fm) / (2 * eps)) * lF).sum(dim=(0, 1)) + (tp - tm) / (2 * eps) * lT
    j_tl = (dfo * lF).sum(dim=(0, 1)) + dto * lT
    rel = ((j_fd - j_tl).abs() / j_tl.abs().clamp_min(1e-300)).cpu().numpy()
    assert np.median(rel) < 1e-7, np.median(rel)
    # a point whose MAX/MIN branch switches inside +-eps has no derivative there
    assert (rel > 1e-4).sum() <= max(1, n // 100), (np.sort(rel)[-5:], n)
    m.close()


def test_implsch_tl_adjoint_dot_product_fp32():
    torch, _ = _torch()
    w, m, st, _ = _spun_up("c2", 0.04, 4)
    dF, dT, dU, rn = _perturbation(torch, st, 3)
    _, dfo, _, dto = _tl(m, st, dF, dT, dU)
    lF, lT = rn(st["f"]), rn(st["tauw"])
    aF, aT, aU = lF.clone(), lT.clone(), torch.empty_like(st["u10"])
    m.implsch_adj_dev(st["f"], st["tauw"], st["u10"], st["udir"], st["roairn"], st["wstar"], aF, aT, aU, stream=_s())
    d = lambda x: x.double()
    lhs = (d(dfo) * d(lF)).sum(dim=(0, 1)) + d(dto) * d(lT)
    rhs = (d(dF) * d(aF)).sum(dim=(0, 1)) + d(dT) * d(aT) + d(dU) * d(aU)
    rel = ((lhs - rhs).abs() / torch.maximum(lhs.abs(), rhs.abs())).cpu().numpy()
    assert np.isfinite(rel).all() and np.median(rel) < 1e-4, (np.median(rel), rel.max())
    m.close()


PROP_CASES = [(1, 0, 0, 0, 0), (1, 1, 0, 1, 1), (1, 1, 1, 0, 1), (0, 1, 1, 0, 1), (0, 0, 0, 0, 0), (1, 0, 1, 1, 0),
              (0, 1, 0, 0, 1)]


@pytest.mark.parametrize("spherical,shallow,current,reduced,refr_d", PROP_CASES)
def test_propags_transpose_dot_product(oracle_mod, spherical, shallow, current, reduced, refr_d):
    torch, dev = _torch()
    from wam_b200 import WamModel
    from wam_b200.model import make_config
    from wam_b200.synth import blob_mask, grf
    rng = np.random.default_rng(40 + 16 * spherical + 8 * shallow + 4 * current + 2 * reduced + refr_d)
    nx, ny = 40, 26
    mask = blob_mask(rng, nx, ny, 0.25, 2)
    xdello = 36000 * 2
    g = oracle_mod.build_grid(nx, ny, 30 * 360000, -10 * 360000, -10 * 360000 + (nx - 1) * xdello, 36000 * 2, xdello,
                              mask, reduced=bool(reduced))
    g["klat"] = g["klat"].astype(np.int32)
    cfg = make_config(24, 25, 0.04177, 1, 600, 300, g["delphi"], shallow_run=bool(shallow),
                      spherical_run=bool(spherical), refraction_d_run=bool(refr_d), refraction_c_run=bool(current),
                      reduced_grid=bool(reduced), precision=8)
    order = mask.T.ravel()
    depth = (15.0 + 300.0 * (0.5 + 0.5 * np.tanh(grf(rng, nx, ny, 4)))).T.ravel()[order]
    m = WamModel(cfg)
    m.set_grid(g)
    m.set_depth(depth)
    if current:
        m.set_current((0.8 * grf(rng, nx, ny, 5)).T.ravel()[order], (0.8 * grf(rng, nx, ny, 5)).T.ravel()[order])
    m.prepare_propagation()
    n, ld = g["nsea"], g["nsea"] + 3
    gen = torch.Generator(device=dev).manual_seed(7)
    d = torch.zeros((25, 24, ld), dtype=torch.float64, device=dev)
    lam = torch.zeros_like(d)
    d[..., :n] = torch.rand((25, 24, n), generator=gen, device=dev, dtype=torch.float64)
    lam[..., :n] = torch.randn((25, 24, n), generator=gen, device=dev, dtype=torch.float64)
    pd = d.clone()
    m.propags_dev(pd, stream=_s())
    plam = lam.clone()
    m.propags_adj_dev(plam, stream=_s())
    lhs = float((pd[..., :n] * lam[..., :n]).sum())
    rhs = float((d[..., :n] * plam[..., :n]).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (lhs, rhs, m.counter)
    assert float(plam[..., n:].abs().max()) == 0.0  # padding untouched
    m.close()


@pytest.mark.parametrize("name,scale,passes", [("c0", 0.2, 3), ("c2", 0.05, 2)])
def test_window_gradient_matches_finite_differences(name, scale, passes):
    torch, dev = _torch()
    from wam_b200.adjoint import WamPass, significant_wave_height, window_cost_and_grad
    w, m, st, nprop = _spun_up(name, scale, 8)
    n = w.nsea
    gen = torch.Generator(device=dev).manual_seed(21)
    points = torch.randperm(n, generator=gen, device=dev)[: max(4, n // 10)]
    us = [st["u10"] * (1.0 + 0.05 * p) for p in range(passes)]
    dfim = torch.tensor(m.table("DFIM"), device=dev, dtype=torch.float64)

    def cost(f0, t0, useq):
        with torch.no_grad():
            f, tw, hs = f0, t0, []
            for p, u in enumerate(useq):
                f, tw = WamPass.apply(f, tw, u, m, nprop, st["udir"], st["roairn"], st["wstar"])
                hs.append(significant_wave_height(f, dfim, points))
            return hs

    hs_ref = cost(st["f"], st["tauw"], us)
    hs_obs = [1.05 * h for h in hs_ref]
    J, gf, gt, gu = window_cost_and_grad(m, st["f"], st["tauw"], us, st["udir"], st["roairn"], st["wstar"], points,
                                         hs_obs, nprop)
    assert gf.shape == st["f"].shape and all(x is not None for x in gu)
    dF = 0.1 * st["f"] * torch.randn(st["f"].shape, generator=gen, device=dev, dtype=torch.float64)
    dT = 0.1 * st["tauw"] * torch.randn(st["tauw"].shape, generator=gen, device=dev, dtype=torch.float64)
    dU = [0.3 * torch.randn(st["u10"].shape, generator=gen, device=dev, dtype=torch.float64) for _ in us]

    def J_at(eps):
        hs = cost(st["f"] + eps * dF, st["tauw"] + eps * dT, [u + eps * du for u, du in zip(us, dU)])
        return sum(float(((h - o) ** 2).sum()) for h, o in zip(hs, hs_obs))

    assert abs(J_at(0.0) - float(J)) <= 1e-12 * float(J)
    eps = 1e-5
    fd = (J_at(eps) - J_at(-eps)) / (2 * eps)
    ad = float((gf * dF).sum() + (gt * dT).sum() + sum((a * b).sum() for a, b in zip(gu, dU)))
    assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
    m.close()


def test_checkpointed_window_through_the_c_abi_matches_autograd():
    """wamgpu_step_ckpt_dev forward and wamgpu_step_adj_dev backward, with the
    Hs misfit's adjoint added between steps, give the autograd harness's
    gradients (FP64)."""
    torch, dev = _torch()
    from wam_b200._lib import WamgpuError
    from wam_b200.adjoint import significant_wave_height, window_cost_and_grad
    w, m, st, nprop = _spun_up("c0", 0.2, 8)
    n, passes = w.nsea, 3
    gen = torch.Generator(device=dev).manual_seed(5)
    points = torch.randperm(n, generator=gen, device=dev)[: max(4, n // 8)]
    us = [st["u10"] * (1.0 + 0.04 * p) for p in range(passes)]
    dfim = torch.tensor(m.table("DFIM"), device=dev, dtype=torch.float64)
    hs_obs = [None] * passes
    J, gf, gt, gu = None, None, None, None
    # observations: 5 % above a plain forward run
    f, tw = st["f"].clone(), st["tauw"].clone()
    ustar, z0, sc = torch.empty_like(tw), torch.empty_like(tw), torch.empty_like(f)
    for p in range(passes):
        m.step_dev(f, nprop, us[p], st["udir"], tw, ustar, z0, st["roairn"], st["wstar"], scratch=sc, stream=_s())
        hs_obs[p] = 1.05 * significant_wave_height(f, dfim, points)
    J, gf, gt, gu = window_cost_and_grad(m, st["f"], st["tauw"], us, st["udir"], st["roairn"], st["wstar"], points,
                                         hs_obs, nprop)
    # the same window through the checkpoint entry points
    ld = st["f"].shape[-1]
    m.checkpoint_reserve(passes, ld)
    f, tw = st["f"].clone(), st["tauw"].clone()
    hs = []
    for p in range(passes):
        m.step_ckpt_dev(p, f, nprop, us[p], st["udir"], tw, ustar, z0, st["roairn"], st["wstar"], scratch=sc, stream=_s())
        hs.append(significant_wave_height(f, dfim, points))
    J2 = sum(float(((h - o) ** 2).sum()) for h, o in zip(hs, hs_obs))
    lam_f, lam_t = torch.zeros_like(st["f"]), torch.zeros_like(st["tauw"])
    lam_u = [torch.empty_like(st["u10"]) for _ in range(passes)]
    for p in reversed(range(passes)):
        g = 16.0 * (hs[p] - hs_obs[p]) / hs[p]  # dJ/dE at the observed points, E = sum DFIM sum F
        lam_f[:, :, points] += dfim[:, None, None] * g[None, None, :]
        m.step_adj_dev(p, nprop, lam_f, lam_t, lam_u[p], st["udir"], st["roairn"], st["wstar"], scratch=sc, stream=_s())
    torch.cuda.synchronize()
    assert abs(J2 - float(J)) <= 1e-12 * float(J)
    rel = lambda a, b: float((a - b).abs().max() / b.abs().max())
    assert rel(lam_f, gf) < 1e-10 and rel(lam_t, gt) < 1e-10, (rel(lam_f, gf), rel(lam_t, gt))
    for a, b in zip(lam_u, gu):
        assert rel(a, b) < 1e-10
    # slots and leading dimension are checked
    with pytest.raises(WamgpuError, match="slot"):
        m.step_adj_dev(passes, nprop, lam_f, lam_t, lam_u[0], st["udir"], st["roairn"], st["wstar"], stream=_s())
    with pytest.raises(WamgpuError, match="ld differs"):
        m.step_adj_dev(0, nprop, lam_f, lam_t, lam_u[0], st["udir"], st["roairn"], st["wstar"], ld=ld + 1, stream=_s())
    m.checkpoint_reserve(0, ld)
    m.close()
