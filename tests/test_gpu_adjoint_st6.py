"""Adjoint of IMPLSCH with ST6 physics (wamgpu_implsch_adj_dev, IPHYS = 2:
SINPUT_ST6 with LFACTOR, SDISSIP_ST6, W3SWL6, the DIA and the implicit
update, wam_source_module.f90:4465-5252) against central finite differences
of the forward kernel in FP64.

IMPLSCH acts point by point, so every sea point gives its own check:
J_p = <lambda, FL3_out> + lambda_T TAUW_out at point p, perturbed along a
random direction of its spectrum and U10.  The discrete decisions (cut-off
indices, the LFACTOR iteration count and its sign sequence, the wind-sea
mask, MAX/MIN branches) are frozen in the adjoint; a perturbation of 1e-7
rarely crosses one, so a few points may disagree, as for ST4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(oracle_mod, name="c1", scale=0.02, steps=3):
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload, vary_sea_state
    w = vary_sea_state(make_workload(name, scale=scale))
    o = oracle_mod.Oracle(w.cfg)
    o.set_grid(w.grid); o.set_fields(w.depth); o.prepare_propagation(); o.prepare_source()
    f = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    for _ in range(steps):
        f, tw, us, zz, _ = o.implsch(f, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, o.indep())
        for _ in range(w.sub_steps):
            f = o.propags(f)
    m = WamModel(dict(w.cfg, precision=8))
    m.set_grid(w.grid); m.set_depth(w.depth); m.prepare_propagation(); m.prepare_source()
    return w, m, f, tw


def test_st6_adjoint_matches_central_differences(oracle_mod):
    import torch
    w, m, f, tw = _state(oracle_mod)
    assert w.cfg["iphys"] == 2
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.asarray(a, np.float64), device=dev)
    F0 = t(np.ascontiguousarray(np.asarray(f).transpose(2, 1, 0)))
    U0, D0, T0, R0, W0 = t(w.u10), t(w.udir), t(tw), t(w.roairn), t(w.wstar)
    g = torch.Generator(device=dev).manual_seed(5)
    rn = lambda x: torch.randn(x.shape, generator=g, device=dev, dtype=x.dtype)
    lF, lT = rn(F0), rn(T0)
    dF, dU = rn(F0) * F0, rn(U0)

    def J(eps):
        F, T = F0 + eps * dF, T0.clone()
        US, Z = torch.zeros_like(T0), torch.zeros_like(T0)
        m.implsch_dev(F, U0 + eps * dU, D0, T, US, Z, R0, W0)
        m.sync()
        return (F * lF).sum(dim=(0, 1)) + T * lT  # per sea point

    aF, aT, aU = lF.clone(), lT.clone(), torch.empty_like(U0)
    m.implsch_adj_dev(F0, T0, U0, D0, R0, W0, aF, aT, aU)
    m.sync()
    assert torch.all(aT == 0), "ST6 does not read the input TAUW"
    grad = (aF * dF).sum(dim=(0, 1)) + aU * dU
    eps = 1e-7
    fd = (J(eps) - J(-eps)) / (2 * eps)
    rel = ((grad - fd).abs() / torch.maximum(fd.abs(), grad.abs()).clamp_min(1e-300)).cpu().numpy()
    assert np.isfinite(rel).all()
    assert np.median(rel) < 1e-6, np.median(rel)
    assert np.mean(rel < 1e-4) >= 0.95, (np.mean(rel < 1e-4), np.sort(rel)[-5:])
    m.close()


def test_st6_checkpointed_window(oracle_mod):
    """Two checkpointed WAMODEL passes (wamgpu_step_ckpt_dev) and their
    adjoints (wamgpu_step_adj_dev) with ST6 physics: the window gradient
    against a central difference of the window cost along a random
    direction of the initial spectrum and of both passes' U10."""
    import torch
    w, m, f, tw = _state(oracle_mod)
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.asarray(a, np.float64), device=dev)
    F0 = t(np.ascontiguousarray(np.asarray(f).transpose(2, 1, 0)))
    D0, T0, R0, W0 = t(w.udir), t(tw), t(w.roairn), t(w.wstar)
    U = [t(w.u10), t(w.u10) * 1.05]
    nprop = w.cfg["idelt"] // w.cfg["idelpro"]
    g = torch.Generator(device=dev).manual_seed(6)
    rn = lambda x: torch.randn(x.shape, generator=g, device=dev, dtype=x.dtype)
    lam = rn(F0)
    dF, dU = rn(F0) * F0, [rn(U[0]), rn(U[1])]
    sc = torch.empty_like(F0)
    m.checkpoint_reserve(2, F0.shape[-1])

    def cost(eps, ckpt=False):
        F, T = F0 + eps * dF, T0.clone()
        US, Z = torch.zeros_like(T0), torch.zeros_like(T0)
        for p in range(2):
            u = U[p] + eps * dU[p]
            if ckpt:
                m.step_ckpt_dev(p, F, nprop, u, D0, T, US, Z, R0, W0, scratch=sc)
            else:
                m.step_dev(F, nprop, u, D0, T, US, Z, R0, W0, scratch=sc)
        m.sync()
        return float((F * lam).sum())

    cost(0.0, ckpt=True)
    lF, lT = lam.clone(), torch.zeros_like(T0)
    lU = [torch.empty_like(U[0]) for _ in range(2)]
    for p in reversed(range(2)):
        m.step_adj_dev(p, nprop, lF, lT, lU[p], D0, R0, W0, scratch=sc)
    m.sync()
    grad = float((lF * dF).sum() + sum((a * b).sum() for a, b in zip(lU, dU)))
    eps = 1e-7
    fd = (cost(eps) - cost(-eps)) / (2 * eps)
    assert abs(grad - fd) <= 1e-5 * abs(fd), (grad, fd)
    m.checkpoint_reserve(0, F0.shape[-1])
    m.close()
