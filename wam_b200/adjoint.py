"""Reverse-mode harness over the C ABI's derivative entry points.

WamPass is a torch.autograd.Function for one WAMODEL pass: NPROP PROPAGS
calls of COUNTER sub-steps each (wam_propagation_module.f90:635-829), then
IMPLSCH (wam_source_module.f90:374-700).  The state is (FL3, TAUW); U10 is a
differentiable forcing.  UDIR, ROAIRN, WSTAR and the depth are held fixed.

The forward pass keeps one checkpoint per pass: the spectrum that enters
IMPLSCH, with TAUW and U10.  The backward pass runs wamgpu_implsch_adj_dev
at that checkpoint, which recomputes IMPLSCH's forward internally, and then
the transpose of PROPAGS NPROP times.

window_cost_and_grad runs an assimilation window of passes with an Hs misfit
at observed sea points, J = sum over passes and observed points of
(Hs - Hs_obs)^2 with Hs = 4 sqrt(sum_m DFIM(m) sum_k F(k, m)), the total
energy as the reference integrates it over the model's bins.  It returns J and
the gradients with respect to the initial spectrum, the initial TAUW and every
pass's U10.

The derivatives are for ST4 (IPHYS=1) physics on a context that covers its
whole grid.  Tensors are CUDA tensors of the context's precision, spectra
shaped (ML, KL, ld) with the sea point fastest.
"""
import torch


def _stream():
    """Handle of torch's current stream for the library calls.  torch's
    default stream is CUDA's legacy default stream, handle 0, which the
    library reads as "the context's own stream"; cudaStreamLegacy (0x1)
    names the legacy stream explicitly."""
    h = torch.cuda.current_stream().cuda_stream
    return h if h else 1


class WamPass(torch.autograd.Function):
    """(fl3, tauw, u10) -> (fl3_new, tauw_new) for one pass of `model`."""

    @staticmethod
    def forward(ctx, fl3, tauw, u10, model, nprop, udir, roairn, wstar):
        s = _stream()
        f = fl3.detach().clone()
        scratch = torch.empty_like(f)
        for _ in range(nprop):
            model.propags_dev(f, scratch=scratch, stream=s)
        f_mid = f.clone()
        tw = tauw.detach().clone()
        ustar, z0 = torch.empty_like(tw), torch.empty_like(tw)
        model.implsch_dev(f, u10.detach(), udir, tw, ustar, z0, roairn, wstar, stream=s)
        ctx.model, ctx.nprop = model, nprop
        ctx.save_for_backward(f_mid, tauw.detach(), u10.detach(), udir, roairn, wstar)
        return f, tw

    @staticmethod
    def backward(ctx, g_f, g_tw):
        f_mid, tw0, u10, udir, roairn, wstar = ctx.saved_tensors
        m, s = ctx.model, _stream()
        lam_f = torch.zeros_like(f_mid) if g_f is None else g_f.detach().clone().contiguous()
        lam_t = torch.zeros_like(tw0) if g_tw is None else g_tw.detach().clone().contiguous()
        lam_u = torch.empty_like(u10)
        m.implsch_adj_dev(f_mid, tw0, u10, udir, roairn, wstar, lam_f, lam_t, lam_u, stream=s)
        scratch = torch.empty_like(lam_f)
        for _ in range(ctx.nprop):
            m.propags_adj_dev(lam_f, scratch=scratch, stream=s)
        return lam_f, lam_t, lam_u, None, None, None, None, None


def significant_wave_height(f, dfim, points):
    """Hs = 4 sqrt(sum_m DFIM(m) sum_k F(k, m)) at the 0-based sea points."""
    e = (f[:, :, points].sum(dim=1) * dfim[:, None]).sum(dim=0)
    return 4.0 * torch.sqrt(e)


def window_cost_and_grad(model, fl3, tauw, u10_seq, udir, roairn, wstar, points, hs_obs, nprop=None):
    """J and its gradients over len(u10_seq) passes.

    u10_seq: a sequence of U10 tensors, one per pass; hs_obs: (passes,
    len(points)) observed Hs after each pass.  Returns (J, dJ/dfl3,
    dJ/dtauw, [dJ/du10 per pass])."""
    if nprop is None:
        nprop = model.cfg["idelt"] // model.cfg["idelpro"]
    dfim = torch.tensor(model.table("DFIM"), device=fl3.device, dtype=fl3.dtype)
    f0 = fl3.detach().clone().requires_grad_(True)
    t0 = tauw.detach().clone().requires_grad_(True)
    us = [u.detach().clone().requires_grad_(True) for u in u10_seq]
    f, tw = f0, t0
    J = torch.zeros((), device=fl3.device, dtype=fl3.dtype)
    for p, u in enumerate(us):
        f, tw = WamPass.apply(f, tw, u, model, nprop, udir, roairn, wstar)
        hs = significant_wave_height(f, dfim, points)
        J = J + ((hs - hs_obs[p]) ** 2).sum()
    J.backward()
    return J.detach(), f0.grad, t0.grad, [u.grad for u in us]
