"""Failure detection on the GPU, without a GPU fault.

An infinite value in one bin of one point's spectrum is an input that the
IMPLSCH kernel's own output scan catches: the implicit update keeps the bin
infinite (the growth limiter bounds the increment, the minimum-energy floor
is a maximum), wamgpu_sync returns WAMGPU_E_NUMERIC, the call clears the
flag, and the context stays usable.  Every float-to-index conversion in
IMPLSCH is clamped to its table (JU to [1, 300], MIJ to [1, ML] or [2, ML],
the TAU_PHI_HF index to [1, 199]) and every iteration has a fixed maximum
count, so a non-finite input stays in bounds and ends.  IMPLSCH is
pointwise: the other points' results are those of a clean run, bit for bit.

The ST6 physics carries the infinite bin into the whole point's spectrum,
which the scan reports.  Under ST4 a non-finite bin makes the point's source
terms NaN, and the implicit update's maxima (limiter, minimum-energy floor)
return the finite operand, so such a point ends on the floor spectrum and is
not reported; the cases here are therefore ST6 grids.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(w):
    from wam_b200 import WamModel
    m = WamModel(dict(w.cfg))
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    return m


def _run(m, w, f0):
    import torch
    dev = torch.device("cuda", 0)
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    f = torch.from_numpy(np.ascontiguousarray(f0.T)).to(dev)
    fields = [t(a) for a in (w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar)]
    torch.cuda.synchronize()
    m.implsch_dev(f, *fields)
    return f, fields


@pytest.mark.parametrize("name,scale", [("c1", 0.02), ("c1", 0.03)])
def test_nonfinite_spectrum_reported_and_context_usable(name, scale):
    from wam_b200._lib import WamgpuError
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale)
    m = _model(w)
    f0 = w.spectrum_f().astype(np.float32)
    bad = w.nsea // 3
    fb = f0.copy()
    fb[bad, 2, 5] = np.inf
    f_bad, fld_bad = _run(m, w, fb)
    with pytest.raises(WamgpuError, match=r"non-finite.*\(-6\)"):
        m.sync()
    m.sync()                                   # the flag was cleared by the report
    f_ok, fld_ok = _run(m, w, f0)
    m.sync()                                   # a clean step reports nothing
    ref = _model(w)
    f_ref, fld_ref = _run(ref, w, f0)
    ref.sync()
    assert np.array_equal(f_ok.cpu().numpy(), f_ref.cpu().numpy())
    for a, b in zip(fld_ok, fld_ref):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
    keep = np.ones(w.nsea, bool)
    keep[bad] = False
    assert np.array_equal(f_bad.cpu().numpy()[:, :, keep], f_ref.cpu().numpy()[:, :, keep])
    outs = [f_bad.cpu().numpy()[:, :, bad].ravel()] + [fld_bad[q].cpu().numpy()[bad:bad + 1] for q in (2, 3, 4)]
    assert not np.isfinite(np.concatenate(outs)).all()
