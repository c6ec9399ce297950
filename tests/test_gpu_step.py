"""The fused WAMODEL-pass entry points against the separate ones, through
the C ABI. Each path runs one pass of the PROP/PHYSICS loop body
(wamodel.f90:286-360) on the same inputs:
  A  nprop x wamgpu_propags_dev, then wamgpu_implsch_dev;
  B  wamgpu_step_dev;
  C  wamgpu_step_host on host arrays, whose copies overlap the kernels in
     chunks of sea points (PROPAGS sub-steps of the chunks as a wavefront).
Results must be bit-identical (spectrum, TAUW, USTAR, Z0 and, with LCFLX,
the flux arrays), with and without current refraction, on grids cut into
a few and into the maximum number of chunks, over two consecutive passes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(w, currents=False, lcflx=False):
    from wam_b200 import WamModel
    cfg = dict(w.cfg, lcflx=int(lcflx))
    if currents:
        cfg["refraction_c_run"] = 1
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    if currents:
        rng = np.random.default_rng(5)
        m.set_current(0.3 * rng.standard_normal(w.nsea), 0.3 * rng.standard_normal(w.nsea))
    m.prepare_propagation()
    m.prepare_source()
    return m


CASES = [("c0", 0.25, False, False), ("c1", 0.02, False, False), ("c1", 0.02, False, True), ("c2", 0.05, True, False),
         ("c1", 0.1, True, False)]


@pytest.mark.parametrize("name,scale,currents,lcflx", CASES,
                         ids=["c0", "c1", "c1-lcflx", "c2-currents", "c1-64-chunks-currents"])
def test_step_paths_identical(name, scale, currents, lcflx):
    import torch
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale)
    m = _model(w, currents, lcflx)
    n, kl, ml = w.nsea, w.cfg["kl"], w.cfg["ml"]
    nprop = w.cfg["idelt"] // w.cfg["idelpro"]
    f0 = w.spectrum_f()
    dev = torch.device("cuda", 0)
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    fields = [w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar]
    # path A and B state on the device
    fa = torch.from_numpy(np.ascontiguousarray(f0.T)).to(dev)
    fb = fa.clone()
    sa = torch.empty_like(fa)
    sb = torch.empty_like(fa)
    A = [t(a) for a in fields]
    B = [t(a) for a in fields]
    # path C state on the host
    fc = f0.copy(order="F")
    C = [np.array(a, np.float32) for a in fields]
    torch.cuda.synchronize()
    for step in range(2):
        u10, udir, tauw, ustar, z0, roairn, wstar = A
        for _ in range(nprop):
            m.propags_dev(fa, scratch=sa)
        m.implsch_dev(fa, u10, udir, tauw, ustar, z0, roairn, wstar)
        m.sync()
        flx_a = m.fluxes() if lcflx else None
        u10, udir, tauw, ustar, z0, roairn, wstar = B
        m.step_dev(fb, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, scratch=sb)
        m.sync()
        flx_b = m.fluxes() if lcflx else None
        u10, udir, tauw, ustar, z0, roairn, wstar = C
        m.step(fc, nprop, u10, udir, tauw, ustar, z0, roairn, wstar)
        flx_c = m.fluxes() if lcflx else None
        assert torch.equal(fa, fb), f"pass {step}: step_dev differs"
        got_c = torch.from_numpy(np.ascontiguousarray(fc.T)).to(dev)
        assert torch.equal(fa, got_c), f"pass {step}: step_host differs, max {(fa - got_c).abs().max().item()}"
        for i in (2, 3, 4):
            assert torch.equal(A[i], B[i]), (step, i)
            assert np.array_equal(A[i].cpu().numpy(), C[i]), (step, i)
        if lcflx:
            assert np.array_equal(flx_a, flx_b) and np.array_equal(flx_a, flx_c)
        assert torch.isfinite(fa).all()
    m.close()
