"""Batched ensembles through the C ABI (wamgpu_batch_*). The members differ in:
  - size (uneven NSEA);
  - KL/ML and ST4/ST6 physics;
  - propagation: deep, or shallow with depth refraction;
  - number of sub-steps.
They advance in shared launches. Results must be bit-identical to each
member's own wamgpu_step_dev, both for direct batched launches (after
autotuning) and for replays of the captured CUDA graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _members():
    from wam_b200.synth import make_ensemble, make_workload
    ws = make_ensemble(n_members=6, seed=99, size_range=(150, 3000))
    ws.append(make_workload("c1", scale=0.02))   # ST6, shallow with depth refraction, 5 sub-steps
    ws.append(make_workload("c0", scale=0.2))    # ST4, deep, 1 deg
    return ws


def _model(w):
    from wam_b200 import WamModel
    m = WamModel(w.cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    return m


def _state(torch, w, dev):
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    f = w.spectrum_device(torch, dev)
    return [f, torch.zeros_like(f)] + [t(a) for a in (w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar)]


def test_batch_matches_members():
    import torch
    from wam_b200.batch import WamBatch
    dev = torch.device("cuda", 0)
    ws = _members()
    models = [_model(w) for w in ws]
    ref = [_state(torch, w, dev) for w in ws]
    bat = [[x.clone() for x in st] for st in ref]
    torch.cuda.synchronize()
    b = WamBatch(models)
    for g, st in enumerate(bat):
        b.set_member(g, *st)
    P, bs = b.tune()
    assert P in (4, 6, 8) and bs in (128, 256)

    def ref_step():
        for w, m, st in zip(ws, models, ref):
            f, sc, u10, udir, tauw, ustar, z0, roairn, wstar = st
            m.step_dev(f, w.cfg["idelt"] // w.cfg["idelpro"], u10, udir, tauw, ustar, z0, roairn, wstar, scratch=sc)
        for m in models:
            m.sync()

    def compare(tag):
        for g, (w, a, c) in enumerate(zip(ws, ref, bat)):
            n = w.nsea
            assert torch.equal(a[0][..., :n], c[0][..., :n]), f"{tag}: member {g} spectrum"
            for i in (4, 5, 6):
                assert torch.equal(a[i], c[i]), f"{tag}: member {g} field {i}"
        assert all(torch.isfinite(c[0]).all() for c in bat)

    for it in range(2):
        ref_step()
        b.step()
        b.sync()
        compare(f"direct pass {it}")
    b.capture()
    for it in range(2):
        ref_step()
        b.step()
        b.sync()
        compare(f"graph pass {it}")
    b.close()
    for m in models:
        m.close()


def test_batch_rejects_unprepared_and_missing_state():
    from wam_b200 import WamModel
    from wam_b200._lib import WamgpuError
    from wam_b200.batch import WamBatch
    from wam_b200.synth import make_workload
    w = make_workload("c0", scale=0.2)
    m = WamModel(w.cfg)
    m.set_grid(w.grid)
    with pytest.raises(WamgpuError, match="not prepared"):
        WamBatch([m])
    m.set_depth(w.depth)
    m.prepare_propagation()
    b = WamBatch([m])
    with pytest.raises(WamgpuError, match="no state"):
        b.step()
    b.close()
    m.close()
