"""Latitude bands on one GPU: two band contexts of one grid (extended ranges,
owned points set with wamgpu_set_owned, the larger COUNTER installed with
wamgpu_set_counter) advanced in lockstep.  Before every PROPAGS sub-step
each band's halo is copied from the other band's owned points.  This is the
exchange that the ranks do over NCCL, here as tensor copies in one process.
The owned points must equal the single-context pass bit for bit: spectra,
TAUW, USTAR and Z0."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,scale", [("c1", 0.02), ("c0", 0.25)])
def test_two_bands_match_whole_grid(name, scale):
    import torch
    from wam_b200 import WamModel
    from wam_b200.halo import exchange_plan, local_grid, partition
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale)
    dev = torch.device("cuda", 0)
    n, nprop = w.nsea, w.cfg["idelt"] // w.cfg["idelpro"]
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    fields = [w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar]
    # whole grid
    g = WamModel(w.cfg)
    g.set_grid(w.grid)
    g.set_depth(w.depth)
    g.prepare_propagation()
    g.prepare_source()
    F = w.spectrum_device(torch, dev)
    SG = torch.empty_like(F)
    G = [t(a) for a in fields]
    # two bands
    parts = partition(w.grid, 2)
    bands = []
    for r, p in enumerate(parts):
        m = WamModel(w.cfg)
        m.set_grid(local_grid(w.grid, p))
        m.set_depth(np.asarray(w.depth)[p["ninf"]:p["nsup"]])
        m.set_owned(p["lo"] - p["ninf"], p["hi"] - p["ninf"])
        _, cnt = m.prepare_propagation()
        bands.append(dict(m=m, p=p, cnt=cnt, f=F[:, :, p["ninf"]:p["nsup"]].clone(), fields=[x[p["ninf"]:p["nsup"]].clone() for x in G]))
    counter = max(b["cnt"] for b in bands)
    assert counter == g.counter
    for b in bands:
        b["m"].set_counter(counter)
        b["m"].prepare_source()
        b["s"] = torch.empty_like(b["f"])
    torch.cuda.synchronize()
    for step in range(2):
        g.step_dev(F, nprop, *G, scratch=SG)
        g.sync()
        src = [b["f"] for b in bands]
        dst = [b["s"] for b in bands]
        for _ in range(nprop * counter):
            for r, b in enumerate(bands):  # halo of band r from the owner
                for q, lo, hi in exchange_plan(parts, r)[1]:
                    pq = parts[q]
                    src[r][:, :, lo - b["p"]["ninf"]:hi - b["p"]["ninf"]] = src[q][:, :, lo - pq["ninf"]:hi - pq["ninf"]]
            for r, b in enumerate(bands):
                b["m"].propags_substep_dev(src[r], dst[r])
            for b in bands:
                b["m"].sync()
            src, dst = dst, src
        for r, b in enumerate(bands):
            b["m"].implsch_dev(src[r], *b["fields"])
            b["m"].sync()
            b["f"], b["s"] = src[r], dst[r]
        for b in bands:
            p = b["p"]
            a, c = p["lo"] - p["ninf"], p["hi"] - p["ninf"]
            assert torch.equal(b["f"][:, :, a:c], F[:, :, p["lo"]:p["hi"]]), f"step {step} spectrum"
            for i in (2, 3, 4):
                assert torch.equal(b["fields"][i][a:c], G[i][p["lo"]:p["hi"]]), f"step {step} field {i}"
    g.close()
    for b in bands:
        b["m"].close()
