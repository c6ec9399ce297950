"""The band driver as the ranks run it: two processes on one GPU over gloo,
each a BandModel (wam_b200/halo.py) with the product kernels over its
latitude band, the halo strips staged through pinned host buffers and the
interior sub-steps overlapped with the exchange.  After two WAMODEL passes
every rank's owned points equal the whole-grid pass of the same process bit
for bit: spectra, TAUW, USTAR and Z0.  The ranks exchange on the host only;
no kernel waits on another rank."""
import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rank(rank, world, port, name, scale, overlap, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    ok = False
    try:
        from wam_b200 import WamModel
        from wam_b200.halo import BandModel, partition
        from wam_b200.synth import make_workload
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        w = make_workload(name, scale=scale)
        nprop = w.cfg["idelt"] // w.cfg["idelpro"]
        t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
        fields = [w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar]
        g = WamModel(w.cfg)
        g.set_grid(w.grid)
        g.set_depth(w.depth)
        g.prepare_propagation()
        g.prepare_source()
        F, G = w.spectrum_device(torch, dev), [t(a) for a in fields]
        SG = torch.empty_like(F)
        parts = partition(w.grid, world)
        p = parts[rank]
        a, b = p["ninf"], p["nsup"]
        bm = BandModel(w.cfg, w.grid, w.depth, parts, rank)
        f = F[:, :, a:b].clone()
        sc = torch.empty_like(f)
        L = [x[a:b].clone() for x in G]
        stream = torch.cuda.Stream(dev)
        torch.cuda.synchronize()
        for step in range(2):
            g.step_dev(F, nprop, *G, scratch=SG)
            g.sync()
            out = bm.step(f, sc, *L, stream=stream, overlap=overlap)
            stream.synchronize()
            if out is not f:
                f, sc = out, f
            lo, hi = p["lo"] - a, p["hi"] - a
            assert torch.equal(f[:, :, lo:hi], F[:, :, p["lo"]:p["hi"]]), f"rank {rank} pass {step}: spectrum"
            for i in (2, 3, 4):
                assert torch.equal(L[i][lo:hi], G[i][p["lo"]:p["hi"]]), f"rank {rank} pass {step}: field {i}"
        dist.barrier()
        ok = True
    finally:
        with open(os.path.join(out_dir, f"rank{rank}.ok"), "w") as fh:
            fh.write("1" if ok else "0")
        dist.destroy_process_group()


@pytest.mark.parametrize("name,scale,overlap", [("c1", 0.02, True), ("c1", 0.02, False), ("c0", 0.5, True)])
def test_band_model_two_ranks_gloo(tmp_path, name, scale, overlap):
    import torch.multiprocessing as mp
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank, args=(world, port, name, scale, overlap, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        assert (tmp_path / f"rank{r}.ok").read_text() == "1"
