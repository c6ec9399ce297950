"""Latitude bands on CPU: the partition and exchange plan of wam_b200.halo,
and two gloo ranks that propagate their bands with the oracle's PROPAGS
(one call per IDELPRO, halo refreshed before each) reproduce the global
propagation of the same grid bit for bit on their owned points."""
import os
import socket

import numpy as np
import pytest


def _workload():
    from wam_b200.synth import make_workload
    return make_workload("c1", scale=0.02)   # spherical shallow grid with depth refraction


@pytest.mark.parametrize("nranks", [2, 3, 5])
def test_partition_and_plan(nranks):
    from wam_b200.halo import band_ranges, exchange_plan, local_grid, partition
    w = _workload()
    n = w.nsea
    r = band_ranges(n, nranks)
    assert r[0][0] == 0 and r[-1][1] == n and all(a[1] == b[0] for a, b in zip(r, r[1:]))
    sizes = [hi - lo for lo, hi in r]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    parts = partition(w.grid, nranks)
    klat = np.asarray(w.grid["klat"]).reshape(-1, n)
    for p in parts:
        lg = local_grid(w.grid, p)
        own = np.arange(p["lo"], p["hi"])
        # every neighbour of an owned point is inside the band's range, renumbered
        lk = np.asarray(lg["klat"]).reshape(-1, lg["nsea"])
        for s in range(klat.shape[0]):
            g = klat[s, own]
            loc = lk[s, own - p["ninf"]]
            assert np.array_equal(np.where(g > 0, g - p["ninf"], 0), loc)
    # what r sends to q is what q receives from r
    for me in range(nranks):
        sends, _ = exchange_plan(parts, me)
        for q, lo, hi in sends:
            assert (me, lo, hi) in exchange_plan(parts, q)[1]


def _rank(rank, world, port, nprop, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Oracle
        from wam_b200.halo import HaloExchange, global_counter, local_grid, partition
        w = _workload()
        parts = partition(w.grid, world)
        p = parts[rank]
        lg = local_grid(w.grid, p)
        o = Oracle(w.cfg)
        o.set_grid(lg)
        o.set_fields(np.asarray(w.depth)[p["ninf"]:p["nsup"]])
        rc, _, cnt = o.prepare_propagation()
        assert rc == 0 and global_counter(cnt) == 1
        f = w.spectrum_f().astype(float)[p["ninf"]:p["nsup"]]
        t = torch.from_numpy(np.ascontiguousarray(f.T))      # (ML, KL, n_ext)
        ex = HaloExchange(parts, rank)
        for _ in range(nprop):
            ex(t)
            t = torch.from_numpy(np.ascontiguousarray(o.propags(np.asfortranarray(t.numpy().T)).T))
        own = t.numpy()[:, :, p["lo"] - p["ninf"]:p["hi"] - p["ninf"]]
        np.save(os.path.join(out_dir, f"band{rank}.npy"), own)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_bands_match_global_propagation_gloo(tmp_path):
    import torch.multiprocessing as mp
    from oracle.oracle import Oracle
    from wam_b200.halo import partition
    world, nprop = 2, 3
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank, args=(world, port, nprop, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    w = _workload()
    o = Oracle(w.cfg)
    o.set_grid(w.grid)
    o.set_fields(w.depth)
    rc, _, cnt = o.prepare_propagation()
    assert rc == 0 and cnt == 1
    f = w.spectrum_f().astype(float)
    for _ in range(nprop):
        f = o.propags(f)
    ref = np.ascontiguousarray(f.T)
    for r, p in enumerate(partition(w.grid, world)):
        got = np.load(tmp_path / f"band{r}.npy")
        assert np.array_equal(got, ref[:, :, p["lo"]:p["hi"]]), r


def _counter_rank(rank, world, port, failing, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        from wam_b200.halo import global_counter
        # COUNTER is the largest of the ranks' values; a CHECK_CFL failure on
        # one rank raises on every rank after the same collective.
        res = []
        res.append(str(global_counter(rank + 1)))
        try:
            global_counter(2, failed=(rank == failing))
            res.append("no error")
        except RuntimeError as e:
            res.append("raised: " + str(e).split(":")[0])
        # the group stays usable after the reported failure
        res.append(str(global_counter(5 - rank)))
        with open(os.path.join(out_dir, f"counter{rank}.txt"), "w") as f:
            f.write("\n".join(res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("failing", [0, 1])
def test_check_cfl_failure_raises_on_every_rank(tmp_path, failing):
    import torch.multiprocessing as mp
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_counter_rank, args=(world, port, failing, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        lines = (tmp_path / f"counter{r}.txt").read_text().splitlines()
        assert lines == [str(world), "raised: CHECK_CFL failed on a rank", "5"], (r, lines)


def _absent_peer_rank(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
    msg = "completed"
    try:
        from wam_b200.halo import HaloExchange, partition
        w = _workload()
        parts = partition(w.grid, world)
        p = parts[rank]
        dist.barrier()
        if rank == 1:
            return           # leaves between steps, with nothing in flight
        t = torch.zeros((w.cfg["ml"], w.cfg["kl"], p["nsup"] - p["ninf"]), dtype=torch.float64)
        try:
            HaloExchange(parts, rank)(t)
        except Exception as e:    # the short process-group timeout ends the exchange
            msg = "error: " + type(e).__name__
        with open(os.path.join(out_dir, f"absent{rank}.txt"), "w") as f:
            f.write(msg)
    finally:
        if rank == 0:
            dist.destroy_process_group()


def test_halo_exchange_with_an_absent_rank_ends_in_error(tmp_path):
    """A rank that leaves between sub-steps: the other rank's next exchange
    ends with an error from the process group's timeout instead of waiting."""
    import torch.multiprocessing as mp
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_absent_peer_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    assert (tmp_path / "absent0.txt").read_text().startswith("error: ")
