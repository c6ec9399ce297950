"""One grid over several ranks in latitude bands.

The layout follows the reference's 1-D MPI decomposition. The south-to-north
ordered sea points are split into contiguous bands: NMEAN = NSEA/P points per
rank, the first NREST ranks one more (wam_mpi_comp_module.f90:607-628). Each
band reads the spectra of its neighbours from a halo, refreshed before every
PROPAGS sub-step (wam_propagation_module.f90:704-709).

The reference packs exactly the needed neighbour points into NINF..NSUP
(wam_mpi_comp_module.f90:1063-1095). Here a rank keeps the contiguous index
range [ninf, nsup) that contains them: owned points plus halo, with neighbour
numbers renumbered to it. That costs a few more exchanged points and gives
the same results.

The library side is wamgpu_set_owned, wamgpu_set_counter and
wamgpu_propags_substep_dev. This module holds the host logic:
  - the partition;
  - the local grids;
  - the exchange plan;
  - a torch.distributed exchange of halo strips (NCCL on GPUs, gloo on CPU);
  - BandModel, one rank's driver of the WAMODEL pass.
"""
import numpy as np


def band_ranges(nsea, nranks):
    """Owned [lo, hi) per rank: NSEA/P points each, the first NSEA mod P ranks one more."""
    nmean, nrest = divmod(nsea, nranks)
    out, lo = [], 0
    for r in range(nranks):
        n = nmean + (1 if r < nrest else 0)
        out.append((lo, lo + n))
        lo += n
    return out


def _neighbours(grid, lo, hi):
    """0-based global numbers of all sea-point neighbours of points lo..hi-1."""
    n = int(grid["nsea"])
    klat = np.asarray(grid["klat"]).reshape(-1)
    klon = np.asarray(grid["klon"]).reshape(-1)
    nb = [klat[lo + n * s:hi + n * s] for s in range(klat.size // n)]
    nb += [klon[lo + n * s:hi + n * s] for s in range(klon.size // n)]
    nb = np.concatenate(nb) if nb else np.zeros(0, np.int64)
    return nb[nb > 0] - 1


def partition(grid, nranks):
    """Per rank a dict lo, hi (owned) and ninf, nsup (owned plus halo), 0-based."""
    parts = []
    for lo, hi in band_ranges(int(grid["nsea"]), nranks):
        nb = _neighbours(grid, lo, hi)
        ninf = int(min(lo, nb.min())) if nb.size else lo
        nsup = int(max(hi, nb.max() + 1)) if nb.size else hi
        parts.append(dict(lo=lo, hi=hi, ninf=ninf, nsup=nsup))
    return parts


def local_grid(grid, part):
    """The grid-module arrays of one band's extended range: KLAT/KLON
    renumbered to it (neighbours outside the range become 0, which only
    affects halo points, never computed); the per-latitude rows unchanged."""
    n = int(grid["nsea"])
    a, b = part["ninf"], part["nsup"]
    m = b - a

    def renumber(arr, slots):
        arr = np.asarray(arr).reshape(slots, n)[:, a:b].astype(np.int64)
        g = arr - 1
        inside = (arr > 0) & (g >= a) & (g < b)
        return np.where(inside, g - a + 1, 0).astype(np.int32).reshape(-1)

    klat = np.asarray(grid["klat"]).reshape(-1)
    klon = np.asarray(grid["klon"]).reshape(-1)
    out = dict(grid)
    out["nsea"] = m
    out["klat"] = renumber(klat, klat.size // n)
    out["klon"] = renumber(klon, klon.size // n)
    out["wlat"] = np.asarray(grid["wlat"]).reshape(-1, n)[:, a:b].reshape(-1).astype(np.float32)
    out["kfromij"] = np.asarray(grid["kfromij"])[a:b].astype(np.int32)
    for key in ("ixlg", "kxlt"):  # per-point grid positions
        if key in grid and np.asarray(grid[key]).size == n:
            out[key] = np.asarray(grid[key])[a:b]
    out.pop("_mask", None)
    return out


def exchange_plan(parts, me):
    """(sends, recvs) of rank `me`: lists of (peer, global lo, global hi) of
    owned points to send to the peer's halo, and of halo points to receive
    from the peer's owned range."""
    mine = parts[me]
    sends, recvs = [], []
    for q, p in enumerate(parts):
        if q == me:
            continue
        # my owned points inside q's extended range are q's halo
        lo, hi = max(mine["lo"], p["ninf"]), min(mine["hi"], p["nsup"])
        if lo < hi:
            sends.append((q, lo, hi))
        # q's owned points inside my extended range are my halo
        lo, hi = max(p["lo"], mine["ninf"]), min(p["hi"], mine["nsup"])
        if lo < hi:
            recvs.append((q, lo, hi))
    return sends, recvs


class HaloExchange:
    """Refreshes the halo of a band's spectrum (a tensor shaped (ML, KL, ld)
    over the band's extended range) from the owning ranks.

    The send and receive strips are allocated once per spectrum shape.  With
    NCCL they stay on the device and the P2P operations are ordered on the
    stream passed (torch's NCCL work waits for that stream, and the stream
    waits for it).  With gloo and a CUDA spectrum the strips are staged
    through pinned host buffers: the host waits only for the strip copies of
    that stream, sends and receives, and queues the halo writes on it.  With
    CPU tensors there is no stream."""

    def __init__(self, parts, me, group=None):
        self.parts, self.me, self.group = parts, me, group
        self.sends, self.recvs = exchange_plan(parts, me)
        self.base = parts[me]["ninf"]
        self._key = None

    def _alloc(self, f):
        import torch
        import torch.distributed as dist
        self._staged = f.is_cuda and dist.get_backend(self.group) != "nccl"
        dev = torch.device("cpu") if self._staged else f.device

        def strip(n):
            return torch.empty((f.shape[0], f.shape[1], n), dtype=f.dtype, device=dev, pin_memory=self._staged)
        self._send = [strip(hi - lo) for _, lo, hi in self.sends]
        self._recv = [strip(hi - lo) for _, lo, hi in self.recvs]
        self._key = (tuple(f.shape), f.dtype, str(f.device))

    def __call__(self, f, stream=None):
        import contextlib
        import torch
        import torch.distributed as dist
        if self._key != (tuple(f.shape), f.dtype, str(f.device)):
            self._alloc(f)
        b = self.base
        ctx = torch.cuda.stream(stream) if (f.is_cuda and stream is not None) else contextlib.nullcontext()
        with ctx:
            for buf, (q, lo, hi) in zip(self._send, self.sends):
                buf.copy_(f[:, :, lo - b:hi - b], non_blocking=True)
            if self._staged:
                torch.cuda.current_stream(f.device).synchronize()  # the strips are on the host
            ops = [dist.P2POp(dist.isend, buf, q, group=self.group) for buf, (q, _, _) in zip(self._send, self.sends)]
            ops += [dist.P2POp(dist.irecv, buf, q, group=self.group) for buf, (q, _, _) in zip(self._recv, self.recvs)]
            if ops:
                if dist.get_backend(self.group) == "nccl":
                    reqs = dist.batch_isend_irecv(ops)
                else:  # one request per strip
                    reqs = [op.op(op.tensor, op.peer, group=self.group) for op in ops]
                for req in reqs:
                    req.wait()
            for buf, (q, lo, hi) in zip(self._recv, self.recvs):
                f[:, :, lo - b:hi - b].copy_(buf, non_blocking=True)
        return f


def global_counter(local_counter, group=None, failed=False):
    """COUNTER agreed over the ranks: the largest of the ranks' own values.
    Every rank takes part even when its own CHECK_CFL failed (failed=True),
    and then every rank raises, as the reference aborts on any processor's
    negative coefficient (propagation:2025-2033)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([int(local_counter), int(bool(failed))], dtype=torch.int64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    if int(t[1].item()):
        raise RuntimeError("CHECK_CFL failed on a rank: negative propagation coefficient, reduce IDELPRO")
    return int(t[0].item())


class BandModel:
    """One rank's share of a grid on its GPU: a WamModel over the band's
    extended range with the owned points set, a halo exchange before every
    PROPAGS sub-step and the global COUNTER.

    The spectrum tensors are (ML, KL, nsup-ninf) over the extended range.
    The per-point fields cover it too; only owned points are integrated."""

    def __init__(self, cfg, grid, depth, parts, me, u=None, v=None, group=None):
        from .model import WamModel
        self.part = parts[me]
        self.lgrid = local_grid(grid, self.part)
        a, b = self.part["ninf"], self.part["nsup"]
        self.m = WamModel(cfg)
        self.m.set_grid(self.lgrid)
        self.m.set_depth(np.asarray(depth)[a:b])
        if u is not None:
            self.m.set_current(np.asarray(u)[a:b], np.asarray(v)[a:b])
        self.m.set_owned(self.part["lo"] - a, self.part["hi"] - a)
        try:
            _, cnt = self.m.prepare_propagation()
            failed = False
        except Exception:
            cnt, failed = 1, True
        self.counter = global_counter(cnt, group, failed)
        self.m.set_counter(self.counter)
        self.m.prepare_source()
        self.exchange = HaloExchange(parts, me, group)
        self.nprop = cfg["idelt"] // cfg["idelpro"]
        self.halo = self.m.halo_width()
        self._xs = None

    def step(self, f, scratch, u10, udir, tauw, ustar, z0, roairn, wstar, stream=None, overlap=True):
        """One WAMODEL pass on `stream` (a torch.cuda.Stream; default: the
        current stream); returns the tensor that holds the new spectrum (f or
        scratch: the sub-steps ping-pong between them).

        With overlap, each sub-step first runs the interior owned points (more
        than the halo width from the band's ends, so they read no halo point)
        on `stream` while the halo exchange runs on a second stream (NCCL) or
        on the host (gloo), and then the points near the band's ends once the
        halo has arrived.  Every kernel computes the same elements from the
        same inputs as the unsplit sub-step."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(f.device)
        h = s.cuda_stream
        o0, o1 = self.part["lo"] - self.part["ninf"], self.part["hi"] - self.part["ninf"]
        i0, i1 = o0 + self.halo, o1 - self.halo
        split = overlap and i0 < i1
        if split and self._xs is None:
            self._xs = torch.cuda.Stream(f.device)
            self._ev = (torch.cuda.Event(), torch.cuda.Event())
        src, dst = f, scratch
        for _ in range(self.nprop * self.counter):
            if split:
                ready, halo = self._ev
                ready.record(s)                                     # src complete
                self.m.propags_substep_range_dev(src, dst, i0, i1, stream=h)
                self._xs.wait_event(ready)
                self.exchange(src, stream=self._xs)                 # halo of src, beside the interior
                halo.record(self._xs)
                s.wait_event(halo)
                if o0 < i0:
                    self.m.propags_substep_range_dev(src, dst, o0, i0, stream=h)
                if i1 < o1:
                    self.m.propags_substep_range_dev(src, dst, i1, o1, stream=h)
            else:
                self.exchange(src, stream=s)
                self.m.propags_substep_dev(src, dst, stream=h)
            src, dst = dst, src
        self.m.implsch_dev(src, u10, udir, tauw, ustar, z0, roairn, wstar, stream=h)
        return src
