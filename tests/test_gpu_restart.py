"""Restart files from and to device buffers (wamgpu_restart_write /
wamgpu_restart_read: SAVE_RESTART_FILE and CONNECT_RESTART,
wam_restart_module.f90:414-591, 109-327) in the reference's sequential
unformatted record layout.  The oracle's record reader and writer
(oracle.read_restart / write_restart) restate that layout: a file the
library writes from the device state reads back there to the same values,
and a file written there reads into the device buffers bit for bit, with and
without the IJ2NEWIJ renumbering."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DATES = {"CDTPRO": "20260101120000", "CDTSOU": "20260101120000", "CDA": "20260101130000",
         "CDTA": "20260101000000", "CDCA": "20260101000000"}


def _state(precision=4):
    import torch
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload
    w = make_workload("c2", scale=0.05)
    cfg = dict(w.cfg, precision=precision)
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    m.prepare_source()
    dev = torch.device("cuda")
    dt = torch.float64 if precision == 8 else torch.float32
    t = lambda a: torch.tensor(np.asarray(a, np.float64), dtype=dt, device=dev)
    F = w.spectrum_device(torch, dev, ld=w.nsea + 3, dtype=dt)
    S = torch.empty_like(F)
    fields = [t(a) for a in (w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn, w.wstar)]
    for _ in range(2):
        m.step_dev(F, w.sub_steps, *fields, scratch=S)
    m.sync()
    rng = np.random.default_rng(2)
    extra = dict(depth=t(w.depth), u=t(rng.standard_normal(w.nsea)), v=t(rng.standard_normal(w.nsea)))
    return w, m, F, fields, extra


@pytest.mark.parametrize("renumber", [False, True])
@pytest.mark.parametrize("precision", [4, 8])
def test_restart_written_from_device(tmp_path, oracle_mod, precision, renumber):
    w, m, F, fields, extra = _state(precision)
    n = w.nsea
    perm = np.random.default_rng(1).permutation(n).astype(np.int32) + 1 if renumber else None
    path = tmp_path / "restart.bin"
    m.restart_write(path, F, fields[0], fields[1], fields[2], DATES, ij2newij=perm, **extra)
    r = oracle_mod.read_restart(path, w.cfg["kl"], w.cfg["ml"], ij2newij=perm)
    assert r["NSEA"] == n and all(r[k] == v for k, v in DATES.items())
    f32 = lambda x: x.cpu().numpy().astype(np.float32)
    fl = F[:, :, :n].cpu().numpy().transpose(2, 1, 0).astype(np.float32)
    assert np.array_equal(r["FL3"], fl)
    for k, x in zip(("U10", "UDIR", "TAUW"), fields[:3]):
        assert np.array_equal(r[k], f32(x)), k
    for k in ("depth", "u", "v"):
        assert np.array_equal(r[k.upper()], f32(extra[k])), k
    m.close()


@pytest.mark.parametrize("renumber", [False, True])
def test_restart_read_into_device(tmp_path, oracle_mod, renumber):
    import torch
    w, m, F, fields, extra = _state(4)
    n, kl, ml = w.nsea, w.cfg["kl"], w.cfg["ml"]
    rng = np.random.default_rng(3)
    perm = rng.permutation(n).astype(np.int32) + 1 if renumber else None
    ref = {"FL3": np.asfortranarray(rng.random((n, kl, ml), dtype=np.float32)),
           **{k: rng.random(n, dtype=np.float32) for k in ("U10", "UDIR", "TAUW", "DEPTH", "U", "V")}}
    path = tmp_path / "restart_ref.bin"
    oracle_mod.write_restart(path, n, DATES, ref["U10"], ref["UDIR"], ref["TAUW"], ref["FL3"], ref["DEPTH"], ref["U"],
                             ref["V"], ij2newij=perm)
    G = torch.zeros_like(F)
    outs = [torch.zeros(n, device="cuda") for _ in range(6)]
    dates = m.restart_read(path, G, outs[0], outs[1], outs[2], depth=outs[3], u=outs[4], v=outs[5], ij2newij=perm)
    assert dates == DATES
    assert np.array_equal(G[:, :, :n].cpu().numpy().transpose(2, 1, 0), ref["FL3"])
    assert torch.count_nonzero(G[:, :, n:]) == 0  # padding beyond NSEA untouched
    for k, t in zip(("U10", "UDIR", "TAUW", "DEPTH", "U", "V"), outs):
        assert np.array_equal(t.cpu().numpy(), ref[k]), k
    m.close()


def test_restart_rejects_other_grids(tmp_path, oracle_mod):
    """CONNECT_RESTART aborts when the file's NSEA is not the model's; here
    the call fails and the buffers stay untouched."""
    import torch
    from wam_b200 import WamgpuError
    w, m, F, fields, extra = _state(4)
    n, kl, ml = w.nsea, w.cfg["kl"], w.cfg["ml"]
    path = tmp_path / "other.bin"
    z = np.zeros(n - 1, np.float32)
    oracle_mod.write_restart(path, n - 1, {"CDTPRO": "20260101000000"}, z, z, z, np.zeros((n - 1, kl, ml), np.float32))
    G = torch.zeros_like(F)
    with pytest.raises(WamgpuError, match="NSEA"):
        m.restart_read(path, G, *[torch.zeros(n, device="cuda") for _ in range(3)])
    assert torch.count_nonzero(G) == 0
    with pytest.raises(WamgpuError):
        m.restart_write(tmp_path / "x.bin", F, *fields[:3], {"CDTPRO": "x", "CDTA": "20260101000000"})  # no depth
    m.close()
