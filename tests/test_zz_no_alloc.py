"""wamgpu_propags_dev_static (F1 ping-pong spectrum in a fixed per-device
array, no allocation) against wamgpu_propags_dev with a caller-owned scratch
on identical spectra: bit-identical over two consecutive calls, for COUNTER
odd and even, FP32 and FP64, with a ragged leading dimension; spectra larger
than the fixed array are rejected before any work is queued, and so is a
context with an owned range (its sub-steps would read halo points of the
shared array that the call never wrote).

Collected last on purpose: it must pass in a fresh process (its first call
does the per-device address lookup) and after every other GPU test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WAMGPU_E_ARG = -1
STATIC_BYTES = 33554432  # WAMGPU_STATIC_SCRATCH_BYTES


def _model(oracle_mod, idelpro, precision=4):
    """Spherical shallow grid, 40x28 at 0.2 deg with depth refraction: COUNTER
    is 1, 2 and 3 at IDELPRO 300, 600 and 900 s."""
    from wam_b200 import WamModel
    from wam_b200.model import make_config
    from wam_b200.synth import blob_mask, grf
    rng = np.random.default_rng(11)
    nx, ny = 40, 28
    mask = blob_mask(rng, nx, ny, 0.25, 2)
    xd = 36000 * 2
    g = oracle_mod.build_grid(nx, ny, 30 * 360000, -10 * 360000, -10 * 360000 + (nx - 1) * xd, xd, xd, mask,
                              reduced=False)
    g["klat"] = g["klat"].astype(np.int32)
    order = mask.T.ravel()
    depth = (15.0 + 300.0 * (0.5 + 0.5 * np.tanh(grf(rng, nx, ny, 4)))).T.ravel()[order].astype(np.float32)
    cfg = make_config(24, 25, 0.04177, 1, 600, idelpro, g["delphi"], shallow_run=True, spherical_run=True,
                      refraction_d_run=True, refraction_c_run=False, reduced_grid=False, precision=precision)
    m = WamModel(cfg)
    m.set_grid(g)
    m.set_depth(depth)
    m.prepare_propagation()
    f = (rng.random((25, 24, g["nsea"])) * np.exp(-np.arange(25) / 6.0)[:, None, None])
    return m, f.astype(np.float64 if precision == 8 else np.float32)


def _static(m, t, ld):
    return m.L.wamgpu_propags_dev_static(m.h, ctypes.c_void_p(t.data_ptr()), ld, None)


def _dtype(torch, precision):
    return torch.float64 if precision == 8 else torch.float32


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("idelpro,counter", [(300, 1), (600, 2), (900, 3)])
def test_static_scratch_matches_propags_dev(oracle_mod, idelpro, counter, precision):
    import torch
    m, f = _model(oracle_mod, idelpro, precision)
    assert m.counter == counter
    n, ld = m.nsea, m.nsea + 5
    a = torch.zeros((25, 24, ld), dtype=_dtype(torch, precision), device="cuda:0")
    a[..., :n] = torch.from_numpy(f).cuda()
    b = a.clone()
    scratch = torch.zeros_like(a)
    torch.cuda.synchronize()
    for call in range(2):
        rc = _static(m, b, ld)
        assert rc == 0, m.L.wamgpu_last_error(m.h).decode()
        m.propags_dev(a, ld=ld, scratch=scratch)
        m.sync()
        assert torch.equal(a[..., :n], b[..., :n]), f"call {call}: max diff {(a - b).abs().max().item()}"
        assert not torch.equal(b[..., :n], torch.from_numpy(f).cuda()), "spectrum did not propagate"
    m.close()


@pytest.mark.parametrize("precision", [4, 8])
def test_static_scratch_rejects_oversize(oracle_mod, precision):
    import torch
    m, f = _model(oracle_mod, 300, precision)
    esize = 8 if precision == 8 else 4
    ld = STATIC_BYTES // (24 * 25 * esize) + 1
    # a buffer that really is ld wide, so even a wrongly accepted call would stay in bounds
    t = torch.zeros((25, 24, ld), dtype=_dtype(torch, precision), device="cuda:0")
    t[..., :m.nsea] = torch.from_numpy(f).cuda()
    before = t.clone()
    torch.cuda.synchronize()
    rc = _static(m, t, ld)
    assert rc == WAMGPU_E_ARG
    assert "static PROPAGS scratch" in m.L.wamgpu_last_error(m.h).decode()
    m.sync()
    assert torch.equal(t, before)
    # the largest accepted leading dimension still runs
    ld_ok = STATIC_BYTES // (24 * 25 * esize)
    assert _static(m, t, ld_ok) == 0, m.L.wamgpu_last_error(m.h).decode()
    m.sync()
    m.close()


def test_static_scratch_rejects_owned_range(oracle_mod):
    """An owned range with COUNTER = 2: the second sub-step would read halo
    points of the fixed array that the first did not write, so the call is
    refused before anything is queued."""
    import torch
    m, f = _model(oracle_mod, 600)
    m.set_owned(0, m.nsea // 2)
    m.prepare_propagation()
    assert m.counter == 2
    t = torch.from_numpy(f).cuda().contiguous()
    before = t.clone()
    torch.cuda.synchronize()
    rc = _static(m, t, m.nsea)
    assert rc == WAMGPU_E_ARG
    assert "owned range" in m.L.wamgpu_last_error(m.h).decode()
    m.sync()
    assert torch.equal(t, before)
    m.close()
