"""CPU checks of the product library: the C ABI loads and exports every
symbol include/wamgpu.h declares, its host table builders agree bit-for-bit
with the oracle's, its grid builder agrees with the oracle's restatement of the
pre-processor, and without a GPU every compute entry point fails loudly."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, coarse_st6_config

FLOAT_TABLES = ["FR", "DF", "DFIM", "GOM", "TH", "COSTH", "SINTH", "DFIMOFR", "FR5", "FRM5", "RHOWG_DFIM", "TFAK",
                "TCGOND", "TSIHKD", "FLMINFR", "AF11", "FKLAP", "FKLAP1", "FKLAM", "FKLAM1", "FRH", "RNLCOEF",
                "SWELLFT", "SATWEIGHTS", "WTAUHF"]
INT_TABLES = ["IKP", "IKP1", "IKM", "IKM1", "K1W", "K2W", "K11W", "K21W", "INLCOEF", "INDICESSAT"]


def _lib():
    from wam_b200 import _lib
    return _lib


def test_library_exports_header_symbols():
    L = _lib()
    lib = L.load()
    header = open(os.path.join(ROOT, "include", "wamgpu.h")).read()
    declared = set(re.findall(r"WAMGPU_API\s+(?:int|const char\*)\s+(wamgpu_\w+)\(", header))
    assert len(declared) >= 17
    for name in declared:
        assert hasattr(lib, name), name
    assert set(L.SIGNATURES) == declared
    assert lib.wamgpu_config_size() == ctypes.sizeof(L.WamgpuConfig)


def _host_table(cfg, name, integer):
    L = _lib()
    lib = L.load()
    fields = {f for f, _ in L.WamgpuConfig._fields_}
    c = L.WamgpuConfig(**{k: v for k, v in cfg.items() if k in fields})
    n = lib.wamgpu_host_table(ctypes.byref(c), name.encode(), None, None)
    assert n >= 0, name
    if integer:
        a = np.zeros(max(n, 1), np.int32)
        lib.wamgpu_host_table(ctypes.byref(c), name.encode(), None, a.ctypes.data_as(L.PI))
    else:
        a = np.zeros(max(n, 1), np.float32)
        lib.wamgpu_host_table(ctypes.byref(c), name.encode(), a.ctypes.data_as(L.PF), None)
    return a[:n]


def _configs():
    from wam_b200.synth import make_workload
    out = [("coarse_st6", coarse_st6_config())]
    for name in ("c0", "c1", "c2", "c4"):
        out.append((name, make_workload(name, scale=0.05).cfg))
    return out


@pytest.mark.parametrize("label,cfg", _configs(), ids=lambda x: x if isinstance(x, str) else "")
def test_host_tables_bit_exact_vs_oracle(oracle_mod, label, cfg):
    o = oracle_mod.Oracle(cfg)
    for t in FLOAT_TABLES:
        got = _host_table(cfg, t, False)
        ref = o.table(t).astype(np.float32)
        assert got.shape == ref.shape, t
        assert np.array_equal(got, ref), (label, t, float(np.abs(got - ref).max()) if got.size else 0)
    for t in INT_TABLES:
        got = _host_table(cfg, t, True)
        assert np.array_equal(got, o.itable(t)), (label, t)


@pytest.mark.parametrize("periodic", [False, True])
def test_grid_builder_matches_oracle(oracle_mod, periodic):
    from wam_b200.grid import regular_grid
    from wam_b200.synth import blob_mask
    rng = np.random.default_rng(7)
    nx, ny = (36, 17) if periodic else (30, 20)
    mask = blob_mask(rng, nx, ny, 0.3, 2)
    dlon = 10.0 if periodic else 1.0
    g = regular_grid(mask, -40.0, 0.0 if periodic else -15.0, 5.0, dlon)
    r = oracle_mod.build_grid(nx, ny, g["amosop"], g["amowep"], g["amoeap"], g["xdella"], g["xdello"], mask)
    assert g["iper"] == r["iper"] == int(periodic)
    assert g["nsea"] == r["nsea"] == int(mask.sum())
    for k in ("klat", "klon", "kfromij", "ixlg", "kxlt"):
        assert np.array_equal(np.asarray(g[k]), r[k]), k
    assert np.array_equal(np.asarray(g["wlat"], np.float64), r["wlat"])
    assert abs(g["delphi"] - r["delphi"]) <= 1e-7 * r["delphi"]
    for k in ("sinph", "cosph", "dellam"):
        assert np.allclose(np.asarray(g[k], np.float64), r[k], rtol=3e-7, atol=3e-7), k


def test_effective_parameter_rules():
    from wam_b200.model import effective_parameters
    st4 = effective_parameters(1, 25, betamax=1.42)
    assert st4["alpha"] == 0.0075 and st4["tauwshelter"] == 0.25 and st4["betamax"] == 1.42
    assert effective_parameters(1, 35)["alpha"] == 0.0062
    assert effective_parameters(2, 35)["tauwshelter"] == 0.0


def test_no_gpu_fails_loudly():
    """Without a device wamgpu_create returns an error; there is no CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from wam_b200 import WamModel, WamgpuError
    with pytest.raises(WamgpuError):
        WamModel(coarse_st6_config())


def test_invalid_configurations_rejected():
    from wam_b200 import WamModel, WamgpuError
    bad = dict(coarse_st6_config(), iphys=0)
    with pytest.raises(WamgpuError):
        WamModel(bad)
    bad = dict(coarse_st6_config(), kl=200)
    with pytest.raises(WamgpuError):
        WamModel(bad)
