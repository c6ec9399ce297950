"""New wind fields on the device (wamgpu_set_wind_grid / wamgpu_wind_dev):
GET_WIND's input path WAM_WIND (wam_wind_module.f90:1063-1216) with the
interpolation tables of INTERPOLATION_TO_GRID (:1224-1377) against the
oracle's float32 restatement.  The interpolation and the speed round every
operation as the reference does and agree bit for bit; the direction
(ATAN2) and the Charnock drag of wind codes 1 and 2 (ALOG) use the device
library's functions: within 4 ulp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MDEG = 360000


def _model(name="c1", scale=0.05):
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale)
    m = WamModel(w.cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    m.prepare_propagation()
    return w, m


def _ulps(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))


@pytest.mark.parametrize("code_in", [3, 1, 2])
def test_wind_interpolated_to_sea_points(oracle_mod, code_in):
    import torch
    w, m = _model()
    g = w.grid
    # a coarser input grid that is not aligned with the model grid
    west_in, south_in = g["amowep"] - 1 * MDEG, g["amosop"] - 1 * MDEG
    dx_in, dy_in = int(3.3 * MDEG), int(2.7 * MDEG)
    east = g["amoeap"] + 1 * MDEG
    north = g["amosop"] + (g["ny"] - 1) * g["xdella"] + 1 * MDEG
    nx_in = (east - west_in) // dx_in + 2
    ny_in = (north - south_in) // dy_in + 2
    rng = np.random.default_rng(4)
    scale = {3: 12.0, 1: 0.5, 2: 0.4}[code_in]
    u_in = (scale * rng.standard_normal((ny_in, nx_in))).astype(np.float32)
    v_in = (scale * rng.standard_normal((ny_in, nx_in))).astype(np.float32)
    if code_in == 2:
        u_in, v_in = np.abs(u_in), np.abs(v_in)
    tab = oracle_mod.wind_tables(g, nx_in, ny_in, west_in, south_in, dx_in, dy_in)
    us_o, ds_o = oracle_mod.wam_wind(u_in, v_in, tab, code_in)
    m.set_wind_grid(g, nx_in, ny_in, west_in, south_in, dx_in, dy_in)
    dev = torch.device("cuda")
    U10, UDIR = torch.zeros(w.nsea, device=dev), torch.zeros(w.nsea, device=dev)
    m.wind_dev(torch.tensor(u_in, device=dev), torch.tensor(v_in, device=dev), U10, UDIR, code_in=code_in)
    m.sync()
    us_g, ds_g = U10.cpu().numpy(), UDIR.cpu().numpy()
    if code_in == 3:
        assert np.array_equal(us_g, us_o)
    else:
        assert _ulps(us_g, us_o).max() <= 4
    assert _ulps(ds_g, ds_o).max() <= 4
    assert us_g.min() >= 2.0 and ds_g.min() >= 0 and ds_g.max() < 2 * np.pi + 1e-6
    m.close()


def test_wind_on_the_model_grid_and_outside(oracle_mod):
    """EQUAL_GRID copies the input at (IFROMIJ, KFROMIJ); an input grid that
    does not cover a sea point is refused, where the reference aborts."""
    import torch
    from wam_b200 import WamgpuError
    w, m = _model()
    g = w.grid
    rng = np.random.default_rng(9)
    u_in = (10 * rng.standard_normal((g["ny"], g["nx"]))).astype(np.float32)
    v_in = (10 * rng.standard_normal((g["ny"], g["nx"]))).astype(np.float32)
    tab = oracle_mod.wind_tables(g, g["nx"], g["ny"], g["amowep"], g["amosop"], g["xdello"], g["xdella"], equal_grid=True)
    us_o, ds_o = oracle_mod.wam_wind(u_in, v_in, tab, 3, equal_grid=True)
    m.set_wind_grid(g, g["nx"], g["ny"], g["amowep"], g["amosop"], g["xdello"], g["xdella"], equal_grid=True)
    dev = torch.device("cuda")
    U10, UDIR = torch.zeros(w.nsea, device=dev), torch.zeros(w.nsea, device=dev)
    m.wind_dev(torch.tensor(u_in, device=dev), torch.tensor(v_in, device=dev), U10, UDIR)
    m.sync()
    assert np.array_equal(U10.cpu().numpy(), us_o)
    assert _ulps(UDIR.cpu().numpy(), ds_o).max() <= 4
    with pytest.raises(WamgpuError):
        m.set_wind_grid(g, 4, 4, g["amowep"], g["amosop"], g["xdello"], g["xdella"])
    m.close()
