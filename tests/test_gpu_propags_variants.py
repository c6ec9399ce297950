"""PROPAGS and CHECK_CFL over every coefficient family of the reference
(PREP_CART_DEEP/SHALLOW(_CUR), PREP_SPHER_DEEP/SHALLOW(_CURR)(_REG),
wam_propagation_module.f90:928-1911), on regular and reduced grids, against
the oracle: total CFL and COUNTER equal, propagated spectra bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = []
for spherical in (0, 1):
    for shallow in (0, 1):
        for current in (0, 1):
            for reduced in ((0, 1) if spherical else (0,)):
                for refr_d in ((0, 1) if shallow and not current else (1,) if current and shallow else (0,)):
                    CASES.append((spherical, shallow, current, reduced, refr_d))


def _case(oracle_mod, spherical, shallow, current, reduced, refr_d, idelpro=600, seed=3):
    from wam_b200.model import make_config
    from wam_b200.synth import blob_mask, grf
    rng = np.random.default_rng(seed + 17 * spherical + 5 * shallow + 3 * current + 2 * reduced + refr_d)
    nx, ny = 48, 30
    mask = blob_mask(rng, nx, ny, 0.25, 2)
    xdello = 36000 * 2  # 0.2 deg
    g = oracle_mod.build_grid(nx, ny, 30 * 360000, -10 * 360000, -10 * 360000 + (nx - 1) * xdello, 36000 * 2, xdello,
                              mask, reduced=bool(reduced))
    n = g["nsea"]
    g["klat"] = g["klat"].astype(np.int32)
    cfg = make_config(24, 25, 0.04177, 1, 600, idelpro, g["delphi"], shallow_run=bool(shallow),
                      spherical_run=bool(spherical), refraction_d_run=bool(refr_d), refraction_c_run=bool(current),
                      reduced_grid=bool(reduced))
    order = mask.T.ravel()
    depth = (15.0 + 300.0 * (0.5 + 0.5 * np.tanh(grf(rng, nx, ny, 4)))).T.ravel()[order].astype(np.float32)
    u = (0.8 * grf(rng, nx, ny, 5)).T.ravel()[order].astype(np.float32) if current else None
    v = (0.8 * grf(rng, nx, ny, 5)).T.ravel()[order].astype(np.float32) if current else None
    f = (rng.random((n, 24, 25)) * np.exp(-np.arange(25) / 6.0)[None, None, :]).astype(np.float32)
    return cfg, g, depth, u, v, np.asfortranarray(f)


@pytest.mark.parametrize("spherical,shallow,current,reduced,refr_d", CASES)
def test_propags_variant_bit_exact(oracle_mod, spherical, shallow, current, reduced, refr_d):
    from wam_b200 import WamModel
    cfg, g, depth, u, v, f = _case(oracle_mod, spherical, shallow, current, reduced, refr_d)
    o = oracle_mod.Oracle(cfg)
    o.set_grid(g)
    o.set_fields(depth, u, v)
    rc, cfl, cnt = o.prepare_propagation()
    m = WamModel(cfg)
    m.set_grid(g)
    m.set_depth(depth)
    if current:
        m.set_current(u, v)
    if rc != 0:
        with pytest.raises(Exception):
            m.prepare_propagation()
        return
    gcfl, gcnt = m.prepare_propagation()
    assert gcnt == cnt and np.float32(gcfl) == np.float32(cfl)
    ref = o.propags(f.astype(float)).astype(np.float32)
    got = f.copy(order="F")
    m.propags(got)
    assert np.array_equal(got, ref), float(np.abs(got - ref).max())


def test_counter_substeps(oracle_mod):
    """A long propagation step (CFL > 1) is split into COUNTER sub-steps (CHECK_CFL :2082-2134)."""
    from wam_b200 import WamModel
    cfg, g, depth, u, v, f = _case(oracle_mod, 1, 1, 0, 0, 1, idelpro=7200)
    o = oracle_mod.Oracle(cfg)
    o.set_grid(g)
    o.set_fields(depth)
    rc, cfl, cnt = o.prepare_propagation()
    assert rc == 0 and cnt > 1
    m = WamModel(cfg)
    m.set_grid(g)
    m.set_depth(depth)
    gcfl, gcnt = m.prepare_propagation()
    assert gcnt == cnt and np.float32(gcfl) == np.float32(cfl)
    ref = o.propags(f.astype(float)).astype(np.float32)
    got = f.copy(order="F")
    m.propags(got)
    assert np.array_equal(got, ref)


def test_grids_with_different_directions_side_by_side(oracle_mod):
    """Two live contexts with KL=24 and KL=36, the second prepared last, each
    propagate with their own direction tables."""
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload
    models = []
    for w in (make_workload("c0", scale=0.2), make_workload("c1", scale=0.02)):
        m = WamModel(w.cfg)
        m.set_grid(w.grid)
        m.set_depth(w.depth)
        m.prepare_propagation()
        models.append((w, m))
    for w, m in models:
        o = oracle_mod.Oracle(w.cfg)
        o.set_grid(w.grid)
        o.set_fields(w.depth)
        o.prepare_propagation()
        f = w.spectrum_f()
        ref = o.propags(f.astype(float)).astype(np.float32)
        got = f.copy(order="F")
        m.propags(got)
        assert np.array_equal(got, ref), w.name
    for _, m in models:
        m.close()
