"""The oracle against the reference's own pinned output (run protocol).

dayfiles/wam_prot_coarse_ST6 is the only output the reference ships for this
path: the DIA index/weight tables, the frequency grid and the table
parameters of its coarse ST6 run.  Integer tables must match exactly.  Float
tables are printed with 8 (DIA weights), 7 (FRH) or 5 (grid) decimals by an
Intel build whose default floating-point model divides through reciprocals,
so they are compared to a few units in the last place of float32.
"""
import numpy as np

from conftest import coarse_st6_config


def test_dia_integer_tables_exact(oracle_mod, golden):
    o = oracle_mod.Oracle(coarse_st6_config())
    rows = golden["dia_freq"]
    assert [r["M"] for r in rows] == list(range(-3, 30))
    for name in ("IKP", "IKP1", "IKM", "IKM1"):
        assert (o.itable(name) == np.array([r[name] for r in rows])).all(), name
    for name in ("K1W", "K2W", "K11W", "K21W"):
        got = o.itable(name).reshape(2, 12).T
        want = np.array([r[name] for r in golden["dia_ang"]])
        assert (got == want).all(), name
    mfrstlw, mlsthg, kfrh = o.itable("DIA_SCALARS")[:3]
    assert (mfrstlw, mlsthg, kfrh) == (-3, 29, 8)


def test_dia_weights(oracle_mod, golden):
    o = oracle_mod.Oracle(coarse_st6_config())
    s = o.table("SCALARS")
    for i, name in enumerate(("ACL1", "ACL2", "CL11", "CL21", "DAL1", "DAL2")):
        assert abs(s[9 + i] - golden[name]) <= 1e-8 + 1e-8 * abs(golden[name]), name
    rows = golden["dia_freq"]
    for name in ("FKLAP", "FKLAP1", "FKLAM", "FKLAM1"):
        got, want = o.table(name), np.array([r[name] for r in rows])
        assert np.abs(got - want).max() <= 8e-8, name   # ~1 ulp of float32 at 0.3-1.0 plus print rounding
    af = o.table("AF11")
    want = np.array([r["AF11"] for r in rows])
    half_unit = 0.5e-3 * 10.0 ** np.floor(np.log10(want) + 1)  # E11.3 prints 3 significant digits
    assert (np.abs(af - want) <= half_unit * 1.001).all()
    assert np.abs(o.table("FRH") - np.array(golden["FRH"])).max() <= 3e-7


def test_frequency_direction_grid(oracle_mod, golden):
    o = oracle_mod.Oracle(coarse_st6_config())
    for name, key in (("FR", "FR_5dp"), ("DFIM", "DFIM_5dp"), ("GOM", "GOM_5dp"), ("C", "C_5dp")):
        got, want = o.table(name), np.array(golden[key])
        assert np.abs(np.round(got, 5) - want).max() <= 1.01e-5, name
    th = o.table("TH").astype(np.float32) * np.float32(180.0 / np.float32(3.1415927))
    assert np.abs(th - np.array(golden["TH_deg"])).max() < 1e-4


def test_table_parameters(oracle_mod, golden):
    o = oracle_mod.Oracle(coarse_st6_config())
    s = o.table("SCALARS")
    assert s[8] == golden["DELU"]
    assert golden["NDEPTH"] == 69 and golden["JUMAX"] == 300
    tf = o.table("TFAK")
    assert tf.size == 69 * 25
    depthe = 1.0 * np.float32(1.1) ** 68
    assert abs(depthe - golden["DEPTHE"]) / golden["DEPTHE"] < 1e-5


def test_effective_parameters_match_protocol(golden):
    from wam_b200.model import effective_parameters
    p = effective_parameters(2, 25, betamax=golden["BETAMAX"], cdfac=golden["CDFAC"])
    assert abs(p["alpha"] - golden["ALPHA"]) < 1e-7
    assert abs(p["zalp"] - golden["ZALP"]) < 1e-7
