"""The single-precision quotients of SINPUT_ST6 (and its adjoint) are formed
as the float rounding of a times the double reciprocal of b (RecipDiv in
wam_b200/csrc/devmath.cuh), which must equal the IEEE single-precision
division a / b bit for bit.  IEEE arithmetic is the same on the host, so
numpy checks the identity here: random significands over the whole exponent
range, divisors near powers of two and with all-ones significands, dividends
close to multiples of the divisor, zeros and results in the subnormal range."""
import numpy as np


def _recip_div(a, b):
    y = 1.0 / b.astype(np.float64)
    return (a.astype(np.float64) * y).astype(np.float32)


def _floats(rng, n, emin, emax, sig=None):
    s = rng.integers(0, 1 << 23, n, dtype=np.uint32) if sig is None else sig
    e = rng.integers(emin + 127, emax + 128, n, dtype=np.uint32)
    return ((e << 23) | s).view(np.float32)


def test_recip_div_equals_ieee_division():
    rng = np.random.default_rng(20261204)
    n = 4_000_000
    cases = [
        (_floats(rng, n, -126, 127), _floats(rng, n, -126, 127)),
        (_floats(rng, n, -40, 40), _floats(rng, n, -20, 20, sig=(rng.integers(0, 1 << 23, n) | 0x7FFF00).astype(np.uint32))),
        (_floats(rng, n, -40, 40), _floats(rng, n, -20, 20, sig=(rng.integers(0, 1 << 23, n) & 0x7F0000).astype(np.uint32))),
        (_floats(rng, n, -126, -100), _floats(rng, n, 0, 30)),           # subnormal and tiny quotients
    ]
    # dividends within a few ulps of k * b
    b = _floats(rng, n, -10, 10)
    k = rng.integers(1, 1 << 12, n).astype(np.float32)
    a = (k * b).astype(np.float32)
    a = a.view(np.uint32) + rng.integers(-2, 3, n).astype(np.uint32)
    cases.append((a.view(np.float32), b))
    cases.append((np.zeros(1000, np.float32), _floats(rng, 1000, -30, 30)))
    with np.errstate(all="ignore"):
        for a, b in cases:
            ok = np.isfinite(a) & np.isfinite(b) & (b != 0)
            a, b = a[ok], b[ok]
            ref = a / b
            got = _recip_div(a, b)
            bad = ref.view(np.uint32) != got.view(np.uint32)
            assert not bad.any(), (a[bad][:5], b[bad][:5], ref[bad][:5], got[bad][:5])
