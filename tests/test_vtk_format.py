"""The VTK value formatter (host build of the device code) against printf "%g".

The reference prints each value with `ofstream << float`, i.e. printf "%g" of
the float widened to double (src/moment_vtk_writer.cu:22,46).  Python's
'%g' % x is a correctly rounded conversion of the same double, so the two must
agree byte for byte; NaN is printed with its sign by the C library ("-nan"),
which Python drops.  The device kernels run the same integer-only code
(lbm_vtk.cu); tests/test_gpu_vtk.py checks the device text against this.
"""
import numpy as np
import pytest

from myfluidsimulation_b200.vtk import format_host


def printf_g(x: np.float32) -> str:
    if np.isnan(x):
        return "-nan" if np.signbit(x) else "nan"
    return "%g" % float(x)


def check(values):
    v = np.asarray(values, np.float32)
    got = format_host(v)
    bad = [(float(x), g, printf_g(x)) for x, g in zip(v, got) if g != printf_g(x)]
    assert not bad, bad[:10]


def test_special_values():
    f = np.float32
    tiny = np.finfo(np.float32).tiny
    check([0.0, -0.0, 1.0, -1.0, 0.5, 1.5, 2.5, 10.0, 100000.0, 999999.0, 1e6, 999999.5, 9999995.0,
           1234565.0, 1234575.0, 0.0001, 0.00009999999, 1e-5, 123456.5, 0.1, 0.2, 0.3, 1.0 / 3.0,
           np.inf, -np.inf, np.nan, -np.nan, np.finfo(np.float32).max, -np.finfo(np.float32).max,
           tiny, np.nextafter(f(0), f(1)), -np.nextafter(f(0), f(1)), np.nextafter(tiny, f(0)),
           1.0000005, 0.99999994, 1e38, 3e-45])


def test_powers_of_ten_and_neighbours():
    vals = []
    for k in range(-45, 39):
        x = np.float32(10.0 ** k)
        for _ in range(4):
            vals += [x, -x]
            x = np.nextafter(x, np.float32(np.inf))
        x = np.float32(10.0 ** k)
        for _ in range(4):
            x = np.nextafter(x, np.float32(0))
            vals += [x]
        # rounding boundaries of 6 digits: d.ddddd5 x 10^k and its neighbours
        if 9.999995 * 10.0 ** k < float(np.finfo(np.float32).max):
            y = np.float32(9.999995 * 10.0 ** k)
            vals += [y, np.nextafter(y, np.float32(0)), np.nextafter(y, np.float32(np.inf))]
    check(vals)


def test_integers_with_ties():
    # integers of 7 digits are exact floats: every tie of the 6th digit is present
    check(np.arange(1_000_000, 1_200_000, 1, dtype=np.float64).astype(np.float32))
    check(np.arange(16_777_000, 16_777_217, 1, dtype=np.float64).astype(np.float32))


@pytest.mark.parametrize("seed", [0, 1])
def test_random_bit_patterns(seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2 ** 32, size=300_000, dtype=np.uint64).astype(np.uint32)
    check(bits.view(np.float32))


def test_lbm_value_ranges():
    rng = np.random.default_rng(7)
    rho = (1.0 + 1e-3 * rng.standard_normal(200_000)).astype(np.float32)
    u = (0.05 * rng.standard_normal(200_000)).astype(np.float32)
    small = (1e-6 * rng.standard_normal(100_000)).astype(np.float32)
    check(rho)
    check(u)
    check(small)
