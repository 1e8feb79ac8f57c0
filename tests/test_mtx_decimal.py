"""The decimal conversion of the device Matrix Market parser
(abhsf_read_mtx_device), run on the host through a test hook: every number
it converts is bitwise what strtod gives (Python's float() rounds the same
way, correctly), and it leaves to the host's parser what it cannot decide --
exact ties, near-ties the 128-bit product cannot split, more than 19
significant digits, subnormal and out-of-range results, other spellings.
The GPU runs the same function (tests/test_gpu_mtx_device.py)."""
import ctypes as C
import math
import random
import struct
from decimal import Decimal, getcontext

import pytest

from abhsf_b200 import capi


def parse(s: str):
    b = s.encode()
    v, u = C.c_double(), C.c_int64()
    rc = capi.lib.abhsf_test_parse_decimal(b, len(b), C.byref(v), C.byref(u))
    return rc, v.value, u.value


def bits(x: float) -> bytes:
    return struct.pack("<d", x)


def check_all(strings):
    converted = 0
    for s in strings:
        rc, v, _ = parse(s)
        if rc == 0:
            converted += 1
            assert bits(v) == bits(float(s)), s
    return converted


def test_typical_spellings_convert_exactly():
    rng = random.Random(11)
    ss = []
    for _ in range(20000):
        x = rng.gauss(0, 1) * 10.0 ** rng.randint(-40, 40)
        ss += [repr(x), "%.17g" % x, "%.16e" % x, "%.15g" % x, "%.7e" % x]
    assert check_all(ss) == len(ss)  # none of these needs the host


def test_random_significands_and_exponents():
    rng = random.Random(12)
    ss = []
    for _ in range(30000):
        d = rng.randint(1, 19)
        m = str(rng.randint(10 ** (d - 1), 10 ** d - 1))
        e = rng.randint(-320, 305)
        ss.append(f"{'-' if rng.random() < 0.5 else ''}{m[0]}.{m[1:]}e{e}")
    assert check_all(ss) > 0.95 * len(ss)


def test_midpoints_are_never_misrounded():
    """Decimal spellings of the exact midpoint between two neighbouring
    doubles, and of its neighbours: ties to even, or left to the host."""
    getcontext().prec = 60
    rng = random.Random(13)
    ss = []
    for _ in range(3000):
        x = abs(rng.gauss(0, 1)) * 10.0 ** rng.randint(-20, 20)
        mid = (Decimal(x) + Decimal(math.nextafter(x, math.inf))) / 2
        for t in (mid, mid.next_plus(), mid.next_minus()):
            ss += ["%.18e" % float(t), format(t.normalize(), "e")]
    ss += [str(2 ** 53 + 2 * k - 1) for k in range(1, 500)]  # integer ties, decided exactly (5^0 is exact)
    check_all(ss)
    assert parse(str(2 ** 53 + 1)) == (0, float(2 ** 53), 16)  # ties to even
    assert parse("0.5000000000000000277555756156289135105907917022705078125")[0] == 1  # too many digits


@pytest.mark.parametrize("text,value,used", [
    ("1.5abc", 1.5, 3), ("1e", 1.0, 1), ("1e+", 1.0, 1), ("-.5", -0.5, 3), (".5e1", 5.0, 4), ("1.", 1.0, 2),
    ("007", 7.0, 3), ("-0.0", -0.0, 4), ("0e999", 0.0, 5),
])
def test_syntax_as_from_chars_reads_it(text, value, used):
    rc, v, u = parse(text)
    assert rc == 0 and bits(v) == bits(value) and u == used


@pytest.mark.parametrize("text", ["+1", "inf", "nan", "-inf", "0x1p3", "1e400", "1e-400", "4.9e-324", ".", "-", "e5",
                                  "12345678901234567890", "1.0000000000000000000001", "1E-2x"])
def test_left_to_the_host(text):
    assert parse(text)[0] == 1
