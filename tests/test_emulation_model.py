"""CPU model of the emulated-FP64 scheme the int8 contraction kernel implements (a restatement of its
arithmetic in numpy, not the kernel): every A row and B column gets a power-of-two scale 2^e with its
largest element in [1/4, 1/2) and S signed base-128 digits, each rounded to nearest, |d| <= 64; the
digit pairs with p + q <= S - 1 are kept, pairs of equal p + q share one int32 level accumulator, and
up to four adjacent levels are combined exactly in int64 before one conversion to FP64.

The tests pin the numerical claims the kernel relies on: the digit bound, the operand's exactness to
2^(e - 7S - 1), the level sums' int32 range at the largest supported contraction, the exactness of
the int64 group combine, and the error falling by about 2^-7 per slice."""
import numpy as np
import pytest

BASE = 128
LGROUP = 4


def scales(x, axis):
    """Power-of-two exponent e per row (axis=1) or column (axis=0) with max|x| / 2^e in [1/4, 1/2)."""
    m = np.max(np.abs(x), axis=axis, keepdims=True)
    e = np.floor(np.log2(np.where(m > 0, m, 1.0))) + 2  # m / 2^e in [1/4, 1/2)
    return e


def digits(x, s, axis):
    """S signed base-128 digits of x / 2^e (rounded to nearest at each step) and the exponents."""
    e = scales(x, axis)
    r = x / np.exp2(e)
    out = []
    for _ in range(s):
        d = np.rint(r * BASE)
        out.append(d.astype(np.int64))
        r = r * BASE - d
    return out, e


def emulated_product(a, b, s):
    """C = A B from the digit pairs p + q <= s - 1: int64 level sums, 4-level int64 groups, FP64."""
    da, ea = digits(a, s, axis=1)  # per row of A
    db, eb = digits(b, s, axis=0)  # per column of B
    levels = [sum(da[p] @ db[lv - p] for p in range(lv + 1)) for lv in range(s)]
    acc = np.zeros(levels[0].shape)
    for g0 in range(0, s, LGROUP):
        g1 = min(g0 + LGROUP, s)
        x = np.zeros(levels[0].shape, dtype=np.int64)
        for lv in range(g0, g1):
            x = x * BASE + levels[lv]
        assert np.max(np.abs(x)) < 2 ** 53  # one exact conversion to FP64
        acc += x.astype(np.float64) * np.exp2(-7.0 * (g1 - 1 + 2))  # weight of the group's last level
    return acc * np.exp2(ea) * np.exp2(eb), levels


@pytest.mark.parametrize("s", [4, 6, 8])
def test_digits_are_bounded_and_exact_to_the_last_place(s):
    rng = np.random.default_rng(s)
    x = rng.uniform(-1, 1, (17, 33)) * np.exp2(rng.integers(-20, 20, (17, 1)))
    d, e = digits(x, s, axis=1)
    assert max(np.max(np.abs(v)) for v in d) <= 64
    back = sum(v.astype(np.float64) * np.exp2(-7.0 * (p + 1)) for p, v in enumerate(d)) * np.exp2(e)
    # exact to 2^(e - 7S - 1) per element
    assert np.all(np.abs(back - x) <= np.exp2(e - 7 * s - 1) * (1 + 1e-12))


# the largest contraction the library accepts: nvir <= 16384, nocc <= 1023, dp = V + O rounded up to 32
DP_MAX = (16384 + 1023 + 31) // 32 * 32


def test_level_sums_fit_int32_at_the_largest_contraction():
    # |level L| <= (L + 1) * dp * 64^2; the kernel's largest level has S terms
    for s in range(4, 9):
        assert s * DP_MAX * 64 * 64 < 2 ** 31
    rng = np.random.default_rng(7)
    a = rng.uniform(-1, 1, (8, 512))
    b = rng.uniform(-1, 1, (512, 8))
    _, levels = emulated_product(a, b, 8)
    for lv, v in enumerate(levels):
        assert np.max(np.abs(v)) <= (lv + 1) * 512 * 64 * 64


def test_int64_group_of_four_levels_stays_below_2_53():
    # |C_l| <= 8 * dp * 64^2 < 2^30 at the largest contraction, so X = sum_l C_l 128^(3 - l) < 2^51.1
    c_max = 8 * DP_MAX * 64 * 64
    assert c_max < 2 ** 30
    bound = sum(c_max * BASE ** (LGROUP - 1 - l) for l in range(LGROUP))
    assert bound < 2 ** 53


def test_error_falls_by_about_2_to_the_7_per_slice():
    rng = np.random.default_rng(11)
    a = rng.uniform(-0.1, 0.1, (24, 340))
    b = rng.uniform(-0.05, 0.05, (340, 24))
    exact = a.astype(np.longdouble) @ b.astype(np.longdouble)
    scale = float(np.max(np.abs(a)) * np.max(np.abs(b)) * a.shape[1])
    errs = {}
    for s in range(3, 8):
        c, _ = emulated_product(a, b, s)
        errs[s] = float(np.max(np.abs(c - exact.astype(np.float64)))) / scale
    for s in range(3, 7):
        assert errs[s + 1] < errs[s] / 32, errs  # about 2^-7 per slice; 2^-5 leaves room
    assert errs[7] < 1e-13, errs
