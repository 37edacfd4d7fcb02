"""The carry chains of zyklop_b200/csrc/field.cuh, restated instruction by
instruction with PTX carry-flag semantics and checked against Python
integers on edge and random operands (CPU only).

The CUDA code drops carries and borrows where its comments prove they
cannot occur (the last madc.hi of a row, the top word of a sum, the final
borrow of a subtraction whose result is known nonnegative).  Here each of
those places asserts that the dropped carry is zero, so a bound that does
not hold fails the test.  Covered: mul_4x4, sqr_4x4, fe_mul_wide
(Karatsuba over 128-bit halves), fe_sqr_wide, fe_redc, the Fp2 product
with two reductions (fp2_mul_call) and the shared-reduction difference of
products (fp_mul_sub_call).  The GPU parity tests check the compiled code
itself; this test pins the arithmetic bounds those sequences rely on."""
import random

import pytest

P = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
M32 = (1 << 32) - 1


class Cc:
    """The carry flag of a chain of .cc instructions."""

    def __init__(self):
        self.f = 0

    def mad_lo(self, a, b, c, cin=False, cout=True):
        v = ((a * b) & M32) + c + (self.f if cin else 0)
        return self._out(v, cout)

    def mad_hi(self, a, b, c, cin=False, cout=True):
        v = ((a * b) >> 32) + c + (self.f if cin else 0)
        return self._out(v, cout)

    def add(self, a, b, cin=False, cout=True):
        return self._out(a + b + (self.f if cin else 0), cout)

    def sub(self, a, b, cin=False, cout=True):
        v = a - b - (self.f if cin else 0)
        if cout:
            self.f = 1 if v < 0 else 0
        else:
            assert v >= 0, "borrow out of a chain that drops it"
        return v & M32

    def _out(self, v, cout):
        if cout:
            self.f = v >> 32
        else:
            assert v >> 32 == 0, "carry out of a chain that drops it"
        return v & M32


def limbs(x, n=8):
    return [(x >> (32 * i)) & M32 for i in range(n)]


def val(ws):
    return sum(w << (32 * i) for i, w in enumerate(ws))


def chain_add(a, b):
    c = Cc()
    return [c.add(x, y, cin=i > 0, cout=i < len(a) - 1) for i, (x, y) in enumerate(zip(a, b))]


def chain_sub(a, b):
    c = Cc()
    return [c.sub(x, y, cin=i > 0, cout=i < len(a) - 1) for i, (x, y) in enumerate(zip(a, b))]


def mul_4x4(x, y):
    x0, x1, x2, x3 = x
    r = [0] * 8
    c = Cc()
    r[0], r[1] = (x0 * y[0]) & M32, (x0 * y[0]) >> 32
    r[2], r[3] = (x2 * y[0]) & M32, (x2 * y[0]) >> 32
    r[1] = c.mad_lo(x1, y[0], r[1])
    r[2] = c.mad_hi(x1, y[0], r[2], cin=True)
    r[3] = c.mad_lo(x3, y[0], r[3], cin=True)
    r[4] = c.mad_hi(x3, y[0], 0, cin=True, cout=False)
    for j in (1, 2, 3):
        yj = y[j]
        r[j] = c.mad_lo(x0, yj, r[j])
        r[j + 1] = c.mad_hi(x0, yj, r[j + 1], cin=True)
        r[j + 2] = c.mad_lo(x2, yj, r[j + 2], cin=True)
        r[j + 3] = c.mad_hi(x2, yj, r[j + 3], cin=True)
        r[j + 4] = c.add(0, 0, cin=True, cout=False)
        r[j + 1] = c.mad_lo(x1, yj, r[j + 1])
        r[j + 2] = c.mad_hi(x1, yj, r[j + 2], cin=True)
        r[j + 3] = c.mad_lo(x3, yj, r[j + 3], cin=True)
        r[j + 4] = c.mad_hi(x3, yj, r[j + 4], cin=True, cout=False)
    return r


def sqr_4x4(x):
    x0, x1, x2, x3 = x
    r = [0] * 8
    c = Cc()
    r[1], r[2] = (x0 * x1) & M32, (x0 * x1) >> 32
    r[3], r[4] = (x1 * x2) & M32, (x1 * x2) >> 32
    r[5], r[6] = (x2 * x3) & M32, (x2 * x3) >> 32
    r[2] = c.mad_lo(x0, x2, r[2])
    r[3] = c.mad_hi(x0, x2, r[3], cin=True)
    r[4] = c.mad_lo(x1, x3, r[4], cin=True)
    r[5] = c.mad_hi(x1, x3, r[5], cin=True)
    r[6] = c.add(r[6], 0, cin=True, cout=False)
    r[3] = c.mad_lo(x0, x3, r[3])
    r[4] = c.mad_hi(x0, x3, r[4], cin=True)
    r[5] = c.add(r[5], 0, cin=True)
    r[6] = c.add(r[6], 0, cin=True)
    r[7] = c.add(0, 0, cin=True, cout=False)
    r[1] = c.add(r[1], r[1])
    for k in range(2, 7):
        r[k] = c.add(r[k], r[k], cin=True)
    r[7] = c.add(r[7], r[7], cin=True, cout=False)
    r[0] = (x0 * x0) & M32
    r[1] = c.mad_hi(x0, x0, r[1])
    r[2] = c.mad_lo(x1, x1, r[2], cin=True)
    r[3] = c.mad_hi(x1, x1, r[3], cin=True)
    r[4] = c.mad_lo(x2, x2, r[4], cin=True)
    r[5] = c.mad_hi(x2, x2, r[5], cin=True)
    r[6] = c.mad_lo(x3, x3, r[6], cin=True)
    r[7] = c.mad_hi(x3, x3, r[7], cin=True, cout=False)
    return r


def mul_wide(a, b):
    """fe_mul_wide: middle product first, then lo, then hi."""
    sa = chain_add(a[0:4] + [0], a[4:8] + [0])
    sb = chain_add(b[0:4] + [0], b[4:8] + [0])
    ca, cb = sa[4], sb[4]
    mid = mul_4x4(sa[:4], sb[:4])
    t = chain_add(mid[4:8] + [0], [v & ((0 - ca) & M32) for v in sb[:4]] + [0])
    mid[4:8], m8 = t[:4], t[4]
    t = chain_add(mid[4:8] + [m8], [v & ((0 - cb) & M32) for v in sa[:4]] + [ca & cb])
    mid[4:8], m8 = t[:4], t[4]
    w = mul_4x4(a[0:4], b[0:4])
    t = chain_sub(mid + [m8], w + [0])
    mid, m8 = t[:8], t[8]
    T = w[0:4] + chain_add(w[4:8] + mid[4:8] + [m8], mid[0:4] + [0] * 5) + [0] * 3
    w = mul_4x4(a[4:8], b[4:8])
    T[8:16] = chain_add(T[8:13] + w[5:8], w[0:5] + [0, 0, 0])
    T[4:16] = chain_sub(T[4:16], w + [0] * 4)
    return T


def sqr_wide(a):
    lo, hi, x = sqr_4x4(a[0:4]), sqr_4x4(a[4:8]), mul_4x4(a[0:4], a[4:8])
    t = chain_add(x + [0], x + [0])
    return lo[0:4] + chain_add(lo[4:8] + hi[0:4] + hi[4:8], t[:8] + [t[8], 0, 0, 0])


def redc(T, m):
    """fe_redc: eight rows fold T_lo, then T_hi is added; one conditional subtraction."""
    inv = (-pow(m, -1, 1 << 32)) % (1 << 32)
    p = limbs(m)
    t = T[0:8] + [0]
    for _ in range(8):
        q = (t[0] * inv) & M32
        c = Cc()
        t[0] = c.mad_lo(q, p[0], t[0])
        t[1] = c.mad_hi(q, p[0], t[1], cin=True)
        t[2] = c.mad_lo(q, p[2], t[2], cin=True)
        t[3] = c.mad_hi(q, p[2], t[3], cin=True)
        t[4] = c.mad_lo(q, p[4], t[4], cin=True)
        t[5] = c.mad_hi(q, p[4], t[5], cin=True)
        t[6] = c.mad_lo(q, p[6], t[6], cin=True)
        t[7] = c.mad_hi(q, p[6], t[7], cin=True)
        t[8] = c.add(t[8], 0, cin=True, cout=False)
        t[1] = c.mad_lo(q, p[1], t[1])
        t[2] = c.mad_hi(q, p[1], t[2], cin=True)
        t[3] = c.mad_lo(q, p[3], t[3], cin=True)
        t[4] = c.mad_hi(q, p[3], t[4], cin=True)
        t[5] = c.mad_lo(q, p[5], t[5], cin=True)
        t[6] = c.mad_hi(q, p[5], t[6], cin=True)
        t[7] = c.mad_lo(q, p[7], t[7], cin=True)
        t[8] = c.mad_hi(q, p[7], t[8], cin=True, cout=False)
        assert t[0] == 0
        t = t[1:9] + [0]
    r = val(chain_add(t[0:8], T[8:16]))
    assert r < 2 * m, "one conditional subtraction is not enough"
    return r - m if r >= m else r


def fp2_mul(a0, a1, b0, b1):
    s, t = chain_add(limbs(a0), limbs(a1)), chain_add(limbs(b0), limbs(b1))
    x, w = mul_wide(s, t), mul_wide(limbs(a0), limbs(b0))
    x = chain_sub(x, w)
    y = chain_add(w, limbs(P * P, 16))
    w = mul_wide(limbs(a1), limbs(b1))
    return redc(chain_sub(y, w), P), redc(chain_sub(x, w), P)


def fp_mul_sub(a, b, c, d):
    x = chain_add(mul_wide(limbs(a), limbs(b)), limbs(P * P, 16))
    return redc(chain_sub(x, mul_wide(limbs(c), limbs(d))), P)


def operands(m, k, seed):
    rng = random.Random(seed)
    edge = [0, 1, 2, m - 1, m - 2, (1 << 128) - 1, 1 << 128, (1 << 253) % m, m // 2]
    return edge + [rng.randrange(m) for _ in range(k)]


@pytest.mark.parametrize("m", [P, R], ids=["fp", "fr"])
def test_product_square_and_reduction(m):
    rinv = pow(1 << 256, -1, m)
    xs = operands(m, 300, 11)
    for i, a in enumerate(xs):
        b = xs[(7 * i + 3) % len(xs)]
        T = mul_wide(limbs(a), limbs(b))
        assert val(T) == a * b
        assert redc(T, m) == a * b * rinv % m
        S = sqr_wide(limbs(a))
        assert val(S) == a * a
        assert redc(S, m) == a * a * rinv % m


def test_wide_products_up_to_2_255():
    """Unreduced sums of two field elements (< 2p < 2^255) enter the products."""
    rng = random.Random(5)
    xs = [(1 << 255) - 1, (1 << 254) + 12345, 2 * P - 2] + [rng.getrandbits(255) for _ in range(100)]
    for a in xs:
        for b in xs[:6]:
            assert val(mul_wide(limbs(a), limbs(b))) == a * b
        assert val(sqr_wide(limbs(a))) == a * a
        assert val(sqr_4x4(limbs(a % (1 << 128), 4))) == (a % (1 << 128)) ** 2


def test_fp2_product_two_reductions():
    rinv = pow(1 << 256, -1, P)
    xs = operands(P, 200, 13)
    cases = [(xs[i], xs[i + 1], xs[i + 2], xs[(5 * i + 1) % len(xs)]) for i in range(len(xs) - 3)]
    cases += [(a, b, c, d) for a in (0, P - 1) for b in (0, P - 1) for c in (0, P - 1) for d in (0, P - 1)]
    for a0, a1, b0, b1 in cases:
        c0, c1 = fp2_mul(a0, a1, b0, b1)
        assert c0 == (a0 * b0 - a1 * b1) * rinv % P
        assert c1 == (a0 * b1 + a1 * b0) * rinv % P


def test_difference_of_products_one_reduction():
    rinv = pow(1 << 256, -1, P)
    xs = operands(P, 200, 17)
    for i in range(len(xs) - 3):
        a, b, c, d = xs[i], xs[i + 1], xs[i + 2], xs[(3 * i + 5) % len(xs)]
        assert fp_mul_sub(a, b, c, d) == (a * b - c * d) * rinv % P
    for a, c in ((0, P - 1), (P - 1, 0), (P - 1, P - 1)):
        assert fp_mul_sub(a, P - 1, c, P - 1) == (a * (P - 1) - c * (P - 1)) * rinv % P
