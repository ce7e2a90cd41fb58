"""The arithmetic of the int8 split form, restated on the host (the kernels are checked on the GPU).

Every operand row is scaled by 2^e with max|v| 2^e in [63, 126) and rounded once to T (|T| < 2^31);
T's four balanced base-256 digits (the bytes of T + 0x80808080, each less 128) are the int8 slices;
a product keeps the ten slice pairs (j, m) with j + m <= 3 and combines them exactly.  The constant
operators are held as n dithered variants, floor(t 2^24 + ((v + h) mod n + 1/2) / n), whose mean over
the n variants is t 2^24 to within 1/(2n).
"""
import numpy as np


def row_exponent(mx):
    f, ex = np.frexp(mx)
    return 7 - ex - (f >= 126.0 / 128.0)


def digits(T):
    """Bytes of T + 0x80808080 (xor 0x80808080), most significant first; signed_bytes makes them the
    balanced digits."""
    u = (np.asarray(T, dtype=np.int64) + 0x80808080) & 0xFFFFFFFF
    u ^= 0x80808080
    return [((u >> (24 - 8 * q)) & 0xFF).astype(np.int64) for q in range(4)]


def signed_bytes(d):
    return np.where(d >= 128, d - 256, d)


def test_row_scale_puts_the_maximum_in_63_126():
    rng = np.random.default_rng(0)
    mx = np.exp(rng.uniform(-40, 40, 20000))
    s = mx * np.ldexp(1.0, row_exponent(mx))
    assert s.min() >= 63.0 and s.max() < 126.0


def test_balanced_digits_rebuild_T_exactly():
    rng = np.random.default_rng(1)
    T = np.concatenate([rng.integers(-(126 << 24), (126 << 24) + 1, 100000),
                        [0, 1, -1, 127, -128, 126 << 24, -(126 << 24), 0x7DFFFF80, -0x7DFFFF80]])
    a = [signed_bytes(d) for d in digits(T)]
    assert all((x >= -128).all() and (x <= 127).all() for x in a)
    rebuilt = a[0] * (1 << 24) + a[1] * (1 << 16) + a[2] * (1 << 8) + a[3]
    np.testing.assert_array_equal(rebuilt, T)


def test_dithered_variants_average_to_the_exact_value():
    rng = np.random.default_rng(2)
    t = rng.uniform(-126, 126, 5000)
    h = rng.integers(0, 1 << 24, t.size)
    for n in (8, 16):
        T = np.stack([np.floor(t * 2.0 ** 24 + (((v + h) & (n - 1)) + 0.5) / n) for v in range(n)])
        err = np.abs(T.mean(axis=0) - t * 2.0 ** 24)
        assert err.max() <= 0.5 / n + 1e-6
        # one variant alone is off by less than one unit (floor of a shifted value)
        assert np.abs(T - t * 2.0 ** 24).max() < 1.0


def test_ten_slice_pairs_give_the_product_to_the_stated_resolution():
    rng = np.random.default_rng(3)
    K = 161
    for _ in range(20):
        s = rng.standard_normal(K)
        x = rng.standard_normal(K)
        es, ex = row_exponent(np.abs(s).max()), row_exponent(np.abs(x).max())
        Ts = np.rint(s * 2.0 ** es * 2 ** 24).astype(np.int64)
        Tx = np.rint(x * 2.0 ** ex * 2 ** 24).astype(np.int64)
        a = [signed_bytes(d) for d in digits(Ts)]
        b = [signed_bytes(d) for d in digits(Tx)]
        D = [sum(int(np.dot(a[j], b[w - j])) for j in range(w + 1)) for w in range(4)]
        assert all(abs(v) < 2 ** 31 for v in D)            # int32 accumulators
        total = (D[0] << 24) + (D[1] << 16) + (D[2] << 8) + D[3]
        y = float(total) * 2.0 ** (-es - ex - 24)
        exact = float(np.dot(s, x))
        # rounding of both rows (2^-25 of each row scale per entry) and the dropped pairs (j + m >= 4)
        scale = np.abs(s).max() * np.abs(x).max() * K
        assert abs(y - exact) <= 2.0 ** -29 * scale
