"""CPU model of the tensor-core contraction's fixed-point arithmetic (digits.cu,
contract_tc.cu): power-of-two row / column scales, four balanced signed base-256 digits,
the digit-pair classes W_c = sum_{i+j=c} A_i B_j (c <= 4) accumulated as S32, and the
FP64 combine 2^(er+ec-46) (W0 2^32 + W1 2^24 + W2 2^16 + W3 2^8 + W4).  No GPU is used here.

Keeping classes up to 4 matters: the dropped products of low digits are of the order of
2^-8c of the row scale times the column scale, whatever the entries' own sizes, so with
c <= 3 a column of many small entries beside one large one (a point set with a heavy node)
would lose ~1e-6 x max|alm|."""
import numpy as np
import pytest

MARGIN = 1.01


def scale_exp(v):
    """Smallest e with 1.01 v <= 2^e (frexp of 1.01 v), 0 for v = 0."""
    if not v > 0:
        return 0
    return int(np.frexp(v * MARGIN)[1])


def digits(x, e):
    """The four signed digit bytes d0..d3 of rint(x 2^(31 - e)) as the kernels form them:
    the bytes of (X + 0x808080) ^ 0x808080 read as int8."""
    X = np.rint(np.ldexp(x, 31 - e)).astype(np.int64)
    assert np.all(np.abs(X) < 2 ** 31 - 2 ** 24)
    Z = ((X + 0x808080) & 0xFFFFFFFF) ^ 0x808080
    b = [(Z >> (8 * (3 - d))) & 0xFF for d in range(4)]           # d0 = top byte
    return [np.where(v >= 128, v - 256, v).astype(np.int64) for v in b], X


def contract(T, F):
    """sum_k T[r, k] F[k, c] through the digit classes (rows of T, columns of F)."""
    R, K = T.shape
    C = F.shape[1]
    out = np.zeros((R, C))
    for r in range(R):
        er = scale_exp(np.abs(T[r]).max())
        a, XA = digits(T[r], er)
        assert np.array_equal(a[0] * 2 ** 24 + a[1] * 2 ** 16 + a[2] * 2 ** 8 + a[3], XA)
        for c in range(C):
            ec = scale_exp(np.abs(F[:, c]).max())
            b, XB = digits(F[:, c], ec)
            W = [sum(int(np.dot(a[i], b[cls - i])) for i in range(max(0, cls - 3), min(cls, 3) + 1))
                 for cls in range(5)]
            assert all(abs(w) < 2 ** 31 for w in W)
            V = (W[0] << 32) + (W[1] << 24) + (W[2] << 16) + (W[3] << 8) + W[4]
            assert abs(V) < 2 ** 63
            out[r, c] = np.ldexp(float(V), er + ec - 46)
    return out


def test_balanced_digits_are_signed_bytes_and_exact():
    rng = np.random.default_rng(0)
    x = rng.normal(size=1000) * np.exp(rng.uniform(-30, 5, 1000))
    e = scale_exp(np.abs(x).max())
    d, X = digits(x, e)
    for v in d:
        assert v.min() >= -128 and v.max() <= 127
    assert np.abs(d[0]).max() <= 127


@pytest.mark.parametrize("K", [64, 1024, 16384])
def test_digit_contraction_matches_fp64(K):
    """Rows spanning hundreds of decades (like high-m table rows) against spread and
    concentrated columns: error within the quantisation bound 2^-30 (max|T| sum|F| +
    max|F| sum|T|) (power-of-two scales are at most 2.02 x the largest entry)."""
    rng = np.random.default_rng(K)
    R, C = 6, 5
    x = np.linspace(0, 0.75, K // 2)
    T = np.empty((R, K))
    for r in range(R):
        p = 40 * r
        row = (1 - x ** 2) ** p * np.cos((r + 3) * 9 * x)
        T[r] = np.concatenate([row, 0.3 * row[::-1]])
    F = rng.normal(size=(K, C))
    F[:, 1] = 0.0
    F[K // 3, 1] = 7.0                 # all weight at one node
    F[:, 2] = np.abs(F[:, 2]) * 1e-3   # many small positive entries and one large
    F[5, 2] = 50.0
    F[:, 4] = 0.0                      # an empty column
    got = contract(T, F)
    ref = T @ F
    for c in range(C):
        bound = 2.0 ** -30 * (np.abs(T).max(axis=1) * np.abs(F[:, c]).sum()
                              + np.abs(F[:, c]).max() * np.abs(T).sum(axis=1)) + 1e-300
        assert np.all(np.abs(got[:, c] - ref[:, c]) <= bound), c
    assert not np.any(got[:, 4])


def test_class_sums_fit_int32_at_the_largest_k():
    """Worst case at K = 2 Nx = 16384: every digit at its extreme -> |W_c| <= 4 K 2^14 = 2^30."""
    K = 16384
    worst = 4 * K * 128 * 128
    assert worst <= 2 ** 30


def test_mixed_magnitude_column_error_is_relative_to_the_entries():
    """One node with half the weight and a thousand small ones: the error stays near the
    quantisation of the entries themselves (the case that needs class 4)."""
    rng = np.random.default_rng(5)
    K = 4096
    x = np.linspace(0, 0.75, K // 2)
    T = np.concatenate([np.cos(40 * x) * (1 - x ** 2) ** 30, 0.5 * np.sin(40 * x)])[None, :]
    F = np.zeros((K, 1))
    F[100, 0] = 1000.0
    F[2048:3048, 0] = rng.uniform(0.5, 1.5, 1000)
    err = abs(contract(T, F)[0, 0] - (T @ F)[0, 0])
    assert err <= 1e-9 * (np.abs(F).sum())
