"""Host restatement of the tensor-core bin sums' fixed-point arithmetic
(directsht_b200/csrc/bin_sums_tc.cu), checked on the CPU.

The kernel rounds every operand to X = rint(x q), q = 2^22 - 2^10, writes X as three
balanced base-256 digits (the bytes of (X + 0x8080) ^ 0x8080, each a signed byte), forms
the eight digit products with five int8 MMAs (B0 and B1 as one operand) into four exact
int32 accumulators W0..W3 and combines them as 2^24 W0 + 2^16 W1 + 2^8 W2 + W3 in int64.
The e^{i c phi} operands come from Chebyshev recurrences in FP64.  These tests pin the
digit split, the grouping of the products, the int32 head-room of a 2048-point piece, the
recurrences' accuracy and the error of a piece's sums against the exact sums of
sht/shared_interp_funcs.py:88-105."""
import numpy as np

Q = 4193280.0  # 2^22 - 2^10


def digits(X):
    """Balanced base-256 digits (d0, d1, d2) of int64 X: the bytes of (X + 0x8080) ^ 0x8080."""
    Z = (np.asarray(X, dtype=np.int64) + 0x8080) ^ 0x8080
    out = []
    for shift in (16, 8, 0):
        b = (Z >> shift) & 0xFF
        out.append(np.where(b >= 128, b - 256, b))
    return out


def w_accumulators(A, B):
    """W0..W3 of the kernel: A (rows x K) and B (cols x K) integer operands, products of
    digits grouped as the five MMAs group them (A_i [B0|B1] lands on W_i and W_(i+1))."""
    a = digits(A)
    b = digits(B)
    B01 = np.concatenate([b[0], b[1]], axis=0)  # one 2N-row operand
    n = B.shape[0]
    W = [np.zeros((A.shape[0], n), dtype=np.int64) for _ in range(4)]
    W[2] += a[0] @ b[2].T
    W[3] += a[1] @ b[2].T
    for i in range(3):
        P = a[i] @ B01.T
        W[i] += P[:, :n]
        W[i + 1] += P[:, n:]
    return W


def test_digits_reconstruct_and_fit_a_signed_byte():
    X = np.arange(-(2**22) + 1, 2**22, 997, dtype=np.int64)
    X = np.concatenate([X, [-(2**22) + 1, 2**22 - 1, 0, 1, -1, 255, -256, 0x7F7F, -0x8080]])
    d0, d1, d2 = digits(X)
    assert np.array_equal(d0 * 65536 + d1 * 256 + d2, X)
    for d in (d0, d1, d2):
        assert d.min() >= -128 and d.max() <= 127


def test_grouped_products_equal_the_exact_product_but_the_lowest():
    rng = np.random.default_rng(1)
    A = rng.integers(-(2**22) + 1, 2**22, size=(6, 300))
    B = rng.integers(-(2**22) + 1, 2**22, size=(5, 300))
    W = w_accumulators(A, B)
    T = (W[0] << 24) + (W[1] << 16) + (W[2] << 8) + W[3]
    a2, b2 = digits(A)[2], digits(B)[2]
    exact = A @ B.T  # < 2^63 here
    assert np.array_equal(T * 256 + a2 @ b2.T, exact)


def test_int32_headroom_of_a_2048_point_piece():
    # worst case: every digit at its extreme, 2048 points
    K = 2048
    A = np.full((1, K), 2**22 - 1, dtype=np.int64)
    B = np.full((1, K), -(2**22) + 1, dtype=np.int64)
    for sa in (1, -1):
        W = w_accumulators(sa * A, B)
        assert max(int(np.abs(w).max()) for w in W) < 2**31
    # the epilogue's int64 value stays below 2^51 (exact conversion through 1.5 * 2^52)
    T = (W[0] << 24) + (W[1] << 16) + (W[2] << 8) + W[3]
    assert int(np.abs(T).max()) * 2 < 2**51


def test_chebyshev_anchors_match_exp():
    rng = np.random.default_rng(2)
    phi = rng.uniform(0, 2 * np.pi, 2000)
    z = np.exp(1j * phi)
    z2 = z * z
    m2 = 2 * z2.real  # 2 cos 2 phi
    worst = 0.0
    # four chains of step 2 over c = 0..63: starts c0 = 0, 1, 32, 33
    for c0 in (0, 1, 32, 33):
        E = z ** c0
        Ep = E * np.conj(z2)  # z^(c0 - 2)
        for u in range(16):
            worst = max(worst, np.abs(E - np.exp(1j * (c0 + 2 * u) * phi)).max())
            E, Ep = m2 * E - Ep, E
    assert worst < 1e-11  # far below the fixed-point step 2^-22


def test_piece_sums_error_within_bound():
    """One 2048-point piece of lognormal(0, 0.5) weights: the fixed-point sums against exact FP64 sums
    of g_k e^{i m phi}, relative to the largest |sum| (the kernel's accuracy claim: below
    1e-7 for pieces of spread weights)."""
    rng = np.random.default_rng(3)
    K, Cf, CH = 2048, 64, 64
    phi = rng.uniform(0, 1.5 * np.pi, K)
    t = rng.uniform(0, 1, K)
    w = rng.lognormal(0, 0.5, K)
    omt = 1 - t
    H = np.stack([w * (2 * t + 1) * omt * omt, w * t * omt * omt, w * t * t * (3 - 2 * t), w * t * t * (t - 1)])
    kscale = np.array([1.0, 0.3, 1.0, 0.3])
    scale = np.abs(H).max() * (1 + 2**-20)
    a = np.arange(16)
    c = np.arange(CH)
    ea = np.exp(1j * Cf * a[:, None] * phi[None, :])          # 16 x K
    ec = np.exp(1j * c[:, None] * phi[None, :])                # CH x K
    # FP32 A operand as the slicers form it: g_k (FP32) times e^{i Cf a phi} (FP32)
    gk = (H / (scale * kscale[:, None])).astype(np.float32)
    rows = []
    for k in range(4):
        L = gk[k][None, :] * ea.astype(np.complex64)
        rows += [L.real, L.imag]
    Lr = np.stack(rows)  # (8, 16, K): (k, re|im) x a
    A = np.rint(Lr.reshape(-1, K).astype(np.float64) * Q).astype(np.int64)
    Bre = np.rint(ec.real * Q).astype(np.int64)
    Bim = np.rint(ec.imag * Q).astype(np.int64)
    B = np.concatenate([Bre, Bim], axis=0)
    W = w_accumulators(A, B)
    T = ((W[0] << 24) + (W[1] << 16) + (W[2] << 8) + W[3]).astype(np.float64) * 256.0 / (Q * Q)
    T = T.reshape(4, 2, 16, 2 * CH)
    got = np.zeros((4, 16 * CH), dtype=complex)
    for k in range(4):
        re = T[k, 0, :, :CH] - T[k, 1, :, CH:]
        im = T[k, 0, :, CH:] + T[k, 1, :, :CH]
        got[k] = ((re + 1j * im) * scale * kscale[k]).reshape(-1)
    m = (Cf * a[:, None] + c[None, :]).reshape(-1)
    exact = np.stack([(H[k][None, :] * np.exp(1j * m[:, None] * phi[None, :])).sum(1) for k in range(4)])
    rel = np.abs(got - exact).max() / np.abs(exact).max()
    assert rel < 1e-7, rel
