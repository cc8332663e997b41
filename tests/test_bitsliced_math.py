"""The arithmetic of the tensor-core (bit-sliced) encode, checked on the CPU.

Multiplication by a constant c in GF(2^16) (polynomial 0x1100B, src/galois.rs)
is GF(2)-linear: bits(c*x) = M_c bits(x).  The tensor form needs, per
coefficient, a 16x16 bit matrix whose ROWS are cheap to produce.  With the
trace form G[i][j] = Tr(a^(i+j)) (a = 2, the generator), M_c^T G = G M_c
(multiplication is self-adjoint under Tr(u*v)), so

    bits(c*x) = G^-1 H_c bits(x),   H_c[i][j] = Tr(c * a^(i+j)),

and H_c is a Hankel matrix: row i is bits i..i+15 of the 31-bit string
T_c = sum_k Tr(c*a^k) 2^k, k < 31.  So a recovery row is
G^-1 (XOR over slices of H_c(r,s) x_s): the kernel builds each row of H
from one shift of T_c, the tensor cores sum the 0/1 products, the parity
of each sum is one bit of y, and G^-1 y is the recovery symbol.
"""
import numpy as np

POLY = 0x1100B


def _tables():
    al = np.zeros(65536, np.int64)
    v = 1
    for k in range(65535):
        al[k] = v
        v <<= 1
        if v & 0x10000:
            v ^= POLY
    lg = np.zeros(65536, np.int64)
    lg[al[:65535]] = np.arange(65535)
    return al, lg


AL, LG = _tables()


def gf_mul(a, b):
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    r = AL[(LG[a] + LG[b]) % 65535]
    return np.where((a == 0) | (b == 0), 0, r)


def trace(y):
    y = np.asarray(y, np.int64)
    acc, z = y.copy(), y.copy()
    for _ in range(15):
        z = gf_mul(z, z)
        acc ^= z
    return acc


def _gf2_inv(m):
    n = m.shape[0]
    a = np.concatenate([m.copy() % 2, np.eye(n, dtype=np.int64)], axis=1)
    for c in range(n):
        p = next(r for r in range(c, n) if a[r, c])
        a[[c, p]] = a[[p, c]]
        for r in range(n):
            if r != c and a[r, c]:
                a[r] ^= a[c]
    return a[:, n:]


TR = trace(AL[:47])                      # Tr(a^k), k < 47
G = np.array([[TR[i + j] for j in range(16)] for i in range(16)], np.int64)
GINV = _gf2_inv(G)


def bits(x):
    return (np.asarray(x, np.int64)[..., None] >> np.arange(16)) & 1


def from_bits(b):
    return (b << np.arange(16)).sum(-1)


def t_string(c):
    """T_c = sum_k Tr(c a^k) 2^k, k < 31."""
    c = np.asarray(c, np.int64)
    return (trace(gf_mul(c[..., None], AL[np.arange(31)])) << np.arange(31)).sum(-1)


def test_trace_is_linear_and_g_is_invertible():
    assert set(np.unique(TR)) <= {0, 1}
    a, b = 0x1234, 0xBEEF
    assert trace(a ^ b) == trace(a) ^ trace(b)
    assert ((G @ GINV) % 2 == np.eye(16, dtype=np.int64)).all()


def test_multiplication_is_self_adjoint_under_the_trace_form():
    rng = np.random.default_rng(1)
    for c in rng.integers(1, 65536, 8):
        M = bits(gf_mul(c, 1 << np.arange(16))).T     # column j = bits of c*a^j
        assert ((M.T @ G) % 2 == (G @ M) % 2).all()


def test_hankel_rows_give_the_product():
    rng = np.random.default_rng(2)
    c = rng.integers(1, 65536, 300)
    x = rng.integers(0, 65536, 300)
    T = t_string(c)
    H = (T[:, None] >> np.arange(16)[None, :])[:, :, None] >> np.arange(16)[None, None, :] & 1  # H[i][j] = bit i+j
    y = (H * bits(x)[:, None, :]).sum(-1) % 2          # y_i = parity of sum_j H[i][j] x_j
    got = from_bits((bits(from_bits(y)) @ GINV.T) % 2)
    assert (got == gf_mul(c, x)).all()


def test_row_is_the_parity_of_summed_slices():
    """One recovery symbol from S slices: XOR of products == G^-1 of the
    parity of the summed 0/1 products (what the MMA accumulates)."""
    rng = np.random.default_rng(3)
    S = 50
    c = rng.integers(1, 65536, S)
    x = rng.integers(0, 65536, S)
    want = np.bitwise_xor.reduce(gf_mul(c, x))
    T = t_string(c)
    A = ((T[:, None, None] >> (np.arange(16)[None, :, None] + np.arange(16)[None, None, :])) & 1)  # [s][i][j]
    D = np.einsum("sij,sj->i", A, bits(x))               # integer sums over slices and bits
    got = from_bits((bits(from_bits(D % 2)) @ GINV.T) % 2)
    assert got == want
