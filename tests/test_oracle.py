"""Pins the CPU oracle (oracle/par2_oracle.c) before anything is compared to it.

Known answers are the reference's own unit tests (galois.rs, reedsolomon.rs,
galois_simd.rs, md5_impl.rs, source.rs, format.rs, packet/*.rs, creator.rs);
hashes are cross-checked against three independent implementations
(Python hashlib/zlib, the reference tree's vendored ISA-L md5_ref.c) and GF
arithmetic against an independent carry-less multiply in Python.
"""
import hashlib
import itertools
import os
import zlib

import numpy as np
import pytest

from par2rust_b200.workloads import deterministic_bytes


# ---- GF(2^16): src/galois.rs:101-184 -------------------------------------
def clmul_mod(a, b, poly=0x1100B):
    r = 0
    while b:
        if b & 1:
            r ^= a
        b >>= 1
        a <<= 1
        if a & 0x10000:
            a ^= poly
    return r


def test_tables_have_expected_sentinels(oracle):
    lg, al = oracle.gf_tables()
    assert lg[0] == 65535 and al[0] == 1 and al[1] == 2 and al[65535] == 0


def test_tables_match_independent_clmul(oracle):
    lg, al = oracle.gf_tables()
    x = 1
    for k in range(65535):
        assert al[k] == x
        x = clmul_mod(x, 2)
    assert sorted(al[:65535]) == list(range(1, 65536))


def test_multiplication_is_commutative_and_matches_clmul(oracle):
    state = 0xCAFEBABE
    for _ in range(2000):
        state = (state * 2654435761 + 1) & 0xFFFFFFFF
        a, b = state & 0xFFFF, state >> 16
        assert oracle.gf_mul(a, b) == oracle.gf_mul(b, a) == clmul_mod(a, b)


def test_zero_identity_inverse_pow(oracle):
    for x in [1, 2, 0xABCD, 0xFFFF]:
        assert oracle.gf_mul(0, x) == 0 == oracle.gf_mul(x, 0)
    for x in [1, 2, 3, 0x100, 0x1234, 0xFFFF]:
        assert oracle.gf_mul(1, x) == x
    for x in range(1, 65536, 7):
        assert oracle.gf_mul(x, oracle.gf_inv(x)) == 1
    for b in [0, 1, 2, 0x1234, 0xFFFF]:
        assert oracle.gf_pow(b, 0) == 1
    for e in [1, 2, 100, 65535]:
        assert oracle.gf_pow(0, e) == 0
    _, al = oracle.gf_tables()
    for k in [0, 1, 2, 100, 1000, 65534]:
        assert oracle.gf_pow(2, k) == al[k % 65535]
    for a in [1, 3, 0x1111, 0xFFFE]:
        a2 = oracle.gf_mul(a, a)
        assert oracle.gf_mul(oracle.gf_mul(a2, a2), a2) == oracle.gf_pow(a, 6)


# ---- RS: src/reedsolomon.rs:159-277 ----------------------------------------
def test_input_bases(oracle):
    lg, al = oracle.gf_tables()
    b = oracle.input_bases(20)
    assert b[0] == 2 and b[1] == al[2]
    logs = [lg[x] for x in b]
    for skip in [0, 3, 5, 6, 9, 10, 15, 17]:
        assert skip not in logs
    big = oracle.input_bases(32768)
    assert len(set(big)) == 32768
    from math import gcd

    want = [al[l] for l in range(65535) if gcd(65535, l) == 1]
    assert big == want


def test_coefficients(oracle):
    b = oracle.input_bases(4)
    for r in range(5):
        for i in range(4):
            assert oracle.coefficient(r, i) == oracle.gf_pow(b[i], r)
    assert all(oracle.coefficient(0, i) == 1 for i in range(3))


def test_mac_identities(oracle):
    out = bytearray(8)
    out[0], out[7] = 0x11, 0x77
    oracle.gf_mul_xor_scalar(0, b"\xff" * 8, out)
    assert out == bytearray([0x11, 0, 0, 0, 0, 0, 0, 0x77])
    out = bytearray([0xAA, 0xBB, 0xCC, 0xDD])
    oracle.gf_mul_xor_scalar(1, bytes([0x12, 0x34, 0x56, 0x78]), out)
    assert out == bytearray([0xAA ^ 0x12, 0xBB ^ 0x34, 0xCC ^ 0x56, 0xDD ^ 0x78])
    inp = bytes([0x11, 0x22, 0xFF, 0x00, 0x99, 0xAB])
    out = bytearray([0x10, 0x20, 0x30, 0x40, 0x50, 0x60])
    exp = bytearray(out)
    for k in range(3):
        p = clmul_mod(0x1234, inp[2 * k] | inp[2 * k + 1] << 8)
        exp[2 * k] ^= p & 0xFF
        exp[2 * k + 1] ^= p >> 8
    oracle.gf_mul_xor_scalar(0x1234, inp, out)
    assert out == exp
    # 2 inputs, 1 recovery -> XOR (rs_encode_roundtrip_with_one_redundancy_block)
    src = bytes(range(16)) + bytes(range(16, 32))
    rec = oracle.encode(src, 2, 16, 1)
    assert bytes(rec) == bytes(a ^ b for a, b in zip(range(16), range(16, 32)))


@pytest.mark.parametrize("coeff", [0x0001, 0x0002, 0x00FF, 0x1234, 0xABCD, 0xFFFF])
def test_table_kernel_matches_scalar(oracle, coeff):
    for ln in [2, 4, 16, 30, 32, 34, 64, 256, 4096]:
        inp = deterministic_bytes(coeff ^ ln, ln)
        a, b = bytearray(ln), bytearray(ln)
        oracle.gf_mul_xor_scalar(coeff, inp, a)
        oracle.gf_mul_xor_table(coeff, inp, b)
        assert a == b


@pytest.mark.parametrize("coeff", [0x0002, 0x00FF, 0x0100, 0x1234, 0x8000, 0xABCD, 0xFFFE, 0xFFFF])
def test_gfni_matrices_all_65536_symbols(oracle, coeff):
    """gfni_affine_matrices_round_trip_a_single_symbol, src/galois_simd.rs:849-874"""
    mats = oracle.gfni_matrices(coeff)
    # vectorised affine evaluation of the four 8x8 blocks
    sym = np.arange(65536, dtype=np.uint32)
    lo, hi = (sym & 0xFF).astype(np.uint8), (sym >> 8).astype(np.uint8)

    def aff(m, x):
        y = np.zeros_like(x)
        for i in range(8):
            row = np.uint8((m >> ((7 - i) * 8)) & 0xFF)
            y |= ((np.unpackbits((row & x)[:, None], axis=1).sum(axis=1) & 1) << i).astype(np.uint8)
        return y

    out_lo = aff(mats[0], lo) ^ aff(mats[1], hi)
    out_hi = aff(mats[2], lo) ^ aff(mats[3], hi)
    got = out_lo.astype(np.uint32) | (out_hi.astype(np.uint32) << 8)
    _, al = oracle.gf_tables()
    lg, _ = oracle.gf_tables()
    lc = lg[coeff]
    want = np.array([0 if s == 0 else al[(lc + lg[s]) % 65535] for s in range(65536)], dtype=np.uint32)
    assert (got == want).all()


def test_cpu_baseline_encode_matches_scalar(oracle):
    for S, slice_, R in [(3, 256, 5), (5, 4096, 33), (2, 132, 3), (1, 4, 2)]:
        src = np.frombuffer(deterministic_bytes(S * 7 + R, S * slice_), dtype=np.uint8)
        a = oracle.encode(src, S, slice_, R)
        b = oracle.encode_fast(src, S, slice_, R, threads=4)
        assert (a == b).all(), (S, slice_, R)


def test_encode_rows_matches_full_encode(oracle):
    S, slice_, R = 7, 4096, 40
    src = np.frombuffer(deterministic_bytes(77, S * slice_), dtype=np.uint8)
    full = oracle.encode(src, S, slice_, R).reshape(R, slice_)
    rows = [0, 1, 17, 39]
    assert (oracle.encode_rows(src, S, slice_, rows) == full[rows]).all()


def test_fast_create_matches_scalar_create(oracle):
    """create(fast=True) (the GFNI port as encoder) gives the scalar create's
    files byte for byte, multi-file and ragged tails included; the GPU tests
    at benchmark sizes compare against the fast form."""
    files = [(b"a.bin", deterministic_bytes(11, 70_001)), (b"b.bin", deterministic_bytes(12, 4096 * 3)),
             (b"c.bin", deterministic_bytes(13, 17))]
    for kind, count in [(oracle.SCHEME_EXPONENTIAL, 0), (oracle.SCHEME_UNIFORM, 3)]:
        a = oracle.create(files, 4096, 21, kind=kind, count=count)
        b = oracle.create(files, 4096, 21, kind=kind, count=count, fast=True)
        assert a == b


# ---- MD5 / CRC32 -------------------------------------------------------------
def test_md5_known_vectors(oracle):
    assert oracle.md5(b"").hex() == "d41d8cd98f00b204e9800998ecf8427e"
    assert oracle.md5(b"abc").hex() == "900150983cd24fb0d6963f7d28e17f72"


def test_md5_three_way_cross_check(oracle):
    ref = oracle.ref_md5_lib()
    for n in [0, 1, 55, 56, 63, 64, 65, 119, 120, 127, 128, 1000, 16384, 65537]:
        d = deterministic_bytes(n, n)
        h = hashlib.md5(d).digest()
        assert oracle.md5(d) == h
        if ref is not None:
            assert oracle.ref_md5(d) == h


def test_crc32_check_value(oracle):
    assert oracle.crc32(b"123456789") == 0xCBF43926
    for n in [0, 1, 3, 4, 5, 100, 4096, 65540]:
        d = deterministic_bytes(n + 1, n)
        assert oracle.crc32(d) == zlib.crc32(d)


# ---- scan: src/source.rs:325-471 --------------------------------------------
def test_scan_zero_padded_last_slice(oracle):
    st, cks, hf, h16, fid = oracle.scan(b"ABCDE", 4, b"file.bin")
    assert st == 0 and len(cks) == 2
    assert cks[0][0] == hashlib.md5(b"ABCD").digest()
    assert cks[1][0] == hashlib.md5(b"E\0\0\0").digest()
    assert hf == hashlib.md5(b"ABCDE").digest() == h16
    assert cks[1][1] == zlib.crc32(b"E\0\0\0")


def test_scan_hash16k_truncation(oracle):
    data = bytes(i & 0xFF for i in range(16384 + 100))
    st, cks, hf, h16, fid = oracle.scan(data, 4096, b"big.bin")
    assert h16 == hashlib.md5(data[:16384]).digest() and hf == hashlib.md5(data).digest()


def test_file_id_derivation(oracle):
    h = b"\x11" * 16
    length = 0x12345678
    name = b"example.dat"
    assert oracle.file_id(h, length, name) == hashlib.md5(h + length.to_bytes(8, "little") + name).digest()


def test_scan_slice_count_and_order(oracle):
    data = bytes(range(17))
    st, cks, *_ = oracle.scan(data, 8, b"x")
    assert len(cks) == 3 and cks[2][0] == hashlib.md5(bytes([16]) + b"\0" * 7).digest()
    data = bytes(((i * 0x9E37) >> 5) & 0xFF for i in range(4096 * 16))
    st, cks, *_ = oracle.scan(data, 16, b"x")
    assert len(cks) == 4096
    for i in [0, 1, 7, 1023, 4095]:
        assert cks[i] == (hashlib.md5(data[16 * i:16 * i + 16]).digest(), zlib.crc32(data[16 * i:16 * i + 16]))


def test_scan_validation(oracle):
    assert oracle.scan(b"", 4, b"x")[0] == -5  # EmptyFile
    assert oracle.scan(b"hi", 0, b"x")[0] == -2  # InvalidSliceSize
    assert oracle.scan(b"hi", 5, b"x")[0] == -2
    assert oracle.scan(b"x", 4, b"")[0] == -3  # InvalidFileName
    assert oracle.scan(b"x", 4, b"bad\0name")[0] == -3


# ---- volumes: src/creator.rs:1347-1619 ---------------------------------------
def test_volume_splits(oracle):
    E, U, L, X = oracle.SCHEME_EXPONENTIAL, oracle.SCHEME_UNIFORM, oracle.SCHEME_LIMITED, oracle.SCHEME_EXPLICIT
    assert oracle.resolve_volume_sizes(1, E) == [1]
    assert oracle.resolve_volume_sizes(2, E) == [1, 1]
    assert oracle.resolve_volume_sizes(4, E) == [1, 1, 2]
    assert oracle.resolve_volume_sizes(10, E) == [1, 1, 2, 4, 2]
    assert oracle.resolve_volume_sizes(200, E) == [1, 1, 2, 4, 8, 16, 32, 64, 72]
    for t in [1, 2, 3, 7, 50, 100, 1000, 65535]:
        s = oracle.resolve_volume_sizes(t, E)
        assert sum(s) == t and all(s)
    assert oracle.resolve_volume_sizes(10, U, count=5) == [2] * 5
    assert oracle.resolve_volume_sizes(13, U, count=4) == [3, 3, 3, 4]
    assert oracle.resolve_volume_sizes(42, U, count=1) == [42]
    assert oracle.resolve_volume_sizes(10, U, count=0) is None
    assert oracle.resolve_volume_sizes(3, U, count=5) is None
    assert oracle.resolve_volume_sizes(2000, U, count=15) == [133] * 14 + [138]
    s = oracle.resolve_volume_sizes(20, L, cap=3, inner=(E,))
    assert all(0 < n <= 3 for n in s) and sum(s) == 20
    assert oracle.resolve_volume_sizes(20, L, cap=4, inner=(U, 2)) == [4, 4, 2, 4, 4, 2]
    assert oracle.resolve_volume_sizes(10, L, cap=0, inner=(E,)) is None
    assert oracle.resolve_volume_sizes(5, X, sizes=[2, 2]) is None
    assert oracle.resolve_volume_sizes(4, X, sizes=[2, 0, 2]) is None
    assert oracle.resolve_volume_sizes(6, X, sizes=[3, 3]) == [3, 3]


def test_volume_names(oracle):
    assert oracle.volume_filename("recovery.par2", 0, 4) == "recovery.vol0+4.par2"
    assert oracle.volume_filename("/a/b/x.par2", 8, 2) == "/a/b/x.vol8+2.par2"
    assert oracle.volume_filename("noext", 1, 1) == "noext.vol1+1.par2"


# ---- packets: src/format.rs, src/packet/*.rs ----------------------------------
def test_create_index_only_layout(oracle):
    files = oracle.create([(b"a.bin", b"hello par2 world")], 4, 0)
    assert len(files) == 1 and files[0][0] == "recovery.par2"
    blob = files[0][1]
    # main packet first: header magic, length, then set id == MD5(body)
    assert blob[:8] == b"PAR2\0PKT"
    plen = int.from_bytes(blob[8:16], "little")
    body = blob[64:plen]
    assert blob[32:48] == hashlib.md5(body).digest()
    assert blob[16:32] == hashlib.md5(blob[32:48] + blob[48:64] + body).digest()
    assert blob[48:64] == b"PAR 2.0\0Main\0\0\0\0"
    # creator packet present with the exact string
    assert b"Created by par2rust v0.1.0" in blob


def test_create_volume_names_exponential(oracle):
    files = oracle.create([(b"a.bin", b"\xab" * (4096 * 4))], 4096, 10, kind=oracle.SCHEME_EXPONENTIAL)
    assert [n for n, _ in files[1:]] == ["recovery.vol0+1.par2", "recovery.vol1+1.par2", "recovery.vol2+2.par2",
                                        "recovery.vol4+4.par2", "recovery.vol8+2.par2"]


def test_create_errors(oracle):
    assert oracle.create([], 4, 0) == -4
    assert oracle.create([(b"a", b"x")], 4, 65536) == -7
    assert oracle.create([(b"a", b"hello par2 world!!!!")], 4, 5, kind=oracle.SCHEME_EXPLICIT, sizes=[2, 2]) == -9


def test_comment_packets(oracle):
    files = oracle.create([(b"a", b"abcd")], 4, 0, comments=["hello", "héllo"])
    blob = files[0][1]
    assert blob.count(b"PAR 2.0\0CommASCI") == 2 and blob.count(b"PAR 2.0\0CommUni\0") == 1
    assert b"h?llo" in blob


# ---- RS decode self-check (replaces upstream `par2 r`) ---------------------
def gf_solve(oracle, M, B):
    """Solve M x = B over GF(2^16) (M k x k ints, B k rows of numpy u16 arrays)."""
    k = len(M)
    M = [row[:] for row in M]
    B = [b.copy() for b in B]
    lg, al = oracle.gf_tables()
    lg = np.array(lg, dtype=np.int64)
    al = np.array(al, dtype=np.uint16)

    def mulv(c, v):  # c * vector
        if c == 0:
            return np.zeros_like(v)
        out = al[(lg[c] + lg[v.astype(np.int64)]) % 65535]
        out[v == 0] = 0
        return out

    for col in range(k):
        piv = next(r for r in range(col, k) if M[r][col])
        M[col], M[piv] = M[piv], M[col]
        B[col], B[piv] = B[piv], B[col]
        inv = oracle.gf_inv(M[col][col])
        M[col] = [oracle.gf_mul(inv, x) for x in M[col]]
        B[col] = mulv(inv, B[col])
        for r in range(k):
            if r != col and M[r][col]:
                f = M[r][col]
                M[r] = [x ^ oracle.gf_mul(f, y) for x, y in zip(M[r], M[col])]
                B[r] = B[r] ^ mulv(f, B[col])
    return B


def decode_check(oracle, src: np.ndarray, S: int, slice_: int, rec: np.ndarray, R: int, erased, rows):
    """Erase `erased` source slices, rebuild them from recovery `rows`, compare."""
    sym = src.view(np.uint16).reshape(S, slice_ // 2)
    rsym = rec.view(np.uint16).reshape(R, slice_ // 2)
    keep = [s for s in range(S) if s not in erased]
    rhs = []
    for r in rows:
        acc = rsym[r].copy()
        for s in keep:  # subtract (XOR) the known columns
            c = oracle.coefficient(r, s)
            if c:
                lg, al = oracle.gf_tables()
                acc ^= np.array([0 if v == 0 else al[(lg[c] + lg[v]) % 65535] for v in sym[s]], dtype=np.uint16)
        rhs.append(acc)
    M = [[oracle.coefficient(r, e) for e in erased] for r in rows]
    sol = gf_solve(oracle, M, rhs)
    for e, x in zip(erased, sol):
        assert (x == sym[e]).all()


def test_oracle_decode_round_trip(oracle):
    S, slice_, R = 6, 64, 4
    src = np.frombuffer(deterministic_bytes(99, S * slice_), dtype=np.uint8).copy()
    rec = oracle.encode(src, S, slice_, R)
    decode_check(oracle, src, S, slice_, rec, R, erased=[1, 4, 5], rows=[0, 2, 3])
