"""ctypes loader for the CPU checker (liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
module.  It exposes the scalar restatement of the par2rust create path
(par2_oracle.c) and the multi-threaded CPU baseline port
(par2_cpu_baseline.c), plus the reference tree's own C MD5 (vendored ISA-L
md5_ref.c, built into _ref/ by the Makefile) when it was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_MD5 = os.path.join(HERE, "_ref", "libmd5_ref.so")

SCHEME_SINGLE, SCHEME_EXPONENTIAL, SCHEME_UNIFORM, SCHEME_LIMITED, SCHEME_EXPLICIT = range(5)


class or_slice_checksum(C.Structure):
    _fields_ = [("md5", C.c_uint8 * 16), ("crc32", C.c_uint32)]


class or_scheme(C.Structure):
    pass


or_scheme._fields_ = [("kind", C.c_int), ("count", C.c_uint32), ("max_blocks_per_volume", C.c_uint32),
                      ("inner", C.POINTER(or_scheme)), ("sizes", C.POINTER(C.c_uint32)), ("n_sizes", C.c_uint32)]


class or_input(C.Structure):
    _fields_ = [("data", C.c_void_p), ("len", C.c_uint64), ("name", C.c_char_p), ("name_len", C.c_size_t)]


_lib = None
_ref = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.or_gf_mul.restype = C.c_uint16
        L.or_gf_pow.restype = C.c_uint16
        L.or_gf_inv.restype = C.c_uint16
        L.or_coefficient.restype = C.c_uint16
        L.or_crc32.restype = C.c_uint32
        L.or_crc32.argtypes = [C.c_void_p, C.c_size_t]
        L.or_md5.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
        L.or_gf_mul_xor_scalar.argtypes = [C.c_uint16, C.c_void_p, C.c_void_p, C.c_size_t]
        L.or_gf_mul_xor_table.argtypes = [C.c_uint16, C.c_void_p, C.c_void_p, C.c_size_t]
        L.or_encode.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32, C.c_void_p]
        L.or_scan.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_char_p, C.c_size_t, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p]
        L.or_file_id.argtypes = [C.c_char_p, C.c_uint64, C.c_char_p, C.c_size_t, C.c_void_p]
        L.or_resolve_volume_sizes.restype = C.c_int64
        L.or_resolve_volume_sizes.argtypes = [C.POINTER(or_scheme), C.c_uint32, C.c_void_p, C.c_uint32]
        L.or_volume_filename.restype = C.c_size_t
        L.or_volume_filename.argtypes = [C.c_char_p, C.c_uint16, C.c_uint32, C.c_char_p, C.c_size_t]
        L.or_create.restype = C.c_int64
        L.or_create.argtypes = [C.POINTER(or_input), C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(or_scheme),
                                C.POINTER(C.c_char_p), C.c_uint32, C.c_char_p, C.POINTER(C.c_void_p),
                                C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.or_set_fast_encode.argtypes = [C.c_int]
        L.or_gfni_matrices.argtypes = [C.c_uint16, C.c_void_p]
        L.or_gfni_apply.argtypes = [C.c_void_p, C.c_uint8, C.c_uint8, C.c_void_p, C.c_void_p]
        L.or_build_main_packet.restype = C.c_size_t
        L.or_build_main_packet.argtypes = [C.c_uint64, C.c_char_p, C.c_uint32, C.c_void_p, C.c_void_p]
        L.or_build_recovery_packet.restype = C.c_size_t
        L.or_build_recovery_packet.argtypes = [C.c_char_p, C.c_uint16, C.c_void_p, C.c_uint64, C.c_void_p]
        L.cb_encode.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_void_p, C.c_int]
        L.cb_encode_rows.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
        L.cb_scan.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.cb_create_timed.restype = C.c_double
        L.cb_create_timed.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_int, C.c_void_p,
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.cb_create_timed_ex.restype = C.c_double
        L.cb_create_timed_ex.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_int, C.c_void_p,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.c_int]
        L.cb_recovery_packet_md5.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32,
                                             C.c_void_p, C.c_int]
        _lib = L
    return _lib


def ref_md5_lib():
    """The reference tree's own MD5 (ISA-L md5_ref.c) or None when not built."""
    global _ref
    if _ref is None and os.path.exists(REF_MD5):
        _ref = C.CDLL(REF_MD5)
        _ref.md5_ref.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32]
    return _ref


def _addr(buf):
    import numpy as np

    a = np.ascontiguousarray(np.frombuffer(buf, dtype=np.uint8) if not isinstance(buf, np.ndarray) else buf)
    return a, a.ctypes.data


# ---- thin Python wrappers ---------------------------------------------------
def md5(data: bytes) -> bytes:
    out = (C.c_uint8 * 16)()
    a, p = _addr(data) if len(data) else (None, None)
    lib().or_md5(p, len(data), out)
    return bytes(out)


def ref_md5(data: bytes) -> bytes:
    r = ref_md5_lib()
    d = (C.c_uint32 * 4)()
    r.md5_ref(bytes(data), d, len(data))
    return b"".join(int(x).to_bytes(4, "little") for x in d)


def crc32(data: bytes) -> int:
    a, p = _addr(data) if len(data) else (None, None)
    return lib().or_crc32(p, len(data))


def gf_tables():
    lg = (C.c_uint16 * 65536)()
    al = (C.c_uint16 * 65536)()
    lib().or_gf_tables(lg, al)
    return list(lg), list(al)


def gf_mul(a, b):
    return lib().or_gf_mul(a, b)


def gf_pow(b, e):
    return lib().or_gf_pow(b, e)


def gf_inv(a):
    return lib().or_gf_inv(a)


def input_bases(n):
    arr = (C.c_uint16 * max(n, 1))()
    lib().or_input_bases(n, arr)
    return list(arr[:n])


def coefficient(r, i):
    return lib().or_coefficient(r, i)


def gf_mul_xor_scalar(coeff, inp: bytes, out: bytearray):
    import numpy as np

    a = np.frombuffer(bytes(inp), dtype=np.uint8)
    o = np.frombuffer(out, dtype=np.uint8)
    lib().or_gf_mul_xor_scalar(coeff, a.ctypes.data, o.ctypes.data, len(a))


def gf_mul_xor_table(coeff, inp: bytes, out: bytearray):
    import numpy as np

    a = np.frombuffer(bytes(inp), dtype=np.uint8)
    o = np.frombuffer(out, dtype=np.uint8)
    lib().or_gf_mul_xor_table(coeff, a.ctypes.data, o.ctypes.data, len(a))


def gfni_matrices(coeff):
    m = (C.c_uint64 * 4)()
    lib().or_gfni_matrices(coeff, m)
    return list(m)


def gfni_apply(mats, lo, hi):
    m = (C.c_uint64 * 4)(*mats)
    a, b = C.c_uint8(), C.c_uint8()
    lib().or_gfni_apply(m, lo, hi, C.byref(a), C.byref(b))
    return a.value, b.value


def encode(src, S: int, slice_size: int, R: int):
    """Scalar reference encode (src/creator.rs:883-1018) -> numpy uint8 R*slice."""
    import numpy as np

    a, p = _addr(src)
    out = np.zeros(R * slice_size, dtype=np.uint8)
    lib().or_encode(p, S, slice_size, R, out.ctypes.data)
    return out


def encode_fast(src, S: int, slice_size: int, R: int, threads: int = 0):
    """CPU baseline encode (GFNI/AVX-512 port, OpenMP)."""
    import numpy as np

    a, p = _addr(src)
    out = np.zeros(R * slice_size, dtype=np.uint8)
    lib().cb_encode(p, 0, S, slice_size, R, out.ctypes.data, threads)
    return out


def encode_rows(src, S: int, slice_size: int, exponents, threads: int = 0):
    """Recovery rows for the listed exponents only (GFNI port, rows in
    parallel) -> numpy uint8 len(exponents) x slice."""
    import numpy as np

    a, p = _addr(src)
    ex = (C.c_uint32 * max(len(exponents), 1))(*exponents)
    out = np.zeros(len(exponents) * slice_size, dtype=np.uint8)
    lib().cb_encode_rows(p, S, slice_size, ex, len(exponents), out.ctypes.data, threads)
    return out.reshape(len(exponents), slice_size)


def scan(data: bytes, slice_size: int, name: bytes):
    """(status, [(md5, crc)], hash_full, hash16k, file_id)"""
    n = (len(data) + slice_size - 1) // slice_size if slice_size else 0
    cks = (or_slice_checksum * max(n, 1))()
    hf, h16, fid = (C.c_uint8 * 16)(), (C.c_uint8 * 16)(), (C.c_uint8 * 16)()
    a, p = _addr(data) if len(data) else (None, None)
    st = lib().or_scan(p, len(data), slice_size, bytes(name), len(name), cks, hf, h16, fid)
    return st, [(bytes(cks[i].md5), cks[i].crc32) for i in range(n if st == 0 else 0)], bytes(hf), bytes(h16), bytes(fid)


def file_id(hash16k: bytes, length: int, name: bytes) -> bytes:
    out = (C.c_uint8 * 16)()
    lib().or_file_id(hash16k, length, name, len(name), out)
    return bytes(out)


def set_id(slice_size: int, file_ids) -> bytes:
    """Recovery set id: MD5 of the main-packet body over the sorted file ids
    (or_build_main_packet, main_packet.rs:25-42)."""
    out = (C.c_uint8 * 16)()
    lib().or_build_main_packet(slice_size, b"".join(file_ids), len(file_ids), out, None)
    return bytes(out)


def recovery_packet_md5(set_id_: bytes, exponent: int, row) -> bytes:
    """Packet MD5 (header bytes 16..32) of the recovery packet of one row
    (or_build_recovery_packet, recovery.rs:11-19)."""
    a, p = _addr(row)
    n = lib().or_build_recovery_packet(set_id_, exponent, p, len(a), None)
    buf = (C.c_uint8 * n)()
    lib().or_build_recovery_packet(set_id_, exponent, p, len(a), buf)
    return bytes(buf)[16:32]


def _scheme_c(kind, count=0, cap=0, inner=None, sizes=None, keep=None):
    keep = keep if keep is not None else []
    s = or_scheme()
    s.kind, s.count, s.max_blocks_per_volume = kind, count, cap
    if inner is not None:
        ic = _scheme_c(*inner, keep=keep)
        keep.append(ic)
        s.inner = C.pointer(ic)
    if sizes is not None:
        arr = (C.c_uint32 * max(len(sizes), 1))(*sizes)
        keep.append(arr)
        s.sizes, s.n_sizes = arr, len(sizes)
    keep.append(s)
    return s


def resolve_volume_sizes(total, kind, count=0, cap=0, inner=None, sizes=None):
    keep = []
    s = _scheme_c(kind, count, cap, inner, sizes, keep)
    n = lib().or_resolve_volume_sizes(C.byref(s), total, None, 0)
    if n < 0:
        return None
    out = (C.c_uint32 * max(n, 1))()
    lib().or_resolve_volume_sizes(C.byref(s), total, out, n)
    return list(out[:n])


def volume_filename(index_path: str, first: int, count: int) -> str:
    buf = C.create_string_buffer(8192)
    lib().or_volume_filename(os.fsencode(index_path), first, count, buf, 8192)
    return os.fsdecode(buf.value)


def create(inputs, slice_size, R, kind=SCHEME_SINGLE, count=0, cap=0, inner=None, sizes=None, comments=(),
           index_path="recovery.par2", fast=False):
    """Whole create in memory: list of (file name, bytes), or a negative status.
    fast=True encodes with the multi-threaded GFNI port (for checks at the
    benchmark sizes, where the scalar encode would take hours)."""
    keep = []
    arr = (or_input * max(len(inputs), 1))()
    for i, (name, data) in enumerate(inputs):
        a, p = _addr(data)
        keep.append(a)
        nb = bytes(name)
        keep.append(nb)
        arr[i].data, arr[i].len, arr[i].name, arr[i].name_len = p, len(a), nb, len(nb)
    s = _scheme_c(kind, count, cap, inner, sizes, keep)
    cm = [c.encode() for c in comments]
    carr = (C.c_char_p * max(len(cm), 1))(*cm)
    blob, sizes_p, names = C.c_void_p(), C.c_void_p(), C.c_void_p()
    lib().or_set_fast_encode(1 if fast else 0)
    try:
        n = lib().or_create(arr, len(inputs), slice_size, R, C.byref(s), carr, len(cm), os.fsencode(index_path),
                            C.byref(blob), C.byref(sizes_p), C.byref(names))
    finally:
        lib().or_set_fast_encode(0)
    if n < 0:
        return n
    fs = C.cast(sizes_p, C.POINTER(C.c_uint64))
    libc = C.CDLL(None)
    out, off, noff = [], 0, 0
    for i in range(n):
        nm = C.string_at(names.value + noff)
        noff += len(nm) + 1
        out.append((os.fsdecode(nm), C.string_at(blob.value + off, fs[i])))
        off += fs[i]
    libc.free(blob)
    libc.free(sizes_p)
    libc.free(names)
    return out


def create_timed(data, slice_size, R, threads=0, want_rec=False, whole_file_md5=True):
    """CPU-baseline create of one in-memory file; (seconds, scan, encode, pkt[, rec]).
    whole_file_md5=False leaves the whole-file MD5 out of the scan."""
    import numpy as np

    a, p = _addr(data)
    rec = np.zeros(R * slice_size, dtype=np.uint8) if want_rec else None
    ts, te, tp = C.c_double(), C.c_double(), C.c_double()
    t = lib().cb_create_timed_ex(p, len(a), slice_size, R, threads, rec.ctypes.data if want_rec else None,
                                 C.byref(ts), C.byref(te), C.byref(tp), 1 if whole_file_md5 else 0)
    if want_rec:
        return t, ts.value, te.value, tp.value, rec
    return t, ts.value, te.value, tp.value


def max_threads() -> int:
    return lib().cb_max_threads()


def kernel_is_gfni512() -> bool:
    return bool(lib().cb_kernel_is_gfni512())
