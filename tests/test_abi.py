"""C ABI of libpar2gpu.so on the CPU: the library loads, exports every entry
point include/par2gpu.h declares, and its pure-host helpers (no device calls)
agree with the oracle."""
import ctypes as C
import hashlib
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "par2gpu.h")
LIB = os.path.join(ROOT, "par2rust_b200", "libpar2gpu.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(p2g_\w+)\s*\(", text, flags=re.M))
    names -= {"p2g_progress_fn"}
    return sorted(names)


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build libpar2gpu.so first (make -C par2rust_b200/csrc)"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (p2g_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    assert len(declared_functions()) >= 30


def test_ffi_signatures_cover_header(p2g):
    from par2rust_b200 import _ffi

    bound = {n for n, _, _ in _ffi.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_build_targets_sm100a_only():
    mk = open(os.path.join(ROOT, "par2rust_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_abi_version(p2g):
    assert p2g._ffi.lib().p2g_abi_version() == 1


def test_host_gf_helpers_match_oracle(p2g, oracle):
    state = 0x1234567
    for _ in range(500):
        state = (state * 6364136223846793005 + 1) & ((1 << 64) - 1)
        a, b, e = state & 0xFFFF, (state >> 16) & 0xFFFF, (state >> 32) & 0xFFFF
        assert p2g.gf_mul(a, b) == oracle.gf_mul(a, b)
        assert p2g.gf_pow(a, e) == oracle.gf_pow(a, e)
    assert p2g.input_bases(32768) == oracle.input_bases(32768)


def test_host_md5_and_file_id(p2g, oracle):
    for n in [0, 1, 55, 56, 64, 100, 1000]:
        d = bytes((i * 7) & 0xFF for i in range(n))
        assert p2g.md5(d) == hashlib.md5(d).digest()
    h = b"\x11" * 16
    assert p2g.compute_file_id(h, 0x12345678, b"example.dat") == oracle.file_id(h, 0x12345678, b"example.dat")


def test_host_packets(p2g):
    set_id = b"\xaa" * 16
    pkt = p2g.build_packet(set_id, b"PAR 2.0\0Creator\0", b"\0" * 8)
    assert len(pkt) == 72 and pkt[:8] == b"PAR2\0PKT" and pkt[32:48] == set_id
    assert int.from_bytes(pkt[8:16], "little") == 72
    assert pkt[16:32] == hashlib.md5(set_id + b"PAR 2.0\0Creator\0" + b"\0" * 8).digest()
    ids = [b"\x20" * 16, b"\x10" * 16, b"\x30" * 16]
    main, sid = p2g.build_main_packet(4096, ids)
    body = main[64:]
    assert body[12:28] == b"\x10" * 16 and body[28:44] == b"\x20" * 16 and body[44:60] == b"\x30" * 16
    assert sid == hashlib.md5(body).digest() == main[32:48]


def test_host_volume_logic(p2g, oracle):
    VS = p2g.VolumeScheme
    assert p2g.resolve_volume_sizes(VS.Exponential(), 10) == [1, 1, 2, 4, 2]
    assert p2g.resolve_volume_sizes(VS.Exponential(), 200) == oracle.resolve_volume_sizes(200, oracle.SCHEME_EXPONENTIAL)
    assert p2g.resolve_volume_sizes(VS.Uniform(4), 13) == [3, 3, 3, 4]
    assert p2g.resolve_volume_sizes(VS.Limited(4, VS.Uniform(2)), 20) == [4, 4, 2, 4, 4, 2]
    assert p2g.resolve_volume_sizes(VS.Single(), 7) == [7]
    assert p2g.resolve_volume_sizes(VS.Explicit([3, 3]), 6) == [3, 3]
    for bad, total in [(VS.Uniform(0), 10), (VS.Uniform(5), 3), (VS.Limited(0, VS.Exponential()), 10),
                       (VS.Explicit([2, 2]), 5), (VS.Explicit([2, 0, 2]), 4), (VS.Explicit([]), 1)]:
        with pytest.raises(p2g.InvalidVolumeScheme):
            p2g.resolve_volume_sizes(bad, total)
    for t in [1, 2, 3, 7, 50, 100, 1000, 65535]:
        assert p2g.resolve_volume_sizes(VS.Exponential(), t) == oracle.resolve_volume_sizes(t, oracle.SCHEME_EXPONENTIAL)
    for path in ["recovery.par2", "/a/b/x.par2", "noext", ".par2", "a.b.par2", "dir/name."]:
        for first, cnt in [(0, 1), (8, 2), (65534, 1)]:
            assert p2g.volume_filename(path, first, cnt) == oracle.volume_filename(path, first, cnt)


def test_errors_map_to_par2error_variants(p2g):
    assert issubclass(p2g.TooManyInputBlocks, p2g.Par2Error)
    assert p2g.InvalidSliceSize.status == 2 and p2g.InvalidVolumeScheme.status == 9


def test_struct_layouts_match_header(tmp_path):
    """Every public struct: the ctypes mirror (which the Rust bindings in the
    integration notes copy) has the C header's size and field offsets, as gcc
    lays them out."""
    import ctypes as C
    import shutil
    import subprocess

    from par2rust_b200 import _ffi

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    structs = {n: getattr(_ffi, n) for n in dir(_ffi)
               if n.startswith("p2g_") and isinstance(getattr(_ffi, n), type) and issubclass(getattr(_ffi, n), C.Structure)}
    assert len(structs) >= 18
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "par2gpu.h"', "int main(void) {"]
    for n, cls in structs.items():
        lines.append(f'    printf("{n} %zu\\n", sizeof({n}));')
        for f in cls._fields_:
            lines.append(f'    printf("{n}.{f[0]} %zu\\n", offsetof({n}, {f[0]}));')
    lines += ["    return 0;", "}"]
    c_file = tmp_path / "layout.c"
    c_file.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(c_file), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                       text=True).stdout.splitlines())
    for n, cls in structs.items():
        assert int(got[n]) == C.sizeof(cls), n
        for f in cls._fields_:
            assert int(got[f"{n}.{f[0]}"]) == getattr(cls, f[0]).offset, f"{n}.{f[0]}"
