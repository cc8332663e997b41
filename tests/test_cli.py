"""The create CLI (src/main.rs): argument semantics through the C ABI, the
par2rust executable's pre-scan errors on the CPU, and whole creates through
the executable on the GPU against the oracle.

The CPU tests port the reference's own unit tests (src/main.rs:558-693) and
the flag rules of build_volume_scheme (:289-337); the GPU tests follow
tests/cli.rs (--out, --comment, --recurse, --input-file, --quiet,
--single-volume), with the written files compared byte for byte with the
oracle's instead of repaired by par2cmdline (absent here).
"""
import os
import subprocess

import pytest

from par2rust_b200.workloads import deterministic_bytes


def test_parses_percent(p2g):
    R = p2g.Redundancy
    assert R.parse("10") == R(percent=10)
    assert R.parse("0") == R(percent=0)
    assert R.parse("250") == R(percent=250)


def test_parses_size_targets(p2g):
    R = p2g.Redundancy
    assert R.parse("k500") == R(target_bytes=500 * 1024)
    assert R.parse("m10") == R(target_bytes=10 * 1024 * 1024)
    assert R.parse("g2") == R(target_bytes=2 * 1024 * 1024 * 1024)
    assert R.parse("M1") == R(target_bytes=1024 * 1024)  # unit letter is case-insensitive


@pytest.mark.parametrize("bad", ["", "abc", "k", "-5"])
def test_redundancy_rejects_bad_input(p2g, bad):
    with pytest.raises(p2g.InvalidArgument):
        p2g.Redundancy.parse(bad)


def test_slice_size_forms(p2g):
    f = p2g.parse_slice_size
    assert f("4096") == 4096 and f("768000") == 768000
    assert f("768000b") == 768000 and f("768000B") == 768000
    assert f("750K") == 750 * 1024 and f("750k") == 750 * 1024
    assert f("1M") == 1 << 20 and f("1m") == 1 << 20
    assert f("2G") == 2 << 30 and f("2g") == 2 << 30


@pytest.mark.parametrize("bad", ["", "b", "K", "abc", "12x", "-5", "99999999999G"])
def test_slice_size_rejects_bad_input_and_overflow(p2g, bad):
    with pytest.raises(p2g.InvalidArgument):
        p2g.parse_slice_size(bad)


def test_resolves_percent_and_target_bytes(p2g):
    R = p2g.Redundancy
    assert p2g.resolve_redundancy(R(percent=10), 100, 4096) == 10
    assert p2g.resolve_redundancy(R(percent=10), 33, 4096) == 4  # ceil(3.3)
    assert p2g.resolve_redundancy(R(target_bytes=8192), 100, 4096) == 2
    assert p2g.resolve_redundancy(R(target_bytes=8193), 100, 4096) == 3


def test_resolve_rejects_zero_result(p2g):
    with pytest.raises(p2g.InvalidVolumeScheme):
        p2g.resolve_redundancy(p2g.Redundancy(percent=0), 1, 4096)


def test_volume_scheme_flags(p2g):
    V, b = p2g.VolumeScheme, p2g.build_volume_scheme
    assert b() == V.Exponential()
    assert b(single_volume=True) == V.Single()
    assert b(uniform=True, recovery_count=40) == V.Uniform(15)   # default count clamp(R, 1, 15)
    assert b(uniform=True, recovery_count=0) == V.Uniform(1)
    assert b(uniform=True, recovery_count=7) == V.Uniform(7)
    assert b(uniform=True, volume_count=3, recovery_count=40) == V.Uniform(3)
    lim = b(limit_size=True, largest_source_length=10 * 4096 + 5, slice_size=4096)
    assert lim.kind == 3 and lim.max_blocks_per_volume == 10 and lim.inner == V.Exponential()
    lim = b(uniform=True, limit_size=True, largest_source_length=100, slice_size=4096, recovery_count=4)
    assert lim.max_blocks_per_volume == 1 and lim.inner == V.Uniform(4)   # cap at least 1
    for bad in [dict(single_volume=True, uniform=True), dict(single_volume=True, limit_size=True),
                dict(single_volume=True, volume_count=2), dict(volume_count=2),
                dict(limit_size=True, largest_source_length=0)]:
        with pytest.raises(p2g.InvalidVolumeScheme):
            b(**bad)


def _cli(p2g, args, cwd, **kw):
    return subprocess.run([p2g.CLI_PATH, *args], cwd=cwd, capture_output=True, text=True, timeout=300, **kw)


def test_cli_errors_before_any_device_work(p2g, tmp_path):
    (tmp_path / "sub").mkdir()
    (tmp_path / "sub" / "a.bin").write_bytes(b"x" * 100)
    r = _cli(p2g, ["create"], tmp_path)
    assert r.returncode == 1 and "missing output archive" in r.stderr
    r = _cli(p2g, ["create", "-q", "out.par2", "sub"], tmp_path)
    assert r.returncode == 1 and "is a directory; pass --recurse" in r.stderr
    r = _cli(p2g, ["c", "out.par2", "nope.bin"], tmp_path)
    assert r.returncode == 1 and r.stderr.startswith("par2rust: error: I/O error:")
    r = _cli(p2g, ["create", "-c", "3", "-r", "10", "out.par2", "sub/a.bin"], tmp_path)
    assert r.returncode == 2 and "cannot be used with" in r.stderr
    r = _cli(p2g, ["create", "-s", "12x", "out.par2", "sub/a.bin"], tmp_path)
    assert r.returncode == 2 and "invalid number" in r.stderr
    r = _cli(p2g, ["create", "out.par2", "-i", "missing.txt"], tmp_path)
    assert r.returncode == 1 and "I/O error" in r.stderr
    assert not list(tmp_path.glob("*.par2"))


# ---- whole creates through the executable (GPU) ----------------------------
def _want(oracle, files, slice_, R, kind, count=0, cap=0, inner=None, comments=(), index="out.par2"):
    return oracle.create(files, slice_, R, kind=kind, count=count, cap=cap, inner=inner, comments=comments,
                         index_path=index)


def _check_dir(tmp_path, want):
    for name, data in want:
        got = (tmp_path / name).read_bytes()
        assert got == data, name


@pytest.mark.gpu
def test_cli_single_volume_and_out_flag(p2g, gpu, oracle, tmp_path):
    data = deterministic_bytes(0xABCD1234, 32 * 1024)
    (tmp_path / "doc.bin").write_bytes(data)
    r = _cli(p2g, ["create", "--single-volume", "-s", "4096", "-c", "5", "backup.par2", "doc.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    vols = sorted(p.name for p in tmp_path.glob("*.vol*"))
    assert vols == ["backup.vol0+5.par2"]
    assert r.stdout.startswith("Wrote 2 files:")
    _check_dir(tmp_path, _want(oracle, [(b"doc.bin", data)], 4096, 5, oracle.SCHEME_SINGLE, index="backup.par2"))
    r = _cli(p2g, ["create", "--out", "via-out.par2", "--quiet", "-c", "3", "doc.bin"], tmp_path)
    assert r.returncode == 0 and r.stdout == "" and (tmp_path / "via-out.par2").exists()
    _check_dir(tmp_path, _want(oracle, [(b"doc.bin", data)], 4096, 3, oracle.SCHEME_EXPONENTIAL, index="via-out.par2"))


@pytest.mark.gpu
def test_cli_comments_recurse_and_input_file(p2g, gpu, oracle, tmp_path):
    (tmp_path / "doc.bin").write_bytes(deterministic_bytes(7, 8192))
    r = _cli(p2g, ["create", "--comment", "hello from par2rust", "--comment", "second note", "--quiet",
                   "with-comments.par2", "doc.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "with-comments.par2").read_bytes().count(b"PAR 2.0\0CommASCI") == 2
    sub = tmp_path / "subdir"
    sub.mkdir()
    (sub / "a.bin").write_bytes(deterministic_bytes(1, 512))
    (sub / "b.bin").write_bytes(deterministic_bytes(2, 512))
    r = _cli(p2g, ["create", "--recurse", "--quiet", "-s", "256", "-c", "2", "recurse.par2", "subdir"], tmp_path)
    assert r.returncode == 0, r.stderr
    idx = (tmp_path / "recurse.par2").read_bytes()
    assert idx.count(b"PAR 2.0\0FileDesc") == 2
    (tmp_path / "inputs.txt").write_text("# listed inputs\nsubdir/a.bin\n\nsubdir/b.bin\n")
    r = _cli(p2g, ["create", "--input-file", "inputs.txt", "--quiet", "-s", "256", "-c", "2", "listed.par2"], tmp_path)
    assert r.returncode == 0, r.stderr
    files = [(b"a.bin", (sub / "a.bin").read_bytes()), (b"b.bin", (sub / "b.bin").read_bytes())]
    _check_dir(tmp_path, _want(oracle, files, 256, 2, oracle.SCHEME_EXPONENTIAL, index="listed.par2"))


@pytest.mark.gpu
def test_cli_redundancy_uniform_and_limit(p2g, gpu, oracle, tmp_path):
    a = deterministic_bytes(11, 70_001)
    b = deterministic_bytes(12, 9_000)
    (tmp_path / "a.bin").write_bytes(a)
    (tmp_path / "b.bin").write_bytes(b)
    files = [(b"a.bin", a), (b"b.bin", b)]
    S = (70_001 + 4095) // 4096 + (9_000 + 4095) // 4096   # 18 + 3
    # -r 25 -> ceil(21 * 25 / 100) = 6 recovery blocks, exponential volumes
    r = _cli(p2g, ["create", "-q", "-r", "25", "pct.par2", "a.bin", "b.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    _check_dir(tmp_path, _want(oracle, files, 4096, -(-S * 25 // 100), oracle.SCHEME_EXPONENTIAL, index="pct.par2"))
    # -rk20 -> ceil(20480 / 4096) = 5 blocks; -u -n 2 -> two uniform volumes
    r = _cli(p2g, ["create", "-q", "-rk20", "-u", "-n", "2", "uni.par2", "a.bin", "b.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    _check_dir(tmp_path, _want(oracle, files, 4096, 5, oracle.SCHEME_UNIFORM, count=2, index="uni.par2"))
    # -l caps each volume at largest / slice = 17 blocks (inner exponential)
    r = _cli(p2g, ["create", "-q", "-c", "40", "-l", "lim.par2", "a.bin", "b.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    _check_dir(tmp_path, _want(oracle, files, 4096, 40, oracle.SCHEME_LIMITED, cap=70_001 // 4096,
                               inner=(oracle.SCHEME_EXPONENTIAL,), index="lim.par2"))
