"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Everything here is integer / byte work, so the bar is bit-exact equality:
recovery slices, MD5 digests, CRC32 values and whole .par2 files.
"""
import hashlib
import os
import zlib

import numpy as np
import pytest

from par2rust_b200.workloads import deterministic_bytes, file_bytes

pytestmark = pytest.mark.gpu


def rnd(seed, n):
    return np.frombuffer(file_bytes(seed * 7919 + 17, n).tobytes(), dtype=np.uint8).copy()


# ---- kernel level ----------------------------------------------------------
@pytest.mark.parametrize("coeff", [0x0000, 0x0001, 0x0002, 0x00FF, 0x0100, 0x1234, 0x8000, 0xABCD, 0xFFFE, 0xFFFF])
def test_gf_mul_xor_matches_scalar(p2g, oracle, gpu, coeff):
    for ln in [2, 4, 16, 30, 32, 34, 62, 64, 96, 100, 1024, 4096, 4098, 65538]:
        inp = deterministic_bytes((coeff << 13) ^ ln, ln)
        init = deterministic_bytes(ln + 5, ln)
        a, b = bytearray(init), bytearray(init)
        oracle.gf_mul_xor_scalar(coeff, inp, a)
        p2g.gf_mul_xor(coeff, inp, b)
        assert a == b, (hex(coeff), ln)


ENC_SHAPES = [
    (1, 4, 1), (2, 16, 1), (3, 64, 5), (5, 4096, 33), (4, 20, 3), (7, 132, 40), (2, 4100, 65),
    (10, 65536, 64), (3, 8192, 200), (9, 2048 * 4 + 16, 31), (33, 256, 97), (1, 8, 300),
]


@pytest.mark.parametrize("S,slice_,R", ENC_SHAPES)
def test_encode_matches_oracle(p2g, oracle, gpu, S, slice_, R):
    src = rnd(S * 1000 + R, S * slice_)
    want = oracle.encode(src, S, slice_, R)
    got = p2g.encode(src, slice_, R)
    assert (want == got).all()


@pytest.mark.parametrize("S,slice_,R", [(5, 4096, 33), (7, 132, 40), (2, 4100, 65), (33, 256, 97), (9, 8208, 31)])
def test_encode_basis_loaded_or_derived_agree(p2g, oracle, gpu, monkeypatch, S, slice_, R):
    # the encode loads a precomputed coefficient basis by default; the kernel
    # that derives it itself (P2G_ENCODE_BASIS=derive) must give the same rows
    src = rnd(S * 7 + R, S * slice_)
    want = oracle.encode(src, S, slice_, R)
    got_load = p2g.encode(src, slice_, R)
    monkeypatch.setenv("P2G_ENCODE_BASIS", "derive")
    got_gen = p2g.encode(src, slice_, R)
    assert (want == got_gen).all() and (want == got_load).all()


@pytest.mark.parametrize("first", [0, 5, 40000, 65496])
def test_encode_first_exponent(p2g, oracle, gpu, monkeypatch, first):
    """c(r,s) = base_s^(first_exponent + r) up to the largest exponent, 65535
    (where base^65535 = 1: the field's multiplicative order); both basis
    modes against gf_pow/gf_mul.  Exponents past 65535 are refused."""
    S, slice_, R = 3, 64, 40
    with pytest.raises(p2g.TooManyRecoveryBlocks):
        p2g.encode(rnd(1, S * slice_), slice_, R, first_exponent=65536 - R + 1)
    src = rnd(77 + first % 1000, S * slice_)
    sym = src.view("<u2").reshape(S, slice_ // 2)
    bases = oracle.input_bases(S)
    want = np.zeros((R, slice_ // 2), np.uint16)
    for r in range(R):
        cs = [oracle.gf_pow(bases[s], first + r) for s in range(S)]
        for k in range(slice_ // 2):
            v = 0
            for s in range(S):
                v ^= oracle.gf_mul(cs[s], int(sym[s, k]))
            want[r, k] = v
    got_load = p2g.encode(src, slice_, R, first_exponent=first).view("<u2").reshape(R, -1)
    monkeypatch.setenv("P2G_ENCODE_BASIS", "derive")
    got_gen = p2g.encode(src, slice_, R, first_exponent=first).view("<u2").reshape(R, -1)
    assert (got_load == want).all() and (got_gen == want).all()


def test_encode_zero_source_gives_zero(p2g, gpu):
    assert not p2g.encode(np.zeros(4 * 1024, np.uint8), 1024, 70).any()


def test_encode_linearity(p2g, gpu):
    S, slice_, R = 6, 4096, 45
    a, b = rnd(1, S * slice_), rnd(2, S * slice_)
    ea, eb, eab = p2g.encode(a, slice_, R), p2g.encode(b, slice_, R), p2g.encode(a ^ b, slice_, R)
    assert ((ea ^ eb) == eab).all()


def test_encode_device_pointers_matches_host(p2g, gpu):
    import torch

    S, slice_, R = 12, 8192, 70
    src = rnd(3, S * slice_)
    want = p2g.encode(src, slice_, R)
    d_src = torch.from_numpy(src).cuda()
    d_rec = torch.zeros(R * slice_, dtype=torch.uint8, device="cuda")
    p2g.encode_device(d_src.data_ptr(), slice_, S, slice_, R, d_rec.data_ptr(), slice_,
                      torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert (d_rec.cpu().numpy() == want).all()


@pytest.mark.parametrize("slice_", [4, 8, 20, 64, 68, 100, 4096, 4100, 65536])
def test_slice_checksums(p2g, gpu, slice_):
    n = 37
    src = rnd(slice_, n * slice_)
    got = p2g.slice_checksums(src, slice_)
    for i in range(n):
        d = src[i * slice_:(i + 1) * slice_].tobytes()
        assert got[i].md5 == hashlib.md5(d).digest()
        assert got[i].crc32 == zlib.crc32(d)


def test_file_hashes(p2g, gpu):
    lens = [1, 3, 55, 56, 63, 64, 65, 119, 120, 1000, 16383, 16384, 16385, 100000, 1 << 20]
    bufs = [rnd(n, n).tobytes() for n in lens]
    got = p2g.file_hashes(bufs)
    for b, (hf, h16) in zip(bufs, got):
        assert hf == hashlib.md5(b).digest()
        assert h16 == hashlib.md5(b[:16384]).digest()


@pytest.mark.parametrize("slice_", [4, 28, 64, 100, 4096, 65540])
def test_recovery_packet_md5(p2g, gpu, slice_):
    R = 9
    rec = rnd(slice_ + 1, R * slice_)
    set_id = bytes(range(16))
    got = p2g.recovery_packet_md5(set_id, rec, slice_, R, first_exponent=3)
    for r in range(R):
        body = (3 + r).to_bytes(4, "little") + rec[r * slice_:(r + 1) * slice_].tobytes()
        assert got[r] == hashlib.md5(set_id + b"PAR 2.0\0RecvSlic" + body).digest()


# ---- whole create, in memory ---------------------------------------------------
def _scheme(p2g, oracle, name, count=0, sizes=None):
    VS = p2g.VolumeScheme
    if name == "single":
        return VS.Single(), dict(kind=oracle.SCHEME_SINGLE)
    if name == "exponential":
        return VS.Exponential(), dict(kind=oracle.SCHEME_EXPONENTIAL)
    if name == "uniform":
        return VS.Uniform(count), dict(kind=oracle.SCHEME_UNIFORM, count=count)
    if name == "explicit":
        return VS.Explicit(sizes), dict(kind=oracle.SCHEME_EXPLICIT, sizes=sizes)
    if name == "limited":
        return VS.Limited(count, VS.Exponential()), dict(kind=oracle.SCHEME_LIMITED, cap=count,
                                                         inner=(oracle.SCHEME_EXPONENTIAL,))
    raise ValueError(name)


PAYLOAD = bytes(((i * 101) & 0xFF) for i in range(17 * 1024 + 37))
CREATE_CASES = [
    ("hello", [(b"a.bin", b"hello par2 world!!!!")], 4, 2, "single", 0, None, []),
    ("payload-single", [(b"p.bin", PAYLOAD)], 4096, 4, "single", 0, None, []),
    ("payload-exp", [(b"p.bin", PAYLOAD)], 4096, 11, "exponential", 0, None, []),
    ("payload-index", [(b"p.bin", PAYLOAD)], 4096, 0, "single", 0, None, []),
    ("multi-uniform", [(b"one", rnd(1, 5000).tobytes()), (b"two.dat", rnd(2, 300).tobytes()),
                       (b"three", rnd(3, 12288).tobytes())], 1024, 7, "uniform", 3, None, ["a comment"]),
    ("explicit-unicode", [(b"x", rnd(4, 20000).tobytes())], 2048, 6, "explicit", 0, [2, 3, 1], ["trés", "ok"]),
    ("limited", [(b"y", rnd(5, 9000).tobytes())], 512, 20, "limited", 3, None, []),
    ("odd-slice", [(b"z", rnd(6, 1001).tobytes()), (b"w", rnd(7, 77).tobytes())], 20, 37, "single", 0, None, []),
    # the limits: 32,768 input slices; 65,535 recovery blocks; thousands of files
    ("max-input-slices", [(b"maxs.bin", rnd(8, 131072).tobytes())], 4, 3, "single", 0, None, []),
    ("max-recovery", [(b"maxr.bin", rnd(9, 40).tobytes())], 4, 65535, "exponential", 0, None, []),
    ("many-files", [(f"f{i:04d}.dat".encode(), rnd(100 + i, 1 + (i * 37) % 200).tobytes()) for i in range(3000)],
     64, 10, "uniform", 4, None, []),
]


@pytest.mark.parametrize("case", CREATE_CASES, ids=[c[0] for c in CREATE_CASES])
def test_create_in_memory_bit_exact(p2g, oracle, gpu, case):
    _, inputs, slice_, R, scheme, count, sizes, comments = case
    vs, okw = _scheme(p2g, oracle, scheme, count, sizes)
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=slice_, recovery_block_count=R, volume_scheme=vs,
                             comments=comments)
    got, srcs = p2g.create_in_memory(opts, [(n, d) for n, d in inputs], return_sources=True)
    want = oracle.create([(n, d) for n, d in inputs], slice_, R, comments=comments, **okw)
    assert [n for n, _ in got] == [n for n, _ in want]
    for (n, a), (_, b) in zip(got, want):
        assert a == b, n
    for (name, data), sf in zip(inputs, srcs):
        st, cks, hf, h16, fid = oracle.scan(data, slice_, name)
        assert sf.hash_full == hf and sf.hash16k == h16 and sf.file_id == fid
        assert [(c.md5, c.crc32) for c in sf.slice_checksums] == cks


@pytest.mark.parametrize("case", CREATE_CASES[:3], ids=[c[0] for c in CREATE_CASES[:3]])
def test_create_in_memory_views_equal_copies(p2g, oracle, gpu, case):
    """copy=False hands out views of the library's buffers; they must hold
    the same bytes as the copies and stay valid after the call returns."""
    _, inputs, slice_, R, scheme, count, sizes, comments = case
    vs, _ = _scheme(p2g, oracle, scheme, count, sizes)
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=slice_, recovery_block_count=R, volume_scheme=vs,
                             comments=comments)
    copies = p2g.create_in_memory(opts, [(n, d) for n, d in inputs])
    views = p2g.create_in_memory(opts, [(n, d) for n, d in inputs], copy=False)
    p2g.create_in_memory(opts, [(n, d) for n, d in inputs], copy=False)  # a later call must not disturb them
    assert [n for n, _ in views] == [n for n, _ in copies]
    for (n, v), (_, b) in zip(views, copies):
        assert isinstance(v, memoryview) and v.readonly
        assert v.tobytes() == b, n
    del copies
    assert views[-1][1].tobytes()[:8] == b"PAR2\0PKT"


@pytest.mark.parametrize("n_slices,R", [(3, 40), (2, 200), (5, 7)])
def test_banded_encode_and_packet_md5(p2g, oracle, gpu, n_slices, R):
    """Large slices split the encode into symbol bands and chain the packet
    MD5 band by band; the files must still match the oracle byte for byte."""
    slice_ = 524288
    data = file_bytes(n_slices * 31 + R, n_slices * slice_ - 1000).tobytes()
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=slice_, recovery_block_count=R,
                             volume_scheme=p2g.VolumeScheme.Exponential())
    got = p2g.create_in_memory(opts, [(b"band.bin", data)])
    want = oracle.create([(b"band.bin", data)], slice_, R, kind=oracle.SCHEME_EXPONENTIAL)
    assert [n for n, _ in got] == [n for n, _ in want]
    assert all(a == b for (_, a), (_, b) in zip(got, want))


@pytest.mark.parametrize("slice_,S,R", [(65540, 100, 30), (132, 3000, 200), (4100, 600, 100), (20004, 800, 40)])
def test_split_tail_with_realigned_slices(p2g, oracle, gpu, slice_, S, R):
    """Slice sizes that are not multiples of 16 (the encode reads a
    realigned copy) in jobs whose planner cuts encode items into
    XOR-accumulating slice ranges: every output byte against the oracle."""
    data = file_bytes(slice_ + S, slice_ * S - 7).tobytes()
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=slice_, recovery_block_count=R,
                             volume_scheme=p2g.VolumeScheme.Exponential())
    got = p2g.create_in_memory(opts, [(b"x.bin", data)])
    want = oracle.create([(b"x.bin", data)], slice_, R, kind=oracle.SCHEME_EXPONENTIAL)
    assert [n for n, _ in got] == [n for n, _ in want]
    assert all(a == b for (_, a), (_, b) in zip(got, want))


@pytest.mark.parametrize("slice_,S,R", [(4100, 600, 100), (65536, 64, 40)])
def test_device_job_writes_nothing_past_the_row(p2g, oracle, gpu, slice_, S, R):
    """A caller's recovery stride wider than the padded row: the job (tail
    split, zeroed columns, accumulating items) leaves the bytes past the
    padded row untouched and the rows equal to the oracle's."""
    import torch

    L = slice_ * S - 11
    host = np.zeros(S * slice_, np.uint8)
    host[:L] = np.frombuffer(file_bytes(S + R, L).tobytes(), np.uint8)
    src = torch.from_numpy(host).cuda()
    bufs = p2g.DeviceJobBuffers(S, 1, slice_, R, src.device)
    padded = (slice_ + 15) // 16 * 16
    stride = padded + 64
    bufs.recovery = torch.full((R * stride,), 0xA5, dtype=torch.uint8, device=src.device)
    bufs.rec_stride = stride
    p2g.run_device_job(src, [L], [b"x.bin"], slice_, R, bufs)
    torch.cuda.synchronize()
    rows = bufs.recovery.view(R, stride).cpu().numpy()
    assert (rows[:, padded:] == 0xA5).all()
    want = np.asarray(oracle.encode(host, S, slice_, R)).reshape(R, slice_)
    assert (rows[:, :slice_] == want).all()


def test_single_16m_bit_exact(p2g, oracle, gpu):
    """16,777,216 B, slice 65,536, R 32, Single: every output byte vs the oracle."""
    data = file_bytes(0x16, 16_777_216)
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=65536, recovery_block_count=32)
    got = p2g.create_in_memory(opts, [(b"source.bin", data)])
    want = oracle.create([(b"source.bin", data)], 65536, 32)
    assert [n for n, _ in got] == [n for n, _ in want]
    assert all(a == b for (_, a), (_, b) in zip(got, want))


def test_bounded_wait_gives_up_and_device_stays_usable(p2g, oracle, gpu):
    """A device wait that can never complete must end in DeviceTimeout (the
    status a job gets when a copy never lands), not a hang, and the next
    create on the same device must still be bit-exact."""
    import time

    for polls in (1, 1 << 12, 1 << 16):
        t0 = time.time()
        with pytest.raises(p2g.DeviceTimeout):
            p2g.check_bounded_wait(polls)
        assert time.time() - t0 < 30
    with pytest.raises(p2g.InvalidArgument):
        p2g.check_bounded_wait(0)
    data = file_bytes(0xB0D, 50_000).tobytes()
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=1024, recovery_block_count=9)
    got = p2g.create_in_memory(opts, [(b"after.bin", data)])
    want = oracle.create([(b"after.bin", data)], 1024, 9)
    assert [n for n, _ in got] == [n for n, _ in want]
    assert all(a == b for (_, a), (_, b) in zip(got, want))


# ---- filesystem entry points -------------------------------------------------
class Capture:
    def __init__(self):
        self.events = []

    def on_event(self, e):
        self.events.append(e)


def test_run_create_scan_fused_agree(p2g, oracle, gpu, tmp_path):
    d1, d2 = tmp_path / "legacy", tmp_path / "fused"
    d1.mkdir()
    d2.mkdir()
    (d1 / "p.bin").write_bytes(PAYLOAD)
    (d2 / "p.bin").write_bytes(PAYLOAD)
    for scheme, R in [(p2g.VolumeScheme.Single(), 4), (p2g.VolumeScheme.Exponential(), 11), (p2g.VolumeScheme.Single(), 0)]:
        src = p2g.SourceFile.scan(d1 / "p.bin", b"p.bin", 4096)
        o1 = p2g.CreateOptions(output=d1 / "recovery.par2", slice_size=4096, recovery_block_count=R, volume_scheme=scheme)
        o2 = p2g.CreateOptions(output=d2 / "recovery.par2", slice_size=4096, recovery_block_count=R, volume_scheme=scheme)
        f1 = p2g.run_create(o1, [src])
        f2 = p2g.run_create_fused(o2, [(d2 / "p.bin", b"p.bin")])
        assert len(f1) == len(f2)
        want = oracle.create([(b"p.bin", PAYLOAD)], 4096, R,
                             kind=oracle.SCHEME_EXPONENTIAL if isinstance(scheme, type(p2g.VolumeScheme.Exponential())) else 0,
                             index_path=str(d1 / "recovery.par2"))
        assert [str(p) for p in f1] == [n for n, _ in want]
        for a, b, (_, w) in zip(f1, f2, want):
            assert a.read_bytes() == b.read_bytes() == w
        assert not list(d1.glob("*.tmp")) and not list(d2.glob("*.tmp"))


def test_encode_progress_from_device_counter(p2g, gpu, tmp_path):
    """run_create_with_progress reports encode progress while the device
    works: ENCODE_PROGRESS events between STARTED and COMPLETED with input
    blocks done strictly rising, below the total until the last one."""
    n, slice_, R = 96 << 20, 65536, 1000
    (tmp_path / "big.bin").write_bytes(file_bytes(0xE7, n).tobytes())
    src = p2g.SourceFile.scan(tmp_path / "big.bin", b"big.bin", slice_)
    S = len(src.slice_checksums)
    cap = Capture()
    opts = p2g.CreateOptions(output=tmp_path / "recovery.par2", slice_size=slice_, recovery_block_count=R,
                             volume_scheme=p2g.VolumeScheme.Uniform(4))
    p2g.run_create_with_progress(opts, [src], cap)
    kinds = [e.kind for e in cap.events]
    a, b = kinds.index("EncodeStarted"), kinds.index("EncodeCompleted")
    prog = [e.input_block_done for e in cap.events[a:b] if e.kind == "EncodeProgress"]
    assert all(e.kind == "EncodeProgress" for e in cap.events[a + 1:b])
    assert prog[-1] == S and all(x < y for x, y in zip(prog, prog[1:]))
    assert len(prog) >= 3, prog  # the job runs for milliseconds: the counter is read several times


def test_scan_matches_oracle(p2g, oracle, gpu, tmp_path):
    for n, slice_ in [(5, 4), (17, 8), (16384 + 100, 4096), (4096 * 16, 16), (1, 4)]:
        data = bytes(((i * 0x9E37) >> 5) & 0xFF for i in range(n))
        (tmp_path / "f").write_bytes(data)
        sf = p2g.SourceFile.scan(tmp_path / "f", b"file.bin", slice_)
        st, cks, hf, h16, fid = oracle.scan(data, slice_, b"file.bin")
        assert sf.length == n and sf.hash_full == hf and sf.hash16k == h16 and sf.file_id == fid
        assert [(c.md5, c.crc32) for c in sf.slice_checksums] == cks


def test_scan_errors(p2g, gpu, tmp_path):
    (tmp_path / "e").write_bytes(b"")
    (tmp_path / "h").write_bytes(b"hi")
    with pytest.raises(p2g.EmptyFile):
        p2g.SourceFile.scan(tmp_path / "e", b"x", 4)
    with pytest.raises(p2g.InvalidSliceSize):
        p2g.SourceFile.scan(tmp_path / "h", b"x", 0)
    with pytest.raises(p2g.InvalidSliceSize):
        p2g.SourceFile.scan(tmp_path / "h", b"x", 5)
    with pytest.raises(p2g.InvalidFileName):
        p2g.SourceFile.scan(tmp_path / "h", b"", 4)
    with pytest.raises(p2g.InvalidFileName):
        p2g.SourceFile.scan(tmp_path / "h", b"bad\0name", 4)
    with pytest.raises(p2g.IoError):
        p2g.SourceFile.scan(tmp_path / "missing", b"x", 4)


def test_fused_create_volume_failure_leaves_no_temp_files(p2g, gpu, tmp_path):
    """A volume whose temp file cannot be created (a directory sits at its
    name) fails the fused create with IoError; the volumes written early
    while the file hashed are removed, and no temp file is left behind."""
    data = file_bytes(0xF1, 300_000).tobytes()
    (tmp_path / "in.bin").write_bytes(data)
    out = tmp_path / "recovery.par2"
    first_vol = p2g.volume_filename(str(out), 0, 1)
    (tmp_path / (os.path.basename(first_vol) + ".par2rust.tmp")).mkdir()
    opts = p2g.CreateOptions(output=out, slice_size=4096, recovery_block_count=11,
                             volume_scheme=p2g.VolumeScheme.Exponential())
    with pytest.raises(p2g.IoError):
        p2g.run_create_fused(opts, [(tmp_path / "in.bin", b"in.bin")])
    assert [p for p in tmp_path.glob("*.par2rust.tmp") if p.is_file()] == []
    assert not os.path.exists(first_vol)


def test_create_errors(p2g, gpu, tmp_path):
    (tmp_path / "a.bin").write_bytes(b"x")
    src = p2g.SourceFile.scan(tmp_path / "a.bin", b"a.bin", 4)
    with pytest.raises(p2g.NoInputFiles):
        p2g.run_create(p2g.CreateOptions(output=tmp_path / "r.par2", slice_size=4), [])
    with pytest.raises(p2g.TooManyRecoveryBlocks):
        p2g.run_create(p2g.CreateOptions(output=tmp_path / "r.par2", slice_size=4, recovery_block_count=65536), [src])
    fake = p2g.SourceFile(name=b"big.bin", path=tmp_path / "big.bin", length=32769 * 4, hash_full=b"\0" * 16,
                          hash16k=b"\0" * 16, file_id=b"\0" * 16,
                          slice_checksums=[p2g.SliceChecksum(b"\0" * 16, 0)] * 32769)
    with pytest.raises(p2g.TooManyInputBlocks) as ei:
        p2g.run_create(p2g.CreateOptions(output=tmp_path / "r.par2", slice_size=4, recovery_block_count=1), [fake])
    assert ei.value.count == 32769 and ei.value.slice_size == 4 and ei.value.suggested > 4 and ei.value.suggested % 4 == 0
    (tmp_path / "w.bin").write_bytes(b"hello par2 world!!!!")
    s2 = p2g.SourceFile.scan(tmp_path / "w.bin", b"w.bin", 4)
    with pytest.raises(p2g.InvalidVolumeScheme):
        p2g.run_create(p2g.CreateOptions(output=tmp_path / "v.par2", slice_size=4, recovery_block_count=5,
                                         volume_scheme=p2g.VolumeScheme.Explicit([2, 2])), [s2])


def test_progress_events_order(p2g, gpu, tmp_path):
    """progress_events_fire_in_order_for_create_with_recovery, src/creator.rs:1720-1812"""
    (tmp_path / "a.bin").write_bytes(b"hello par2 world!!!!")
    rep = Capture()
    src = p2g.SourceFile.scan_with_progress(tmp_path / "a.bin", b"a.bin", 4, rep)
    files = p2g.run_create_with_progress(
        p2g.CreateOptions(output=tmp_path / "recovery.par2", slice_size=4, recovery_block_count=2), [src], rep)
    assert len(files) == 2
    k = [e.kind for e in rep.events]
    first_encode, first_index, first_volume = k.index("EncodeStarted"), k.index("IndexWritten"), k.index("VolumeWritten")
    last_encode_end = len(k) - 1 - k[::-1].index("EncodeCompleted")
    assert first_encode > 0 and first_index < first_encode and first_volume > last_encode_end
    enc = [e for e in rep.events if e.kind == "EncodeProgress"][-1]
    assert enc.input_block_done == enc.input_blocks == 5
    scn = [e for e in rep.events if e.kind == "ScanProgress"][-1]
    assert scn.slices_done == scn.total_slices == 5
    assert k.count("EncodeStarted") == 1 and k.count("EncodeCompleted") == 1


def test_write_index_file(p2g, gpu, tmp_path):
    (tmp_path / "a.bin").write_bytes(b"hello par2")
    src = p2g.SourceFile.scan(tmp_path / "a.bin", b"a.bin", 4)
    out = p2g.write_index_file(p2g.CreateOptions(output=tmp_path / "recovery.par2", slice_size=4), [src])
    assert out == tmp_path / "recovery.par2" and out.exists()


# ---- the two device-job pipelines ---------------------------------------------
# Jobs run as one persistent launch by default; the multi-stream banded
# pipeline (P2G_BANDED, and jobs whose whole-file MD5 is on the device) must
# give the same bytes: folded and unfolded tail groups, realigned slices,
# several files, > 256 recovery rows.
@pytest.mark.parametrize("lens,slice_,R", [
    ([300_001], 4096, 48), ([5000, 70000, 1], 1024, 300), ([9000, 4100 * 3], 4100, 7),
    ([2_000_000, 17], 16384, 70), ([1_100_000], 65536, 33),
])
def test_device_job_persistent_equals_banded(p2g, gpu, monkeypatch, lens, slice_, R):
    import torch

    S = sum((n + slice_ - 1) // slice_ for n in lens)
    host = np.zeros(S * slice_, np.uint8)
    off = 0
    for i, n in enumerate(lens):
        host[off:off + n] = rnd(i + 3 * R, n)
        off += (n + slice_ - 1) // slice_ * slice_
    src = torch.from_numpy(host).cuda()
    names = [f"f{i}.bin".encode() for i in range(len(lens))]

    def run():
        # whole-file MD5 on the device too (file-hash items / the banded pipeline's file kernel)
        b = p2g.run_device_job(src, lens, names, slice_, R, skip_hash_full=False)
        torch.cuda.synchronize()
        rows = b.recovery.view(-1, b.rec_stride)[:R, :slice_].cpu().numpy().copy()
        return (rows, b.checksums[:20 * S].cpu().numpy().copy(), b.hash16k[:16 * len(lens)].cpu().numpy().copy(),
                b.packet_md5[:16 * R].cpu().numpy().copy(), b.set_id, b.hash_full[:16 * len(lens)].cpu().numpy().copy())

    persistent = run()
    monkeypatch.setenv("P2G_BANDED", "1")
    banded = run()
    for k, (x, y) in enumerate(zip(persistent, banded)):
        assert (np.asarray(x) == np.asarray(y)).all() if not isinstance(x, bytes) else x == y, k
    off = 0
    for i, n in enumerate(lens):  # hash_full against hashlib
        assert persistent[5][16 * i:16 * i + 16].tobytes() == hashlib.md5(host[off:off + n].tobytes()).digest(), i
        off += (n + slice_ - 1) // slice_ * slice_



def test_create_in_memory_pinned_inputs_equal_pageable(p2g, oracle, gpu):
    """Many page-locked inputs are uploaded by one kernel that reads them
    over the bus: odd lengths, slice tails to zero, pointers at odd offsets
    inside a pinned allocation, and files of several 4 MiB segments give the
    same bytes as the same inputs from pageable memory, and as the oracle."""
    import torch

    rng = np.random.default_rng(21)
    lens = [int(x) for x in rng.integers(1, 300_000, size=30)] + [9 * 1024 * 1024 + 13, 65536, 1]
    pool = torch.empty(sum(lens) + 64 * len(lens), dtype=torch.uint8, pin_memory=True)
    pinned, pageable, off = [], [], 0
    for i, n in enumerate(lens):
        off += 1 + (i % 7)  # odd offsets: the copy takes its byte path there
        data = rnd(500 + i, n)
        view = pool[off:off + n]
        view.numpy()[:] = data
        pinned.append((f"p{i:02d}.bin".encode(), view))
        pageable.append((f"p{i:02d}.bin".encode(), data.tobytes()))
        off += n
    opts = p2g.CreateOptions(output="pin.par2", slice_size=65536, recovery_block_count=12,
                             volume_scheme=p2g.VolumeScheme.Uniform(3))
    a = p2g.create_in_memory(opts, pinned)
    b = p2g.create_in_memory(opts, pageable)
    assert [n for n, _ in a] == [n for n, _ in b]
    for (n, x), (_, y) in zip(a, b):
        assert x == y, n
    want = oracle.create([(n, d) for n, d in pageable], 65536, 12, kind=oracle.SCHEME_UNIFORM, count=3,
                         index_path="pin.par2")
    for (n, x), (m, y) in zip(a, want):
        assert n == m and x == y, n
