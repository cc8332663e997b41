"""Batched create: many jobs in one persistent, graph-captured launch.

GPU tests compare every output of every job in a heterogeneous batch with
the oracle (recovery rows, slice MD5/CRC32, hash16k, set id, packet MD5s),
with the plain per-job device path, and with the same job batched alone:
results must be byte-identical however the job is mixed.  CPU tests cover
the planner (items, tile search, predicted makespan).
"""
import math

import numpy as np
import pytest

from par2rust_b200.workloads import file_bytes


def _tail_fold(R):
    tail = R - (R - 1) // 32 * 32
    return 4 if tail <= 8 else 2 if tail <= 16 else 1


def _shape_items(slice_, S, R):
    """(scan + CRC, encode, set-id) item counts at the widest tiles: the last
    row group is folded over `fold` tiles inside each band of up to 64 bands."""
    Np = (slice_ + 15) // 16 * 16 // 2
    tiles = math.ceil(Np / 2048)
    enc = 0
    if R:
        F = _tail_fold(R)
        bt = max(1, math.ceil(tiles / 64))
        bt = math.ceil(bt / F) * F
        for t0 in range(0, tiles, bt):
            n = min(tiles, t0 + bt) - t0
            enc += n * (math.ceil(R / 32) - 1) + math.ceil(n / F)
    crc_per_item = min(256, max(1, (4 << 20) // slice_))  # CRC items of ~4 MiB
    return math.ceil(S / 256) + math.ceil(S / crc_per_item), enc, 1


# ---- planner (CPU) -----------------------------------------------------------
def test_plan_counts_items(p2g):
    shapes = [(4096, 74, 48, 1), (1024, 600, 300, 3), (65536, 4, 0, 1), (1048576, 300, 20, 5), (4100, 10, 7, 2)]
    info, tiles = p2g.batch_plan(shapes, ctas=148, flags=p2g.BATCH_NO_AUTOTUNE)
    scan = sum(_shape_items(sl, S, R)[0] for sl, S, R, _ in shapes)
    enc = sum(_shape_items(sl, S, R)[1] for sl, S, R, _ in shapes)
    assert info.scan_items == scan and info.encode_items == enc and info.setid_items == len(shapes)
    assert info.items == info.scan_items + info.encode_items + info.setid_items
    for (sl, S, R, _), ts in zip(shapes, tiles):
        Np = (sl + 15) // 16 * 16 // 2
        if R == 0:
            assert ts == 0
        else:
            assert ts % 8 == 0 and 0 < ts <= 2048 and ts >= min(Np, 64) // 8 * 8
    assert info.predicted_ms > 0


def test_plan_autotune_splits_tiles_of_a_lone_job(p2g):
    # one job, 1 row group, 16 tiles of 2048: 16 of 148 CTAs busy; finer tiles
    # spread it wider and the simulated makespan must drop by a quarter or
    # more (not in proportion: every slice of a tile also pays a fixed cost)
    shapes = [(65536, 2000, 20, 1)]
    base, t0 = p2g.batch_plan(shapes, ctas=148, flags=p2g.BATCH_NO_AUTOTUNE)
    tuned, t1 = p2g.batch_plan(shapes, ctas=148)
    assert t0 == [2048] and t1[0] < 2048
    assert tuned.predicted_ms < 0.75 * base.predicted_ms
    assert tuned.encode_items > base.encode_items


def test_plan_large_batch_is_near_its_bound(p2g):
    from par2rust_b200 import workloads as W

    jobs = W.batch_256()
    shapes = [(j.slice_size, j.slices, j.recovery, len(j.file_lengths)) for j in jobs]
    info, tiles = p2g.batch_plan(shapes, ctas=148)
    assert info.jobs == 256 and info.scan_items == sum(_shape_items(j.slice_size, j.slices, j.recovery)[0] for j in jobs)
    # the mixed batch has ~43 SM-seconds of encode work: ~290 ms on 148 SMs
    assert 250 < info.predicted_ms < 400


SPLIT_SHAPES = [(524288, 1027, 200), (65536, 256, 32), (4100, 600, 100), (262144, 4096, 100), (16384, 6104, 1000),
                (524288, 256, 200), (65540, 100, 30)]


@pytest.mark.parametrize("slice_,S,R", SPLIT_SHAPES)
def test_device_job_plan_covers_every_slice_of_every_tile_once(p2g, slice_, S, R):
    """The single-job planner may cut encode items of the last bands into
    slice ranges (tail split).  For every (row group, first symbol) the
    pieces must tile the input slices exactly once; pieces are accumulating
    exactly when they do not cover all slices, and start at or after the
    zeroed columns; items with the same band share it, in symbol order."""
    items, zero_from, bands = p2g.plan_device_job(slice_, S, R)
    Np = (slice_ + 15) // 16 * 16 // 2
    assert items and 0 <= zero_from <= Np
    tensor = items[0]["fold"] == 0  # tensor-core tiles: 16 rows, at most 240 symbols
    assert all((it["fold"] == 0) == tensor for it in items)
    RG = (R + 15) // 16 if tensor else (R + 31) // 32
    pieces = {}
    for it in items:
        assert 0 <= it["row_group"] < RG and it["fold"] in ((0,) if tensor else (1, 2, 4))
        assert it["fold"] <= 1 or it["row_group"] == RG - 1
        assert not tensor or (it["symbols"] <= 240 and it["first_symbol"] % 240 == 0)
        # tensor-core pieces start on whole 16-slice stages of the A image
        assert not tensor or it["first_slice"] % 16 == 0
        assert 0 < it["symbols"] and it["first_symbol"] + it["symbols"] <= Np
        assert 0 <= it["first_slice"] and it["first_slice"] + it["slices"] <= S and it["slices"] > 0
        assert it["accumulate"] == (0 if it["slices"] == S else 1)
        if it["accumulate"]:
            assert it["first_symbol"] >= zero_from
        if bands:
            assert it["band"] < bands
        pieces.setdefault((it["row_group"], it["first_symbol"]), []).append(
            (it["first_slice"], it["slices"], it["symbols"], it["fold"], it["band"]))
    for key, ps in pieces.items():
        ps.sort()
        # the pieces of one tile are cut only along the slices
        assert len({(syms, fold, band) for _, _, syms, fold, band in ps}) == 1, (key, ps)
        at = 0
        for s0, sn, *_ in ps:
            assert s0 == at, (key, ps)
            at += sn
        assert at == S, key
    if bands:
        # bands follow the symbols: within a row group, a later tile never has an
        # earlier band, and unfolded tiles at one symbol share a band across groups
        band_at = {}
        for rg in range(RG):
            seq = sorted((n0, ps[0][4]) for (g, n0), ps in pieces.items() if g == rg)
            assert all(a[1] <= b[1] for a, b in zip(seq, seq[1:])), (rg, seq)
        for (g, n0), ps in pieces.items():
            if ps[0][3] <= 1:
                assert band_at.setdefault(n0, ps[0][4]) == ps[0][4], (g, n0)
    # every row group covers every symbol (a folded tail item covers `fold` tiles)
    for rg in range(RG):
        cover = sorted((it["first_symbol"], it["symbols"]) for it in items if it["row_group"] == rg and it["first_slice"] == 0)
        at = 0
        for n0, syms in cover:
            assert n0 == at, (rg, n0, at)
            at += syms
        assert at == Np, rg
    # the plan is cached: a second call returns the same items
    again, z2, b2 = p2g.plan_device_job(slice_, S, R)
    assert again == items and z2 == zero_from and b2 == bands


def test_device_job_plan_splits_the_538mb_job(p2g, monkeypatch):
    """On the lookup kernel the 538 MB job's last bands are cut into slice
    ranges (its 1.5 ms items would otherwise end in lockstep); the tensor-core
    plan's 14,209 short items (1,093 symbol tiles x 13 row tiles) need no cut."""
    monkeypatch.setenv("P2G_ENCODE_VARIANT", "lut")
    items, zero_from, bands = p2g.plan_device_job(524288, 1027, 200)
    acc = [it for it in items if it["accumulate"]]
    assert bands > 1 and acc and zero_from < 262144
    assert not any(it["accumulate"] for it in p2g.plan_device_job(524288, 1027, 200, with_chains=False)[0])
    monkeypatch.setenv("P2G_ENCODE_VARIANT", "tensor")
    items, zero_from, bands = p2g.plan_device_job(524288, 1027, 200)
    assert len(items) == 1093 * 13 and all(it["fold"] == 0 for it in items) and bands > 1


def test_staged_groups_cover_jobs_in_order(p2g):
    # equal jobs: the first group gets about half of the others' share
    r = p2g.staged_groups([10] * 70, 4)
    assert r == [(0, 10), (10, 30), (30, 50), (50, 70)]
    # every split covers all jobs once, in order, without empty groups
    rng = np.random.default_rng(3)
    for _ in range(200):
        sizes = list(rng.integers(1, 1000, rng.integers(1, 40)))
        g = int(rng.integers(1, 6))
        r = p2g.staged_groups(sizes, g)
        assert r[0][0] == 0 and r[-1][1] == len(sizes) and 1 <= len(r) <= min(g, len(sizes))
        assert all(a < b for a, b in r) and all(b == c for (_, b), (c, _) in zip(r, r[1:]))
    # one job holding most bytes cannot be split
    assert p2g.staged_groups([1, 1, 1000], 4) == [(0, 3)]
    assert p2g.staged_groups([1000, 1, 1], 3) == [(0, 1), (1, 2), (2, 3)]
    assert p2g.staged_groups([5], 4) == [(0, 1)]


def test_plan_rejects_bad_shapes(p2g):
    with pytest.raises(p2g.InvalidSliceSize):
        p2g.batch_plan([(4098, 10, 5, 1)])
    with pytest.raises(p2g.TooManyRecoveryBlocks):
        p2g.batch_plan([(4096, 10, 70000, 1)])
    with pytest.raises(p2g.InvalidArgument):
        p2g.batch_plan([(4096, 0, 5, 1)])


# ---- device (GPU) -----------------------------------------------------------
# (files, slice, R, name prefix): ragged files, slice sizes that are and are not
# multiples of 16, a job without recovery rows, > 256 rows (two packet-MD5
# passes), > 256 slices (several scan items), 40 files (sorting file ids),
# two identical files (equal file ids), a one-slice job, the smallest slice
JOB_SET = [
    ([300_001], 4096, 48),
    ([5000, 70000, 1], 1024, 300),
    ([9000, 4100 * 3], 4100, 7),
    ([200_000], 65536, 0),
    ([100 + 73 * i for i in range(40)], 512, 5),
    ("dup", 256, 3),
    ([65536], 65536, 1),
    ([600 * 1024 - 5], 1024, 33),
    ([40], 4, 2),
    ([1_000_000, 2_000_003, 17], 16384, 60),
]


def _files(k, spec):
    if spec == "dup":
        d = file_bytes(991, 3000).tobytes()
        return [(b"same.bin", d), (b"same.bin", d)]
    return [(f"j{k}_f{i}.bin".encode(), file_bytes(k * 1000 + i + 1, n).tobytes()) for i, n in enumerate(spec)]


def _make_job(p2g, k, spec, slice_, R):
    import torch

    files = _files(k, spec)
    S = sum((len(d) + slice_ - 1) // slice_ for _, d in files)
    host = np.zeros(S * slice_, np.uint8)
    off = 0
    for _, d in files:
        host[off:off + len(d)] = np.frombuffer(d, np.uint8)
        off += (len(d) + slice_ - 1) // slice_ * slice_
    src = torch.from_numpy(host).cuda()
    bufs = p2g.DeviceJobBuffers(S, len(files), slice_, R, src.device)
    # whole-file MD5s on the device as well (file-hash items)
    spec_ = p2g.BatchJobSpec(src, [len(d) for _, d in files], [n for n, _ in files], slice_, R, bufs, hash_full=True)
    return spec_, files, host


def _outputs(spec):
    b = spec.bufs
    S, R, n = spec.input_slices, spec.recovery_count, len(spec.file_lengths)
    rec = b.recovery.view(-1, b.rec_stride)[:R, :spec.slice_size].cpu().numpy().copy() if R else None
    return {
        "rec": rec,
        "checks": b.checksums[:20 * S].cpu().numpy().copy(),
        "h16k": b.hash16k[:16 * n].cpu().numpy().copy(),
        "pkt": b.packet_md5[:16 * R].cpu().numpy().copy() if R else None,
        "set_id": b.set_id_device.cpu().numpy().tobytes(),
        "hfull": b.hash_full[:16 * n].cpu().numpy().copy(),
    }


def _expected(oracle, files, host, slice_, R):
    S = len(host) // slice_
    cks, h16s, fids, hfs = [], [], [], []
    for name, d in files:
        st, c, hf, h16, fid = oracle.scan(d, slice_, name)
        assert st == 0
        cks += c
        h16s.append(h16)
        fids.append(fid)
        hfs.append(hf)
    sid = oracle.set_id(slice_, fids)
    rec = np.asarray(oracle.encode(host, S, slice_, R)).reshape(R, slice_) if R else None
    pkt = [oracle.recovery_packet_md5(sid, r, rec[r].tobytes()) for r in range(R)] if R else []
    return cks, h16s, sid, rec, pkt, hfs


@pytest.fixture(scope="module")
def batch_jobs(p2g):
    return [_make_job(p2g, k, spec, sl, R) for k, (spec, sl, R) in enumerate(JOB_SET)]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["by-shape", "tensor", "lut"])
def test_batch_matches_oracle(p2g, oracle, gpu, batch_jobs, variant):
    """Every job of a heterogeneous batch against the oracle, with the encode
    on the kernel the cost model picks for the batch, or forced to either."""
    import torch

    flags = {"by-shape": 0, "tensor": p2g.BATCH_TENSOR, "lut": p2g.BATCH_LUT}[variant]
    for j, _, _ in batch_jobs:  # no stale rows from an earlier run
        j.bufs.recovery.fill_(0xA5)
        j.bufs.packet_md5.zero_()
    b = p2g.Batch([j for j, _, _ in batch_jobs], flags=flags)
    b.launch()
    torch.cuda.synchronize()
    b.check()
    info = b.info()
    assert info.jobs == len(JOB_SET) and info.setid_items == len(JOB_SET)
    for k, (spec, files, host) in enumerate(batch_jobs):
        got = _outputs(spec)
        cks, h16s, sid, rec, pkt, hfs = _expected(oracle, files, host, spec.slice_size, spec.recovery_count)
        assert got["hfull"].tobytes() == b"".join(hfs), f"job {k} hash_full"
        ch = got["checks"].reshape(-1, 20)
        assert [(bytes(r[:16]), int.from_bytes(bytes(r[16:]), "little")) for r in ch] == cks, f"job {k} checksums"
        assert got["h16k"].tobytes() == b"".join(h16s), f"job {k} hash16k"
        assert got["set_id"] == sid, f"job {k} set id"
        if spec.recovery_count:
            assert (got["rec"] == rec).all(), f"job {k} recovery rows"
            assert got["pkt"].tobytes() == b"".join(pkt), f"job {k} packet md5"
    b.close()


@pytest.mark.gpu
def test_batch_matches_plain_device_job(p2g, gpu, batch_jobs):
    import torch

    b = p2g.Batch([j for j, _, _ in batch_jobs])
    b.launch()
    torch.cuda.synchronize()
    b.check()
    for k, (spec, _, _) in enumerate(batch_jobs):
        got = _outputs(spec)
        plain = p2g.run_device_job(spec.src, spec.file_lengths, spec.names, spec.slice_size, spec.recovery_count,
                                   skip_hash_full=True)
        torch.cuda.synchronize()
        S, R, n = spec.input_slices, spec.recovery_count, len(spec.file_lengths)
        assert (plain.checksums[:20 * S].cpu().numpy() == got["checks"]).all(), k
        assert (plain.hash16k[:16 * n].cpu().numpy() == got["h16k"]).all(), k
        assert plain.set_id == got["set_id"], k
        if R:
            prec = plain.recovery.view(-1, plain.rec_stride)[:R, :spec.slice_size].cpu().numpy()
            assert (prec == got["rec"]).all(), k
            assert (plain.packet_md5[:16 * R].cpu().numpy() == got["pkt"]).all(), k
    b.close()


@pytest.mark.gpu
def test_batch_job_alone_equals_in_mix(p2g, gpu, batch_jobs):
    import torch

    mix = p2g.Batch([j for j, _, _ in batch_jobs])
    mix.launch()
    torch.cuda.synchronize()
    mix.check()
    in_mix = [_outputs(j) for j, _, _ in batch_jobs]
    for k, (spec, _, _) in enumerate(batch_jobs):
        for t in (spec.bufs.recovery, spec.bufs.checksums, spec.bufs.hash16k, spec.bufs.packet_md5,
                  spec.bufs.set_id_device, spec.bufs.hash_full):
            t.fill_(0xA5)
        alone = p2g.Batch([spec])
        alone.launch()
        torch.cuda.synchronize()
        alone.check()
        got = _outputs(spec)
        for key in ("checks", "h16k", "set_id", "hfull"):
            assert np.array_equal(np.frombuffer(bytes(got[key]), np.uint8),
                                  np.frombuffer(bytes(in_mix[k][key]), np.uint8)), (k, key)
        if spec.recovery_count:
            assert (got["rec"] == in_mix[k]["rec"]).all() and (got["pkt"] == in_mix[k]["pkt"]).all(), k
        alone.close()
    mix.close()


@pytest.mark.gpu
def test_staged_batch_from_host_equals_batch(p2g, gpu, batch_jobs):
    """Sources uploaded group by group beside the running groups: every
    output must equal one Batch over all jobs, on two runs in a row."""
    import torch

    specs = [j for j, _, _ in batch_jobs]
    ref = p2g.Batch(specs)
    ref.launch()
    torch.cuda.synchronize()
    ref.check()
    want = [_outputs(j) for j in specs]
    ref.close()
    hosts = [torch.from_numpy(h).pin_memory() for _, _, h in batch_jobs]
    outs = [tuple(torch.empty(t.numel(), dtype=torch.uint8).pin_memory()
                  for t in (j.bufs.recovery, j.bufs.checksums, j.bufs.packet_md5, j.bufs.hash16k,
                            j.bufs.set_id_device)) for j in specs]
    staged = p2g.StagedBatch(specs, hosts, outs, groups=3)
    assert len(staged.ranges) >= 2 and staged.ranges[0][0] == 0 and staged.ranges[-1][1] == len(specs)
    assert all(a < b and b == c for (a, b), (c, _) in zip(staged.ranges, staged.ranges[1:]))
    for _ in range(2):
        for j in specs:  # the device copies must come from the host sources
            j.src.fill_(0x5A)
            for t in (j.bufs.recovery, j.bufs.checksums, j.bufs.packet_md5, j.bufs.hash16k, j.bufs.set_id_device):
                t.fill_(0xA5)
        for o in outs:
            for t in o:
                t.fill_(0)
        staged.launch()
        torch.cuda.synchronize()
        staged.check()
        for k, (j, w, o) in enumerate(zip(specs, want, outs)):
            S, R, n = j.input_slices, j.recovery_count, len(j.file_lengths)
            assert o[1][:20 * S].numpy().tobytes() == w["checks"].tobytes(), k
            assert o[3][:16 * n].numpy().tobytes() == w["h16k"].tobytes(), k
            assert o[4].numpy().tobytes() == w["set_id"], k
            if R:
                rec = o[0].view(-1, j.bufs.rec_stride)[:R, :j.slice_size].numpy()
                assert (rec == w["rec"]).all(), k
                assert o[2][:16 * R].numpy().tobytes() == w["pkt"].tobytes(), k
    staged.close()


@pytest.mark.gpu
def test_batch_graph_replay_direct_launch_and_derived_basis_agree(p2g, gpu, batch_jobs):
    import torch

    jobs = [j for j, _, _ in batch_jobs]
    g = p2g.Batch(jobs)
    g.launch()
    torch.cuda.synchronize()
    first = [_outputs(j) for j in jobs]
    for j in jobs:
        j.bufs.recovery.zero_()
        j.bufs.packet_md5.zero_()
        j.bufs.set_id_device.zero_()
    g.launch()
    g.launch()  # a replay right behind another on the same stream
    torch.cuda.synchronize()
    g.check()
    for flags in (p2g.BATCH_NO_GRAPH, p2g.BATCH_DERIVE_BASIS, p2g.BATCH_NO_AUTOTUNE | p2g.BATCH_DERIVE_BASIS):
        for j in jobs:
            j.bufs.recovery.zero_()
            j.bufs.packet_md5.zero_()
        d = p2g.Batch(jobs, flags=flags)
        d.launch()
        torch.cuda.synchronize()
        d.check()
        for k, j in enumerate(jobs):
            o = _outputs(j)
            assert o["set_id"] == first[k]["set_id"]
            if j.recovery_count:
                assert (o["rec"] == first[k]["rec"]).all() and (o["pkt"] == first[k]["pkt"]).all(), (flags, k)
        d.close()
    g.close()


@pytest.mark.gpu
def test_batch_validation(p2g, gpu, batch_jobs):
    import torch

    spec = batch_jobs[0][0]
    bad = p2g.BatchJobSpec(spec.src, [0], [b"x"], 4096, 4, spec.bufs)
    with pytest.raises(p2g.EmptyFile):
        p2g.Batch([bad])
    odd = p2g.BatchJobSpec(spec.src[1:], [10], [b"x"], 4096, 4, spec.bufs)
    with pytest.raises(p2g.InvalidArgument):
        p2g.Batch([odd])
    with pytest.raises(p2g.InvalidSliceSize):
        p2g.Batch([p2g.BatchJobSpec(spec.src, [10], [b"x"], 4098, 4, spec.bufs)])
    torch.cuda.synchronize()


@pytest.mark.parametrize("slice_,S,R,want", [
    (524288, 1027, 200, "tensor"),   # the 538 MB job: 5.4 ms on the tensor cores against 9.0 ms
    (262144, 8723, 2000, "tensor"),  # many_2000's shape
    (524288, 1027, 16, "tensor"),    # 0.49 ms against 1.01 ms
    (262144, 64, 32, "lut"),         # small: 0.084 ms on the lookup kernel against 0.107 ms
    (4096, 40, 3, "lut"),
])
def test_planner_picks_the_encode_kernel_by_shape(p2g, monkeypatch, slice_, S, R, want):
    """With no flag or environment override, the single-job planner puts the
    encode on the kernel its cost model finds faster for the shape (measured
    times in the comments); tensor-core items report fold 0."""
    monkeypatch.delenv("P2G_ENCODE_VARIANT", raising=False)
    items, _, _ = p2g.plan_device_job(slice_, S, R)
    got = "tensor" if items[0]["fold"] == 0 else "lut"
    assert got == want, (slice_, S, R, got)
