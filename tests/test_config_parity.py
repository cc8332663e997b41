"""Bit-exactness at the benchmark shapes, on the GPU, against the oracle.

- single_538m (538,218,411 B, slice 524,288, R 200, Exponential): the exact
  job the benchmark times -- p2g_run_device_job with the default persistent
  plan and its tail split -- every recovery row, slice checksum, hash16k,
  set id and packet MD5; then the public in-memory create, whose index and
  nine volume files must equal the oracle's byte for byte
  (src/creator.rs:883-1018 encode, :1025-1042 volume layout).
- many_2000 (2,000 files, slice 262,144, R 2,000, Uniform{15}): every slice
  checksum, hash16k, hash_full (on the device for many files), the set id,
  every packet MD5 over the device's rows, and a seeded sample of 32 rows
  (0, 1 and 1,999 always) against the oracle's encode of those rows; the
  index file through the public create against the oracle's.
"""
import numpy as np
import pytest

from par2rust_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device_src(job, dev):
    import torch

    sl = job.slice_size
    src = torch.zeros(job.slices * sl, dtype=torch.uint8, device=dev)
    files, off = [], 0
    for n, sd in zip(job.file_lengths, job.seeds):
        f = W.file_bytes(sd, n)
        files.append(f)
        src[off:off + n] = torch.from_numpy(f).to(dev)
        off += (n + sl - 1) // sl * sl
    return src, files


def test_single_538m_job_and_files_bit_exact(p2g, gpu, oracle):
    import torch

    from oracle import parity

    job = W.single_538m()
    sl, R, S = job.slice_size, job.recovery, job.slices
    assert (S, job.file_lengths[0]) == (1027, 538_218_411)
    src, files = _device_src(job, torch.device("cuda"))
    names = [b"source.bin"]
    bufs = p2g.run_device_job(src, job.file_lengths, names, sl, R, skip_hash_full=True)
    torch.cuda.synchronize()
    out = parity.device_outputs(bufs, S, 1, sl, R)
    bad = parity.check_device_job(files, names, sl, R, out["rec"], out["checks"], out["hash16k"], bufs.set_id,
                                  out["packet_md5"])
    assert not bad, bad
    del src, bufs
    torch.cuda.empty_cache()
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=sl, recovery_block_count=R,
                             volume_scheme=p2g.VolumeScheme.Exponential())
    got = p2g.create_in_memory(opts, [(names[0], files[0])])
    want = oracle.create([(names[0], files[0])], sl, R, kind=oracle.SCHEME_EXPONENTIAL, fast=True)
    assert [n for n, _ in got] == [n for n, _ in want] and len(want) == 10
    for (n, a), (_, b) in zip(got, want):
        assert a == b, f"{n} differs from the oracle"


def test_many_2000_hashes_packets_and_sampled_rows_bit_exact(p2g, gpu, oracle):
    import torch

    from oracle import parity

    job = W.many_2000(seed=3)
    sl, R, S, n = job.slice_size, job.recovery, job.slices, len(job.file_lengths)
    assert n == 2000 and R == 2000 and S > 5000
    src, files = _device_src(job, torch.device("cuda"))
    names = [f"file{i:04d}.bin".encode() for i in range(n)]
    bufs = p2g.run_device_job(src, job.file_lengths, names, sl, R)
    torch.cuda.synchronize()
    out = parity.device_outputs(bufs, S, n, sl, R)
    rows = parity.sample_rows(R, 32, seed=3)
    assert {0, 1, R - 1} <= set(rows)
    bad = parity.check_device_job(files, names, sl, R, out["rec"], out["checks"], out["hash16k"], bufs.set_id,
                                  out["packet_md5"], hash_full=out["hash_full"], rows=rows)
    assert not bad, bad
    del src, bufs
    torch.cuda.empty_cache()
    # the index file of the public create (critical packets only: no recovery data)
    opts = p2g.CreateOptions(output="many.par2", slice_size=sl, recovery_block_count=R,
                             volume_scheme=p2g.VolumeScheme.Uniform(15))
    got = p2g.create_in_memory(opts, list(zip(names, files)), copy=False)
    want = oracle.create(list(zip(names, files)), sl, 0, index_path="many.par2")
    assert got[0][0] == want[0][0] == "many.par2" and len(got) == 16
    assert bytes(got[0][1]) == want[0][1]
