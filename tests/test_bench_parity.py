"""The benchmark's own parity checks, on CPU: the serving sweep's sample of
requests is drawn within its cost bounds, outputs equal to the oracle's pass,
and a single flipped bit in any kept output is reported as a mismatch.

The "device" outputs here are the oracle's own (a scan, the set id, the
encode and the packet MD5s of each sampled request), so the check is
exercised without a GPU; the GPU run feeds it what the serving loop
returned.
"""
import numpy as np
import pytest

import bench
from par2rust_b200 import workloads as W


def _oracle_outputs(oracle, job, i):
    from oracle import parity

    files = [W.file_bytes(sd, ln) for ln, sd in zip(job.file_lengths, job.seeds)]
    names = [f"req{i:05d}_f{k:02d}.bin".encode() for k in range(len(files))]
    cks, h16, fids = [], b"", []
    for f, nm in zip(files, names):
        st, c, _hf, h, fid = oracle.scan(f, job.slice_size, nm)
        assert st == 0
        cks += c
        h16 += h
        fids.append(fid)
    sid = oracle.set_id(job.slice_size, fids)
    R = job.recovery
    rec = oracle.encode_fast(parity.padded_source(files, job.slice_size), job.slices, job.slice_size, R)
    rec = np.asarray(rec).reshape(R, job.slice_size)
    return {"recovery": [rec[r].tobytes() for r in range(R)],
            "checksums": b"".join(m + c.to_bytes(4, "little") for m, c in cks), "hash16k": h16, "set_id": sid,
            "packet_md5": b"".join(oracle.recovery_packet_md5(sid, r, rec[r].tobytes()) for r in range(R))}


@pytest.fixture(scope="module")
def sample(oracle):
    jobs = W.serve_requests(400, seed=5)
    pick = bench.serve_parity_pick(jobs, n_sample=3, max_bytes=8 << 20, max_macs=3e10, seed=5)
    kept = {i: _oracle_outputs(oracle, jobs[i], i) for i in sorted(pick)}
    return jobs, pick, kept


def test_serve_parity_pick_stays_within_its_bounds(sample):
    jobs, pick, _ = sample
    assert 1 <= len(pick) <= 4  # the seeded sample plus the smallest candidate
    for i in pick:
        j = jobs[i]
        assert j.source_bytes <= 8 << 20
        assert j.slices * j.recovery * (j.slice_size // 2) <= 3e10 / 3
    small = min(range(len(jobs)), key=lambda k: jobs[k].source_bytes)
    assert small in pick


def test_serve_parity_accepts_the_oracle_outputs(sample):
    jobs, _, kept = sample
    res = bench.serve_parity(jobs, kept)
    assert res["result"] == "bit-exact", res["mismatches"]
    assert res["requests_checked"] == sorted(kept)


@pytest.mark.parametrize("field", ["recovery", "checksums", "hash16k", "set_id", "packet_md5"])
def test_serve_parity_reports_one_flipped_bit(sample, field):
    jobs, _, kept = sample
    i = sorted(kept)[0]
    out = dict(kept[i])
    if field == "recovery":
        rows = list(out["recovery"])
        b = bytearray(rows[-1])
        b[len(b) // 2] ^= 0x10
        rows[-1] = bytes(b)
        out["recovery"] = rows
    else:
        b = bytearray(out[field])
        b[-1] ^= 0x01
        out[field] = bytes(b)
    res = bench.serve_parity(jobs, {i: out})
    assert res["result"] == "MISMATCH" and i in res["mismatches"]
