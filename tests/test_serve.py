"""Serving loop: create requests admitted by HBM footprint and run in device
waves shared with the other resident jobs (continuous batching).

Every job's outputs are checked against the oracle, and against the same job
served alone: a request's results must not depend on what it was mixed with.
The HBM budget is set below the mix's total footprint so admission has to
queue requests and admit them as earlier ones are released.
"""
import time

import numpy as np
import pytest

from par2rust_b200.workloads import file_bytes

pytestmark = pytest.mark.gpu

# (file lengths, slice, R): with wave_ms=2 an encode item holds at most ~300
# slices of 2048 symbols, so jobs A and G run as XOR-accumulated slice chunks;
# B has two packet items; C needs realigned slices; D has no recovery rows
MIX = [
    ([2_000_000], 4096, 40),
    ([5000, 70000, 1], 1024, 300),
    ([9000, 4100 * 3], 4100, 7),
    ([200_000], 65536, 0),
    ([100 + 97 * i for i in range(12)], 512, 5),
    ([3_000_000], 65536, 10),
    ([700 * 16384 - 3], 16384, 60),
]
BUDGET = 13_000_000  # holds the largest job (12.45 MB), below the mix total (19.0 MB)


def _seeds(k, n):
    return [(k * 7919 + f * 104729 + 1) & (2**64 - 1) for f in range(n)]


def _names(k, n):
    return [f"req{k}_f{i}.bin".encode() for i in range(n)]


def _footprint(lens, slice_, R):
    S = sum((n + slice_ - 1) // slice_ for n in lens)
    return S * slice_ + R * ((slice_ + 15) // 16 * 16)


def _drain(srv, want, timeout=120.0):
    """Collect `want` results, reading each job's outputs and releasing it as
    it arrives (completed jobs hold their budget until released)."""
    got, outs = {}, {}
    t_end = time.time() + timeout
    while len(got) < want and time.time() < t_end:
        for r in srv.poll(wait_ms=50):
            got[r.ticket] = r
            outs[r.ticket] = srv.outputs(r) if r.status == 0 else None
            srv.release(r.ticket)
    assert len(got) == want, f"{len(got)} of {want} jobs completed"
    return got, outs


def _expected(oracle, k, lens, slice_, R):
    files = [(nm, file_bytes(sd, n).tobytes()) for nm, sd, n in zip(_names(k, len(lens)), _seeds(k, len(lens)), lens)]
    cks, h16s, fids = [], [], []
    host = b""
    for name, d in files:
        st, c, _hf, h16, fid = oracle.scan(d, slice_, name)
        assert st == 0
        cks += c
        h16s.append(h16)
        fids.append(fid)
        host += d + bytes((-len(d)) % slice_)
    sid = oracle.set_id(slice_, fids)
    S = len(host) // slice_
    rec = np.asarray(oracle.encode(np.frombuffer(host, np.uint8), S, slice_, R)).reshape(R, slice_) if R else None
    pkt = b"".join(oracle.recovery_packet_md5(sid, r, rec[r].tobytes()) for r in range(R))
    ck = b"".join(m + c.to_bytes(4, "little") for m, c in cks)
    return {"checksums": ck, "hash16k": b"".join(h16s), "set_id": sid,
            "recovery": [rec[r].tobytes() for r in range(R)] if R else [], "packet_md5": pkt}


def _serve(p2g, jobs, budget, wave_ms=2.0):
    srv = p2g.Server(hbm_budget=budget, wave_ms=wave_ms)
    tickets = {}
    for k, (lens, slice_, R) in jobs:
        tickets[srv.submit_seeded(lens, _seeds(k, len(lens)), _names(k, len(lens)), slice_, R, tag=k)] = k
    done, raw = _drain(srv, len(jobs))
    outs = {}
    for t, r in done.items():
        assert r.status == 0, (tickets[t], r.status)
        outs[tickets[t]] = raw[t]
    stats = srv.stats()
    srv.close()
    return outs, done, stats


@pytest.mark.parametrize("variant", ["by-shape", "tensor"])
def test_serve_mix_matches_oracle_and_respects_budget(p2g, oracle, gpu, variant, monkeypatch):
    """The mix against the oracle.  With the tensor-core encode forced, the
    jobs whose A image fits (R 10 on 64 KiB slices, R 7 on realigned 4,100-byte
    slices) run tensor-core items, and waves alternate the two kinds."""
    if variant == "tensor":
        monkeypatch.setenv("P2G_ENCODE_VARIANT", "tensor")
    jobs = list(enumerate(MIX))
    assert sum(_footprint(*j) for _, j in jobs) > BUDGET  # admission must queue
    outs, done, stats = _serve(p2g, jobs, BUDGET)
    assert stats["completed"] == len(MIX) and stats["released"] == len(MIX)
    assert 0 < stats["peak_resident_bytes"] <= BUDGET
    assert stats["waves"] >= 2
    for k, (lens, slice_, R) in jobs:
        want = _expected(oracle, k, lens, slice_, R)
        got = outs[k]
        for key in ("checksums", "hash16k", "set_id", "packet_md5"):
            assert got[key] == want[key], (k, key)
        assert got["recovery"] == want["recovery"], (k, "recovery")
    for r in done.values():
        assert r.submit_s <= r.admit_s <= r.done_s


def test_serve_each_job_alone_equals_in_mix(p2g, gpu):
    jobs = list(enumerate(MIX))
    mixed, _, _ = _serve(p2g, jobs, BUDGET)
    for k, job in jobs:
        alone, _, st = _serve(p2g, [(k, job)], BUDGET)
        assert st["waves"] >= 1
        assert alone[k] == mixed[k], f"job {k} differs alone vs in the mix"


def test_serve_host_source_equals_seeded(p2g, gpu):
    import torch

    k, (lens, slice_, R) = 1, MIX[1]
    host = b"".join(file_bytes(sd, n).tobytes() + bytes((-n) % slice_) for sd, n in zip(_seeds(k, len(lens)), lens))
    pinned = torch.frombuffer(bytearray(host), dtype=torch.uint8).pin_memory()
    srv = p2g.Server(hbm_budget=BUDGET, wave_ms=2.0)
    t = srv.submit_host(pinned, lens, _names(k, len(lens)), slice_, R)
    done, raw = _drain(srv, 1)
    assert done[t].status == 0
    got = raw[t]
    srv.close()
    seeded, _, _ = _serve(p2g, [(k, (lens, slice_, R))], BUDGET)
    assert got == seeded[k]


def test_serve_rejects_bad_requests(p2g, gpu):
    srv = p2g.Server(hbm_budget=1_000_000, wave_ms=2.0)
    with pytest.raises(p2g.InvalidArgument):  # can never fit the budget
        srv.submit_seeded([2_000_000], [1], [b"big"], 4096, 8)
    with pytest.raises(p2g.EmptyFile):
        srv.submit_seeded([0], [1], [b"empty"], 4096, 8)
    with pytest.raises(p2g.InvalidSliceSize):
        srv.submit_seeded([100], [1], [b"x"], 4098, 8)
    assert srv.stats()["submitted"] == 0
    srv.close()
