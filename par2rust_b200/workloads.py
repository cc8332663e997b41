"""Seeded synthetic create workloads.

Bytes come from a splitmix64 counter stream (Vigna's public-domain
generator): word k of a file is mix(seed + (k+1)*GAMMA), stored
little-endian, truncated to the file length.  Sizes and per-job choices come
from a separate splitmix64 "meta" stream.  GF(2^16) multiply, MD5 and CRC32
costs do not depend on the byte values, so uniform random bytes stand in
for real files.

Named workloads (sizes as used by the benchmark and the parity tests):
  single_16m      1 file, 16,777,216 B, slice 65,536, R 32, Single
  single_538m     1 file, 538,218,411 B, slice 524,288, R 200, Exponential
  many_2000       2,000 files log-uniform in [1 KiB, 8 MiB], slice 262,144,
                  R 2,000, Uniform{15}
  batch_256       256 jobs, 1-16 files log-uniform in [4 KiB, 64 MiB],
                  slice in {16K, 64K, 256K, 1M}, R = max(1, ceil(f*S)),
                  f ~ U[0.01, 0.20], total <= 24 GiB
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

GAMMA = 0x9E3779B97F4A7C15
MASK = (1 << 64) - 1


def _mix(z: int) -> int:
    z = (z + 0) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


class Meta:
    """splitmix64 scalar stream for sizes and choices."""

    def __init__(self, seed: int):
        self.state = seed & MASK

    def next(self) -> int:
        self.state = (self.state + GAMMA) & MASK
        return _mix(self.state)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))

    def log_uniform(self, lo: int, hi: int) -> int:
        u = self.uniform()
        return int(math.floor(math.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))))

    def randint(self, lo: int, hi: int) -> int:  # inclusive
        return lo + self.next() % (hi - lo + 1)


def file_seed(cfg_seed: int, job: int, f: int) -> int:
    return _mix((cfg_seed ^ (job << 20) ^ f) & MASK)


def file_bytes(seed: int, length: int) -> np.ndarray:
    """splitmix64 counter stream, numpy (host)."""
    nwords = (length + 7) // 8
    k = np.arange(1, nwords + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * np.uint64(GAMMA)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z.view(np.uint8)[:length].copy()


def file_bytes_torch(seed: int, length: int, device="cuda"):
    """The same stream generated on the device (torch int64 wraps mod 2^64)."""
    import torch

    nwords = (length + 7) // 8

    def c(v):  # uint64 constant as the int64 with the same bits
        return v - (1 << 64) if v >= (1 << 63) else v

    k = torch.arange(1, nwords + 1, dtype=torch.int64, device=device)
    z = c(seed & MASK) + k * c(GAMMA)

    def srl(x, s):  # logical right shift on int64 bits
        return (x >> s) & ((1 << (64 - s)) - 1)

    z = (z ^ srl(z, 30)) * c(0xBF58476D1CE4E5B9)
    z = (z ^ srl(z, 27)) * c(0x94D049BB133111EB)
    z = z ^ srl(z, 31)
    return z.view(torch.uint8)[:length]


def deterministic_bytes(seed: int, length: int) -> bytes:
    """The reference's fixture LCG (tests/common/mod.rs:46-57,
    src/galois_simd.rs:772-782): state = seed*0x9E3779B97F4A7C15, then
    state = state*6364136223846793005 + 1442695040888963407, byte = state>>33."""
    state = (seed * 0x9E3779B97F4A7C15) & MASK
    out = bytearray(length)
    for i in range(length):
        state = (state * 6364136223846793005 + 1442695040888963407) & MASK
        out[i] = (state >> 33) & 0xFF
    return bytes(out)


@dataclass
class Job:
    slice_size: int
    recovery: int
    file_lengths: List[int]
    seeds: List[int] = field(default_factory=list)
    scheme: str = "single"
    scheme_count: int = 0

    @property
    def slices(self) -> int:
        return sum((n + self.slice_size - 1) // self.slice_size for n in self.file_lengths)

    @property
    def source_bytes(self) -> int:
        return sum(self.file_lengths)


def single_16m() -> Job:
    return Job(65536, 32, [16_777_216], [file_seed(1, 0, 0)], "single")


def single_538m() -> Job:
    return Job(524288, 200, [538_218_411], [file_seed(2, 0, 0)], "exponential")


def many_2000(seed: int = 3) -> Job:
    m = Meta(seed ^ 0xA5A5A5A5A5A5A5A5)
    while True:
        lens = [m.log_uniform(1024, 8 << 20) for _ in range(2000)]
        j = Job(262144, 2000, lens, [file_seed(seed, 0, f) for f in range(2000)], "uniform", 15)
        if j.slices <= 32768:
            return j


def batch_256(seed: int = 4, cap: int = 24 << 30, n_jobs: int = 256) -> List[Job]:
    """n_jobs jobs (256 by default) whose total source stays within `cap`;
    a draw that would exceed the cap (or 32,768 slices) is redrawn, so the
    cap must leave room for n_jobs jobs (~57 MB each on average)."""
    m = Meta(seed ^ 0xA5A5A5A5A5A5A5A5)
    jobs, total = [], 0
    slices = [16384, 65536, 262144, 1048576]
    draws = 0
    while len(jobs) < n_jobs:
        draws += 1
        if draws > 100 * n_jobs:
            raise ValueError(f"cannot fit {n_jobs} jobs under a {cap}-byte cap")
        nf = m.randint(1, 16)
        lens = [m.log_uniform(4096, 64 << 20) for _ in range(nf)]
        ss = slices[m.randint(0, 3)]
        f = 0.01 + 0.19 * m.uniform()
        S = sum((n + ss - 1) // ss for n in lens)
        R = max(1, math.ceil(f * S))
        if S > 32768 or total + sum(lens) > cap:
            continue
        jid = len(jobs)
        jobs.append(Job(ss, R, lens, [file_seed(seed, jid, i) for i in range(nf)], "single"))
        total += sum(lens)
    return jobs


def job_cost(job: Job) -> int:
    """Relative device cost of a create job: GF multiply-accumulates
    (input slices x recovery rows x symbols per slice) plus the bytes hashed."""
    return job.slices * max(job.recovery, 1) * (job.slice_size // 2) + 4 * job.source_bytes


def shard_jobs(jobs: List[Job], rank: int, world: int) -> List[int]:
    """Indices of the jobs rank `rank` of `world` runs.  Jobs are independent,
    so GPUs share no data: greedy longest-processing-time assignment by
    job_cost, deterministic on every rank (ties broken by job index)."""
    if world <= 1:
        return list(range(len(jobs)))
    load = [0] * world
    owner = [0] * len(jobs)
    for i in sorted(range(len(jobs)), key=lambda k: (-job_cost(jobs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += job_cost(jobs[i])
    return [i for i in range(len(jobs)) if owner[i] == rank]


SERVE_SLICES = [16384, 65536, 262144, 1048576]


def serve_requests(n: int = 10_000, seed: int = 5) -> List[Job]:
    """Serving-loop requests: job totals log-uniform in [1 MiB, 2 GiB], split
    into 1-32 files (random cut weights, each file >= 1 byte); slice drawn
    from {16K, 64K, 256K, 1M} as in the batched config, raised to the
    smallest slice of that set with at most 32,768 slices when the draw
    exceeds it; R = max(1, ceil(f*S)), f ~ U[0.01, 0.20]."""
    m = Meta(seed ^ 0xA5A5A5A5A5A5A5A5)
    jobs = []
    for jid in range(n):
        total = m.log_uniform(1 << 20, 2 << 30)
        nf = m.randint(1, 32)
        w = [m.uniform() + 1e-9 for _ in range(nf)]
        sw = sum(w)
        lens = [max(1, int(total * x / sw)) for x in w]
        lens[-1] = max(1, total - sum(lens[:-1]))
        k = m.randint(0, 3)
        f = 0.01 + 0.19 * m.uniform()
        while True:
            ss = SERVE_SLICES[k]
            S = sum((x + ss - 1) // ss for x in lens)
            if S <= 32768 or k == len(SERVE_SLICES) - 1:
                break
            k += 1
        R = max(1, math.ceil(f * S))
        jobs.append(Job(ss, R, lens, [file_seed(seed, jid, i) for i in range(nf)], "single"))
    return jobs


def poisson_arrivals(n: int, rate: float, seed: int) -> List[float]:
    """Open-loop arrival times (seconds from 0) of n requests at `rate` per
    second: exponential gaps from a splitmix64 stream."""
    m = Meta(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += -math.log(1.0 - m.uniform()) / rate
        out.append(t)
    return out
