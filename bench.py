#!/usr/bin/env python3
"""PAR2 create benchmark: encode source GB/s on B200.

Workload (default): one 538,218,411-byte file of seeded random bytes, slice
524,288 (1,027 input slices, the last zero-padded), 200 recovery blocks,
Exponential volume split.

  value      device-resident step: the source already in HBM; one step is the
             device work of one create job -- coefficient basis + Reed-Solomon
             encode + per-slice MD5/CRC32 + hash16k + recovery-packet MD5
             (the whole-file MD5 chain is one serial stream; it is timed
             separately as file_md5_device_chain_gbs and counted in e2e).
             Timed with CUDA events on the launching stream; max over ranks.
  e2e        the same metric through the public API (p2g_create_in_memory):
             pinned host source -> H2D -> device job -> whole-file MD5 ->
             D2H of recovery rows + checksums -> index/volume bytes in memory.
  roofline   the timed step's encode against the unit it is bound by: the
             tensor pipe (nominal dense FP4, 2 x 256 e2m1 FLOP per GF MAC) when
             the planner runs tensor-core items, else the shared-memory lookup
             bound of the LUT kernel; `lookup_roofline` and `hbm_roofline`
             beside it, and `encode_only` times each encode kernel alone.
  cpu_baseline  the reference's CPU create path (C port with the GFNI/AVX-512
             kernel, all host threads) on a bounded sample of the same file.

`--impl reference` times only that CPU path on this config (rank 0 only).
Launched under torchrun for N>1: one independent job replica per rank (the
path shards by job; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PUBLISHED_E2E_GBS = 0.0975  # par2rust create, same shape, Apple M4 10 threads (5.52 s)

WORKLOADS = {
    "single_538m": dict(length=538_218_411, slice=524_288, R=200, scheme="exponential", seed=2),
    "single_16m": dict(length=16_777_216, slice=65_536, R=32, scheme="single", seed=1),
    # profiling case: same slice size and recovery count, 256 slices (134 MB > L2)
    "prof_256x512k": dict(length=256 * 524_288, slice=524_288, R=200, scheme="exponential", seed=2),
    # 256 independent jobs in one persistent launch vs the plain per-job path
    "batch_256": dict(batch=True, n_jobs=256, seed=4),
    # serving loop: open-loop Poisson arrivals of create requests
    "serve": dict(serve=True, seed=5),
    # dense contraction: 2,000 files log-uniform in [1 KiB, 8 MiB], R 2,000, Uniform{15}
    "many_2000": dict(many=True, seed=3),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single_538m", choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the device MD5-chain rate probe")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-vs-plain section of the default (single-file) run")
    ap.add_argument("--no-many", action="store_true", help="skip the many_2000 section of the default run")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the timed step's outputs")
    ap.add_argument("--serve-requests", type=int, default=2_000,
                    help="serving section of the default run: requests per arrival rate (0 skips it)")
    ap.add_argument("--serve-fracs", default="0.5,0.85",
                    help="serving section of the default run: arrival rates as fractions of the probed capacity")
    ap.add_argument("--batch-jobs", type=int, default=256, help="jobs in the batched comparison")
    ap.add_argument("--requests", type=int, default=2_000,
                    help="serving: requests per arrival rate (the full mix is 10,000: ~8-13 min per rate)")
    ap.add_argument("--rates", default="", help="serving: comma-separated arrival rates (jobs/s); default "
                                                "0.5,0.8,0.95 x the capacity measured by a closed-batch probe")
    ap.add_argument("--probe-jobs", type=int, default=200, help="serving: jobs in the capacity probe")
    ap.add_argument("--wave-ms", type=float, default=20.0, help="serving: target device time per wave")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                      "-i", str(self.idx), "-lms", "20"], stdout=open(self.path, "w"),
                                     stderr=subprocess.DEVNULL)
        # the timed region is short (~0.1 s): start it only once sampling runs
        t_end = time.time() + 5.0
        while time.time() < t_end and os.path.getsize(self.path) == 0:
            time.sleep(0.01)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


FP4_DENSE_TFLOPS = 9000.0  # nominal dense FP4 (block-scaled e2m1) tensor rate of one B200


def measured_bf16():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return json.load(open(p)).get("bf16_tflops") if os.path.exists(p) else None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def cpu_baseline(data_np, wl, target_s, threads=0, steps=1, warmup=0):
    """Time the CPU port on a bounded prefix of the same file; GB/s of source."""
    from oracle import oracle as orc

    slice_, R = wl["slice"], wl["R"]
    n_slices = (len(data_np) + slice_ - 1) // slice_
    # calibrate on a small prefix, then size the sample to ~target_s
    probe = min(n_slices, 8)
    t, *_ = orc.create_timed(data_np[:probe * slice_], slice_, R, threads)
    per_slice = max(t / probe, 1e-6)
    take = int(min(n_slices, max(probe, target_s / per_slice)))
    sample = data_np[:min(len(data_np), take * slice_)]
    for _ in range(warmup):
        orc.create_timed(sample, slice_, R, threads)
    times = []
    parts = None
    for _ in range(max(steps, 1)):
        t, ts, te, tp = orc.create_timed(sample, slice_, R, threads)
        times.append(t)
        parts = (ts, te, tp)
    tt = sum(times) / len(times)
    # the same work as the device-resident `value` (which leaves the
    # whole-file MD5 to the host, where e2e counts it): one more pass without it
    t_nf, *_ = orc.create_timed(sample, slice_, R, threads, whole_file_md5=False)
    return {
        "value": len(sample) / tt / 1e9, "unit": "GB/s", "cores": threads or orc.max_threads(),
        "value_without_file_md5": len(sample) / t_nf / 1e9,
        "kind": "port",
        "sample": f"first {take} of {n_slices} slices ({len(sample)} B) of the same file, R={R}: scan "
                  f"(per-slice MD5+CRC32 joined with the whole-file MD5), encode "
                  f"({'GFNI-AVX512' if orc.kernel_is_gfni512() else 'byte-table'} kernel), "
                  f"recovery-packet MD5s of the exponential volumes",
        "seconds_per_step": tt, "scan_s": parts[0], "encode_s": parts[1], "packet_md5_s": parts[2],
    }, tt


def run_reference(args, wl):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import numpy as np

    from par2rust_b200 import workloads as W

    data = W.file_bytes(W.file_seed(wl["seed"], 0, 0), wl["length"])
    # each step is a bounded sample sized so warmup+steps take about two minutes in total
    per_step = max(1.0, min(args.cpu_seconds, 120.0 / max(1, args.steps + args.warmup)))
    cb, tt = cpu_baseline(data, wl, target_s=per_step, steps=args.steps, warmup=args.warmup)
    line = {
        "metric": "encode source GB/s", "value": cb["value"], "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": cb["value"] / PUBLISHED_E2E_GBS, "dtype": "u16", "data": "synthetic",
        "impl": "reference",
        "config": config_dict(args, wl),
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def batch_specs(dev, n_jobs=256, seed=4):
    """The mixed batch on the device: each job's files generated in place
    (seeded splitmix64 bytes), slice-padded, with its output buffers."""
    import torch

    import par2rust_b200 as p2g
    from par2rust_b200 import workloads as W

    jobs = W.batch_256(seed=seed, n_jobs=n_jobs)
    specs = []
    for k, j in enumerate(jobs):
        src = torch.zeros(j.slices * j.slice_size, dtype=torch.uint8, device=dev)
        off = 0
        for n, sd in zip(j.file_lengths, j.seeds):
            src[off:off + n] = W.file_bytes_torch(sd, n, device=dev)
            off += (n + j.slice_size - 1) // j.slice_size * j.slice_size
        names = [f"job{k:03d}_file{i:02d}.bin".encode() for i in range(len(j.file_lengths))]
        bufs = p2g.DeviceJobBuffers(j.slices, len(names), j.slice_size, j.recovery, dev)
        specs.append(p2g.BatchJobSpec(src, list(j.file_lengths), names, j.slice_size, j.recovery, bufs))
    return jobs, specs


def batch_parity(jobs, specs, snap, seed=4, n_sample=8, max_macs=3e11):
    """Oracle check of a seeded sample of the batch's jobs (every recovery
    row, slice checksum, hash16k, set id and packet MD5 of each), drawn
    among jobs whose CPU encode stays within the budget."""
    import random

    from oracle import parity
    from par2rust_b200 import workloads as W

    cost = lambda j: j.slices * j.recovery * (j.slice_size // 2)
    cand = [k for k, j in enumerate(jobs) if cost(j) <= max_macs / n_sample]
    pick = sorted(random.Random(seed).sample(cand, min(n_sample, len(cand))))
    t0 = time.perf_counter()
    bad = {}
    for k in pick:
        j, sp = jobs[k], specs[k]
        rec, ck, h16, pkt, sid = snap[k]
        R, S, n = j.recovery, j.slices, len(j.file_lengths)
        files = [W.file_bytes(sd, ln) for ln, sd in zip(j.file_lengths, j.seeds)]
        rows = rec.view(-1, sp.bufs.rec_stride)[:R, :j.slice_size].cpu().numpy()
        b = parity.check_device_job(files, sp.names, j.slice_size, R, rows, ck[:20 * S].cpu().numpy(),
                                    h16[:16 * n].cpu().numpy().reshape(n, 16), sid, pkt[:16 * R].cpu().numpy())
        if b:
            bad[k] = b[:5]
    return {"result": "bit-exact" if not bad else "MISMATCH", "jobs_checked": pick,
            "macs_checked": sum(cost(jobs[k]) for k in pick), "seconds": time.perf_counter() - t0,
            "what": "every recovery row (GFNI port), slice MD5/CRC32, hash16k, set id and packet MD5 of each "
                    "sampled job against the oracle", "mismatches": bad}


def bench_batch(dev, steps, warmup, plain_steps=1, n_jobs=256, e2e_steps=0):
    """Batched persistent launch vs the same jobs run one after another through
    the plain per-job device path (p2g_run_device_job), both with the sources
    resident in HBM and hash_full left to the host; outputs compared."""
    import torch

    import par2rust_b200 as p2g

    jobs, specs = batch_specs(dev, n_jobs)
    total = sum(j.source_bytes for j in jobs)
    macs = sum(j.slices * j.recovery * (j.slice_size // 2) for j in jobs)
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    batch = p2g.Batch(specs)
    plan_s = time.perf_counter() - t0
    info = batch.info()
    for _ in range(warmup):
        batch.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    batch.check()
    l0 = p2g.kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        batch.launch(stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    batch.check()
    launches = (p2g.kernel_launch_count() - l0) // max(steps, 1)
    ms = ev0.elapsed_time(ev1) / steps
    snap = [(s.bufs.recovery.clone(), s.bufs.checksums.clone(), s.bufs.hash16k.clone(), s.bufs.packet_md5.clone(),
             bytes(s.bufs.set_id_device.cpu().numpy())) for s in specs]

    def plain_step():
        for s in specs:
            p2g.run_device_job(s.src, s.file_lengths, s.names, s.slice_size, s.recovery_count, s.bufs,
                               stream=stream.cuda_stream, skip_hash_full=True)

    plain_step()  # warm: first-call scratch growth
    torch.cuda.synchronize()
    pl0 = p2g.kernel_launch_count()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(plain_steps):
        plain_step()
    b.record(stream)
    torch.cuda.synchronize()
    plain_launches = (p2g.kernel_launch_count() - pl0) // max(plain_steps, 1)
    plain_ms = a.elapsed_time(b) / plain_steps
    same = True
    for s, (rec, ck, h16, pkt, sid) in zip(specs, snap):
        R = s.recovery_count
        rs = s.bufs.rec_stride
        same &= torch.equal(rec.view(-1, rs)[:R, :s.slice_size], s.bufs.recovery.view(-1, rs)[:R, :s.slice_size])
        same &= torch.equal(ck, s.bufs.checksums) and torch.equal(h16, s.bufs.hash16k)
        same &= torch.equal(pkt[:16 * R], s.bufs.packet_md5[:16 * R]) and sid == s.bufs.set_id
    par = batch_parity(jobs, specs, snap)
    out = {
        "parity": par,
        "workload": f"batch_{n_jobs} (mixed jobs: 1-16 files log-uniform in [4 KiB, 64 MiB], slice in "
                    "{16K,64K,256K,1M}, R 1-20% of slices, seed 4)",
        "jobs": n_jobs, "files": sum(len(j.file_lengths) for j in jobs), "source_bytes": total,
        "recovery_bytes": sum(j.recovery * j.slice_size for j in jobs), "gf_macs": macs,
        "batched_gbs": total / (ms * 1e-3) / 1e9, "batched_ms": ms,
        "plain_gbs": total / (plain_ms * 1e-3) / 1e9, "plain_ms": plain_ms,
        "batched_over_plain": plain_ms / ms, "identical_to_plain": bool(same),
        "batched_launches_per_step": launches, "plain_launches_per_step": plain_launches,
        "lut_frac": macs / (ms * 1e-3) / (32 * 148 * 1965e6),
        "plan": {"items": info.items, "encode_items": info.encode_items, "scan_items": info.scan_items,
                 "ctas": info.ctas, "predicted_ms": info.predicted_ms, "plan_and_capture_s": plan_s,
                 "scratch_bytes": info.device_bytes},
        "hash_full": "not on the device in either arm (the host hashes whole files while reading them)",
    }
    if e2e_steps:
        # pinned host sources -> H2D -> batched launch -> D2H of every output
        hosts = [torch.empty(s.src.numel(), dtype=torch.uint8, pin_memory=True) for s in specs]
        for h, s in zip(hosts, specs):
            h.copy_(s.src)
        outs = [(torch.empty(s.bufs.recovery.numel(), dtype=torch.uint8, pin_memory=True),
                 torch.empty(s.bufs.checksums.numel(), dtype=torch.uint8, pin_memory=True),
                 torch.empty(s.bufs.packet_md5.numel(), dtype=torch.uint8, pin_memory=True),
                 torch.empty(s.bufs.hash16k.numel(), dtype=torch.uint8, pin_memory=True),
                 torch.empty(16, dtype=torch.uint8, pin_memory=True)) for s in specs]
        h2d = sum(h.numel() for h in hosts)
        d2h = sum(sum(t.numel() for t in o) for o in outs)

        def e2e_step():
            for h, s in zip(hosts, specs):
                s.src.copy_(h, non_blocking=True)
            batch.launch(stream.cuda_stream)
            for o, s in zip(outs, specs):
                for t, d in zip(o, (s.bufs.recovery, s.bufs.checksums, s.bufs.packet_md5, s.bufs.hash16k,
                                    s.bufs.set_id_device)):
                    t.copy_(d, non_blocking=True)
            torch.cuda.synchronize()

        e2e_step()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        es_serial = (time.perf_counter() - t0) / e2e_steps
        batch.check()

        # the same through StagedBatch: uploads of later groups overlap the
        # running groups, downloads follow each group
        staged = p2g.StagedBatch(specs, hosts, outs, groups=6)

        def staged_step():
            staged.launch(stream.cuda_stream)
            torch.cuda.synchronize()

        staged_step()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            staged_step()
        es = (time.perf_counter() - t0) / e2e_steps
        staged.check()
        same_staged = all(torch.equal(o[0], rec.cpu()) and torch.equal(o[1], ck.cpu()) and torch.equal(o[2], pkt.cpu())
                          for o, (rec, ck, h16, pkt, sid) in zip(outs, snap))
        staged.close()
        out["e2e"] = {"value": total / es / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                      "seconds_per_step": es, "groups": len(staged.ranges), "identical_to_batched": bool(same_staged),
                      "serial_seconds_per_step": es_serial,
                      "api": "StagedBatch (p2g_batch_launch per group) with pinned host sources (H2D overlapped "
                             "with the running groups) and pinned output copies (D2H)"}
    batch.close()
    del specs, snap
    torch.cuda.empty_cache()
    return out


def serve_cpu_baseline(jobs, target_s, threads=0):
    """The CPU port on whole requests of the serving mix, in order, until
    about target_s seconds of CPU work (each request's files as one buffer)."""
    import numpy as np

    from oracle import oracle as orc
    from par2rust_b200 import workloads as W

    done_bytes, spent, n = 0, 0.0, 0
    for j in jobs:
        data = np.concatenate([W.file_bytes(sd, ln) for ln, sd in zip(j.file_lengths, j.seeds)])
        t, *_ = orc.create_timed(data, j.slice_size, j.recovery, threads)
        done_bytes += len(data)
        spent += t
        n += 1
        if spent >= target_s:
            break
    return {"value": done_bytes / spent / 1e9, "unit": "GB/s", "cores": threads or orc.max_threads(), "kind": "port",
            "sample": f"the first {n} requests of the serving mix ({done_bytes} B), each request's files as one "
                      "buffer (scan + encode + packet MD5s)", "seconds": spent}, spent


def serve_parity_pick(jobs, n_sample=8, max_bytes=64 << 20, max_macs=2e11, seed=5):
    """A seeded sample of requests whose oracle check stays cheap (source
    and CPU encode bounded), always including the smallest request."""
    import random

    cost = lambda j: j.slices * j.recovery * (j.slice_size // 2)
    cand = [k for k, j in enumerate(jobs) if j.source_bytes <= max_bytes and cost(j) <= max_macs / n_sample]
    if not cand:
        return set()
    pick = set(random.Random(seed).sample(cand, min(n_sample, len(cand))))
    pick.add(min(cand, key=lambda k: jobs[k].source_bytes))
    return pick


def serve_parity(jobs, kept):
    """Oracle check of the sampled requests' outputs as the serving loop
    returned them mid-sweep: every recovery row (GFNI port), slice MD5/CRC32,
    hash16k, set id and packet MD5."""
    import numpy as np

    from oracle import parity
    from par2rust_b200 import workloads as W

    t0 = time.perf_counter()
    bad = {}
    for i, out in sorted(kept.items()):
        j = jobs[i]
        R, n, sl = j.recovery, len(j.file_lengths), j.slice_size
        files = [W.file_bytes(sd, ln) for ln, sd in zip(j.file_lengths, j.seeds)]
        names = [f"req{i:05d}_f{k:02d}.bin".encode() for k in range(n)]
        rec = (np.frombuffer(b"".join(out["recovery"]), np.uint8).reshape(R, sl) if R
               else np.zeros((0, sl), np.uint8))
        b = parity.check_device_job(files, names, sl, R, rec, np.frombuffer(out["checksums"], np.uint8),
                                    np.frombuffer(out["hash16k"], np.uint8).reshape(n, 16), out["set_id"],
                                    np.frombuffer(out["packet_md5"], np.uint8))
        if b:
            bad[i] = b[:5]
    return {"result": "bit-exact" if not bad else "MISMATCH", "requests_checked": sorted(kept),
            "source_bytes_checked": sum(jobs[i].source_bytes for i in kept), "seconds": time.perf_counter() - t0,
            "mismatches": bad}


def serve_run(srv, jobs, arrivals, p2g, keep=()):
    """Open loop: submit job i at arrivals[i] (server clock from now), a
    poller thread reads each completed job's set id and packet MD5s back and
    releases it; for the requests in `keep` it first copies every output to
    the host (returned under "kept", for the oracle check after the run).
    Returns per-job latencies and totals."""
    import threading

    n = len(jobs)
    lat, done_bytes, d2h = [], [0], [0]
    kept = {}
    last_done = [0.0]
    finished = threading.Event()

    errors = []

    def poller():
        got = 0
        try:
            while got < n:
                for r in srv.poll(wait_ms=20):
                    got += 1
                    if r.status != 0:
                        raise RuntimeError(f"request {r.tag} failed with status {r.status}")
                    if r.tag in keep:
                        kept[r.tag] = out = srv.outputs(r)
                        d2h[0] += sum(len(v) if isinstance(v, bytes) else sum(map(len, v)) for v in out.values())
                    else:
                        p2g.copy_to_host(r.ptr["set_id"], 16)
                        p2g.copy_to_host(r.ptr["packet_md5"], 16 * r.recovery_count)
                        d2h[0] += 16 + 16 * r.recovery_count
                    srv.release(r.ticket)
                    lat.append(r.done_s - r.submit_s)
                    done_bytes[0] += r.source_bytes
                    last_done[0] = max(last_done[0], r.done_s)
        except Exception as e:  # surfaced by the submitting thread
            errors.append(e)
        finished.set()

    th = threading.Thread(target=poller, daemon=True)
    t0 = srv.now()
    th.start()
    for i, (j, at) in enumerate(zip(jobs, arrivals)):
        while True:
            wait = t0 + at - srv.now()
            if wait <= 0:
                break
            time.sleep(min(wait, 0.002))
        names = [f"req{i:05d}_f{k:02d}.bin".encode() for k in range(len(j.file_lengths))]
        srv.submit_seeded(j.file_lengths, j.seeds, names, j.slice_size, j.recovery, tag=i)
        if errors:
            break
    finished.wait()
    th.join()
    if errors:
        raise errors[0]
    span = last_done[0] - t0
    lat.sort()
    pct = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]
    return {"requests": n, "source_bytes": done_bytes[0], "seconds": span, "gbs": done_bytes[0] / span / 1e9,
            "jobs_per_s": n / span, "p50_ms": pct(0.50) * 1e3, "p99_ms": pct(0.99) * 1e3,
            "mean_ms": sum(lat) / len(lat) * 1e3, "max_ms": lat[-1] * 1e3, "d2h_bytes": d2h[0], "kept": kept}


def bench_serve(requests, rate_fracs=(0.5, 0.8, 0.95), rates=None, probe_jobs=200, wave_ms=20.0, seed=5,
                local=0, check_parity=True):
    """The serving loop on the request mix: a closed-batch capacity probe,
    then open-loop Poisson arrivals at each rate (fractions of that capacity
    unless explicit rates are given).  Returns the sweep and its clocks."""
    import par2rust_b200 as p2g
    from par2rust_b200 import workloads as W

    jobs = W.serve_requests(requests, seed=seed)
    budget = 120_000_000_000
    srv = p2g.Server(hbm_budget=budget, wave_ms=wave_ms)
    clocks = ClockSampler(local)
    clocks.start()
    probe = jobs[:min(probe_jobs, len(jobs))]
    pr = serve_run(srv, probe, [0.0] * len(probe), p2g)
    pr.pop("kept")
    cap_jobs = pr["jobs_per_s"]
    rates = list(rates) if rates else [f * cap_jobs for f in rate_fracs]
    keep = serve_parity_pick(jobs, seed=seed) if check_parity else set()
    sweep, kept = [], []
    for ri, rate in enumerate(rates):
        arr = W.poisson_arrivals(len(jobs), rate, seed=100 + ri)
        res = serve_run(srv, jobs, arr, p2g, keep=keep)
        kept.append(res.pop("kept"))
        res["rate_jobs_per_s"] = rate
        res["offered_gbs"] = rate * sum(j.source_bytes for j in jobs) / len(jobs) / 1e9
        st = srv.stats()
        res["waves_total"] = st["waves"]
        res["peak_resident_gb"] = st["peak_resident_bytes"] / 1e9
        sweep.append(res)
        print(json.dumps({"serve_point": res}), file=sys.stderr, flush=True)
    clk = clocks.stop()
    waves = srv.stats()["waves"]
    srv.close()
    for res, kp in zip(sweep, kept):  # outside the sweep: the oracle runs on the host
        res["parity"] = serve_parity(jobs, kp) if keep else None
    parity_all = (None if not keep else
                  "bit-exact" if all(r["parity"]["result"] == "bit-exact" for r in sweep) else "MISMATCH")
    return {
        "workload": f"serve: {len(jobs)} requests per rate, totals log-uniform [1 MiB, 2 GiB] in 1-32 files, "
                    "slice {16K,64K,256K,1M} (smallest with <= 32768 slices), R 1-20% of slices, Poisson arrivals",
        "hbm_budget_bytes": budget, "wave_ms": wave_ms, "requests_per_rate": len(jobs),
        "total_source_bytes": sum(j.source_bytes for j in jobs), "capacity_probe": pr, "sweep": sweep,
        "p50_ms": [r["p50_ms"] for r in sweep], "p99_ms": [r["p99_ms"] for r in sweep],
        "rates_jobs_per_s": [r["rate_jobs_per_s"] for r in sweep], "gbs": [r["gbs"] for r in sweep],
        "clocks": clk, "waves": waves, "jobs": jobs, "parity": parity_all,
        "parity_what": "per rate, a seeded sample of requests (source <= 64 MiB) keeps every output; each is "
                       "checked against the oracle after the sweep: every recovery row, slice MD5/CRC32, hash16k, "
                       "set id and packet MD5",
    }


def run_serve(args, wl):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    rates = [float(x) for x in args.rates.split(",") if x]
    res = bench_serve(args.requests, rates=rates, probe_jobs=args.probe_jobs, wave_ms=args.wave_ms, seed=wl["seed"],
                      local=local, check_parity=not args.no_parity)
    jobs = res.pop("jobs")
    cb = None
    if not args.no_cpu_baseline:
        cb, _ = serve_cpu_baseline(jobs, args.cpu_seconds)
    top = res["sweep"][-1]
    line = {
        "metric": "serving: source GB/s and p50/p99 job latency per arrival rate", "value": top["gbs"],
        "unit": "GB/s", "n_gpus": 1, "steps": len(res["sweep"]), "warmup": 1, "ms_per_step": top["seconds"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
        "data": "synthetic (request bytes generated on the device from per-file seeds)",
        "config": {"workload": res["workload"], "hbm_budget_bytes": res["hbm_budget_bytes"], "wave_ms": args.wave_ms,
                   "total_source_bytes": res["total_source_bytes"], "parallelism": "1 GPU"},
        "capacity_probe": res["capacity_probe"], "sweep": res["sweep"],
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"], "parity": res["parity"],
        "e2e": {"value": top["gbs"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": top["d2h_bytes"],
                "note": "host clock from each request's submit to its completion; sources generated on the device"},
        "roofline": None, "cpu_baseline": cb, "clocks": res["clocks"], "gpu_launches": res["waves"],
    }
    print(json.dumps(line), flush=True)
    return 0


def bench_many(dev, steps, warmup, e2e_steps, cpu_seconds, no_cpu_baseline=False, seed=3, parity_rows=32):
    """many_2000: one create job over 2,000 files with 2,000 recovery blocks
    through the plain per-job device path; its encode alone with both
    kernels; e2e through p2g_create_in_memory; a sampled oracle check."""
    import numpy as np
    import torch

    import par2rust_b200 as p2g
    from par2rust_b200 import workloads as W

    job = W.many_2000(seed=seed)
    sl, R, S = job.slice_size, job.recovery, job.slices
    names = [f"file{i:04d}.bin".encode() for i in range(len(job.file_lengths))]
    src = torch.zeros(S * sl, dtype=torch.uint8, device=dev)
    off = 0
    for n, sd in zip(job.file_lengths, job.seeds):
        src[off:off + n] = W.file_bytes_torch(sd, n, device=dev)
        off += (n + sl - 1) // sl * sl
    bufs = p2g.DeviceJobBuffers(S, len(names), sl, R, dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        p2g.run_device_job(src, job.file_lengths, names, sl, R, bufs, skip_hash_full=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    l0 = p2g.kernel_launch_count()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        p2g.run_device_job(src, job.file_lengths, names, sl, R, bufs, skip_hash_full=True)
    b.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = p2g.kernel_launch_count() - l0
    ms = a.elapsed_time(b) / steps
    total = job.source_bytes
    macs = S * R * (sl // 2)
    # parity of the timed job's outputs (hash_full runs on the host in the timed step)
    from oracle import parity

    files = [W.file_bytes(sd, n) for n, sd in zip(job.file_lengths, job.seeds)]
    out = parity.device_outputs(bufs, S, len(names), sl, R)
    rows = parity.sample_rows(R, parity_rows, seed=seed)
    t0 = time.perf_counter()
    bad = parity.check_device_job(files, names, sl, R, out["rec"], out["checks"], out["hash16k"], bufs.set_id,
                                  out["packet_md5"], rows=rows)
    par = {"result": "bit-exact" if not bad else "MISMATCH", "rows_checked": rows, "seconds": time.perf_counter() - t0,
           "what": f"{len(rows)} sampled recovery rows (0, 1 and {R - 1} always), every slice MD5/CRC32, hash16k, "
                   "the set id and every packet MD5", "mismatches": bad[:10]}
    # the encode alone, each kernel
    enc = {}
    for label, variant in (("lut", p2g.ENCODE_LUT), ("tensor", p2g.ENCODE_TENSOR)):
        ts = []
        for i in range(warmup + steps):
            x, y = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            x.record(stream)
            p2g.encode_device(src.data_ptr(), sl, S, sl, R, bufs.recovery.data_ptr(), bufs.rec_stride,
                              stream.cuda_stream, variant=variant)
            y.record(stream)
            torch.cuda.synchronize()
            if i >= warmup:
                ts.append(x.elapsed_time(y))
        enc[label] = sum(ts) / len(ts)
    e2e = None
    if e2e_steps:
        host = [torch.empty(n, dtype=torch.uint8, pin_memory=True) for n in job.file_lengths]
        for h, f in zip(host, files):
            h.numpy()[:] = f
        opts = p2g.CreateOptions(output="many.par2", slice_size=sl, recovery_block_count=R,
                                 volume_scheme=p2g.VolumeScheme.Uniform(15))
        inputs = list(zip(names, host))
        p2g.create_in_memory(opts, inputs, copy=False)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            got = None  # the previous step's outputs are freed before the next step
            got = p2g.create_in_memory(opts, inputs, copy=False)
        es = (time.perf_counter() - t0) / e2e_steps
        e2e = {"value": total / es / 1e9, "unit": "GB/s", "h2d_bytes_per_step": total,
               "d2h_bytes_per_step": R * sl + S * 20 + 16 * R, "seconds_per_step": es,
               "api": "p2g_create_in_memory (2,000 pinned host files; volumes returned as views "
                      "of the library's buffers, copy=False)", "output_files": len(got)}
        del host, got
    cb = None
    if not no_cpu_baseline:
        from oracle import oracle as orc

        data = np.concatenate(files[:200])
        n_sl = max(1, min(len(data) // sl, int(cpu_seconds * 4)))
        sample = data[:n_sl * sl]
        t, *_ = orc.create_timed(sample, sl, R, 0)
        cb = {"value": len(sample) / t / 1e9, "unit": "GB/s", "cores": orc.max_threads(), "kind": "port",
              "sample": f"{n_sl} slices ({len(sample)} B) of the first files, R={R}", "seconds": t}
    del src, bufs
    torch.cuda.empty_cache()
    lut_peak = 32 * 148 * 1965e6
    return {
        "workload": "many_2000: 2,000 files log-uniform [1 KiB, 8 MiB], slice 262,144, R 2,000, Uniform{15}",
        "files": len(names), "source_bytes": total, "input_slices": S, "recovery_blocks": R, "gf_macs": macs,
        "value": total / (ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": ms, "steps": steps,
        "encode_only_ms": enc, "encode_gf_mac_per_s": {k: macs / (v * 1e-3) for k, v in enc.items()},
        "lut_frac_of_lookup_bound": macs / (enc["lut"] * 1e-3) / lut_peak,
        "tensor_frac_of_nominal_fp4": 2 * 256 * macs / (enc["tensor"] * 1e-3) / 1e12 / FP4_DENSE_TFLOPS,
        "e2e": e2e, "parity": par, "cpu_baseline": cb, "clocks": clk, "gpu_launches": launches,
    }


def run_many(args, wl):
    """--workload many_2000: the dense-contraction job as the measured step."""
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    res = bench_many(dev, args.steps, args.warmup, args.e2e_steps, args.cpu_seconds, args.no_cpu_baseline,
                     seed=wl["seed"])
    line = {
        "metric": "encode source GB/s", "value": res["value"], "unit": "GB/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": res["workload"], "files": res["files"], "source_bytes": res["source_bytes"],
                   "input_slices": res["input_slices"], "recovery_blocks": res["recovery_blocks"],
                   "parallelism": "1 GPU"},
        "e2e": res["e2e"], "parity": res["parity"]["result"], "many_2000": res,
        "cpu_baseline": res["cpu_baseline"], "clocks": res["clocks"], "gpu_launches": res["gpu_launches"],
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_batch(args, wl):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    per_step = max(1.0, min(args.cpu_seconds, 120.0 / max(1, args.steps + args.warmup)))
    vals = []
    cb = None
    for _ in range(args.steps):
        cb, spent = batch_cpu_baseline(per_step)
        vals.append(spent)
    line = {
        "metric": "encode source GB/s (batched)", "value": cb["value"], "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(vals) / len(vals) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "impl": "reference", "config": {"workload": "batch_256", "parallelism": "host threads"},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args, wl):
    S = (wl["length"] + wl["slice"] - 1) // wl["slice"]
    return {"workload": args.workload, "file_bytes": wl["length"], "files": 1, "slice_size": wl["slice"],
            "input_slices": S, "recovery_blocks": wl["R"], "volume_scheme": wl["scheme"],
            "parallelism": f"replicas x{args.gpus} (one independent job per GPU)",
            "l2": "inputs larger than L2: each step reads the whole padded source"}


def batch_cpu_baseline(target_s, threads=0):
    """The CPU port on whole jobs of the mixed batch, in batch order, until
    about target_s seconds of CPU work (each job's files as one buffer)."""
    import numpy as np

    from oracle import oracle as orc
    from par2rust_b200 import workloads as W

    done_bytes, spent, jobs_done = 0, 0.0, 0
    for j in W.batch_256():
        data = np.concatenate([W.file_bytes(sd, n) for n, sd in zip(j.file_lengths, j.seeds)])
        t, *_ = orc.create_timed(data, j.slice_size, j.recovery, threads)
        done_bytes += len(data)
        spent += t
        jobs_done += 1
        if spent >= target_s:
            break
    return {"value": done_bytes / spent / 1e9, "unit": "GB/s", "cores": threads or orc.max_threads(), "kind": "port",
            "sample": f"the first {jobs_done} jobs of the batch ({done_bytes} B), each job's files hashed and encoded "
                      "as one buffer (scan + encode + packet MD5s)", "seconds": spent}, spent


def run_batch(args, wl):
    """--workload batch_256: the batched launch is the measured step."""
    import torch
    import torch.distributed as dist

    import par2rust_b200 as p2g

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    clocks = ClockSampler(local)
    clocks.start()
    res = bench_batch(dev, args.steps, args.warmup, plain_steps=1, n_jobs=args.batch_jobs or wl["n_jobs"],
                      e2e_steps=args.e2e_steps)
    clk = clocks.stop()
    t = torch.tensor([res["batched_ms"]], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * res["source_bytes"] / (ms_max * 1e-3) / 1e9
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, _ = batch_cpu_baseline(args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    hbm_peak, peak_kind = measured_peaks()
    alg = res["source_bytes"] + res["recovery_bytes"]
    line = {
        "metric": "encode source GB/s (batched)", "value": value, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": res["workload"], "jobs": res["jobs"], "files": res["files"],
                   "source_bytes": res["source_bytes"], "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (14.7 GB of sources per step)"},
        "batched": res,
        "e2e": res.get("e2e"),
        "roofline": {"bound": "hbm", "achieved": alg / (ms_max * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": alg / (ms_max * 1e-3) / 1e9 / hbm_peak, "traffic": None, "peak_source": peak_kind,
                     "kernel": "batch_kernel (whole step)", "algorithmic_bytes": alg},
        "lut_roofline": {"achieved": res["gf_macs"] / (ms_max * 1e-3), "peak": 32 * 148 * 1965e6,
                         "unit": "GF(2^16) MAC/s", "frac": res["lut_frac"]},
        "cpu_baseline": cb, "clocks": clk, "gpu_launches": res["batched_launches_per_step"] * args.steps,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        if wl.get("serve"):
            rank, _, _ = dist_env()
            if rank != 0:
                return 0
            from par2rust_b200 import workloads as W

            cb, spent = serve_cpu_baseline(W.serve_requests(args.requests, seed=wl["seed"]), args.cpu_seconds)
            print(json.dumps({"metric": "serving: source GB/s and p50/p99 job latency per arrival rate",
                              "value": cb["value"], "unit": "GB/s", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
                              "ms_per_step": spent * 1e3, "higher_is_better": True, "scaling": "weak",
                              "vs_baseline": None, "dtype": "u16", "data": "synthetic", "impl": "reference",
                              "config": {"workload": "serve"}, "cpu_baseline": cb,
                              "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        if wl.get("batch"):
            return run_reference_batch(args, wl)
        if wl.get("many"):
            rank, _, _ = dist_env()
            if rank != 0:
                return 0
            import numpy as np

            from oracle import oracle as orc
            from par2rust_b200 import workloads as W

            job = W.many_2000(seed=wl["seed"])
            data = np.concatenate([W.file_bytes(sd, n) for n, sd in list(zip(job.file_lengths, job.seeds))[:200]])
            n_sl = max(1, min(len(data) // job.slice_size, int(args.cpu_seconds * 4)))
            sample = data[:n_sl * job.slice_size]
            ts = [orc.create_timed(sample, job.slice_size, job.recovery, 0)[0] for _ in range(max(1, args.steps))]
            v = len(sample) / (sum(ts) / len(ts)) / 1e9
            print(json.dumps({"metric": "encode source GB/s", "value": v, "unit": "GB/s", "n_gpus": args.gpus,
                              "steps": args.steps, "warmup": 0, "ms_per_step": sum(ts) / len(ts) * 1e3,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
                              "data": "synthetic", "impl": "reference", "config": {"workload": "many_2000"},
                              "cpu_baseline": {"value": v, "unit": "GB/s", "cores": orc.max_threads(), "kind": "port",
                                               "sample": f"{n_sl} slices of the first files, R={job.recovery}"},
                              "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
                  flush=True)
            return 0
        return run_reference(args, wl)
    if wl.get("batch"):
        return run_batch(args, wl)
    if wl.get("serve"):
        return run_serve(args, wl)
    if wl.get("many"):
        return run_many(args, wl)

    import numpy as np
    import torch
    import torch.distributed as dist

    import par2rust_b200 as p2g
    from par2rust_b200 import workloads as W

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    L, slice_, R = wl["length"], wl["slice"], wl["R"]
    S = (L + slice_ - 1) // slice_
    name = b"source.bin"
    info = p2g.device_info()

    # source: seeded bytes generated on the device into a slice-padded buffer
    seed = W.file_seed(wl["seed"], rank, 0)
    src = torch.zeros(S * slice_, dtype=torch.uint8, device=dev)
    src[:L] = W.file_bytes_torch(seed, L, device=dev)
    bufs = p2g.DeviceJobBuffers(S, 1, slice_, R, dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()


    # ---- value: device-resident job ----
    for _ in range(args.warmup):
        p2g.run_device_job(src, [L], [name], slice_, R, bufs, skip_hash_full=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = p2g.kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        p2g.run_device_job(src, [L], [name], slice_, R, bufs, skip_hash_full=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = p2g.kernel_launch_count() - launches0
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * L / (ms_max * 1e-3) / 1e9

    # ---- parity of the timed step: every output of the last step ----
    parity_res = None
    if rank == 0 and not args.no_parity:
        from oracle import parity

        t0 = time.perf_counter()
        data_np = src[:L].cpu().numpy()
        out = parity.device_outputs(bufs, S, 1, slice_, R)
        bad = parity.check_device_job([data_np], [name], slice_, R, out["rec"], out["checks"], out["hash16k"],
                                      bufs.set_id, out["packet_md5"])
        parity_res = {"result": "bit-exact" if not bad else "MISMATCH", "seconds": time.perf_counter() - t0,
                      "what": "the last timed step's outputs: all recovery rows (oracle GFNI port, pinned to the "
                              "scalar restatement), every slice MD5/CRC32, hash16k, the set id and every packet MD5",
                      "mismatches": bad[:10]}
        del data_np, out

    # ---- the encode alone, each kernel (CUDA events per launch) ----
    def encode_ms(variant, env=None):
        if env:
            os.environ.update(env)
        ts = []
        for i in range(args.warmup + args.steps):
            x, y = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            x.record(stream)
            p2g.encode_device(src.data_ptr(), slice_, S, slice_, R, bufs.recovery.data_ptr(), bufs.rec_stride,
                              stream.cuda_stream, variant=variant)
            y.record(stream)
            torch.cuda.synchronize()
            if i >= args.warmup:
                ts.append(x.elapsed_time(y))
        for k in env or {}:
            del os.environ[k]
        return sum(ts) / len(ts)

    enc_lut = encode_ms(p2g.ENCODE_LUT)
    enc_derive = encode_ms(p2g.ENCODE_LUT, {"P2G_ENCODE_BASIS": "derive"})
    enc_tensor = encode_ms(p2g.ENCODE_TENSOR)
    hbm_peak, peak_kind = measured_peaks()
    alg_bytes = S * slice_ + R * slice_  # padded source read once + recovery written once
    macs = S * R * (slice_ // 2)
    lut_peak = 32 * 148 * 1965e6  # 2 shared-memory u16 lookups per MAC at 128 B/clk/SM, max clock
    # which encode the step's plan runs: the planner reports tensor-core items with fold 0
    plan_items, _, _ = p2g.plan_device_job(slice_, S, R)
    step_tensor = bool(plan_items) and all(it["fold"] == 0 for it in plan_items)
    traffic = None  # DRAM bytes per batch_kernel launch (ncu, profiles/)
    tp = os.path.join(ROOT, "profiles", "batch_kernel_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get(args.workload)
        except Exception:
            traffic = None

    # ---- e2e: public API with pinned host input ----
    host_src = torch.empty(L, dtype=torch.uint8, pin_memory=True)
    host_src.copy_(src[:L])
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=slice_, recovery_block_count=R,
                             volume_scheme=p2g.VolumeScheme.Exponential() if wl["scheme"] == "exponential"
                             else p2g.VolumeScheme.Single())
    e2e_val, e2e_s, files = None, None, []
    if args.e2e_steps > 0:
        p2g.create_in_memory(opts, [(name, host_src)], copy=False)  # warm
        barrier()
        e2e_t = []
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            files = None  # the previous step's outputs are freed before the next step
            files = p2g.create_in_memory(opts, [(name, host_src)], copy=False)
            torch.cuda.synchronize()
            e2e_t.append(time.perf_counter() - t0)
        et = torch.tensor([sum(e2e_t) / len(e2e_t)], device=dev)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e_s = float(et.item())
        e2e_val = world * L / e2e_s / 1e9

    # ---- the same through the file API: source file in, .par2 files out ----
    e2e_files = None
    if args.e2e_steps > 0 and rank == 0 and world == 1:
        import tempfile

        with tempfile.TemporaryDirectory(prefix="p2g_bench_") as td:
            sp = os.path.join(td, "source.bin")
            host_src.numpy().tofile(sp)
            fopts = p2g.CreateOptions(output=os.path.join(td, "recovery.par2"), slice_size=slice_, recovery_block_count=R,
                                      volume_scheme=opts.volume_scheme)
            p2g.run_create_fused(fopts, [(sp, name)])  # warm (page cache, pinned buffers)
            ft = []
            for _ in range(args.e2e_steps):
                t0 = time.perf_counter()
                written = p2g.run_create_fused(fopts, [(sp, name)])
                ft.append(time.perf_counter() - t0)
            fs = sum(ft) / len(ft)
            e2e_files = {"value": L / fs / 1e9, "unit": "GB/s", "seconds_per_step": fs,
                         "api": "p2g_run_create_fused (source file mapped from the page cache; index and "
                                f"{len(written) - 1} volume files written to a temporary directory)",
                         "bytes_written": sum(os.path.getsize(w) for w in written)}
    d2h = R * slice_ + S * 20 + 16 * R + 32

    # device single-chain MD5 rate (the whole-file hash on the device)
    chain_gbs = None
    if not args.no_extras:
        t0 = time.perf_counter()
        p2g.run_device_job(src[:64 * 1024 * 1024], [64 * 1024 * 1024], [name], slice_, 0, None)
        torch.cuda.synchronize()
        chain_gbs = 64 * 1024 * 1024 / (time.perf_counter() - t0) / 1e9
    del src, bufs
    torch.cuda.empty_cache()

    # ---- batched persistent launch vs the plain path on the mixed batch ----
    batched = None
    if world == 1 and not args.no_batch:
        batched = bench_batch(dev, args.steps, args.warmup, plain_steps=1, n_jobs=args.batch_jobs)

    # ---- the dense contraction: 2,000 files, R 2,000 ----
    many = None
    if world == 1 and not args.no_many:
        many = bench_many(dev, max(2, args.steps // 3), args.warmup, 1 if args.e2e_steps else 0,
                          max(2.0, args.cpu_seconds / 3), args.no_cpu_baseline)

    # ---- serving: p50/p99 job latency at two arrival rates ----
    serving = None
    if world == 1 and args.serve_requests > 0:
        serving = bench_serve(args.serve_requests, rate_fracs=tuple(float(x) for x in args.serve_fracs.split(",")),
                              local=local, check_parity=not args.no_parity)
        serving.pop("jobs")

    # ---- CPU baseline (rank 0, N=1) ----
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, _ = cpu_baseline(host_src.numpy(), wl, target_s=args.cpu_seconds)
        # and on one core, on a shorter sample (the scalar chains set the pace)
        c1, _ = cpu_baseline(host_src.numpy(), wl, target_s=max(2.0, args.cpu_seconds / 4), threads=1)
        cb["one_thread"] = {"value": c1["value"], "unit": c1["unit"], "seconds_per_step": c1["seconds_per_step"],
                            "sample": c1["sample"]}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    step_macs = macs / (ms_max * 1e-3)
    lookup_roofline = {"bound": "smem", "achieved": step_macs, "peak": lut_peak, "unit": "GF(2^16) MAC/s",
                       "frac": step_macs / lut_peak,
                       "peak_source": "computed: 2 shared-memory u16 lookups per GF MAC at 128 B/clk/SM, 148 SMs, "
                                      "1965 MHz (the lookup kernel's design bound)"}
    kernel_note = ("batch_kernel (one launch per step: encode items, slice MD5/CRC32, packet-MD5 chains) + "
                   + ("a_image_kernel" if step_tensor else "basis_kernel")
                   + "; timed per step with events on the launching stream")
    if step_tensor:
        # 16 x 16 e2m1 products (mul + add) per GF MAC on the tensor pipe
        step_tflops = 2 * 256 * macs / (ms_max * 1e-3) / 1e12
        roofline = {"bound": "tensor", "achieved": step_tflops, "peak": FP4_DENSE_TFLOPS, "unit": "TFLOP/s",
                    "frac": step_tflops / FP4_DENSE_TFLOPS, "traffic": traffic,
                    "peak_source": "nominal dense FP4 (kind::mxf4) rate of B200; MEASURED_PEAKS.json holds no FP4 "
                                   "figure (its bf16 GEMM: %s TFLOP/s)" % measured_bf16(),
                    "kernel": kernel_note + "; encode items on tcgen05 kind::mxf4", "kernel_ms": ms_max,
                    "macs_per_launch": macs, "e2m1_flop_per_launch": 2 * 256 * macs}
    else:
        roofline = dict(lookup_roofline, traffic=traffic, kernel=kernel_note, kernel_ms=ms_max, macs_per_launch=macs)
    line = {
        "metric": "encode source GB/s", "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_E2E_GBS, "dtype": "u16", "data": "synthetic",
        "config": config_dict(args, wl),
        "parity": parity_res["result"] if parity_res else None,
        "parity_detail": parity_res,
        "e2e": {"value": e2e_val, "unit": "GB/s", "h2d_bytes_per_step": L, "d2h_bytes_per_step": d2h,
                "seconds_per_step": e2e_s, "api": "p2g_create_in_memory (pinned host source; volumes returned as views of "
                "the library's buffers, copy=False)",
                "output_files": len(files)},
        "e2e_files": e2e_files,
        # the binding unit of the timed step's encode: the tensor pipe (tcgen05
        # items) or the shared-memory lookups (lookup-table items)
        "roofline": roofline,
        "step_encode": "tensor" if step_tensor else "lut",
        "lookup_roofline": lookup_roofline,
        "hbm_roofline": {"bound": "hbm", "achieved": alg_bytes / (ms_max * 1e-3) / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": alg_bytes / (ms_max * 1e-3) / 1e9 / hbm_peak, "traffic": traffic,
                         "peak_source": peak_kind, "algorithmic_bytes": alg_bytes},
        "encode_only": {
            "lut": {"kernel": "basis_kernel + encode_lut_kernel (p2g_encode, one launch)", "kernel_ms": enc_lut,
                    "gf_mac_per_s": macs / (enc_lut * 1e-3), "frac_of_lookup_bound": macs / (enc_lut * 1e-3) / lut_peak,
                    "kernel_ms_basis_derived": enc_derive},
            "tensor": {"kernel": "a_image_kernel + encode_mma_kernel (tcgen05 kind::mxf4, p2g_encode)",
                       "kernel_ms": enc_tensor, "gf_mac_per_s": macs / (enc_tensor * 1e-3),
                       "e2m1_tflops": 2 * 256 * macs / (enc_tensor * 1e-3) / 1e12,
                       "frac_of_nominal_fp4": 2 * 256 * macs / (enc_tensor * 1e-3) / 1e12 / FP4_DENSE_TFLOPS}},
        "cpu_baseline": cb,
        "clocks": clk,
        "gpu_launches": launches,
        "file_md5_device_chain_gbs": chain_gbs,
        "batched": batched,
        "many_2000": many,
        "serving": serving,
        "device": info,
        "baseline_note": "vs_baseline divides by the reference's published end-to-end create rate for this "
                         "shape (0.0975 GB/s, Apple M4, 10 threads)",
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
