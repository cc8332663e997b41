"""Device-output checks against the CPU oracle -- TEST INFRASTRUCTURE.

Used by tests/ and by bench.py's parity check of the workloads it times
(outside every timed region).  Nothing here is on the product path: it only
compares what the library produced with what the oracle computes for the
same input bytes.

check_device_job() takes one create job's device outputs (copied to host
numpy arrays) and returns a list of mismatch descriptions; an empty list
means bit-exact.  Recovery rows are compared either all (the GFNI port
encode, itself pinned to the scalar restatement of src/reedsolomon.rs:87-126
by tests/test_oracle.py) or on a given set of rows (oracle.encode_rows).
Slice checksums, hash16k, hash_full and file ids follow src/source.rs:145-309
(oracle.scan); the set id src/packet/main_packet.rs:25-42; packet MD5s
src/packet/recovery.rs:11-19 over the device's own rows.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from . import oracle as orc


def padded_source(files: Sequence[np.ndarray], slice_size: int) -> np.ndarray:
    """The files back to back in caller order, each zero-padded to whole
    slices: the encoder's input (src/creator.rs:895-900)."""
    S = sum((len(f) + slice_size - 1) // slice_size for f in files)
    out = np.zeros(S * slice_size, dtype=np.uint8)
    off = 0
    for f in files:
        out[off:off + len(f)] = f
        off += (len(f) + slice_size - 1) // slice_size * slice_size
    return out


def check_device_job(files: Sequence[np.ndarray], names: Sequence[bytes], slice_size: int, R: int,
                     rec: np.ndarray, checks: np.ndarray, hash16k: np.ndarray, set_id: bytes,
                     packet_md5: np.ndarray, hash_full: Optional[np.ndarray] = None,
                     rows: Optional[Sequence[int]] = None, first_exponent: int = 0) -> List[str]:
    """Mismatches between one job's device outputs and the oracle.

    rec: R x slice_size recovery rows; checks: S x 20 IFSC records; hash16k /
    hash_full: n x 16; packet_md5: R x 16.  rows=None compares every row."""
    bad: List[str] = []
    S = sum((len(f) + slice_size - 1) // slice_size for f in files)
    want_checks, fids = [], []
    for k, (f, name) in enumerate(zip(files, names)):
        st, cks, hf, h16, fid = orc.scan(np.ascontiguousarray(f, dtype=np.uint8), slice_size, name)
        if st != 0:
            bad.append(f"oracle scan of file {k} failed ({st})")
            return bad
        want_checks += cks
        fids.append(fid)
        if bytes(hash16k[k]) != h16:
            bad.append(f"hash16k of file {k}")
        if hash_full is not None and bytes(hash_full[k]) != hf:
            bad.append(f"hash_full of file {k}")
    got = checks.reshape(S, 20)
    for s, (md5, crc) in enumerate(want_checks):
        if bytes(got[s, :16]) != md5 or int.from_bytes(bytes(got[s, 16:20]), "little") != crc:
            bad.append(f"slice checksum {s}")
            if len(bad) > 20:
                return bad
    sid = orc.set_id(slice_size, fids)
    if sid != set_id:
        bad.append("set id")
    if R == 0:
        return bad
    src = padded_source(files, slice_size)
    rec = rec.reshape(R, slice_size)
    if rows is None and first_exponent == 0:
        want = orc.encode_fast(src, S, slice_size, R).reshape(R, slice_size)
        rows = list(range(R))
    else:
        rows = list(range(R)) if rows is None else sorted(set(rows))
        want = np.zeros((R, slice_size), dtype=np.uint8)
        want[rows] = orc.encode_rows(src, S, slice_size, [first_exponent + r for r in rows])
    for r in rows:
        if not np.array_equal(rec[r], want[r]):
            bad.append(f"recovery row {r}")
            if len(bad) > 20:
                return bad
    pm = packet_md5.reshape(R, 16)
    for r in range(R):
        if bytes(pm[r]) != orc.recovery_packet_md5(sid, first_exponent + r, rec[r]):
            bad.append(f"packet md5 {r}")
            if len(bad) > 20:
                return bad
    return bad


def sample_rows(R: int, n: int, seed: int) -> List[int]:
    """Rows 0, 1 and R-1 plus a seeded sample, n in all (or every row)."""
    if R <= n:
        return list(range(R))
    rng = np.random.default_rng(seed)
    pick = {0, 1, R - 1}
    while len(pick) < n:
        pick.add(int(rng.integers(0, R)))
    return sorted(pick)


def device_outputs(bufs, S: int, n_files: int, slice_size: int, R: int) -> dict:
    """Host copies of a DeviceJobBuffers' outputs, shaped for check_device_job."""
    rs = bufs.rec_stride
    rec = bufs.recovery.view(-1, rs)[:R, :slice_size].cpu().numpy() if R else np.zeros((0, slice_size), np.uint8)
    return {"rec": rec, "checks": bufs.checksums[:20 * S].cpu().numpy(),
            "hash16k": bufs.hash16k[:16 * n_files].cpu().numpy().reshape(n_files, 16),
            "hash_full": bufs.hash_full[:16 * n_files].cpu().numpy().reshape(n_files, 16),
            "packet_md5": bufs.packet_md5[:16 * max(R, 1)].cpu().numpy()[:16 * R]}
