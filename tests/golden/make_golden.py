#!/usr/bin/env python3
"""Regenerates tests/golden/golden.json from the CPU oracle.

The reference crate cannot be built here (Rust toolchain absent, crates not
vendored), so golden outputs come from oracle/par2_oracle.c after it has
been pinned against the reference's own known answers (tests/test_oracle.py:
RFC 1321 MD5 vectors, the CRC-32 check value, GF sentinels, base/coefficient
tables, the GFNI all-symbol check, scan/packet/volume layouts) and three
independent MD5s.  Inputs are deterministic: the reference's fixture LCG
(tests/common/mod.rs:46-57) or fixed byte patterns from the reference tests.

    python tests/golden/make_golden.py      # rewrites golden.json
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from par2rust_b200.workloads import deterministic_bytes  # noqa: E402

PAYLOAD = bytes(((i * 101) & 0xFF) for i in range(17 * 1024 + 37))  # creator.rs:1853-1855

# name: (inputs as (display name, generator spec), slice, R, scheme kwargs, comments)
CASES = {
    "hello_r2": ([("a.bin", "text:hello par2 world!!!!")], 4, 2, {}, []),
    "payload_single_r4": ([("p.bin", "payload")], 4096, 4, {}, []),
    "payload_exp_r11": ([("p.bin", "payload")], 4096, 11, {"kind": oracle.SCHEME_EXPONENTIAL}, []),
    "payload_index_only": ([("p.bin", "payload")], 4096, 0, {}, []),
    "lcg_multi_uniform": ([("one.bin", "lcg:1:5000"), ("two.bin", "lcg:2:300"), ("three.bin", "lcg:3:12288")],
                          1024, 7, {"kind": oracle.SCHEME_UNIFORM, "count": 3}, ["golden comment", "naïve"]),
    "lcg_odd_slice_r37": ([("z", "lcg:6:1001"), ("w", "lcg:7:77")], 20, 37, {}, []),
    "lcg_exp_r64": ([("big.bin", "lcg:9:70000")], 2048, 64, {"kind": oracle.SCHEME_EXPONENTIAL}, []),
}


def make_bytes(spec: str) -> bytes:
    if spec == "payload":
        return PAYLOAD
    if spec.startswith("text:"):
        return spec[5:].encode()
    _, seed, n = spec.split(":")
    return deterministic_bytes(int(seed), int(n))


def main():
    lg, al = oracle.gf_tables()
    out = {
        "gf": {
            "log_sha256": hashlib.sha256(b"".join(x.to_bytes(2, "little") for x in lg)).hexdigest(),
            "antilog_sha256": hashlib.sha256(b"".join(x.to_bytes(2, "little") for x in al)).hexdigest(),
            "first_bases": oracle.input_bases(64),
            "bases_32768_sha256": hashlib.sha256(
                b"".join(x.to_bytes(2, "little") for x in oracle.input_bases(32768))).hexdigest(),
        },
        "md5": {"": oracle.md5(b"").hex(), "abc": oracle.md5(b"abc").hex()},
        "crc32_check": oracle.crc32(b"123456789"),
        "encode_small": {},
        "creates": {},
    }
    src = deterministic_bytes(42, 3 * 8)
    out["encode_small"] = {"src": src.hex(), "S": 3, "slice": 8, "R": 4,
                           "recovery": bytes(oracle.encode(src, 3, 8, 4)).hex()}
    for name, (inputs, slice_, R, kw, comments) in CASES.items():
        ins = [(n.encode(), make_bytes(spec)) for n, spec in inputs]
        files = oracle.create(ins, slice_, R, comments=comments, **kw)
        out["creates"][name] = {
            "inputs": inputs, "slice": slice_, "R": R, "scheme": kw, "comments": comments,
            "files": [{"name": n, "length": len(b), "sha256": hashlib.sha256(b).hexdigest(),
                       **({"hex": b.hex()} if len(b) <= 2048 else {})} for n, b in files],
        }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
