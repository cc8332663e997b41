"""Committed golden vectors (tests/golden/golden.json, made by
tests/golden/make_golden.py): the oracle must keep reproducing them (CPU) and
the device path must produce the same bytes (GPU)."""
import hashlib
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import make_bytes  # noqa: E402

G = json.load(open(os.path.join(HERE, "golden", "golden.json")))


def test_oracle_reproduces_gf_and_hash_vectors(oracle):
    lg, al = oracle.gf_tables()
    assert hashlib.sha256(b"".join(x.to_bytes(2, "little") for x in lg)).hexdigest() == G["gf"]["log_sha256"]
    assert hashlib.sha256(b"".join(x.to_bytes(2, "little") for x in al)).hexdigest() == G["gf"]["antilog_sha256"]
    assert oracle.input_bases(64) == G["gf"]["first_bases"]
    assert oracle.md5(b"abc").hex() == G["md5"]["abc"] == "900150983cd24fb0d6963f7d28e17f72"
    assert oracle.crc32(b"123456789") == G["crc32_check"] == 0xCBF43926
    e = G["encode_small"]
    assert bytes(oracle.encode(bytes.fromhex(e["src"]), e["S"], e["slice"], e["R"])).hex() == e["recovery"]


@pytest.mark.parametrize("name", sorted(G["creates"]))
def test_oracle_reproduces_creates(oracle, name):
    c = G["creates"][name]
    ins = [(n.encode(), make_bytes(spec)) for n, spec in c["inputs"]]
    files = oracle.create(ins, c["slice"], c["R"], comments=c["comments"], **c["scheme"])
    assert [(n, len(b), hashlib.sha256(b).hexdigest()) for n, b in files] == \
        [(f["name"], f["length"], f["sha256"]) for f in c["files"]]


def _scheme(p2g, kw):
    kind = kw.get("kind", 0)
    if kind == 1:
        return p2g.VolumeScheme.Exponential()
    if kind == 2:
        return p2g.VolumeScheme.Uniform(kw["count"])
    return p2g.VolumeScheme.Single()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(G["creates"]))
def test_device_reproduces_golden_creates(p2g, gpu, name):
    c = G["creates"][name]
    ins = [(n.encode(), make_bytes(spec)) for n, spec in c["inputs"]]
    opts = p2g.CreateOptions(output="recovery.par2", slice_size=c["slice"], recovery_block_count=c["R"],
                             volume_scheme=_scheme(p2g, c["scheme"]), comments=c["comments"])
    files = p2g.create_in_memory(opts, ins)
    assert [(n, len(b), hashlib.sha256(b).hexdigest()) for n, b in files] == \
        [(f["name"], f["length"], f["sha256"]) for f in c["files"]]
    for (n, b), f in zip(files, c["files"]):
        if "hex" in f:
            assert b.hex() == f["hex"]


@pytest.mark.gpu
def test_device_reproduces_encode_small(p2g, gpu):
    e = G["encode_small"]
    assert bytes(p2g.encode(bytes.fromhex(e["src"]), e["slice"], e["R"])).hex() == e["recovery"]
