"""The tensor-core (tcgen05, kind::mxf4) encode against the oracle and the
lookup kernel.

Shapes cover a single slice, R = 1, one and two 8-row halves of a 16-row
tile (R = 8, 9, 16, 17), a last symbol tile of 8 symbols (Np = 248), ragged
slices (4,100 B: 2,056 symbols), slice counts that are not a multiple of the
4-slice K-step, non-zero first exponents, and a 538 MB-like slice size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [  # (S, slice, R, first_exponent)
    (1, 64, 1, 0), (1, 496, 8, 0), (2, 496, 9, 0), (3, 4096, 16, 0), (5, 4096, 17, 0), (6, 960, 33, 0),
    (7, 4100, 20, 0), (9, 2048, 48, 7), (13, 65536, 3, 65530), (37, 65536, 200, 0), (64, 8192, 129, 100),
]


@pytest.mark.parametrize("S,slice_,R,fe", SHAPES)
def test_tensor_encode_matches_oracle(p2g, gpu, oracle, S, slice_, R, fe):
    from par2rust_b200.workloads import file_bytes

    src = file_bytes(7 * S + R, S * slice_)
    got = p2g.encode(src, slice_, R, first_exponent=fe, variant=p2g.ENCODE_TENSOR).reshape(R, slice_)
    if fe == 0:
        want = oracle.encode_fast(src, S, slice_, R).reshape(R, slice_)
    else:
        want = oracle.encode_rows(src, S, slice_, [fe + r for r in range(R)])
    assert np.array_equal(got, want)


def test_tensor_encode_equals_lut_on_device(p2g, gpu):
    """Device pointers, 256 slices x 512 KiB, R 200: both kernels, same bytes,
    and bytes past the padded row untouched."""
    import torch

    S, sl, R = 256, 524288, 200
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    src = torch.randint(0, 256, (S * sl,), dtype=torch.uint8, device="cuda", generator=g)
    rs = sl + 64
    a = torch.full((R * rs,), 0x33, dtype=torch.uint8, device="cuda")
    b = torch.full((R * rs,), 0x33, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    p2g.encode_device(src.data_ptr(), sl, S, sl, R, a.data_ptr(), rs, stream, variant=p2g.ENCODE_LUT, wait=True)
    p2g.encode_device(src.data_ptr(), sl, S, sl, R, b.data_ptr(), rs, stream, variant=p2g.ENCODE_TENSOR, wait=True)
    torch.cuda.synchronize()
    assert torch.equal(a.view(R, rs)[:, :sl], b.view(R, rs)[:, :sl])
    assert bool((b.view(R, rs)[:, sl:] == 0x33).all())


def test_tensor_encode_large_sums_stay_exact(p2g, gpu, oracle):
    """All-ones sources make every product sum as large as the data allows
    (about half of the 16 S terms of each dot product): 8,192 slices take the
    fp32 sums to ~65,000, where a lossy accumulator would flip parities."""
    S, sl, R = 8192, 64, 40
    src = np.full(S * sl, 0xFF, dtype=np.uint8)
    got = p2g.encode(src, sl, R, variant=p2g.ENCODE_TENSOR).reshape(R, sl)
    want = oracle.encode_fast(src, S, sl, R).reshape(R, sl)
    assert np.array_equal(got, want)


DEVICE_JOB_SHAPES = [  # (file lengths, slice, R): tail split, ragged slices, several files, R % 16 != 0
    ([100 * 524288 - 777], 524288, 200), ([600 * 4100 - 3], 4100, 100), ([100 * 65540], 65540, 30),
    ([70_001, 4096 * 9, 123], 4096, 17), ([16_777_216], 65536, 32),
]


@pytest.mark.parametrize("lengths,slice_,R", DEVICE_JOB_SHAPES)
def test_device_job_on_tensor_cores_matches_oracle(p2g, gpu, oracle, lengths, slice_, R):
    """The whole device job (persistent kernel with tensor-core encode items,
    packet-MD5 chains per band, the tail split's accumulating pieces) against
    the oracle: every row, checksum, hash and packet MD5."""
    import torch

    from oracle import parity
    from par2rust_b200.workloads import file_bytes

    files = [file_bytes(31 * k + R, n) for k, n in enumerate(lengths)]
    src = torch.from_numpy(parity.padded_source(files, slice_)).cuda()
    names = [f"f{k}.bin".encode() for k in range(len(files))]
    S = src.numel() // slice_
    bufs = p2g.run_device_job(src, lengths, names, slice_, R, variant=p2g.ENCODE_TENSOR)
    torch.cuda.synchronize()
    out = parity.device_outputs(bufs, S, len(files), slice_, R)
    bad = parity.check_device_job(files, names, slice_, R, out["rec"], out["checks"], out["hash16k"], bufs.set_id,
                                  out["packet_md5"], hash_full=out["hash_full"])
    assert not bad, bad


@pytest.mark.parametrize("variant", ["tensor", "lut"])
def test_device_encodes_on_two_streams_keep_their_scratch_apart(p2g, gpu, variant):
    """Two device-pointer encodes with different exponents on two streams,
    issued back to back: the library's coefficient scratch is shared, so the
    second waits for the first; each result equals the same encode alone."""
    import torch

    v = p2g.ENCODE_TENSOR if variant == "tensor" else p2g.ENCODE_LUT
    S, sl, R = 96, 65536, 40
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    src = torch.randint(0, 256, (S * sl,), dtype=torch.uint8, device="cuda", generator=g)
    alone = []
    for fe in (0, 9000):
        out = torch.zeros(R * sl, dtype=torch.uint8, device="cuda")
        p2g.encode_device(src.data_ptr(), sl, S, sl, R, out.data_ptr(), sl, torch.cuda.current_stream().cuda_stream,
                          variant=v, wait=True, first_exponent=fe)
        alone.append(out)
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    a = torch.zeros(R * sl, dtype=torch.uint8, device="cuda")
    b = torch.zeros(R * sl, dtype=torch.uint8, device="cuda")
    for _ in range(3):
        p2g.encode_device(src.data_ptr(), sl, S, sl, R, a.data_ptr(), sl, s1.cuda_stream, variant=v, first_exponent=0)
        p2g.encode_device(src.data_ptr(), sl, S, sl, R, b.data_ptr(), sl, s2.cuda_stream, variant=v,
                          first_exponent=9000)
    torch.cuda.synchronize()
    assert torch.equal(a, alone[0]) and torch.equal(b, alone[1])


def test_device_jobs_on_two_streams_keep_their_scratch_apart(p2g, gpu):
    """Two device jobs (different sources) issued back to back on two streams
    share the library's descriptor, A image and staging buffers: each must
    give what it gives alone."""
    import torch

    sl, L = 65536, 96 * 65536 - 1000
    S = (L + sl - 1) // sl
    srcs = []
    for seed in (1, 2):
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        t = torch.zeros(S * sl, dtype=torch.uint8, device="cuda")
        t[:L] = torch.randint(0, 256, (L,), dtype=torch.uint8, device="cuda", generator=g)
        srcs.append(t)
    alone = []
    for t in srcs:
        bufs = p2g.run_device_job(t, [L], [b"f.bin"], sl, 40, skip_hash_full=True)
        torch.cuda.synchronize()
        alone.append((bufs.recovery.clone(), bufs.packet_md5.clone(), bufs.checksums.clone()))
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    got = []
    for t, st in zip(srcs, (s1, s2)):
        got.append(p2g.run_device_job(t, [L], [b"f.bin"], sl, 40, stream=st.cuda_stream, skip_hash_full=True))
    torch.cuda.synchronize()
    for b, (rec, pkt, cks) in zip(got, alone):
        assert torch.equal(b.recovery, rec) and torch.equal(b.packet_md5, pkt) and torch.equal(b.checksums, cks)
