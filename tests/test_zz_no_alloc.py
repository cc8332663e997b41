"""p2g_encode_noalloc: the encode for callers that cannot let the library
allocate device memory (their allocator or memory pool owns every byte, or
a cudaMalloc would synchronise the device on a latency-critical path).

It must give exactly the bytes of the regular entry point, p2g_encode, on
consecutive calls that share its fixed scratch array, and refuse jobs whose
scratch would not fit.  This file is collected last on purpose and also
passes on its own in a fresh process (the first call does the per-device
set-up).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _job(_ffi, src, S, slice_, R, rec, stream):
    return _ffi.p2g_encode_job(src=src.data_ptr(), src_stride=slice_, input_count=S, slice_size=slice_,
                               recovery_count=R, first_exponent=0, recovery=rec.data_ptr(), recovery_stride=slice_,
                               flags=1, stream=stream)


def test_noalloc_matches_encode_on_two_calls(p2g, gpu):
    import torch

    from par2rust_b200 import _ffi
    from par2rust_b200.workloads import file_bytes

    lib = _ffi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    shapes = [(37, 65536, 200), (5, 4096, 33)]  # two calls in a row, different sizes and contents
    for call, (S, slice_, R) in enumerate(shapes):
        src = torch.from_numpy(file_bytes(1000 + call, S * slice_)).cuda()
        want = torch.zeros(R * slice_, dtype=torch.uint8, device="cuda")
        got = torch.full((R * slice_,), 0xA5, dtype=torch.uint8, device="cuda")
        assert lib.p2g_encode(C.byref(_job(_ffi, src, S, slice_, R, want, stream))) == 0
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = lib.p2g_encode_noalloc(C.byref(_job(_ffi, src, S, slice_, R, got, stream)))
        assert st == 0, lib.p2g_last_error_message()
        torch.cuda.synchronize()
        if call > 0:  # past the first call's per-device set-up: no device memory taken
            assert torch.cuda.mem_get_info()[0] == free_before
        assert torch.equal(got, want), f"call {call}: p2g_encode_noalloc differs from p2g_encode"


def test_noalloc_rejects_jobs_beyond_its_scratch(p2g, gpu):
    import torch

    from par2rust_b200 import _ffi

    lib = _ffi.lib()
    S, slice_, R = 4097, 16, 96  # 4097 * ceil(96/32) = 12291 row groups > 8192
    src = torch.zeros(S * slice_, dtype=torch.uint8, device="cuda")
    rec = torch.zeros(R * slice_, dtype=torch.uint8, device="cuda")
    st = lib.p2g_encode_noalloc(C.byref(_job(_ffi, src, S, slice_, R, rec, torch.cuda.current_stream().cuda_stream)))
    assert st == p2g.InvalidArgument.status
    assert b"scratch" in lib.p2g_last_error_message()
    assert not rec.any()


def test_noalloc_edge_shapes_match_encode(p2g, gpu):
    """Ragged slices with their 16-byte row padding, a recovery stride wider
    than the padded row (bytes past it stay untouched), high first
    exponents, an R whose last row group folds, and the waiting form that
    reads the device error flag back: each equal to p2g_encode."""
    import torch

    from par2rust_b200 import _ffi
    from par2rust_b200.workloads import file_bytes

    lib = _ffi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # (S, slice, src_stride, R, recovery_stride, first_exponent, flags)
    cases = [(9, 4100, 4112, 20, 4112, 0, 1), (7, 4100, 4112, 33, 4160, 0, 1 | p2g.ENCODE_WAIT),
             (11, 8192, 8192, 30, 8192, 65500, 1), (5, 2048, 2048, 48, 2048, 17, 1 | p2g.ENCODE_WAIT)]
    for k, (S, sl, ss, R, rs, fe, flags) in enumerate(cases):
        # source rows with their padding inside the buffer (it is read)
        src = torch.zeros(S * ss, dtype=torch.uint8, device="cuda")
        src.view(S, ss)[:, :sl] = torch.from_numpy(file_bytes(2000 + k, S * sl).reshape(S, sl)).cuda()
        want = torch.full((R * rs,), 0x5C, dtype=torch.uint8, device="cuda")
        got = torch.full((R * rs,), 0x5C, dtype=torch.uint8, device="cuda")
        mk = lambda rec, fl: _ffi.p2g_encode_job(src=src.data_ptr(), src_stride=ss, input_count=S, slice_size=sl,
                                                 recovery_count=R, first_exponent=fe, recovery=rec.data_ptr(),
                                                 recovery_stride=rs, flags=fl, stream=stream)
        assert lib.p2g_encode(C.byref(mk(want, flags))) == 0, lib.p2g_last_error_message()
        assert lib.p2g_encode_noalloc(C.byref(mk(got, flags))) == 0, lib.p2g_last_error_message()
        torch.cuda.synchronize()
        w, g = want.view(R, rs), got.view(R, rs)
        assert torch.equal(g[:, :sl], w[:, :sl]), f"case {k}: rows differ from p2g_encode"
        pad = (sl + 15) // 16 * 16
        assert bool((g[:, pad:] == 0x5C).all()), f"case {k}: bytes past the padded row were written"
