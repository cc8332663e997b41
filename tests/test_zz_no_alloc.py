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
