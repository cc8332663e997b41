"""par2rust_b200 -- B200 PAR2 create engine, Python mirror of the par2rust API.

The names follow the reference crate's public surface (src/lib.rs:42-61):
``run_create``, ``run_create_with_progress``, ``run_create_fused``,
``write_index_file``, ``CreateOptions``, ``VolumeScheme``, ``SourceFile``
(with ``scan`` / ``scan_with_progress``), ``ProgressEvent``,
``ProgressReporter``, ``Par2Error`` and the ``MAX_*`` limits.  Every call
goes through the C ABI of ``libpar2gpu.so`` (include/par2gpu.h); the
Reed-Solomon accumulator and all bulk hashing run as sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Callable, Iterable, List, Optional, Sequence, Tuple, Union

from . import _ffi
from ._ffi import lib

MAX_FILES = 32_768
MAX_INPUT_BLOCKS = 32_768
MAX_RECOVERY_BLOCKS = 65_535
HASH16K_LEN = 16 * 1024

HOST_POINTERS = 0
DEVICE_POINTERS = 1
JOB_SKIP_HASH_FULL = 2
ENCODE_WAIT = 4  # p2g_encode / p2g_encode_noalloc: wait and report a device timeout
ENCODE_LUT = 8  # p2g_encode: force the shared-memory lookup kernel
ENCODE_TENSOR = 16  # p2g_encode: force the tensor-core (tcgen05) bit-sliced kernel


# ---------------------------------------------------------------------------
# Errors: Par2Error variants (src/error.rs:7-41)
# ---------------------------------------------------------------------------
class Par2Error(Exception):
    status = -1


class IoError(Par2Error):
    status = 1


class InvalidSliceSize(Par2Error):
    status = 2


class InvalidFileName(Par2Error):
    status = 3


class NoInputFiles(Par2Error):
    status = 4


class EmptyFile(Par2Error):
    status = 5


class TooManyFiles(Par2Error):
    status = 6


class TooManyRecoveryBlocks(Par2Error):
    status = 7


class TooManyInputBlocks(Par2Error):
    status = 8

    def __init__(self, msg, count=0, slice_size=0, suggested=0):
        super().__init__(msg)
        self.count, self.slice_size, self.suggested = count, slice_size, suggested


class InvalidVolumeScheme(Par2Error):
    status = 9


class InvalidArgument(Par2Error):
    status = 20


class CudaError(Par2Error):
    status = 21


class OutOfMemory(Par2Error):
    status = 22


class DeviceTimeout(Par2Error):
    status = 23


_ERRORS = {c.status: c for c in (IoError, InvalidSliceSize, InvalidFileName, NoInputFiles, EmptyFile, TooManyFiles,
                                 TooManyRecoveryBlocks, TooManyInputBlocks, InvalidVolumeScheme, InvalidArgument,
                                 CudaError, OutOfMemory, DeviceTimeout)}


def _check(status: int) -> None:
    if status == 0:
        return
    msg = (lib().p2g_last_error_message() or b"").decode("utf-8", "replace")
    cls = _ERRORS.get(status, Par2Error)
    if cls is TooManyInputBlocks:
        d = _ffi.p2g_error_detail()
        lib().p2g_last_error_detail(C.byref(d))
        raise TooManyInputBlocks(msg, d.count, d.slice_size, d.suggested)
    raise cls(msg)


# ---------------------------------------------------------------------------
# VolumeScheme (src/creator.rs:111-139) and CreateOptions (:142-173)
# ---------------------------------------------------------------------------
class VolumeScheme:
    kind = 0

    @staticmethod
    def Single() -> "VolumeScheme":
        return _Single()

    @staticmethod
    def Exponential() -> "VolumeScheme":
        return _Exponential()

    @staticmethod
    def Uniform(count: int) -> "VolumeScheme":
        return _Uniform(count)

    @staticmethod
    def Limited(max_blocks_per_volume: int, inner: "VolumeScheme") -> "VolumeScheme":
        return _Limited(max_blocks_per_volume, inner)

    @staticmethod
    def Explicit(sizes: Sequence[int]) -> "VolumeScheme":
        return _Explicit(list(sizes))

    def _to_c(self, keep: list) -> _ffi.p2g_volume_scheme:
        s = _ffi.p2g_volume_scheme()
        s.kind = self.kind
        s.count = getattr(self, "count", 0)
        s.max_blocks_per_volume = getattr(self, "max_blocks_per_volume", 0)
        inner = getattr(self, "inner", None)
        if inner is not None:
            ic = inner._to_c(keep)
            keep.append(ic)
            s.inner = C.pointer(ic)
        sizes = getattr(self, "sizes", None)
        if sizes is not None:
            arr = (C.c_uint32 * max(len(sizes), 1))(*sizes)
            keep.append(arr)
            s.explicit_sizes = arr
            s.explicit_count = len(sizes)
        return s

    def __eq__(self, other):
        return type(self) is type(other) and self.__dict__ == other.__dict__

    def __repr__(self):
        args = ", ".join(f"{k}={v!r}" for k, v in self.__dict__.items())
        return f"VolumeScheme.{type(self).__name__.lstrip('_')}({args})"


class _Single(VolumeScheme):
    kind = 0


class _Exponential(VolumeScheme):
    kind = 1


class _Uniform(VolumeScheme):
    kind = 2

    def __init__(self, count):
        self.count = int(count)


class _Limited(VolumeScheme):
    kind = 3

    def __init__(self, max_blocks_per_volume, inner):
        self.max_blocks_per_volume = int(max_blocks_per_volume)
        self.inner = inner


class _Explicit(VolumeScheme):
    kind = 4

    def __init__(self, sizes):
        self.sizes = [int(x) for x in sizes]


@dataclass
class CreateOptions:
    output: Union[str, Path] = ""
    slice_size: int = 4096
    recovery_block_count: int = 0
    volume_scheme: VolumeScheme = field(default_factory=VolumeScheme.Single)
    comments: List[str] = field(default_factory=list)

    def _to_c(self, keep: list) -> _ffi.p2g_create_options:
        o = _ffi.p2g_create_options()
        out = os.fsencode(str(self.output))
        keep.append(out)
        o.output = out
        o.slice_size = int(self.slice_size)
        o.recovery_block_count = int(self.recovery_block_count)
        o.volume_scheme = self.volume_scheme._to_c(keep)
        if self.comments:
            enc = [c.encode("utf-8") for c in self.comments]
            arr = (C.c_char_p * len(enc))(*enc)
            keep.extend([enc, arr])
            o.comments = arr
            o.comment_count = len(enc)
        return o


# ---------------------------------------------------------------------------
# Progress (src/progress.rs)
# ---------------------------------------------------------------------------
_EVENT_NAMES = ["ScanStarted", "ScanProgress", "ScanCompleted", "EncodeStarted", "EncodeProgress",
                "EncodeCompleted", "IndexWritten", "VolumeWritten"]


@dataclass
class ProgressEvent:
    kind: str
    path: Optional[str] = None
    total_slices: int = 0
    slices_done: int = 0
    volume_index: int = 0
    total_volumes: int = 0
    input_blocks: int = 0
    recovery_blocks: int = 0
    input_block_done: int = 0


class ProgressReporter:
    """Receiver for progress events (ProgressReporter::on_event)."""

    def on_event(self, event: ProgressEvent) -> None:  # pragma: no cover - interface
        raise NotImplementedError


def _progress_cb(reporter):
    if reporter is None:
        return _ffi.PROGRESS_FN(), None

    def cb(evp, _user):
        e = evp.contents
        reporter.on_event(ProgressEvent(
            kind=_EVENT_NAMES[e.kind], path=e.path.decode("utf-8", "replace") if e.path else None,
            total_slices=e.total_slices, slices_done=e.slices_done, volume_index=e.volume_index,
            total_volumes=e.total_volumes, input_blocks=e.input_blocks, recovery_blocks=e.recovery_blocks,
            input_block_done=e.input_block_done))

    f = _ffi.PROGRESS_FN(cb)
    return f, f


# ---------------------------------------------------------------------------
# SourceFile (src/source.rs:28-136)
# ---------------------------------------------------------------------------
@dataclass
class SliceChecksum:
    md5: bytes
    crc32: int


@dataclass
class SourceFile:
    name: bytes
    path: Path
    length: int
    hash_full: bytes
    hash16k: bytes
    file_id: bytes
    slice_checksums: List[SliceChecksum]

    @staticmethod
    def scan(path, display_name: bytes, slice_size: int) -> "SourceFile":
        return SourceFile.scan_with_progress(path, display_name, slice_size, None)

    @staticmethod
    def scan_with_progress(path, display_name: bytes, slice_size: int,
                           reporter: Optional[ProgressReporter]) -> "SourceFile":
        sf = _ffi.p2g_source_file()
        name = bytes(display_name)
        nbuf = (C.c_uint8 * max(len(name), 1)).from_buffer_copy(name or b"\0")
        cb, _keep = _progress_cb(reporter)
        _check(lib().p2g_scan_with_progress(os.fsencode(str(path)), nbuf, len(name), int(slice_size), cb, None,
                                            C.byref(sf)))
        try:
            return SourceFile._from_c(sf)
        finally:
            lib().p2g_source_file_free(C.byref(sf))

    @staticmethod
    def _from_c(sf: _ffi.p2g_source_file) -> "SourceFile":
        n = sf.slice_count
        cks = [SliceChecksum(bytes(sf.slice_checksums[i].md5), int(sf.slice_checksums[i].crc32)) for i in range(n)]
        return SourceFile(name=C.string_at(sf.name, sf.name_len), path=Path(os.fsdecode(sf.path or b"")),
                          length=sf.length, hash_full=bytes(sf.hash_full), hash16k=bytes(sf.hash16k),
                          file_id=bytes(sf.file_id), slice_checksums=cks)

    def _to_c(self, keep: list) -> _ffi.p2g_source_file:
        sf = _ffi.p2g_source_file()
        nb = (C.c_uint8 * max(len(self.name), 1)).from_buffer_copy(self.name or b"\0")
        pb = os.fsencode(str(self.path))
        arr = (_ffi.p2g_slice_checksum * max(len(self.slice_checksums), 1))()
        for i, sc in enumerate(self.slice_checksums):
            arr[i].md5[:] = list(sc.md5)
            arr[i].crc32 = sc.crc32
        keep.extend([nb, pb, arr])
        sf.name = C.cast(nb, C.POINTER(C.c_uint8))
        sf.name_len = len(self.name)
        sf.path = pb
        sf.length = self.length
        sf.hash_full[:] = list(self.hash_full)
        sf.hash16k[:] = list(self.hash16k)
        sf.file_id[:] = list(self.file_id)
        sf.slice_checksums = C.cast(arr, C.POINTER(_ffi.p2g_slice_checksum))
        sf.slice_count = len(self.slice_checksums)
        return sf


def _sources_to_c(sources: Sequence[SourceFile], keep: list):
    arr = (_ffi.p2g_source_file * max(len(sources), 1))()
    for i, s in enumerate(sources):
        arr[i] = s._to_c(keep)
    return arr


def _path_list(pl: _ffi.p2g_path_list) -> List[Path]:
    out = [Path(os.fsdecode(pl.paths[i])) for i in range(pl.count)]
    lib().p2g_path_list_free(C.byref(pl))
    return out


# ---------------------------------------------------------------------------
# Create entry points (src/creator.rs:182-860)
# ---------------------------------------------------------------------------
def run_create(opts: CreateOptions, sources: Sequence[SourceFile]) -> List[Path]:
    return run_create_with_progress(opts, sources, None)


def run_create_with_progress(opts: CreateOptions, sources: Sequence[SourceFile],
                             reporter: Optional[ProgressReporter]) -> List[Path]:
    keep: list = []
    o = opts._to_c(keep)
    arr = _sources_to_c(sources, keep)
    pl = _ffi.p2g_path_list()
    cb, _k = _progress_cb(reporter)
    _check(lib().p2g_run_create_with_progress(C.byref(o), arr, len(sources), cb, None, C.byref(pl)))
    return _path_list(pl)


def run_create_fused(opts: CreateOptions, inputs: Sequence[Tuple[Union[str, Path], bytes]],
                     reporter: Optional[ProgressReporter] = None) -> List[Path]:
    keep: list = []
    o = opts._to_c(keep)
    arr = (_ffi.p2g_input * max(len(inputs), 1))()
    for i, (p, name) in enumerate(inputs):
        pb = os.fsencode(str(p))
        nb = (C.c_uint8 * max(len(name), 1)).from_buffer_copy(bytes(name) or b"\0")
        keep.extend([pb, nb])
        arr[i].path = pb
        arr[i].display_name = C.cast(nb, C.POINTER(C.c_uint8))
        arr[i].name_len = len(name)
    pl = _ffi.p2g_path_list()
    cb, _k = _progress_cb(reporter)
    _check(lib().p2g_run_create_fused(C.byref(o), arr, len(inputs), cb, None, C.byref(pl)))
    return _path_list(pl)


def write_index_file(opts: CreateOptions, sources: Sequence[SourceFile]) -> Path:
    keep: list = []
    o = opts._to_c(keep)
    arr = _sources_to_c(sources, keep)
    out = C.c_void_p()
    _check(lib().p2g_write_index_file(C.byref(o), arr, len(sources), C.byref(out)))
    p = C.string_at(out.value)
    lib().p2g_string_free(out)
    return Path(os.fsdecode(p))


class _OutputSetOwner:
    """Frees a library-owned p2g_output_set once no view of it is left."""

    def __init__(self, os_):
        self.os_ = os_
        # bound now: at interpreter exit the module globals may be gone first
        self._free = lib().p2g_output_set_free
        self._byref = C.byref

    def __del__(self):
        self._free(self._byref(self.os_))


def create_in_memory(opts: CreateOptions, inputs: Sequence[Tuple[bytes, object]],
                     return_sources: bool = False, copy: bool = True):
    """run_create_fused without a filesystem.

    ``inputs`` are (display_name, data) pairs; data is any buffer (bytes,
    numpy array, pinned torch tensor, ...).  Returns a list of
    (file_name, bytes) for the index and each volume, plus the scanned
    SourceFile records when ``return_sources``.  With ``copy=False`` the
    file contents are read-only memoryviews of the library's buffers (no
    copy into Python bytes); the buffers are freed when the last view goes.
    """
    keep: list = []
    o = opts._to_c(keep)
    arr = (_ffi.p2g_buffer_input * max(len(inputs), 1))()
    for i, (name, data) in enumerate(inputs):
        ptr, length = _host_buffer(data, keep)
        nb = (C.c_uint8 * max(len(name), 1)).from_buffer_copy(bytes(name) or b"\0")
        keep.append(nb)
        arr[i].data = ptr
        arr[i].length = length
        arr[i].display_name = C.cast(nb, C.POINTER(C.c_uint8))
        arr[i].name_len = len(name)
    srcs = (_ffi.p2g_source_file * max(len(inputs), 1))() if return_sources else None
    os_ = _ffi.p2g_output_set()
    _check(lib().p2g_create_in_memory(C.byref(o), arr, len(inputs), srcs, C.byref(os_)))
    files = []
    if copy:
        for i in range(os_.count):
            f = os_.files[i]
            files.append((os.fsdecode(f.name), C.string_at(f.data, f.length)))
        lib().p2g_output_set_free(C.byref(os_))
    else:
        owner = _OutputSetOwner(os_)
        for i in range(os_.count):
            f = os_.files[i]
            buf = (C.c_uint8 * f.length).from_address(C.cast(f.data, C.c_void_p).value)
            buf._owner = owner  # the view keeps buf, buf keeps the output set
            files.append((os.fsdecode(f.name), memoryview(buf).cast("B").toreadonly()))
    if not return_sources:
        return files
    out_src = []
    for i in range(len(inputs)):
        out_src.append(SourceFile._from_c(srcs[i]))
        lib().p2g_source_file_free(C.byref(srcs[i]))
    return files, out_src


def _host_buffer(data, keep: list) -> Tuple[int, int]:
    """(address, length) of a host buffer without copying when possible."""
    if hasattr(data, "data_ptr") and hasattr(data, "is_cuda"):  # torch tensor (CPU)
        if data.is_cuda:
            raise InvalidArgument("expected a host tensor")
        t = data.contiguous()
        keep.append(t)
        return t.data_ptr(), t.numel() * t.element_size()
    import numpy as np

    a = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    a = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
    keep.append(a)
    return a.ctypes.data, a.nbytes


# ---------------------------------------------------------------------------
# Kernel-level seams
# ---------------------------------------------------------------------------
def check_bounded_wait(polls: int = 1 << 16) -> None:
    """Run the library's device-wait failure path on purpose (a barrier that
    nothing completes, waited for at most ``polls`` tries).  Raises
    DeviceTimeout, as a job whose copy never lands would; the device stays
    usable afterwards."""
    _check(lib().p2g_check_bounded_wait(int(polls)))


def gf_mul_xor(coeff: int, input: bytes, output: bytearray) -> None:
    """output ^= coeff * input over LE GF(2^16) symbols (gf_mul_xor_dispatch)."""
    import numpy as np

    inp = np.frombuffer(bytes(input), dtype=np.uint8)
    out = np.frombuffer(output, dtype=np.uint8)
    _check(lib().p2g_gf_mul_xor(int(coeff), inp.ctypes.data, out.ctypes.data, len(inp), HOST_POINTERS, None))


def encode(src, slice_size: int, recovery_count: int, first_exponent: int = 0, input_count: Optional[int] = None,
           variant: int = 0):
    """encode_all_recovery_blocks over host memory: src holds input_count
    zero-padded slices back to back; returns recovery bytes (R*slice)."""
    import numpy as np

    a = np.ascontiguousarray(np.frombuffer(src, dtype=np.uint8) if not isinstance(src, np.ndarray) else src)
    a = a.view(np.uint8).reshape(-1)
    S = input_count if input_count is not None else a.nbytes // slice_size
    out = np.zeros(recovery_count * slice_size, dtype=np.uint8)
    job = _ffi.p2g_encode_job(src=a.ctypes.data, src_stride=slice_size, input_count=S, slice_size=slice_size,
                              recovery_count=recovery_count, first_exponent=first_exponent,
                              recovery=out.ctypes.data, recovery_stride=slice_size, flags=HOST_POINTERS | variant,
                              stream=None)
    _check(lib().p2g_encode(C.byref(job)))
    return out


def encode_device(src_ptr: int, src_stride: int, input_count: int, slice_size: int, recovery_count: int,
                  rec_ptr: int, rec_stride: int, stream: int = 0, first_exponent: int = 0, wait: bool = False,
                  variant: int = 0) -> None:
    """p2g_encode on device buffers, enqueued on `stream`; with wait=True
    the call waits for it and raises DeviceTimeout if a device wait gave up.
    variant: 0 (chosen by shape), ENCODE_LUT or ENCODE_TENSOR."""
    job = _ffi.p2g_encode_job(src=src_ptr, src_stride=src_stride, input_count=input_count, slice_size=slice_size,
                              recovery_count=recovery_count, first_exponent=first_exponent, recovery=rec_ptr,
                              recovery_stride=rec_stride, flags=DEVICE_POINTERS | (ENCODE_WAIT if wait else 0) | variant,
                              stream=stream or None)
    _check(lib().p2g_encode(C.byref(job)))


def slice_checksums(src, slice_size: int, count: Optional[int] = None) -> List[SliceChecksum]:
    import numpy as np

    a = np.ascontiguousarray(np.frombuffer(src, dtype=np.uint8) if not isinstance(src, np.ndarray) else src)
    n = count if count is not None else a.nbytes // slice_size
    out = (_ffi.p2g_slice_checksum * max(n, 1))()
    _check(lib().p2g_slice_checksums(a.ctypes.data, slice_size, n, slice_size, C.addressof(out), HOST_POINTERS, None))
    return [SliceChecksum(bytes(out[i].md5), int(out[i].crc32)) for i in range(n)]


def file_hashes(buffers: Sequence[bytes]) -> List[Tuple[bytes, bytes]]:
    """(hash_full, hash16k) per buffer, computed on the device."""
    import numpy as np

    arrs = [np.frombuffer(bytes(b) + b"\0" * 4, dtype=np.uint8) for b in buffers]
    n = len(arrs)
    ptrs = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in arrs])
    lens = (C.c_uint64 * max(n, 1))(*[len(b) for b in buffers])
    hf = (C.c_uint8 * (16 * max(n, 1)))()
    h16 = (C.c_uint8 * (16 * max(n, 1)))()
    _check(lib().p2g_file_hashes(ptrs, lens, n, C.addressof(hf), C.addressof(h16), HOST_POINTERS, None))
    return [(bytes(hf[16 * i:16 * i + 16]), bytes(h16[16 * i:16 * i + 16])) for i in range(n)]


def recovery_packet_md5(set_id: bytes, recovery, slice_size: int, count: int, first_exponent: int = 0) -> List[bytes]:
    import numpy as np

    a = np.ascontiguousarray(np.frombuffer(recovery, dtype=np.uint8) if not isinstance(recovery, np.ndarray) else recovery)
    out = (C.c_uint8 * (16 * max(count, 1)))()
    _check(lib().p2g_recovery_packet_md5(bytes(set_id), a.ctypes.data, slice_size, count, slice_size, first_exponent,
                                         C.addressof(out), HOST_POINTERS, None))
    return [bytes(out[16 * i:16 * i + 16]) for i in range(count)]


class DeviceJobBuffers:
    """Device outputs of one create job (torch uint8 CUDA tensors)."""

    def __init__(self, S: int, n_files: int, slice_size: int, recovery_count: int, device):
        import torch

        self.rec_stride = (slice_size + 15) // 16 * 16
        self.recovery = torch.empty(max(recovery_count, 1) * self.rec_stride, dtype=torch.uint8, device=device)
        self.checksums = torch.empty(max(S, 1) * 20, dtype=torch.uint8, device=device)
        self.hash_full = torch.empty(max(n_files, 1) * 16, dtype=torch.uint8, device=device)
        self.hash16k = torch.empty(max(n_files, 1) * 16, dtype=torch.uint8, device=device)
        self.packet_md5 = torch.empty(max(recovery_count, 1) * 16, dtype=torch.uint8, device=device)
        self.set_id_device = torch.empty(16, dtype=torch.uint8, device=device)  # written by batched runs
        self.set_id = b""


def run_device_job(src, file_lengths: Sequence[int], names: Sequence[bytes], slice_size: int, recovery_count: int,
                   bufs: Optional[DeviceJobBuffers] = None, stream: Optional[int] = None,
                   skip_hash_full: bool = False, variant: int = 0) -> DeviceJobBuffers:
    """The device work of one create job over a device-resident source.

    ``src`` is a CUDA uint8 tensor holding the files back to back, each
    starting on a slice boundary and zero-padded to whole slices.  Work is
    ordered on ``stream`` (default: torch's current stream).
    """
    import torch

    S = sum((n + slice_size - 1) // slice_size for n in file_lengths)
    if bufs is None:
        bufs = DeviceJobBuffers(S, len(file_lengths), slice_size, recovery_count, src.device)
    if stream is None:
        stream = torch.cuda.current_stream(src.device).cuda_stream
    n = len(file_lengths)
    lens = (C.c_uint64 * max(n, 1))(*file_lengths)
    nbufs = [C.create_string_buffer(bytes(x), len(x)) for x in names]
    nptrs = (C.c_void_p * max(n, 1))(*[C.addressof(b) for b in nbufs])
    nlens = (C.c_size_t * max(n, 1))(*[len(x) for x in names])
    job = _ffi.p2g_device_job()
    job.src = src.data_ptr()
    job.file_count = n
    job.file_lengths = lens
    job.names = nptrs
    job.name_lens = nlens
    job.slice_size = slice_size
    job.recovery_count = recovery_count
    job.recovery = bufs.recovery.data_ptr()
    job.recovery_stride = bufs.rec_stride
    job.checksums = bufs.checksums.data_ptr()
    job.hash_full = bufs.hash_full.data_ptr()
    job.hash16k = bufs.hash16k.data_ptr()
    job.packet_md5 = bufs.packet_md5.data_ptr()
    job.flags = (JOB_SKIP_HASH_FULL if skip_hash_full else 0) | variant
    job.stream = stream
    _check(lib().p2g_run_device_job(C.byref(job)))
    bufs.set_id = bytes(job.set_id_out)
    return bufs


# ---------------------------------------------------------------------------
# Batched create (no counterpart in the reference, which creates one set at a
# time): many jobs in one persistent, graph-captured launch.
# ---------------------------------------------------------------------------
BATCH_NO_GRAPH = 1
BATCH_NO_AUTOTUNE = 2
BATCH_DERIVE_BASIS = 4
BATCH_TENSOR = 8  # every job's encode on the tensor cores
BATCH_LUT = 16  # every job's encode on the lookup kernel (neither: one kernel per batch, by cost)


@dataclass
class BatchJobSpec:
    """One job of a batch: a device source laid out as for run_device_job and
    the buffers its outputs go to."""
    src: object
    file_lengths: Sequence[int]
    names: Sequence[bytes]
    slice_size: int
    recovery_count: int
    bufs: DeviceJobBuffers
    hash_full: bool = False  # whole-file MD5s on the device too (into bufs.hash_full)

    @property
    def input_slices(self) -> int:
        return sum((n + self.slice_size - 1) // self.slice_size for n in self.file_lengths)


@dataclass
class BatchInfo:
    jobs: int
    items: int
    encode_items: int
    scan_items: int
    setid_items: int
    ctas: int
    predicted_ms: float
    device_bytes: int


def _batch_info(ci: "_ffi.p2g_batch_info") -> BatchInfo:
    return BatchInfo(ci.jobs, ci.items, ci.encode_items, ci.scan_items, ci.setid_items, ci.ctas,
                     ci.predicted_ms, ci.device_bytes)


class Batch:
    """A planned batch of create jobs (p2g_batch_create).  ``launch`` enqueues
    one run of every job on a stream; after synchronising, ``check`` raises
    DeviceTimeout if a bounded device wait gave up.  Per job the outputs equal
    run_device_job(..., skip_hash_full=True); the set id lands in
    ``bufs.set_id_device``."""

    def __init__(self, jobs: Sequence[BatchJobSpec], flags: int = 0):
        self._keep = []
        arr = (_ffi.p2g_batch_job * len(jobs))()
        for i, j in enumerate(jobs):
            n = len(j.file_lengths)
            lens = (C.c_uint64 * max(n, 1))(*j.file_lengths)
            nbufs = [C.create_string_buffer(bytes(x), len(x)) for x in j.names]
            nptrs = (C.c_void_p * max(n, 1))(*[C.addressof(b) for b in nbufs])
            nlens = (C.c_size_t * max(n, 1))(*[len(x) for x in j.names])
            self._keep += [lens, nbufs, nptrs, nlens]
            b = j.bufs
            arr[i] = _ffi.p2g_batch_job(src=j.src.data_ptr(), file_count=n, file_lengths=lens, names=nptrs,
                                        name_lens=nlens, slice_size=j.slice_size, recovery_count=j.recovery_count,
                                        recovery=b.recovery.data_ptr(), recovery_stride=b.rec_stride,
                                        checksums=b.checksums.data_ptr(), hash16k=b.hash16k.data_ptr(),
                                        packet_md5=b.packet_md5.data_ptr(), set_id=b.set_id_device.data_ptr(),
                                        hash_full=b.hash_full.data_ptr() if j.hash_full else None)
        self.jobs = list(jobs)
        h = C.c_void_p()
        _check(lib().p2g_batch_create(arr, len(jobs), flags, C.byref(h)))
        self._h = h

    def launch(self, stream: Optional[int] = None) -> None:
        import torch

        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        _check(lib().p2g_batch_launch(self._h, stream))

    def check(self) -> None:
        _check(lib().p2g_batch_check(self._h))

    def info(self) -> BatchInfo:
        ci = _ffi.p2g_batch_info()
        _check(lib().p2g_batch_get_info(self._h, C.byref(ci)))
        return _batch_info(ci)

    def tile(self, job: int) -> int:
        return lib().p2g_batch_job_tile(self._h, job)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().p2g_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def staged_groups(sizes: Sequence[int], groups: int) -> List[Tuple[int, int]]:
    """Consecutive job ranges [a, b) for StagedBatch: about equal source bytes
    per group, the first group half as large; a job is never split, so a
    single large job can leave fewer groups than asked."""
    n = len(sizes)
    groups = max(1, min(int(groups), n))
    total = max(1, sum(sizes))
    shares = [0.5] + [1.0] * (groups - 1)
    unit = total / sum(shares)
    bounds, acc, k, edge = [], 0, 0, shares[0] * unit
    for i, sz in enumerate(sizes):
        acc += sz
        if acc >= edge and k < groups - 1 and i + 1 < n:
            bounds.append(i + 1)
            k += 1
            edge += shares[k] * unit
    bounds = [0] + bounds + [n]
    return [(a, b) for a, b in zip(bounds, bounds[1:]) if b > a]


def plan_device_job(slice_size: int, input_slices: int, recovery_count: int, file_count: int = 1,
                    with_chains: bool = True, ctas: int = 148):
    """The encode items p2g_run_device_job would run (host-only planner):
    returns (items, zero_from_symbol, bands); each item is a dict with
    row_group, fold, first_symbol, symbols, band, first_slice, slices and
    accumulate."""
    n = C.c_uint32()
    z = C.c_uint32()
    nb = C.c_uint32()
    _check(lib().p2g_plan_device_job(slice_size, input_slices, recovery_count, file_count, int(with_chains), ctas,
                                     None, 0, C.byref(n), C.byref(z), C.byref(nb)))
    arr = (_ffi.p2g_plan_item * max(n.value, 1))()
    _check(lib().p2g_plan_device_job(slice_size, input_slices, recovery_count, file_count, int(with_chains), ctas,
                                     C.cast(arr, C.c_void_p), n.value, C.byref(n), C.byref(z), C.byref(nb)))
    items = [{f: getattr(arr[i], f) for f, _ in _ffi.p2g_plan_item._fields_} for i in range(n.value)]
    return items, z.value, nb.value


class StagedBatch:
    """Batched create for jobs whose sources sit in pinned host memory.

    The jobs are cut into ``groups`` consecutive batches of about equal
    source bytes (the first one half as large, so the device starts early).
    All uploads are queued at once on a copy stream; group g's batch launches
    on the compute stream when its own uploads are done.  So group g+1's
    sources cross PCIe while group g runs.  Each group's outputs download on a
    third stream as soon as that group ends.  Outputs equal one Batch over all
    jobs.

    ``hosts[i]`` is job i's pinned source (its first ``hosts[i].numel()``
    bytes go to ``jobs[i].src``).  ``outputs[i]``, when given, is a tuple of
    pinned tensors (recovery, checksums, packet_md5, hash16k, set_id) that
    receive the job's device buffers of the same names.
    """

    def __init__(self, jobs: Sequence[BatchJobSpec], hosts: Sequence[object], outputs=None, groups: int = 6,
                 flags: int = 0):
        import torch

        if len(hosts) != len(jobs) or (outputs is not None and len(outputs) != len(jobs)):
            raise InvalidArgument("one pinned source (and output set) per job")
        self.ranges = staged_groups([int(h.numel()) for h in hosts], groups)
        self.jobs, self.hosts, self.outputs = list(jobs), list(hosts), outputs
        self.batches = [Batch(self.jobs[a:b], flags) for a, b in self.ranges]
        self._up = torch.cuda.Stream()
        self._down = torch.cuda.Stream()

    def launch(self, stream: Optional[int] = None) -> None:
        """Enqueue uploads, launches and downloads; the caller synchronises."""
        import torch

        comp = torch.cuda.current_stream() if stream is None else torch.cuda.ExternalStream(stream)
        self._up.wait_stream(comp)  # the previous run's readers of the sources are done
        uploaded = []
        with torch.cuda.stream(self._up):
            for a, b in self.ranges:
                for i in range(a, b):
                    n = self.hosts[i].numel()
                    self.jobs[i].src.view(-1)[:n].copy_(self.hosts[i].view(-1), non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self._up)
                uploaded.append(ev)
        for (a, b), batch, ev in zip(self.ranges, self.batches, uploaded):
            comp.wait_event(ev)
            batch.launch(comp.cuda_stream)
            if self.outputs is None:
                continue
            done = torch.cuda.Event()
            done.record(comp)
            self._down.wait_event(done)
            with torch.cuda.stream(self._down):
                for i in range(a, b):
                    bf = self.jobs[i].bufs
                    for t, d in zip(self.outputs[i], (bf.recovery, bf.checksums, bf.packet_md5, bf.hash16k,
                                                      bf.set_id_device)):
                        t.copy_(d, non_blocking=True)
        comp.wait_stream(self._down)

    def check(self) -> None:
        for b in self.batches:
            b.check()

    def close(self) -> None:
        for b in self.batches:
            b.close()


# ---------------------------------------------------------------------------
# Serving loop (no counterpart in the reference): continuous batching of
# create requests on the device.
# ---------------------------------------------------------------------------
SOURCE_HOST = 0
SOURCE_SEEDED = 1


@dataclass
class ServerResult:
    ticket: int
    tag: int
    status: int
    submit_s: float
    admit_s: float
    done_s: float
    source_bytes: int
    input_slices: int
    recovery_count: int
    file_count: int
    slice_size: int
    ptr: dict  # device pointers: src, recovery, checksums, hash16k, packet_md5, set_id
    recovery_stride: int

    @property
    def latency_s(self) -> float:
        return self.done_s - self.submit_s


def copy_to_host(device_ptr: int, nbytes: int) -> bytes:
    buf = C.create_string_buffer(max(nbytes, 1))
    _check(lib().p2g_copy_to_host(buf, device_ptr, nbytes))
    return buf.raw[:nbytes]


class Server:
    """Create-request server (p2g_server_*): jobs are admitted by HBM
    footprint and run in device waves shared with the other resident jobs.
    ``submit_*`` returns a ticket; ``poll`` returns completed jobs, whose
    device outputs stay valid until ``release``."""

    def __init__(self, hbm_budget: int = 0, wave_ms: float = 0.0, max_jobs: int = 0):
        o = _ffi.p2g_server_options(hbm_budget=hbm_budget, wave_ms=wave_ms, max_jobs=max_jobs, flags=0)
        h = C.c_void_p()
        _check(lib().p2g_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self._slices = {}
        self._keep = {}

    def _submit(self, file_lengths, names, slice_size, recovery_count, kind, host_src=None, seeds=None, tag=0):
        n = len(file_lengths)
        lens = (C.c_uint64 * max(n, 1))(*file_lengths)
        nbufs = [C.create_string_buffer(bytes(x), len(x)) for x in names]
        nptrs = (C.c_void_p * max(n, 1))(*[C.addressof(b) for b in nbufs])
        nlens = (C.c_size_t * max(n, 1))(*[len(x) for x in names])
        sd = (C.c_uint64 * max(n, 1))(*(seeds or [0] * n))
        job = _ffi.p2g_server_job(file_count=n, file_lengths=lens, names=nptrs, name_lens=nlens,
                                  slice_size=slice_size, recovery_count=recovery_count, source_kind=kind,
                                  host_src=host_src, file_seeds=sd, tag=tag)
        t = C.c_uint64()
        _check(lib().p2g_server_submit(self._h, C.byref(job), C.byref(t)))
        self._slices[t.value] = slice_size
        return t.value

    def submit_seeded(self, file_lengths: Sequence[int], seeds: Sequence[int], names: Sequence[bytes],
                      slice_size: int, recovery_count: int, tag: int = 0) -> int:
        return self._submit(file_lengths, names, slice_size, recovery_count, SOURCE_SEEDED, seeds=list(seeds), tag=tag)

    def submit_host(self, host_src, file_lengths: Sequence[int], names: Sequence[bytes], slice_size: int,
                    recovery_count: int, tag: int = 0) -> int:
        """host_src: the files back to back, slice-padded (a pinned torch tensor
        copies asynchronously); kept referenced until the job is released."""
        ptr = host_src.data_ptr() if hasattr(host_src, "data_ptr") else host_src.ctypes.data
        t = self._submit(file_lengths, names, slice_size, recovery_count, SOURCE_HOST, host_src=ptr, tag=tag)
        self._keep[t] = host_src
        return t

    def poll(self, max_results: int = 1024, wait_ms: int = 0) -> List[ServerResult]:
        arr = (_ffi.p2g_server_result * max_results)()
        n = C.c_uint32()
        _check(lib().p2g_server_poll(self._h, arr, max_results, C.byref(n), wait_ms))
        out = []
        for r in arr[:n.value]:
            out.append(ServerResult(r.ticket, r.tag, r.status, r.submit_s, r.admit_s, r.done_s, r.source_bytes,
                                    r.input_slices, r.recovery_count, r.file_count, self._slices.get(r.ticket, 0),
                                    {"src": r.src, "recovery": r.recovery, "checksums": r.checksums,
                                     "hash16k": r.hash16k, "packet_md5": r.packet_md5, "set_id": r.set_id},
                                    r.recovery_stride))
        return out

    def outputs(self, res: ServerResult) -> dict:
        """Copy a completed job's outputs to host bytes."""
        R, S, n = res.recovery_count, res.input_slices, res.file_count
        rec = copy_to_host(res.ptr["recovery"], R * res.recovery_stride) if R else b""
        rows = [rec[r * res.recovery_stride:r * res.recovery_stride + res.slice_size] for r in range(R)]
        return {"recovery": rows, "checksums": copy_to_host(res.ptr["checksums"], 20 * S),
                "hash16k": copy_to_host(res.ptr["hash16k"], 16 * n),
                "packet_md5": copy_to_host(res.ptr["packet_md5"], 16 * R) if R else b"",
                "set_id": copy_to_host(res.ptr["set_id"], 16)}

    def release(self, ticket: int) -> None:
        _check(lib().p2g_server_release(self._h, ticket))
        self._keep.pop(ticket, None)
        self._slices.pop(ticket, None)

    def stats(self) -> dict:
        st = _ffi.p2g_server_stats()
        _check(lib().p2g_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _ffi.p2g_server_stats._fields_}

    def now(self) -> float:
        return lib().p2g_server_now(self._h)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().p2g_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_plan(shapes: Sequence[Tuple[int, int, int, int]], ctas: int = 148, flags: int = 0
               ) -> Tuple[BatchInfo, List[int]]:
    """The batch planner alone (no device): shapes are (slice_size,
    input_slices, recovery_count, file_count); returns the plan summary and
    each job's tile width (0 for jobs without recovery rows)."""
    arr = (_ffi.p2g_batch_shape * len(shapes))(*[_ffi.p2g_batch_shape(*s) for s in shapes])
    ci = _ffi.p2g_batch_info()
    tiles = (C.c_uint32 * max(len(shapes), 1))()
    _check(lib().p2g_batch_plan(arr, len(shapes), ctas, flags, C.byref(ci), tiles))
    return _batch_info(ci), list(tiles[:len(shapes)])


# ---------------------------------------------------------------------------
# Host helpers of the reference's public modules
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Create CLI glue (src/main.rs): the par2rust executable beside the library
# is a shell around these.
# ---------------------------------------------------------------------------
CLI_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "par2rust")


def parse_slice_size(s: str) -> int:
    """parse_slice_size (src/main.rs:464-487); InvalidArgument on bad input."""
    v = C.c_uint64()
    _check(lib().p2g_parse_slice_size(s.encode(), C.byref(v)))
    return v.value


@dataclass(frozen=True)
class Redundancy:
    """The -r value (src/main.rs:489-531): Percent(percent) or TargetBytes(target_bytes)."""
    percent: Optional[int] = None
    target_bytes: Optional[int] = None

    @staticmethod
    def parse(s: str) -> "Redundancy":
        r = _ffi.p2g_redundancy()
        _check(lib().p2g_parse_redundancy(s.encode(), C.byref(r)))
        return Redundancy(target_bytes=r.target_bytes) if r.is_bytes else Redundancy(percent=r.percent)

    def _to_c(self) -> "_ffi.p2g_redundancy":
        r = _ffi.p2g_redundancy()
        if self.target_bytes is not None:
            r.is_bytes, r.target_bytes = 1, self.target_bytes
        else:
            r.percent = self.percent
        return r


def resolve_redundancy(r: Redundancy, total_input_blocks: int, slice_size: int) -> int:
    """resolve_redundancy (src/main.rs:533-556) for inputs of this many slices."""
    out = C.c_uint32()
    c = r._to_c()
    _check(lib().p2g_resolve_redundancy(C.byref(c), total_input_blocks, slice_size, C.byref(out)))
    return out.value


def build_volume_scheme(single_volume: bool = False, uniform: bool = False, limit_size: bool = False,
                        volume_count: Optional[int] = None, largest_source_length: int = 0, slice_size: int = 4096,
                        recovery_count: int = 0) -> VolumeScheme:
    """build_volume_scheme (src/main.rs:289-337) from the CLI's volume flags."""
    f = _ffi.p2g_cli_volume_flags(int(single_volume), int(uniform), int(limit_size), int(volume_count is not None),
                                  volume_count or 0)
    out, inner = _ffi.p2g_volume_scheme(), _ffi.p2g_volume_scheme()
    _check(lib().p2g_build_volume_scheme(C.byref(f), largest_source_length, slice_size, recovery_count, C.byref(out),
                                         C.byref(inner)))

    def conv(sc):
        if sc.kind == 0:
            return VolumeScheme.Single()
        if sc.kind == 1:
            return VolumeScheme.Exponential()
        if sc.kind == 2:
            return VolumeScheme.Uniform(sc.count)
        return VolumeScheme.Limited(sc.max_blocks_per_volume, conv(inner))

    return conv(out)


def input_bases(count: int) -> List[int]:
    arr = (C.c_uint16 * max(count, 1))()
    _check(lib().p2g_input_bases(count, arr))
    return list(arr[:count])


def gf_mul(a: int, b: int) -> int:
    return lib().p2g_gf_mul(a, b)


def gf_pow(base: int, exp: int) -> int:
    return lib().p2g_gf_pow(base, exp)


def resolve_volume_sizes(scheme: VolumeScheme, total: int) -> List[int]:
    keep: list = []
    sc = scheme._to_c(keep)
    n = C.c_uint32()
    _check(lib().p2g_resolve_volume_sizes(C.byref(sc), total, None, 0, C.byref(n)))
    out = (C.c_uint32 * max(n.value, 1))()
    _check(lib().p2g_resolve_volume_sizes(C.byref(sc), total, out, n.value, C.byref(n)))
    return list(out[:n.value])


def volume_filename(index_path, first_exponent: int, count: int) -> str:
    p = lib().p2g_volume_filename(os.fsencode(str(index_path)), first_exponent, count)
    s = C.string_at(p)
    lib().p2g_string_free(p)
    return os.fsdecode(s)


def build_packet(set_id: bytes, type_tag: bytes, body: bytes) -> bytes:
    n = lib().p2g_build_packet(set_id, type_tag, body, len(body), None)
    out = (C.c_uint8 * n)()
    lib().p2g_build_packet(set_id, type_tag, body, len(body), C.addressof(out))
    return bytes(out)


def build_main_packet(slice_size: int, file_ids: Sequence[bytes]) -> Tuple[bytes, bytes]:
    """(packet bytes, set_id)"""
    ids = b"".join(file_ids)
    sid = (C.c_uint8 * 16)()
    n = lib().p2g_build_main_packet(slice_size, ids, len(file_ids), None, None)
    out = (C.c_uint8 * n)()
    lib().p2g_build_main_packet(slice_size, ids, len(file_ids), C.addressof(sid), C.addressof(out))
    return bytes(out), bytes(sid)


def compute_file_id(hash16k: bytes, length: int, name: bytes) -> bytes:
    out = (C.c_uint8 * 16)()
    lib().p2g_compute_file_id(hash16k, length, name, len(name), C.addressof(out))
    return bytes(out)


def md5(data: bytes) -> bytes:
    out = (C.c_uint8 * 16)()
    lib().p2g_md5(data, len(data), C.addressof(out))
    return bytes(out)


def kernel_launch_count() -> int:
    return int(lib().p2g_kernel_launch_count())


def device_info() -> str:
    buf = C.create_string_buffer(256)
    _check(lib().p2g_device_info(buf, 256))
    return buf.value.decode()


__all__ = [
    "MAX_FILES", "MAX_INPUT_BLOCKS", "MAX_RECOVERY_BLOCKS", "HASH16K_LEN", "Par2Error", "IoError", "InvalidSliceSize",
    "InvalidFileName", "NoInputFiles", "EmptyFile", "TooManyFiles", "TooManyRecoveryBlocks", "TooManyInputBlocks",
    "InvalidVolumeScheme", "InvalidArgument", "CudaError", "OutOfMemory", "DeviceTimeout", "VolumeScheme",
    "CreateOptions", "ProgressEvent", "ProgressReporter", "SliceChecksum", "SourceFile", "run_create",
    "run_create_with_progress", "run_create_fused", "write_index_file", "create_in_memory", "gf_mul_xor", "encode",
    "encode_device", "slice_checksums", "file_hashes", "recovery_packet_md5", "input_bases", "gf_mul", "gf_pow",
    "resolve_volume_sizes", "volume_filename", "build_packet", "build_main_packet", "compute_file_id", "md5",
    "kernel_launch_count", "device_info", "DeviceJobBuffers", "run_device_job", "BATCH_NO_GRAPH",
    "BATCH_NO_AUTOTUNE", "BATCH_DERIVE_BASIS", "SOURCE_HOST", "SOURCE_SEEDED", "ServerResult", "Server",
    "copy_to_host", "BatchJobSpec", "BatchInfo", "Batch", "batch_plan",
]
