"""ctypes binding of libpar2gpu.so (the C ABI in include/par2gpu.h).

The shared library is built in-tree by ``__graft_entry__.build()`` (or
``make -C par2rust_b200/csrc``).  Loading fails loudly when it is missing:
there is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpar2gpu.so")


class p2g_error_detail(C.Structure):
    _fields_ = [("count", C.c_uint64), ("slice_size", C.c_uint64), ("suggested", C.c_uint64)]


class p2g_slice_checksum(C.Structure):
    _fields_ = [("md5", C.c_uint8 * 16), ("crc32", C.c_uint32)]


class p2g_source_file(C.Structure):
    _fields_ = [
        ("name", C.POINTER(C.c_uint8)),
        ("name_len", C.c_size_t),
        ("path", C.c_char_p),
        ("length", C.c_uint64),
        ("hash_full", C.c_uint8 * 16),
        ("hash16k", C.c_uint8 * 16),
        ("file_id", C.c_uint8 * 16),
        ("slice_checksums", C.POINTER(p2g_slice_checksum)),
        ("slice_count", C.c_uint64),
    ]


class p2g_volume_scheme(C.Structure):
    pass


p2g_volume_scheme._fields_ = [
    ("kind", C.c_uint32),
    ("count", C.c_uint32),
    ("max_blocks_per_volume", C.c_uint32),
    ("inner", C.POINTER(p2g_volume_scheme)),
    ("explicit_sizes", C.POINTER(C.c_uint32)),
    ("explicit_count", C.c_uint32),
]


class p2g_create_options(C.Structure):
    _fields_ = [
        ("output", C.c_char_p),
        ("slice_size", C.c_uint64),
        ("recovery_block_count", C.c_uint32),
        ("volume_scheme", p2g_volume_scheme),
        ("comments", C.POINTER(C.c_char_p)),
        ("comment_count", C.c_uint32),
    ]


class p2g_progress_event(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("path", C.c_char_p),
        ("total_slices", C.c_uint64),
        ("slices_done", C.c_uint64),
        ("volume_index", C.c_uint32),
        ("total_volumes", C.c_uint32),
        ("input_blocks", C.c_uint64),
        ("recovery_blocks", C.c_uint32),
        ("input_block_done", C.c_uint64),
    ]


PROGRESS_FN = C.CFUNCTYPE(None, C.POINTER(p2g_progress_event), C.c_void_p)


class p2g_path_list(C.Structure):
    _fields_ = [("paths", C.POINTER(C.c_char_p)), ("count", C.c_uint32)]


class p2g_input(C.Structure):
    _fields_ = [("path", C.c_char_p), ("display_name", C.POINTER(C.c_uint8)), ("name_len", C.c_size_t)]


class p2g_buffer_input(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("length", C.c_uint64),
        ("display_name", C.POINTER(C.c_uint8)),
        ("name_len", C.c_size_t),
    ]


class p2g_plan_item(C.Structure):
    _fields_ = [("row_group", C.c_uint32), ("fold", C.c_uint32), ("first_symbol", C.c_uint32), ("symbols", C.c_uint32),
                ("band", C.c_uint32), ("first_slice", C.c_uint32), ("slices", C.c_uint32), ("accumulate", C.c_uint32)]


class p2g_output_file(C.Structure):
    _fields_ = [("name", C.c_char_p), ("data", C.POINTER(C.c_uint8)), ("length", C.c_uint64)]


class p2g_output_set(C.Structure):
    _fields_ = [("files", C.POINTER(p2g_output_file)), ("count", C.c_uint32)]


class p2g_encode_job(C.Structure):
    _fields_ = [
        ("src", C.c_void_p),
        ("src_stride", C.c_uint64),
        ("input_count", C.c_uint32),
        ("slice_size", C.c_uint64),
        ("recovery_count", C.c_uint32),
        ("first_exponent", C.c_uint16),
        ("recovery", C.c_void_p),
        ("recovery_stride", C.c_uint64),
        ("flags", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class p2g_device_job(C.Structure):
    _fields_ = [
        ("src", C.c_void_p),
        ("file_count", C.c_uint32),
        ("file_lengths", C.POINTER(C.c_uint64)),
        ("names", C.POINTER(C.c_void_p)),
        ("name_lens", C.POINTER(C.c_size_t)),
        ("slice_size", C.c_uint64),
        ("recovery_count", C.c_uint32),
        ("recovery", C.c_void_p),
        ("recovery_stride", C.c_uint64),
        ("checksums", C.c_void_p),
        ("hash_full", C.c_void_p),
        ("hash16k", C.c_void_p),
        ("packet_md5", C.c_void_p),
        ("set_id_out", C.c_uint8 * 16),
        ("flags", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class p2g_batch_job(C.Structure):
    _fields_ = [
        ("src", C.c_void_p),
        ("file_count", C.c_uint32),
        ("file_lengths", C.POINTER(C.c_uint64)),
        ("names", C.POINTER(C.c_void_p)),
        ("name_lens", C.POINTER(C.c_size_t)),
        ("slice_size", C.c_uint64),
        ("recovery_count", C.c_uint32),
        ("recovery", C.c_void_p),
        ("recovery_stride", C.c_uint64),
        ("checksums", C.c_void_p),
        ("hash16k", C.c_void_p),
        ("packet_md5", C.c_void_p),
        ("set_id", C.c_void_p),
        ("hash_full", C.c_void_p),
    ]


class p2g_batch_info(C.Structure):
    _fields_ = [
        ("jobs", C.c_uint32),
        ("items", C.c_uint32),
        ("encode_items", C.c_uint32),
        ("scan_items", C.c_uint32),
        ("setid_items", C.c_uint32),
        ("ctas", C.c_uint32),
        ("predicted_ms", C.c_double),
        ("device_bytes", C.c_uint64),
    ]


class p2g_batch_shape(C.Structure):
    _fields_ = [
        ("slice_size", C.c_uint64),
        ("input_slices", C.c_uint32),
        ("recovery_count", C.c_uint32),
        ("file_count", C.c_uint32),
    ]


class p2g_server_options(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("wave_ms", C.c_double), ("max_jobs", C.c_uint32), ("flags", C.c_uint32)]


class p2g_server_job(C.Structure):
    _fields_ = [
        ("file_count", C.c_uint32),
        ("file_lengths", C.POINTER(C.c_uint64)),
        ("names", C.POINTER(C.c_void_p)),
        ("name_lens", C.POINTER(C.c_size_t)),
        ("slice_size", C.c_uint64),
        ("recovery_count", C.c_uint32),
        ("source_kind", C.c_uint32),
        ("host_src", C.c_void_p),
        ("file_seeds", C.POINTER(C.c_uint64)),
        ("tag", C.c_uint64),
    ]


class p2g_server_result(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("tag", C.c_uint64),
        ("status", C.c_int32),
        ("submit_s", C.c_double),
        ("admit_s", C.c_double),
        ("done_s", C.c_double),
        ("source_bytes", C.c_uint64),
        ("input_slices", C.c_uint32),
        ("recovery_count", C.c_uint32),
        ("file_count", C.c_uint32),
        ("src", C.c_void_p),
        ("recovery", C.c_void_p),
        ("recovery_stride", C.c_uint64),
        ("checksums", C.c_void_p),
        ("hash16k", C.c_void_p),
        ("packet_md5", C.c_void_p),
        ("set_id", C.c_void_p),
    ]


class p2g_server_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("admitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("released", C.c_uint64),
        ("waves", C.c_uint64),
        ("items", C.c_uint64),
        ("queued", C.c_uint32),
        ("resident", C.c_uint32),
        ("resident_bytes", C.c_uint64),
        ("peak_resident_bytes", C.c_uint64),
        ("budget_bytes", C.c_uint64),
    ]


class p2g_redundancy(C.Structure):
    _fields_ = [("is_bytes", C.c_uint32), ("percent", C.c_uint32), ("target_bytes", C.c_uint64)]


class p2g_cli_volume_flags(C.Structure):
    _fields_ = [("single_volume", C.c_uint32), ("uniform", C.c_uint32), ("limit_size", C.c_uint32),
                ("has_volume_count", C.c_uint32), ("volume_count", C.c_uint32)]


# (name, restype, argtypes) for every entry point of include/par2gpu.h
SIGNATURES = [
    ("p2g_last_error_message", C.c_char_p, []),
    ("p2g_last_error_detail", None, [C.POINTER(p2g_error_detail)]),
    ("p2g_abi_version", C.c_int, []),
    ("p2g_source_file_free", None, [C.POINTER(p2g_source_file)]),
    ("p2g_path_list_free", None, [C.POINTER(p2g_path_list)]),
    ("p2g_string_free", None, [C.c_void_p]),
    ("p2g_scan", C.c_int, [C.c_char_p, C.POINTER(C.c_uint8), C.c_size_t, C.c_uint64, C.POINTER(p2g_source_file)]),
    ("p2g_scan_with_progress", C.c_int,
     [C.c_char_p, C.POINTER(C.c_uint8), C.c_size_t, C.c_uint64, PROGRESS_FN, C.c_void_p, C.POINTER(p2g_source_file)]),
    ("p2g_run_create", C.c_int,
     [C.POINTER(p2g_create_options), C.POINTER(p2g_source_file), C.c_uint32, C.POINTER(p2g_path_list)]),
    ("p2g_run_create_with_progress", C.c_int,
     [C.POINTER(p2g_create_options), C.POINTER(p2g_source_file), C.c_uint32, PROGRESS_FN, C.c_void_p,
      C.POINTER(p2g_path_list)]),
    ("p2g_run_create_fused", C.c_int,
     [C.POINTER(p2g_create_options), C.POINTER(p2g_input), C.c_uint32, PROGRESS_FN, C.c_void_p,
      C.POINTER(p2g_path_list)]),
    ("p2g_write_index_file", C.c_int,
     [C.POINTER(p2g_create_options), C.POINTER(p2g_source_file), C.c_uint32, C.POINTER(C.c_void_p)]),
    ("p2g_create_in_memory", C.c_int,
     [C.POINTER(p2g_create_options), C.POINTER(p2g_buffer_input), C.c_uint32, C.POINTER(p2g_source_file),
      C.POINTER(p2g_output_set)]),
    ("p2g_output_set_free", None, [C.POINTER(p2g_output_set)]),
    ("p2g_gf_mul_xor", C.c_int, [C.c_uint16, C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_void_p]),
    ("p2g_encode", C.c_int, [C.POINTER(p2g_encode_job)]),
    ("p2g_encode_noalloc", C.c_int, [C.POINTER(p2g_encode_job)]),
    ("p2g_check_bounded_wait", C.c_int, [C.c_uint32]),
    ("p2g_plan_device_job", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
      C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("p2g_slice_checksums", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("p2g_file_hashes", C.c_int,
     [C.POINTER(C.c_void_p), C.POINTER(C.c_uint64), C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("p2g_recovery_packet_md5", C.c_int,
     [C.c_char_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint16, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("p2g_run_device_job", C.c_int, [C.POINTER(p2g_device_job)]),
    ("p2g_batch_create", C.c_int, [C.POINTER(p2g_batch_job), C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("p2g_batch_launch", C.c_int, [C.c_void_p, C.c_void_p]),
    ("p2g_batch_check", C.c_int, [C.c_void_p]),
    ("p2g_batch_get_info", C.c_int, [C.c_void_p, C.POINTER(p2g_batch_info)]),
    ("p2g_batch_job_tile", C.c_uint32, [C.c_void_p, C.c_uint32]),
    ("p2g_batch_destroy", None, [C.c_void_p]),
    ("p2g_batch_plan", C.c_int,
     [C.POINTER(p2g_batch_shape), C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(p2g_batch_info),
      C.POINTER(C.c_uint32)]),
    ("p2g_server_create", C.c_int, [C.POINTER(p2g_server_options), C.POINTER(C.c_void_p)]),
    ("p2g_server_submit", C.c_int, [C.c_void_p, C.POINTER(p2g_server_job), C.POINTER(C.c_uint64)]),
    ("p2g_server_poll", C.c_int,
     [C.c_void_p, C.POINTER(p2g_server_result), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
    ("p2g_server_release", C.c_int, [C.c_void_p, C.c_uint64]),
    ("p2g_server_get_stats", C.c_int, [C.c_void_p, C.POINTER(p2g_server_stats)]),
    ("p2g_server_now", C.c_double, [C.c_void_p]),
    ("p2g_server_destroy", None, [C.c_void_p]),
    ("p2g_copy_to_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    ("p2g_input_bases", C.c_int, [C.c_uint32, C.POINTER(C.c_uint16)]),
    ("p2g_gf_mul", C.c_uint16, [C.c_uint16, C.c_uint16]),
    ("p2g_gf_pow", C.c_uint16, [C.c_uint16, C.c_uint32]),
    ("p2g_resolve_volume_sizes", C.c_int,
     [C.POINTER(p2g_volume_scheme), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(C.c_uint32)]),
    ("p2g_volume_filename", C.c_void_p, [C.c_char_p, C.c_uint16, C.c_uint32]),
    ("p2g_build_packet", C.c_size_t, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t, C.c_void_p]),
    ("p2g_build_main_packet", C.c_size_t, [C.c_uint64, C.c_char_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("p2g_compute_file_id", None, [C.c_char_p, C.c_uint64, C.c_char_p, C.c_size_t, C.c_void_p]),
    ("p2g_md5", None, [C.c_char_p, C.c_size_t, C.c_void_p]),
    ("p2g_parse_slice_size", C.c_int, [C.c_char_p, C.POINTER(C.c_uint64)]),
    ("p2g_parse_redundancy", C.c_int, [C.c_char_p, C.POINTER(p2g_redundancy)]),
    ("p2g_resolve_redundancy", C.c_int, [C.POINTER(p2g_redundancy), C.c_uint64, C.c_uint64, C.POINTER(C.c_uint32)]),
    ("p2g_build_volume_scheme", C.c_int,
     [C.POINTER(p2g_cli_volume_flags), C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(p2g_volume_scheme),
      C.POINTER(p2g_volume_scheme)]),
    ("p2g_kernel_launch_count", C.c_uint64, []),
    ("p2g_device_info", C.c_int, [C.c_char_p, C.c_size_t]),
]

_lib = None


def lib() -> C.CDLL:
    """Load libpar2gpu.so once; raise (never fall back) when it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C par2rust_b200/csrc` "
                "(or __graft_entry__.build()); par2rust_b200 has no CPU fallback")
        h = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib
