// p2g_internal.h -- launch wrappers shared between the kernel file and the
// host pipeline of libpar2gpu.so.  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/par2gpu.h"

namespace p2g {

// GF(2^16) constants of src/galois.rs:15-18.
constexpr uint32_t kFieldLimit = 65535u;
constexpr uint32_t kFieldGenerator = 0x1100Bu;

// Encode kernel geometry: 32 recovery rows per CTA ("row group"), 256
// threads, NCH chunks of 8 symbols per lane.
constexpr int kRowsPerGroup = 32;
constexpr int kEncThreads = 256;
constexpr int kEncChunks = 4;
constexpr int kEncTileSymbols = (kEncThreads / 32) * kEncChunks * 64;  // 2048
constexpr int kEncStages = 4;

// Byte offsets of one file inside a device source buffer (used by the
// per-file MD5 kernel).
struct FileSpan {
    uint64_t offset;  // byte offset of the first byte
    uint64_t length;  // bytes hashed
};

// Upload the log/antilog and input-logbase tables into the module's
// __device__ arrays of the current device (idempotent per device).
cudaError_t upload_tables();

// Number of kernels launched so far (all wrappers bump it).
uint64_t launch_count();

cudaError_t launch_basis(uint16_t* basis, uint32_t S, uint32_t RG, uint32_t R, uint32_t first_exp,
                         cudaStream_t st);
cudaError_t launch_encode(const uint8_t* src, uint64_t src_stride, uint32_t S, const uint16_t* basis,
                          uint32_t RG, uint32_t R, uint64_t slice_size, uint8_t* rec,
                          uint64_t rec_stride, int* err, cudaStream_t st);
cudaError_t launch_gf_mul_xor(uint16_t coeff, const uint8_t* in, uint8_t* out, size_t len,
                              cudaStream_t st);
cudaError_t launch_md5_slices(const uint8_t* src, uint64_t stride, uint32_t count,
                              uint64_t slice_size, p2g_slice_checksum* out, cudaStream_t st);
cudaError_t launch_crc_slices(const uint8_t* src, uint64_t stride, uint32_t count,
                              uint64_t slice_size, p2g_slice_checksum* out, cudaStream_t st);
cudaError_t launch_md5_files(const uint8_t* base, const FileSpan* spans, uint32_t n,
                             uint8_t* out16, cudaStream_t st);
cudaError_t launch_md5_recovery(const uint8_t* rec, uint64_t stride, uint32_t count,
                                uint64_t slice_size, const uint8_t set_id[16], uint32_t first_exp,
                                uint8_t* out16, cudaStream_t st);
cudaError_t launch_realign(const uint8_t* src, uint64_t src_stride, uint8_t* dst,
                           uint64_t dst_stride, uint32_t count, uint64_t slice_size,
                           cudaStream_t st);

// Size in bytes of the coefficient-basis scratch for S slices and RG groups.
inline size_t basis_bytes(uint32_t S, uint32_t RG) { return (size_t)S * RG * 512 * sizeof(uint16_t); }

}  // namespace p2g
