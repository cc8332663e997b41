// p2g_internal.h -- launch wrappers shared between the kernel file and the
// host pipeline of libpar2gpu.so.  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "../../include/par2gpu.h"

namespace p2g {

// GF(2^16) constants of src/galois.rs:15-18.
constexpr uint32_t kFieldLimit = 65535u;
constexpr uint32_t kFieldGenerator = 0x1100Bu;

// Encode kernel geometry: 32 recovery rows per CTA ("row group"), 512
// threads, NCH chunks of 8 symbols per lane.
constexpr int kRowsPerGroup = 32;
constexpr int kEncThreads = 512;  // 16 warps: one 16-row block of each table build per warp
constexpr int kEncChunks = 2;
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
// Packet-MD5 continuation over message blocks [b_from, b_to) (state: 4
// words per row, kept between calls).
cudaError_t launch_md5_recovery_range(const uint8_t* rec, uint64_t stride, uint32_t count, uint64_t slice_size,
                                      const uint8_t set_id[16], uint32_t first_exp, uint32_t* state,
                                      uint64_t b_from, uint64_t b_to, bool final, uint8_t* out16, cudaStream_t st);
cudaError_t launch_realign(const uint8_t* src, uint64_t src_stride, uint8_t* dst,
                           uint64_t dst_stride, uint32_t count, uint64_t slice_size,
                           cudaStream_t st);

// Banded encode: band b covers symbol positions [begin, end) of every row in
// tiles of ts symbols; bands are launched in order on one stream.
struct EncodeBand {
    uint32_t begin, end, ts;
};
struct EncodePlan {
    uint32_t Np = 0;  // symbol positions processed per slice (slice rounded up to 16 B)
    std::vector<EncodeBand> bands;
};
// banded: cut into whole-wave bands (packet-MD5 pipelining); reserve/reserve_ms:
// SMs held by slice-MD5 blocks at the start of the job and for how long.
EncodePlan plan_encode(uint64_t slice_size, uint32_t S, uint32_t RG, bool banded, uint32_t reserve,
                       double reserve_ms);
cudaError_t launch_encode_band(const EncodePlan& pl, uint32_t band, const uint8_t* src, uint64_t src_stride,
                               uint32_t S, const uint16_t* basis, uint32_t RG, uint32_t R, uint8_t* rec,
                               uint64_t rec_stride, int* err, cudaStream_t st);
// Blocks (one SM each) that a hash launch over `streams` MD5 streams occupies.
uint32_t hash_blocks(uint32_t streams);

// Encode tiling: tile size (symbols, multiple of 8) and tile count for Np
// symbols, RG row groups and `sms` SMs.
void choose_tiles(uint32_t Np, uint32_t RG, uint32_t sms, uint32_t* ts_out, uint32_t* tiles_out);

// Heap-free variants used by the allocation-free entry point.
cudaError_t upload_tables_noheap();
cudaError_t launch_encode_noheap(const uint8_t* src, uint64_t src_stride, uint32_t S, const uint16_t* basis,
                                 uint32_t RG, uint32_t R, uint64_t slice_size, uint8_t* rec, uint64_t rec_stride,
                                 int* err, cudaStream_t st);

// Size in bytes of the coefficient-basis scratch for S slices and RG groups.
inline size_t basis_bytes(uint32_t S, uint32_t RG) { return (size_t)S * RG * 512 * sizeof(uint16_t); }

}  // namespace p2g
