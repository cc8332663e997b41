// p2g_internal.h -- launch wrappers shared between the kernel file and the
// host pipeline of libpar2gpu.so.  Not part of the public ABI.
#pragma once
#include <cuda.h>  // CUtensorMap and its enums (the encode function is looked up at run time)
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "../../include/par2gpu.h"

namespace p2g {

// CUDA error -> status (P2G_ERR_OOM for allocation failures, else
// P2G_ERR_CUDA) with the message set; clears the runtime's last error.
p2g_status cuda_fail(cudaError_t e, const char* what);
#define P2G_CU(call)                                                \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ::p2g::cuda_fail(_e, #call);  \
    } while (0)
#define P2G_TRY(expr)                \
    do {                             \
        p2g_status _s = (expr);      \
        if (_s != P2G_OK) return _s; \
    } while (0)

// Select the engine's device, check it is sm_100 and upload the GF tables
// (idempotent; serialised with the engine's other calls).
p2g_status ensure_device_ready();

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

// Number of kernels launched so far (all wrappers bump it; graph replays
// add their kernel count with add_launches).
uint64_t launch_count();
void add_launches(uint64_t n);

cudaError_t launch_basis(uint16_t* basis, uint32_t S, uint32_t RG, uint32_t R, uint32_t first_exp,
                         cudaStream_t st);
// basis == nullptr: the kernel derives the coefficient basis itself (from
// first_exp); otherwise it loads the launch_basis layout.
cudaError_t launch_encode(const uint8_t* src, uint64_t src_stride, uint32_t S, const uint16_t* basis,
                          uint32_t RG, uint32_t R, uint64_t slice_size, uint8_t* rec,
                          uint64_t rec_stride, int* err, cudaStream_t st, uint32_t first_exp = 0);
// One block waits (at most `polls` tries) on an mbarrier nothing arrives on;
// *gave_up becomes 1 when the bound fired.
cudaError_t launch_bounded_wait_probe(int* gave_up, uint32_t polls, cudaStream_t st);
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
// Copies n_seg segments from page-locked host memory to the device in one
// launch: seg (device memory) holds 3 words per segment -- host source,
// device destination, length | zero padding after it << 40.
cudaError_t launch_gather_host(const uint64_t* seg, uint32_t n_seg, cudaStream_t st);

// Banded encode: band b covers symbol positions [begin, end) of every row in
// tiles of ts symbols; bands are launched in order on one stream.
struct EncodeBand {
    uint32_t begin, end, ts;
};
struct EncodePlan {
    uint32_t Np = 0;    // symbol positions processed per slice (slice rounded up to 16 B)
    uint32_t fold = 1;  // fold of the last row group (tail_fold)
    std::vector<EncodeBand> bands;
};
// Fold of the last row group for R recovery rows: 4 when it has <= 8 real
// rows, 2 when <= 16, else 1 (its CTA then covers fold tiles).
uint32_t tail_fold(uint32_t R);
// banded: cut into whole-wave bands (packet-MD5 pipelining); reserve/reserve_ms:
// SMs held by slice-MD5 blocks at the start of the job and for how long.
EncodePlan plan_encode(uint64_t slice_size, uint32_t S, uint32_t RG, bool banded, uint32_t reserve,
                       double reserve_ms, uint32_t fold = 1);
cudaError_t launch_encode_band(const EncodePlan& pl, uint32_t band, const uint8_t* src, uint64_t src_stride,
                               uint32_t S, const uint16_t* basis, uint32_t RG, uint32_t R, uint8_t* rec,
                               uint64_t rec_stride, int* err, cudaStream_t st, uint32_t first_exp = 0);
// Blocks (one SM each) that a hash launch over `streams` MD5 streams occupies.
uint32_t hash_blocks(uint32_t streams);

// Encode tiling: tile size (symbols, multiple of 8) and tile count for Np
// symbols, RG row groups and `sms` SMs.
void choose_tiles(uint32_t Np, uint32_t RG, uint32_t sms, uint32_t* ts_out, uint32_t* tiles_out, uint32_t fold = 1);

// Heap-free variants used by the allocation-free entry point.
cudaError_t upload_tables_noheap();
cudaError_t launch_encode_noheap(const uint8_t* src, uint64_t src_stride, uint32_t S, const uint16_t* basis,
                                 uint32_t RG, uint32_t R, uint64_t slice_size, uint8_t* rec, uint64_t rec_stride,
                                 int* err, cudaStream_t st);

// Device addresses of the GF antilog and input-logbase tables (after upload_tables).
cudaError_t gf_device_tables(const uint16_t** antilog, const uint16_t** logbase);

// The encode on the tensor cores (p2g_mma.cu): a_image_kernel fills `aimg`
// (mma_aimg_bytes(S, R) of scratch) with the A operand of every 16-row tile
// and K-step, then the persistent tcgen05 kernel accumulates 16-row x
// 240-symbol tiles over all S slices.  src rows are read in whole 16-byte
// units, as by launch_encode, through a 2-D tensor map (16-byte aligned src
// and src_stride).
size_t mma_aimg_bytes(uint32_t S, uint32_t R);
// K-steps (4 slices) per 16-row tile in that image: whole 16-slice stages.
constexpr uint32_t mma_image_steps(uint32_t S) { return (S + 15) / 16 * 4; }
// The source as a 2-D tensor map of Np u16 symbols x S slices for the
// tensor-core tiles (cuTensorMapEncodeTiled, found through the runtime).
cudaError_t make_src_map(CUtensorMap* map, const void* src, uint64_t stride, uint32_t S, uint32_t Np);
cudaError_t launch_encode_mma(const uint8_t* src, uint64_t src_stride, uint32_t S, uint64_t slice_size, uint32_t R,
                              uint32_t first_exp, uint8_t* aimg, uint8_t* rec, uint64_t rec_stride, int* err,
                              cudaStream_t st);

// Size in bytes of the coefficient-basis scratch for S slices and RG groups.
inline size_t basis_bytes(uint32_t S, uint32_t RG) { return (size_t)S * RG * 512 * sizeof(uint16_t); }

// ---------------------------------------------------------------------------
// Batched create (p2g_batch.cpp): the work items of many jobs run in one
// persistent launch, one CTA per SM popping items off a device queue.
// ---------------------------------------------------------------------------
enum BatchItemKind : uint32_t {
    kItemScan = 0,    // slice MD5 of up to kScanSlices slices
    kItemEncode = 1,  // one (row group, symbol tile) of the accumulator
    kItemSetId = 3,   // hash16k, file ids and set id
    kItemPacket = 4,  // packet MD5s of recovery rows [a, a+b) (set id already written)
    kItemCrc = 5,     // slice CRC32 of slices [a, a+b)
    kItemFileHash = 6,  // whole-file MD5 (hash_full) of files [a, a+b), one lane each
    kItemEncodeMma = 7,  // one (16-row tile, 240-symbol tile) of the accumulator on the tensor cores
};
constexpr uint64_t kCrcItemBytes = 4u << 20;  // source bytes per CRC item
constexpr uint32_t kItemKindMask = 0x7Fu;
constexpr uint32_t kItemAccumulate = 0x80u;  // encode: XOR partial sums into zeroed rows
constexpr uint32_t kScanSlices = 256;        // one slice per MD5 lane
constexpr uint32_t kChainRows = 256;         // recovery rows per packet-MD5 chain token

// Encode item fields: kind_rg = kItemEncode | acc | rg << 8 | log2(fold) << 24;
// b = band << 16 | symbols.
inline uint32_t encode_kind(uint32_t rg, uint32_t fold, bool acc) {
    return kItemEncode | (acc ? kItemAccumulate : 0u) | (rg << 8) | ((fold == 4 ? 2u : fold == 2 ? 1u : 0u) << 24);
}

// Tensor-core encode item: kind_rg = kItemEncodeMma | acc | row tile << 8;
// a = first symbol, b = band << 16 | symbols (<= 240), s0/sn as for kItemEncode.
inline uint32_t encode_mma_kind(uint32_t rt, bool acc) {
    return kItemEncodeMma | (acc ? kItemAccumulate : 0u) | (rt << 8);
}
constexpr uint32_t kMmaTileSymbols = 240;  // symbols of a tensor-core tile (its MMA N)
constexpr uint32_t kMmaTileRows = 16;      // recovery rows of a tensor-core tile

struct BatchItem {
    uint32_t job;
    uint32_t kind_rg;  // kind in bits 0-6 (+ kItemAccumulate); encode: row group in bits 8-23,
                       // log2 fold in bits 24-25
    uint32_t a, b;     // scan: first slice, count; encode: first symbol, band << 16 | symbols;
                       // packet: first row, row count
    uint32_t s0, sn;   // encode: input slices [s0, s0+sn) (sn == 0: all of the job's)
};

// Device descriptor of one job.  The CTA that completes a job's last encode
// item (or runs its finish item) also derives the job's hash16k values, file
// ids, set id and recovery-packet MD5s.
struct BatchJob {
    const uint8_t* src;        // files back to back, each on a slice boundary, zero-padded
    const uint8_t* esrc;       // encode source: src, or a copy with 16-byte aligned slices
    uint16_t* basis;           // [s][row group][16][32] precomputed basis, or null: derived per slice
    uint8_t* rec;              // recovery row r at rec + r*rec_stride
    p2g_slice_checksum* checks;
    uint8_t* h16k;             // 16 bytes per file
    uint8_t* pkt;              // 16 bytes per recovery row
    uint8_t* set_id;           // 16 bytes
    uint8_t* hfull;            // 16 bytes per file (whole-file MD5), when file-hash items run
    const uint64_t* files;     // 2 per file: byte offset in src, length
    const uint8_t* names;      // display names, each starting 4-byte aligned
    const uint32_t* name_off;  // 2 per file: offset into names, length
    uint8_t* scratch;          // 16*n file ids, then the 12+16*n main-packet body
    // Recovery-packet MD5 in chain segments: the symbol range is cut into
    // n_bands bands of band_syms; when the last encode item of a band
    // completes, the chains of every 256-row block advance over that band's
    // bytes (n_bands 0: packets are separate items, as in the serving loop).
    uint32_t* bstate;            // per run, zeroed: [n_bands] items done, [Q] next band, [Q] token, [1] set id ready
    const uint32_t* band_items;  // [n_bands] encode items per band
    uint32_t* chain;             // 4 words of MD5 state per recovery row
    uint64_t slice, estride, rec_stride;
    uint32_t S, R, RG, n_files;
    uint32_t n_bands, band_syms;
    uint32_t ts, first_exp;  // ts: tile width (sub-tile width of folded items)
    uint32_t vec;            // slices and file starts of src are 16-byte aligned
    uint32_t mma;            // encode items run on the tensor cores (kItemEncodeMma)
    uint8_t* aimg;           // mma: the A operand image (mma_aimg_bytes)
    uint32_t Rpad, ksteps;   // mma: R rounded up to whole 16-row tiles; the image's K-steps per tile
    CUtensorMap src_map;     // mma: esrc as a 2-D tensor (make_src_map); 64-byte aligned
};

// Items of one job run alone through the persistent kernel (the plain
// device-job path): scans / set-id item / packet-MD5 chains as requested.
struct SingleJobPlan {
    std::vector<BatchItem> items;    // job index 0
    std::vector<uint32_t> band_items;  // empty: no chains
    uint32_t band_syms = 0, ts = 0;
    // recovery columns [zero_from_sym, Np) are written by XOR-accumulating
    // items: the caller zeroes them first (Np: none)
    uint32_t zero_from_sym = 0;
    double predicted_ms = 0;
};
// file_bytes: largest file (non-zero: whole-file MD5 items, 256 files each);
// split_tail: the caller zeroes the columns from zero_from_sym, so the last
// bands' encode items may be cut into accumulating slice ranges.
// mma: encode items on the tensor cores (kItemEncodeMma).
SingleJobPlan plan_single_job(uint64_t slice, uint32_t S, uint32_t R, uint32_t n_files, bool scans, bool set_id,
                              bool chains, uint32_t ctas, uint64_t file_bytes = 0, bool split_tail = false,
                              bool mma = false);
// Shared memory of one batch CTA.
size_t batch_smem_bytes();
// Fills every job's basis (one launch; blockIdx.y = job).
cudaError_t launch_basis_batch(const BatchJob* jobs, uint32_t n_jobs, uint64_t max_words, cudaStream_t st);
// The persistent kernel: `ctas` CTAs; ctl[0] queue head, ctl[1+j] completed
// encode items of job j (zeroed before each launch).
// Seeded synthetic files (3 words per file in `spans`: offset, length,
// padded length; one seed per file), blockIdx.y = file.
cudaError_t launch_seeded_fill(uint8_t* base, const uint64_t* spans, const uint64_t* seeds, uint32_t n_files,
                               uint64_t max_padded, cudaStream_t st);
// Cost model shared by the batch planner and the server's wave builder
// (milliseconds of one CTA).
double est_md5_ms(uint64_t bytes);
double est_encode_item_ms(uint32_t slices, uint32_t syms);
double est_mma_item_ms(uint32_t slices);
// CTA-milliseconds of a job's encode on the lookup or the tensor-core kernel
// (cost model), and whether the tensor cores are the cheaper.
double encode_cost_ms(uint64_t slice, uint32_t S, uint32_t R, bool mma);
bool prefer_mma(uint64_t slice, uint32_t S, uint32_t R);
double est_scan_item_ms(uint64_t slice, uint32_t count);
double est_crc_item_ms(uint64_t slice, uint32_t count);
// slices per CRC item: ~kCrcItemBytes, at least 1, at most kScanSlices
inline uint32_t crc_item_slices(uint64_t slice) {
    const uint64_t n = kCrcItemBytes / slice;
    return (uint32_t)(n < 1 ? 1 : n > kScanSlices ? kScanSlices : n);
}
double est_set_id_ms(uint32_t files);
double est_packet_item_ms(uint64_t slice, uint32_t rows);
// Sets the batch kernel's shared-memory attribute (call before stream capture).
cudaError_t prepare_batch_kernel();
// mma: the batch has tensor-core encode items (the CTAs allocate TMEM and
// need the G^-1 tables of mma_tables_ready()).
cudaError_t launch_batch(const BatchJob* jobs, const BatchItem* items, uint32_t n_items, uint32_t* ctl, int* err,
                         uint32_t ctas, cudaStream_t st, bool mma = false);
// Device address of the 512 G^-1 table entries (256 for the low byte, 256 for
// the high) after a one-time set-up of the tensor-core tables on this device.
cudaError_t mma_tables_ready(const uint16_t** ginv);
// Fills every tensor-core job's A image (blockIdx.y = job); max_bytes: the
// largest image.
cudaError_t launch_a_image_batch(const BatchJob* jobs, uint32_t n_jobs, uint64_t max_bytes, cudaStream_t st);
int device_sm_count();

}  // namespace p2g
