/*
 * par2gpu.h -- C ABI of the B200 PAR2 create engine (libpar2gpu.so).
 *
 * Drop-in boundary for the create path of javi11/par2rust v0.1.0.  Each entry
 * point below names the reference interface it replaces (file:line within the
 * par2rust crate).  Plain pointers and sizes only; no CUDA or torch types in
 * the signatures (streams are passed as `void *` holding a cudaStream_t).
 *
 * Threading: calls are synchronous and thread-safe; the library serialises
 * work on its per-process device context.  Progress callbacks run on the
 * calling thread.  Strings and arrays returned by the library are owned by
 * the caller and released with the matching p2g_*_free function.
 *
 * Errors: every entry point returns a p2g_status.  The P2G_ERR_* values from
 * IO to INVALID_VOLUME_SCHEME map one to one onto the reference's Par2Error
 * variants (src/error.rs:7-41); p2g_last_error_message() gives the same text
 * and p2g_last_error_detail() the TooManyInputBlocks fields (thread-local).
 */
#ifndef PAR2GPU_H
#define PAR2GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P2G_ABI_VERSION 1

/* src/creator.rs:102-108 */
#define P2G_MAX_FILES 32768u
#define P2G_MAX_INPUT_BLOCKS 32768u
#define P2G_MAX_RECOVERY_BLOCKS 65535u
/* src/source.rs:17 */
#define P2G_HASH16K_LEN 16384u

/* Par2Error, src/error.rs:7-41, plus the device-side failures. */
typedef enum p2g_status {
    P2G_OK = 0,
    P2G_ERR_IO = 1,                      /* Par2Error::Io */
    P2G_ERR_INVALID_SLICE_SIZE = 2,      /* Par2Error::InvalidSliceSize */
    P2G_ERR_INVALID_FILE_NAME = 3,       /* Par2Error::InvalidFileName */
    P2G_ERR_NO_INPUT_FILES = 4,          /* Par2Error::NoInputFiles */
    P2G_ERR_EMPTY_FILE = 5,              /* Par2Error::EmptyFile */
    P2G_ERR_TOO_MANY_FILES = 6,          /* Par2Error::TooManyFiles */
    P2G_ERR_TOO_MANY_RECOVERY_BLOCKS = 7,/* Par2Error::TooManyRecoveryBlocks */
    P2G_ERR_TOO_MANY_INPUT_BLOCKS = 8,   /* Par2Error::TooManyInputBlocks */
    P2G_ERR_INVALID_VOLUME_SCHEME = 9,   /* Par2Error::InvalidVolumeScheme */
    P2G_ERR_INVALID_ARGUMENT = 20,       /* bad pointer / alignment / size at the ABI */
    P2G_ERR_CUDA = 21,                   /* CUDA runtime error or no usable device */
    P2G_ERR_OOM = 22,                    /* device or pinned-host allocation failed */
    P2G_ERR_TIMEOUT = 23                 /* a bounded device wait gave up */
} p2g_status;

/* Par2Error::TooManyInputBlocks{count, slice_size, suggested}, src/error.rs:29-37 */
typedef struct p2g_error_detail {
    uint64_t count;
    uint64_t slice_size;
    uint64_t suggested;
} p2g_error_detail;

const char *p2g_last_error_message(void);
void p2g_last_error_detail(p2g_error_detail *out);
int p2g_abi_version(void);

/* SliceChecksum, src/source.rs:28-31.  20 bytes, exactly one IFSC entry
 * (md5 ‖ crc32 little-endian), src/packet/file_verify.rs:12-23. */
typedef struct p2g_slice_checksum {
    uint8_t md5[16];
    uint32_t crc32;
} p2g_slice_checksum;

/* SourceFile, src/source.rs:37-47.  Filled by p2g_scan; freed with
 * p2g_source_file_free.  Callers may also fill one themselves (as the
 * reference's tests fabricate SourceFile values). */
typedef struct p2g_source_file {
    uint8_t *name;      /* display name bytes, no NUL terminator required */
    size_t name_len;
    char *path;         /* NUL-terminated on-disk path */
    uint64_t length;
    uint8_t hash_full[16];
    uint8_t hash16k[16];
    uint8_t file_id[16];
    p2g_slice_checksum *slice_checksums;
    uint64_t slice_count;
} p2g_source_file;
void p2g_source_file_free(p2g_source_file *sf);

/* VolumeScheme, src/creator.rs:111-139. */
typedef enum p2g_scheme_kind {
    P2G_SCHEME_SINGLE = 0,
    P2G_SCHEME_EXPONENTIAL = 1,
    P2G_SCHEME_UNIFORM = 2,  /* Uniform{count} */
    P2G_SCHEME_LIMITED = 3,  /* Limited{max_blocks_per_volume, inner} */
    P2G_SCHEME_EXPLICIT = 4  /* Explicit(sizes) */
} p2g_scheme_kind;
typedef struct p2g_volume_scheme {
    uint32_t kind;
    uint32_t count;
    uint32_t max_blocks_per_volume;
    const struct p2g_volume_scheme *inner;
    const uint32_t *explicit_sizes;
    uint32_t explicit_count;
} p2g_volume_scheme;

/* CreateOptions, src/creator.rs:142-173 (defaults: slice 4096, R 0, Single). */
typedef struct p2g_create_options {
    const char *output;
    uint64_t slice_size;
    uint32_t recovery_block_count;
    p2g_volume_scheme volume_scheme;
    const char *const *comments; /* UTF-8 strings */
    uint32_t comment_count;
} p2g_create_options;

/* ProgressEvent, src/progress.rs:26-60. */
typedef enum p2g_event_kind {
    P2G_EV_SCAN_STARTED = 0,
    P2G_EV_SCAN_PROGRESS = 1,
    P2G_EV_SCAN_COMPLETED = 2,
    P2G_EV_ENCODE_STARTED = 3,
    P2G_EV_ENCODE_PROGRESS = 4,
    P2G_EV_ENCODE_COMPLETED = 5,
    P2G_EV_INDEX_WRITTEN = 6,
    P2G_EV_VOLUME_WRITTEN = 7
} p2g_event_kind;
typedef struct p2g_progress_event {
    uint32_t kind;
    const char *path;
    uint64_t total_slices;
    uint64_t slices_done;
    uint32_t volume_index;
    uint32_t total_volumes;
    uint64_t input_blocks;
    uint32_t recovery_blocks;
    uint64_t input_block_done;
} p2g_progress_event;
/* ProgressReporter::on_event, src/progress.rs:18-20 */
typedef void (*p2g_progress_fn)(const p2g_progress_event *ev, void *user);

typedef struct p2g_path_list {
    char **paths;
    uint32_t count;
} p2g_path_list;
void p2g_path_list_free(p2g_path_list *pl);
void p2g_string_free(char *s);

/* ---- create pipeline ------------------------------------------------- */

/* SourceFile::scan, src/source.rs:53-55 / scan_with_progress :59-136.
 * Per-slice MD5+CRC32, hash16k and hash_full run on the device. */
p2g_status p2g_scan(const char *path, const uint8_t *display_name, size_t name_len,
                    uint64_t slice_size, p2g_source_file *out);
p2g_status p2g_scan_with_progress(const char *path, const uint8_t *display_name,
                                  size_t name_len, uint64_t slice_size, p2g_progress_fn cb,
                                  void *user, p2g_source_file *out);

/* run_create, src/creator.rs:182-184 / run_create_with_progress :188-321.
 * Writes the index and volume files; `out` lists them, index first. */
p2g_status p2g_run_create(const p2g_create_options *opts, const p2g_source_file *sources,
                          uint32_t n, p2g_path_list *out);
p2g_status p2g_run_create_with_progress(const p2g_create_options *opts,
                                        const p2g_source_file *sources, uint32_t n,
                                        p2g_progress_fn cb, void *user, p2g_path_list *out);

/* run_create_fused, src/creator.rs:447-700: inputs are (path, display name)
 * pairs; each file is read once and scanned and encoded from the same
 * device-resident copy. */
typedef struct p2g_input {
    const char *path;
    const uint8_t *display_name;
    size_t name_len;
} p2g_input;
p2g_status p2g_run_create_fused(const p2g_create_options *opts, const p2g_input *inputs,
                                uint32_t n, p2g_progress_fn cb, void *user, p2g_path_list *out);

/* write_index_file, src/creator.rs:847-860 */
p2g_status p2g_write_index_file(const p2g_create_options *opts, const p2g_source_file *sources,
                                uint32_t n, char **out_path);

/* In-memory form of run_create_fused (no filesystem): the same index and
 * volume bytes, returned in caller-freed buffers.  `sources_out`, when not
 * NULL, receives n scanned SourceFile records (free each with
 * p2g_source_file_free).  Inputs are host pointers (pinned memory is copied
 * without staging). */
typedef struct p2g_buffer_input {
    const uint8_t *data;
    uint64_t length;
    const uint8_t *display_name;
    size_t name_len;
} p2g_buffer_input;
typedef struct p2g_output_file {
    char *name;
    uint8_t *data;
    uint64_t length;
} p2g_output_file;
typedef struct p2g_output_set {
    p2g_output_file *files;
    uint32_t count;
} p2g_output_set;
p2g_status p2g_create_in_memory(const p2g_create_options *opts, const p2g_buffer_input *inputs,
                                uint32_t n, p2g_source_file *sources_out, p2g_output_set *out);
void p2g_output_set_free(p2g_output_set *os);

/* ---- failure-path check (no counterpart in the reference) ------------
 * Every device wait in this library is bounded: when a copy or a chain
 * step it waits for never completes, the kernel gives up, records it, and
 * the call returns P2G_ERR_TIMEOUT with the device still usable.  This runs
 * that path on purpose: one block waits on a barrier that nothing ever
 * completes, for at most `polls` tries (1..2^24), and the call returns
 * P2G_ERR_TIMEOUT when the bound fired (it always should). */
p2g_status p2g_check_bounded_wait(uint32_t polls);

/* ---- hot-path seams -------------------------------------------------- */

/* Pointer placement for the seams below. */
#define P2G_HOST_POINTERS 0u
#define P2G_DEVICE_POINTERS 1u

/* gf_mul_xor_dispatch, src/galois_simd.rs:640-643 (and the scalar reference
 * gf_mul_xor_scalar, src/reedsolomon.rs:87-126): out ^= coeff * in over
 * little-endian GF(2^16) symbols.  len must be even. */
p2g_status p2g_gf_mul_xor(uint16_t coeff, const uint8_t *input, uint8_t *output, size_t len,
                          uint32_t flags, void *stream);

/* encode_all_recovery_blocks, src/creator.rs:883-1018 (RsEncoder
 * src/reedsolomon.rs:39-60): recovery[r] = XOR_s c(r,s) * source[s] with
 * c(r,s) = base_s ^ (first_exponent + r).  Source slice s is read at
 * src + s*src_stride (zero-padded slices), recovery row r is written at
 * recovery + r*recovery_stride.  With P2G_DEVICE_POINTERS, src_stride and
 * recovery_stride must be multiples of 16 and both pointers 16-byte
 * aligned, and the work is enqueued on `stream` (0 = legacy default); a
 * call waits on `stream` for the previous device-pointer call's use of the
 * library's scratch (coefficient tables, error word), whatever its stream
 * (not while `stream` is being captured into a graph: captured calls must
 * not overlap other device-pointer encodes).
 * Device rows are read and written in whole 16-byte units: bytes
 * [slice_size, round_up(slice_size, 16)) of every source row are read --
 * for the last row too, so src must be readable up to
 * (input_count-1)*src_stride + round_up(slice_size, 16) -- and the same
 * bytes of every recovery row receive unspecified values (bytes
 * [0, slice_size) do not depend on them).  With P2G_ENCODE_WAIT the call
 * waits for its work on `stream` and returns P2G_ERR_TIMEOUT when a
 * bounded device wait gave up (the rows are then not valid); without it a
 * device timeout is not reported. */
#define P2G_ENCODE_WAIT 4u
/* Encode kernel: by default chosen per shape; these force the shared-memory
 * lookup kernel or the tensor-core (tcgen05) bit-sliced kernel.  Both give
 * the same bytes. */
#define P2G_ENCODE_LUT 8u
#define P2G_ENCODE_TENSOR 16u
typedef struct p2g_encode_job {
    const uint8_t *src;
    uint64_t src_stride;
    uint32_t input_count;
    uint64_t slice_size;
    uint32_t recovery_count;
    uint16_t first_exponent;
    uint8_t *recovery;
    uint64_t recovery_stride;
    uint32_t flags;
    void *stream;
} p2g_encode_job;
p2g_status p2g_encode(const p2g_encode_job *job);

/* p2g_encode without any allocation by the library.  No counterpart in the
 * reference: it exists for callers that must own all device memory (a
 * caching allocator or memory pool that accounts for every byte, a hard
 * memory cap, or a latency-critical path where cudaMalloc/cudaFree would
 * synchronise the device), and so cannot let the library call cudaMalloc.
 * Device pointers only (P2G_DEVICE_POINTERS), same alignment rules as
 * p2g_encode.  Its scratch is a fixed 8 MiB array inside the library
 * (present on every GPU that loads it, until exit), which limits a call to
 * input_count * ceil(recovery_count/32) <= 8192; larger jobs get
 * P2G_ERR_INVALID_ARGUMENT.  The first call on a device uploads tables and
 * looks up the scratch address; make that first call before any stream
 * capture.  All calls share the one scratch array, so calls whose work
 * overlaps on the GPU (other streams, other threads) race: order them on one
 * stream or synchronise between them.  Work is enqueued on `stream`; the
 * padding reads and writes of p2g_encode's device form apply.  Its device
 * error flag is part of the shared scratch: P2G_ENCODE_WAIT waits for the
 * call's work and reads the flag back into a local variable (no allocation),
 * returning P2G_ERR_TIMEOUT when a bounded device wait gave up. */
p2g_status p2g_encode_noalloc(const p2g_encode_job *job);

/* The per-slice half of scan_via_mmap, src/source.rs:165-220: MD5 and
 * CRC32 of `count` slices (slice i at src + i*src_stride, slice_size bytes,
 * already zero-padded). */
p2g_status p2g_slice_checksums(const uint8_t *src, uint64_t src_stride, uint32_t count,
                               uint64_t slice_size, p2g_slice_checksum *out, uint32_t flags,
                               void *stream);

/* The file half of scan_via_mmap, src/source.rs:222-228: hash_full (MD5 of
 * the real bytes) and hash16k (MD5 of the first min(len,16384) bytes) of
 * `n` files, file f at data[f] (host or device per flags). */
p2g_status p2g_file_hashes(const uint8_t *const *data, const uint64_t *lengths, uint32_t n,
                           uint8_t *hash_full_out, uint8_t *hash16k_out, uint32_t flags,
                           void *stream);

/* The packet MD5 of build_recovery_packet + build_packet
 * (src/packet/recovery.rs:11-19, src/format.rs:33-54): for each row r,
 * MD5(set_id ‖ "PAR 2.0\0RecvSlic" ‖ le32(first_exponent+r) ‖ row r). */
p2g_status p2g_recovery_packet_md5(const uint8_t set_id[16], const uint8_t *recovery,
                                   uint64_t recovery_stride, uint32_t count, uint64_t slice_size,
                                   uint16_t first_exponent, uint8_t *md5_out, uint32_t flags,
                                   void *stream);

/* One whole create job with the source already in device memory: the
 * device work of run_create_fused minus file I/O.  `src` holds the n files
 * back to back in caller order, each starting on a slice boundary and
 * zero-padded to a whole number of slices (slice s at src + s*slice_size).
 * Produces, in device memory: recovery rows (recovery_stride apart), the
 * per-slice checksums, hash16k and (unless P2G_JOB_SKIP_HASH_FULL) hash_full
 * per file, and the recovery-packet MD5s.  The set id is derived on the host
 * from the device hash16k values (src/source.rs:303-309,
 * src/packet/main_packet.rs:25-42); names are the files' display names.
 * All work is ordered on `stream`. */
#define P2G_JOB_SKIP_HASH_FULL 2u
/* p2g_device_job.flags may also carry P2G_ENCODE_LUT or P2G_ENCODE_TENSOR
 * to force the encode kernel (by default it is chosen by shape). */
typedef struct p2g_device_job {
    const uint8_t *src;
    uint32_t file_count;
    const uint64_t *file_lengths;       /* host array */
    const uint8_t *const *names;        /* host array of display names */
    const size_t *name_lens;
    uint64_t slice_size;
    uint32_t recovery_count;
    uint8_t *recovery;                  /* device */
    uint64_t recovery_stride;
    p2g_slice_checksum *checksums;      /* device, one per input slice */
    uint8_t *hash_full;                 /* device, 16 per file */
    uint8_t *hash16k;                   /* device, 16 per file */
    uint8_t *packet_md5;                /* device, 16 per recovery row */
    uint8_t set_id_out[16];             /* host, filled */
    uint32_t flags;
    void *stream;
} p2g_device_job;
p2g_status p2g_run_device_job(p2g_device_job *job);

/* ---- batched create (no counterpart in par2rust, which runs one create
 * at a time: run_create, src/creator.rs:188-321) ------------------------
 * Many independent create jobs, each described like p2g_device_job, run in
 * one persistent launch: one CTA per SM pops (job, row group, symbol tile)
 * encode items and (job, 256-slice) scan items off a device queue; the CTA
 * that completes a job's last encode item derives that job's hash16k, file
 * ids, set id (on the device) and recovery-packet MD5s.  Per job the device
 * outputs are byte-identical to p2g_run_device_job; hash_full is computed
 * only when its output is given (one chain per file, which bounds the batch by
 * its largest file), else it stays with the caller, who usually hashes files
 * on the host while reading them.  An autotuner picks each job's
 * tile width and the queue order by simulating the launch with a cost model.
 * Coefficient bases are precomputed into batch scratch (S x ceil(R/32) x
 * 1 KiB per job) while the batch's total stays within 16 GiB
 * (P2G_BATCH_BASIS_BUDGET bytes); beyond that, or with
 * P2G_BATCH_DERIVE_BASIS, each encode item derives its basis in the kernel.
 * The launch sequence (queue reset, bases, any realignment, the persistent
 * kernel) is captured once into a CUDA graph and replayed. */
typedef struct p2g_batch_job {
    const uint8_t *src;                 /* device, 16-byte aligned; layout as in p2g_device_job */
    uint32_t file_count;
    const uint64_t *file_lengths;       /* host array */
    const uint8_t *const *names;        /* host array of display names */
    const size_t *name_lens;
    uint64_t slice_size;
    uint32_t recovery_count;
    uint8_t *recovery;                  /* device, 16-byte aligned */
    uint64_t recovery_stride;           /* multiple of 16, >= slice_size rounded up to 16 */
    p2g_slice_checksum *checksums;      /* device, one per input slice */
    uint8_t *hash16k;                   /* device, 16 per file */
    uint8_t *packet_md5;                /* device, 16 per recovery row */
    uint8_t *set_id;                    /* device, 16 bytes, 4-byte aligned */
    uint8_t *hash_full;                 /* device, 16 per file, 4-byte aligned; NULL: the caller hashes
                                           whole files itself (one serial MD5 chain per file) */
} p2g_batch_job;

typedef struct p2g_batch p2g_batch;     /* opaque */

typedef struct p2g_batch_info {
    uint32_t jobs, items;
    uint32_t encode_items, scan_items, setid_items;
    uint32_t ctas;                      /* persistent CTAs (one per SM) */
    double predicted_ms;                /* the autotuner's makespan estimate */
    uint64_t device_bytes;              /* scratch the batch holds (bases, tables, queue) */
} p2g_batch_info;

/* Shape of one job, for the host-only planner. */
typedef struct p2g_batch_shape {
    uint64_t slice_size;
    uint32_t input_slices;
    uint32_t recovery_count;
    uint32_t file_count;
} p2g_batch_shape;

#define P2G_BATCH_NO_GRAPH 1u           /* launch directly instead of replaying a CUDA graph */
#define P2G_BATCH_NO_AUTOTUNE 2u        /* widest tiles and cost order, no tile search */
#define P2G_BATCH_DERIVE_BASIS 4u       /* no basis scratch: encode items derive their bases */
#define P2G_BATCH_TENSOR 8u             /* every job's encode on the tensor cores (tcgen05) */
#define P2G_BATCH_LUT 16u               /* every job's encode on the shared-memory lookup kernel
                                           (neither flag: one kernel for the whole batch, the
                                           cheaper for its jobs by the cost model) */

/* Validate the jobs (the checks of p2g_run_device_job), plan the items and
 * allocate the batch's device scratch.  The job buffers must stay valid
 * while the batch is used; contents may change between launches. */
p2g_status p2g_batch_create(const p2g_batch_job *jobs, uint32_t n, uint32_t flags, p2g_batch **out);
/* Enqueue one run of the whole batch on `stream` (one run at a time per batch). */
p2g_status p2g_batch_launch(p2g_batch *batch, void *stream);
/* After the run's stream has been synchronised: P2G_ERR_TIMEOUT when a
 * bounded device wait gave up, else P2G_OK. */
p2g_status p2g_batch_check(p2g_batch *batch);
p2g_status p2g_batch_get_info(const p2g_batch *batch, p2g_batch_info *out);
/* Tile width (symbols) the autotuner chose for job `job`; 0 if out of range. */
uint32_t p2g_batch_job_tile(const p2g_batch *batch, uint32_t job);
void p2g_batch_destroy(p2g_batch *batch);
/* The planner alone (no device): items and predicted makespan for `ctas`
 * CTAs; tiles_out (optional, n entries) receives each job's tile width. */
p2g_status p2g_batch_plan(const p2g_batch_shape *shapes, uint32_t n, uint32_t ctas, uint32_t flags,
                          p2g_batch_info *info, uint32_t *tiles_out);

/* The plan one device job (p2g_run_device_job) runs when it computes the
 * slice checksums and derives the set id on the device and leaves hash_full
 * to the host (P2G_JOB_SKIP_HASH_FULL, or a single large file), from the
 * host-only planner, for inspection; P2G_TAIL_SPLIT=0 in the environment
 * turns the tail split off here as it does for the job, and the encode
 * kernel is chosen as for the job (P2G_ENCODE_VARIANT, else by shape).  Lookup
 * kernel items cover 32-row groups (fold 1, 2 or 4 for a short last group);
 * tensor-core items have fold 0 and cover 16-row tiles of at most 240
 * symbols.  It returns up to `cap` encode items as (row group, fold,
 * first symbol, symbols, band, first slice, slice count, accumulate), the
 * number of encode items, and the first symbol of the columns that are
 * zeroed for accumulating items (the padded row width when there are none).
 * `with_chains` plans packet-MD5 chains as the job with packet MD5s does. */
typedef struct p2g_plan_item {
    uint32_t row_group, fold, first_symbol, symbols, band, first_slice, slices, accumulate;
} p2g_plan_item;
p2g_status p2g_plan_device_job(uint64_t slice_size, uint32_t input_slices, uint32_t recovery_count,
                               uint32_t file_count, uint32_t with_chains, uint32_t ctas,
                               p2g_plan_item *items, uint32_t cap, uint32_t *n_items,
                               uint32_t *zero_from_symbol, uint32_t *band_count);

/* ---- serving loop (no counterpart in par2rust, which runs one create at
 * a time) ------------------------------------------------------------------
 * A request loop with continuous batching.  Submitted create jobs wait in
 * arrival order until their footprint (padded source + recovery rows) fits
 * the HBM budget beside the resident jobs; admission then allocates their
 * device memory from the stream-ordered pool and brings the source in.  The
 * device runs back-to-back "waves" of the persistent batch kernel, each
 * taking a fair share of work items from every resident job, so requests
 * that arrive while others are on the GPU start in the next wave and their
 * work overlaps.  Outputs (as for p2g_batch_job, hash_full excluded) stay in
 * device memory until the caller releases the job.  A scheduler thread
 * inside the library drives admission and waves; all calls are thread-safe.
 * A job's encode runs on the tensor cores when the cost model prefers that
 * and its coefficient image (recovery_count x input slices x 128 bytes,
 * counted in its footprint) is at most a quarter of its source bytes, else
 * on the lookup kernel; P2G_ENCODE_VARIANT=lut|tensor in the environment
 * overrides the preference.  Each job's outputs are byte-identical to the
 * same job run alone. */
typedef struct p2g_server p2g_server;   /* opaque */
typedef struct p2g_server_options {
    uint64_t hbm_budget;                /* bytes of source + recovery resident jobs may hold (0: 120e9) */
    double wave_ms;                     /* target device time of one wave (0: 20) */
    uint32_t max_jobs;                  /* resident job slots (0: 1024) */
    uint32_t flags;                     /* reserved, 0 */
} p2g_server_options;

#define P2G_SOURCE_HOST 0u              /* host_src: the files back to back, slice-padded, copied at admission
                                           (pinned memory copies asynchronously); keep it until the job completes */
#define P2G_SOURCE_SEEDED 1u            /* file_seeds: each file generated on the device as the splitmix64 counter
                                           stream of its seed (synthetic requests for benchmarks and tests) */
typedef struct p2g_server_job {
    uint32_t file_count;
    const uint64_t *file_lengths;       /* host arrays, copied at submit */
    const uint8_t *const *names;
    const size_t *name_lens;
    uint64_t slice_size;
    uint32_t recovery_count;
    uint32_t source_kind;
    const uint8_t *host_src;
    const uint64_t *file_seeds;
    uint64_t tag;                       /* caller's id, returned with the result */
} p2g_server_job;

typedef struct p2g_server_result {
    uint64_t ticket, tag;
    int32_t status;                     /* P2G_OK or the job's failure */
    double submit_s, admit_s, done_s;   /* server clock (p2g_server_now) */
    uint64_t source_bytes;
    uint32_t input_slices, recovery_count, file_count;
    const uint8_t *src;                 /* device pointers, valid until p2g_server_release */
    const uint8_t *recovery;
    uint64_t recovery_stride;
    const p2g_slice_checksum *checksums;
    const uint8_t *hash16k;
    const uint8_t *packet_md5;
    const uint8_t *set_id;
} p2g_server_result;

typedef struct p2g_server_stats {
    uint64_t submitted, admitted, completed, released;
    uint64_t waves, items;
    uint32_t queued, resident;
    uint64_t resident_bytes, peak_resident_bytes, budget_bytes;
} p2g_server_stats;

p2g_status p2g_server_create(const p2g_server_options *opts, p2g_server **out);
/* Validates (as p2g_run_device_job) and queues one job; never blocks on the device. */
p2g_status p2g_server_submit(p2g_server *server, const p2g_server_job *job, uint64_t *ticket);
/* Up to cap completed jobs not yet polled; waits up to wait_ms for the first. */
p2g_status p2g_server_poll(p2g_server *server, p2g_server_result *out, uint32_t cap, uint32_t *n_out,
                           uint32_t wait_ms);
/* Frees a completed job's device memory (after the caller's reads of it have finished). */
p2g_status p2g_server_release(p2g_server *server, uint64_t ticket);
p2g_status p2g_server_get_stats(p2g_server *server, p2g_server_stats *out);
double p2g_server_now(p2g_server *server);
/* Stops the scheduler, waits for the device, frees every job. */
void p2g_server_destroy(p2g_server *server);
/* Synchronous device-to-host copy of result bytes (for callers that do not
 * link the CUDA runtime themselves). */
p2g_status p2g_copy_to_host(void *dst, const void *device_src, uint64_t bytes);

/* ---- host helpers of the reference's public format/packet modules ----- */

/* generate_input_bases, src/reedsolomon.rs:130-149 */
p2g_status p2g_input_bases(uint32_t count, uint16_t *out);
/* gf_mul / gf_pow, src/galois.rs:57-87 */
uint16_t p2g_gf_mul(uint16_t a, uint16_t b);
uint16_t p2g_gf_pow(uint16_t base, uint32_t exp);
/* resolve_volume_sizes, src/creator.rs:325-431: returns the volume count in
 * *n_out (sizes written when out != NULL and cap allows). */
p2g_status p2g_resolve_volume_sizes(const p2g_volume_scheme *scheme, uint32_t total,
                                    uint32_t *out, uint32_t cap, uint32_t *n_out);
/* derive_volume_filename, src/creator.rs:1046-1057 (caller frees) */
char *p2g_volume_filename(const char *index_path, uint16_t first_exponent, uint32_t count);
/* build_packet, src/format.rs:33-54; returns the packet length, writes when out != NULL */
size_t p2g_build_packet(const uint8_t set_id[16], const uint8_t type_tag[16],
                        const uint8_t *body, size_t body_len, uint8_t *out);
/* build_main_packet, src/packet/main_packet.rs:25-42 */
size_t p2g_build_main_packet(uint64_t slice_size, const uint8_t *file_ids, uint32_t n,
                             uint8_t set_id_out[16], uint8_t *out);
/* compute_file_id, src/source.rs:303-309 */
void p2g_compute_file_id(const uint8_t hash16k[16], uint64_t length, const uint8_t *name,
                         size_t name_len, uint8_t out[16]);
/* host MD5 used for packet framing (md5_impl::digest, src/md5_impl.rs:24-48) */
void p2g_md5(const uint8_t *data, size_t len, uint8_t out[16]);

/* ---- create CLI glue (src/main.rs) ------------------------------------
 * The argument semantics of `par2rust create`: they decide the bytes a
 * create writes (-r sets the recovery count, -l caps volume sizes).  The
 * par2rust executable built beside libpar2gpu.so is a shell around these
 * and the create entry points above.  Errors carry the reference's texts. */

/* parse_slice_size, src/main.rs:464-487: a bare integer (bytes) or one with
 * a suffix b/B (bytes), k/K (KiB), m/M (MiB), g/G (GiB).  Bad input:
 * P2G_ERR_INVALID_ARGUMENT. */
p2g_status p2g_parse_slice_size(const char *s, uint64_t *out);

/* Redundancy, src/main.rs:489-531: the `-r` value, a percentage of the
 * input ("10") or a target recovery-data size with a unit prefix ("k500",
 * "m10", "g2"; case-insensitive).  Bad input: P2G_ERR_INVALID_ARGUMENT. */
typedef struct p2g_redundancy {
    uint32_t is_bytes;     /* 0: Percent(percent), 1: TargetBytes(target_bytes) */
    uint32_t percent;
    uint64_t target_bytes;
} p2g_redundancy;
p2g_status p2g_parse_redundancy(const char *s, p2g_redundancy *out);

/* resolve_redundancy, src/main.rs:533-556: the recovery count for inputs of
 * `total_input_blocks` slices: ceil(total * percent / 100) or
 * ceil(target_bytes / slice_size), saturated to u32; 0 blocks is
 * P2G_ERR_INVALID_VOLUME_SCHEME. */
p2g_status p2g_resolve_redundancy(const p2g_redundancy *r, uint64_t total_input_blocks,
                                  uint64_t slice_size, uint32_t *out);

/* build_volume_scheme, src/main.rs:289-337: the VolumeScheme of the
 * --single-volume / -u / -l / -n flags.  -u without -n uses
 * clamp(recovery_count, 1, 15) volumes; -l wraps the scheme in Limited with
 * max(largest_source_length / slice_size, 1) blocks per volume, its inner
 * scheme written to *inner_out (out->inner points there).  Conflicting flags:
 * P2G_ERR_INVALID_VOLUME_SCHEME. */
typedef struct p2g_cli_volume_flags {
    uint32_t single_volume;
    uint32_t uniform;          /* -u */
    uint32_t limit_size;       /* -l */
    uint32_t has_volume_count; /* -n given */
    uint32_t volume_count;
} p2g_cli_volume_flags;
p2g_status p2g_build_volume_scheme(const p2g_cli_volume_flags *flags, uint64_t largest_source_length,
                                   uint64_t slice_size, uint32_t recovery_count,
                                   p2g_volume_scheme *out, p2g_volume_scheme *inner_out);

/* ---- device / runtime info ------------------------------------------- */
/* Number of kernel launches this process has issued through the library
 * (monotonic); lets callers count device work inside a timed region. */
uint64_t p2g_kernel_launch_count(void);
/* 0 when a device is usable; fills a short description. */
p2g_status p2g_device_info(char *buf, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
