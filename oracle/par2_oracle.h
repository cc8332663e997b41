/*
 * par2_oracle.h -- CPU restatement of the par2rust create path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm load it
 * to compute the expected bytes on the CPU.  Nothing in the par2rust_b200
 * product links, loads or calls it.
 *
 * Every function restates a function of the reference crate (javi11/par2rust
 * v0.1.0); the citation on each declaration is the reference file:line it
 * follows.  MD5 is OpenSSL's (the reference's `fast-md5` backend,
 * src/md5_impl.rs:50-88) and CRC-32 is zlib's crc32(), the same CRC-32/IEEE
 * (reflected 0xEDB88320, init/xorout 0xFFFFFFFF) that crc32fast 1.5.0
 * computes at src/source.rs:172,181,275.
 */
#ifndef PAR2_ORACLE_H
#define PAR2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GF(2^16), src/galois.rs ------------------------------------------ */
/* build_tables, src/galois.rs:33-53 (copies the 65536-entry tables out) */
void or_gf_tables(uint16_t *log_out, uint16_t *antilog_out);
uint16_t or_gf_mul(uint16_t a, uint16_t b);          /* src/galois.rs:57-69 */
uint16_t or_gf_pow(uint16_t base, uint32_t exp);     /* src/galois.rs:74-87 */
uint16_t or_gf_inv(uint16_t a);                      /* src/galois.rs:91-99 */

/* ---- Reed-Solomon, src/reedsolomon.rs --------------------------------- */
/* generate_input_bases, src/reedsolomon.rs:130-149 */
int or_input_bases(uint32_t count, uint16_t *out);
/* RsEncoder::coefficient, src/reedsolomon.rs:56-60 (first_exponent 0) */
uint16_t or_coefficient(uint32_t recovery_idx, uint32_t input_idx);
/* gf_mul_xor_scalar, src/reedsolomon.rs:87-126 */
void or_gf_mul_xor_scalar(uint16_t coeff, const uint8_t *in, uint8_t *out, size_t len);
/* gf_mul_xor_table_scalar + CoeffTables::new, src/galois_simd.rs:45-69 */
void or_gf_mul_xor_table(uint16_t coeff, const uint8_t *in, uint8_t *out, size_t len);
/* GfniTables::from_coeff + apply_scalar, src/galois_simd/gfni.rs:78-141 */
void or_gfni_matrices(uint16_t coeff, uint64_t mats[4]);
void or_gfni_apply(const uint64_t mats[4], uint8_t lo, uint8_t hi, uint8_t *out_lo, uint8_t *out_hi);
/* encode_all_recovery_blocks' single pass, src/creator.rs:883-1018:
 * src holds `S` zero-padded slices back to back (slice i at i*slice_size),
 * out receives R slices (recovery i = exponent i), zeroed first. */
void or_encode(const uint8_t *src, uint32_t S, uint64_t slice_size, uint32_t R, uint8_t *out);
/* or_create encodes with cb_encode (the multi-threaded port) when on != 0. */
void or_set_fast_encode(int on);
void cb_encode(const uint8_t *src, uint32_t s_begin, uint32_t s_end, uint64_t slice_size, uint32_t R, uint8_t *out,
               int threads);

/* ---- hashes ------------------------------------------------------------ */
void or_md5(const uint8_t *data, size_t len, uint8_t out[16]);  /* md5_impl::digest */
uint32_t or_crc32(const uint8_t *data, size_t len);             /* crc32fast::hash */

/* ---- scan, src/source.rs ------------------------------------------------ */
typedef struct {
    uint8_t md5[16];
    uint32_t crc32;
} or_slice_checksum; /* SliceChecksum, src/source.rs:28-31 (IFSC entry layout) */

/* scan_via_mmap semantics over an in-memory file, src/source.rs:145-232:
 * per-slice MD5+CRC32 of the zero-padded slice, hash_full over the real
 * bytes, hash16k over the first min(len,16384) bytes; then compute_file_id,
 * src/source.rs:303-309.  `checksums` must hold ceil(len/slice) entries.
 * Returns 0, or a negative or_status code for the validation errors of
 * src/source.rs:65-75. */
int or_scan(const uint8_t *data, uint64_t len, uint64_t slice_size,
            const uint8_t *name, size_t name_len,
            or_slice_checksum *checksums, uint8_t hash_full[16],
            uint8_t hash16k[16], uint8_t file_id[16]);
/* compute_file_id, src/source.rs:303-309 */
void or_file_id(const uint8_t hash16k[16], uint64_t length, const uint8_t *name,
                size_t name_len, uint8_t out[16]);

/* ---- packets, src/format.rs + src/packet/ files ------------------------- */
/* Every builder writes into `out` (if non-NULL) and returns the byte count. */
size_t or_build_packet(const uint8_t set_id[16], const uint8_t type[16],
                       const uint8_t *body, size_t body_len, uint8_t *out); /* format.rs:33-54 */
size_t or_build_main_packet(uint64_t slice_size, const uint8_t *file_ids, uint32_t n,
                            uint8_t set_id_out[16], uint8_t *out); /* main_packet.rs:25-42 */
size_t or_build_file_desc_packet(const uint8_t set_id[16], const uint8_t file_id[16],
                                 const uint8_t hash_full[16], const uint8_t hash16k[16],
                                 uint64_t length, const uint8_t *name, size_t name_len,
                                 uint8_t *out); /* file_desc.rs:17-28 */
size_t or_build_file_verify_packet(const uint8_t set_id[16], const uint8_t file_id[16],
                                   const or_slice_checksum *cks, uint64_t n,
                                   uint8_t *out); /* file_verify.rs:12-23 */
size_t or_build_creator_packet(const uint8_t set_id[16], uint8_t *out); /* creator.rs:8-14 */
/* comment.rs:15-81; `comment` is UTF-8 */
size_t or_build_comment_packets(const uint8_t set_id[16], const char *comment, uint8_t *out);
size_t or_build_recovery_packet(const uint8_t set_id[16], uint16_t exponent,
                                const uint8_t *slice, uint64_t slice_size,
                                uint8_t *out); /* recovery.rs:11-19 */

/* ---- volumes, src/creator.rs ------------------------------------------ */
enum { OR_SCHEME_SINGLE = 0, OR_SCHEME_EXPONENTIAL = 1, OR_SCHEME_UNIFORM = 2,
       OR_SCHEME_LIMITED = 3, OR_SCHEME_EXPLICIT = 4 };
typedef struct or_scheme {
    int kind;
    uint32_t count;                 /* Uniform{count} */
    uint32_t max_blocks_per_volume; /* Limited */
    const struct or_scheme *inner;  /* Limited */
    const uint32_t *sizes;          /* Explicit */
    uint32_t n_sizes;
} or_scheme;
/* resolve_volume_sizes, src/creator.rs:325-431.  Returns the volume count
 * (written to `out` when non-NULL, capacity `cap`), or -1 on
 * InvalidVolumeScheme. */
int64_t or_resolve_volume_sizes(const or_scheme *scheme, uint32_t total, uint32_t *out, uint32_t cap);
/* derive_volume_filename, src/creator.rs:1046-1057 (returns strlen) */
size_t or_volume_filename(const char *index_path, uint16_t first_exp, uint32_t count, char *out, size_t cap);

/* ---- whole create, src/creator.rs:188-321 ----------------------------- */
enum { OR_OK = 0, OR_ERR_INVALID_SLICE_SIZE = -2, OR_ERR_INVALID_FILE_NAME = -3,
       OR_ERR_NO_INPUT_FILES = -4, OR_ERR_EMPTY_FILE = -5, OR_ERR_TOO_MANY_FILES = -6,
       OR_ERR_TOO_MANY_RECOVERY_BLOCKS = -7, OR_ERR_TOO_MANY_INPUT_BLOCKS = -8,
       OR_ERR_INVALID_VOLUME_SCHEME = -9, OR_ERR_NOMEM = -10 };
typedef struct {
    const uint8_t *data;
    uint64_t len;
    const uint8_t *name;
    size_t name_len;
} or_input;
/* Scans every input (SourceFile::scan) and runs run_create_with_progress's
 * byte production without touching the filesystem.  `out_blob` receives the
 * concatenation of every output file (index first, then volumes in exponent
 * order); `out_sizes[i]` the length of file i; `out_names` the file names
 * (each NUL-terminated, concatenated).  The caller frees the three buffers
 * with free().  Returns the number of files or a negative OR_ERR_* code. */
int64_t or_create(const or_input *inputs, uint32_t n, uint64_t slice_size, uint32_t R,
                  const or_scheme *scheme, const char *const *comments, uint32_t n_comments,
                  const char *index_path, uint8_t **out_blob, uint64_t **out_sizes,
                  char **out_names);

#ifdef __cplusplus
}
#endif
#endif
