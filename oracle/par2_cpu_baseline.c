/*
 * par2_cpu_baseline.c -- the reference's multi-threaded CPU create path,
 * restated in C for timing on the GPU host's own cores.
 *
 * TEST / BENCHMARK INFRASTRUCTURE ONLY (bench.py's cpu_baseline leg and its
 * `--impl reference` arm).  The reference crate is Rust and cannot be built
 * in this image (no cargo, crates.io dependencies not vendored), so this is a
 * port of its fast path with the same structure:
 *   - encode: per input slice, build the R per-coefficient tables in
 *     parallel, then split the R recovery buffers into ceil(R/workers)
 *     chunks, one per worker (src/creator.rs:931-995); the inner kernel is
 *     the GFNI + AVX-512BW affine kernel (src/galois_simd/gfni.rs:314-402,
 *     picked first by detect_dispatch, src/galois_simd.rs:605-636), with the
 *     byte-table scalar kernel (src/galois_simd.rs:59-69) when the host lacks
 *     GFNI/AVX-512BW;
 *   - scan: per-slice MD5 + CRC32 in parallel joined with the whole-file MD5
 *     and 16k hash on another task (src/source.rs:156-230, rayon::join);
 *   - volumes: one task per volume file, recovery-packet MD5s serial within a
 *     volume (src/creator.rs:296-314, 1025-1042).
 * MD5 = OpenSSL (the `fast-md5` backend), CRC32 = zlib.
 */
#define _GNU_SOURCE
#include "par2_oracle.h"

#include <immintrin.h>
#include <omp.h>
#include <openssl/evp.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    uint16_t coeff;
    uint64_t mats[4];  /* ll, lh, hl, hh (GfniTables) */
    uint16_t lo[256];  /* CoeffTables (fallback kernel) */
    uint16_t hi[256];
} cb_tables;

static int cb_have_gfni512(void) {
    __builtin_cpu_init();
    return __builtin_cpu_supports("gfni") && __builtin_cpu_supports("avx512f") &&
           __builtin_cpu_supports("avx512bw");
}

/* CoeffSimdTables::new, src/galois_simd.rs:683-715 */
static void cb_build_tables(cb_tables *t, uint16_t coeff, int gfni) {
    t->coeff = coeff;
    if (coeff <= 1) return; /* Trivial */
    if (gfni) {
        or_gfni_matrices(coeff, t->mats);
    } else {
        for (uint32_t s = 0; s < 256; s++) {
            t->lo[s] = or_gf_mul(coeff, (uint16_t)s);
            t->hi[s] = or_gf_mul(coeff, (uint16_t)(s << 8));
        }
    }
}

__attribute__((target("gfni,avx512f,avx512bw"))) static void
cb_mul_xor_gfni512(const cb_tables *t, const uint8_t *in, uint8_t *out, size_t len) {
    const __m512i m_ll = _mm512_set1_epi64((long long)t->mats[0]);
    const __m512i m_lh = _mm512_set1_epi64((long long)t->mats[1]);
    const __m512i m_hl = _mm512_set1_epi64((long long)t->mats[2]);
    const __m512i m_hh = _mm512_set1_epi64((long long)t->mats[3]);
    const __m512i deint = _mm512_broadcast_i32x4(
        _mm_setr_epi8(0, 2, 4, 6, 8, 10, 12, 14, 1, 3, 5, 7, 9, 11, 13, 15));
    const __m512i inter = _mm512_broadcast_i32x4(
        _mm_setr_epi8(0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15));
    const __m512i p_lo = _mm512_setr_epi64(0, 2, 4, 6, 8, 10, 12, 14);
    const __m512i p_hi = _mm512_setr_epi64(1, 3, 5, 7, 9, 11, 13, 15);
    const __m512i p_i0 = _mm512_setr_epi64(0, 8, 1, 9, 2, 10, 3, 11);
    const __m512i p_i1 = _mm512_setr_epi64(4, 12, 5, 13, 6, 14, 7, 15);
    size_t chunks = len / 128;
    for (size_t c = 0; c < chunks; c++) {
        const uint8_t *ip = in + c * 128;
        uint8_t *op = out + c * 128;
        __m512i d0 = _mm512_shuffle_epi8(_mm512_loadu_si512(ip), deint);
        __m512i d1 = _mm512_shuffle_epi8(_mm512_loadu_si512(ip + 64), deint);
        __m512i lows = _mm512_permutex2var_epi64(d0, p_lo, d1);
        __m512i highs = _mm512_permutex2var_epi64(d0, p_hi, d1);
        __m512i olo = _mm512_xor_si512(_mm512_gf2p8affine_epi64_epi8(lows, m_ll, 0),
                                       _mm512_gf2p8affine_epi64_epi8(highs, m_lh, 0));
        __m512i ohi = _mm512_xor_si512(_mm512_gf2p8affine_epi64_epi8(lows, m_hl, 0),
                                       _mm512_gf2p8affine_epi64_epi8(highs, m_hh, 0));
        __m512i r0 = _mm512_shuffle_epi8(_mm512_permutex2var_epi64(olo, p_i0, ohi), inter);
        __m512i r1 = _mm512_shuffle_epi8(_mm512_permutex2var_epi64(olo, p_i1, ohi), inter);
        _mm512_storeu_si512(op, _mm512_xor_si512(_mm512_loadu_si512(op), r0));
        _mm512_storeu_si512(op + 64, _mm512_xor_si512(_mm512_loadu_si512(op + 64), r1));
    }
    for (size_t off = chunks * 128; off + 2 <= len; off += 2) {
        uint8_t lo, hi;
        or_gfni_apply(t->mats, in[off], in[off + 1], &lo, &hi);
        out[off] ^= lo;
        out[off + 1] ^= hi;
    }
}

/* gf_mul_xor_with_tables, src/galois_simd.rs:720-766 */
static void cb_mul_xor(const cb_tables *t, const uint8_t *in, uint8_t *out, size_t len, int gfni) {
    if (t->coeff == 0) return;
    if (t->coeff == 1) {
        for (size_t i = 0; i < len; i++) out[i] ^= in[i];
        return;
    }
    if (gfni) {
        cb_mul_xor_gfni512(t, in, out, len);
        return;
    }
    for (size_t k = 0; k < len / 2; k++) {
        uint16_t p = t->lo[in[2 * k]] ^ t->hi[in[2 * k + 1]];
        out[2 * k] ^= (uint8_t)p;
        out[2 * k + 1] ^= (uint8_t)(p >> 8);
    }
}

int cb_kernel_is_gfni512(void) { return cb_have_gfni512(); }

/* encode_all_recovery_blocks' hot loop (src/creator.rs:931-1007) over the
 * input slices [s_begin, s_end); `src` points at slice s_begin and the
 * slices follow back to back.  `out` is XORed into (zero it for a fresh
 * encode). */
void cb_encode(const uint8_t *src, uint32_t s_begin, uint32_t s_end, uint64_t slice_size,
               uint32_t R, uint8_t *out, int threads) {
    int gfni = cb_have_gfni512();
    if (threads <= 0) threads = omp_get_max_threads();
    uint16_t *bases = (uint16_t *)malloc(sizeof(uint16_t) * (s_end ? s_end : 1));
    or_input_bases(s_end, bases);
    cb_tables *tabs = (cb_tables *)malloc(sizeof(cb_tables) * (R ? R : 1));
    uint32_t chunk = (R + (uint32_t)threads - 1) / (uint32_t)threads;
    if (chunk == 0) chunk = 1;
    uint32_t nchunks = (R + chunk - 1) / chunk;
#pragma omp parallel num_threads(threads)
    {
        for (uint32_t s = s_begin; s < s_end; s++) {
#pragma omp for schedule(static)
            for (uint32_t r = 0; r < R; r++) cb_build_tables(&tabs[r], or_gf_pow(bases[s], r), gfni);
            const uint8_t *in = src + (size_t)(s - s_begin) * slice_size;
#pragma omp for schedule(static)
            for (uint32_t c = 0; c < nchunks; c++) {
                uint32_t r1 = (c + 1) * chunk < R ? (c + 1) * chunk : R;
                for (uint32_t r = c * chunk; r < r1; r++)
                    cb_mul_xor(&tabs[r], in, out + (size_t)r * slice_size, slice_size, gfni);
            }
        }
    }
    free(tabs);
    free(bases);
}

/* Selected recovery rows only: out row k = XOR_s gf_pow(base_s, exps[k]) *
 * slice s over the S slices at src (back to back), i.e. row exps[k] of
 * encode_all_recovery_blocks (src/creator.rs:931-1007) -- for spot checks of
 * jobs whose full encode is too long for the CPU.  Rows run in parallel. */
void cb_encode_rows(const uint8_t *src, uint32_t S, uint64_t slice_size, const uint32_t *exps, uint32_t n,
                    uint8_t *out, int threads) {
    int gfni = cb_have_gfni512();
    if (threads <= 0) threads = omp_get_max_threads();
    uint16_t *bases = (uint16_t *)malloc(sizeof(uint16_t) * (S ? S : 1));
    or_input_bases(S, bases);
    memset(out, 0, (size_t)n * slice_size);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (uint32_t k = 0; k < n; k++) {
        cb_tables t;
        for (uint32_t s = 0; s < S; s++) {
            cb_build_tables(&t, or_gf_pow(bases[s], exps[k]), gfni);
            cb_mul_xor(&t, src + (size_t)s * slice_size, out + (size_t)k * slice_size, slice_size, gfni);
        }
    }
    free(bases);
}

static void cb_md5(const uint8_t *d, size_t n, uint8_t out[16]) {
    unsigned int l = 16;
    EVP_Digest(d, n, out, &l, EVP_md5(), NULL);
}

/* scan_via_mmap, src/source.rs:145-232: per-slice hashes on the pool joined
 * with the whole-file hashes on one task.  whole_file 0 leaves out the
 * whole-file MD5 (hash_full is then zero): the work a device job does when
 * that hash is placed on the host. */
static void cb_scan_ex(const uint8_t *data, uint64_t len, uint64_t slice_size, or_slice_checksum *cks,
                       uint8_t hash_full[16], uint8_t hash16k[16], int threads, int whole_file) {
    if (threads <= 0) threads = omp_get_max_threads();
    uint64_t n = (len + slice_size - 1) / slice_size;
#pragma omp parallel num_threads(threads)
#pragma omp single
    {
#pragma omp task
        {
            if (whole_file)
                cb_md5(data, len, hash_full);
            else
                memset(hash_full, 0, 16);
            cb_md5(data, len < 16384 ? len : 16384, hash16k);
        }
#pragma omp taskloop grainsize(1)
        for (uint64_t i = 0; i < n; i++) {
            uint64_t st = i * slice_size, en = st + slice_size < len ? st + slice_size : len;
            if (en - st == slice_size) {
                cb_md5(data + st, slice_size, cks[i].md5);
                cks[i].crc32 = or_crc32(data + st, slice_size);
            } else {
                uint8_t *pad = (uint8_t *)calloc(slice_size, 1);
                memcpy(pad, data + st, en - st);
                cb_md5(pad, slice_size, cks[i].md5);
                cks[i].crc32 = or_crc32(pad, slice_size);
                free(pad);
            }
        }
#pragma omp taskwait
    }
}

void cb_scan(const uint8_t *data, uint64_t len, uint64_t slice_size, or_slice_checksum *cks,
             uint8_t hash_full[16], uint8_t hash16k[16], int threads) {
    cb_scan_ex(data, len, slice_size, cks, hash_full, hash16k, threads, 1);
}

/* Recovery packet MD5s, one task per volume, serial inside a volume
 * (src/creator.rs:296-314 with build_volume_packet :1025-1042). */
void cb_recovery_packet_md5(const uint8_t set_id[16], const uint8_t *rec, uint32_t R,
                            uint64_t slice_size, const uint32_t *vol_sizes, uint32_t n_vol,
                            uint8_t *out_md5, int threads) {
    if (threads <= 0) threads = omp_get_max_threads();
    uint32_t *first = (uint32_t *)malloc(sizeof(uint32_t) * (n_vol ? n_vol : 1));
    uint32_t acc = 0;
    for (uint32_t v = 0; v < n_vol; v++) {
        first[v] = acc;
        acc += vol_sizes[v];
    }
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (uint32_t v = 0; v < n_vol; v++) {
        EVP_MD_CTX *ctx = EVP_MD_CTX_new();
        for (uint32_t k = 0; k < vol_sizes[v]; k++) {
            uint32_t e = first[v] + k;
            if (e >= R) break;
            uint8_t head[36];
            memcpy(head, set_id, 16);
            memcpy(head + 16, "PAR 2.0\0RecvSlic", 16);
            head[32] = (uint8_t)e;
            head[33] = (uint8_t)(e >> 8);
            head[34] = 0;
            head[35] = 0;
            unsigned int l = 16;
            EVP_DigestInit_ex(ctx, EVP_md5(), NULL);
            EVP_DigestUpdate(ctx, head, 36);
            EVP_DigestUpdate(ctx, rec + (size_t)e * slice_size, slice_size);
            EVP_DigestFinal_ex(ctx, out_md5 + 16 * (size_t)e, &l);
        }
        EVP_MD_CTX_free(ctx);
    }
    free(first);
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* One create over a single in-memory file: scan (with file hashes), encode
 * all R rows, and the recovery-packet MD5s of an exponential volume split.
 * This is the compute of `par2rust create -s slice -c R` minus file I/O.
 * Returns seconds; `rec_out` (R*slice bytes, may be NULL) receives recovery. */
double cb_create_timed_ex(const uint8_t *data, uint64_t len, uint64_t slice_size, uint32_t R,
                          int threads, uint8_t *rec_out, double *t_scan, double *t_encode,
                          double *t_pkt, int whole_file) {
    if (threads <= 0) threads = omp_get_max_threads();
    uint64_t S = (len + slice_size - 1) / slice_size;
    or_slice_checksum *cks = (or_slice_checksum *)calloc(S, sizeof *cks);
    uint8_t hf[16], h16[16], fid[16], set_id[16];
    double t0 = now_s();
    cb_scan_ex(data, len, slice_size, cks, hf, h16, threads, whole_file);
    or_file_id(h16, len, (const uint8_t *)"source.bin", 10, fid);
    uint8_t mp[128];
    or_build_main_packet(slice_size, fid, 1, set_id, mp);
    double t1 = now_s();
    /* SourceReader zero-pads the tail slice: pad it into a copy of the last slice only */
    uint8_t *rec = rec_out ? rec_out : (uint8_t *)malloc((size_t)R * slice_size);
    memset(rec, 0, (size_t)R * slice_size);
    uint64_t full = len / slice_size;
    if (full) cb_encode(data, 0, (uint32_t)full, slice_size, R, rec, threads);
    if (full < S) {
        uint8_t *tail = (uint8_t *)calloc(slice_size, 1);
        memcpy(tail, data + full * slice_size, len - full * slice_size);
        cb_encode(tail, (uint32_t)full, (uint32_t)S, slice_size, R, rec, threads);
        free(tail);
    }
    double t2 = now_s();
    or_scheme ex = {OR_SCHEME_EXPONENTIAL, 0, 0, NULL, NULL, 0};
    uint32_t vs[64];
    int64_t nv = R ? or_resolve_volume_sizes(&ex, R, vs, 64) : 0;
    uint8_t *pm = (uint8_t *)malloc(16 * (size_t)(R ? R : 1));
    if (nv > 0) cb_recovery_packet_md5(set_id, rec, R, slice_size, vs, (uint32_t)nv, pm, threads);
    double t3 = now_s();
    free(pm);
    if (!rec_out) free(rec);
    free(cks);
    if (t_scan) *t_scan = t1 - t0;
    if (t_encode) *t_encode = t2 - t1;
    if (t_pkt) *t_pkt = t3 - t2;
    return t3 - t0;
}

double cb_create_timed(const uint8_t *data, uint64_t len, uint64_t slice_size, uint32_t R,
                       int threads, uint8_t *rec_out, double *t_scan, double *t_encode,
                       double *t_pkt) {
    return cb_create_timed_ex(data, len, slice_size, R, threads, rec_out, t_scan, t_encode, t_pkt, 1);
}

int cb_max_threads(void) { return omp_get_max_threads(); }
