/*
 * par2_oracle.c -- CPU restatement of the par2rust create path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke()
 * and bench.py's CPU legs.  The par2rust_b200 product never links it.
 * Each function cites the reference (javi11/par2rust v0.1.0) file:line that
 * it restates.  Plain scalar C on purpose: this file is the readable
 * statement of the algorithm, not a fast path (the fast CPU baseline lives
 * in par2_cpu_baseline.c).
 */
#define _GNU_SOURCE
#include "par2_oracle.h"

#include <openssl/evp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

/* src/galois.rs:15-18 */
#define FIELD_COUNT 65536u
#define FIELD_LIMIT 65535u
#define FIELD_GENERATOR 0x1100Bu
/* src/source.rs:17 */
#define HASH16K_LEN 16384u
/* src/creator.rs:102-108 */
#define MAX_FILES 32768u
#define MAX_INPUT_BLOCKS 32768u
#define MAX_RECOVERY_BLOCKS 65535u

static uint16_t g_log[FIELD_COUNT];
static uint16_t g_antilog[FIELD_COUNT];
static int g_tables_ready = 0;

/* build_tables, src/galois.rs:33-53 */
static void build_tables(void) {
    if (g_tables_ready) return;
    uint32_t b = 1;
    for (uint32_t l = 0; l < FIELD_LIMIT; l++) {
        g_log[b] = (uint16_t)l;
        g_antilog[l] = (uint16_t)b;
        b <<= 1;
        if (b & FIELD_COUNT) b ^= FIELD_GENERATOR;
    }
    g_log[0] = (uint16_t)FIELD_LIMIT;
    g_antilog[FIELD_LIMIT] = 0;
    g_tables_ready = 1;
}

void or_gf_tables(uint16_t *log_out, uint16_t *antilog_out) {
    build_tables();
    if (log_out) memcpy(log_out, g_log, sizeof g_log);
    if (antilog_out) memcpy(antilog_out, g_antilog, sizeof g_antilog);
}

/* gf_mul, src/galois.rs:57-69 */
uint16_t or_gf_mul(uint16_t a, uint16_t b) {
    if (a == 0 || b == 0) return 0;
    build_tables();
    uint32_t sum = (uint32_t)g_log[a] + g_log[b];
    uint32_t idx = sum >= FIELD_LIMIT ? sum - FIELD_LIMIT : sum;
    return g_antilog[idx];
}

/* gf_pow, src/galois.rs:74-87 */
uint16_t or_gf_pow(uint16_t base, uint32_t exp) {
    if (exp == 0) return 1;
    if (base == 0) return 0;
    build_tables();
    uint64_t prod = (uint64_t)g_log[base] * exp;
    return g_antilog[(uint32_t)(prod % FIELD_LIMIT)];
}

/* gf_inv, src/galois.rs:91-99 (returns 0 for a == 0 instead of panicking) */
uint16_t or_gf_inv(uint16_t a) {
    if (a == 0) return 0;
    build_tables();
    uint32_t log_inv = (FIELD_LIMIT - g_log[a]) % FIELD_LIMIT;
    return g_antilog[log_inv];
}

/* gcd, src/reedsolomon.rs:151-157 */
static uint32_t gcd_u32(uint32_t a, uint32_t b) {
    while (b) {
        uint32_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

/* generate_input_bases, src/reedsolomon.rs:130-149 */
int or_input_bases(uint32_t count, uint16_t *out) {
    build_tables();
    uint32_t n = 0, logbase = 0;
    while (n < count) {
        if (logbase >= FIELD_LIMIT) return -1; /* the reference panics here */
        if (gcd_u32(FIELD_LIMIT, logbase) == 1) out[n++] = g_antilog[logbase];
        logbase++;
    }
    return 0;
}

static uint16_t *g_bases = NULL;
static uint32_t g_bases_n = 0;

static const uint16_t *bases_upto(uint32_t count) {
    if (count > g_bases_n) {
        uint16_t *nb = (uint16_t *)realloc(g_bases, (size_t)count * sizeof(uint16_t));
        if (!nb) return NULL;
        g_bases = nb;
        or_input_bases(count, g_bases);
        g_bases_n = count;
    }
    return g_bases;
}

/* RsEncoder::coefficient, src/reedsolomon.rs:56-60; exponent r = recovery_idx
 * because encode_all_recovery_blocks uses first_exponent 0 (creator.rs:915). */
uint16_t or_coefficient(uint32_t recovery_idx, uint32_t input_idx) {
    const uint16_t *b = bases_upto(input_idx + 1);
    return or_gf_pow(b[input_idx], recovery_idx);
}

/* gf_mul_xor_scalar, src/reedsolomon.rs:87-126 */
void or_gf_mul_xor_scalar(uint16_t coeff, const uint8_t *in, uint8_t *out, size_t len) {
    if (coeff == 0) return;
    if (coeff == 1) {
        for (size_t i = 0; i < len; i++) out[i] ^= in[i];
        return;
    }
    build_tables();
    uint32_t log_coeff = g_log[coeff];
    for (size_t k = 0; k < len / 2; k++) {
        uint32_t sym = (uint32_t)in[2 * k] | ((uint32_t)in[2 * k + 1] << 8);
        uint32_t product = 0;
        if (sym != 0) {
            uint32_t sum = log_coeff + g_log[sym];
            uint32_t idx = sum >= FIELD_LIMIT ? sum - FIELD_LIMIT : sum;
            product = g_antilog[idx];
        }
        out[2 * k] ^= (uint8_t)product;
        out[2 * k + 1] ^= (uint8_t)(product >> 8);
    }
}

/* CoeffTables::new + gf_mul_xor_table_scalar, src/galois_simd.rs:45-69 */
void or_gf_mul_xor_table(uint16_t coeff, const uint8_t *in, uint8_t *out, size_t len) {
    uint16_t lo[256], hi[256];
    for (uint32_t s = 0; s < 256; s++) {
        lo[s] = or_gf_mul(coeff, (uint16_t)s);
        hi[s] = or_gf_mul(coeff, (uint16_t)(s << 8));
    }
    for (size_t k = 0; k < len / 2; k++) {
        uint16_t prod = lo[in[2 * k]] ^ hi[in[2 * k + 1]];
        out[2 * k] ^= (uint8_t)prod;
        out[2 * k + 1] ^= (uint8_t)(prod >> 8);
    }
}

/* GfniTables::from_coeff, src/galois_simd/gfni.rs:78-118.  mats = ll, lh, hl, hh. */
void or_gfni_matrices(uint16_t coeff, uint64_t mats[4]) {
    uint16_t cols[16];
    for (uint32_t j = 0; j < 16; j++) cols[j] = or_gf_mul(coeff, (uint16_t)(1u << j));
    const uint32_t bases[4][2] = {{0, 0}, {0, 8}, {8, 0}, {8, 8}}; /* (out, in) bit bases */
    for (int m = 0; m < 4; m++) {
        uint64_t acc = 0;
        for (uint32_t i = 0; i < 8; i++) {
            uint8_t row = 0;
            for (uint32_t ip = 0; ip < 8; ip++) {
                uint32_t bit = (cols[bases[m][1] + ip] >> (bases[m][0] + i)) & 1u;
                row |= (uint8_t)(bit << ip);
            }
            acc |= (uint64_t)row << ((7 - i) * 8);
        }
        mats[m] = acc;
    }
}

/* affine_apply, src/galois_simd/gfni.rs:133-141 */
static uint8_t affine_apply(uint64_t mat, uint8_t x) {
    uint8_t y = 0;
    for (uint32_t i = 0; i < 8; i++) {
        uint8_t row = (uint8_t)(mat >> ((7 - i) * 8));
        y |= (uint8_t)((__builtin_popcount(row & x) & 1) << i);
    }
    return y;
}

/* GfniTables::apply_scalar, src/galois_simd/gfni.rs:124-128 */
void or_gfni_apply(const uint64_t mats[4], uint8_t lo, uint8_t hi, uint8_t *out_lo, uint8_t *out_hi) {
    *out_lo = affine_apply(mats[0], lo) ^ affine_apply(mats[1], hi);
    *out_hi = affine_apply(mats[2], lo) ^ affine_apply(mats[3], hi);
}

/* The single-pass loop of encode_all_recovery_blocks, src/creator.rs:883-1018:
 * recovery buffers start zeroed (:921-923); for every input slice in global
 * order, every recovery row r accumulates coefficient(r, input)·slice. */
void or_encode(const uint8_t *src, uint32_t S, uint64_t slice_size, uint32_t R, uint8_t *out) {
    memset(out, 0, (size_t)R * slice_size);
    bases_upto(S ? S : 1);
    for (uint32_t s = 0; s < S; s++) {
        const uint8_t *in = src + (size_t)s * slice_size;
        for (uint32_t r = 0; r < R; r++) {
            uint16_t c = or_gf_pow(g_bases[s], r);
            or_gf_mul_xor_scalar(c, in, out + (size_t)r * slice_size, slice_size);
        }
    }
}

/* md5_impl::digest, src/md5_impl.rs:84-88 (OpenSSL backend) */
void or_md5(const uint8_t *data, size_t len, uint8_t out[16]) {
    unsigned int n = 16;
    EVP_Digest(data, len, out, &n, EVP_md5(), NULL);
}

/* crc32fast::hash (CRC-32/IEEE), src/source.rs:172 */
uint32_t or_crc32(const uint8_t *data, size_t len) {
    uLong c = crc32(0L, Z_NULL, 0);
    while (len > 0) {
        uInt chunk = len > 0x40000000u ? 0x40000000u : (uInt)len;
        c = crc32(c, data, chunk);
        data += chunk;
        len -= chunk;
    }
    return (uint32_t)c;
}

static void put_le64(uint8_t *p, uint64_t v) {
    for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (8 * i));
}
static void put_le32(uint8_t *p, uint32_t v) {
    for (int i = 0; i < 4; i++) p[i] = (uint8_t)(v >> (8 * i));
}

/* compute_file_id, src/source.rs:303-309 */
void or_file_id(const uint8_t hash16k[16], uint64_t length, const uint8_t *name, size_t name_len,
                uint8_t out[16]) {
    uint8_t *buf = (uint8_t *)malloc(24 + name_len);
    memcpy(buf, hash16k, 16);
    put_le64(buf + 16, length);
    if (name_len) memcpy(buf + 24, name, name_len);
    or_md5(buf, 24 + name_len, out);
    free(buf);
}

/* SourceFile::scan_with_progress validation (src/source.rs:65-75) and
 * scan_via_mmap (src/source.rs:145-232), then compute_file_id. */
int or_scan(const uint8_t *data, uint64_t len, uint64_t slice_size, const uint8_t *name,
            size_t name_len, or_slice_checksum *checksums, uint8_t hash_full[16],
            uint8_t hash16k[16], uint8_t file_id[16]) {
    if (name_len == 0 || memchr(name, 0, name_len)) return OR_ERR_INVALID_FILE_NAME;
    if (slice_size == 0 || slice_size % 4 != 0) return OR_ERR_INVALID_SLICE_SIZE;
    if (len == 0) return OR_ERR_EMPTY_FILE;
    uint64_t n_slices = (len + slice_size - 1) / slice_size;
    uint8_t *pad = NULL;
    for (uint64_t i = 0; i < n_slices; i++) {
        uint64_t start = i * slice_size;
        uint64_t end = start + slice_size < len ? start + slice_size : len;
        if (end - start == slice_size) {
            or_md5(data + start, slice_size, checksums[i].md5);
            checksums[i].crc32 = or_crc32(data + start, slice_size);
        } else { /* trailing partial slice is zero-padded, src/source.rs:176-183 */
            if (!pad) pad = (uint8_t *)calloc(slice_size, 1);
            memset(pad, 0, slice_size);
            memcpy(pad, data + start, end - start);
            or_md5(pad, slice_size, checksums[i].md5);
            checksums[i].crc32 = or_crc32(pad, slice_size);
        }
    }
    free(pad);
    or_md5(data, len, hash_full);                                  /* :224 */
    or_md5(data, len < HASH16K_LEN ? len : HASH16K_LEN, hash16k);  /* :225-226 */
    or_file_id(hash16k, len, name, name_len, file_id);
    return 0;
}

/* ---- packets ----------------------------------------------------------- */
/* src/format.rs:3-15 */
static const uint8_t PACKET_MAGIC[8] = {'P', 'A', 'R', '2', 0, 'P', 'K', 'T'};
static const uint8_t TYPE_FILE_DESC[16] = "PAR 2.0\0FileDesc";
static const uint8_t TYPE_FILE_VERIFY[16] = "PAR 2.0\0IFSC\0\0\0\0";
static const uint8_t TYPE_MAIN[16] = "PAR 2.0\0Main\0\0\0\0";
static const uint8_t TYPE_RECOVERY[16] = "PAR 2.0\0RecvSlic";
static const uint8_t TYPE_CREATOR[16] = "PAR 2.0\0Creator\0";
static const uint8_t TYPE_COMMENT_ASCII[16] = "PAR 2.0\0CommASCI";
static const uint8_t TYPE_COMMENT_UNICODE[16] = "PAR 2.0\0CommUni\0";
/* src/packet/creator.rs:3 */
static const char CREATOR_STRING[] = "Created by par2rust v0.1.0";

static size_t round_up_4(size_t n) { return (n + 3) & ~(size_t)3; } /* format.rs:23-25 */

/* build_packet, src/format.rs:33-54 */
size_t or_build_packet(const uint8_t set_id[16], const uint8_t type[16], const uint8_t *body,
                       size_t body_len, uint8_t *out) {
    size_t packet_len = 64 + body_len;
    if (!out) return packet_len;
    uint8_t *hin = (uint8_t *)malloc(32 + body_len);
    memcpy(hin, set_id, 16);
    memcpy(hin + 16, type, 16);
    if (body_len) memcpy(hin + 32, body, body_len);
    uint8_t h[16];
    or_md5(hin, 32 + body_len, h);
    free(hin);
    memcpy(out, PACKET_MAGIC, 8);
    put_le64(out + 8, packet_len);
    memcpy(out + 16, h, 16);
    memcpy(out + 32, set_id, 16);
    memcpy(out + 48, type, 16);
    if (body_len) memcpy(out + 64, body, body_len);
    return packet_len;
}

static int cmp16(const void *a, const void *b) { return memcmp(a, b, 16); }

/* build_main_packet, src/packet/main_packet.rs:25-42 */
size_t or_build_main_packet(uint64_t slice_size, const uint8_t *file_ids, uint32_t n,
                            uint8_t set_id_out[16], uint8_t *out) {
    size_t body_len = 12 + 16 * (size_t)n;
    uint8_t *body = (uint8_t *)malloc(body_len);
    put_le64(body, slice_size);
    put_le32(body + 8, n);
    if (n) memcpy(body + 12, file_ids, 16 * (size_t)n);
    qsort(body + 12, n, 16, cmp16);
    uint8_t set_id[16];
    or_md5(body, body_len, set_id);
    if (set_id_out) memcpy(set_id_out, set_id, 16);
    size_t r = or_build_packet(set_id, TYPE_MAIN, body, body_len, out);
    free(body);
    return r;
}

/* build_file_desc_packet, src/packet/file_desc.rs:17-28 */
size_t or_build_file_desc_packet(const uint8_t set_id[16], const uint8_t file_id[16],
                                 const uint8_t hash_full[16], const uint8_t hash16k[16],
                                 uint64_t length, const uint8_t *name, size_t name_len,
                                 uint8_t *out) {
    size_t body_len = 56 + round_up_4(name_len);
    if (!out) return 64 + body_len;
    uint8_t *body = (uint8_t *)calloc(body_len, 1);
    memcpy(body, file_id, 16);
    memcpy(body + 16, hash_full, 16);
    memcpy(body + 32, hash16k, 16);
    put_le64(body + 48, length);
    if (name_len) memcpy(body + 56, name, name_len);
    size_t r = or_build_packet(set_id, TYPE_FILE_DESC, body, body_len, out);
    free(body);
    return r;
}

/* build_file_verify_packet, src/packet/file_verify.rs:12-23 */
size_t or_build_file_verify_packet(const uint8_t set_id[16], const uint8_t file_id[16],
                                   const or_slice_checksum *cks, uint64_t n, uint8_t *out) {
    size_t body_len = 16 + 20 * (size_t)n;
    if (!out) return 64 + body_len;
    uint8_t *body = (uint8_t *)malloc(body_len);
    memcpy(body, file_id, 16);
    for (uint64_t i = 0; i < n; i++) {
        memcpy(body + 16 + 20 * i, cks[i].md5, 16);
        put_le32(body + 16 + 20 * i + 16, cks[i].crc32);
    }
    size_t r = or_build_packet(set_id, TYPE_FILE_VERIFY, body, body_len, out);
    free(body);
    return r;
}

/* build_creator_packet, src/packet/creator.rs:8-14 */
size_t or_build_creator_packet(const uint8_t set_id[16], uint8_t *out) {
    size_t n = strlen(CREATOR_STRING);
    size_t body_len = round_up_4(n);
    uint8_t body[64] = {0};
    memcpy(body, CREATOR_STRING, n);
    return or_build_packet(set_id, TYPE_CREATOR, body, body_len, out);
}

/* Decode UTF-8 into code points (the input is a Rust String, so valid UTF-8). */
static size_t utf8_decode(const char *s, uint32_t *cps) {
    size_t n = 0;
    const unsigned char *p = (const unsigned char *)s;
    while (*p) {
        uint32_t c;
        if (*p < 0x80) {
            c = *p++;
        } else if ((*p & 0xE0) == 0xC0) {
            c = ((uint32_t)(p[0] & 0x1F) << 6) | (p[1] & 0x3F);
            p += 2;
        } else if ((*p & 0xF0) == 0xE0) {
            c = ((uint32_t)(p[0] & 0x0F) << 12) | ((uint32_t)(p[1] & 0x3F) << 6) | (p[2] & 0x3F);
            p += 3;
        } else {
            c = ((uint32_t)(p[0] & 0x07) << 18) | ((uint32_t)(p[1] & 0x3F) << 12) |
                ((uint32_t)(p[2] & 0x3F) << 6) | (p[3] & 0x3F);
            p += 4;
        }
        cps[n++] = c;
    }
    return n;
}

/* build_comment_packet_pair + ascii/unicode builders, src/packet/comment.rs:23-81 */
size_t or_build_comment_packets(const uint8_t set_id[16], const char *comment, uint8_t *out) {
    size_t slen = strlen(comment);
    uint32_t *cps = (uint32_t *)malloc((slen + 1) * sizeof(uint32_t));
    size_t ncp = utf8_decode(comment, cps);
    int non_ascii = 0;
    for (size_t i = 0; i < ncp; i++) non_ascii |= cps[i] >= 0x80;

    /* ASCII variant: non-ASCII code points become '?' (comment.rs:45-62) */
    size_t abody_len = round_up_4(ncp);
    uint8_t *abody = (uint8_t *)calloc(abody_len ? abody_len : 1, 1);
    for (size_t i = 0; i < ncp; i++) abody[i] = cps[i] < 0x80 ? (uint8_t)cps[i] : '?';
    size_t total = 64 + abody_len;
    uint8_t ascii_md5[16] = {0};
    if (out) {
        or_build_packet(set_id, TYPE_COMMENT_ASCII, abody, abody_len, out);
        memcpy(ascii_md5, out + 16, 16);
    } else {
        uint8_t *tmp = (uint8_t *)malloc(total);
        or_build_packet(set_id, TYPE_COMMENT_ASCII, abody, abody_len, tmp);
        memcpy(ascii_md5, tmp + 16, 16);
        free(tmp);
    }
    free(abody);

    if (non_ascii) { /* Unicode variant: link ‖ UTF-16LE, padded to 4 (comment.rs:64-81) */
        size_t units = 0;
        for (size_t i = 0; i < ncp; i++) units += cps[i] >= 0x10000 ? 2 : 1;
        size_t ubody_len = round_up_4(16 + 2 * units);
        uint8_t *ubody = (uint8_t *)calloc(ubody_len, 1);
        memcpy(ubody, ascii_md5, 16);
        size_t o = 16;
        for (size_t i = 0; i < ncp; i++) {
            uint32_t c = cps[i];
            if (c >= 0x10000) {
                c -= 0x10000;
                uint16_t h = (uint16_t)(0xD800 + (c >> 10)), l = (uint16_t)(0xDC00 + (c & 0x3FF));
                ubody[o++] = (uint8_t)h; ubody[o++] = (uint8_t)(h >> 8);
                ubody[o++] = (uint8_t)l; ubody[o++] = (uint8_t)(l >> 8);
            } else {
                ubody[o++] = (uint8_t)c; ubody[o++] = (uint8_t)(c >> 8);
            }
        }
        if (out) or_build_packet(set_id, TYPE_COMMENT_UNICODE, ubody, ubody_len, out + total);
        total += 64 + ubody_len;
        free(ubody);
    }
    free(cps);
    return total;
}

/* build_recovery_packet, src/packet/recovery.rs:11-19 */
size_t or_build_recovery_packet(const uint8_t set_id[16], uint16_t exponent, const uint8_t *slice,
                                uint64_t slice_size, uint8_t *out) {
    size_t body_len = 4 + slice_size;
    if (!out) return 64 + body_len;
    uint8_t *body = (uint8_t *)malloc(body_len);
    put_le32(body, exponent);
    memcpy(body + 4, slice, slice_size);
    size_t r = or_build_packet(set_id, TYPE_RECOVERY, body, body_len, out);
    free(body);
    return r;
}

/* ---- volume sizes, src/creator.rs:325-431 ----------------------------- */
typedef struct {
    uint32_t *v;
    size_t n, cap;
} u32vec;
static void vpush(u32vec *a, uint32_t x) {
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 16;
        a->v = (uint32_t *)realloc(a->v, a->cap * sizeof(uint32_t));
    }
    a->v[a->n++] = x;
}

static int resolve(const or_scheme *sc, uint32_t total, u32vec *out) {
    switch (sc->kind) {
    case OR_SCHEME_SINGLE: /* :327 */
        vpush(out, total);
        return 0;
    case OR_SCHEME_EXPONENTIAL: { /* exponential_split, :367-385 */
        uint32_t remaining = total, next = 1;
        size_t count = 0;
        while (remaining > 0) {
            uint32_t take = next < remaining ? next : remaining;
            vpush(out, take);
            count++;
            remaining -= take;
            if (count >= 2) next = next > 0x7FFFFFFFu ? 0xFFFFFFFFu : next * 2;
        }
        return 0;
    }
    case OR_SCHEME_UNIFORM: { /* uniform_split, :390-409 */
        if (sc->count == 0 || sc->count > total) return -1;
        uint32_t base = total / sc->count, rem = total - base * sc->count;
        for (uint32_t i = 0; i + 1 < sc->count; i++) vpush(out, base);
        vpush(out, base + rem);
        return 0;
    }
    case OR_SCHEME_LIMITED: { /* :330-341 + cap_volume_sizes, :414-431 */
        if (sc->max_blocks_per_volume == 0 || !sc->inner) return -1;
        u32vec inner = {0};
        if (resolve(sc->inner, total, &inner) != 0) {
            free(inner.v);
            return -1;
        }
        uint32_t cap = sc->max_blocks_per_volume;
        for (size_t i = 0; i < inner.n; i++) {
            uint32_t n = inner.v[i];
            if (n <= cap) {
                vpush(out, n);
            } else {
                while (n > cap) {
                    vpush(out, cap);
                    n -= cap;
                }
                if (n > 0) vpush(out, n);
            }
        }
        free(inner.v);
        return 0;
    }
    case OR_SCHEME_EXPLICIT: { /* :342-359 */
        if (sc->n_sizes == 0) return -1;
        uint64_t sum = 0;
        for (uint32_t i = 0; i < sc->n_sizes; i++) {
            if (sc->sizes[i] == 0) return -1;
            sum += sc->sizes[i];
        }
        if (sum != total) return -1;
        for (uint32_t i = 0; i < sc->n_sizes; i++) vpush(out, sc->sizes[i]);
        return 0;
    }
    }
    return -1;
}

int64_t or_resolve_volume_sizes(const or_scheme *scheme, uint32_t total, uint32_t *out, uint32_t cap) {
    u32vec v = {0};
    if (resolve(scheme, total, &v) != 0) {
        free(v.v);
        return -1;
    }
    for (size_t i = 0; out && i < v.n && i < cap; i++) out[i] = v.v[i];
    int64_t n = (int64_t)v.n;
    free(v.v);
    return n;
}

/* derive_volume_filename, src/creator.rs:1046-1057: Path::file_stem/extension
 * semantics on the last component (a leading dot is part of the stem). */
size_t or_volume_filename(const char *index_path, uint16_t first_exp, uint32_t count, char *out,
                          size_t cap) {
    const char *slash = strrchr(index_path, '/');
    size_t parent_len = slash ? (size_t)(slash - index_path) : 0;
    const char *fname = slash ? slash + 1 : index_path;
    size_t flen = strlen(fname);
    const char *dot = strrchr(fname, '.');
    char stem[4096], ext[4096];
    if (flen == 0) {
        strcpy(stem, "par2rust");
        strcpy(ext, "par2");
    } else if (!dot || dot == fname) {
        snprintf(stem, sizeof stem, "%s", fname);
        strcpy(ext, "par2");
    } else {
        snprintf(stem, sizeof stem, "%.*s", (int)(dot - fname), fname);
        snprintf(ext, sizeof ext, "%s", dot + 1);
    }
    char buf[8192];
    int n;
    if (slash)
        n = snprintf(buf, sizeof buf, "%.*s/%s.vol%u+%u.%s", (int)parent_len, index_path, stem,
                     (unsigned)first_exp, (unsigned)count, ext);
    else
        n = snprintf(buf, sizeof buf, "%s.vol%u+%u.%s", stem, (unsigned)first_exp, (unsigned)count, ext);
    if (out && cap) snprintf(out, cap, "%s", buf);
    return (size_t)n;
}

/* ---- run_create_with_progress, src/creator.rs:188-321 ----------------- */
typedef struct {
    uint8_t *p;
    size_t n, cap;
} bytes_t;
static void bappend(bytes_t *b, const uint8_t *src, size_t n) {
    if (b->n + n > b->cap) {
        size_t nc = b->cap ? b->cap : 4096;
        while (nc < b->n + n) nc *= 2;
        b->p = (uint8_t *)realloc(b->p, nc);
        b->cap = nc;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
}

/* Large checks (hundreds of MB, hundreds of recovery rows) take hours on the
 * scalar encode; with this set, or_create encodes with the multi-threaded
 * GFNI port of par2_cpu_baseline.c instead (same bytes: the tests compare
 * the two).  Everything else in or_create is unchanged. */
static int g_fast_encode = 0;
void or_set_fast_encode(int on) { g_fast_encode = on; }

int64_t or_create(const or_input *inputs, uint32_t n, uint64_t slice_size, uint32_t R,
                  const or_scheme *scheme, const char *const *comments, uint32_t n_comments,
                  const char *index_path, uint8_t **out_blob, uint64_t **out_sizes, char **out_names) {
    /* validation order of run_create_with_progress (:193-218) after the scans */
    if (n == 0) return OR_ERR_NO_INPUT_FILES;
    if (n > MAX_FILES) return OR_ERR_TOO_MANY_FILES;
    if (R > MAX_RECOVERY_BLOCKS) return OR_ERR_TOO_MANY_RECOVERY_BLOCKS;
    if (slice_size == 0 || slice_size % 4) return OR_ERR_INVALID_SLICE_SIZE;

    /* SourceFile::scan for each input */
    or_slice_checksum **cks = (or_slice_checksum **)calloc(n, sizeof *cks);
    uint64_t *nsl = (uint64_t *)calloc(n, sizeof *nsl);
    uint8_t(*hf)[16] = calloc(n, 16), (*h16)[16] = calloc(n, 16), (*fid)[16] = calloc(n, 16);
    uint64_t total_blocks = 0;
    int64_t rc = 0;
    for (uint32_t f = 0; f < n; f++) {
        nsl[f] = inputs[f].len ? (inputs[f].len + slice_size - 1) / slice_size : 0;
        cks[f] = (or_slice_checksum *)calloc(nsl[f] ? nsl[f] : 1, sizeof(or_slice_checksum));
        int r = or_scan(inputs[f].data, inputs[f].len, slice_size, inputs[f].name, inputs[f].name_len,
                        cks[f], hf[f], h16[f], fid[f]);
        if (r) {
            rc = r;
            goto done;
        }
        total_blocks += nsl[f];
    }
    if (total_blocks > MAX_INPUT_BLOCKS) {
        rc = OR_ERR_TOO_MANY_INPUT_BLOCKS;
        goto done;
    }

    { /* critical packets (:219-235) */
        uint8_t set_id[16];
        bytes_t crit = {0}, blob = {0};
        size_t mlen = or_build_main_packet(slice_size, NULL, 0, NULL, NULL) + 16 * (size_t)n;
        uint8_t *tmp = (uint8_t *)malloc(mlen);
        or_build_main_packet(slice_size, (const uint8_t *)fid, n, set_id, tmp);
        bappend(&crit, tmp, mlen);
        free(tmp);
        for (uint32_t f = 0; f < n; f++) {
            size_t l = or_build_file_desc_packet(set_id, fid[f], hf[f], h16[f], inputs[f].len,
                                                 inputs[f].name, inputs[f].name_len, NULL);
            tmp = (uint8_t *)malloc(l);
            or_build_file_desc_packet(set_id, fid[f], hf[f], h16[f], inputs[f].len, inputs[f].name,
                                      inputs[f].name_len, tmp);
            bappend(&crit, tmp, l);
            free(tmp);
            l = or_build_file_verify_packet(set_id, fid[f], cks[f], nsl[f], NULL);
            tmp = (uint8_t *)malloc(l);
            or_build_file_verify_packet(set_id, fid[f], cks[f], nsl[f], tmp);
            bappend(&crit, tmp, l);
            free(tmp);
        }
        uint8_t cbuf[256];
        size_t cl = or_build_creator_packet(set_id, cbuf);
        bappend(&crit, cbuf, cl);
        for (uint32_t c = 0; c < n_comments; c++) {
            size_t l = or_build_comment_packets(set_id, comments[c], NULL);
            tmp = (uint8_t *)malloc(l);
            or_build_comment_packets(set_id, comments[c], tmp);
            bappend(&crit, tmp, l);
            free(tmp);
        }

        u32vec sizes = {0};
        if (R > 0 && resolve(scheme, R, &sizes) != 0) { /* :244 */
            free(crit.p);
            free(sizes.v);
            rc = OR_ERR_INVALID_VOLUME_SCHEME;
            goto done;
        }
        size_t nfiles = 1 + sizes.n;
        uint64_t *fsizes = (uint64_t *)calloc(nfiles, sizeof(uint64_t));
        bytes_t names = {0};
        bappend(&blob, crit.p, crit.n);
        fsizes[0] = crit.n;
        bappend(&names, (const uint8_t *)index_path, strlen(index_path) + 1);

        if (R > 0) {
            /* encode_all_recovery_blocks: inputs in caller order, padded slices */
            uint8_t *src = (uint8_t *)calloc(total_blocks * slice_size, 1);
            uint64_t o = 0;
            for (uint32_t f = 0; f < n; f++) {
                memcpy(src + o * slice_size, inputs[f].data, inputs[f].len);
                o += nsl[f];
            }
            uint8_t *rec = (uint8_t *)malloc((size_t)R * slice_size);
            if (g_fast_encode) { /* the multi-threaded GFNI port, pinned to or_encode by the tests */
                memset(rec, 0, (size_t)R * slice_size);
                cb_encode(src, 0, (uint32_t)total_blocks, slice_size, R, rec, 0);
            } else
                or_encode(src, (uint32_t)total_blocks, slice_size, R, rec);
            free(src);
            uint32_t first = 0;
            for (size_t v = 0; v < sizes.n; v++) { /* build_volume_packet, :1025-1042 */
                size_t before = blob.n;
                bappend(&blob, crit.p, crit.n);
                size_t pl = 64 + 4 + slice_size;
                uint8_t *pkt = (uint8_t *)malloc(pl);
                for (uint32_t k = 0; k < sizes.v[v]; k++) {
                    uint16_t e = (uint16_t)(first + k);
                    or_build_recovery_packet(set_id, e, rec + (size_t)e * slice_size, slice_size, pkt);
                    bappend(&blob, pkt, pl);
                }
                free(pkt);
                bappend(&blob, crit.p, crit.n);
                fsizes[1 + v] = blob.n - before;
                char name[8192];
                or_volume_filename(index_path, (uint16_t)first, sizes.v[v], name, sizeof name);
                bappend(&names, (const uint8_t *)name, strlen(name) + 1);
                first += sizes.v[v];
            }
            free(rec);
        }
        free(sizes.v);
        free(crit.p);
        *out_blob = blob.p;
        *out_sizes = fsizes;
        *out_names = (char *)names.p;
        rc = (int64_t)nfiles;
    }
done:
    for (uint32_t f = 0; f < n; f++) free(cks[f]);
    free(cks);
    free(nsl);
    free(hf);
    free(h16);
    free(fid);
    return rc;
}
