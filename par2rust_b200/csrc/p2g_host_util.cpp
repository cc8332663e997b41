// p2g_host_util.cpp -- host-side packet framing, volume logic, GF helpers,
// host MD5 and the error channel of libpar2gpu.so.
#include "p2g_host_util.h"

#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>

namespace p2g {

// ---------------------------------------------------------------------------
// Error channel: the text of Par2Error's Display impls (src/error.rs:7-41).
// ---------------------------------------------------------------------------
static thread_local std::string t_msg;
static thread_local p2g_error_detail t_detail = {0, 0, 0};

p2g_status set_error(p2g_status st, const char* fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_msg = buf;
    return st;
}
void set_error_detail(uint64_t count, uint64_t slice_size, uint64_t suggested) {
    t_detail.count = count;
    t_detail.slice_size = slice_size;
    t_detail.suggested = suggested;
}
void clear_error() {
    t_msg.clear();
    t_detail = {0, 0, 0};
}

}  // namespace p2g

extern "C" const char* p2g_last_error_message(void) { return p2g::t_msg.c_str(); }
extern "C" void p2g_last_error_detail(p2g_error_detail* out) {
    if (out) *out = p2g::t_detail;
}
extern "C" int p2g_abi_version(void) { return P2G_ABI_VERSION; }

namespace p2g {

// ---------------------------------------------------------------------------
// MD5, RFC 1321.  Host-side only: frames the small packets (main, file
// description, IFSC, creator, comments) and derives file ids; the bulk
// hashing runs on the device.
// ---------------------------------------------------------------------------
static inline uint32_t rol(uint32_t x, int s) { return (x << s) | (x >> (32 - s)); }


// Fully unrolled compression, written for the shortest dependent chain
// through b (the value the previous step produced), since one core runs the
// serial chain of a whole-file hash: the message word and constant are added
// to a before the round function; H groups y ^ z, which does not wait for b;
// and G = (x & z) | (y & ~z) is added as two disjoint terms, (y & ~z) early
// and (x & z) last, so its chain is AND, ADD instead of XOR, AND, XOR, ADD.
#define HM_F(x, y, z) ((z) ^ ((x) & ((y) ^ (z))))
#define HM_H(x, y, z) ((x) ^ ((y) ^ (z)))
#define HM_I(x, y, z) ((y) ^ ((x) | ~(z)))
#define HM_STEP(f, a, b, c, d, x, t, s) \
    (a) += (x) + (t);                   \
    (a) += f((b), (c), (d));            \
    (a) = rol((a), (s)) + (b);
#define HM_STEP_G(a, b, c, d, x, t, s) \
    (a) += (x) + (t) + ((c) & ~(d));   \
    (a) += (b) & (d);                  \
    (a) = rol((a), (s)) + (b);

static void md5_block(uint32_t st[4], const uint8_t* p) {
    uint32_t m[16];
    memcpy(m, p, 64);  // little-endian host
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
    HM_STEP(HM_F, a, b, c, d, m[0], 0xd76aa478, 7) HM_STEP(HM_F, d, a, b, c, m[1], 0xe8c7b756, 12)
    HM_STEP(HM_F, c, d, a, b, m[2], 0x242070db, 17) HM_STEP(HM_F, b, c, d, a, m[3], 0xc1bdceee, 22)
    HM_STEP(HM_F, a, b, c, d, m[4], 0xf57c0faf, 7) HM_STEP(HM_F, d, a, b, c, m[5], 0x4787c62a, 12)
    HM_STEP(HM_F, c, d, a, b, m[6], 0xa8304613, 17) HM_STEP(HM_F, b, c, d, a, m[7], 0xfd469501, 22)
    HM_STEP(HM_F, a, b, c, d, m[8], 0x698098d8, 7) HM_STEP(HM_F, d, a, b, c, m[9], 0x8b44f7af, 12)
    HM_STEP(HM_F, c, d, a, b, m[10], 0xffff5bb1, 17) HM_STEP(HM_F, b, c, d, a, m[11], 0x895cd7be, 22)
    HM_STEP(HM_F, a, b, c, d, m[12], 0x6b901122, 7) HM_STEP(HM_F, d, a, b, c, m[13], 0xfd987193, 12)
    HM_STEP(HM_F, c, d, a, b, m[14], 0xa679438e, 17) HM_STEP(HM_F, b, c, d, a, m[15], 0x49b40821, 22)
    HM_STEP_G(a, b, c, d, m[1], 0xf61e2562, 5) HM_STEP_G(d, a, b, c, m[6], 0xc040b340, 9)
    HM_STEP_G(c, d, a, b, m[11], 0x265e5a51, 14) HM_STEP_G(b, c, d, a, m[0], 0xe9b6c7aa, 20)
    HM_STEP_G(a, b, c, d, m[5], 0xd62f105d, 5) HM_STEP_G(d, a, b, c, m[10], 0x02441453, 9)
    HM_STEP_G(c, d, a, b, m[15], 0xd8a1e681, 14) HM_STEP_G(b, c, d, a, m[4], 0xe7d3fbc8, 20)
    HM_STEP_G(a, b, c, d, m[9], 0x21e1cde6, 5) HM_STEP_G(d, a, b, c, m[14], 0xc33707d6, 9)
    HM_STEP_G(c, d, a, b, m[3], 0xf4d50d87, 14) HM_STEP_G(b, c, d, a, m[8], 0x455a14ed, 20)
    HM_STEP_G(a, b, c, d, m[13], 0xa9e3e905, 5) HM_STEP_G(d, a, b, c, m[2], 0xfcefa3f8, 9)
    HM_STEP_G(c, d, a, b, m[7], 0x676f02d9, 14) HM_STEP_G(b, c, d, a, m[12], 0x8d2a4c8a, 20)
    HM_STEP(HM_H, a, b, c, d, m[5], 0xfffa3942, 4) HM_STEP(HM_H, d, a, b, c, m[8], 0x8771f681, 11)
    HM_STEP(HM_H, c, d, a, b, m[11], 0x6d9d6122, 16) HM_STEP(HM_H, b, c, d, a, m[14], 0xfde5380c, 23)
    HM_STEP(HM_H, a, b, c, d, m[1], 0xa4beea44, 4) HM_STEP(HM_H, d, a, b, c, m[4], 0x4bdecfa9, 11)
    HM_STEP(HM_H, c, d, a, b, m[7], 0xf6bb4b60, 16) HM_STEP(HM_H, b, c, d, a, m[10], 0xbebfbc70, 23)
    HM_STEP(HM_H, a, b, c, d, m[13], 0x289b7ec6, 4) HM_STEP(HM_H, d, a, b, c, m[0], 0xeaa127fa, 11)
    HM_STEP(HM_H, c, d, a, b, m[3], 0xd4ef3085, 16) HM_STEP(HM_H, b, c, d, a, m[6], 0x04881d05, 23)
    HM_STEP(HM_H, a, b, c, d, m[9], 0xd9d4d039, 4) HM_STEP(HM_H, d, a, b, c, m[12], 0xe6db99e5, 11)
    HM_STEP(HM_H, c, d, a, b, m[15], 0x1fa27cf8, 16) HM_STEP(HM_H, b, c, d, a, m[2], 0xc4ac5665, 23)
    HM_STEP(HM_I, a, b, c, d, m[0], 0xf4292244, 6) HM_STEP(HM_I, d, a, b, c, m[7], 0x432aff97, 10)
    HM_STEP(HM_I, c, d, a, b, m[14], 0xab9423a7, 15) HM_STEP(HM_I, b, c, d, a, m[5], 0xfc93a039, 21)
    HM_STEP(HM_I, a, b, c, d, m[12], 0x655b59c3, 6) HM_STEP(HM_I, d, a, b, c, m[3], 0x8f0ccc92, 10)
    HM_STEP(HM_I, c, d, a, b, m[10], 0xffeff47d, 15) HM_STEP(HM_I, b, c, d, a, m[1], 0x85845dd1, 21)
    HM_STEP(HM_I, a, b, c, d, m[8], 0x6fa87e4f, 6) HM_STEP(HM_I, d, a, b, c, m[15], 0xfe2ce6e0, 10)
    HM_STEP(HM_I, c, d, a, b, m[6], 0xa3014314, 15) HM_STEP(HM_I, b, c, d, a, m[13], 0x4e0811a1, 21)
    HM_STEP(HM_I, a, b, c, d, m[4], 0xf7537e82, 6) HM_STEP(HM_I, d, a, b, c, m[11], 0xbd3af235, 10)
    HM_STEP(HM_I, c, d, a, b, m[2], 0x2ad7d2bb, 15) HM_STEP(HM_I, b, c, d, a, m[9], 0xeb86d391, 21)
    st[0] += a;
    st[1] += b;
    st[2] += c;
    st[3] += d;
}

Md5Ctx::Md5Ctx() : total(0), fill(0) {
    st[0] = 0x67452301u;
    st[1] = 0xefcdab89u;
    st[2] = 0x98badcfeu;
    st[3] = 0x10325476u;
}
void Md5Ctx::update(const void* data, size_t len) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    total += len;
    if (fill) {
        const size_t take = std::min(len, 64 - fill);
        memcpy(buf + fill, p, take);
        fill += take;
        p += take;
        len -= take;
        if (fill == 64) {
            md5_block(st, buf);
            fill = 0;
        }
    }
    while (len >= 64) {
        md5_block(st, p);
        p += 64;
        len -= 64;
    }
    if (len) {
        memcpy(buf, p, len);
        fill = len;
    }
}
Md5 Md5Ctx::finish() {
    const uint64_t bits = total * 8;
    const uint8_t pad = 0x80;
    update(&pad, 1);
    const uint8_t zero[64] = {0};
    update(zero, fill <= 56 ? 56 - fill : 120 - fill);
    uint8_t lenb[8];
    for (int i = 0; i < 8; ++i) lenb[i] = (uint8_t)(bits >> (8 * i));
    update(lenb, 8);
    Md5 out;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(st[i] >> (8 * j));
    return out;
}
Md5 md5_of(const void* data, size_t len) {
    Md5Ctx c;
    c.update(data, len);
    return c.finish();
}

// ---------------------------------------------------------------------------
// GF(2^16) host helpers (src/galois.rs:33-87, src/reedsolomon.rs:130-157).
// ---------------------------------------------------------------------------
struct GfTables {
    uint16_t log[65536];
    uint16_t antilog[65536];
    GfTables() {
        uint32_t b = 1;
        for (uint32_t l = 0; l < 65535u; l++) {
            log[b] = (uint16_t)l;
            antilog[l] = (uint16_t)b;
            b <<= 1;
            if (b & 0x10000u) b ^= 0x1100Bu;
        }
        log[0] = 65535;
        antilog[65535] = 0;
    }
};
static const GfTables& gft() {
    static GfTables t;
    return t;
}
uint16_t gf_mul(uint16_t a, uint16_t b) {
    if (!a || !b) return 0;
    uint32_t s = (uint32_t)gft().log[a] + gft().log[b];
    if (s >= 65535u) s -= 65535u;
    return gft().antilog[s];
}
uint16_t gf_pow(uint16_t base, uint32_t exp) {
    if (exp == 0) return 1;
    if (base == 0) return 0;
    return gft().antilog[(uint32_t)(((uint64_t)gft().log[base] * exp) % 65535u)];
}
void input_bases(uint32_t count, uint16_t* out) {
    uint32_t n = 0;
    for (uint32_t l = 0; l < 65535u && n < count; l++) {
        uint32_t x = 65535u, y = l;
        while (y) {
            uint32_t t = x % y;
            x = y;
            y = t;
        }
        if (x == 1) out[n++] = gft().antilog[l];
    }
}

// ---------------------------------------------------------------------------
// Packets (src/format.rs:3-54 and src/packet/*.rs).
// ---------------------------------------------------------------------------
const uint8_t kTypeMain[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'M', 'a', 'i', 'n', 0, 0, 0, 0};
const uint8_t kTypeFileDesc[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'F', 'i', 'l', 'e', 'D', 'e', 's', 'c'};
const uint8_t kTypeFileVerify[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'I', 'F', 'S', 'C', 0, 0, 0, 0};
const uint8_t kTypeRecovery[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'R', 'e', 'c', 'v', 'S', 'l', 'i', 'c'};
const uint8_t kTypeCreator[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'C', 'r', 'e', 'a', 't', 'o', 'r', 0};
const uint8_t kTypeCommentAscii[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'C', 'o', 'm', 'm', 'A', 'S', 'C', 'I'};
const uint8_t kTypeCommentUnicode[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'C', 'o', 'm', 'm', 'U', 'n', 'i', 0};
const char kCreatorString[] = "Created by par2rust v0.1.0";
static const uint8_t kMagic[8] = {'P', 'A', 'R', '2', 0, 'P', 'K', 'T'};

static inline void put_le(uint8_t* p, uint64_t v, int n) {
    for (int i = 0; i < n; ++i) p[i] = (uint8_t)(v >> (8 * i));
}
static inline size_t round_up_4(size_t n) { return (n + 3) & ~(size_t)3; }

void append_packet(std::vector<uint8_t>& out, const Md5& set_id, const uint8_t type[16], const uint8_t* body,
                   size_t body_len) {
    Md5Ctx c;
    c.update(set_id.data(), 16);
    c.update(type, 16);
    c.update(body, body_len);
    const Md5 h = c.finish();
    const size_t at = out.size();
    out.resize(at + 64 + body_len);
    uint8_t* p = out.data() + at;
    memcpy(p, kMagic, 8);
    put_le(p + 8, 64 + body_len, 8);
    memcpy(p + 16, h.data(), 16);
    memcpy(p + 32, set_id.data(), 16);
    memcpy(p + 48, type, 16);
    if (body_len) memcpy(p + 64, body, body_len);
}

Md5 build_main_packet(uint64_t slice_size, const std::vector<Md5>& file_ids, std::vector<uint8_t>& out) {
    std::vector<Md5> sorted = file_ids;
    std::sort(sorted.begin(), sorted.end());
    std::vector<uint8_t> body(12 + 16 * sorted.size());
    put_le(body.data(), slice_size, 8);
    put_le(body.data() + 8, (uint32_t)sorted.size(), 4);
    for (size_t i = 0; i < sorted.size(); ++i) memcpy(body.data() + 12 + 16 * i, sorted[i].data(), 16);
    const Md5 set_id = md5_of(body.data(), body.size());
    append_packet(out, set_id, kTypeMain, body.data(), body.size());
    return set_id;
}

void append_file_desc(std::vector<uint8_t>& out, const Md5& set_id, const Md5& file_id, const uint8_t hash_full[16],
                      const uint8_t hash16k[16], uint64_t length, const uint8_t* name, size_t name_len) {
    std::vector<uint8_t> body(56 + round_up_4(name_len), 0);
    memcpy(body.data(), file_id.data(), 16);
    memcpy(body.data() + 16, hash_full, 16);
    memcpy(body.data() + 32, hash16k, 16);
    put_le(body.data() + 48, length, 8);
    if (name_len) memcpy(body.data() + 56, name, name_len);
    append_packet(out, set_id, kTypeFileDesc, body.data(), body.size());
}

void append_file_verify(std::vector<uint8_t>& out, const Md5& set_id, const Md5& file_id,
                        const p2g_slice_checksum* cks, uint64_t n) {
    std::vector<uint8_t> body(16 + 20 * n);
    memcpy(body.data(), file_id.data(), 16);
    for (uint64_t i = 0; i < n; ++i) {
        memcpy(body.data() + 16 + 20 * i, cks[i].md5, 16);
        put_le(body.data() + 16 + 20 * i + 16, cks[i].crc32, 4);
    }
    append_packet(out, set_id, kTypeFileVerify, body.data(), body.size());
}

void append_creator(std::vector<uint8_t>& out, const Md5& set_id) {
    const size_t n = strlen(kCreatorString);
    std::vector<uint8_t> body(round_up_4(n), 0);
    memcpy(body.data(), kCreatorString, n);
    append_packet(out, set_id, kTypeCreator, body.data(), body.size());
}

// UTF-8 -> code points (Rust Strings are valid UTF-8; invalid bytes map to U+FFFD).
static std::vector<uint32_t> utf8_codepoints(const char* s) {
    std::vector<uint32_t> cps;
    const unsigned char* p = (const unsigned char*)s;
    while (*p) {
        uint32_t c;
        int n;
        if (*p < 0x80) { c = *p; n = 1; }
        else if ((*p & 0xE0) == 0xC0) { c = *p & 0x1F; n = 2; }
        else if ((*p & 0xF0) == 0xE0) { c = *p & 0x0F; n = 3; }
        else if ((*p & 0xF8) == 0xF0) { c = *p & 0x07; n = 4; }
        else { cps.push_back(0xFFFD); ++p; continue; }
        bool ok = true;
        for (int i = 1; i < n; ++i) {
            if ((p[i] & 0xC0) != 0x80) { ok = false; break; }
            c = (c << 6) | (p[i] & 0x3F);
        }
        if (!ok) { cps.push_back(0xFFFD); ++p; continue; }
        cps.push_back(c);
        p += n;
    }
    return cps;
}

// build_comment_packet_pair, src/packet/comment.rs:23-81
void append_comments(std::vector<uint8_t>& out, const Md5& set_id, const char* comment) {
    const std::vector<uint32_t> cps = utf8_codepoints(comment);
    bool non_ascii = false;
    std::vector<uint8_t> abody(round_up_4(cps.size()), 0);
    for (size_t i = 0; i < cps.size(); ++i) {
        abody[i] = cps[i] < 0x80 ? (uint8_t)cps[i] : (uint8_t)'?';
        non_ascii |= cps[i] >= 0x80;
    }
    const size_t at = out.size();
    append_packet(out, set_id, kTypeCommentAscii, abody.data(), abody.size());
    if (!non_ascii) return;
    std::vector<uint8_t> ubody(out.begin() + at + 16, out.begin() + at + 32);  // ASCII packet MD5
    for (uint32_t c : cps) {
        if (c >= 0x10000) {
            c -= 0x10000;
            const uint16_t hs = (uint16_t)(0xD800 + (c >> 10)), ls = (uint16_t)(0xDC00 + (c & 0x3FF));
            ubody.push_back((uint8_t)hs); ubody.push_back((uint8_t)(hs >> 8));
            ubody.push_back((uint8_t)ls); ubody.push_back((uint8_t)(ls >> 8));
        } else {
            ubody.push_back((uint8_t)c); ubody.push_back((uint8_t)(c >> 8));
        }
    }
    while (ubody.size() % 4) ubody.push_back(0);
    append_packet(out, set_id, kTypeCommentUnicode, ubody.data(), ubody.size());
}

void recovery_packet_header(uint8_t out[68], const Md5& set_id, const uint8_t pkt_md5[16], uint64_t slice_size,
                            uint32_t exponent) {
    memcpy(out, kMagic, 8);
    put_le(out + 8, 64 + 4 + slice_size, 8);
    memcpy(out + 16, pkt_md5, 16);
    memcpy(out + 32, set_id.data(), 16);
    memcpy(out + 48, kTypeRecovery, 16);
    put_le(out + 64, exponent, 4);
}

Md5 file_id_of(const uint8_t hash16k[16], uint64_t length, const uint8_t* name, size_t name_len) {
    Md5Ctx c;
    c.update(hash16k, 16);
    uint8_t l[8];
    put_le(l, length, 8);
    c.update(l, 8);
    c.update(name, name_len);
    return c.finish();
}

// ---------------------------------------------------------------------------
// Validation shared by the create entry points (src/creator.rs:193-218,
// :461-508, src/source.rs:65-75).
// ---------------------------------------------------------------------------
p2g_status check_common(uint32_t n, uint32_t R, uint64_t slice) {
    if (n == 0) return set_error(P2G_ERR_NO_INPUT_FILES, "no input files supplied");
    if (n > P2G_MAX_FILES)
        return set_error(P2G_ERR_TOO_MANY_FILES, "too many input files (%u); PAR2 limit is 32768", n);
    if (R > P2G_MAX_RECOVERY_BLOCKS)
        return set_error(P2G_ERR_TOO_MANY_RECOVERY_BLOCKS, "recovery block count %u exceeds PAR2 limit of 65535", R);
    if (slice == 0 || slice % 4)
        return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size %llu: must be > 0 and a multiple of 4",
                         (unsigned long long)slice);
    return P2G_OK;
}
p2g_status check_name(const uint8_t* name, size_t len, const char* path) {
    if (len == 0 || !name || memchr(name, 0, len))
        return set_error(P2G_ERR_INVALID_FILE_NAME,
                         "filename \"%s\" is empty or contains a NUL byte; PAR2 does not permit either",
                         path ? path : "");
    return P2G_OK;
}
p2g_status check_total_blocks(uint64_t total_blocks, uint64_t total_bytes, uint64_t slice) {
    if (total_blocks > P2G_MAX_INPUT_BLOCKS) {
        const uint64_t raw = (total_bytes + P2G_MAX_INPUT_BLOCKS - 1) / P2G_MAX_INPUT_BLOCKS;
        const uint64_t suggested = (raw + 3) / 4 * 4;
        set_error_detail(total_blocks, slice, suggested);
        return set_error(P2G_ERR_TOO_MANY_INPUT_BLOCKS,
                         "too many input blocks (%llu) at slice_size %llu; PAR2 caps total slices at 32768 — retry "
                         "with slice_size >= %llu",
                         (unsigned long long)total_blocks, (unsigned long long)slice, (unsigned long long)suggested);
    }
    return P2G_OK;
}

// ---------------------------------------------------------------------------
// Volumes
// ---------------------------------------------------------------------------
p2g_status resolve_volume_sizes(const p2g_volume_scheme& sc, uint32_t total, std::vector<uint32_t>& out) {
    out.clear();
    switch (sc.kind) {
    case P2G_SCHEME_SINGLE:
        out.push_back(total);
        return P2G_OK;
    case P2G_SCHEME_EXPONENTIAL: {  // exponential_split, src/creator.rs:367-385
        uint32_t remaining = total, next = 1;
        while (remaining > 0) {
            const uint32_t take = std::min(next, remaining);
            out.push_back(take);
            remaining -= take;
            if (out.size() >= 2) next = next > 0x7FFFFFFFu ? 0xFFFFFFFFu : next * 2;
        }
        return P2G_OK;
    }
    case P2G_SCHEME_UNIFORM: {  // uniform_split, :390-409
        if (sc.count == 0)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME, "invalid volume scheme: Uniform scheme requires count > 0");
        if (sc.count > total)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                             "invalid volume scheme: Uniform scheme count (%u) exceeds recovery block total (%u)",
                             sc.count, total);
        const uint32_t base = total / sc.count, rem = total - base * sc.count;
        for (uint32_t i = 0; i + 1 < sc.count; ++i) out.push_back(base);
        out.push_back(base + rem);
        return P2G_OK;
    }
    case P2G_SCHEME_LIMITED: {  // :330-341 + cap_volume_sizes :414-431
        if (sc.max_blocks_per_volume == 0)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                             "invalid volume scheme: Limited scheme requires max_blocks_per_volume > 0");
        if (!sc.inner)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME, "invalid volume scheme: Limited scheme needs an inner scheme");
        std::vector<uint32_t> inner;
        p2g_status st = resolve_volume_sizes(*sc.inner, total, inner);
        if (st != P2G_OK) return st;
        const uint32_t cap = sc.max_blocks_per_volume;
        for (uint32_t n : inner) {
            if (n <= cap) {
                out.push_back(n);
            } else {
                while (n > cap) {
                    out.push_back(cap);
                    n -= cap;
                }
                if (n > 0) out.push_back(n);
            }
        }
        return P2G_OK;
    }
    case P2G_SCHEME_EXPLICIT: {  // :342-359
        if (sc.explicit_count == 0 || !sc.explicit_sizes)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                             "invalid volume scheme: explicit scheme requires at least one volume");
        uint64_t sum = 0;
        for (uint32_t i = 0; i < sc.explicit_count; ++i) {
            if (sc.explicit_sizes[i] == 0)
                return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                                 "invalid volume scheme: explicit scheme volumes must each have >0 recovery blocks");
            sum += sc.explicit_sizes[i];
        }
        if (sum != total)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                             "invalid volume scheme: explicit volume sizes sum to %llu, expected %u",
                             (unsigned long long)sum, total);
        out.assign(sc.explicit_sizes, sc.explicit_sizes + sc.explicit_count);
        return P2G_OK;
    }
    }
    return set_error(P2G_ERR_INVALID_VOLUME_SCHEME, "invalid volume scheme: unknown kind %u", sc.kind);
}

// derive_volume_filename, src/creator.rs:1046-1057 (Path::file_stem /
// Path::extension semantics on the last component).
std::string volume_filename(const std::string& index_path, uint16_t first_exp, uint32_t count) {
    const size_t slash = index_path.rfind('/');
    const std::string parent = slash == std::string::npos ? std::string() : index_path.substr(0, slash);
    const std::string fname = slash == std::string::npos ? index_path : index_path.substr(slash + 1);
    std::string stem, ext;
    const size_t dot = fname.rfind('.');
    if (fname.empty()) {
        stem = "par2rust";
        ext = "par2";
    } else if (dot == std::string::npos || dot == 0) {
        stem = fname;
        ext = "par2";
    } else {
        stem = fname.substr(0, dot);
        ext = fname.substr(dot + 1);
    }
    const std::string leaf = stem + ".vol" + std::to_string(first_exp) + "+" + std::to_string(count) + "." + ext;
    if (slash == std::string::npos) return leaf;
    return parent + "/" + leaf;
}

// write_atomic, src/creator.rs:1070-1087: tmp file, fsync, rename.
p2g_status write_atomic(const std::string& path, const std::vector<std::pair<const uint8_t*, size_t>>& pieces) {
    const std::string tmp = path + ".par2rust.tmp";
    const int fd = open(tmp.c_str(), O_WRONLY | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
    if (fd < 0) return set_error(P2G_ERR_IO, "I/O error: %s: %s", tmp.c_str(), strerror(errno));
    for (const auto& pc : pieces) {
        const uint8_t* p = pc.first;
        size_t left = pc.second;
        while (left) {
            const ssize_t w = write(fd, p, left > (1u << 30) ? (1u << 30) : left);
            if (w < 0) {
                if (errno == EINTR) continue;
                const int e = errno;
                close(fd);
                return set_error(P2G_ERR_IO, "I/O error: %s: %s", tmp.c_str(), strerror(e));
            }
            p += w;
            left -= (size_t)w;
        }
    }
    if (fsync(fd) != 0) {
        const int e = errno;
        close(fd);
        return set_error(P2G_ERR_IO, "I/O error: %s: %s", tmp.c_str(), strerror(e));
    }
    close(fd);
    if (rename(tmp.c_str(), path.c_str()) != 0)
        return set_error(P2G_ERR_IO, "I/O error: %s: %s", path.c_str(), strerror(errno));
    return P2G_OK;
}

}  // namespace p2g

// ---------------------------------------------------------------------------
// C ABI: host helpers mirrored from the reference's public modules.
// ---------------------------------------------------------------------------
extern "C" p2g_status p2g_input_bases(uint32_t count, uint16_t* out) {
    if (count > P2G_MAX_INPUT_BLOCKS || (count && !out))
        return p2g::set_error(P2G_ERR_INVALID_ARGUMENT, "input base count %u exceeds 32768", count);
    p2g::input_bases(count, out);
    return P2G_OK;
}
extern "C" uint16_t p2g_gf_mul(uint16_t a, uint16_t b) { return p2g::gf_mul(a, b); }
extern "C" uint16_t p2g_gf_pow(uint16_t base, uint32_t exp) { return p2g::gf_pow(base, exp); }
extern "C" p2g_status p2g_resolve_volume_sizes(const p2g_volume_scheme* scheme, uint32_t total, uint32_t* out,
                                               uint32_t cap, uint32_t* n_out) {
    if (!scheme) return p2g::set_error(P2G_ERR_INVALID_ARGUMENT, "scheme is NULL");
    std::vector<uint32_t> v;
    p2g_status st = p2g::resolve_volume_sizes(*scheme, total, v);
    if (st != P2G_OK) return st;
    if (n_out) *n_out = (uint32_t)v.size();
    for (size_t i = 0; out && i < v.size() && i < cap; ++i) out[i] = v[i];
    return P2G_OK;
}
extern "C" char* p2g_volume_filename(const char* index_path, uint16_t first_exponent, uint32_t count) {
    const std::string s = p2g::volume_filename(index_path ? index_path : "", first_exponent, count);
    char* r = (char*)malloc(s.size() + 1);
    memcpy(r, s.c_str(), s.size() + 1);
    return r;
}
extern "C" size_t p2g_build_packet(const uint8_t set_id[16], const uint8_t type_tag[16], const uint8_t* body,
                                   size_t body_len, uint8_t* out) {
    if (!out) return 64 + body_len;
    std::vector<uint8_t> v;
    p2g::Md5 sid;
    memcpy(sid.data(), set_id, 16);
    p2g::append_packet(v, sid, type_tag, body, body_len);
    memcpy(out, v.data(), v.size());
    return v.size();
}
extern "C" size_t p2g_build_main_packet(uint64_t slice_size, const uint8_t* file_ids, uint32_t n,
                                        uint8_t set_id_out[16], uint8_t* out) {
    std::vector<p2g::Md5> ids(n);
    for (uint32_t i = 0; i < n; ++i) memcpy(ids[i].data(), file_ids + 16 * i, 16);
    std::vector<uint8_t> v;
    const p2g::Md5 sid = p2g::build_main_packet(slice_size, ids, v);
    if (set_id_out) memcpy(set_id_out, sid.data(), 16);
    if (out) memcpy(out, v.data(), v.size());
    return v.size();
}
extern "C" void p2g_compute_file_id(const uint8_t hash16k[16], uint64_t length, const uint8_t* name,
                                    size_t name_len, uint8_t out[16]) {
    const p2g::Md5 id = p2g::file_id_of(hash16k, length, name, name_len);
    memcpy(out, id.data(), 16);
}
extern "C" void p2g_md5(const uint8_t* data, size_t len, uint8_t out[16]) {
    const p2g::Md5 h = p2g::md5_of(data, len);
    memcpy(out, h.data(), 16);
}
