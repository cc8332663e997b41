// p2g_host_util.h -- host-side pieces of the create path that stay on the
// CPU: packet framing, volume splitting and naming, GF helpers, the host MD5
// used to frame packets, and the thread-local error channel.
#pragma once
#include <stdarg.h>
#include <stddef.h>
#include <stdint.h>

#include <array>
#include <string>
#include <vector>

#include "../../include/par2gpu.h"

namespace p2g {

using Md5 = std::array<uint8_t, 16>;

// ---- error channel (thread-local) ----
p2g_status set_error(p2g_status st, const char* fmt, ...);
void set_error_detail(uint64_t count, uint64_t slice_size, uint64_t suggested);
void clear_error();

// ---- host MD5 (RFC 1321), incremental ----
struct Md5Ctx {
    uint32_t st[4];
    uint64_t total;
    uint8_t buf[64];
    size_t fill;
    Md5Ctx();
    void update(const void* data, size_t len);
    Md5 finish();
};
Md5 md5_of(const void* data, size_t len);

// ---- GF(2^16) (src/galois.rs) ----
uint16_t gf_mul(uint16_t a, uint16_t b);
uint16_t gf_pow(uint16_t base, uint32_t exp);
void input_bases(uint32_t count, uint16_t* out);

// ---- packets (src/format.rs, src/packet/*) ----
extern const uint8_t kTypeMain[16], kTypeFileDesc[16], kTypeFileVerify[16], kTypeRecovery[16],
    kTypeCreator[16], kTypeCommentAscii[16], kTypeCommentUnicode[16];
extern const char kCreatorString[];
void append_packet(std::vector<uint8_t>& out, const Md5& set_id, const uint8_t type[16],
                   const uint8_t* body, size_t body_len);
Md5 build_main_packet(uint64_t slice_size, const std::vector<Md5>& file_ids, std::vector<uint8_t>& out);
void append_file_desc(std::vector<uint8_t>& out, const Md5& set_id, const Md5& file_id,
                      const uint8_t hash_full[16], const uint8_t hash16k[16], uint64_t length,
                      const uint8_t* name, size_t name_len);
void append_file_verify(std::vector<uint8_t>& out, const Md5& set_id, const Md5& file_id,
                        const p2g_slice_checksum* cks, uint64_t n);
void append_creator(std::vector<uint8_t>& out, const Md5& set_id);
void append_comments(std::vector<uint8_t>& out, const Md5& set_id, const char* comment);
// 64-byte header of a recovery packet whose packet MD5 is already known.
void recovery_packet_header(uint8_t out[68], const Md5& set_id, const uint8_t pkt_md5[16],
                            uint64_t slice_size, uint32_t exponent);
Md5 file_id_of(const uint8_t hash16k[16], uint64_t length, const uint8_t* name, size_t name_len);

// ---- volumes (src/creator.rs:325-431, 1046-1057) ----
// Returns P2G_OK or P2G_ERR_INVALID_VOLUME_SCHEME (message set).
p2g_status resolve_volume_sizes(const p2g_volume_scheme& sc, uint32_t total, std::vector<uint32_t>& out);
std::string volume_filename(const std::string& index_path, uint16_t first_exp, uint32_t count);

// ---- validation shared by the create entry points (src/creator.rs:193-218,
// :461-508, src/source.rs:65-75); each sets the error message ----
p2g_status check_common(uint32_t n, uint32_t R, uint64_t slice);
p2g_status check_name(const uint8_t* name, size_t len, const char* path);
p2g_status check_total_blocks(uint64_t total_blocks, uint64_t total_bytes, uint64_t slice);

// ---- filesystem ----
p2g_status write_atomic(const std::string& path, const std::vector<std::pair<const uint8_t*, size_t>>& pieces);

}  // namespace p2g
