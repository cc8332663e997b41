// p2g_cli_args.cpp -- the create CLI's argument semantics (src/main.rs of
// par2rust): slice-size suffixes, the -r redundancy forms and their
// resolution to a recovery count, and the volume scheme built from the
// -u / -l / -n / --single-volume flags.  These decide which bytes a create
// writes (-r sets R, -l caps volumes), so they are exported over the C ABI
// and the par2rust CLI (p2g_cli.cpp) is a thin shell around them.
#include <inttypes.h>
#include <stdio.h>
#include <string.h>

#include <string>

#include "p2g_host_util.h"

using namespace p2g;

namespace {
// Rust's u64::from_str: an optional '+', then one or more ASCII digits, no
// overflow.  false on anything else.
bool parse_u64(const std::string& s, uint64_t* out) {
    size_t i = 0;
    if (i < s.size() && s[i] == '+') ++i;
    if (i == s.size()) return false;
    uint64_t v = 0;
    for (; i < s.size(); ++i) {
        const char c = s[i];
        if (c < '0' || c > '9') return false;
        const uint64_t d = (uint64_t)(c - '0');
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    *out = v;
    return true;
}
}  // namespace

// parse_slice_size, src/main.rs:464-487
extern "C" p2g_status p2g_parse_slice_size(const char* s, uint64_t* out) {
    clear_error();
    if (!s || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL argument");
    const std::string str(s);
    if (str.empty()) return set_error(P2G_ERR_INVALID_ARGUMENT, "slice size is empty");
    const char last = str.back();
    uint32_t shift = 0;
    std::string digits = str;
    switch (last) {
        case 'b': case 'B': shift = 0; digits.pop_back(); break;
        case 'k': case 'K': shift = 10; digits.pop_back(); break;
        case 'm': case 'M': shift = 20; digits.pop_back(); break;
        case 'g': case 'G': shift = 30; digits.pop_back(); break;
        default: break;
    }
    if (digits.empty())
        return set_error(P2G_ERR_INVALID_ARGUMENT, "slice size '%s' is missing a numeric value", s);
    uint64_t n = 0;
    if (!parse_u64(digits, &n))
        return set_error(P2G_ERR_INVALID_ARGUMENT, "slice size '%s' has invalid number '%s'", s, digits.c_str());
    if (shift && n > (UINT64_MAX >> shift))
        return set_error(P2G_ERR_INVALID_ARGUMENT, "slice size '%s' overflows u64", s);
    *out = n << shift;
    return P2G_OK;
}

// Redundancy::from_str, src/main.rs:496-531.  A size target's shift is not
// overflow-checked there (checked_shl only rejects shift >= 64), so it wraps
// here too.
extern "C" p2g_status p2g_parse_redundancy(const char* s, p2g_redundancy* out) {
    clear_error();
    if (!s || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL argument");
    const std::string str(s);
    if (str.empty()) return set_error(P2G_ERR_INVALID_ARGUMENT, "redundancy value is empty");
    uint32_t shift = 0;
    switch (str[0]) {
        case 'k': case 'K': shift = 10; break;
        case 'm': case 'M': shift = 20; break;
        case 'g': case 'G': shift = 30; break;
        default: break;
    }
    memset(out, 0, sizeof *out);
    if (shift) {
        const std::string rest = str.substr(1);
        if (rest.empty()) return set_error(P2G_ERR_INVALID_ARGUMENT, "redundancy '%s' is missing a numeric value", s);
        uint64_t n = 0;
        if (!parse_u64(rest, &n))
            return set_error(P2G_ERR_INVALID_ARGUMENT, "redundancy '%s' has invalid number '%s'", s, rest.c_str());
        out->is_bytes = 1;
        out->target_bytes = n << shift;
        return P2G_OK;
    }
    uint64_t n = 0;
    if (!parse_u64(str, &n) || n > UINT32_MAX)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "redundancy '%s' is not a percentage or [gmk]N value", s);
    out->percent = (uint32_t)n;
    return P2G_OK;
}

// resolve_redundancy, src/main.rs:533-556
extern "C" p2g_status p2g_resolve_redundancy(const p2g_redundancy* r, uint64_t total_input_blocks, uint64_t slice_size,
                                             uint32_t* out) {
    clear_error();
    if (!r || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL argument");
    uint64_t blocks;
    if (r->is_bytes) {
        const uint64_t d = slice_size ? slice_size : 1;
        blocks = r->target_bytes / d + (r->target_bytes % d ? 1 : 0);
    } else {
        const uint64_t p = r->percent;
        const uint64_t num = (p && total_input_blocks > UINT64_MAX / p) ? UINT64_MAX : total_input_blocks * p;
        blocks = num / 100 + (num % 100 ? 1 : 0);
    }
    if (blocks == 0) {
        if (r->is_bytes)
            return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                             "invalid volume scheme: -r TargetBytes(%" PRIu64
                             ") resolves to 0 recovery blocks (input is too small or value too low)",
                             r->target_bytes);
        return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                         "invalid volume scheme: -r Percent(%u) resolves to 0 recovery blocks (input is too small or "
                         "value too low)",
                         r->percent);
    }
    *out = blocks > UINT32_MAX ? UINT32_MAX : (uint32_t)blocks;
    return P2G_OK;
}

// build_volume_scheme, src/main.rs:289-337 (default_uniform_count :283-287)
extern "C" p2g_status p2g_build_volume_scheme(const p2g_cli_volume_flags* f, uint64_t largest_source_length,
                                              uint64_t slice_size, uint32_t recovery_count, p2g_volume_scheme* out,
                                              p2g_volume_scheme* inner_out) {
    clear_error();
    if (!f || !out || !inner_out) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL argument");
    memset(out, 0, sizeof *out);
    memset(inner_out, 0, sizeof *inner_out);
    if (f->single_volume && (f->uniform || f->limit_size || f->has_volume_count))
        return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                         "invalid volume scheme: --single-volume cannot be combined with -u, -l, or -n");
    if (f->single_volume) {
        out->kind = P2G_SCHEME_SINGLE;
        return P2G_OK;
    }
    if (f->has_volume_count && !f->uniform)
        return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                         "invalid volume scheme: -n/--volume-count currently requires -u/--uniform");
    p2g_volume_scheme inner;
    memset(&inner, 0, sizeof inner);
    if (f->uniform) {
        inner.kind = P2G_SCHEME_UNIFORM;
        inner.count = f->has_volume_count ? f->volume_count
                                          : (recovery_count < 1 ? 1u : recovery_count > 15 ? 15u : recovery_count);
    } else {
        inner.kind = P2G_SCHEME_EXPONENTIAL;
    }
    if (!f->limit_size) {
        *out = inner;
        return P2G_OK;
    }
    if (largest_source_length == 0)
        return set_error(P2G_ERR_INVALID_VOLUME_SCHEME,
                         "invalid volume scheme: -l/--limit-size requires at least one non-empty source file");
    if (!slice_size) return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size 0: must be > 0 and a multiple of 4");
    uint64_t cap = largest_source_length / slice_size;
    if (cap < 1) cap = 1;
    *inner_out = inner;
    out->kind = P2G_SCHEME_LIMITED;
    out->max_blocks_per_volume = cap > UINT32_MAX ? UINT32_MAX : (uint32_t)cap;
    out->inner = inner_out;
    return P2G_OK;
}
