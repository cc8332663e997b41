// p2g_kernels.cu -- sm_100a kernels of the PAR2 create path.
//
//   basis_kernel      per (input slice, row group): c(r,s)*2^j, j<16, the 16
//                     GF(2^16) products every lookup table is built from
//   encode_lut_kernel the Reed-Solomon accumulator recovery[r] ^= c(r,s)*src[s]
//                     (src/reedsolomon.rs:56-126, src/creator.rs:934-1007)
//   md5_*_kernel      multi-buffer MD5, one stream per thread
//                     (src/source.rs:165-228, src/format.rs:33-54)
//   crc_slices_kernel CRC-32/IEEE per slice, one warp per slice
//                     (src/source.rs:172,181)
//
// GF(2^16) arithmetic follows src/galois.rs: polynomial 0x1100B, generator
// 2, symbols are little-endian u16 pairs of bytes.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "p2g_internal.h"
#include "p2g_mma_tile.cuh"

namespace p2g {

// log/antilog tables (src/galois.rs:33-53) and the logarithms of the input
// bases (src/reedsolomon.rs:130-149: the i-th integer coprime to 65535).
__device__ uint16_t d_log[65536];
__device__ uint16_t d_antilog[65536];
__device__ uint16_t d_logbase[32768];

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
static inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

cudaError_t upload_tables() {
    static std::mutex mu;
    static bool done[256] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 256 && done[dev]) return cudaSuccess;
    std::vector<uint16_t> lg(65536), al(65536), lb(32768);
    uint32_t b = 1;
    for (uint32_t l = 0; l < kFieldLimit; l++) {
        lg[b] = (uint16_t)l;
        al[l] = (uint16_t)b;
        b <<= 1;
        if (b & 0x10000u) b ^= kFieldGenerator;
    }
    lg[0] = (uint16_t)kFieldLimit;
    al[kFieldLimit] = 0;
    uint32_t n = 0;
    for (uint32_t l = 0; l < kFieldLimit && n < 32768; l++) {
        uint32_t x = kFieldLimit, y = l;
        while (y) {
            uint32_t t = x % y;
            x = y;
            y = t;
        }
        if (x == 1) lb[n++] = (uint16_t)l;
    }
    if ((e = cudaMemcpyToSymbol(d_log, lg.data(), 65536 * 2)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(d_antilog, al.data(), 65536 * 2)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(d_logbase, lb.data(), 32768 * 2)) != cudaSuccess) return e;
    if (dev >= 0 && dev < 256) done[dev] = true;
    return cudaSuccess;
}

// Device addresses of the antilog and input-logbase tables (for kernels in
// other translation units, which cannot name these arrays directly).
cudaError_t gf_device_tables(const uint16_t** antilog, const uint16_t** logbase) {
    void* a = nullptr;
    void* l = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&a, d_antilog);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&l, d_logbase);
    *antilog = static_cast<const uint16_t*>(a);
    *logbase = static_cast<const uint16_t*>(l);
    return e;
}

// ---------------------------------------------------------------------------
// PTX helpers: shared-memory addressing, mbarrier, 1-D bulk TMA copies.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Ends an mbarrier object's life, so that its bytes may hold other data.
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~2^22 polls (each poll may suspend briefly)
// and reports failure instead of spinning forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Global -> shared bulk copy (no multicast), completion counted on `bar`.
// dst, src and bytes must be multiples of 16.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// x*m + y as one IMAD (m a run-time value keeps ptxas from rewriting it)
__device__ __forceinline__ uint32_t mad1(uint32_t x, uint32_t m, uint32_t y) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(m), "r"(y));
    return r;
}
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr));
    return v;
}
__device__ __forceinline__ void sts32(uint32_t addr, uint32_t v) {
    asm volatile("st.shared.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ void sts16(uint32_t addr, uint16_t v) {
    asm volatile("st.shared.b16 [%0], %1;" ::"r"(addr), "h"(v) : "memory");
}
__device__ __forceinline__ uint32_t lds32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

// ---------------------------------------------------------------------------
// Coefficient basis.  c(r,s) = base_s^(first_exp+r) = 2^(logbase_s*(first_exp+r)
// mod 65535) (RsEncoder::coefficient + gf_pow, src/reedsolomon.rs:56-60,
// src/galois.rs:74-87); the basis entry j is c*2^j = antilog[log c + j].
// Layout [s][rg][jj][hi][32 rows] u16 (j = 8*hi + jj): one contiguous 1 KiB
// block per (s, rg), ordered so that a warp's basis loads in the table build
// (lane = row pair + 16*hi) hit 32 distinct banks.  Rows r >= R get 0 (their
// tables are all-zero and never stored).
// ---------------------------------------------------------------------------
// fold > 1: the last row group's rows repeat its first 32/fold rows (the
// layout a folded encode CTA builds its replicated tables from; an unfolded
// CTA only stores rows < R, which are the same either way).
//
// One warp per (s, rg) block, lane = table row: one exponent and one antilog
// lookup per row give c, then c*2^(j+1) = (c*2^j)*2, a shift that folds the
// generator polynomial 0x1100B back in when bit 15 falls off.  Each store of
// the warp writes 32 consecutive u16 (one 64-byte run).
__device__ __forceinline__ void basis_fill(uint16_t* __restrict__ basis, uint32_t S, uint32_t RG, uint32_t R,
                                           uint32_t first_exp, uint64_t warp_start, uint64_t warp_step,
                                           uint32_t fold = 1) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t blocks = (uint64_t)S * RG;
    for (uint64_t sg = warp_start; sg < blocks; sg += warp_step) {
        const uint32_t rg = (uint32_t)(sg % RG);
        const uint32_t s = (uint32_t)(sg / RG);
        const uint32_t r = rg * kRowsPerGroup + (rg + 1 == RG ? lane & (31u >> (fold >> 1)) : lane);
        uint32_t v = 0;
        if (r < R) {
            // logbase * e < 2^33; 2^32 = 1 (mod 65535), so fold the high word in
            const uint64_t p = (uint64_t)d_logbase[s] * (first_exp + r);
            uint32_t x = (uint32_t)p;
            x = (x & 0xFFFFu) + (x >> 16);
            x = (x & 0xFFFFu) + (x >> 16) + (uint32_t)(p >> 32);
            x = (x & 0xFFFFu) + (x >> 16);
            if (x >= kFieldLimit) x -= kFieldLimit;
            v = d_antilog[x];
        }
        uint16_t* out = basis + sg * 512 + lane;
#pragma unroll
        for (uint32_t j = 0; j < 16; ++j) {
            out[((j & 7u) * 2u + (j >> 3)) * 32u] = (uint16_t)v;
            v = ((v << 1) & 0xFFFFu) ^ ((v & 0x8000u) ? 0x100Bu : 0u);
        }
    }
}

__global__ void basis_kernel(uint16_t* __restrict__ basis, uint32_t S, uint32_t RG, uint32_t R,
                             uint32_t first_exp, uint32_t fold) {
    basis_fill(basis, S, RG, R, first_exp, ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
               ((uint64_t)gridDim.x * blockDim.x) >> 5, fold);
}

// ---------------------------------------------------------------------------
// Reed-Solomon accumulator, split byte tables in shared memory.
//
// A CTA owns 32 recovery rows (row group rg) and a tile of NT symbol
// positions, and keeps its 32 x NT accumulator in registers for the whole
// pass over the S input slices.  Per input slice it builds, from the 16
// basis products, the two byte tables of all 32 coefficients:
//     lo[v] = c*v,  hi[v] = c*(v<<8),   v < 256,
// stored "row-major over coefficients": table row v is 128 bytes = 32 u32
// words, words 0..15 the lo products of rows (2p, 2p+1), words 16..31 the
// hi products.  A lookup of one symbol byte thus returns the products of 8
// rows with one 16-byte shared load, and c*x = lo[x & 255] ^ hi[x >> 8].
//
// Lane mapping: 4 lanes (k = 0..3, rows 8k..8k+7) per symbol, 8 symbols
// (lane groups g) per warp instruction.  Even groups look up lo first, odd
// groups hi first, so each 8-lane quarter reads one 64-byte lo segment
// (banks 0-15) and one 64-byte hi segment (banks 16-31): conflict-free.
//
// Source tiles and basis blocks are staged by 1-D bulk TMA copies into a
// kEncStages-deep ring guarded by mbarriers; one __syncthreads per slice
// separates table builds (double-buffered) from lookups.
// ---------------------------------------------------------------------------
constexpr int kTabBytes = 256 * 128;
__device__ uint32_t d_row_bytes = 128;

__host__ __device__ constexpr int ctz5(int u) {
    return (u & 1) ? 0 : (u & 2) ? 1 : (u & 4) ? 2 : (u & 8) ? 3 : 4;
}

// FMAX: largest row-group fold the CTA may run (a stage holds FMAX tiles);
// STAGES: depth of the TMA ring.
template <int NCH, int FMAX = 1, int STAGES = kEncStages>
__host__ __device__ constexpr size_t encode_bars_offset() {
    return 2 * kTabBytes + (size_t)STAGES * (FMAX * (kEncThreads / 32) * NCH * 64 * 2 + 1024);
}
template <int NCH, int FMAX = 1, int STAGES = kEncStages>
__host__ __device__ constexpr size_t encode_smem_bytes() {
    return encode_bars_offset<NCH, FMAX, STAGES>() + STAGES * sizeof(uint64_t);
}

// One (row group, symbol tile) work unit of the accumulator: 32 rows x
// tile_syms symbols from n0, over all S input slices.  `phase` holds the
// mbarrier parity of each stage's next use, so a persistent CTA can run
// tiles back to back on the same barriers; it is advanced on return.
// Returns false (uniformly over the CTA) when a bounded TMA wait gave up;
// copies still in flight have then been waited for.
//
// GEN: derive the 16 basis products of each slice in the kernel instead of
// loading them: warp w (= j) lane l (= row) looks up c*2^j =
// antilog[(logbase_s * (first_exp + r) mod 65535 + j) mod 65535], two
// slices ahead, into one of two 1 KiB slots (no basis buffer in HBM).
//
// s0 / accumulate: the tile covers input slices [s0, s0+S) only; with
// accumulate it XORs its partial sums into the recovery rows (atomic XOR
// reductions, so chunks of one tile may run concurrently on rows that start
// zeroed).
//
// fold (1, 2 or 4; <= FMAX): a row group with at most 32/fold real rows
// replicates its coefficients fold times across the 32 table rows, and lane
// k's row quad then serves sub-tile k >> (2 - log2 fold) of fold adjacent
// sub-tiles of sub_syms symbols.  Lookups keep the 32-row bank pattern (each
// lane still reads quad k of a table row), so a short last row group costs
// 1/fold of a full one instead of a full one.
__device__ __forceinline__ uint32_t mod_field(uint32_t x) {  // x mod 65535 for x < 2^32
    x = (x & 0xFFFFu) + (x >> 16);
    x = (x & 0xFFFFu) + (x >> 16);
    return x >= kFieldLimit ? x - kFieldLimit : x;
}
__device__ __forceinline__ void red_xor4(uint8_t* p, const uint4& v) {
    uint32_t* q = reinterpret_cast<uint32_t*>(p);
    asm volatile("red.global.xor.b32 [%0], %1;" ::"l"(q), "r"(v.x) : "memory");
    asm volatile("red.global.xor.b32 [%0], %1;" ::"l"(q + 1), "r"(v.y) : "memory");
    asm volatile("red.global.xor.b32 [%0], %1;" ::"l"(q + 2), "r"(v.z) : "memory");
    asm volatile("red.global.xor.b32 [%0], %1;" ::"l"(q + 3), "r"(v.w) : "memory");
}

template <int NCH, bool GEN = false, int FMAX = 1, int STAGES = kEncStages>
__device__ __forceinline__ bool encode_tile(const uint8_t* __restrict__ src, uint64_t src_stride, uint32_t S,
                                            const uint16_t* __restrict__ basis, uint32_t RG, uint32_t rg,
                                            uint32_t R, uint32_t n0, uint32_t tile_syms,
                                            uint8_t* __restrict__ rec, uint64_t rec_stride, uint8_t* smem,
                                            uint32_t& phase, uint32_t first_exp = 0, uint32_t s0 = 0,
                                            bool accumulate = false, uint32_t fold = 1, uint32_t sub_syms = 0) {
    constexpr int WARPS = kEncThreads / 32;
    constexpr int NT = FMAX * WARPS * NCH * 64;  // symbol capacity of a stage (tile_syms <= NT)
    static_assert(!GEN || WARPS == 16, "derived basis: one warp per basis product j");
    uint8_t* tabs = smem;
    uint8_t* src_st = smem + 2 * kTabBytes;
    uint8_t* bas_st = src_st + STAGES * NT * 2;
    uint64_t* bars = reinterpret_cast<uint64_t*>(bas_st + STAGES * 1024);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile_bytes = tile_syms * 2;
    const uint32_t ph = phase;
    src += (size_t)s0 * src_stride;
    if (!GEN) basis += (size_t)s0 * RG * 512;
    const uint16_t* lbase = d_logbase + s0;
    auto parity = [&](uint32_t s) { return ((ph >> (s % STAGES)) ^ (s / STAGES)) & 1u; };

    auto issue = [&](uint32_t s, int st) {
        mbar_arrive_expect_tx(&bars[st], GEN ? tile_bytes : tile_bytes + 1024);
        tma_load_1d(src_st + st * NT * 2, src + (size_t)s * src_stride + (size_t)n0 * 2, tile_bytes,
                    &bars[st]);
        if (!GEN) tma_load_1d(bas_st + st * 1024, basis + ((size_t)s * RG + rg) * 512, 1024, &bars[st]);
    };
    if (tid == 0)
        for (int st = 0; st < STAGES && (uint32_t)st < S; ++st) issue(st, st);

    // derived basis: this thread's (j = warp, row = lane) entry and its offset in a slot
    const uint32_t g_row = rg * kRowsPerGroup + (lane & (31u >> (fold >> 1)));  // replicated when folded
    // exponent mod 65535 (the coefficient is 2^(logbase * e mod 65535)), so
    // the product below stays under 2^32 for first_exp + row >= 65536 too
    const uint32_t g_exp = (first_exp + g_row) % kFieldLimit;
    const bool g_live = g_row < R;
    const uint32_t g_off = (uint32_t)((((warp & 7) * 2 + (warp >> 3)) * 32 + lane) * 2);
    auto gen_value = [&](uint32_t lb) -> uint16_t {
        if (!g_live) return 0;
        uint32_t k = mod_field(lb * g_exp) + (uint32_t)warp;
        if (k >= kFieldLimit) k -= kFieldLimit;
        return d_antilog[k];
    };
    auto gen_slot = [&](uint32_t s) { return smem_u32(bas_st) + (s & 1u) * 1024 + g_off; };
    uint16_t g_v = 0;   // basis value of slice s+2, stored at the end of iteration s
    uint32_t g_lb = 0;  // logbase of slice s+3
    if (GEN) {
        if (S > 0) sts16(gen_slot(0), gen_value(lbase[0]));
        if (S > 1) sts16(gen_slot(1), gen_value(lbase[1]));
        if (S > 2) g_v = gen_value(lbase[2]);
        if (S > 3) g_lb = lbase[3];
        __syncthreads();
    }

    // Table build: the 256 table rows are 16 blocks of 16; warp w builds
    // blocks w, w+WARPS, ...  Thread (word column wc = lane) writes the 16
    // entries v = 16*block + u of its column with a Gray-code walk over the
    // low 4 bits of v; the high 4 bits select the starting XOR.
    const uint32_t bas_u32 = smem_u32(bas_st), tab_u32 = smem_u32(tabs);
    auto build = [&](int t, int st) {
        const int p = lane & 15, h = lane >> 4;
        uint32_t b[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) b[jj] = lds32(bas_u32 + st * 1024 + (jj * 32 + h * 16 + p) * 4);
        for (int blk = warp; blk < 16; blk += WARPS) {
            uint32_t e = 0;
#pragma unroll
            for (int jj = 4; jj < 8; ++jj)
                if ((blk >> (jj - 4)) & 1) e ^= b[jj];
            const uint32_t row0 = tab_u32 + t * kTabBytes + (uint32_t)(blk * 16) * 128 + lane * 4;
            sts32(row0, e);
#pragma unroll
            for (int u = 1; u < 16; ++u) {
                e ^= b[ctz5(u)];
                sts32(row0 + (uint32_t)(u ^ (u >> 1)) * 128, e);
            }
        }
    };

    const int g = lane >> 2, k = lane & 3, odd = g & 1;
    const uint32_t offA = odd ? (64 + 16 * k) : 16 * k;
    const uint32_t offB = odd ? 16 * k : (64 + 16 * k);
    const uint32_t selA0 = odd ? 0x4441u : 0x4440u, selB0 = odd ? 0x4440u : 0x4441u;
    const uint32_t selA1 = odd ? 0x4443u : 0x4442u, selB1 = odd ? 0x4442u : 0x4443u;
    // folded: this lane's sub-tile, its symbol limit and its rows' quad
    const uint32_t sub = fold == 1 ? 0u : (uint32_t)k >> (fold == 2 ? 1 : 0);
    if (fold == 1) sub_syms = tile_syms;
    const uint32_t lim = tile_syms > sub * sub_syms ? min(sub_syms, tile_syms - sub * sub_syms) : 0u;
    const uint32_t kq = (uint32_t)k & (3u >> (fold >> 1));
    const uint32_t src_u32 = smem_u32(src_st) + sub * sub_syms * 2 + (uint32_t)(warp * NCH * 8 + g) * 16;
    // 128 = bytes per table row; read at run time so the address multiply-add
    // stays an IMAD (FMA pipe) instead of integer-ALU shift+add
    const uint32_t row_bytes = *reinterpret_cast<volatile const uint32_t*>(&d_row_bytes);

    uint32_t acc[NCH][8][4];
#pragma unroll
    for (int j = 0; j < NCH; ++j)
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[j][i][q] = 0u;

    int bad = 0;
    if (S > 0) {
        if (!mbar_wait_bounded(&bars[0], parity(0))) bad = 1;
        build(0, 0);
    }
    if (__syncthreads_or(bad)) {
        if (tid == 0)
            for (uint32_t s2 = 1; s2 < S && s2 < (uint32_t)STAGES; ++s2) mbar_wait_bounded(&bars[s2], parity(s2));
        return false;
    }

    for (uint32_t s = 0; s < S; ++s) {
        const int st = (int)(s % STAGES);
        const int t = (int)(s & 1);
        if (s + 1 < S) {
            const int st1 = (int)((s + 1) % STAGES);
            if (!mbar_wait_bounded(&bars[st1], parity(s + 1))) bad = 1;
            build(t ^ 1, GEN ? (int)((s + 1) & 1) : st1);  // GEN: the slice's slot
        }
        const uint32_t baseA = tab_u32 + t * kTabBytes + offA;
        const uint32_t baseB = tab_u32 + t * kTabBytes + offB;
        const uint32_t sbase = src_u32 + st * NT * 2;
#pragma unroll
        for (int j = 0; j < NCH; ++j) {
            if ((uint32_t)(warp * NCH * 8 + j * 8 + g) * 8 >= lim) continue;  // chunk outside the (sub-)tile
            const uint4 w4 = lds128(sbase + j * 128);
            const uint32_t ws[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const uint32_t bA = __byte_perm(ws[m], 0u, hh ? selA1 : selA0);
                    const uint32_t bB = __byte_perm(ws[m], 0u, hh ? selB1 : selB0);
                    const uint4 A = lds128(mad1(bA, row_bytes, baseA));
                    const uint4 B = lds128(mad1(bB, row_bytes, baseB));
                    const int i = 2 * m + hh;
                    acc[j][i][0] ^= A.x ^ B.x;
                    acc[j][i][1] ^= A.y ^ B.y;
                    acc[j][i][2] ^= A.z ^ B.z;
                    acc[j][i][3] ^= A.w ^ B.w;
                }
            }
        }
        if (GEN && s + 2 < S) {  // slot s&1 was last read by build(s), before the previous barrier
            sts16(gen_slot(s), g_v);
            if (s + 3 < S) {
                g_v = gen_value(g_lb);
                if (s + 4 < S) g_lb = lbase[s + 4];
            }
        }
        if (__syncthreads_or(bad)) {
            if (tid == 0)  // drain copies still in flight before the CTA's shared memory goes away
                for (uint32_t s2 = s + 1; s2 < S && s2 < s + STAGES; ++s2)
                    mbar_wait_bounded(&bars[s2 % STAGES], parity(s2));
            return false;
        }
        if (tid == 0 && s + STAGES < S) issue(s + STAGES, st);
    }
    // stage st was used ceil((S - st) / STAGES) times: flip its parity if odd
    uint32_t flip = 0;
#pragma unroll
    for (int st = 0; st < STAGES; ++st)
        if ((uint32_t)st < S && (((S - 1 - st) / STAGES) & 1u) == 0) flip |= 1u << st;
    phase = ph ^ flip;

    // Epilogue: transpose (symbol-major, row pairs packed) into row-major
    // 16-byte runs of 8 symbols and store.
#pragma unroll
    for (int j = 0; j < NCH; ++j) {
        const uint32_t chunk = (uint32_t)(warp * NCH * 8 + j * 8 + g);
        const uint32_t n = n0 + sub * sub_syms + chunk * 8;
        if (chunk * 8 < lim) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t re = rg * kRowsPerGroup + 8 * kq + 2 * q;
                uint4 we, wo;
                we.x = __byte_perm(acc[j][0][q], acc[j][1][q], 0x5410);
                we.y = __byte_perm(acc[j][2][q], acc[j][3][q], 0x5410);
                we.z = __byte_perm(acc[j][4][q], acc[j][5][q], 0x5410);
                we.w = __byte_perm(acc[j][6][q], acc[j][7][q], 0x5410);
                wo.x = __byte_perm(acc[j][0][q], acc[j][1][q], 0x7632);
                wo.y = __byte_perm(acc[j][2][q], acc[j][3][q], 0x7632);
                wo.z = __byte_perm(acc[j][4][q], acc[j][5][q], 0x7632);
                wo.w = __byte_perm(acc[j][6][q], acc[j][7][q], 0x7632);
                uint8_t* pe = rec + (size_t)re * rec_stride + (size_t)n * 2;
                uint8_t* po = pe + rec_stride;
                if (accumulate) {
                    if (re < R) red_xor4(pe, we);
                    if (re + 1 < R) red_xor4(po, wo);
                } else {
                    if (re < R) *reinterpret_cast<uint4*>(pe) = we;
                    if (re + 1 < R) *reinterpret_cast<uint4*>(po) = wo;
                }
            }
        }
    }
    return true;
}

// tail_fold: fold of the last row group (1, 2, 4); its CTA for tile t covers
// tail_fold adjacent tiles, so the grid's tail-group CTAs past the band exit.
template <int NCH, bool GEN>
__global__ void __launch_bounds__(kEncThreads, 1)
    encode_lut_kernel(const uint8_t* __restrict__ src, uint64_t src_stride, uint32_t S,
                      const uint16_t* __restrict__ basis, uint32_t RG, uint32_t R, uint32_t sym_begin,
                      uint32_t sym_end, uint32_t TS, uint8_t* __restrict__ rec, uint64_t rec_stride,
                      uint32_t first_exp, uint32_t tail_fold, int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + encode_bars_offset<NCH, 4>());
    const uint32_t tile = blockIdx.x / RG, rg = blockIdx.x % RG;
    const uint32_t fold = rg + 1 == RG ? tail_fold : 1u;
    const uint32_t n0 = sym_begin + tile * TS * fold;
    if (n0 >= sym_end) return;  // uniform: empty tile at the end of a band
    if (threadIdx.x == 0) {
        for (int st = 0; st < kEncStages; ++st) mbar_init(&bars[st], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    if (!encode_tile<NCH, GEN, 4>(src, src_stride, S, basis, RG, rg, R, n0, min(TS * fold, sym_end - n0), rec,
                                  rec_stride, smem, phase, first_exp, 0, false, fold, TS) &&
        threadIdx.x == 0)
        atomicOr(err, 1);
}

// ---------------------------------------------------------------------------
// Single-coefficient multiply-XOR over arbitrary buffers (the kernel-level
// seam gf_mul_xor_dispatch, src/galois_simd.rs:640-643).  Byte tables in
// shared memory (CoeffTables, src/galois_simd.rs:45-54).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint16_t dev_gf_mul(uint32_t a, uint32_t b) {
    if (a == 0 || b == 0) return 0;
    uint32_t s = (uint32_t)d_log[a] + d_log[b];
    if (s >= kFieldLimit) s -= kFieldLimit;
    return d_antilog[s];
}

__global__ void gf_mul_xor_kernel(uint16_t coeff, const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                                  uint64_t nsym) {
    __shared__ uint16_t lo[256], hi[256];
    for (int t = threadIdx.x; t < 256; t += blockDim.x) {
        lo[t] = dev_gf_mul(coeff, (uint32_t)t);
        hi[t] = dev_gf_mul(coeff, (uint32_t)t << 8);
    }
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nsym;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)in[2 * i] | ((uint32_t)in[2 * i + 1] << 8);
        const uint32_t p = lo[x & 0xFF] ^ hi[x >> 8];
        out[2 * i] ^= (uint8_t)p;
        out[2 * i + 1] ^= (uint8_t)(p >> 8);
    }
}

// ---------------------------------------------------------------------------
// MD5 (RFC 1321), one message stream per thread.  The message is
// prefix words ‖ data bytes; the prefix length is a multiple of 4 and data is
// 4-byte aligned.  Whole 64-byte blocks inside the data run a software-
// pipelined loop (next block's loads issued before the current compress).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t rotl32(uint32_t x, int s) { return __funnelshift_l(x, x, s); }

#define P2G_F(x, y, z) ((z) ^ ((x) & ((y) ^ (z))))
#define P2G_G(x, y, z) ((y) ^ ((z) & ((x) ^ (y))))
#define P2G_H(x, y, z) ((x) ^ (y) ^ (z))
#define P2G_I(x, y, z) ((y) ^ ((x) | ~(z)))
// a + x + t does not depend on the previous step's output (b), so it is
// formed first; the chain through b is then round function -> add ->
// rotate -> add.
#define P2G_STEP(f, a, b, c, d, x, t, s)                    \
    {                                                       \
        const uint32_t _axt = (a) + ((x) + (t));            \
        (a) = rotl32(_axt + f((b), (c), (d)), (s)) + (b);   \
    }

__device__ __forceinline__ void md5_compress(uint32_t st[4], const uint32_t m[16]) {
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
    P2G_STEP(P2G_F, a, b, c, d, m[0], 0xd76aa478u, 7);
    P2G_STEP(P2G_F, d, a, b, c, m[1], 0xe8c7b756u, 12);
    P2G_STEP(P2G_F, c, d, a, b, m[2], 0x242070dbu, 17);
    P2G_STEP(P2G_F, b, c, d, a, m[3], 0xc1bdceeeu, 22);
    P2G_STEP(P2G_F, a, b, c, d, m[4], 0xf57c0fafu, 7);
    P2G_STEP(P2G_F, d, a, b, c, m[5], 0x4787c62au, 12);
    P2G_STEP(P2G_F, c, d, a, b, m[6], 0xa8304613u, 17);
    P2G_STEP(P2G_F, b, c, d, a, m[7], 0xfd469501u, 22);
    P2G_STEP(P2G_F, a, b, c, d, m[8], 0x698098d8u, 7);
    P2G_STEP(P2G_F, d, a, b, c, m[9], 0x8b44f7afu, 12);
    P2G_STEP(P2G_F, c, d, a, b, m[10], 0xffff5bb1u, 17);
    P2G_STEP(P2G_F, b, c, d, a, m[11], 0x895cd7beu, 22);
    P2G_STEP(P2G_F, a, b, c, d, m[12], 0x6b901122u, 7);
    P2G_STEP(P2G_F, d, a, b, c, m[13], 0xfd987193u, 12);
    P2G_STEP(P2G_F, c, d, a, b, m[14], 0xa679438eu, 17);
    P2G_STEP(P2G_F, b, c, d, a, m[15], 0x49b40821u, 22);

    P2G_STEP(P2G_G, a, b, c, d, m[1], 0xf61e2562u, 5);
    P2G_STEP(P2G_G, d, a, b, c, m[6], 0xc040b340u, 9);
    P2G_STEP(P2G_G, c, d, a, b, m[11], 0x265e5a51u, 14);
    P2G_STEP(P2G_G, b, c, d, a, m[0], 0xe9b6c7aau, 20);
    P2G_STEP(P2G_G, a, b, c, d, m[5], 0xd62f105du, 5);
    P2G_STEP(P2G_G, d, a, b, c, m[10], 0x02441453u, 9);
    P2G_STEP(P2G_G, c, d, a, b, m[15], 0xd8a1e681u, 14);
    P2G_STEP(P2G_G, b, c, d, a, m[4], 0xe7d3fbc8u, 20);
    P2G_STEP(P2G_G, a, b, c, d, m[9], 0x21e1cde6u, 5);
    P2G_STEP(P2G_G, d, a, b, c, m[14], 0xc33707d6u, 9);
    P2G_STEP(P2G_G, c, d, a, b, m[3], 0xf4d50d87u, 14);
    P2G_STEP(P2G_G, b, c, d, a, m[8], 0x455a14edu, 20);
    P2G_STEP(P2G_G, a, b, c, d, m[13], 0xa9e3e905u, 5);
    P2G_STEP(P2G_G, d, a, b, c, m[2], 0xfcefa3f8u, 9);
    P2G_STEP(P2G_G, c, d, a, b, m[7], 0x676f02d9u, 14);
    P2G_STEP(P2G_G, b, c, d, a, m[12], 0x8d2a4c8au, 20);

    P2G_STEP(P2G_H, a, b, c, d, m[5], 0xfffa3942u, 4);
    P2G_STEP(P2G_H, d, a, b, c, m[8], 0x8771f681u, 11);
    P2G_STEP(P2G_H, c, d, a, b, m[11], 0x6d9d6122u, 16);
    P2G_STEP(P2G_H, b, c, d, a, m[14], 0xfde5380cu, 23);
    P2G_STEP(P2G_H, a, b, c, d, m[1], 0xa4beea44u, 4);
    P2G_STEP(P2G_H, d, a, b, c, m[4], 0x4bdecfa9u, 11);
    P2G_STEP(P2G_H, c, d, a, b, m[7], 0xf6bb4b60u, 16);
    P2G_STEP(P2G_H, b, c, d, a, m[10], 0xbebfbc70u, 23);
    P2G_STEP(P2G_H, a, b, c, d, m[13], 0x289b7ec6u, 4);
    P2G_STEP(P2G_H, d, a, b, c, m[0], 0xeaa127fau, 11);
    P2G_STEP(P2G_H, c, d, a, b, m[3], 0xd4ef3085u, 16);
    P2G_STEP(P2G_H, b, c, d, a, m[6], 0x04881d05u, 23);
    P2G_STEP(P2G_H, a, b, c, d, m[9], 0xd9d4d039u, 4);
    P2G_STEP(P2G_H, d, a, b, c, m[12], 0xe6db99e5u, 11);
    P2G_STEP(P2G_H, c, d, a, b, m[15], 0x1fa27cf8u, 16);
    P2G_STEP(P2G_H, b, c, d, a, m[2], 0xc4ac5665u, 23);

    P2G_STEP(P2G_I, a, b, c, d, m[0], 0xf4292244u, 6);
    P2G_STEP(P2G_I, d, a, b, c, m[7], 0x432aff97u, 10);
    P2G_STEP(P2G_I, c, d, a, b, m[14], 0xab9423a7u, 15);
    P2G_STEP(P2G_I, b, c, d, a, m[5], 0xfc93a039u, 21);
    P2G_STEP(P2G_I, a, b, c, d, m[12], 0x655b59c3u, 6);
    P2G_STEP(P2G_I, d, a, b, c, m[3], 0x8f0ccc92u, 10);
    P2G_STEP(P2G_I, c, d, a, b, m[10], 0xffeff47du, 15);
    P2G_STEP(P2G_I, b, c, d, a, m[1], 0x85845dd1u, 21);
    P2G_STEP(P2G_I, a, b, c, d, m[8], 0x6fa87e4fu, 6);
    P2G_STEP(P2G_I, d, a, b, c, m[15], 0xfe2ce6e0u, 10);
    P2G_STEP(P2G_I, c, d, a, b, m[6], 0xa3014314u, 15);
    P2G_STEP(P2G_I, b, c, d, a, m[13], 0x4e0811a1u, 21);
    P2G_STEP(P2G_I, a, b, c, d, m[4], 0xf7537e82u, 6);
    P2G_STEP(P2G_I, d, a, b, c, m[11], 0xbd3af235u, 10);
    P2G_STEP(P2G_I, c, d, a, b, m[2], 0x2ad7d2bbu, 15);
    P2G_STEP(P2G_I, b, c, d, a, m[9], 0xeb86d391u, 21);
    st[0] += a;
    st[1] += b;
    st[2] += c;
    st[3] += d;
}

// CG: load through L2 only (data written earlier in the same launch by
// other CTAs or by this one); otherwise through the read-only path.
template <bool VEC, bool CG = false>
__device__ __forceinline__ void md5_load_block(uint32_t m[16], const uint8_t* p) {
    if (VEC) {
        const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint4 v = CG ? __ldcg(q + i) : __ldg(q + i);
            m[4 * i] = v.x;
            m[4 * i + 1] = v.y;
            m[4 * i + 2] = v.z;
            m[4 * i + 3] = v.w;
        }
    } else {
        const uint32_t* q = reinterpret_cast<const uint32_t*>(p);
#pragma unroll
        for (int i = 0; i < 16; ++i) m[i] = CG ? __ldcg(q + i) : __ldg(q + i);
    }
}

// Word at stream byte offset q (multiple of 4) of prefix ‖ data ‖ MD5 padding.
__device__ uint32_t md5_stream_word(const uint32_t* pre, uint32_t pre_bytes, const uint8_t* data,
                                    uint64_t len, uint64_t total, uint64_t last_start, uint64_t q) {
    if (q == last_start + 56) return (uint32_t)(total << 3);
    if (q == last_start + 60) return (uint32_t)(total >> 29);
    if (q < pre_bytes) return pre[q >> 2];
    const uint64_t d = q - pre_bytes;
    // L2-only loads: the data may have been written earlier in the same launch
    if (d + 4 <= len) return __ldcg(reinterpret_cast<const uint32_t*>(data + d));
    uint32_t w = 0;
    for (int t = 0; t < 4; ++t) {
        const uint64_t pos = d + t;
        const uint32_t byte = pos < len ? (uint32_t)__ldcg(data + pos) : (pos == len ? 0x80u : 0u);
        w |= byte << (8 * t);
    }
    return w;
}

// Blocks [b_from, b_to) of the padded message prefix ‖ data.
template <bool VEC, bool CG = false>
__device__ void md5_range(uint32_t st[4], const uint32_t* pre, uint32_t pre_bytes, const uint8_t* data, uint64_t len,
                          uint64_t b_from, uint64_t b_to) {
    const uint64_t total = pre_bytes + len;
    const uint64_t nblocks = (total + 8) / 64 + 1;
    const uint64_t last_start = (nblocks - 1) * 64;
    const uint64_t fb0 = (pre_bytes + 63) / 64;  // first block wholly after the prefix
    const uint64_t fb1 = total / 64;             // blocks below this hold no padding
    if (b_to > nblocks) b_to = nblocks;
    uint64_t b = b_from;
    uint32_t m[16];
    for (; b < fb0 && b < b_to; ++b) {
#pragma unroll
        for (int i = 0; i < 16; ++i) m[i] = md5_stream_word(pre, pre_bytes, data, len, total, last_start, 64 * b + 4 * i);
        md5_compress(st, m);
    }
    const uint64_t fast_end = fb1 < b_to ? fb1 : b_to;
    if (b < fast_end) {
        md5_load_block<VEC, CG>(m, data + 64 * b - pre_bytes);
        for (; b < fast_end; ++b) {
            uint32_t nx[16];
            const uint64_t nb = b + 1 < fast_end ? b + 1 : b;
            md5_load_block<VEC, CG>(nx, data + 64 * nb - pre_bytes);
            md5_compress(st, m);
#pragma unroll
            for (int i = 0; i < 16; ++i) m[i] = nx[i];
        }
    }
    for (; b < b_to; ++b) {
#pragma unroll
        for (int i = 0; i < 16; ++i) m[i] = md5_stream_word(pre, pre_bytes, data, len, total, last_start, 64 * b + 4 * i);
        md5_compress(st, m);
    }
}

__device__ __forceinline__ void md5_init(uint32_t st[4]) {
    st[0] = 0x67452301u;
    st[1] = 0xefcdab89u;
    st[2] = 0x98badcfeu;
    st[3] = 0x10325476u;
}

template <bool VEC>
__device__ void md5_stream(uint32_t st[4], const uint32_t* pre, uint32_t pre_bytes, const uint8_t* data,
                           uint64_t len) {
    md5_init(st);
    md5_range<VEC>(st, pre, pre_bytes, data, len, 0, ~0ull);
}

// ---------------------------------------------------------------------------
// Staged MD5 streams.  With 32 lanes of a warp each hashing a different
// stream, direct global loads leave every block waiting on 32 scattered
// cache lines.  Instead each lane pulls its stream through a private ring of
// kRingUnits 64-byte units in shared memory with cp.async, kRingAhead units
// ahead of the block being compressed, and reads message words back with
// 128-bit shared loads.  PW = prefix words (the message is PW prefix words
// ‖ data); data must be 16-byte aligned when VEC (else 4-byte copies).
// Blocks that contain prefix words, padding, or data past the last whole
// copy unit take the direct (generic) path.
// ---------------------------------------------------------------------------
constexpr int kHashThreads = 256;  // 8 warps: two MD5 warps per SM sub-partition keep full chain speed
constexpr int kRingUnits = 8;
constexpr int kRingAhead = 4;
constexpr int kRingLaneBytes = kRingUnits * 64 + 16;  // +16: lanes land on distinct bank groups

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int PW, bool VEC, int UNITS = kRingUnits, int AHEAD = kRingAhead>
__device__ void md5_range_ring(uint32_t st[4], const uint32_t* pre, const uint8_t* data, uint64_t len,
                               uint64_t b_from, uint64_t b_to, uint32_t ring) {
    constexpr uint32_t pre_bytes = 4 * PW;
    constexpr int SH = (4 - (PW & 3)) & 3;  // word offset of a block's first word in its aligned quad
    constexpr int NQ = SH ? 5 : 4;          // quads touched per block
    const uint64_t total = pre_bytes + len;
    const uint64_t nblocks = (total + 8) / 64 + 1;
    const uint64_t last_start = (nblocks - 1) * 64;
    if (b_to > nblocks) b_to = nblocks;
    // whole 64-byte units that can go through the ring
    const uint64_t fetch_bytes = VEC ? (len & ~15ull) : (len & ~3ull);
    const uint64_t n_units = fetch_bytes / 64;
    // ring-eligible blocks: no prefix word, all data words inside whole units
    const uint64_t rb0 = (pre_bytes + 63) / 64;
    const uint64_t rb1 = n_units * 16 >= 16 - PW ? (n_units * 16 + PW) / 16 : 0;  // blocks b with 16b+16-PW <= 16*n_units
    uint64_t b = b_from;
    uint32_t m[16];
    auto generic = [&](uint64_t blk) {
#pragma unroll
        for (int i = 0; i < 16; ++i) m[i] = md5_stream_word(pre, pre_bytes, data, len, total, last_start, 64 * blk + 4 * i);
        md5_compress(st, m);
    };
    for (; b < b_to && (b < rb0 || b >= rb1); ++b) generic(b);
    const uint64_t fast_end = rb1 < b_to ? rb1 : b_to;
    if (b < fast_end) {
        auto fetch = [&](uint64_t u, uint32_t slot) {  // one unit = one commit group (possibly empty)
            if (u < n_units) {
                const uint8_t* g = data + 64 * u;
                const uint32_t d = ring + slot * 64;
                if (VEC) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) cp_async16(d + 16 * q, g + 16 * q);
                } else {
#pragma unroll
                    for (int q = 0; q < 16; ++q) cp_async4(d + 4 * q, g + 4 * q);
                }
            }
            cp_async_commit();
        };
        // units of block b: [lo(b), hi(b)] with hi(b) = floor((16b + 15 - PW) / 16)
        const uint64_t first_w = 16 * b - PW;
        const uint64_t u_lo = first_w / 16;
        const uint64_t u_hi0 = (first_w + 15) / 16;
        for (uint64_t u = u_lo; u < u_hi0 + AHEAD; ++u) fetch(u, (uint32_t)(u % UNITS));
        // Each block moves the ring by one unit (16 words): the next unit to
        // fetch, its slot and the slot of the block's first aligned quad are
        // stepped as 32-bit counters, so no 64-bit remainder (the ring need
        // not be a power of two) sits between one compress and the next.
        constexpr uint32_t RW = 16 * UNITS;  // ring size in words
        uint64_t u_next = u_hi0 + AHEAD;
        uint32_t f_slot = (uint32_t)(u_next % UNITS);
        uint32_t w_slot = (uint32_t)(((16 * b - PW) & ~3ull) % RW);
        for (; b < fast_end; ++b) {
            fetch(u_next, f_slot);
            ++u_next;
            f_slot = f_slot + 1 == (uint32_t)UNITS ? 0u : f_slot + 1;
            cp_async_wait<AHEAD>();
            uint32_t q[NQ * 4];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                uint32_t widx = w_slot + 4 * i;
                if (widx >= RW) widx -= RW;
                const uint4 v = lds128(ring + widx * 4);
                q[4 * i] = v.x;
                q[4 * i + 1] = v.y;
                q[4 * i + 2] = v.z;
                q[4 * i + 3] = v.w;
            }
            w_slot = w_slot + 16 >= RW ? w_slot + 16 - RW : w_slot + 16;
#pragma unroll
            for (int i = 0; i < 16; ++i) m[i] = q[SH + i];
            md5_compress(st, m);
        }
        cp_async_wait<0>();
    }
    for (; b < b_to; ++b) generic(b);
}

template <bool VEC>
__global__ void __launch_bounds__(kHashThreads) md5_slices_kernel(const uint8_t* __restrict__ src, uint64_t stride,
                                                                  uint32_t count, uint64_t slice_size,
                                                                  p2g_slice_checksum* __restrict__ out) {
    extern __shared__ __align__(16) uint8_t ring[];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t st[4];
    md5_init(st);
    md5_range_ring<0, VEC>(st, nullptr, src + (size_t)i * stride, slice_size, 0, ~0ull,
                           smem_u32(ring) + threadIdx.x * kRingLaneBytes);
    uint32_t* o = reinterpret_cast<uint32_t*>(&out[i]);
    o[0] = st[0];
    o[1] = st[1];
    o[2] = st[2];
    o[3] = st[3];
}

template <bool VEC>
__global__ void __launch_bounds__(kHashThreads) md5_files_kernel(const uint8_t* __restrict__ base,
                                                                 const FileSpan* __restrict__ spans, uint32_t n,
                                                                 uint8_t* __restrict__ out16) {
    extern __shared__ __align__(16) uint8_t ring[];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t st[4];
    const FileSpan sp = spans[i];
    md5_init(st);
    md5_range_ring<0, VEC>(st, nullptr, base + sp.offset, sp.length, 0, ~0ull,
                           smem_u32(ring) + threadIdx.x * kRingLaneBytes);
    uint32_t* o = reinterpret_cast<uint32_t*>(out16 + 16 * (size_t)i);
    o[0] = st[0];
    o[1] = st[1];
    o[2] = st[2];
    o[3] = st[3];
}

struct RecvPrefix {
    uint32_t w[8];  // set_id ‖ "PAR 2.0\0RecvSlic"
};

template <bool VEC>
__global__ void __launch_bounds__(kHashThreads) md5_recovery_kernel(const uint8_t* __restrict__ rec, uint64_t stride, uint32_t count,
                                    uint64_t slice_size, RecvPrefix pfx, uint32_t first_exp,
                                    uint8_t* __restrict__ out16) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    uint32_t pre[9];
#pragma unroll
    for (int i = 0; i < 8; ++i) pre[i] = pfx.w[i];
    pre[8] = first_exp + r;  // exponent as le32 (src/packet/recovery.rs:15)
    extern __shared__ __align__(16) uint8_t ring[];
    uint32_t st[4];
    md5_init(st);
    md5_range_ring<9, VEC>(st, pre, rec + (size_t)r * stride, slice_size, 0, ~0ull,
                            smem_u32(ring) + threadIdx.x * kRingLaneBytes);
    uint32_t* o = reinterpret_cast<uint32_t*>(out16 + 16 * (size_t)r);
    o[0] = st[0];
    o[1] = st[1];
    o[2] = st[2];
    o[3] = st[3];
}

// Continuation form: blocks [b_from, b_to) of each row's packet message,
// with the chain state kept in `state` (4 words per row) between calls.
// b_from == 0 starts a chain; `final` writes the digest instead of the state.
template <bool VEC>
__global__ void __launch_bounds__(kHashThreads) md5_recovery_range_kernel(const uint8_t* __restrict__ rec, uint64_t stride, uint32_t count,
                                          uint64_t slice_size, RecvPrefix pfx, uint32_t first_exp,
                                          uint32_t* __restrict__ state, uint64_t b_from, uint64_t b_to, int final,
                                          uint8_t* __restrict__ out16) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    uint32_t pre[9];
#pragma unroll
    for (int i = 0; i < 8; ++i) pre[i] = pfx.w[i];
    pre[8] = first_exp + r;
    extern __shared__ __align__(16) uint8_t ring[];
    uint32_t st[4];
    if (b_from == 0) {
        md5_init(st);
    } else {
        const uint4 v = reinterpret_cast<const uint4*>(state)[r];
        st[0] = v.x;
        st[1] = v.y;
        st[2] = v.z;
        st[3] = v.w;
    }
    md5_range_ring<9, VEC>(st, pre, rec + (size_t)r * stride, slice_size, b_from, b_to,
                            smem_u32(ring) + threadIdx.x * kRingLaneBytes);
    if (final) {
        uint32_t* o = reinterpret_cast<uint32_t*>(out16 + 16 * (size_t)r);
        o[0] = st[0];
        o[1] = st[1];
        o[2] = st[2];
        o[3] = st[3];
    } else {
        reinterpret_cast<uint4*>(state)[r] = make_uint4(st[0], st[1], st[2], st[3]);
    }
}

// ---------------------------------------------------------------------------
// CRC-32/IEEE (reflected polynomial 0xEDB88320, init and final xor
// 0xFFFFFFFF), one warp per slice.  Lane l runs the table-driven register
// update (four 256-entry tables, four bytes per step) over its contiguous
// chunk from register value 0 (lane 0 from 0xFFFFFFFF); the chunk results
// are then moved to the end of the slice by multiplying with x^(8*bytes
// after the chunk) mod P and XORed together.  In the reflected register
// bit 31 is the x^0 coefficient, so "times x" is a right shift that folds
// the polynomial back in when bit 0 falls off.
// ---------------------------------------------------------------------------
constexpr uint32_t kCrcPoly = 0xEDB88320u;

__device__ __forceinline__ uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
    uint32_t prod = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        if (a & (0x80000000u >> i)) prod ^= b;
        b = (b >> 1) ^ ((b & 1u) ? kCrcPoly : 0u);
    }
    return prod;
}

__device__ uint32_t x_pow_8n(uint64_t n) {
    uint32_t result = 0x80000000u;  // x^0
    uint32_t base = 0x00800000u;    // x^8
    while (n) {
        if (n & 1) result = gf2_mulmod(result, base);
        base = gf2_mulmod(base, base);
        n >>= 1;
    }
    return result;
}

// Slicing-by-4 tables T[t][b] (T[0] the byte table) into shared memory,
// built by all threads of the block (contains __syncthreads).
__device__ __forceinline__ void crc_tables_build(uint32_t (*T)[256]) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t c = (uint32_t)i;
        for (int b = 0; b < 8; ++b) c = (c >> 1) ^ ((c & 1u) ? kCrcPoly : 0u);
        T[0][i] = c;
    }
    __syncthreads();
    for (int t = 1; t < 4; ++t) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) {
            const uint32_t v = T[t - 1][i];
            T[t][i] = (v >> 8) ^ T[0][v & 0xFF];
        }
        __syncthreads();
    }
}

// Lane chunk of a slice of W = slice_size/4 words: [start, end) words, and
// K = x^(8 * bytes after the chunk) mod P that moves its partial CRC to the
// end of the slice.
struct CrcLane {
    uint64_t start, end;
    uint32_t K;
};
template <bool VEC>
__device__ __forceinline__ CrcLane crc_lane(uint64_t slice_size, int lane) {
    const uint64_t W = slice_size / 4;
    uint64_t cw = (W + 31) / 32;
    if (VEC) cw = (cw + 3) & ~3ull;
    CrcLane c;
    c.start = min((uint64_t)lane * cw, W);
    c.end = min(c.start + cw, W);
    c.K = x_pow_8n(slice_size - c.end * 4);
    return c;
}

// CRC32 of one slice by one warp (all 32 lanes call it with the same p).
template <bool VEC>
__device__ __forceinline__ uint32_t crc_slice_warp(const uint32_t* __restrict__ p, const CrcLane& cl, int lane,
                                                   const uint32_t (*T)[256]) {
    uint32_t c = lane == 0 ? 0xFFFFFFFFu : 0u;
    uint64_t w = cl.start;
    if (VEC && w + 4 <= cl.end) {
        // the next 16 bytes are loaded before the current 16 are folded in,
        // so a lane has two loads in flight instead of one
        uint4 nxt = __ldg(reinterpret_cast<const uint4*>(p + w));
        for (; w + 4 <= cl.end; w += 4) {
            const uint4 v = nxt;
            if (w + 8 <= cl.end) nxt = __ldg(reinterpret_cast<const uint4*>(p + w + 4));
            const uint32_t vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                c ^= vv[q];
                c = T[3][c & 0xFF] ^ T[2][(c >> 8) & 0xFF] ^ T[1][(c >> 16) & 0xFF] ^ T[0][c >> 24];
            }
        }
    }
    for (; w < cl.end; ++w) {
        c ^= __ldg(p + w);
        c = T[3][c & 0xFF] ^ T[2][(c >> 8) & 0xFF] ^ T[1][(c >> 16) & 0xFF] ^ T[0][c >> 24];
    }
    c = gf2_mulmod(c, cl.K);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c ^= __shfl_xor_sync(0xFFFFFFFFu, c, o);
    return c ^ 0xFFFFFFFFu;
}

template <bool VEC>
__global__ void __launch_bounds__(64) crc_slices_kernel(const uint8_t* __restrict__ src, uint64_t stride,
                                                         uint32_t count, uint64_t slice_size,
                                                         p2g_slice_checksum* __restrict__ out) {
    __shared__ uint32_t T[4][256];
    crc_tables_build(T);
    const int lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    const CrcLane cl = crc_lane<VEC>(slice_size, lane);
    for (uint64_t s = (uint64_t)blockIdx.x * wpb + (threadIdx.x >> 5); s < count; s += (uint64_t)gridDim.x * wpb) {
        const uint32_t c = crc_slice_warp<VEC>(reinterpret_cast<const uint32_t*>(src + (size_t)s * stride), cl, lane, T);
        if (lane == 0) out[s].crc32 = c;
    }
}

__global__ void realign_kernel(const uint8_t* __restrict__ src, uint64_t src_stride, uint8_t* __restrict__ dst,
                               uint64_t dst_stride, uint32_t count, uint64_t slice_size) {
    const uint64_t wps = slice_size / 4;
    const uint64_t total = wps * count;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t s = i / wps, w = i % wps;
        reinterpret_cast<uint32_t*>(dst + s * dst_stride)[w] =
            reinterpret_cast<const uint32_t*>(src + s * src_stride)[w];
    }
}

// Upload of page-locked host inputs in one launch: segment k copies len
// bytes from seg[3k] (a host address the device reads directly, over the
// bus) to seg[3k+1] and then zeroes pad bytes after them (the tail of a
// file's last slice).  One CTA per segment at a time; 16-byte accesses when
// both ends are 16-byte aligned, else bytes.  seg[3k+2] = len | pad << 40.
__global__ void gather_host_kernel(const uint64_t* __restrict__ seg, uint32_t n_seg) {
    for (uint32_t k = blockIdx.x; k < n_seg; k += gridDim.x) {
        const uint8_t* s = reinterpret_cast<const uint8_t*>(seg[3 * k]);
        uint8_t* d = reinterpret_cast<uint8_t*>(seg[3 * k + 1]);
        const uint64_t len = seg[3 * k + 2] & ((1ull << 40) - 1), pad = seg[3 * k + 2] >> 40;
        uint64_t done = 0;
        if ((((uintptr_t)s | (uintptr_t)d) & 15) == 0) {
            const uint64_t n16 = len / 16;
            for (uint64_t i = threadIdx.x; i < n16; i += blockDim.x)
                reinterpret_cast<uint4*>(d)[i] = reinterpret_cast<const uint4*>(s)[i];
            done = n16 * 16;
        }
        for (uint64_t i = done + threadIdx.x; i < len; i += blockDim.x) d[i] = s[i];
        for (uint64_t i = threadIdx.x; i < pad; i += blockDim.x) d[len + i] = 0;
    }
}

// ---------------------------------------------------------------------------
// Batched create.  One CTA per SM pops work items off a device queue until
// it is empty.  Items of one job never wait for one another: the CTA whose
// encode item completes a job (counted with an atomic after a release fence)
// runs that job's finish step itself, so the launch has no inter-CTA waits.
//
// Shared memory: the encode region (tables, TMA ring, mbarriers), a cp.async
// ring of kBatchRingLane bytes for each of the kHashThreads MD5 lanes, the
// CRC32 tables and a few words of per-CTA state.
// ---------------------------------------------------------------------------
// The persistent kernel runs its encode items on a 3-deep TMA ring (3 slices
// of lead, ~4.5 us, hide any load) so that its MD5 streams get a 6-unit ring
// (4 units ahead, like the dedicated hash kernels) beside an encode stage
// that holds a folded tail item (4 tiles).
constexpr int kBatchEncStages = 3;
constexpr size_t kBatchEncBytes = (encode_smem_bytes<kEncChunks, 4, kBatchEncStages>() + 15) / 16 * 16;
constexpr int kBatchRingUnits = 6;
constexpr int kBatchRingAhead = 4;
constexpr int kBatchRingLane = kBatchRingUnits * 64 + 16;
constexpr size_t kBatchRingBytes = (size_t)kHashThreads * kBatchRingLane;
// Tensor-core items reuse the encode region and the MD5 rings for their
// operand and input rings; their barriers, the TMEM address, an abort flag,
// the pipeline state and the G^-1 tables live past the other regions, so
// they persist across items.  The MD5 rings start past the tensor-core input
// stages: a tile's producer issues the next tile's first input stages before
// the CTA has counted the tile's band, and the packet-MD5 chains that a band
// completes run on the rings meanwhile (the rings then overlap only operand
// stages, which are idle between tiles).
constexpr size_t kBatchRingOff = ((kBatchEncBytes > (size_t)mma::kInStages * mma::kInStageBytes
                                       ? kBatchEncBytes
                                       : (size_t)mma::kInStages * mma::kInStageBytes) + 15) / 16 * 16;
constexpr size_t kBatchMmaBarsOff = kBatchRingOff + kBatchRingBytes + 4 * 256 * 4 + 64;
// the G^-1 tables of tensor-core items, copied once per launch, after the
// pipeline state words
constexpr size_t kBatchGinvOff = kBatchMmaBarsOff + mma::kBarBytes + 32;
// the next tile a tensor-core tile's producer claimed (one mma::Tile)
constexpr size_t kBatchNextTileOff = (kBatchGinvOff + mma::kGinvBytes + 15) / 16 * 16;
constexpr size_t kBatchSmem = kBatchNextTileOff + 64;
static_assert(sizeof(mma::Tile) <= 64 && kBatchNextTileOff % 16 == 0, "next-tile slot");
static_assert(kBatchEncBytes % 16 == 0 && kBatchRingOff % 16 == 0, "MD5 rings must start 16-byte aligned");
static_assert(mma::kRingBytes <= kBatchRingOff + kBatchRingBytes,
              "tensor-core rings fit the encode region and the MD5 rings");
static_assert(kBatchMmaBarsOff % 8 == 0 && kBatchSmem <= 227 * 1024, "batch shared memory");
size_t batch_smem_bytes() { return kBatchSmem; }

// The tile of a tensor-core item.
__device__ __forceinline__ mma::Tile batch_mma_tile_of(const BatchJob& J, const BatchItem& it) {
    mma::Tile T;
    T.src_map = &J.src_map;
    T.aimg = J.aimg;
    T.rec = J.rec;
    T.rec_stride = J.rec_stride;
    T.s0 = it.s0;
    T.sn = it.sn ? it.sn : J.S - it.s0;
    T.ksteps = J.ksteps;
    T.R = J.R;
    T.r0 = ((it.kind_rg >> 8) & 0xFFFFu) * kMmaTileRows;
    T.n0 = it.a;
    T.syms = it.b & 0xFFFFu;
    T.accumulate = (it.kind_rg & kItemAccumulate) ? 1u : 0u;
    return T;
}

// One tensor-core item of the batch kernel, all threads: 14 operand-building
// warps (warps 2..15).  Kept out of line, with its pipeline state in shared
// memory (words [2..6] past the barriers: operand stages, tiles, drains,
// input stages, stages issued ahead), so that it adds no registers to the
// other item kinds.
//
// The CTA's next item is claimed from the queue here, by the producer thread
// once it has issued this tile's last input stage (a few K-steps before the
// tile ends, about when the CTA would otherwise claim it); its index goes to
// *held (shared memory, read by every thread after this returns) and its
// first input stages are issued at once.  Nothing is claimed ahead
// (held = kNoHeldItem) once the error flag is set, when the queue head is not
// a tensor-core item, or when fewer than kClaimMargin other tiles of this
// tile's band are unfinished: the CTA that completes a band runs its
// packet-MD5 chains next, and a claimed item would wait behind them.
constexpr uint32_t kNoHeldItem = 0xFFFFFFFFu;
constexpr uint32_t kClaimMargin = 8;
__device__ __noinline__ bool batch_mma_tile(const BatchJob* __restrict__ jobs, const BatchItem* __restrict__ items,
                                            uint32_t n_items, uint32_t* __restrict__ ctl, const int* err,
                                            uint32_t idx, uint32_t* held) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint32_t* mm = reinterpret_cast<uint32_t*>(smem + kBatchMmaBarsOff + mma::kBarBytes);
    const uint16_t* gsm = reinterpret_cast<const uint16_t*>(smem + kBatchGinvOff);  // filled at launch start
    // Earlier items stored to this shared memory through the generic proxy;
    // the tile's bulk and tensor copies write it through the async proxy.
    // Order the two before any copy is issued.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    const BatchItem it = items[idx];
    const BatchJob& J = jobs[it.job];
    mma::Pipe P;
    P.ring = smem_u32(smem);
    P.bars = smem_u32(smem + kBatchMmaBarsOff);
    P.tmem = mm[0];
    P.ginv = gsm;
    P.abort_flag = mm + 1;
    P.g = mm[2];
    P.tcount = mm[3];
    P.drains = mm[4];
    P.gi = mm[5];
    P.pre = mm[6];
    if (threadIdx.x == 0) mma::tensormap_acquire(&J.src_map);  // written by the host's upload of the jobs
    const mma::Tile T = batch_mma_tile_of(J, it);
    // producer thread only (thread 0); the tile goes to its shared-memory slot
    auto claim_next = [&]() -> const mma::Tile* {
        *held = kNoHeldItem;
        if (*reinterpret_cast<const volatile int*>(err)) return nullptr;
        if (J.n_bands) {
            const uint32_t band = it.b >> 16;
            const uint32_t done = *reinterpret_cast<const volatile uint32_t*>(&J.bstate[band]);
            if (done + kClaimMargin >= J.band_items[band]) return nullptr;
        }
        const uint32_t h = *reinterpret_cast<const volatile uint32_t*>(&ctl[0]);
        if (h >= n_items || (items[h].kind_rg & kItemKindMask) != kItemEncodeMma) return nullptr;
        const uint32_t nidx = atomicAdd(&ctl[0], 1u);
        *held = nidx;
        if (nidx >= n_items) return nullptr;
        const BatchItem nit = items[nidx];
        if ((nit.kind_rg & kItemKindMask) != kItemEncodeMma) return nullptr;
        const BatchJob& Jn = jobs[nit.job];
        mma::tensormap_acquire(&Jn.src_map);
        mma::Tile* slot = reinterpret_cast<mma::Tile*>(smem + kBatchNextTileOff);
        *slot = batch_mma_tile_of(Jn, nit);
        return slot;
    };
    const bool ok = mma::run_tile<14>(P, T, claim_next);  // ends with a CTA barrier
    if (threadIdx.x == 0) {
        mm[2] = P.g;
        mm[3] = P.tcount;
        mm[4] = P.drains;
        mm[5] = P.gi;
        mm[6] = P.pre;
    }
    __syncthreads();
    return ok;
}

__device__ __forceinline__ void store_digest(uint8_t* out, const uint32_t st[4]) {
    uint32_t* o = reinterpret_cast<uint32_t*>(out);  // 4-byte aligned
    o[0] = st[0];
    o[1] = st[1];
    o[2] = st[2];
    o[3] = st[3];
}

// a < b comparing the 16 digest bytes in order (words hold them little-endian)
__device__ __forceinline__ bool id_less(const uint4& a, const uint4& b) {
    const uint32_t x[4] = {a.x, a.y, a.z, a.w}, y[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t p = __byte_perm(x[i], 0u, 0x0123), q = __byte_perm(y[i], 0u, 0x0123);
        if (p != q) return p < q;
    }
    return false;
}
__device__ __forceinline__ bool id_eq(const uint4& a, const uint4& b) {
    return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}

// The MD5 items (scan, file hash, packets, chain segments) are kept out of
// line: their chain loops then get registers of their own rather than a
// share of the persistent kernel's 128, which spills.
//
// Slice MD5 of slices [first, first+count) of job J on the kHashThreads
// lanes (one slice each, staged through the lane's ring).  The other warps
// idle: the lanes are bound by their chains, and the SM is the item's alone.
template <bool VEC>
__device__ __noinline__ void batch_scan(const BatchJob& J, uint32_t first, uint32_t count, uint32_t ring) {
    const int tid = threadIdx.x;
    if (tid < kHashThreads && (uint32_t)tid < count) {
        const uint32_t s = first + tid;
        uint32_t st[4];
        md5_init(st);
        md5_range_ring<0, VEC, kBatchRingUnits, kBatchRingAhead>(st, nullptr, J.src + (size_t)s * J.slice, J.slice,
                                                                 0, ~0ull, ring + tid * kBatchRingLane);
        store_digest(J.checks[s].md5, st);
    }
}

// Whole-file MD5 (hash_full, src/source.rs:222-228) of files [first,
// first+count) of job J, one file per MD5 lane: a serial chain each.
template <bool VEC>
__device__ __noinline__ void batch_file_hash(const BatchJob& J, uint32_t first, uint32_t count, uint32_t ring) {
    const int tid = threadIdx.x;
    if (tid < kHashThreads && (uint32_t)tid < count) {
        const uint32_t f = first + tid;
        uint32_t st[4];
        md5_init(st);
        md5_range_ring<0, VEC, kBatchRingUnits, kBatchRingAhead>(st, nullptr, J.src + J.files[2 * f],
                                                                 J.files[2 * f + 1], 0, ~0ull,
                                                                 ring + tid * kBatchRingLane);
        store_digest(J.hfull + 16 * (size_t)f, st);
    }
}

// Slice CRC32 of slices [first, first+count): one slice per warp at a time
// over all 16 warps (CRC streams from DRAM; its items are a few MB each so
// the work spreads over many SMs).
template <bool VEC>
__device__ __forceinline__ void batch_crc(const BatchJob& J, uint32_t first, uint32_t count,
                                          const uint32_t (*T)[256]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const CrcLane cl = crc_lane<VEC>(J.slice, lane);
    for (uint32_t i = (uint32_t)warp; i < count; i += kEncThreads / 32) {
        const uint32_t s = first + i;
        const uint32_t c = crc_slice_warp<VEC>(reinterpret_cast<const uint32_t*>(J.src + (size_t)s * J.slice), cl, lane, T);
        if (lane == 0) J.checks[s].crc32 = c;
    }
}

// Set-id step of job J (all threads of the CTA): hash16k of each file and
// its file id MD5(hash16k ‖ length le64 ‖ name) (src/source.rs:303-309); the
// main-packet body slice_size le64 ‖ count le32 ‖ file ids in byte order,
// whose MD5 is the set id (src/packet/main_packet.rs:25-42).  The set id
// goes to J.set_id and to sid[0..3] (shared memory).
template <bool VEC>
__device__ void batch_set_id(const BatchJob& J, uint32_t ring, uint32_t* sid) {
    const int tid = threadIdx.x;
    const uint32_t n = J.n_files;
    uint4* ids = reinterpret_cast<uint4*>(J.scratch);
    uint8_t* body = J.scratch + 16 * (size_t)n;
    if (tid < kHashThreads) {
        for (uint32_t f = tid; f < n; f += kHashThreads) {
            const uint64_t off = J.files[2 * f], len = J.files[2 * f + 1];
            uint32_t h[4];
            md5_init(h);
            md5_range_ring<0, VEC, kBatchRingUnits, kBatchRingAhead>(
                h, nullptr, J.src + off, len < P2G_HASH16K_LEN ? len : P2G_HASH16K_LEN, 0, ~0ull,
                ring + tid * kBatchRingLane);
            store_digest(J.h16k + 16 * (size_t)f, h);
            const uint32_t pre[6] = {h[0], h[1], h[2], h[3], (uint32_t)len, (uint32_t)(len >> 32)};
            uint32_t id[4];
            md5_init(id);
            md5_range<false>(id, pre, 24, J.names + J.name_off[2 * f], J.name_off[2 * f + 1], 0, ~0ull);
            __stcg(ids + f, make_uint4(id[0], id[1], id[2], id[3]));
        }
    }
    __syncthreads();
    // rank sort: ties keep file order (equal ids are interchangeable anyway)
    for (uint32_t f = tid; f < n; f += blockDim.x) {
        const uint4 me = __ldcg(ids + f);
        uint32_t rank = 0;
        for (uint32_t g = 0; g < n; ++g) {
            const uint4 o = __ldcg(ids + g);
            rank += (id_less(o, me) || (g < f && id_eq(o, me))) ? 1u : 0u;
        }
        uint32_t* d = reinterpret_cast<uint32_t*>(body + 12 + 16 * (size_t)rank);
        __stcg(d, me.x);
        __stcg(d + 1, me.y);
        __stcg(d + 2, me.z);
        __stcg(d + 3, me.w);
    }
    if (tid == 0) {
        uint32_t* b = reinterpret_cast<uint32_t*>(body);
        __stcg(b, (uint32_t)J.slice);
        __stcg(b + 1, (uint32_t)(J.slice >> 32));
        __stcg(b + 2, n);
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t s[4];
        md5_init(s);
        md5_range<false, true>(s, nullptr, 0, body, 12 + 16 * (uint64_t)n, 0, ~0ull);
        sid[0] = s[0];
        sid[1] = s[1];
        sid[2] = s[2];
        sid[3] = s[3];
        uint32_t* o = reinterpret_cast<uint32_t*>(J.set_id);
        __stcg(o, s[0]);
        __stcg(o + 1, s[1]);
        __stcg(o + 2, s[2]);
        __stcg(o + 3, s[3]);
    }
    __syncthreads();
}

// Packet MD5 of recovery rows [r0, r1) of job J (all threads of the CTA):
// MD5(set_id ‖ "PAR 2.0\0RecvSlic" ‖ exponent le32 ‖ row)
// (src/packet/recovery.rs:15, src/format.rs:33-54).
__device__ __noinline__ void batch_packets(const BatchJob& J, uint32_t ring, const uint32_t* sid, uint32_t r0, uint32_t r1) {
    const int tid = threadIdx.x;
    if (tid < kHashThreads) {
        for (uint32_t r = r0 + tid; r < r1; r += kHashThreads) {
            // set id ‖ "PAR 2.0\0" "RecvSlic" as little-endian words ‖ exponent
            const uint32_t pre[9] = {sid[0], sid[1], sid[2], sid[3], 0x20524150u, 0x00302E32u, 0x76636552u,
                                     0x63696C53u, J.first_exp + r};
            uint32_t st[4];
            md5_init(st);
            md5_range_ring<9, true, kBatchRingUnits, kBatchRingAhead>(
                st, pre, J.rec + (size_t)r * J.rec_stride, J.slice, 0, ~0ull, ring + tid * kBatchRingLane);
            store_digest(J.pkt + 16 * (size_t)r, st);
        }
    }
    __syncthreads();
}

// Chain segment: rows of block q advance over the message blocks that bands
// b..b_last completed (set id ‖ type ‖ exponent ‖ row bytes; the last band
// also pads and writes the digests).  State between passes lives in J.chain.
__device__ __noinline__ void advance_rows(const BatchJob& J, uint32_t q, uint32_t b, uint32_t b_last, uint32_t ring,
                                          const uint32_t* sid) {
    const int tid = threadIdx.x;
    const uint64_t total = 36 + J.slice;
    const uint64_t nblocks = (total + 8) / 64 + 1;
    const uint32_t Np = (uint32_t)((J.slice + 15) / 16 * 8);
    auto done_bytes = [&](uint32_t band) {  // row bytes final once bands 0..band are encoded
        const uint64_t end = min((uint64_t)Np, (uint64_t)(band + 1) * J.band_syms);
        return min(J.slice, 2 * end);
    };
    const bool final = b_last + 1 == J.n_bands;
    const uint64_t from = b == 0 ? 0 : (36 + done_bytes(b - 1)) / 64;
    const uint64_t to = final ? nblocks : (36 + done_bytes(b_last)) / 64;
    const uint32_t r = q * kChainRows + tid;
    if (tid < (int)kChainRows && r < J.R) {
        const uint32_t pre[9] = {sid[0], sid[1], sid[2], sid[3], 0x20524150u, 0x00302E32u, 0x76636552u,
                                 0x63696C53u, J.first_exp + r};
        uint32_t st[4];
        if (from == 0) {
            md5_init(st);
        } else {
            const uint4 v = __ldcg(reinterpret_cast<const uint4*>(J.chain) + r);
            st[0] = v.x;
            st[1] = v.y;
            st[2] = v.z;
            st[3] = v.w;
        }
        md5_range_ring<9, true, kBatchRingUnits, kBatchRingAhead>(st, pre, J.rec + (size_t)r * J.rec_stride,
                                                                  J.slice, from, to, ring + tid * kBatchRingLane);
        if (final)
            store_digest(J.pkt + 16 * (size_t)r, st);
        else
            __stcg(reinterpret_cast<uint4*>(J.chain) + r, make_uint4(st[0], st[1], st[2], st[3]));
        __threadfence();  // the next token holder, on another SM, reads this state
    }
    __syncthreads();
}

// Take block q's chain token if it is free and advance its rows over every
// band that is ready, in order; after releasing the token, look once more
// (a band that became ready while the token was held was left to us).  Each
// pass either advances at least one band or returns, so this ends.  No CTA
// waits for another: a busy token means its holder will see the new band.
constexpr uint32_t kChainBandsPerPass = 16;
__device__ void try_advance(const BatchJob& J, uint32_t q, uint32_t ring, uint32_t* misc) {
    const int tid = threadIdx.x;
    const uint32_t nb = J.n_bands, Q = (J.R + kChainRows - 1) / kChainRows;
    uint32_t* done = J.bstate;
    uint32_t* next = done + nb;
    uint32_t* busy = next + Q;
    uint32_t* sid_ready = busy + Q;
    auto ready = [&](uint32_t b) {
        return b < nb && atomicAdd(sid_ready, 0u) != 0 && atomicAdd(&done[b], 0u) == J.band_items[b];
    };
    for (;;) {
        if (tid == 0) misc[2] = atomicCAS(&busy[q], 0u, 1u) == 0u ? 1u : 0u;
        __syncthreads();
        const bool got = misc[2] != 0;
        __syncthreads();
        if (!got) return;
        for (;;) {
            // every band that is ready in a row goes in one pass: one chain
            // state load and store, one ring start and one hand-over for all
            if (tid == 0) {
                const uint32_t b = atomicAdd(&next[q], 0u);
                uint32_t k = 0;
                while (k < kChainBandsPerPass && ready(b + k)) ++k;
                misc[3] = b;
                misc[2] = k;
            }
            __syncthreads();
            const uint32_t k = misc[2];
            const uint32_t b = misc[3];
            if (k && tid < 4) misc[4 + tid] = __ldcg(reinterpret_cast<const uint32_t*>(J.set_id) + tid);
            __syncthreads();
            if (!k) break;
            __threadfence();  // acquire: the bands' rows and the set id
            advance_rows(J, q, b, b + k - 1, ring, misc + 4);
            if (tid == 0) {
                __threadfence();
                atomicExch(&next[q], b + k);
            }
            __syncthreads();
        }
        if (tid == 0) {
            __threadfence();
            atomicExch(&busy[q], 0u);
            __threadfence();
            misc[2] = ready(atomicAdd(&next[q], 0u)) ? 1u : 0u;
        }
        __syncthreads();
        const bool again = misc[2] != 0;
        __syncthreads();
        if (!again) return;
    }
}

__device__ void advance_all(const BatchJob& J, uint32_t ring, uint32_t* misc) {
    const uint32_t Q = (J.R + kChainRows - 1) / kChainRows;
    for (uint32_t q = 0; q < Q; ++q) try_advance(J, q, ring, misc);
}

// MMA: the launch has tensor-core items (mma_ginv set).  The variant without
// them keeps the other item kinds' code free of the tensor pipeline's
// registers.
template <bool MMA>
__global__ void __launch_bounds__(kEncThreads, 1)
    batch_kernel(const BatchJob* __restrict__ jobs, const BatchItem* __restrict__ items, uint32_t n_items,
                 uint32_t* __restrict__ ctl, int* __restrict__ err, const uint16_t* __restrict__ mma_ginv) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* enc = smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(enc + encode_bars_offset<kEncChunks, 4, kBatchEncStages>());
    uint8_t* ring_p = smem + kBatchRingOff;
    uint32_t(*T)[256] = reinterpret_cast<uint32_t(*)[256]>(ring_p + kBatchRingBytes);
    // [0] item [1] last [2..3] chain tokens [4..7] set id [8] item claimed ahead by a tensor-core tile
    uint32_t* misc = reinterpret_cast<uint32_t*>(ring_p + kBatchRingBytes + 4 * 256 * 4);
    const uint32_t ring = smem_u32(ring_p);
    const int tid = threadIdx.x;
    // tensor-core items (mma_ginv set): TMEM for the whole launch, barriers
    // and scale factors set up once.  mma_misc: [0] TMEM address, [1] abort
    // flag, [2..6] pipeline state.
    uint32_t* mma_misc = reinterpret_cast<uint32_t*>(smem + kBatchMmaBarsOff + mma::kBarBytes);
    const uint32_t mma_bars = smem_u32(smem + kBatchMmaBarsOff);
    // The lookup items' barriers lie inside the tensor-core input stages.
    // Launches with tensor-core items set them up only around a lookup item
    // and invalidate them after it (an mbarrier's bytes may hold other data
    // only once it is invalidated); such launches plan no lookup items.
    if (tid == 0) {
        misc[8] = kNoHeldItem;
        if (!MMA)
            for (int st = 0; st < kBatchEncStages; ++st) mbar_init(&bars[st], 1);
        if (MMA) {
            mma::init_bars(mma_bars, 14);
            mma_misc[1] = mma_misc[2] = mma_misc[3] = mma_misc[4] = mma_misc[5] = mma_misc[6] = 0;
        }
        fence_mbar_init();
    }
    if (MMA && (tid >> 5) == 1) mma::tmem_alloc(smem_u32(mma_misc));
    if (MMA) mma::tc_fence_before();
    crc_tables_build(T);  // ends with __syncthreads
    if (MMA) {
        mma::tc_fence_after();
        if ((tid >> 5) >= 4 && (tid >> 5) < 8) mma::sf_fill(mma_misc[0], (uint32_t)(tid >> 5) & 3u);
        uint16_t* gsm = reinterpret_cast<uint16_t*>(smem + kBatchGinvOff);
        for (int i = tid; i < 512; i += kEncThreads) gsm[i] = mma_ginv[i];
        mma::tc_fence_before();
        __syncthreads();
        mma::tc_fence_after();
    }
    uint32_t phase = 0;
    for (;;) {
        if (tid == 0) {
            // an item a tensor-core tile claimed ahead runs next whatever the
            // error flag says: its first input copies may be in flight
            const uint32_t h = misc[8];
            misc[8] = kNoHeldItem;
            misc[0] = h != kNoHeldItem ? h
                      : *reinterpret_cast<volatile int*>(err) ? n_items
                                                                : atomicAdd(&ctl[0], 1u);
        }
        __syncthreads();
        const uint32_t idx = misc[0];
        if (idx >= n_items) break;
        const BatchItem it = items[idx];
        const BatchJob& J = jobs[it.job];
        const uint32_t kind = it.kind_rg & kItemKindMask;
        if (kind == kItemScan) {
            if (J.vec)
                batch_scan<true>(J, it.a, it.b, ring);
            else
                batch_scan<false>(J, it.a, it.b, ring);
            __syncthreads();
            continue;
        }
        if (kind == kItemFileHash) {
            if (J.vec)
                batch_file_hash<true>(J, it.a, it.b, ring);
            else
                batch_file_hash<false>(J, it.a, it.b, ring);
            __syncthreads();
            continue;
        }
        if (kind == kItemCrc) {
            if (J.vec)
                batch_crc<true>(J, it.a, it.b, T);
            else
                batch_crc<false>(J, it.a, it.b, T);
            __syncthreads();
            continue;
        }
        if (kind == kItemSetId) {
            if (J.vec)
                batch_set_id<true>(J, ring, misc + 4);
            else
                batch_set_id<false>(J, ring, misc + 4);
            if (J.n_bands && J.R) {  // chain segments may start
                if (tid == 0) {
                    __threadfence();
                    atomicExch(J.bstate + J.n_bands + 2 * ((J.R + kChainRows - 1) / kChainRows), 1u);
                }
                __syncthreads();
                advance_all(J, ring, misc);
            }
            continue;
        }
        if (kind == kItemPacket) {
            if (tid < 4) misc[4 + tid] = __ldcg(reinterpret_cast<const uint32_t*>(J.set_id) + tid);
            __syncthreads();
            batch_packets(J, ring, misc + 4, it.a, it.a + it.b);
            continue;
        }
        if (MMA && kind == kItemEncodeMma) {
            const bool ok = batch_mma_tile(jobs, items, n_items, ctl, err, idx, misc + 8);
            // the builders' generic stores come before any later item's bulk
            // copies (async proxy) into the same bytes
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (!ok) {
                if (tid == 0) atomicOr(err, 1);
                break;
            }
            if (!J.n_bands) continue;
            const uint32_t band = it.b >> 16;
            __threadfence();  // release this tile's rows before counting it
            __syncthreads();
            if (tid == 0) misc[1] = (atomicAdd(&J.bstate[band], 1u) + 1 == J.band_items[band]) ? 1u : 0u;
            __syncthreads();
            if (!misc[1]) continue;
            __threadfence();  // acquire: the whole band is visible from here on
            advance_all(J, ring, misc);
            continue;
        }
        if (kind == kItemEncode) {
            if (MMA) {  // its barriers, set up for this item alone (nothing is in flight now)
                if (tid == 0) {
                    for (int st = 0; st < kBatchEncStages; ++st) mbar_init(&bars[st], 1);
                    fence_mbar_init();
                }
                phase = 0;
                __syncthreads();
            }
            // the job's precomputed basis when it has one, else derived per slice
            const uint32_t rg = (it.kind_rg >> 8) & 0xFFFFu, sn = it.sn ? it.sn : J.S;
            const uint32_t fold = 1u << ((it.kind_rg >> 24) & 3u);
            const uint32_t syms = it.b & 0xFFFFu, band = it.b >> 16;
            const bool acc = (it.kind_rg & kItemAccumulate) != 0;
            const bool ok = J.basis ? encode_tile<kEncChunks, false, 4, kBatchEncStages>(J.esrc, J.estride, sn, J.basis, J.RG, rg, J.R,
                                                                         it.a, syms, J.rec, J.rec_stride, enc, phase,
                                                                         J.first_exp, it.s0, acc, fold, J.ts)
                                    : encode_tile<kEncChunks, true, 4, kBatchEncStages>(J.esrc, J.estride, sn, nullptr, J.RG, rg, J.R,
                                                                        it.a, syms, J.rec, J.rec_stride, enc, phase,
                                                                        J.first_exp, it.s0, acc, fold, J.ts);
            if (MMA) {  // the barriers' bytes go back to the tensor-core input stages
                __syncthreads();
                if (tid == 0)
                    for (int st = 0; st < kBatchEncStages; ++st) mbar_inval(&bars[st]);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
            }
            if (!ok) {
                if (tid == 0) atomicOr(err, 1);
                break;
            }
            if (!J.n_bands) continue;
            __threadfence();  // release this tile's rows before counting it
            __syncthreads();
            if (tid == 0) misc[1] = (atomicAdd(&J.bstate[band], 1u) + 1 == J.band_items[band]) ? 1u : 0u;
            __syncthreads();
            if (!misc[1]) continue;
            __threadfence();  // acquire: the whole band is visible from here on
            advance_all(J, ring, misc);
        }
    }
    if (MMA) {  // every MMA issued has completed before TMEM is given back
        mma::tc_fence_before();
        __syncthreads();
        if (tid == 0 && mma_misc[6]) {
            // input stages issued ahead for a tile that did not run (the loop
            // always runs a claimed tile, so this stays idle): they land before
            // the CTA exits
            const mma::Bars B(mma_bars);
            for (uint32_t q = mma_misc[5]; q < mma_misc[5] + mma_misc[6]; ++q)
                mma::bar_drain(B.in_full + 8 * (q % mma::kInStages), (q / mma::kInStages) & 1u);
        }
        if ((tid >> 5) == 1) {
            if ((tid & 31) == 0) {
                const mma::Bars B(mma_bars);
                mma::mma_commit(B.drain);
                mma::bar_drain(B.drain, mma_misc[4] & 1u);
            }
            __syncwarp();
            mma::tc_fence_after();
            mma::tmem_free(mma_misc[0]);
        }
    }
}

// Seeded synthetic source: file f of a job occupies [off, off+padded) of
// `base`; its bytes are the splitmix64 counter stream of seed f (8-byte word
// k = mix(seed + (k+1)*0x9E3779B97F4A7C15), little-endian) for `len` bytes,
// then zeros.  Offsets are multiples of 4 (slice boundaries).
__device__ __forceinline__ uint64_t splitmix_word(uint64_t seed, uint64_t k) {
    uint64_t z = seed + (k + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__global__ void seeded_fill_kernel(uint8_t* __restrict__ base, const uint64_t* __restrict__ spans,
                                   const uint64_t* __restrict__ seeds) {
    const uint64_t off = spans[3 * blockIdx.y], len = spans[3 * blockIdx.y + 1], padded = spans[3 * blockIdx.y + 2];
    const uint64_t seed = seeds[blockIdx.y];
    uint32_t* dst = reinterpret_cast<uint32_t*>(base + off);
    const uint64_t words = padded / 4;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = 0;
        const uint64_t b = 4 * w;
        if (b < len) {
            const uint64_t z = splitmix_word(seed, w >> 1);
            v = (w & 1) ? (uint32_t)(z >> 32) : (uint32_t)z;
            if (b + 4 > len) v &= 0xFFFFFFFFu >> (8 * (b + 4 - len));
        }
        dst[w] = v;
    }
}

__global__ void basis_batch_kernel(const BatchJob* __restrict__ jobs) {
    const BatchJob& J = jobs[blockIdx.y];
    if (!J.R || !J.basis) return;
    // the last row group replicated as the folded encode items build it (tail_fold)
    const uint32_t tail = J.R - (J.R - 1) / kRowsPerGroup * kRowsPerGroup;
    const uint32_t fold = tail <= 8 ? 4u : tail <= 16 ? 2u : 1u;
    basis_fill(J.basis, J.S, J.RG, J.R, J.first_exp, ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
               ((uint64_t)gridDim.x * blockDim.x) >> 5, fold);
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Tile size for Np symbol positions and RG row groups on `sms` SMs (one CTA
// each).  Per input slice a CTA spends about one shared-memory wavefront per
// symbol of its tile on lookups plus a fixed ~384 on building its tables, so
// pick the tile count minimising ceil(tiles*RG/sms) * (tile + 384): the
// fewest, fullest waves.
uint32_t tail_fold(uint32_t R) {
    if (!R) return 1;
    const uint32_t tail = R - (R - 1) / kRowsPerGroup * kRowsPerGroup;  // rows of the last group, 1..32
    return tail <= 8 ? 4u : tail <= 16 ? 2u : 1u;
}
// CTAs of `tiles` tiles over RG row groups whose last one is folded
static inline uint64_t eff_ctas(uint64_t tiles, uint32_t RG, uint32_t fold) {
    return tiles * (RG - 1) + (tiles + fold - 1) / fold;
}
// tiles per band so that its CTAs fit `budget` SMs (at least 1)
static inline uint32_t tiles_for_budget(uint32_t budget, uint32_t RG, uint32_t fold) {
    uint32_t t = (uint32_t)((uint64_t)budget * fold / ((uint64_t)(RG - 1) * fold + 1));
    while (t > 1 && eff_ctas(t, RG, fold) > budget) --t;
    return t ? t : 1;
}

void choose_tiles(uint32_t Np, uint32_t RG, uint32_t sms, uint32_t* ts_out, uint32_t* tiles_out, uint32_t fold) {
    constexpr uint64_t kBuildCost = 384;
    const uint32_t tmin = (Np + kEncTileSymbols - 1) / kEncTileSymbols;
    uint64_t best_cost = ~0ull;
    uint32_t best_ts = kEncTileSymbols, best_t = tmin;
    for (uint32_t t = tmin; t <= 4 * tmin + 8; ++t) {
        const uint32_t ts = ((Np + t - 1) / t + 7) & ~7u;
        if (ts == 0 || ts > (uint32_t)kEncTileSymbols) continue;
        const uint32_t tt = (Np + ts - 1) / ts;
        const uint64_t waves = (eff_ctas(tt, RG, fold) + sms - 1) / sms;
        const uint64_t cost = waves * (ts + kBuildCost);
        if (cost < best_cost) {
            best_cost = cost;
            best_ts = ts;
            best_t = tt;
        }
    }
    *ts_out = best_ts;
    *tiles_out = best_t;
}

cudaError_t launch_basis(uint16_t* basis, uint32_t S, uint32_t RG, uint32_t R, uint32_t first_exp,
                         cudaStream_t st) {
    const uint64_t total = (uint64_t)S * RG;  // 1 KiB blocks, one warp each
    if (!total) return cudaSuccess;
    const uint64_t want = (total + 7) / 8;
    const unsigned blocks = (unsigned)(want < (uint64_t)sm_count() * 16 ? want : (uint64_t)sm_count() * 16);
    basis_kernel<<<blocks, 256, 0, st>>>(basis, S, RG, R, first_exp, tail_fold(R));
    count_launch();
    return cudaGetLastError();
}

static cudaError_t encode_attr() {
    constexpr size_t smem = encode_smem_bytes<kEncChunks, 4>();
    static bool attr_set[256] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 256 || !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(encode_lut_kernel<kEncChunks, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(encode_lut_kernel<kEncChunks, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 256) attr_set[dev] = true;
    }
    return cudaSuccess;
}

// Band plan.  The symbol range is cut into bands of whole waves so bands
// finish in order and the recovery-packet MD5 chains can follow band by band
// (one SM kept free for them).  While the slice-MD5 blocks run (`reserve`
// SMs for about `reserve_ms`), bands are sized to leave those SMs alone;
// the plan keeps that only when it beats sharing SMs with them (which slows
// the bands involved about twofold).  Per input slice a CTA spends ~1 shared-
// memory wavefront per tile symbol plus ~384 on its tables; 0.78 of the peak
// wavefront rate at ~1.9 GHz estimates band times.
static double est_band_ms(uint32_t S, uint32_t ts, uint32_t waves) {
    return (double)S * (ts + 384.0) * waves / (0.78 * 1.9e6);
}

static void split_even(EncodePlan& pl, uint32_t begin, uint32_t RG, uint32_t budget, double* ms, uint32_t S) {
    if (begin >= pl.Np) return;
    const uint32_t tiles = tiles_for_budget(budget, RG, pl.fold);
    const uint32_t waves = (uint32_t)((eff_ctas(tiles, RG, pl.fold) + budget - 1) / budget);
    const uint64_t rem = pl.Np - begin;
    const uint64_t per = (uint64_t)tiles * kEncTileSymbols;
    const uint32_t B = (uint32_t)((rem + per - 1) / per);
    const uint32_t ts = (uint32_t)(((rem + (uint64_t)B * tiles - 1) / ((uint64_t)B * tiles) + 7) & ~7ull);
    for (uint32_t b = 0; b < B; ++b) {
        const uint64_t s0 = begin + (uint64_t)b * tiles * ts;
        if (s0 >= pl.Np) break;
        const uint32_t s1 = (uint32_t)std::min<uint64_t>(pl.Np, s0 + (uint64_t)tiles * ts);
        pl.bands.push_back({(uint32_t)s0, s1, ts});
        if (ms) *ms += est_band_ms(S, ts, waves);
    }
}

EncodePlan plan_encode(uint64_t slice_size, uint32_t S, uint32_t RG, bool banded, uint32_t reserve,
                       double reserve_ms, uint32_t fold) {
    EncodePlan pl;
    pl.Np = (uint32_t)(((slice_size + 15) & ~15ull) / 2);
    pl.fold = fold;
    const uint32_t sms = (uint32_t)sm_count();
    uint32_t ts1 = 0, t1 = 0;
    choose_tiles(pl.Np, RG, sms, &ts1, &t1, fold);
    EncodePlan c = pl;  // C: one launch, packet MD5 after it
    c.bands.push_back({0, pl.Np, ts1});
    if (!banded || sms < 4) return c;
    // Banded plans run each band as one wave, which lasts as long as its
    // slowest CTA; a folded tail CTA (4x the source reads of one tile) runs
    // ~15% longer than the others, which cancels its saving there, so bands
    // keep the last row group unfolded.
    if (fold != 1) {
        EncodePlan unfolded = plan_encode(slice_size, S, RG, banded, reserve, reserve_ms, 1);
        if (unfolded.bands.size() > 1) return unfolded;
        return c;
    }
    const double chain_ms_per_byte = 7.2e-4 / 64;  // one MD5 chain: ~0.72 us per 64-byte block
    const uint32_t waves1 = (uint32_t)((eff_ctas(t1, RG, fold) + sms - 1) / sms);
    const double ms_c = est_band_ms(S, ts1, waves1) + 2.0 * pl.Np * chain_ms_per_byte + reserve_ms;
    auto tail = [&](const EncodePlan& p) {  // last band's packet-MD5 step + per-band launch/drain
        const EncodeBand& l = p.bands.back();
        return 2.0 * (l.end - l.begin) * chain_ms_per_byte + 0.02 * p.bands.size();
    };
    // A: bands with one SM kept for the packet MD5; slice MD5 shares SMs
    EncodePlan a = pl;
    double ms_a = 0;
    split_even(a, 0, RG, sms - 1, &ms_a, S);
    ms_a += std::min(reserve_ms, ms_a) + tail(a);  // bands overlapping the slice MD5 run ~2x slower
    // B: early bands leave the slice-MD5 SMs alone, later bands use them
    EncodePlan b = pl;
    double ms_b = 1e30;
    if (reserve && reserve + 2 < sms) {
        const uint32_t budget = sms - reserve - 1;
        const uint32_t tiles = tiles_for_budget(budget, RG, fold);
        const uint32_t waves = (uint32_t)((eff_ctas(tiles, RG, fold) + budget - 1) / budget);
        uint32_t sym = 0;
        ms_b = 0;
        while (sym < pl.Np && ms_b < reserve_ms) {
            const uint32_t s1 = (uint32_t)std::min<uint64_t>(pl.Np, sym + (uint64_t)tiles * kEncTileSymbols);
            b.bands.push_back({sym, s1, (uint32_t)kEncTileSymbols});
            ms_b += est_band_ms(S, kEncTileSymbols, waves);
            sym = s1;
        }
        split_even(b, sym, RG, sms - 1, &ms_b, S);
        ms_b += tail(b);
    }
    const size_t kMaxBands = 64;
    if (a.bands.size() > kMaxBands) ms_a = 1e30;
    if (b.bands.size() > kMaxBands) ms_b = 1e30;
    if (ms_c <= ms_a && ms_c <= ms_b) return c;
    return ms_b < ms_a ? b : a;
}

cudaError_t launch_encode_band(const EncodePlan& pl, uint32_t band, const uint8_t* src, uint64_t src_stride,
                               uint32_t S, const uint16_t* basis, uint32_t RG, uint32_t R, uint8_t* rec,
                               uint64_t rec_stride, int* err, cudaStream_t st, uint32_t first_exp) {
    constexpr size_t smem = encode_smem_bytes<kEncChunks, 4>();
    cudaError_t e = encode_attr();
    if (e != cudaSuccess) return e;
    if (band >= pl.bands.size() || !R) return cudaSuccess;
    const EncodeBand& bd = pl.bands[band];
    if (bd.begin >= bd.end) return cudaSuccess;
    const uint32_t tiles = (bd.end - bd.begin + bd.ts - 1) / bd.ts;
    if (basis)
        encode_lut_kernel<kEncChunks, false><<<tiles * RG, kEncThreads, smem, st>>>(
            src, src_stride, S, basis, RG, R, bd.begin, bd.end, bd.ts, rec, rec_stride, first_exp, pl.fold, err);
    else  // coefficient basis derived in the kernel
        encode_lut_kernel<kEncChunks, true><<<tiles * RG, kEncThreads, smem, st>>>(
            src, src_stride, S, nullptr, RG, R, bd.begin, bd.end, bd.ts, rec, rec_stride, first_exp, pl.fold, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_encode(const uint8_t* src, uint64_t src_stride, uint32_t S, const uint16_t* basis,
                          uint32_t RG, uint32_t R, uint64_t slice_size, uint8_t* rec, uint64_t rec_stride,
                          int* err, cudaStream_t st, uint32_t first_exp) {
    const EncodePlan pl = plan_encode(slice_size, S, RG, false, 0, 0.0, tail_fold(R));
    return launch_encode_band(pl, 0, src, src_stride, S, basis, RG, R, rec, rec_stride, err, st, first_exp);
}

// Diagnostic for the failure path every TMA wait in this file takes: an
// mbarrier that nothing ever arrives on, waited for with the same bounded
// poll loop (`polls` tries instead of the production limit).  The wait gives
// up, the kernel records it in *gave_up and returns; nothing faults or hangs.
__global__ void bounded_wait_probe_kernel(int* __restrict__ gave_up, uint32_t polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    bool ok = false;
    for (uint32_t it = 0; it < polls && !ok; ++it) ok = mbar_try_wait(&bar, 0);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(gave_up, 1);
}

cudaError_t launch_bounded_wait_probe(int* gave_up, uint32_t polls, cudaStream_t st) {
    bounded_wait_probe_kernel<<<1, 32, 0, st>>>(gave_up, polls);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gf_mul_xor(uint16_t coeff, const uint8_t* in, uint8_t* out, size_t len, cudaStream_t st) {
    const uint64_t nsym = len / 2;
    if (!nsym) return cudaSuccess;
    const uint64_t want = (nsym + 255) / 256;
    const unsigned blocks = (unsigned)(want < (uint64_t)sm_count() * 8 ? want : (uint64_t)sm_count() * 8);
    gf_mul_xor_kernel<<<blocks, 256, 0, st>>>(coeff, in, out, nsym);
    count_launch();
    return cudaGetLastError();
}

// Hash blocks run long serial chains; any long-running warp sharing an SM
// with an encode CTA slows that CTA (its per-slice barrier waits for the
// slowest warp) and with it the whole band.  So hash blocks claim almost all
// of an SM's shared memory: nothing else can be resident beside them.
static int exclusive_smem() {
    static int v = 0;
    if (!v) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (v <= 0) v = 48 * 1024;
    }
    return v;
}
template <class K>
static cudaError_t allow_exclusive(K kernel) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, exclusive_smem());
}
struct HashGrid {
    unsigned blocks, threads;
    size_t smem;
};
static HashGrid hash_grid(uint32_t streams) {
    const unsigned warps = (streams + 31) / 32;
    const unsigned wpb = warps < (unsigned)(kHashThreads / 32) ? warps : (unsigned)(kHashThreads / 32);
    HashGrid g;
    g.threads = wpb * 32;
    g.blocks = (streams + g.threads - 1) / g.threads;
    g.smem = (size_t)exclusive_smem();
    return g;
}
uint32_t hash_blocks(uint32_t streams) { return streams ? hash_grid(streams).blocks : 0; }

cudaError_t launch_md5_slices(const uint8_t* src, uint64_t stride, uint32_t count, uint64_t slice_size,
                              p2g_slice_checksum* out, cudaStream_t st) {
    if (!count) return cudaSuccess;
    const HashGrid g = hash_grid(count);
    const bool vec = ((uintptr_t)src % 16 == 0) && (stride % 16 == 0);
    cudaError_t e;
    if (vec) {
        if ((e = allow_exclusive(md5_slices_kernel<true>)) != cudaSuccess) return e;
        md5_slices_kernel<true><<<g.blocks, g.threads, g.smem, st>>>(src, stride, count, slice_size, out);
    } else {
        if ((e = allow_exclusive(md5_slices_kernel<false>)) != cudaSuccess) return e;
        md5_slices_kernel<false><<<g.blocks, g.threads, g.smem, st>>>(src, stride, count, slice_size, out);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_crc_slices(const uint8_t* src, uint64_t stride, uint32_t count, uint64_t slice_size,
                              p2g_slice_checksum* out, cudaStream_t st) {
    if (!count) return cudaSuccess;
    const unsigned tpb = 64, wpb = tpb / 32;
    const uint64_t want = (count + wpb - 1) / wpb;
    const unsigned blocks = (unsigned)(want < (uint64_t)sm_count() * 8 ? want : (uint64_t)sm_count() * 8);
    const bool vec = ((uintptr_t)src % 16 == 0) && (stride % 16 == 0) && (slice_size % 16 == 0);
    if (vec)
        crc_slices_kernel<true><<<blocks, tpb, 0, st>>>(src, stride, count, slice_size, out);
    else
        crc_slices_kernel<false><<<blocks, tpb, 0, st>>>(src, stride, count, slice_size, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_md5_files(const uint8_t* base, const FileSpan* spans, uint32_t n, uint8_t* out16,
                             cudaStream_t st) {
    if (!n) return cudaSuccess;
    const HashGrid g = hash_grid(n);
    cudaError_t e = allow_exclusive(md5_files_kernel<false>);
    if (e != cudaSuccess) return e;
    // file starts are only known to be 4-byte aligned: 4-byte ring copies
    md5_files_kernel<false><<<g.blocks, g.threads, g.smem, st>>>(base, spans, n, out16);
    count_launch();
    return cudaGetLastError();
}

static RecvPrefix recv_prefix(const uint8_t set_id[16]) {
    RecvPrefix pfx;
    static const uint8_t kType[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'R', 'e', 'c', 'v', 'S', 'l', 'i', 'c'};
    uint8_t raw[32];
    for (int i = 0; i < 16; ++i) raw[i] = set_id[i];
    for (int i = 0; i < 16; ++i) raw[16 + i] = kType[i];
    for (int i = 0; i < 8; ++i)
        pfx.w[i] = (uint32_t)raw[4 * i] | ((uint32_t)raw[4 * i + 1] << 8) | ((uint32_t)raw[4 * i + 2] << 16) |
                   ((uint32_t)raw[4 * i + 3] << 24);
    return pfx;
}

cudaError_t launch_md5_recovery(const uint8_t* rec, uint64_t stride, uint32_t count, uint64_t slice_size,
                                const uint8_t set_id[16], uint32_t first_exp, uint8_t* out16, cudaStream_t st) {
    if (!count) return cudaSuccess;
    const HashGrid g = hash_grid(count);
    cudaError_t e;
    // 16-byte ring copies only when every row starts 16-byte aligned
    if ((uintptr_t)rec % 16 == 0 && stride % 16 == 0) {
        if ((e = allow_exclusive(md5_recovery_kernel<true>)) != cudaSuccess) return e;
        md5_recovery_kernel<true><<<g.blocks, g.threads, g.smem, st>>>(rec, stride, count, slice_size,
                                                                        recv_prefix(set_id), first_exp, out16);
    } else {
        if ((e = allow_exclusive(md5_recovery_kernel<false>)) != cudaSuccess) return e;
        md5_recovery_kernel<false><<<g.blocks, g.threads, g.smem, st>>>(rec, stride, count, slice_size,
                                                                         recv_prefix(set_id), first_exp, out16);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_md5_recovery_range(const uint8_t* rec, uint64_t stride, uint32_t count, uint64_t slice_size,
                                      const uint8_t set_id[16], uint32_t first_exp, uint32_t* state,
                                      uint64_t b_from, uint64_t b_to, bool final, uint8_t* out16, cudaStream_t st) {
    if (!count || (b_from >= b_to && !final)) return cudaSuccess;
    const HashGrid g = hash_grid(count);
    cudaError_t e;
    if ((uintptr_t)rec % 16 == 0 && stride % 16 == 0) {
        if ((e = allow_exclusive(md5_recovery_range_kernel<true>)) != cudaSuccess) return e;
        md5_recovery_range_kernel<true><<<g.blocks, g.threads, g.smem, st>>>(
            rec, stride, count, slice_size, recv_prefix(set_id), first_exp, state, b_from, b_to, final ? 1 : 0, out16);
    } else {
        if ((e = allow_exclusive(md5_recovery_range_kernel<false>)) != cudaSuccess) return e;
        md5_recovery_range_kernel<false><<<g.blocks, g.threads, g.smem, st>>>(
            rec, stride, count, slice_size, recv_prefix(set_id), first_exp, state, b_from, b_to, final ? 1 : 0, out16);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_realign(const uint8_t* src, uint64_t src_stride, uint8_t* dst, uint64_t dst_stride,
                           uint32_t count, uint64_t slice_size, cudaStream_t st) {
    const uint64_t total = slice_size / 4 * count;
    if (!total) return cudaSuccess;
    const uint64_t want = (total + 255) / 256;
    const unsigned blocks = (unsigned)(want < (uint64_t)sm_count() * 16 ? want : (uint64_t)sm_count() * 16);
    realign_kernel<<<blocks, 256, 0, st>>>(src, src_stride, dst, dst_stride, count, slice_size);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather_host(const uint64_t* seg, uint32_t n_seg, cudaStream_t st) {
    if (!n_seg) return cudaSuccess;
    const unsigned blocks = n_seg < (uint32_t)sm_count() * 4 ? n_seg : (unsigned)sm_count() * 4;
    gather_host_kernel<<<blocks, 512, 0, st>>>(seg, n_seg);
    count_launch();
    return cudaGetLastError();
}

int device_sm_count() { return sm_count(); }

cudaError_t launch_basis_batch(const BatchJob* jobs, uint32_t n_jobs, uint64_t max_words, cudaStream_t st) {
    if (!n_jobs || !max_words) return cudaSuccess;
    const uint64_t want = (max_words / 512 + 7) / 8;  // one warp per 1 KiB block
    const unsigned bx = (unsigned)(want < (uint64_t)sm_count() * 4 ? want : (uint64_t)sm_count() * 4);
    basis_batch_kernel<<<dim3(bx, n_jobs), 256, 0, st>>>(jobs);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_seeded_fill(uint8_t* base, const uint64_t* spans, const uint64_t* seeds, uint32_t n_files,
                               uint64_t max_padded, cudaStream_t st) {
    if (!n_files || !max_padded) return cudaSuccess;
    const uint64_t want = (max_padded / 4 + 255) / 256;
    const unsigned bx = (unsigned)(want < (uint64_t)sm_count() * 8 ? want : (uint64_t)sm_count() * 8);
    seeded_fill_kernel<<<dim3(bx, n_files), 256, 0, st>>>(base, spans, seeds);
    count_launch();
    return cudaGetLastError();
}

cudaError_t prepare_batch_kernel() {
    static bool attr_set[256] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 256 || !attr_set[dev]) {
        cudaError_t e =
            cudaFuncSetAttribute(batch_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 256) attr_set[dev] = true;
    }
    return cudaSuccess;
}

cudaError_t launch_batch(const BatchJob* jobs, const BatchItem* items, uint32_t n_items, uint32_t* ctl, int* err,
                         uint32_t ctas, cudaStream_t st, bool mma) {
    if (!n_items) return cudaSuccess;
    cudaError_t e = prepare_batch_kernel();
    if (e != cudaSuccess) return e;
    const uint16_t* ginv = nullptr;
    if (mma && (e = mma_tables_ready(&ginv)) != cudaSuccess) return e;
    if (mma)
        batch_kernel<true><<<ctas, kEncThreads, kBatchSmem, st>>>(jobs, items, n_items, ctl, err, ginv);
    else
        batch_kernel<false><<<ctas, kEncThreads, kBatchSmem, st>>>(jobs, items, n_items, ctl, err, nullptr);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Heap-free helpers for the allocation-free entry point (p2g_noalloc.cu):
// same tables and the same single-launch encode as above, but without any
// host or device allocation.
// ---------------------------------------------------------------------------
cudaError_t upload_tables_noheap() {
    static uint16_t lg[65536], al[65536], lb[32768];
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    uint32_t b = 1;
    for (uint32_t l = 0; l < kFieldLimit; l++) {
        lg[b] = (uint16_t)l;
        al[l] = (uint16_t)b;
        b <<= 1;
        if (b & 0x10000u) b ^= kFieldGenerator;
    }
    lg[0] = (uint16_t)kFieldLimit;
    al[kFieldLimit] = 0;
    uint32_t n = 0;
    for (uint32_t l = 0; l < kFieldLimit && n < 32768; l++) {
        uint32_t x = kFieldLimit, y = l;
        while (y) {
            const uint32_t t = x % y;
            x = y;
            y = t;
        }
        if (x == 1) lb[n++] = (uint16_t)l;
    }
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(d_log, lg, sizeof lg)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(d_antilog, al, sizeof al)) != cudaSuccess) return e;
    return cudaMemcpyToSymbol(d_logbase, lb, sizeof lb);
}

cudaError_t launch_encode_noheap(const uint8_t* src, uint64_t src_stride, uint32_t S, const uint16_t* basis,
                                 uint32_t RG, uint32_t R, uint64_t slice_size, uint8_t* rec, uint64_t rec_stride,
                                 int* err, cudaStream_t st) {
    constexpr size_t smem = encode_smem_bytes<kEncChunks, 4>();
    cudaError_t e = encode_attr();
    if (e != cudaSuccess) return e;
    const uint32_t Np = (uint32_t)(((slice_size + 15) & ~15ull) / 2);
    uint32_t ts = 0, tiles = 0;
    choose_tiles(Np, RG, (uint32_t)sm_count(), &ts, &tiles);
    if (!R || !tiles) return cudaSuccess;
    encode_lut_kernel<kEncChunks, false><<<tiles * RG, kEncThreads, smem, st>>>(src, src_stride, S, basis, RG, R, 0,
                                                                                Np, ts, rec, rec_stride, 0, 1, err);
    count_launch();
    return cudaGetLastError();
}

}  // namespace p2g
