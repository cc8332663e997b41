// p2g_mma_tile.cuh -- device code of the tensor-core (tcgen05, kind::mxf4)
// encode shared by its standalone kernel (p2g_mma.cu) and the persistent
// batch kernel (p2g_kernels.cu).
//
// The arithmetic (bits(c*x) = G^-1 H_c bits(x), H_c a Hankel matrix from the
// 31-bit trace string T_c) is explained at the top of p2g_mma.cu.  Here: the
// shared-memory and TMEM layout of one CTA and the work of one 16-row x
// 240-symbol tile over a range of input slices.
//
// The A operand (the coefficients' bit matrices) depends only on the 16-row
// tile and the K-step, so it is built once per job in global memory (the A
// image, a_image_index below) and every tile copies it in.  The B operand
// (the source symbols' bit planes) is built per tile in shared memory.
//
// Shared memory (from `ring`, 1024-aligned): kInStages input stages of
// 40,448 B, each covering kInSteps K-steps (16 input slices): the A image of
// those 4 K-steps (4 x 8 KiB: the two 8-row halves' 128 operand rows of 32
// B, one bulk copy) and the tile's symbols of those slices ([slice][240
// symbols], 7,680 B, one 2-D tensor copy); then kOpStages operand stages of
// kOpSteps K-steps of B rows (8 KiB slots of 7,680 B).  The MMAs read A from
// the input stage, so an input stage is free again when the MMAs of its last
// K-step have completed.  Both operands are K-major without swizzle: core
// matrices of 8 rows x 16 B, K halves 128 B apart, 8-row groups 256 B apart.
// TMEM: the two fp32 accumulators at columns 0 and 256 (240 columns each),
// scale factors 1.0 at 496-511.
#pragma once
#include <stdint.h>

namespace p2g {
namespace mma {

constexpr uint32_t kN = 240;        // symbols per tile (MMA N)
constexpr uint32_t kTileRows = 16;  // recovery rows per tile (two M = 128 MMAs)
constexpr uint32_t kKSlices = 4;    // input slices per K-step (K = 64 e2m1 values)
constexpr uint32_t kOpSteps = 4;    // K-steps per operand stage
constexpr int kOpStages = 2;
constexpr uint32_t kInSteps = 4;                     // K-steps per input stage
constexpr uint32_t kInSlices = kInSteps * kKSlices;  // 16 input slices per input stage
constexpr int kInStages = 3;
constexpr uint32_t kAccCol1 = 256;                // TMEM column of the second accumulator
constexpr uint32_t kSfaCol = 496, kSfbCol = 504;  // scale factors (all 1.0)
constexpr uint32_t kATileBytes = 4096;            // 128 rows x 32 B
constexpr uint32_t kAStepBytes = 2 * kATileBytes;  // both halves of one K-step
constexpr uint32_t kBTileBytes = kN * 32;         // 240 rows x 32 B
constexpr uint32_t kBSlotBytes = 8192;
constexpr uint32_t kOpStageBytes = kOpSteps * kBSlotBytes;
constexpr uint32_t kSrcSliceBytes = kN * 2;
constexpr uint32_t kInABytes = kInSteps * kAStepBytes;         // 32 KiB
constexpr uint32_t kInSrcBytes = kInSlices * kSrcSliceBytes;   // 7,680 B
constexpr uint32_t kInStageBytes = kInABytes + kInSrcBytes;    // 40,448 B
constexpr uint32_t kRingBytes = kInStages * kInStageBytes + kOpStages * kOpStageBytes;
constexpr uint32_t kGinvBytes = 1024;             // G^-1 tables: 256 lo then 256 hi u16
constexpr uint32_t kNumBars = 2 * kInStages + 2 * kOpStages + 3;
constexpr uint32_t kBarBytes = kNumBars * 8;
static_assert(kInStageBytes % 128 == 0 && kInABytes % 128 == 0, "tensor copies land 128-byte aligned");
static_assert(kBTileBytes <= kBSlotBytes, "B tile fits its slot");
constexpr uint32_t kOpPerIn = kInSteps / kOpSteps;  // operand stages per input stage
static_assert(kInSteps % kOpSteps == 0, "an input stage feeds whole operand stages");

// The A image in global memory: for 16-row tile rt and K-step k (slices 4k ..
// 4k+3), 8 KiB laid out as in shared memory -- byte
//   ((rt * ksteps + k) * 2 + t) * 4096 + grp * 256 + kh * 128 + m8 * 16
// holds operand row m = 8 grp + m8 of half t (recovery row 16 rt + 8 t + m /
// 16, bit i = m % 16), K half kh (slices 4k + 2kh, 4k + 2kh + 1): 8 e2m1
// bytes per slice, the spread of bits i..i+15 of T_c.  ksteps = a_image_steps
// (S): whole input stages, zero past S and R.
__host__ __device__ constexpr uint32_t a_image_steps(uint32_t S) {
    return (S + kInSlices - 1) / kInSlices * kInSteps;
}

// Instruction descriptor of kind::mxf4 with UE8M0 block scales: A and B
// e2m1 (format 1 at bits 7 and 10), K-major, N >> 3 at bit 17, scale format
// UE8M0 at bit 23, M >> 4 at bit 24, scale-factor ids 0, dense K = 64.
constexpr uint32_t kIdesc = (1u << 7) | (1u << 10) | ((kN >> 3) << 17) | (1u << 23) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when it gave up (it then sets the abort flag) or when
// another role has given up.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, volatile uint32_t* abort_flag) {
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        if (bar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 255u && *abort_flag) return false;
    }
    *abort_flag = 1u;
    return false;
}
// Waits (bounded) for a phase without looking at the abort flag: for
// copies and MMAs in flight, which land whatever happened elsewhere.
__device__ __forceinline__ void bar_drain(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 22) && !bar_try_wait(bar, parity); ++it) {
    }
}
__device__ __forceinline__ void tma_1d(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
// 2-D tiled tensor copy: the box at (x, y) of the tensor map `map` (a generic
// address of a CUtensorMap in kernel-parameter or global memory).  x times
// the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_2d(uint32_t dst, const void* map, int32_t x, int32_t y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
// Before the first copy through a tensor map that ordinary stores wrote to
// global memory (the batch job descriptors).
__device__ __forceinline__ void tensormap_acquire(const void* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Shared-memory matrix descriptor, K-major, no swizzle: start >> 4, leading
// (K-half) byte offset >> 4 at bit 16, stride (8-row group) byte offset >> 4
// at bit 32, version 1 at bit 46.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void mma_mxf4(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t sfa,
                                         uint32_t sfb, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %6, 0;\n"
        " tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%4], [%5], p;\n}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(kIdesc), "r"(sfa), "r"(sfb), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, uint32_t v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr), "r"(v)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// 16 bits -> 16 e2m1 values (0 or 1.0 = 0x2), 8 bytes.  Bit pairs (4q, 4q+1)
// go to byte q of the low word, pairs (4q+2, 4q+3) to byte q of the high
// word, each pair through a 4-entry byte table (PRMT).  A and B go through
// the same map, so K positions pair bit j with bit j.
__device__ __forceinline__ uint2 spread16(uint32_t x) {
    constexpr uint32_t kPairs = 0x22200200u;  // byte g = e2m1 pair of bits (g & 1, g >> 1)
    return make_uint2(__byte_perm(kPairs, 0u, x & 0x3333u), __byte_perm(kPairs, 0u, (x >> 2) & 0x3333u));
}
__device__ __forceinline__ void sts64(uint32_t addr, uint2 v) {
    asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(addr), "r"(v.x), "r"(v.y) : "memory");
}
__device__ __forceinline__ void sts128(uint32_t addr, uint2 lo, uint2 hi) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(lo.x), "r"(lo.y), "r"(hi.x), "r"(hi.y)
                 : "memory");
}
__device__ __forceinline__ uint32_t lds_b32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}
__device__ __forceinline__ uint32_t lds_u16(uint32_t addr) {
    uint16_t v;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(addr));
    return v;
}

// Barrier block: in_full[kInStages], in_empty[kInStages], op_full[kOpStages],
// op_empty[kOpStages], acc_full, acc_empty, drain.
struct Bars {
    uint32_t in_full, in_empty, op_full, op_empty, acc_full, acc_empty, drain;
    __device__ explicit Bars(uint32_t b)
        : in_full(b), in_empty(b + 8 * kInStages), op_full(b + 16 * kInStages),
          op_empty(b + 16 * kInStages + 8 * kOpStages), acc_full(b + 16 * kInStages + 16 * kOpStages),
          acc_empty(acc_full + 8), drain(acc_full + 16) {}
};
// One thread: counts for `ngen` operand-building warps.  An input stage is
// released by the MMA warp's commit after its last K-step (the builders have
// read it by then: the MMAs waited for their operands).
__device__ __forceinline__ void init_bars(uint32_t b, uint32_t ngen) {
    const Bars B(b);
    for (int i = 0; i < kInStages; ++i) {
        bar_init(B.in_full + 8 * i, 1);
        bar_init(B.in_empty + 8 * i, 1);
    }
    for (int i = 0; i < kOpStages; ++i) {
        bar_init(B.op_full + 8 * i, ngen);
        bar_init(B.op_empty + 8 * i, 1);
    }
    bar_init(B.acc_full, 1);
    bar_init(B.acc_empty, ngen);
    bar_init(B.drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// The whole of TMEM (one warp; the slot receives the base address), and
// given up again at the end by the same warp.
__device__ __forceinline__ void tmem_alloc(uint32_t slot) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(slot) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t tmem) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}
// Scale factors 1.0 (UE8M0 127) over the 32 lanes of warp quadrant q,
// columns 496..511 (called by four warps with distinct quadrants).
__device__ __forceinline__ void sf_fill(uint32_t tmem, uint32_t q) {
    const uint32_t t = tmem + ((32 * q) << 16) + kSfaCol;
    tmem_st8(t, 0x7F7F7F7Fu);
    tmem_st8(t + 8, 0x7F7F7F7Fu);
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// One tile: recovery rows [r0, r0+16) x symbols [n0, n0+syms) over input
// slices [s0, s0+sn), s0 a multiple of 16 and s0+sn a multiple of 4 or S.
// src_map: 2-D tensor map over the source (u16 symbols x input slices, the
// slice stride a multiple of 16 bytes; symbols and slices past its extent
// read 0); n0 is a multiple of 8.  aimg: the job's A image (ksteps =
// a_image_steps(S)).  accumulate: XOR the tile into the rows (the caller
// zeroed them) instead of storing it.
struct Tile {
    const void* src_map;
    const uint8_t* aimg;
    uint8_t* rec;
    uint64_t rec_stride;
    uint32_t s0, sn, ksteps, R, r0, n0, syms, accumulate;
};

// Per-CTA pipeline state, the same in every thread: operand stages, input
// stages, tiles and drains so far (ring positions and barrier parities follow
// from them).
struct Pipe {
    uint32_t ring, bars, tmem;
    const uint16_t* ginv;  // shared memory
    volatile uint32_t* abort_flag;
    uint32_t g, gi, tcount, drains;
    uint32_t pre;  // input stages of the coming tile already issued by the previous call
};

// All threads of the CTA call this.  Warp 0 lane 0 streams the inputs, warp
// 1 lane 0 issues the MMAs, warps 2 .. 2+NGEN-1 build the B operand and run
// the epilogue (the first eight of them; warp w reads TMEM lanes
// 32*(w%4)..).  Other warps idle.  Returns false (uniformly, after a CTA
// barrier) when a bounded wait gave up; copies and MMAs in flight have then
// landed.
// next_fn: called once, by the producer thread alone, after it has issued
// this tile's last input stage; it returns the tile this CTA runs next (it
// stays valid until the producer has issued its first stages), or null.
// The producer then issues that tile's first input stages while this tile's
// last K-steps and epilogue run, so the next tile starts without a copy
// round trip.  Only the producer thread's P.pre counts (the stages it issued
// ahead); the next call must be for that same tile.  When any role's wait
// gives up, the producer waits for every copy it issued, the next tile's
// included, before this returns.
template <int NGEN, class NextFn>
__device__ __forceinline__ bool run_tile(Pipe& P, const Tile& T, NextFn&& next_fn) {
    static_assert(NGEN >= 8, "eight warps cover the two accumulators' four lane quadrants");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Bars B(P.bars);
    const uint32_t in0 = P.ring, op0 = P.ring + kInStages * kInStageBytes;
    const uint32_t KS = (T.sn + kKSlices - 1) / kKSlices, NI = (KS + kInSteps - 1) / kInSteps;
    const uint32_t NS = (KS + kOpSteps - 1) / kOpSteps;  // operand stages
    const uint32_t g0 = P.g, gi0 = P.gi, tc = P.tcount, rt = T.r0 / kTileRows;
    // a tensor copy's x offset must be 16-byte aligned, the A image is cut in
    // whole input stages (the same in every thread)
    if ((T.n0 & 7u) || (T.s0 % kInSlices)) return false;
    // producer: the input-stage position after the last copy it issued and
    // has not drained (0: none), the next tile's first stages included
    uint32_t issued_end = 0;
    bool ok = true;
    if (warp == 0) {
        if (lane == 0) {
            // stages [0, P.pre) of this tile went out with the previous tile
            uint32_t gi = gi0 + P.pre;
            auto issue = [&](const Tile& U, uint32_t rtu, uint32_t k, uint32_t gi_) {
                const uint32_t st = gi_ % kInStages;
                if (!bar_wait(B.in_empty + 8 * st, ((gi_ / kInStages) & 1u) ^ 1u, P.abort_flag)) return false;
                const uint32_t sa = U.s0 + k * kInSlices;
                const uint32_t dst = in0 + st * kInStageBytes;
                bar_expect_tx(B.in_full + 8 * st, kInStageBytes);
                tma_1d(dst, U.aimg + ((size_t)rtu * U.ksteps + sa / kKSlices) * kAStepBytes, kInABytes,
                       B.in_full + 8 * st);
                tma_2d(dst + kInABytes, U.src_map, (int32_t)U.n0, (int32_t)sa, B.in_full + 8 * st);
                return true;
            };
            // slices past the tile's range (up to 15) are copied too: the
            // builders mask their B rows
            for (uint32_t k = P.pre; k < NI; ++k, ++gi)
                if (!issue(T, rt, k, gi)) {
                    ok = false;
                    break;
                }
            const Tile* U = ok ? next_fn() : nullptr;
            if (U && !(U->n0 & 7u) && !(U->s0 % kInSlices)) {
                const uint32_t NI_next = ((U->sn + kKSlices - 1) / kKSlices + kInSteps - 1) / kInSteps;
                const uint32_t want = NI_next < (uint32_t)kInStages ? NI_next : (uint32_t)kInStages;
                for (uint32_t k = 0; k < want; ++k, ++gi)
                    if (!issue(*U, U->r0 / kTileRows, k, gi)) {
                        ok = false;
                        break;
                    }
            }
            if (!ok) {  // copies issued but maybe not consumed land before the stages are reused
                for (uint32_t q = gi > gi0 + kInStages ? gi - kInStages : gi0; q < gi; ++q)
                    bar_drain(B.in_full + 8 * (q % kInStages), (q / kInStages) & 1u);
            } else {
                issued_end = gi;  // >= gi0 + NI: this tile's stages all went out
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const bool two = T.R - T.r0 > 8;
            if (!bar_wait(B.acc_empty, (tc & 1u) ^ 1u, P.abort_flag)) ok = false;
            tc_fence_after();
            uint32_t g = g0;
            for (uint32_t p = 0; ok && p < NS; ++p, ++g) {
                const uint32_t so = g % kOpStages, gi = gi0 + p / kOpPerIn, si = gi % kInStages;
                // the A rows were copied with the input stage, which the builders waited for
                if (!bar_wait(B.op_full + 8 * so, (g / kOpStages) & 1u, P.abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (uint32_t ks = 0; ks < kOpSteps; ++ks) {
                    const uint32_t k = p * kOpSteps + ks;
                    if (k >= KS) break;
                    const uint32_t a = in0 + si * kInStageBytes + ((p % kOpPerIn) * kOpSteps + ks) * kAStepBytes;
                    const uint64_t bdesc = smem_desc(op0 + so * kOpStageBytes + ks * kBSlotBytes, 128, 256);
                    mma_mxf4(P.tmem, smem_desc(a, 128, 256), bdesc, P.tmem + kSfaCol, P.tmem + kSfbCol, k > 0);
                    if (two)
                        mma_mxf4(P.tmem + kAccCol1, smem_desc(a + kATileBytes, 128, 256), bdesc, P.tmem + kSfaCol,
                                 P.tmem + kSfbCol, k > 0);
                }
                mma_commit(B.op_empty + 8 * so);
                if (p % kOpPerIn == kOpPerIn - 1 || p == NS - 1) mma_commit(B.in_empty + 8 * si);
            }
            if (ok) {
                mma_commit(B.acc_full);
            } else {  // every MMA issued completes before its stages or TMEM are reused
                mma_commit(B.drain);
                bar_drain(B.drain, P.drains & 1u);
            }
        }
    } else if (warp < 2 + NGEN) {
        const int gw = warp - 2;
        // A lane writes one 16-byte K half (2 slices) of one B row: symbols
        // m8 of 8-row group 2v+gsub, K half kh -- each quarter warp stores 128
        // contiguous bytes.  Per operand stage the builders share 15 warp
        // units per K-step (v = 0..14: the 30 8-row groups of the 240
        // symbols), dealt round-robin over the warps.  A unit: two 32-bit
        // loads from the input stage (the words holding symbol n of slices
        // 2kh and 2kh+1), the symbol's half, spread16, one 16-byte store.
        const uint32_t m8 = (uint32_t)lane & 7u, kh = ((uint32_t)lane >> 3) & 1u, gsub = (uint32_t)lane >> 4;
        const uint32_t lane_off = kh * 128 + m8 * 16;
        constexpr int kUnits = 15 * (int)kOpSteps;
        constexpr int kTasks = (kUnits + NGEN - 1) / NGEN;
        // fixed for the tile, per task: input offset (from the input stage,
        // first operand stage of the pair), operand offset (from the operand
        // stage), shift | slice within the operand stage << 8, and the
        // 2-bit-pair mask (0 for symbols past the tile).  Tasks past the units
        // load from offset 0 and store nothing.
        uint32_t t_in[kTasks], t_op[kTasks], t_fl[kTasks], t_m[kTasks];
#pragma unroll
        for (int j = 0; j < kTasks; ++j) {
            const uint32_t u = (uint32_t)gw + (uint32_t)j * NGEN;
            const uint32_t ks = u / 15u, v = u % 15u;
            const uint32_t grp = 2 * v + gsub, n = grp * 8 + m8;
            if (u >= (uint32_t)kUnits) {
                t_in[j] = t_op[j] = t_fl[j] = t_m[j] = 0;
            } else {
                t_in[j] = kInABytes + (ks * kKSlices + 2 * kh) * kSrcSliceBytes + ((n * 2) & ~3u);
                t_op[j] = ks * kBSlotBytes + grp * 256 + lane_off;
                t_fl[j] = ((n & 1u) * 16) | ((ks * kKSlices + 2 * kh) << 8);
                t_m[j] = n < T.syms ? 0x3333u : 0u;
            }
        }
        uint32_t g = g0;
        for (uint32_t p = 0; p < NS; ++p, ++g) {
            const uint32_t half = p % kOpPerIn, gi = gi0 + p / kOpPerIn, si = gi % kInStages, so = g % kOpStages;
            if ((half == 0 && !bar_wait(B.in_full + 8 * si, (gi / kInStages) & 1u, P.abort_flag)) ||
                !bar_wait(B.op_empty + 8 * so, ((g / kOpStages) & 1u) ^ 1u, P.abort_flag)) {
                ok = false;
                break;
            }
            // this operand stage's symbols: K-steps kOpSteps*half .. of the input stage
            const uint32_t ins = in0 + si * kInStageBytes + half * kOpSteps * kKSlices * kSrcSliceBytes;
            const uint32_t ops = op0 + so * kOpStageBytes;
            // slices of this operand stage: [first, first + 4 kOpSteps); past sn the K positions get 0
            const int32_t klim = (int32_t)T.sn - (int32_t)(p * kOpSteps * kKSlices);
            const bool full = klim >= (int32_t)(kOpSteps * kKSlices);
#pragma unroll
            for (int j = 0; j < kTasks; ++j) {
                const uint32_t fl = t_fl[j];
                const uint32_t a0 = ins + t_in[j];
                const uint32_t x0 = lds_b32(a0), x1 = lds_b32(a0 + kSrcSliceBytes);
                uint32_t m0 = t_m[j], m1 = t_m[j];
                if (!full) {
                    const int32_t sl = (int32_t)(fl >> 8);
                    if (sl >= klim) m0 = 0;
                    if (sl + 1 >= klim) m1 = 0;
                }
                const uint32_t sh = fl & 31u;
                // spread16 of 16 bits y: pairs (4q, 4q+1) from y & 0x3333, pairs (4q+2, 4q+3) from (y >> 2) & 0x3333
                constexpr uint32_t kPairs = 0x22200200u;
                const uint2 w0 = make_uint2(__byte_perm(kPairs, 0u, (x0 >> sh) & m0),
                                            __byte_perm(kPairs, 0u, (x0 >> (sh + 2)) & m0));
                const uint2 w1 = make_uint2(__byte_perm(kPairs, 0u, (x1 >> sh) & m1),
                                            __byte_perm(kPairs, 0u, (x1 >> (sh + 2)) & m1));
                if ((uint32_t)gw + (uint32_t)j * NGEN < (uint32_t)kUnits) sts128(ops + t_op[j], w0, w1);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) bar_arrive(B.op_full + 8 * so);
        }
        if (ok && !bar_wait(B.acc_full, tc & 1u, P.abort_flag)) ok = false;
        if (ok && gw < 8) {
            tc_fence_after();
            const uint32_t q = (uint32_t)warp & 3u, t = (uint32_t)gw >> 2;
            const uint32_t ra = T.r0 + 8 * t + 2 * q, rb = ra + 1;
            if (ra < T.R) {
                for (uint32_t c0 = 0; c0 < kN; c0 += 32) {
                    uint32_t v[32];
                    tmem_ld32(P.tmem + ((32 * q) << 16) + t * kAccCol1 + c0, v);
                    uint32_t mine = 0;
                    // parity of each count: the counts are integers below
                    // 16 * 32768 = 2^19, so in count + 2^23 the mantissa's
                    // lowest bit is the count's (one add, no conversion)
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const uint32_t par = __float_as_uint(__uint_as_float(v[j]) + 8388608.0f) & 1u;
                        const uint32_t b = __ballot_sync(0xFFFFFFFFu, par);
                        if (lane == j) mine = b;
                    }
                    // ballot lanes 0-15: the bits of row ra, lanes 16-31: row rb
                    const uint32_t col = c0 + (uint32_t)lane;
                    const uint32_t ya = mine & 0xFFFFu, yb = mine >> 16;
                    const uint32_t va = P.ginv[ya & 0xFFu] ^ P.ginv[256 + (ya >> 8)];
                    const uint32_t vb = rb < T.R ? P.ginv[yb & 0xFFu] ^ P.ginv[256 + (yb >> 8)] : 0u;
                    if (T.accumulate) {
                        // pairs of columns as 32-bit words (tiles start on an even symbol)
                        const uint32_t wa = va | (__shfl_down_sync(0xFFFFFFFFu, va, 1) << 16);
                        const uint32_t wb = vb | (__shfl_down_sync(0xFFFFFFFFu, vb, 1) << 16);
                        if (!(lane & 1) && col < T.syms) {
                            uint8_t* p = T.rec + (size_t)ra * T.rec_stride + (size_t)(T.n0 + col) * 2;
                            atomicXor(reinterpret_cast<unsigned int*>(p), wa);
                            if (rb < T.R) atomicXor(reinterpret_cast<unsigned int*>(p + T.rec_stride), wb);
                        }
                    } else if (col < T.syms) {
                        uint8_t* p = T.rec + (size_t)ra * T.rec_stride + (size_t)(T.n0 + col) * 2;
                        *reinterpret_cast<uint16_t*>(p) = (uint16_t)va;
                        if (rb < T.R) *reinterpret_cast<uint16_t*>(p + T.rec_stride) = (uint16_t)vb;
                    }
                }
            }
        }
        tc_fence_before();
        __syncwarp();
        if (ok && lane == 0) bar_arrive(B.acc_empty);
    }
    const bool bad = __syncthreads_or(!ok) != 0;
    if (bad && issued_end) {
        // another role gave up: the copies the producer issued (this tile's
        // last stages, the next tile's first) land before the stages are
        // reused or the CTA exits
        for (uint32_t q = issued_end - kInStages; q < issued_end; ++q)
            if (q >= gi0) bar_drain(B.in_full + 8 * (q % kInStages), (q / kInStages) & 1u);
    }
    P.g += NS;
    P.gi += NI;
    P.pre = bad || !issued_end ? 0u : issued_end - gi0 - NI;
    P.tcount += 1;
    if (bad) P.drains += 1;
    return !bad;
}

}  // namespace mma
}  // namespace p2g
