// p2g_mma.cu -- the Reed-Solomon accumulator on the tensor cores (tcgen05,
// kind::mxf4), as a bit-sliced GF(2) product.
//
// recovery[r] = XOR_s c(r,s) * source[s] over GF(2^16) (src/reedsolomon.rs:
// 87-126, src/creator.rs:934-1007).  Multiplication by a constant c is
// GF(2)-linear on the 16 bits of a symbol.  With the trace form
// G[i][j] = Tr(a^(i+j)) (a = 2) multiplication is self-adjoint, which gives
//
//     bits(c * x) = G^-1 H_c bits(x),   H_c[i][j] = Tr(c * a^(i+j)),
//
// and H_c is a Hankel matrix: its row i is bits i..i+15 of the 31-bit trace
// string T_c = sum_{k<31} Tr(c a^k) 2^k.  So one recovery symbol is
//
//     rec[r][n] = G^-1 ( parity of  sum_s sum_j H_c(r,s)[i][j] * bit_j(src[s][n]) )_i ,
//
// an integer matrix product D = A * B^T with 0/1 entries:
//     A[(r,i), (s,j)] = bit (i+j) of T_c(r,s)       (M = 16 rows per recovery row)
//     B[n, (s,j)]     = bit j of src[s][n]           (N = symbols)
// summed over K = 16 S, of which only the parity is kept.  0 and 1 are exact
// e2m1 values (1.0 = 0x2), all scale factors are 1.0 (UE8M0 127), and the
// fp32 accumulator holds the sums exactly (at most 16 * 32768 < 2^24).
//
// Tile: 16 recovery rows (two M = 128 MMAs, 8 rows x 16 bits each) x 240
// symbols (N), accumulated in TMEM over all input slices, K-step = 4 slices
// (K = 64 e2m1 values = 32 bytes per operand row).  a_image_kernel first
// writes the A operand of the whole job to global memory (R x S x 128 bytes,
// built once instead of once per symbol tile).  Warp roles:
//   warp 0       TMA producer: per 16 input slices, one bulk copy of their A
//                rows and one 2-D tensor copy of the tile's source symbols
//   warp 1       TMEM allocation; lane 0 issues the MMAs and commits
//   warps 2..15  B operand builders (source symbols spread to e2m1 in the
//                canonical K-major layout, 16-byte K halves), then (warps
//                2..9) the epilogue: tcgen05.ld of the sums, parity, one
//                ballot per column (= two recovery symbols), G^-1, store.
// The tile pipeline itself is p2g_mma_tile.cuh, shared with the persistent
// batch kernel's tensor-core items.
// Every mbarrier wait is bounded; a wait that gives up sets the error flag,
// stops all roles, drains copies and MMAs in flight and frees TMEM.
#include <mutex>

#include "p2g_internal.h"
#include "p2g_mma_tile.cuh"

namespace p2g {

// T_c = d_trace_lo[c & 255] ^ d_trace_hi[c >> 8]; G^-1 y likewise from two
// 256-entry tables of 16-bit columns, d_ginv[0..255] for the low byte of y
// and d_ginv[256..511] for the high byte.
__device__ uint32_t d_trace_lo[256], d_trace_hi[256];
__device__ uint16_t d_ginv[512];

namespace {

using namespace mma;
constexpr int kGenWarps = 15;  // 60 B units per operand stage: four each
constexpr int kThreads = 64 + 32 * kGenWarps;

// shared memory layout (bytes): the rings, G^-1 tables, barriers, misc
constexpr uint32_t kOffOp = 0;
constexpr uint32_t kOffIn = kOffOp + kOpStages * kOpStageBytes;
constexpr uint32_t kOffGinv = kRingBytes;
constexpr uint32_t kOffBars = kOffGinv + kGinvBytes;
constexpr uint32_t kOffMisc = kOffBars + kBarBytes;
constexpr uint32_t kSmemBytes = kOffMisc + 16;
static_assert(kSmemBytes > 116 * 1024, "one CTA per SM: TMEM is allocated whole");
static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");
static_assert(mma_image_steps(1027) == a_image_steps(1027) && mma_image_steps(32) == a_image_steps(32),
              "host and device agree on the A image layout");

}  // namespace

// Trace string of the coefficient c(r,s) = base_s ^ (first_exp + r) =
// 2^(logbase_s * (first_exp + r) mod 65535) (RsEncoder::coefficient,
// src/reedsolomon.rs:56-60; gf_pow src/galois.rs:74-87).
__device__ __forceinline__ uint32_t coef_trace(uint32_t s, uint32_t r, uint32_t first_exp,
                                               const uint16_t* __restrict__ antilog,
                                               const uint16_t* __restrict__ logbase) {
    const uint32_t e = (first_exp + r) % kFieldLimit;
    uint32_t k = (uint32_t)logbase[s] * e;  // < 2^32
    k = (k & 0xFFFFu) + (k >> 16);
    k = (k & 0xFFFFu) + (k >> 16);
    if (k >= kFieldLimit) k -= kFieldLimit;
    const uint32_t c = antilog[k];
    return d_trace_lo[c & 0xFFu] ^ d_trace_hi[c >> 8];
}

// The A image of one job (layout: a_image_steps in p2g_mma_tile.cuh), one
// 16-byte K half of an operand row per step of the loop: rows of recovery
// row r >= R and slices s >= S are 0.
__device__ __forceinline__ void fill_a_image(uint8_t* __restrict__ aimg, uint32_t S, uint32_t R, uint32_t first_exp,
                                             const uint16_t* __restrict__ antilog,
                                             const uint16_t* __restrict__ logbase, uint64_t i0, uint64_t step) {
    const uint32_t ksteps = a_image_steps(S), n_row = (R + kTileRows - 1) / kTileRows;
    const uint64_t total = (uint64_t)n_row * ksteps * (kAStepBytes / 16);
    for (uint64_t i = i0; i < total; i += step) {
        const uint32_t c = (uint32_t)(i % (kAStepBytes / 16));  // byte c*16 = t*4096 + grp*256 + kh*128 + m8*16
        const uint64_t q = i / (kAStepBytes / 16);
        const uint32_t k = (uint32_t)(q % ksteps), rt = (uint32_t)(q / ksteps);
        const uint32_t t = c >> 8, grp = (c >> 4) & 15u, kh = (c >> 3) & 1u, m8 = c & 7u;
        const uint32_t m = grp * 8 + m8, r = rt * kTileRows + 8 * t + (m >> 4), bit = m & 15u;
        const uint32_t s0 = k * kKSlices + 2 * kh;
        const uint32_t T0 = (r < R && s0 < S) ? coef_trace(s0, r, first_exp, antilog, logbase) : 0u;
        const uint32_t T1 = (r < R && s0 + 1 < S) ? coef_trace(s0 + 1, r, first_exp, antilog, logbase) : 0u;
        const uint2 v0 = spread16((T0 >> bit) & 0xFFFFu), v1 = spread16((T1 >> bit) & 0xFFFFu);
        reinterpret_cast<uint4*>(aimg)[i] = make_uint4(v0.x, v0.y, v1.x, v1.y);
    }
}

__global__ void a_image_kernel(uint8_t* __restrict__ aimg, const uint16_t* __restrict__ antilog,
                               const uint16_t* __restrict__ logbase, uint32_t S, uint32_t R, uint32_t first_exp) {
    fill_a_image(aimg, S, R, first_exp, antilog, logbase, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x,
                 (uint64_t)gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(kThreads, 1)
    encode_mma_kernel(const __grid_constant__ CUtensorMap src_map, uint32_t S, uint32_t Np,
                      const uint8_t* __restrict__ aimg, uint32_t R, uint8_t* __restrict__ rec,
                      uint64_t rec_stride, uint32_t n_row_tiles, uint32_t n_tiles, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    uint16_t* ginv = reinterpret_cast<uint16_t*>(smem + kOffGinv);  // [0,256) lo, [256,512) hi
    uint32_t* misc = reinterpret_cast<uint32_t*>(smem + kOffMisc);  // [0] TMEM base, [1] abort
    mma::Pipe P;
    P.ring = smem_addr(smem + kOffOp);
    P.bars = smem_addr(smem + kOffBars);
    P.ginv = ginv;
    P.abort_flag = misc + 1;
    P.g = P.gi = P.tcount = P.drains = P.pre = 0;
    if (tid == 0) {
        init_bars(P.bars, kGenWarps);
        misc[1] = 0;
    }
    for (int i = tid; i < 512; i += kThreads) ginv[i] = d_ginv[i];
    if (warp == 1) tmem_alloc(smem_addr(misc));  // the whole of TMEM: two accumulators and the scale factors
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    P.tmem = misc[0];
    if (warp >= 4 && warp < 8) sf_fill(P.tmem, (uint32_t)warp & 3u);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // tiles in order of symbol tile, row tile fastest: concurrent CTAs share
    // their source bytes in L2
    bool ok = true;
    auto tile_of = [&](uint32_t tile) {
        Tile T;
        T.src_map = &src_map;
        T.aimg = aimg;
        T.rec = rec;
        T.rec_stride = rec_stride;
        T.s0 = 0;
        T.sn = S;
        T.ksteps = a_image_steps(S);
        T.R = R;
        T.r0 = (tile % n_row_tiles) * kTileRows;
        T.n0 = (tile / n_row_tiles) * kN;
        T.syms = min(kN, Np - T.n0);
        T.accumulate = 0;
        return T;
    };
    for (uint32_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x) {
        const Tile T = tile_of(tile);
        const uint32_t nt = tile + gridDim.x;
        Tile Tn;
        ok = run_tile<kGenWarps>(P, T, [&]() -> const Tile* {
            if (nt >= n_tiles) return nullptr;
            Tn = tile_of(nt);
            return &Tn;
        });
    }
    if (tid == 0 && !ok) atomicOr(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_free(P.tmem);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {
// Trace strings and G^-1 from the field itself (polynomial 0x1100B,
// generator 2).  Returns false if G were singular (it never is).
bool build_trace_tables(uint32_t tlo[256], uint32_t thi[256], uint16_t glo[256], uint16_t ghi[256]) {
    std::vector<uint32_t> al(65536), lg(65536);
    uint32_t b = 1;
    for (uint32_t l = 0; l < kFieldLimit; ++l) {
        al[l] = b;
        lg[b] = l;
        b <<= 1;
        if (b & 0x10000u) b ^= kFieldGenerator;
    }
    auto mul = [&](uint32_t x, uint32_t y) -> uint32_t {
        return (x && y) ? al[(lg[x] + lg[y]) % kFieldLimit] : 0u;
    };
    auto trace = [&](uint32_t y) {  // y + y^2 + ... + y^(2^15), in {0, 1}
        uint32_t acc = y, z = y;
        for (int i = 0; i < 15; ++i) {
            z = mul(z, z);
            acc ^= z;
        }
        return acc;
    };
    uint32_t tr[47];
    for (uint32_t k = 0; k < 47; ++k) tr[k] = trace(al[k]);
    uint32_t tbit[16];  // T of the basis element 2^b
    for (uint32_t bb = 0; bb < 16; ++bb) {
        tbit[bb] = 0;
        for (uint32_t k = 0; k < 31; ++k) tbit[bb] |= (tr[bb + k] & 1u) << k;
    }
    // G[i][j] = Tr(a^(i+j)); invert over GF(2): rows as 32-bit [G | I]
    uint32_t rows[16];
    for (uint32_t i = 0; i < 16; ++i) {
        rows[i] = 1u << (16 + i);
        for (uint32_t j = 0; j < 16; ++j) rows[i] |= (tr[i + j] & 1u) << j;
    }
    for (uint32_t c = 0; c < 16; ++c) {
        uint32_t p = c;
        while (p < 16 && !((rows[p] >> c) & 1u)) ++p;
        if (p == 16) return false;
        std::swap(rows[c], rows[p]);
        for (uint32_t r = 0; r < 16; ++r)
            if (r != c && ((rows[r] >> c) & 1u)) rows[r] ^= rows[c];
    }
    uint16_t gcol[16];  // column j of G^-1 as a 16-bit vector over i
    for (uint32_t j = 0; j < 16; ++j) {
        gcol[j] = 0;
        for (uint32_t i = 0; i < 16; ++i) gcol[j] |= (uint16_t)(((rows[i] >> (16 + j)) & 1u) << i);
    }
    for (uint32_t v = 0; v < 256; ++v) {
        tlo[v] = thi[v] = 0;
        glo[v] = ghi[v] = 0;
        for (uint32_t bb = 0; bb < 8; ++bb)
            if ((v >> bb) & 1u) {
                tlo[v] ^= tbit[bb];
                thi[v] ^= tbit[bb + 8];
                glo[v] ^= gcol[bb];
                ghi[v] ^= gcol[bb + 8];
            }
    }
    return true;
}

cudaError_t mma_prepare() {
    static std::mutex mu;
    static bool done[256] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 256 && done[dev]) return cudaSuccess;
    static uint32_t tlo[256], thi[256];
    static uint16_t glo[256], ghi[256];
    if (!build_trace_tables(tlo, thi, glo, ghi)) return cudaErrorInvalidValue;
    if ((e = cudaMemcpyToSymbol(d_trace_lo, tlo, sizeof tlo)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(d_trace_hi, thi, sizeof thi)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(d_ginv, glo, sizeof glo)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(d_ginv, ghi, sizeof ghi, sizeof glo)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(encode_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes)) !=
        cudaSuccess)
        return e;
    if (dev >= 0 && dev < 256) done[dev] = true;
    return cudaSuccess;
}
}  // namespace

cudaError_t mma_tables_ready(const uint16_t** ginv) {
    cudaError_t e = mma_prepare();
    if (e != cudaSuccess) return e;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, d_ginv);
    *ginv = static_cast<const uint16_t*>(p);
    return e;
}

// The A images of every tensor-core job of a batch (blockIdx.y = job).
__global__ void a_image_batch_kernel(const BatchJob* __restrict__ jobs, const uint16_t* __restrict__ antilog,
                                     const uint16_t* __restrict__ logbase) {
    const BatchJob& J = jobs[blockIdx.y];
    if (!J.mma || !J.R || !J.aimg) return;
    fill_a_image(J.aimg, J.S, J.R, J.first_exp, antilog, logbase, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x,
                 (uint64_t)gridDim.x * blockDim.x);
}

cudaError_t launch_a_image_batch(const BatchJob* jobs, uint32_t n_jobs, uint64_t max_bytes, cudaStream_t st) {
    if (!n_jobs || !max_bytes) return cudaSuccess;
    const uint16_t* g = nullptr;
    cudaError_t e = mma_tables_ready(&g);
    if (e != cudaSuccess) return e;
    const uint16_t *antilog = nullptr, *logbase = nullptr;
    if ((e = gf_device_tables(&antilog, &logbase)) != cudaSuccess) return e;
    const uint64_t want = (max_bytes / 16 + 255) / 256;
    const unsigned bx = (unsigned)std::min<uint64_t>(want, (uint64_t)device_sm_count() * 8);
    a_image_batch_kernel<<<dim3(bx, n_jobs), 256, 0, st>>>(jobs, antilog, logbase);
    add_launches(1);
    return cudaGetLastError();
}

size_t mma_aimg_bytes(uint32_t S, uint32_t R) {
    return (size_t)((R + kTileRows - 1) / kTileRows) * a_image_steps(S) * kAStepBytes;
}

// The source as a 2-D tensor of u16 symbols: Np symbols per input slice, S
// slices `stride` bytes apart (16-byte aligned base and stride), read in
// boxes of 240 symbols x 16 slices, zeros past either extent.
cudaError_t make_src_map(CUtensorMap* map, const void* src, uint64_t stride, uint32_t S, uint32_t Np) {
    using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                     const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeTiled encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<EncodeTiled>(fn);
    });
    if (!encode) return cudaErrorNotSupported;
    if ((uintptr_t)src % 16 || stride % 16 || !S || !Np) return cudaErrorInvalidValue;
    const cuuint64_t dims[2] = {Np, S};
    const cuuint64_t strides[1] = {stride};
    const cuuint32_t box[2] = {kN, kInSlices};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void*>(src), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_encode_mma(const uint8_t* src, uint64_t src_stride, uint32_t S, uint64_t slice_size, uint32_t R,
                              uint32_t first_exp, uint8_t* aimg, uint8_t* rec, uint64_t rec_stride, int* err,
                              cudaStream_t st) {
    if (!S || !R) return cudaSuccess;
    cudaError_t e = mma_prepare();
    if (e != cudaSuccess) return e;
    const uint16_t *antilog = nullptr, *logbase = nullptr;
    if ((e = gf_device_tables(&antilog, &logbase)) != cudaSuccess) return e;
    const uint32_t Np = (uint32_t)(((slice_size + 15) & ~15ull) / 2);
    CUtensorMap map;
    if ((e = make_src_map(&map, src, src_stride, S, Np)) != cudaSuccess) return e;
    const uint32_t n_row = (R + kTileRows - 1) / kTileRows;
    const uint32_t n_sym = (Np + kN - 1) / kN;
    const uint64_t chunks = mma_aimg_bytes(S, R) / 16;
    const int sms = device_sm_count();
    const unsigned cb = (unsigned)std::min<uint64_t>((chunks + 255) / 256, (uint64_t)sms * 8);
    a_image_kernel<<<cb, 256, 0, st>>>(aimg, antilog, logbase, S, R, first_exp);
    add_launches(1);
    const uint64_t tiles = (uint64_t)n_sym * n_row;
    const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)sms);
    encode_mma_kernel<<<grid, kThreads, kSmemBytes, st>>>(map, S, Np, aimg, R, rec, rec_stride, n_row,
                                                          (uint32_t)tiles, err);
    add_launches(1);
    return cudaGetLastError();
}

}  // namespace p2g
