// p2g_batch.cpp -- batched create: many independent create jobs in one
// persistent, graph-captured launch (p2g_batch_* in include/par2gpu.h).
//
// Planning.  Each job becomes work items: scan items (slice MD5 + CRC32 of
// up to kScanSlices slices), encode items (one row group x one symbol tile
// over all of the job's input slices) and, for a job without recovery rows,
// one finish item.  A job's finish step (hash16k, file ids, set id, packet
// MD5s) runs on the CTA that completes its last encode item.
//
// Autotuning.  Items are popped in a fixed order by whichever CTA is free,
// so the launch is list scheduling.  The planner simulates it with a cost
// model (per-slice encode cost ~ tile + 384 shared-memory wavefronts at 78%
// of peak, ~0.72 us per 64-byte MD5 block of a chain) for the queue order
// "longest item + tail first", then searches each large job's tile width
// (1x, 2x, 4x, 8x its minimum tile count) for the shortest simulated makespan.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <queue>
#include <tuple>
#include <vector>

#include "p2g_host_util.h"
#include "p2g_internal.h"

namespace p2g {
namespace {

// Calibrated on the persistent kernel's per-item timelines: an encode item
// costs 0.62 us per slice plus 0.433 ns per symbol and slice (1.49 ms for
// 1027 slices x 1920 symbols, 0.187 ms for 256 x 256), a folded tail item
// 15 % more, an accumulating item 4 % more; a scan chain steps 64 bytes in
// 0.76 us, a packet chain in 0.81 us; CRC32 streams at ~10 GB/s per CTA.
constexpr double kEncRate = 2.309e6;    // symbols per ms per CTA, per slice
constexpr double kBuildCost = 1430.0;   // per-slice fixed cost (table build, barrier, copy wait) in symbols
constexpr double kChainMs = 7.6e-4;         // one MD5 chain step of 64 bytes
constexpr double kFoldCost = 1.15, kAccCost = 1.04;
// A finer tiling or a tail split must beat the current plan by 3 % in the
// simulation: the model is good to a few percent, and smaller pieces cost
// more in ways it does not see.
constexpr double kPlanMargin = 0.97;
constexpr double kItemMs = 0.003;          // pop, descriptor loads, pipeline fill

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }
// Device bytes a batch may spend on precomputed coefficient bases
// (P2G_BATCH_BASIS_BUDGET overrides; default 16 GiB).
uint64_t basis_budget() {
    const char* e = getenv("P2G_BATCH_BASIS_BUDGET");
    return e ? strtoull(e, nullptr, 10) : (16ull << 30);
}
inline double md5_ms(uint64_t bytes) { return (double)((bytes + 8) / 64 + 1) * kChainMs; }

struct PlanJob {
    uint64_t slice = 0;
    uint32_t S = 0, R = 0, n = 0, RG = 0, Np = 0;
    uint32_t ts = 0, tiles = 0;  // chosen tiling
    double finish = 0;           // finish-step estimate
    // work the job needs (all by default): slice checksums, the set-id item,
    // packet-MD5 chains
    bool scans = true, set_id = true, chains = true;
    uint64_t file_bytes = 0;  // largest file, when whole-file MD5 items run (0: none)
    // Tail split (single job with chains; the caller zeroes the columns of the
    // split bands): the encode items of the last split_bands bands are cut
    // into split_chunks slice ranges that XOR-accumulate into the rows.
    // split_chunks 0: the caller does not zero, never split.
    uint32_t split_bands = 0, split_chunks = 0;
    // Encode on the tensor cores: 16-row x 240-symbol items (kItemEncodeMma);
    // RG then counts 16-row tiles and ts is fixed at 240.
    bool mma = false;
};

double finish_ms(const PlanJob& j) { return est_set_id_ms(j.n) + est_packet_item_ms(j.slice, j.R); }
inline double encode_ms(const PlanJob& j, uint32_t syms) {
    return j.mma ? est_mma_item_ms(j.S) : est_encode_item_ms(j.S, syms);
}
inline double scan_ms(const PlanJob& j, uint32_t count) { return est_scan_item_ms(j.slice, count); }

void set_tiling(PlanJob& j, uint32_t tiles) {
    const uint32_t ts = (uint32_t)std::min<uint64_t>(round_up((j.Np + tiles - 1) / tiles, 8), kEncTileSymbols);
    j.ts = ts;
    j.tiles = (j.Np + ts - 1) / ts;
}
inline uint32_t min_tiles(const PlanJob& j) { return (j.Np + kEncTileSymbols - 1) / kEncTileSymbols; }

struct Plan {
    std::vector<BatchItem> items;
    std::vector<std::vector<uint32_t>> band_items;  // per job: encode items of each band
    std::vector<uint32_t> band_syms;                // per job
    uint32_t n_scan = 0, n_crc = 0, n_enc = 0, n_setid = 0;
    double makespan = 0;
};

constexpr uint32_t kMaxBands = 64;  // packet-MD5 chain segments per job (64: 10.27 ms vs 10.59 at 16 for 538 MB / R 200)

// Bands of job j: runs of band_tiles consecutive tiles, a multiple of the
// tail fold so that no folded item straddles two bands.
void job_bands(const PlanJob& j, uint32_t* band_tiles, uint32_t* n_bands) {
    const uint32_t F = j.mma ? 1u : tail_fold(j.R);
    uint32_t bt = std::max<uint32_t>(1, (j.tiles + kMaxBands - 1) / kMaxBands);
    bt = (bt + F - 1) / F * F;
    *band_tiles = bt;
    *n_bands = (j.tiles + bt - 1) / bt;
}
// one chain segment of every 256-row block over one band's bytes
inline double chain_ms(const PlanJob& j, uint32_t band_syms) {
    return ceil(j.R / (double)kChainRows) * md5_ms(2ull * band_syms) * 1.07 + kItemMs;
}

// Items of all jobs in queue order: every job's set-id item (its chains wait
// for it), then the MD5 scan items, longest first, then the encode items job
// by job (largest job first), band by band, tile-major within a band so a
// tile's row groups run together and share its source reads in L2, and last
// the short CRC items, which fill the ragged final round of the encode.  A
// folded item covers the last row group of `fold` adjacent tiles.
Plan build_items(const std::vector<PlanJob>& jobs) {
    Plan p;
    p.band_items.resize(jobs.size());
    p.band_syms.assign(jobs.size(), 0);
    std::vector<std::pair<double, BatchItem>> pre, post;
    struct JobItems {
        double key;
        uint32_t job;
        std::vector<BatchItem> items;
    };
    std::vector<JobItems> enc;
    for (uint32_t ji = 0; ji < (uint32_t)jobs.size(); ++ji) {
        const PlanJob& j = jobs[ji];
        if (j.set_id) {
            pre.push_back({1e30, {ji, kItemSetId, 0, 0, 0, 0}});
            p.n_setid++;
        }
        for (uint32_t f = 0; j.file_bytes && f < j.n; f += kScanSlices)  // longest chains: right after set ids
            pre.push_back({1e29, {ji, kItemFileHash, f, std::min(kScanSlices, j.n - f), 0, 0}});
        for (uint32_t s = 0; j.scans && s < j.S; s += kScanSlices) {
            const uint32_t cnt = std::min(kScanSlices, j.S - s);
            pre.push_back({scan_ms(j, cnt), {ji, kItemScan, s, cnt, 0, 0}});
            p.n_scan++;
        }
        const uint32_t cper = crc_item_slices(j.slice);
        for (uint32_t s = 0; j.scans && s < j.S; s += cper) {
            const uint32_t cnt = std::min(cper, j.S - s);
            post.push_back({est_crc_item_ms(j.slice, cnt), {ji, kItemCrc, s, cnt, 0, 0}});
            p.n_crc++;
        }
        if (!j.R) continue;
        uint32_t bt = 0, nb = 0;
        job_bands(j, &bt, &nb);
        const uint32_t F = j.mma ? 1u : tail_fold(j.R);
        p.band_syms[ji] = bt * j.ts;
        p.band_items[ji].assign(nb, 0);
        std::vector<uint32_t>& counts = p.band_items[ji];
        JobItems e{0.0, ji, {}};
        const uint32_t first_split = j.chains && j.split_chunks > 1 && j.split_bands
                                         ? nb - std::min(nb, j.split_bands) : nb;
        for (uint32_t b = 0; b < nb; ++b) {
            const uint32_t t0 = b * bt, t1 = std::min(j.tiles, t0 + bt);
            const uint32_t C = b >= first_split ? j.split_chunks : 1;
            // tensor-core ranges start on whole 16-slice stages of the A image
            const uint32_t cs = j.mma ? ((j.S + C - 1) / C + 15) / 16 * 16 : (j.S + C - 1) / C;
            auto push = [&](uint32_t rg, uint32_t fold, uint32_t n0, uint32_t syms) {
                for (uint32_t s0 = 0; s0 < j.S; s0 += cs) {
                    const uint32_t sn = C > 1 ? std::min(cs, j.S - s0) : 0;
                    e.items.push_back({ji, encode_kind(rg, fold, C > 1), n0, (b << 16) | syms, s0, sn});
                    e.key += est_encode_item_ms(sn ? sn : j.S, std::min(j.ts, syms));
                    counts[b]++;
                }
            };
            if (j.mma) {  // tile-major: the row tiles of one symbol tile share its source reads in L2
                for (uint32_t t = t0; t < t1; ++t) {
                    const uint32_t n0 = t * j.ts, syms = std::min(j.ts, j.Np - n0);
                    for (uint32_t rt = 0; rt < j.RG; ++rt)
                        for (uint32_t s0 = 0; s0 < j.S; s0 += cs) {
                            const uint32_t sn = C > 1 ? std::min(cs, j.S - s0) : 0;
                            e.items.push_back({ji, encode_mma_kind(rt, C > 1), n0, (b << 16) | syms, s0, sn});
                            e.key += est_mma_item_ms(sn ? sn : j.S);
                            counts[b]++;
                        }
                }
                continue;
            }
            for (uint32_t t = t0; t < t1; ++t) {
                const uint32_t n0 = t * j.ts, syms = std::min(j.ts, j.Np - n0);
                for (uint32_t rg = 0; rg + 1 < j.RG; ++rg) push(rg, 1, n0, syms);
                if ((t - t0) % F == 0) {
                    const uint32_t end = std::min(std::min((t + F) * j.ts, t1 * j.ts), j.Np);
                    push(j.RG - 1, F, n0, end - n0);
                }
            }
        }
        if (j.chains) {
            e.key += nb * chain_ms(j, p.band_syms[ji]);
        } else {  // no chain segments: the encode items count nothing
            counts.clear();
            p.band_syms[ji] = 0;
        }
        p.n_enc += (uint32_t)e.items.size();
        enc.push_back(std::move(e));
    }
    std::stable_sort(pre.begin(), pre.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::stable_sort(enc.begin(), enc.end(), [](const JobItems& a, const JobItems& b) {
        if (a.key != b.key) return a.key > b.key;
        return a.job < b.job;
    });
    std::stable_sort(post.begin(), post.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    for (auto& x : pre) p.items.push_back(x.second);
    for (auto& e : enc) p.items.insert(p.items.end(), e.items.begin(), e.items.end());
    for (auto& x : post) p.items.push_back(x.second);
    return p;
}

double item_ms(const PlanJob& j, const BatchItem& it) {
    switch (it.kind_rg & kItemKindMask) {
    case kItemScan: return scan_ms(j, it.b);
    case kItemCrc: return est_crc_item_ms(j.slice, it.b);
    case kItemFileHash: return md5_ms(j.file_bytes) + kItemMs;
    case kItemEncodeMma:
        return est_mma_item_ms(it.sn ? it.sn : j.S) * ((it.kind_rg & kItemAccumulate) ? kAccCost : 1.0);
    case kItemEncode: {
        double ms = est_encode_item_ms(it.sn ? it.sn : j.S, std::min(j.ts, it.b & 0xFFFFu));
        if ((it.kind_rg >> 24) & 3u) ms *= kFoldCost;
        if (it.kind_rg & kItemAccumulate) ms *= kAccCost;
        return ms;
    }
    default: return est_set_id_ms(j.n);
    }
}

// List-scheduling simulation: each item goes to the CTA that frees first.
// A job's packet chains advance band by band in order: band b's segment
// starts when the band's last item ends and the previous segment is done.
// (The advancing CTA's time is charged to it when the chain was waiting for
// that band; a band that completes while the chain is busy is picked up by
// the chain's holder.)
double simulate(const std::vector<PlanJob>& jobs, const Plan& p, uint32_t ctas) {
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    for (uint32_t c = 0; c < ctas; ++c) free_at.push(0.0);
    std::vector<std::vector<uint32_t>> left = p.band_items;
    std::vector<std::vector<double>> done(jobs.size());
    for (size_t ji = 0; ji < jobs.size(); ++ji) done[ji].assign(p.band_items[ji].size(), 0.0);
    double end = 0;
    for (const BatchItem& it : p.items) {
        double t = free_at.top();
        free_at.pop();
        const PlanJob& j = jobs[it.job];
        t += item_ms(j, it);
        const uint32_t kd = it.kind_rg & kItemKindMask;
        if ((kd == kItemEncode || kd == kItemEncodeMma) && !left[it.job].empty()) {
            const uint32_t b = it.b >> 16;
            done[it.job][b] = std::max(done[it.job][b], t);
            --left[it.job][b];
        }
        end = std::max(end, t);
        free_at.push(t);
    }
    for (size_t ji = 0; ji < jobs.size(); ++ji) {
        double chain = 0;
        for (double d : done[ji]) chain = std::max(chain, d) + chain_ms(jobs[ji], p.band_syms[ji]);
        end = std::max(end, chain);
    }
    return end;
}

Plan plan_tiles(std::vector<PlanJob>& jobs, uint32_t ctas, uint32_t flags);

// A job alone with packet chains: its items run in rounds of equal length,
// so several bands complete together at the end of each round and the last
// round leaves the chains a burst of bands to hash after the encode is done.
// Cutting the items of the last bands into slice ranges spreads their
// completions out; the simulation picks how many bands and how many pieces.
Plan plan_batch(std::vector<PlanJob>& jobs, uint32_t ctas, uint32_t flags) {
    Plan best = plan_tiles(jobs, ctas, flags);
    if (jobs.size() != 1 || !jobs[0].split_chunks || !jobs[0].chains || !jobs[0].R ||
        (flags & P2G_BATCH_NO_AUTOTUNE))
        return best;
    PlanJob& j = jobs[0];
    const uint32_t nb = (uint32_t)best.band_items[0].size();
    if (nb < 2) {
        j.split_bands = 0;
        j.split_chunks = 1;
        return best;
    }
    const uint32_t per_band = std::max(1u, best.band_items[0][0]);
    const uint32_t wave = std::max(1u, (ctas + per_band - 1) / per_band);
    uint32_t bb = 0, bc = 1;
    for (uint32_t bands : {wave, 2 * wave, 3 * wave, 4 * wave, nb / 2, nb}) {
        for (uint32_t chunks : {2u, 4u, 8u}) {
            j.split_bands = std::min(bands, nb);
            j.split_chunks = chunks;
            Plan p = build_items(jobs);
            p.makespan = simulate(jobs, p, ctas);
            if (p.makespan < best.makespan * kPlanMargin) {
                best = std::move(p);
                bb = j.split_bands;
                bc = chunks;
            }
        }
    }
    j.split_bands = bb;
    j.split_chunks = bc;
    return best;
}

Plan plan_tiles(std::vector<PlanJob>& jobs, uint32_t ctas, uint32_t flags) {
    for (PlanJob& j : jobs) {
        j.split_bands = 0;  // tiles are chosen unsplit

        j.Np = (uint32_t)(round_up(j.slice, 16) / 2);
        j.finish = finish_ms(j);
        if (j.mma) {  // fixed tile: one MMA N wide, 16 rows (two M = 128 halves) high
            j.RG = (j.R + kMmaTileRows - 1) / kMmaTileRows;
            j.ts = kMmaTileSymbols;
            j.tiles = (j.Np + j.ts - 1) / j.ts;
            continue;
        }
        j.RG = (j.R + kRowsPerGroup - 1) / kRowsPerGroup;
        set_tiling(j, min_tiles(j));
        if (jobs.size() == 1 && j.R && !(flags & P2G_BATCH_NO_AUTOTUNE)) {
            // alone on the GPU, equal items run in rounds of the CTAs that
            // the (long) MD5 scan items leave free: take the tile count with
            // the fewest, fullest rounds (choose_tiles)
            const uint32_t scans = j.scans ? (j.S + kScanSlices - 1) / kScanSlices : 0;
            const uint32_t free_ctas = ctas > scans + 16 ? ctas - scans : ctas;
            uint32_t ts = 0, tiles = 0;
            choose_tiles(j.Np, j.RG, free_ctas, &ts, &tiles, tail_fold(j.R));
            j.ts = ts;
            j.tiles = tiles;
        }
    }
    Plan best = build_items(jobs);
    best.makespan = simulate(jobs, best, ctas);
    if (flags & P2G_BATCH_NO_AUTOTUNE) return best;
    // lower bound at the widest tiles: all work spread evenly over the CTAs
    double total = 0;
    for (const BatchItem& it : best.items) total += item_ms(jobs[it.job], it);
    for (uint32_t ji = 0; ji < (uint32_t)jobs.size(); ++ji)
        total += best.band_items[ji].size() * chain_ms(jobs[ji], best.band_syms[ji]);
    const double bound = total / ctas;
    if (best.makespan <= 1.02 * bound) return best;
    // try finer tilings for the jobs with the longest encode items
    std::vector<uint32_t> order;
    for (uint32_t i = 0; i < (uint32_t)jobs.size(); ++i)
        if (jobs[i].R && !jobs[i].mma) order.push_back(i);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return encode_ms(jobs[a], jobs[a].ts) > encode_ms(jobs[b], jobs[b].ts);
    });
    if (order.size() > 24) order.resize(24);
    for (uint32_t ji : order) {
        PlanJob& j = jobs[ji];
        const uint32_t base = min_tiles(j), keep = j.tiles;
        uint32_t best_tiles = keep;
        for (uint32_t mult : {2u, 4u, 8u}) {
            const uint32_t t = base * mult;
            if ((j.Np + t - 1) / t < 64) continue;  // tiles too small to pay for their table builds
            set_tiling(j, t);
            Plan p = build_items(jobs);
            p.makespan = simulate(jobs, p, ctas);
            if (p.makespan < best.makespan * kPlanMargin) {
                best = std::move(p);
                best_tiles = j.tiles;
            }
        }
        set_tiling(j, best_tiles);
        if (best.makespan <= 1.02 * bound) break;
    }
    return best;
}

}  // namespace

double est_md5_ms(uint64_t bytes) { return md5_ms(bytes); }
// A tensor-core item: one K-step (4 slices) of operand building and two
// MMAs, plus the pipeline fill and the epilogue.
// Per 4-slice K-step and per tile on one SM, from the standalone kernel on
// 14,209 tiles of 16 rows x 240 symbols (96 per SM): 1.93 ms at 256 slices,
// 5.38 ms at 1,024.
constexpr double kMmaStepMs = 1.87e-4, kMmaFixedMs = 0.005;
double est_mma_item_ms(uint32_t slices) { return (slices + 3) / 4 * kMmaStepMs + kMmaFixedMs + kItemMs; }
// Whether a job's encode runs on the tensor cores: by the cost of its items
// on a full GPU (the lookup kernel folds a short last row group; the tensor
// tiles are 16 rows high and 240 symbols wide).
// CTA-milliseconds of a job's encode items on either kernel.
double encode_cost_ms(uint64_t slice, uint32_t S, uint32_t R, bool mma) {
    if (!R || !S) return 0;
    const uint32_t Np = (uint32_t)(round_up(slice, 16) / 2);
    if (mma)
        return (double)((Np + kMmaTileSymbols - 1) / kMmaTileSymbols) * ((R + kMmaTileRows - 1) / kMmaTileRows) *
               est_mma_item_ms(S);
    const uint32_t RG = (R + kRowsPerGroup - 1) / kRowsPerGroup, F = tail_fold(R);
    return (double)((Np + kEncTileSymbols - 1) / kEncTileSymbols) * (RG - 1 + (F > 1 ? kFoldCost / F : 1.0)) *
           est_encode_item_ms(S, std::min<uint32_t>(Np, kEncTileSymbols));
}
bool prefer_mma(uint64_t slice, uint32_t S, uint32_t R) {
    return R && S && encode_cost_ms(slice, S, R, true) < encode_cost_ms(slice, S, R, false);
}
double est_encode_item_ms(uint32_t slices, uint32_t syms) {
    return (double)slices * (round_up(syms, 8) + kBuildCost) / kEncRate + kItemMs;
}
double est_scan_item_ms(uint64_t slice, uint32_t count) {
    (void)count;  // the lanes run their chains side by side
    return md5_ms(slice) + kItemMs;
}
// CRC32 streams from DRAM at ~10 GB/s per SM (16 warps)
double est_crc_item_ms(uint64_t slice, uint32_t count) { return (double)slice * count / 1e7 + kItemMs; }
double est_set_id_ms(uint32_t files) {
    const double hashes = ceil(files / 256.0) * (md5_ms(P2G_HASH16K_LEN) + md5_ms(24 + 256));
    const double sort = (double)files * files / 512.0 * 4e-6;
    return hashes + sort + md5_ms(12 + 16ull * files) + kItemMs;
}
double est_packet_item_ms(uint64_t slice, uint32_t rows) { return ceil(rows / 256.0) * md5_ms(36 + slice) + kItemMs; }

// Plans depend only on the job's shape, and the search (tilings, tail
// splits, each simulated) costs milliseconds of host time, so single-job
// plans are kept per shape: repeated jobs of one shape plan once.
namespace {
struct PlanKey {
    uint64_t slice, file_bytes;
    uint32_t S, R, n, ctas, flags;
    bool operator<(const PlanKey& o) const {
        return std::tie(slice, file_bytes, S, R, n, ctas, flags) <
               std::tie(o.slice, o.file_bytes, o.S, o.R, o.n, o.ctas, o.flags);
    }
};
std::mutex g_plan_mu;
std::map<PlanKey, SingleJobPlan> g_plans;
size_t g_plan_items = 0;                    // items held by the cached plans
constexpr size_t kMaxCachedPlans = 256;
constexpr size_t kMaxCachedItems = 1u << 20;  // 24 MiB of items
SingleJobPlan plan_single_job_uncached(uint64_t slice, uint32_t S, uint32_t R, uint32_t n_files, bool scans,
                                       bool set_id, bool chains, uint32_t ctas, uint64_t file_bytes,
                                       bool split_tail, bool mma);
}  // namespace

SingleJobPlan plan_single_job(uint64_t slice, uint32_t S, uint32_t R, uint32_t n_files, bool scans, bool set_id,
                              bool chains, uint32_t ctas, uint64_t file_bytes, bool split_tail, bool mma) {
    const PlanKey key{slice, file_bytes, S, R, n_files, ctas,
                      (scans ? 1u : 0u) | (set_id ? 2u : 0u) | (chains ? 4u : 0u) | (split_tail ? 8u : 0u) |
                          (mma ? 16u : 0u)};
    {
        std::lock_guard<std::mutex> lk(g_plan_mu);
        auto it = g_plans.find(key);
        if (it != g_plans.end()) return it->second;
    }
    SingleJobPlan p =
        plan_single_job_uncached(slice, S, R, n_files, scans, set_id, chains, ctas, file_bytes, split_tail, mma);
    std::lock_guard<std::mutex> lk(g_plan_mu);
    if (g_plans.size() >= kMaxCachedPlans || g_plan_items + p.items.size() > kMaxCachedItems) {
        g_plans.clear();
        g_plan_items = 0;
    }
    if (g_plans.emplace(key, p).second) g_plan_items += p.items.size();
    return p;
}

namespace {
SingleJobPlan plan_single_job_uncached(uint64_t slice, uint32_t S, uint32_t R, uint32_t n_files, bool scans,
                                       bool set_id, bool chains, uint32_t ctas, uint64_t file_bytes,
                                       bool split_tail, bool mma) {
    std::vector<PlanJob> jobs(1);
    jobs[0].mma = mma && R;
    jobs[0].slice = slice;
    jobs[0].S = S;
    jobs[0].R = R;
    jobs[0].n = std::max(1u, n_files);
    jobs[0].scans = scans;
    jobs[0].set_id = set_id;
    jobs[0].chains = chains && R;
    jobs[0].file_bytes = file_bytes;
    jobs[0].split_chunks = split_tail ? 1 : 0;  // non-zero: the split search may run
    Plan p = plan_batch(jobs, ctas, 0);
    SingleJobPlan out;
    out.zero_from_sym = jobs[0].Np;
    if (jobs[0].split_chunks > 1 && jobs[0].split_bands) {
        const uint32_t nb = (uint32_t)p.band_items[0].size();
        out.zero_from_sym = (nb - std::min(nb, jobs[0].split_bands)) * p.band_syms[0];
    }
    out.items = std::move(p.items);
    out.band_items = p.band_items[0];
    out.band_syms = p.band_syms[0];
    out.ts = jobs[0].ts;
    out.predicted_ms = p.makespan;
    return out;
}
}  // namespace

// ---------------------------------------------------------------------------
// The batch object
// ---------------------------------------------------------------------------
}  // namespace p2g

struct p2g_batch {
    int device = -1;
    uint32_t flags = 0;
    uint32_t n_jobs = 0, n_items = 0, ctas = 0;
    p2g::Plan plan;
    std::vector<p2g::PlanJob> shape;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    p2g::BatchJob* d_jobs = nullptr;
    p2g::BatchItem* d_items = nullptr;
    uint32_t* d_ctl = nullptr;  // queue head, per-job chain state, then the error word
    uint64_t err_word = 0;      // index of the error word in d_ctl
    size_t ctl_bytes = 0;
    uint64_t max_basis_words = 0;
    uint64_t max_aimg_bytes = 0;  // tensor-core jobs: largest A image to fill per run
    struct Realign {
        const uint8_t* src;
        uint8_t* dst;
        uint64_t slice, estride;
        uint32_t S;
    };
    std::vector<Realign> realigns;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t kernels_per_run = 0;
};

namespace p2g {
namespace {

p2g_status enqueue_run(p2g_batch* b, cudaStream_t st) {
    int* err = reinterpret_cast<int*>(b->d_ctl + b->err_word);
    P2G_CU(cudaMemsetAsync(b->d_ctl, 0, b->ctl_bytes, st));
    if (b->max_basis_words) P2G_CU(launch_basis_batch(b->d_jobs, b->n_jobs, b->max_basis_words, st));
    if (b->max_aimg_bytes) P2G_CU(launch_a_image_batch(b->d_jobs, b->n_jobs, b->max_aimg_bytes, st));
    for (const auto& r : b->realigns) P2G_CU(launch_realign(r.src, r.slice, r.dst, r.estride, r.S, r.slice, st));
    P2G_CU(launch_batch(b->d_jobs, b->d_items, b->n_items, b->d_ctl, err, b->ctas, st, b->max_aimg_bytes != 0));
    return P2G_OK;
}

void release(p2g_batch* b) {
    if (!b) return;
    if (b->device >= 0) cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->arena) cudaFree(b->arena);
    delete b;
}

void fill_info(const p2g_batch* b, p2g_batch_info* out) {
    out->jobs = b->n_jobs;
    out->items = b->n_items;
    out->encode_items = b->plan.n_enc;
    out->scan_items = b->plan.n_scan + b->plan.n_crc;
    out->setid_items = b->plan.n_setid;
    out->ctas = b->ctas;
    out->predicted_ms = b->plan.makespan;
    out->device_bytes = b->arena_bytes;
}

}  // namespace
}  // namespace p2g

using namespace p2g;

extern "C" p2g_status p2g_plan_device_job(uint64_t slice_size, uint32_t input_slices, uint32_t recovery_count,
                                          uint32_t file_count, uint32_t with_chains, uint32_t ctas,
                                          p2g_plan_item* items, uint32_t cap, uint32_t* n_items,
                                          uint32_t* zero_from_symbol, uint32_t* band_count) {
    clear_error();
    if (!ctas || !input_slices || input_slices > P2G_MAX_INPUT_BLOCKS || (cap && !items))
        return set_error(P2G_ERR_INVALID_ARGUMENT, "plan needs ctas > 0, 1..32768 input slices and an item array");
    P2G_TRY(check_common(std::max(1u, file_count), recovery_count, slice_size));
    // as run_device_job_persistent plans a job with device slice checksums, a
    // device set id and hash_full off the device; P2G_TAIL_SPLIT=0 turns the
    // tail split off there and here alike
    const char* ts = getenv("P2G_TAIL_SPLIT");
    const bool split_tail = !(ts && !strcmp(ts, "0"));
    // the encode kernel the job would use (P2G_ENCODE_VARIANT, else the cost model)
    const char* ev = getenv("P2G_ENCODE_VARIANT");
    const bool mma = ev && !strcmp(ev, "tensor") ? true
                     : ev && !strcmp(ev, "lut")  ? false
                                                 : prefer_mma(slice_size, input_slices, recovery_count);
    const SingleJobPlan pl = plan_single_job(slice_size, input_slices, recovery_count, std::max(1u, file_count),
                                             true, true, with_chains && recovery_count, ctas, 0, split_tail,
                                             mma && recovery_count);
    uint32_t n = 0;
    for (const BatchItem& it : pl.items) {
        const uint32_t kind = it.kind_rg & kItemKindMask;
        if (kind != kItemEncode && kind != kItemEncodeMma) continue;
        if (n < cap)
            items[n] = {(it.kind_rg >> 8) & 0xFFFFu, kind == kItemEncodeMma ? 0u : 1u << ((it.kind_rg >> 24) & 3u),
                        it.a, it.b & 0xFFFFu, it.b >> 16, it.s0, it.sn ? it.sn : input_slices,
                        (it.kind_rg & kItemAccumulate) ? 1u : 0u};
        ++n;
    }
    if (n_items) *n_items = n;
    if (zero_from_symbol) *zero_from_symbol = pl.zero_from_sym;
    if (band_count) *band_count = (uint32_t)pl.band_items.size();
    return P2G_OK;
}

extern "C" p2g_status p2g_batch_plan(const p2g_batch_shape* shapes, uint32_t n, uint32_t ctas, uint32_t flags,
                                     p2g_batch_info* info, uint32_t* tiles_out) {
    clear_error();
    if (!shapes || !n || !ctas) return set_error(P2G_ERR_INVALID_ARGUMENT, "batch plan needs shapes and ctas > 0");
    std::vector<PlanJob> jobs(n);
    for (uint32_t i = 0; i < n; ++i) {
        P2G_TRY(check_common(std::max(1u, shapes[i].file_count), shapes[i].recovery_count, shapes[i].slice_size));
        if (!shapes[i].input_slices || shapes[i].input_slices > P2G_MAX_INPUT_BLOCKS)
            return set_error(P2G_ERR_INVALID_ARGUMENT, "job %u: input slice count must be in [1, 32768]", i);
        jobs[i].slice = shapes[i].slice_size;
        jobs[i].S = shapes[i].input_slices;
        jobs[i].R = shapes[i].recovery_count;
        jobs[i].n = std::max(1u, shapes[i].file_count);
    }
    const Plan p = plan_batch(jobs, ctas, flags);
    if (info) {
        p2g_batch tmp;
        tmp.n_jobs = n;
        tmp.n_items = (uint32_t)p.items.size();
        tmp.ctas = ctas;
        tmp.plan = p;
        fill_info(&tmp, info);
    }
    if (tiles_out)
        for (uint32_t i = 0; i < n; ++i) tiles_out[i] = jobs[i].R ? jobs[i].ts : 0;
    return P2G_OK;
}

extern "C" p2g_status p2g_batch_create(const p2g_batch_job* jobs, uint32_t n, uint32_t flags, p2g_batch** out) {
    clear_error();
    if (!out) return set_error(P2G_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!jobs || !n) return set_error(P2G_ERR_INVALID_ARGUMENT, "a batch needs at least one job");
    if (n > 65535) return set_error(P2G_ERR_INVALID_ARGUMENT, "a batch holds at most 65535 jobs");
    // ---- validation (as p2g_run_device_job) ----
    std::vector<PlanJob> shape(n);
    uint64_t total_files = 0, names_bytes = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const p2g_batch_job& jb = jobs[i];
        P2G_TRY(check_common(jb.file_count, jb.recovery_count, jb.slice_size));
        if (!jb.src || (uintptr_t)jb.src % 16 || !jb.checksums || !jb.hash16k || !jb.set_id ||
            (uintptr_t)jb.set_id % 4 || !jb.file_lengths || !jb.names || !jb.name_lens)
            return set_error(P2G_ERR_INVALID_ARGUMENT,
                             "batch job %u: src (16-byte aligned), checksums, hash16k, set_id (4-byte aligned), "
                             "file lengths and names are required", i);
        if (jb.recovery_count && (!jb.recovery || !jb.packet_md5 || (uintptr_t)jb.recovery % 16 ||
                                  jb.recovery_stride % 16 || jb.recovery_stride < round_up(jb.slice_size, 16)))
            return set_error(P2G_ERR_INVALID_ARGUMENT,
                             "batch job %u: recovery rows need a 16-byte aligned buffer, recovery_stride a multiple "
                             "of 16 and >= round_up(slice,16), and packet_md5", i);
        uint64_t S = 0, total = 0;
        for (uint32_t f = 0; f < jb.file_count; ++f) {
            P2G_TRY(check_name(jb.names[f], jb.name_lens[f], ""));
            if (jb.file_lengths[f] == 0) return set_error(P2G_ERR_EMPTY_FILE, "batch job %u: input file %u is empty", i, f);
            S += (jb.file_lengths[f] + jb.slice_size - 1) / jb.slice_size;
            total += jb.file_lengths[f];
            names_bytes += round_up(jb.name_lens[f], 4);
        }
        P2G_TRY(check_total_blocks(S, total, jb.slice_size));
        total_files += jb.file_count;
        shape[i].slice = jb.slice_size;
        shape[i].S = (uint32_t)S;
        shape[i].R = jb.recovery_count;
        shape[i].n = jb.file_count;
        if (jb.hash_full) {
            if ((uintptr_t)jb.hash_full % 4)
                return set_error(P2G_ERR_INVALID_ARGUMENT, "batch job %u: hash_full must be 4-byte aligned", i);
            for (uint32_t f = 0; f < jb.file_count; ++f)
                shape[i].file_bytes = std::max<uint64_t>(shape[i].file_bytes, jb.file_lengths[f]);
        }
    }
    // One encode kernel for the whole launch: forced by the flags (or
    // P2G_ENCODE_VARIANT), else the one the cost model prefers for the
    // batch's total encode work.  Lookup and tensor-core items are not mixed
    // in one launch: mixed launches gave wrong recovery bytes for a few
    // tensor-core tiles, and with the proxy fences between item kinds a
    // 256-job mixed launch still ran into a bounded wait (each kind alone is
    // bit-exact).
    const char* ev = getenv("P2G_ENCODE_VARIANT");
    bool use_mma;
    if (flags & P2G_BATCH_TENSOR) {
        use_mma = true;
    } else if (flags & P2G_BATCH_LUT) {
        use_mma = false;
    } else if (ev && (!strcmp(ev, "tensor") || !strcmp(ev, "lut"))) {
        use_mma = !strcmp(ev, "tensor");
    } else {
        double lut = 0, mma = 0;
        for (uint32_t i = 0; i < n; ++i) {
            lut += encode_cost_ms(shape[i].slice, shape[i].S, shape[i].R, false);
            mma += encode_cost_ms(shape[i].slice, shape[i].S, shape[i].R, true);
        }
        use_mma = mma < lut;
    }
    for (uint32_t i = 0; i < n; ++i) shape[i].mma = use_mma && shape[i].R;
    P2G_TRY(ensure_device_ready());
    p2g_batch* b = new p2g_batch();
    cudaGetDevice(&b->device);
    b->flags = flags;
    b->n_jobs = n;
    b->ctas = (uint32_t)device_sm_count();
    b->plan = plan_batch(shape, b->ctas, flags);
    b->shape = shape;
    b->n_items = (uint32_t)b->plan.items.size();

    // ---- device arena: descriptors, items, queue, tables, scratch, bases ----
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = round_up(off + bytes, 256);
        return o;
    };
    const size_t o_jobs = take(sizeof(BatchJob) * n);
    const size_t o_items = take(sizeof(BatchItem) * b->n_items);
    // control block, zeroed before each run: queue head, each job's chain
    // state (band counts, next band and token per 256-row block, set-id flag),
    // then the error word
    std::vector<uint64_t> bstate_off(n);
    uint64_t ctl_words = 1;
    for (uint32_t i = 0; i < n; ++i) {
        bstate_off[i] = ctl_words;
        const uint32_t Q = (shape[i].R + kChainRows - 1) / kChainRows;
        ctl_words += b->plan.band_items[i].size() + 2 * Q + 1;
    }
    b->err_word = ctl_words;
    b->ctl_bytes = sizeof(uint32_t) * (ctl_words + 1);
    const size_t o_ctl = take(b->ctl_bytes);
    std::vector<size_t> o_bands(n), o_chain(n);
    for (uint32_t i = 0; i < n; ++i) {
        o_bands[i] = take(4 * std::max<size_t>(1, b->plan.band_items[i].size()));
        o_chain[i] = take(16ull * std::max(1u, shape[i].R));
    }
    const size_t o_files = take(16 * total_files);
    const size_t o_noff = take(8 * total_files);
    const size_t o_names = take(names_bytes);
    // Precomputed bases load faster (a derived basis adds ~6% to an encode
    // item) but take S x row groups x 1 KiB each: keep them while they fit.
    uint64_t basis_total = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (shape[i].R && !shape[i].mma) basis_total += basis_bytes(shape[i].S, shape[i].RG);
    const bool load_basis = !(flags & P2G_BATCH_DERIVE_BASIS) && basis_total <= basis_budget();
    std::vector<size_t> o_scratch(n), o_basis(n, 0), o_real(n, 0), o_aimg(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        o_scratch[i] = take(32ull * shape[i].n + 12);
        if (shape[i].mma) o_aimg[i] = take(mma_aimg_bytes(shape[i].S, shape[i].R));
        if (load_basis && shape[i].R && !shape[i].mma) o_basis[i] = take(basis_bytes(shape[i].S, shape[i].RG));
        if (shape[i].R && jobs[i].slice_size % 16) o_real[i] = take(round_up(jobs[i].slice_size, 16) * shape[i].S);
    }
    b->arena_bytes = off;
    cudaError_t e = cudaMalloc(&b->arena, off);
    if (e != cudaSuccess) {
        release(b);
        return cuda_fail(e, "batch arena");
    }
    uint8_t* A = static_cast<uint8_t*>(b->arena);
    b->d_jobs = reinterpret_cast<BatchJob*>(A + o_jobs);
    b->d_items = reinterpret_cast<BatchItem*>(A + o_items);
    b->d_ctl = reinterpret_cast<uint32_t*>(A + o_ctl);

    // ---- host images of the tables ----
    std::vector<BatchJob> hj(n);
    std::vector<uint64_t> hfiles(2 * total_files);
    std::vector<uint32_t> hnoff(2 * total_files);
    std::vector<uint8_t> hnames(names_bytes, 0);
    uint64_t fcur = 0, ncur = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const p2g_batch_job& jb = jobs[i];
        BatchJob& d = hj[i];
        memset(&d, 0, sizeof d);
        d.src = jb.src;
        d.slice = jb.slice_size;
        d.S = shape[i].S;
        d.R = jb.recovery_count;
        d.RG = shape[i].RG;
        d.n_files = jb.file_count;
        d.rec = jb.recovery;
        d.rec_stride = jb.recovery_stride;
        d.checks = jb.checksums;
        d.h16k = jb.hash16k;
        d.pkt = jb.packet_md5;
        d.set_id = jb.set_id;
        d.hfull = jb.hash_full;
        d.files = reinterpret_cast<const uint64_t*>(A + o_files) + 2 * fcur;
        d.name_off = reinterpret_cast<const uint32_t*>(A + o_noff) + 2 * fcur;
        d.names = A + o_names;
        d.scratch = A + o_scratch[i];
        d.n_bands = (uint32_t)b->plan.band_items[i].size();
        d.band_syms = b->plan.band_syms[i];
        d.ts = shape[i].ts;
        d.bstate = b->d_ctl + bstate_off[i];
        d.band_items = reinterpret_cast<const uint32_t*>(A + o_bands[i]);
        d.chain = reinterpret_cast<uint32_t*>(A + o_chain[i]);
        d.first_exp = 0;
        d.vec = jb.slice_size % 16 == 0 ? 1u : 0u;
        d.basis = load_basis && d.R && !shape[i].mma ? reinterpret_cast<uint16_t*>(A + o_basis[i]) : nullptr;
        if (d.R && jb.slice_size % 16) {
            d.esrc = A + o_real[i];
            d.estride = round_up(jb.slice_size, 16);
            b->realigns.push_back({jb.src, A + o_real[i], jb.slice_size, d.estride, d.S});
        } else {
            d.esrc = jb.src;
            d.estride = jb.slice_size;
        }
        if (shape[i].mma) {
            d.mma = 1;
            d.Rpad = (d.R + kMmaTileRows - 1) / kMmaTileRows * kMmaTileRows;
            d.ksteps = mma_image_steps(d.S);
            d.aimg = A + o_aimg[i];
            b->max_aimg_bytes = std::max<uint64_t>(b->max_aimg_bytes, mma_aimg_bytes(d.S, d.R));
            if (e == cudaSuccess) e = make_src_map(&d.src_map, d.esrc, d.estride, d.S, (uint32_t)(d.estride / 2));
        }
        if (d.basis) b->max_basis_words = std::max<uint64_t>(b->max_basis_words, (uint64_t)d.S * d.RG * 512);
        uint64_t first = 0;
        for (uint32_t f = 0; f < jb.file_count; ++f, ++fcur) {
            hfiles[2 * fcur] = first * jb.slice_size;
            hfiles[2 * fcur + 1] = jb.file_lengths[f];
            first += (jb.file_lengths[f] + jb.slice_size - 1) / jb.slice_size;
            hnoff[2 * fcur] = (uint32_t)ncur;
            hnoff[2 * fcur + 1] = (uint32_t)jb.name_lens[f];
            memcpy(hnames.data() + ncur, jb.names[f], jb.name_lens[f]);
            ncur += round_up(jb.name_lens[f], 4);
        }
    }
    auto up = [&](size_t o, const void* src, size_t bytes) {
        return bytes ? cudaMemcpy(A + o, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i)
        if (!b->plan.band_items[i].empty())
            e = cudaMemcpy(A + o_bands[i], b->plan.band_items[i].data(), 4 * b->plan.band_items[i].size(),
                           cudaMemcpyHostToDevice);
    if (e != cudaSuccess || (e = up(o_jobs, hj.data(), sizeof(BatchJob) * n)) != cudaSuccess ||
        (e = up(o_items, b->plan.items.data(), sizeof(BatchItem) * b->n_items)) != cudaSuccess ||
        (e = up(o_files, hfiles.data(), 8 * hfiles.size())) != cudaSuccess ||
        (e = up(o_noff, hnoff.data(), 4 * hnoff.size())) != cudaSuccess ||
        (e = up(o_names, hnames.data(), hnames.size())) != cudaSuccess) {
        release(b);
        return cuda_fail(e, "batch tables upload");
    }
    b->kernels_per_run = 1 + (b->max_basis_words ? 1 : 0) + (b->max_aimg_bytes ? 1 : 0) + (uint32_t)b->realigns.size();

    // ---- capture the run into a CUDA graph ----
    if (!(flags & P2G_BATCH_NO_GRAPH)) {
        if ((e = prepare_batch_kernel()) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking)) != cudaSuccess) {
            release(b);
            return cuda_fail(e, "batch graph stream");
        }
        if ((e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
            release(b);
            return cuda_fail(e, "batch graph capture");
        }
        const p2g_status s = enqueue_run(b, b->cap);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(b->cap, &g);
        b->graph = g;
        if (s != P2G_OK) {
            release(b);
            return s;
        }
        if (e != cudaSuccess || (e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) {
            release(b);
            return cuda_fail(e, "batch graph instantiate");
        }
    }
    *out = b;
    return P2G_OK;
}

extern "C" p2g_status p2g_batch_launch(p2g_batch* b, void* stream) {
    clear_error();
    if (!b) return set_error(P2G_ERR_INVALID_ARGUMENT, "batch is NULL");
    P2G_CU(cudaSetDevice(b->device));
    const cudaStream_t st = (cudaStream_t)stream;
    if (b->exec) {
        P2G_CU(cudaGraphLaunch(b->exec, st));
        add_launches(b->kernels_per_run);
        return P2G_OK;
    }
    return enqueue_run(b, st);
}

extern "C" p2g_status p2g_batch_check(p2g_batch* b) {
    clear_error();
    if (!b) return set_error(P2G_ERR_INVALID_ARGUMENT, "batch is NULL");
    P2G_CU(cudaSetDevice(b->device));
    int h = 0;
    P2G_CU(cudaMemcpy(&h, b->d_ctl + b->err_word, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) return set_error(P2G_ERR_TIMEOUT, "a bounded device wait gave up in the batch kernel (TMA stage never completed)");
    return P2G_OK;
}

extern "C" p2g_status p2g_batch_get_info(const p2g_batch* b, p2g_batch_info* out) {
    clear_error();
    if (!b || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "batch or out is NULL");
    fill_info(b, out);
    return P2G_OK;
}

extern "C" uint32_t p2g_batch_job_tile(const p2g_batch* b, uint32_t job) {
    if (!b || job >= b->n_jobs || !b->shape[job].R) return 0;
    return b->shape[job].ts;
}

extern "C" void p2g_batch_destroy(p2g_batch* b) { release(b); }
