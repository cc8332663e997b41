// p2g_server.cpp -- serving loop: create jobs admitted as they arrive, with
// continuous batching on the device (p2g_server_* in include/par2gpu.h).
//
// Admission.  Requests wait in arrival order until their footprint (padded
// source + recovery rows) fits the HBM budget beside the jobs already
// resident and a descriptor slot is free.  Admission allocates the job's
// device memory from the stream-ordered pool, brings its source in (H2D
// copy or seeded generation), zeroes its recovery rows and uploads its
// descriptor, all on the copy stream, then records a ready event.
//
// Waves.  The device runs a sequence of persistent batch-kernel launches
// ("waves", ~wave_ms of work each, two in flight).  Each wave takes work
// items from every resident job whose source is ready, a fair share per job
// (processor sharing), so a request that arrives while others run starts in
// the next wave instead of waiting for them to finish.  A job's items:
//   scan    slice MD5 + CRC32, 256 slices per item
//   set id  hash16k, file ids, set id
//   encode  (row group, symbol tile, slice chunk); chunks of one tile XOR
//           into zeroed rows, so no item runs longer than ~wave_ms/4
//   packet  recovery-packet MD5s of up to 256 rows, issued once every
//           encode item and the set-id item of the job have completed
// A job is complete when its last item's wave has completed; its outputs
// stay in device memory until the caller releases it.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "p2g_host_util.h"
#include "p2g_internal.h"

namespace p2g {
namespace {

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

constexpr int kWaveBufs = 3;        // item buffers (two waves in flight + one being built)
constexpr uint32_t kWaveItems = 1u << 16;

struct SJob {
    uint64_t ticket = 0, tag = 0;
    // request
    std::vector<uint64_t> lens, seeds;
    std::vector<std::string> names;
    uint64_t slice = 0;
    uint32_t S = 0, R = 0, RG = 0, Np = 0, n = 0;
    uint32_t source_kind = 0;
    const uint8_t* host_src = nullptr;
    uint64_t source_bytes = 0, footprint = 0;
    // encode on the tensor cores (items of kind kItemEncodeMma); the job's A
    // image then lives in its device allocation (aimg_bytes)
    bool mma = false;
    uint64_t aimg_bytes = 0;
    // device memory (one allocation) and the tables uploaded with it
    void* mem = nullptr;
    BatchJob desc{};
    std::vector<uint64_t> h_files, h_fill;
    std::vector<uint32_t> h_noff;
    std::vector<uint8_t> h_names;
    uint32_t slot = ~0u;
    cudaEvent_t ready = nullptr;
    bool is_ready = false;
    // work
    std::deque<BatchItem> todo;    // scan, set-id and encode items not yet issued
    std::deque<double> todo_ms;    // estimated ms of each todo item
    uint32_t enc_total = 0, enc_done = 0, scan_total = 0, scan_done = 0;
    bool setid_done = false;
    uint32_t pkt_issued = 0, pkt_done = 0;  // rows
    uint32_t outstanding = 0;
    double enc_ms = 0, pkt_ms_per_item = 0;
    // state
    int state = 0;  // 0 queued, 1 resident, 2 complete, 3 released
    bool counted = false;  // footprint added to the resident bytes (admitted)
    int32_t status = P2G_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

struct Wave {
    cudaEvent_t ev = nullptr;
    int buf = 0;
    std::vector<std::pair<SJob*, BatchItem>> items;
};

}  // namespace
}  // namespace p2g

struct p2g_server {
    int device = -1;
    uint64_t budget = 0;
    double wave_ms = 0;
    uint32_t max_jobs = 0, ctas = 0;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread th;
    bool stop = false;
    p2g_status fatal = P2G_OK;
    std::string fatal_msg;
    uint64_t next_ticket = 1;
    std::deque<std::unique_ptr<p2g::SJob>> queue;  // waiting for admission
    std::vector<std::unique_ptr<p2g::SJob>> live;  // resident or complete, not released
    std::vector<uint32_t> free_slots;
    std::deque<p2g::SJob*> completed;             // not yet polled
    std::deque<p2g::Wave> inflight;
    uint64_t resident_bytes = 0, peak_bytes = 0;
    p2g_server_stats st{};
    cudaStream_t exec = nullptr, copy = nullptr;
    p2g::BatchJob* d_jobs = nullptr;
    p2g::BatchItem* d_items[p2g::kWaveBufs] = {};
    p2g::BatchItem* h_items[p2g::kWaveBufs] = {};
    uint32_t* d_ctl[p2g::kWaveBufs] = {};
    int* d_err = nullptr;
    int* h_err = nullptr;  // pinned, one word per wave buffer
    bool buf_busy[p2g::kWaveBufs] = {};
    uint32_t rr = 0;  // round-robin start for the next wave

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace p2g {
namespace {

p2g_status fail_cuda(p2g_server* s, cudaError_t e, const char* what) {
    cudaGetLastError();
    s->fatal = e == cudaErrorMemoryAllocation ? P2G_ERR_OOM : P2G_ERR_CUDA;
    s->fatal_msg = std::string(what) + ": " + cudaGetErrorString(e);
    return s->fatal;
}
#define SRV_CU(s, call)                                              \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return fail_cuda((s), _e, #call);     \
    } while (0)

// Items of a newly admitted job (all but the packet items).
void plan_job(p2g_server* s, SJob& j) {
    const uint32_t ts = std::min<uint32_t>(j.Np, kEncTileSymbols) / 8 * 8;
    const uint32_t tiles = (j.Np + ts - 1) / ts;
    // slices per encode item: at most ~wave_ms/4 of work
    const double per_slice = est_encode_item_ms(1, ts) - est_encode_item_ms(0, ts);
    uint32_t chunk = (uint32_t)std::max(1.0, floor(s->wave_ms / 4.0 / per_slice));
    chunk = std::min(chunk, j.S);
    const uint32_t chunks = (j.S + chunk - 1) / chunk;
    for (uint32_t a = 0; a < j.S; a += kScanSlices) {
        const uint32_t cnt = std::min(kScanSlices, j.S - a);
        j.todo.push_back({j.slot, kItemScan, a, cnt, 0, 0});
        j.todo_ms.push_back(est_scan_item_ms(j.slice, cnt));
        j.scan_total++;
    }
    const uint32_t cper = crc_item_slices(j.slice);
    for (uint32_t a = 0; a < j.S; a += cper) {
        const uint32_t cnt = std::min(cper, j.S - a);
        j.todo.push_back({j.slot, kItemCrc, a, cnt, 0, 0});
        j.todo_ms.push_back(est_crc_item_ms(j.slice, cnt));
        j.scan_total++;
    }
    j.todo.push_back({j.slot, kItemSetId, 0, 0, 0, 0});
    j.todo_ms.push_back(est_set_id_ms(j.n));
    if (j.R && j.mma) {
        // tensor-core items: 16-row tiles x 240 symbols, slice chunks on whole
        // 16-slice stages of the A image, again at most ~wave_ms/4 each
        const double per_stage = est_mma_item_ms(16) - est_mma_item_ms(0);
        uint32_t mchunk = (uint32_t)std::max(1.0, floor(s->wave_ms / 4.0 / per_stage)) * 16;
        if (mchunk >= j.S) mchunk = j.S;
        const uint32_t mchunks = (j.S + mchunk - 1) / mchunk;
        const uint32_t mtiles = (j.Np + kMmaTileSymbols - 1) / kMmaTileSymbols;
        const uint32_t RT = (j.R + kMmaTileRows - 1) / kMmaTileRows;
        for (uint32_t t = 0; t < mtiles; ++t) {
            const uint32_t n0 = t * kMmaTileSymbols, syms = std::min(kMmaTileSymbols, j.Np - n0);
            for (uint32_t c = 0; c < mchunks; ++c) {
                const uint32_t s0 = c * mchunk, sn = std::min(mchunk, j.S - s0);
                for (uint32_t rt = 0; rt < RT; ++rt) {
                    j.todo.push_back({j.slot, encode_mma_kind(rt, mchunks > 1), n0, syms, s0, sn});
                    j.todo_ms.push_back(est_mma_item_ms(sn));
                    j.enc_total++;
                }
            }
        }
    } else if (j.R) {
        const bool acc = chunks > 1;
        const uint32_t F = tail_fold(j.R);  // the last row group covers F tiles per item
        for (uint32_t t = 0; t < tiles; ++t) {
            const uint32_t n0 = t * ts, syms = std::min(ts, j.Np - n0);
            for (uint32_t c = 0; c < chunks; ++c) {
                const uint32_t s0 = c * chunk, sn = std::min(chunk, j.S - s0);
                for (uint32_t rg = 0; rg < j.RG; ++rg) {
                    uint32_t fold = 1, n = syms;
                    if (rg + 1 == j.RG && F > 1) {
                        if (t % F) continue;  // covered by the folded item of tile t - t % F
                        fold = F;
                        n = std::min((t + F) * ts, j.Np) - n0;
                    }
                    j.todo.push_back({j.slot, encode_kind(rg, fold, acc), n0, n, s0, sn});
                    j.todo_ms.push_back(est_encode_item_ms(sn, syms));
                    j.enc_total++;
                }
            }
        }
    }
    j.pkt_ms_per_item = est_packet_item_ms(j.slice, std::min(j.R, kScanSlices));
}

// Admit queued jobs in arrival order while budget and slots allow.
p2g_status admit(p2g_server* s) {
    while (!s->queue.empty() && !s->free_slots.empty()) {
        SJob& j = *s->queue.front();
        if (s->resident_bytes + j.footprint > s->budget) break;
        const uint64_t rec_stride = round_up(j.slice, 16);
        const uint64_t src_b = round_up((uint64_t)j.S * j.slice, 256);
        const uint64_t rec_b = round_up((uint64_t)std::max(j.R, 1u) * rec_stride, 256);
        const uint64_t chk_b = round_up(20ull * j.S, 256);
        const uint64_t small_b = round_up(16ull * j.n, 256) * 2 + 256 + round_up(16ull * std::max(j.R, 1u), 256) +
                                 round_up(32ull * j.n + 12, 256) + round_up(j.h_names.size() + 4, 256) +
                                 round_up(8ull * j.n, 256) + round_up(24ull * j.n, 256) + round_up(8ull * j.n, 256);
        const uint64_t realign_b = j.slice % 16 ? round_up((uint64_t)j.S * rec_stride, 256) : 0;
        const uint64_t aimg_b = j.mma ? round_up(j.aimg_bytes, 256) : 0;
        const uint64_t total = src_b + rec_b + chk_b + small_b + realign_b + aimg_b;
        cudaError_t e = cudaMallocAsync(&j.mem, total, s->copy);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            j.mem = nullptr;
            bool any_resident = false;
            for (auto& up : s->live) any_resident |= up->mem != nullptr;
            if (any_resident) break;  // the pool cannot place it now: retry after a release
            // nothing else holds device memory: the job can never be placed
            j.status = P2G_ERR_OOM;
            j.state = 2;
            j.t_admit = j.t_done = s->now();
            s->completed.push_back(&j);
            s->st.completed++;
            s->live.push_back(std::move(s->queue.front()));
            s->queue.pop_front();
            s->cv_done.notify_all();
            continue;
        }
        if (e != cudaSuccess) return fail_cuda(s, e, "cudaMallocAsync");
        uint8_t* m = static_cast<uint8_t*>(j.mem);
        uint64_t off = 0;
        auto take = [&](uint64_t b) {
            uint8_t* p = m + off;
            off += round_up(b, 256);
            return p;
        };
        BatchJob& d = j.desc;
        memset(&d, 0, sizeof d);
        uint8_t* src = take(src_b);
        d.src = src;
        d.rec = take(rec_b);
        d.checks = reinterpret_cast<p2g_slice_checksum*>(take(chk_b));
        d.h16k = take(16ull * j.n);
        d.pkt = take(16ull * std::max(j.R, 1u));
        d.set_id = take(16);
        d.scratch = take(32ull * j.n + 12);
        uint8_t* names = take(j.h_names.size() + 4);
        uint64_t* files = reinterpret_cast<uint64_t*>(take(16ull * j.n));
        uint32_t* noff = reinterpret_cast<uint32_t*>(take(8ull * j.n));
        uint64_t* fill = reinterpret_cast<uint64_t*>(take(24ull * j.n));
        uint64_t* seeds = reinterpret_cast<uint64_t*>(take(8ull * j.n));
        d.names = names;
        d.files = files;
        d.name_off = noff;
        d.slice = j.slice;
        d.S = j.S;
        d.R = j.R;
        d.RG = j.RG;
        d.n_files = j.n;
        d.rec_stride = rec_stride;
        d.n_bands = 0;  // packet MD5s run as their own items
        d.ts = std::min<uint32_t>(j.Np, kEncTileSymbols) / 8 * 8;
        d.first_exp = 0;
        d.vec = j.slice % 16 == 0 ? 1u : 0u;
        d.basis = nullptr;  // derived per slice: no basis memory per resident job
        if (realign_b) {
            d.esrc = take(realign_b);
            d.estride = rec_stride;
        } else {
            d.esrc = src;
            d.estride = j.slice;
        }
        if (j.mma) {
            d.mma = 1;
            d.aimg = take(aimg_b);
            d.Rpad = (j.R + kMmaTileRows - 1) / kMmaTileRows * kMmaTileRows;
            d.ksteps = mma_image_steps(j.S);
            const cudaError_t me = make_src_map(&d.src_map, d.esrc, d.estride, j.S, (uint32_t)(d.estride / 2));
            if (me != cudaSuccess) return fail_cuda(s, me, "tensor map");
        }
        const uint32_t slot = s->free_slots.back();
        s->free_slots.pop_back();
        j.slot = slot;
        cudaStream_t c = s->copy;
        SRV_CU(s, cudaMemcpyAsync(files, j.h_files.data(), 16ull * j.n, cudaMemcpyHostToDevice, c));
        SRV_CU(s, cudaMemcpyAsync(noff, j.h_noff.data(), 8ull * j.n, cudaMemcpyHostToDevice, c));
        SRV_CU(s, cudaMemcpyAsync(names, j.h_names.data(), j.h_names.size(), cudaMemcpyHostToDevice, c));
        if (j.source_kind == P2G_SOURCE_SEEDED) {
            SRV_CU(s, cudaMemcpyAsync(fill, j.h_fill.data(), 24ull * j.n, cudaMemcpyHostToDevice, c));
            SRV_CU(s, cudaMemcpyAsync(seeds, j.seeds.data(), 8ull * j.n, cudaMemcpyHostToDevice, c));
            uint64_t mx = 0;
            for (uint32_t f = 0; f < j.n; ++f) mx = std::max(mx, j.h_fill[3 * f + 2]);
            SRV_CU(s, launch_seeded_fill(src, fill, seeds, j.n, mx, c));
        } else {
            SRV_CU(s, cudaMemcpyAsync(src, j.host_src, (uint64_t)j.S * j.slice, cudaMemcpyHostToDevice, c));
        }
        if (realign_b) SRV_CU(s, launch_realign(src, j.slice, const_cast<uint8_t*>(d.esrc), rec_stride, j.S, j.slice, c));
        if (j.R) SRV_CU(s, cudaMemsetAsync(d.rec, 0, (uint64_t)j.R * rec_stride, c));
        SRV_CU(s, cudaMemcpyAsync(s->d_jobs + slot, &j.desc, sizeof(BatchJob), cudaMemcpyHostToDevice, c));
        if (j.mma) SRV_CU(s, launch_a_image_batch(s->d_jobs + slot, 1, j.aimg_bytes, c));
        SRV_CU(s, cudaEventCreateWithFlags(&j.ready, cudaEventDisableTiming));
        SRV_CU(s, cudaEventRecord(j.ready, c));
        plan_job(s, j);
        j.state = 1;
        j.t_admit = s->now();
        s->resident_bytes += j.footprint;
        j.counted = true;
        s->peak_bytes = std::max(s->peak_bytes, s->resident_bytes);
        s->st.admitted++;
        s->live.push_back(std::move(s->queue.front()));
        s->queue.pop_front();
    }
    return P2G_OK;
}

void complete_if_done(p2g_server* s, SJob& j) {
    if (j.state != 1 || j.outstanding) return;
    const bool done = j.status != P2G_OK ||
                      (j.todo.empty() && j.scan_done == j.scan_total && j.setid_done && j.enc_done == j.enc_total &&
                       j.pkt_done == j.R);
    if (!done) return;
    j.state = 2;
    j.t_done = s->now();
    s->completed.push_back(&j);
    s->st.completed++;
    s->cv_done.notify_all();
}

// Retire completed waves (in order).
p2g_status retire(p2g_server* s, bool block) {
    while (!s->inflight.empty()) {
        Wave& w = s->inflight.front();
        cudaError_t q = block ? cudaEventSynchronize(w.ev) : cudaEventQuery(w.ev);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) return fail_cuda(s, q, "wave");
        const bool err = s->h_err[w.buf] != 0;
        for (auto& [j, it] : w.items) {
            j->outstanding--;
            if (err) {
                j->status = P2G_ERR_TIMEOUT;
                continue;
            }
            switch (it.kind_rg & kItemKindMask) {
            case kItemScan:
            case kItemCrc: j->scan_done++; break;
            case kItemSetId: j->setid_done = true; break;
            case kItemEncode:
            case kItemEncodeMma: j->enc_done++; break;
            case kItemPacket: j->pkt_done += it.b; break;
            }
        }
        for (auto& [j, it] : w.items) complete_if_done(s, *j);
        cudaEventDestroy(w.ev);
        s->buf_busy[w.buf] = false;
        s->inflight.pop_front();
    }
    return P2G_OK;
}

// Build and launch one wave if there is work; returns true if launched.
p2g_status launch_wave(p2g_server* s, bool* launched) {
    *launched = false;
    int buf = -1;
    for (int b = 0; b < kWaveBufs; ++b)
        if (!s->buf_busy[b]) {
            buf = b;
            break;
        }
    if (buf < 0) return P2G_OK;
    // eligible jobs, in admission order starting at the round-robin cursor
    std::vector<SJob*> el;
    for (auto& up : s->live) {
        SJob& j = *up;
        if (j.state != 1 || j.status != P2G_OK) continue;
        if (!j.is_ready) {
            const cudaError_t q = cudaEventQuery(j.ready);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) return fail_cuda(s, q, "source ready");
            j.is_ready = true;
        }
        const bool pkt_ok = j.setid_done && j.enc_done == j.enc_total && j.pkt_issued < j.R;
        if (!j.todo.empty() || pkt_ok) el.push_back(&j);
    }
    if (el.empty()) return P2G_OK;
    const double budget = s->wave_ms * s->ctas;
    const double share = budget / el.size();
    Wave w;
    w.buf = buf;
    double used = 0;
    // A launch runs one kind of encode item: the first encode item taken
    // sets it, and a job whose next item is of the other kind waits for a
    // later wave (its scan, set-id and packet items run in either kind).
    int wave_mma = -1;
    auto take_from = [&](SJob& j, double quota) {
        double got = 0;
        while (got < quota && w.items.size() < kWaveItems) {
            if (!j.todo.empty()) {
                const BatchItem it = j.todo.front();
                const uint32_t kd = it.kind_rg & kItemKindMask;
                if (kd == kItemEncode || kd == kItemEncodeMma) {
                    const int km = kd == kItemEncodeMma ? 1 : 0;
                    if (wave_mma < 0) wave_mma = km;
                    if (wave_mma != km) break;
                }
                const double ms = j.todo_ms.front();
                j.todo.pop_front();
                j.todo_ms.pop_front();
                w.items.push_back({&j, it});
                j.outstanding++;
                got += ms;
            } else if (j.setid_done && j.enc_done == j.enc_total && j.pkt_issued < j.R) {
                const uint32_t rows = std::min(kScanSlices, j.R - j.pkt_issued);
                w.items.push_back({&j, {j.slot, kItemPacket, j.pkt_issued, rows, 0, 0}});
                j.pkt_issued += rows;
                j.outstanding++;
                got += j.pkt_ms_per_item;
            } else {
                break;
            }
        }
        return got;
    };
    const size_t n_el = el.size();
    for (size_t k = 0; k < n_el; ++k) used += take_from(*el[(s->rr + k) % n_el], share);
    for (size_t k = 0; k < n_el && used < budget; ++k) used += take_from(*el[k], budget - used);  // oldest first
    s->rr++;
    if (w.items.empty()) return P2G_OK;
    // longest items first inside the wave
    std::vector<std::pair<double, BatchItem>> order;
    order.reserve(w.items.size());
    for (auto& [j, it] : w.items) {
        const uint32_t k = it.kind_rg & kItemKindMask;
        const double ms = k == kItemEncode      ? est_encode_item_ms(it.sn, std::min(it.b & 0xFFFFu, j->desc.ts))
                          : k == kItemEncodeMma ? est_mma_item_ms(it.sn)
                          : k == kItemScan ? est_scan_item_ms(j->slice, it.b)
                          : k == kItemCrc ? est_crc_item_ms(j->slice, it.b)
                          : k == kItemSetId ? est_set_id_ms(j->n)
                                            : est_packet_item_ms(j->slice, it.b);
        order.push_back({ms, it});
    }
    std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    for (size_t i = 0; i < order.size(); ++i) s->h_items[buf][i] = order[i].second;
    const uint32_t n = (uint32_t)order.size();
    cudaStream_t e = s->exec;
    SRV_CU(s, cudaMemcpyAsync(s->d_items[buf], s->h_items[buf], sizeof(BatchItem) * n, cudaMemcpyHostToDevice, e));
    SRV_CU(s, cudaMemsetAsync(s->d_ctl[buf], 0, sizeof(uint32_t) * (1 + s->max_jobs), e));
    SRV_CU(s, launch_batch(s->d_jobs, s->d_items[buf], n, s->d_ctl[buf], s->d_err, s->ctas, e, wave_mma == 1));
    SRV_CU(s, cudaMemcpyAsync(s->h_err + buf, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, e));
    SRV_CU(s, cudaEventCreateWithFlags(&w.ev, cudaEventDisableTiming));
    SRV_CU(s, cudaEventRecord(w.ev, e));
    s->buf_busy[buf] = true;
    s->st.waves++;
    s->st.items += n;
    s->inflight.push_back(std::move(w));
    *launched = true;
    return P2G_OK;
}

void scheduler(p2g_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        p2g_status r = retire(s, false);
        if (r == P2G_OK) r = admit(s);
        bool launched = false;
        if (r == P2G_OK && s->inflight.size() < 2) r = launch_wave(s, &launched);
        if (r != P2G_OK) {  // device error: fail every job, stop scheduling
            for (auto& up : s->live)
                if (up->state == 1) {
                    up->status = s->fatal;
                    up->outstanding = 0;
                    complete_if_done(s, *up);
                }
            s->cv_done.notify_all();
            s->cv_work.wait(lk, [s] { return s->stop; });
            break;
        }
        if (launched) continue;
        // nothing to launch: poll the waves in flight every 100 us, or sleep
        // until a submit or a release
        s->cv_work.wait_for(lk, std::chrono::microseconds(s->inflight.empty() ? 2000 : 100));
    }
}

void free_job_memory(p2g_server* s, SJob& j) {
    if (j.mem) cudaFreeAsync(j.mem, s->copy);
    j.mem = nullptr;
    if (j.ready) cudaEventDestroy(j.ready);
    j.ready = nullptr;
    if (j.slot != ~0u) s->free_slots.push_back(j.slot);
    j.slot = ~0u;
    if (j.counted) s->resident_bytes -= j.footprint;
    j.counted = false;
}

}  // namespace
}  // namespace p2g

using namespace p2g;

extern "C" p2g_status p2g_server_create(const p2g_server_options* opts, p2g_server** out) {
    clear_error();
    if (!out) return set_error(P2G_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    P2G_TRY(ensure_device_ready());
    std::unique_ptr<p2g_server> s(new p2g_server());
    cudaGetDevice(&s->device);
    s->budget = opts && opts->hbm_budget ? opts->hbm_budget : 120000000000ull;
    s->wave_ms = opts && opts->wave_ms > 0 ? opts->wave_ms : 20.0;
    s->max_jobs = opts && opts->max_jobs ? opts->max_jobs : 1024;
    s->ctas = (uint32_t)device_sm_count();
    s->t0 = std::chrono::steady_clock::now();
    int lo = 0, hi = 0;
    P2G_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    P2G_CU(cudaStreamCreateWithPriority(&s->exec, cudaStreamNonBlocking, lo));
    P2G_CU(cudaStreamCreateWithPriority(&s->copy, cudaStreamNonBlocking, hi));  // admissions ahead of waves
    cudaMemPool_t pool;
    P2G_CU(cudaDeviceGetDefaultMemPool(&pool, s->device));
    uint64_t keep = ~0ull;  // keep freed job memory in the pool
    P2G_CU(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    P2G_CU(cudaMalloc(&s->d_jobs, sizeof(BatchJob) * s->max_jobs));
    P2G_CU(cudaMalloc(&s->d_err, sizeof(int)));
    P2G_CU(cudaMemset(s->d_err, 0, sizeof(int)));
    P2G_CU(cudaHostAlloc(&s->h_err, sizeof(int) * kWaveBufs, cudaHostAllocDefault));
    for (int b = 0; b < kWaveBufs; ++b) {
        P2G_CU(cudaMalloc(&s->d_items[b], sizeof(BatchItem) * kWaveItems));
        P2G_CU(cudaHostAlloc(&s->h_items[b], sizeof(BatchItem) * kWaveItems, cudaHostAllocDefault));
        P2G_CU(cudaMalloc(&s->d_ctl[b], sizeof(uint32_t) * (1 + s->max_jobs)));
        s->h_err[b] = 0;
    }
    P2G_CU(prepare_batch_kernel());
    for (uint32_t i = s->max_jobs; i-- > 0;) s->free_slots.push_back(i);
    p2g_server* raw = s.release();
    try {
        raw->th = std::thread(scheduler, raw);
    } catch (const std::exception& e) {  // no thread for the scheduler: nothing was started
        p2g_server_destroy(raw);
        return set_error(P2G_ERR_INVALID_ARGUMENT, "cannot start the server's scheduler thread: %s", e.what());
    }
    *out = raw;
    return P2G_OK;
}

extern "C" p2g_status p2g_server_submit(p2g_server* s, const p2g_server_job* rq, uint64_t* ticket) {
    clear_error();
    if (!s || !rq) return set_error(P2G_ERR_INVALID_ARGUMENT, "server or job is NULL");
    P2G_TRY(check_common(rq->file_count, rq->recovery_count, rq->slice_size));
    if (!rq->file_lengths || !rq->names || !rq->name_lens)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "file lengths and names are required");
    if (rq->source_kind == P2G_SOURCE_HOST ? !rq->host_src : rq->source_kind != P2G_SOURCE_SEEDED || !rq->file_seeds)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "a host source or per-file seeds are required");
    std::unique_ptr<SJob> j(new SJob());
    j->slice = rq->slice_size;
    j->R = rq->recovery_count;
    j->n = rq->file_count;
    j->tag = rq->tag;
    j->source_kind = rq->source_kind;
    j->host_src = rq->host_src;
    uint64_t S = 0;
    for (uint32_t f = 0; f < j->n; ++f) {
        P2G_TRY(check_name(rq->names[f], rq->name_lens[f], ""));
        const uint64_t len = rq->file_lengths[f];
        if (!len) return set_error(P2G_ERR_EMPTY_FILE, "input file %u is empty", f);
        const uint64_t sl = (len + j->slice - 1) / j->slice;
        j->lens.push_back(len);
        j->h_files.push_back(S * j->slice);
        j->h_files.push_back(len);
        j->h_fill.push_back(S * j->slice);
        j->h_fill.push_back(len);
        j->h_fill.push_back(sl * j->slice);
        j->h_noff.push_back((uint32_t)j->h_names.size());
        j->h_noff.push_back((uint32_t)rq->name_lens[f]);
        j->h_names.insert(j->h_names.end(), rq->names[f], rq->names[f] + rq->name_lens[f]);
        j->h_names.resize(round_up(j->h_names.size(), 4), 0);
        if (rq->source_kind == P2G_SOURCE_SEEDED) j->seeds.push_back(rq->file_seeds[f]);
        S += sl;
        j->source_bytes += len;
    }
    P2G_TRY(check_total_blocks(S, j->source_bytes, j->slice));
    j->S = (uint32_t)S;
    j->RG = (j->R + kRowsPerGroup - 1) / kRowsPerGroup;
    j->Np = (uint32_t)(round_up(j->slice, 16) / 2);
    j->footprint = S * j->slice + (uint64_t)j->R * round_up(j->slice, 16);
    // tensor-core encode when the cost model prefers it and the A image
    // (R x S x 128 B) stays within a quarter of the source bytes
    const char* ev = getenv("P2G_ENCODE_VARIANT");  // "lut" / "tensor" force a kind (tensor: if the image fits)
    const bool want_mma = ev && !strcmp(ev, "lut") ? false
                          : ev && !strcmp(ev, "tensor") ? true
                                                        : prefer_mma(j->slice, j->S, j->R);
    if (j->R && want_mma && 4 * mma_aimg_bytes(j->S, j->R) <= S * j->slice) {
        j->mma = true;
        j->aimg_bytes = mma_aimg_bytes(j->S, j->R);
        j->footprint += j->aimg_bytes;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal != P2G_OK) return set_error(s->fatal, "server stopped: %s", s->fatal_msg.c_str());
    if (j->footprint > s->budget)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "job footprint %llu bytes exceeds the server's HBM budget %llu",
                         (unsigned long long)j->footprint, (unsigned long long)s->budget);
    j->ticket = s->next_ticket++;
    j->t_submit = s->now();
    if (ticket) *ticket = j->ticket;
    s->queue.push_back(std::move(j));
    s->st.submitted++;
    s->cv_work.notify_all();
    return P2G_OK;
}

extern "C" p2g_status p2g_server_poll(p2g_server* s, p2g_server_result* out, uint32_t cap, uint32_t* n_out,
                                      uint32_t wait_ms) {
    clear_error();
    if (!s || (!out && cap) || !n_out) return set_error(P2G_ERR_INVALID_ARGUMENT, "server, out or n_out is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->completed.empty() && wait_ms)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] { return !s->completed.empty(); });
    uint32_t n = 0;
    while (n < cap && !s->completed.empty()) {
        SJob& j = *s->completed.front();
        s->completed.pop_front();
        p2g_server_result& r = out[n++];
        memset(&r, 0, sizeof r);
        r.ticket = j.ticket;
        r.tag = j.tag;
        r.status = j.status;
        r.submit_s = j.t_submit;
        r.admit_s = j.t_admit;
        r.done_s = j.t_done;
        r.source_bytes = j.source_bytes;
        r.input_slices = j.S;
        r.recovery_count = j.R;
        r.file_count = j.n;
        r.src = j.desc.src;
        r.recovery = j.desc.rec;
        r.recovery_stride = j.desc.rec_stride;
        r.checksums = j.desc.checks;
        r.hash16k = j.desc.h16k;
        r.packet_md5 = j.desc.pkt;
        r.set_id = j.desc.set_id;
    }
    *n_out = n;
    return P2G_OK;
}

extern "C" p2g_status p2g_server_release(p2g_server* s, uint64_t ticket) {
    clear_error();
    if (!s) return set_error(P2G_ERR_INVALID_ARGUMENT, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t i = 0; i < s->live.size(); ++i) {
        SJob& j = *s->live[i];
        if (j.ticket != ticket) continue;
        if (j.state != 2) return set_error(P2G_ERR_INVALID_ARGUMENT, "job %llu is not complete", (unsigned long long)ticket);
        cudaSetDevice(s->device);
        free_job_memory(s, j);
        j.state = 3;
        s->st.released++;
        s->live.erase(s->live.begin() + i);
        s->cv_work.notify_all();
        return P2G_OK;
    }
    return set_error(P2G_ERR_INVALID_ARGUMENT, "unknown ticket %llu", (unsigned long long)ticket);
}

extern "C" p2g_status p2g_server_get_stats(p2g_server* s, p2g_server_stats* out) {
    clear_error();
    if (!s || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "server or out is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->queued = (uint32_t)s->queue.size();
    uint32_t res = 0;
    for (auto& up : s->live) res += up->state == 1;
    out->resident = res;
    out->resident_bytes = s->resident_bytes;
    out->peak_resident_bytes = s->peak_bytes;
    out->budget_bytes = s->budget;
    return s->fatal != P2G_OK ? set_error(s->fatal, "server stopped: %s", s->fatal_msg.c_str()) : P2G_OK;
}

extern "C" double p2g_server_now(p2g_server* s) { return s ? s->now() : 0.0; }

extern "C" p2g_status p2g_copy_to_host(void* dst, const void* device_src, uint64_t bytes) {
    clear_error();
    if (!bytes) return P2G_OK;
    if (!dst || !device_src) return set_error(P2G_ERR_INVALID_ARGUMENT, "dst or device_src is NULL");
    P2G_TRY(ensure_device_ready());
    P2G_CU(cudaMemcpy(dst, device_src, bytes, cudaMemcpyDeviceToHost));
    return P2G_OK;
}

extern "C" void p2g_server_destroy(p2g_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->exec);
    cudaStreamSynchronize(s->copy);
    for (auto& w : s->inflight) cudaEventDestroy(w.ev);
    for (auto& up : s->live) free_job_memory(s, *up);
    cudaStreamSynchronize(s->copy);
    for (int b = 0; b < kWaveBufs; ++b) {
        cudaFree(s->d_items[b]);
        cudaFreeHost(s->h_items[b]);
        cudaFree(s->d_ctl[b]);
    }
    cudaFree(s->d_jobs);
    cudaFree(s->d_err);
    cudaFreeHost(s->h_err);
    cudaStreamDestroy(s->exec);
    cudaStreamDestroy(s->copy);
    delete s;
}
