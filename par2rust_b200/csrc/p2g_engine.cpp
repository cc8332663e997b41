// p2g_engine.cpp -- device context, hot-path seams and the create pipeline
// of libpar2gpu.so (the C ABI declared in include/par2gpu.h).
//
// Device data layout for one create job:
//   src      the input files back to back in caller order, each starting on a
//            slice boundary and zero-padded to whole slices: input slice s is
//            src + s*slice_size (the global input index of
//            src/creator.rs:895-900 / :757-775).
//   rec      recovery row r (exponent first_exp + r) at rec + r*rec_stride,
//            rec_stride = slice_size rounded up to 16 bytes.
//   basis    [s][row group][16][32] u16 coefficient-basis scratch.
//   checks   one 20-byte IFSC record (md5 ‖ crc32) per input slice.
#include <cuda_runtime.h>
#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "p2g_host_util.h"
#include "p2g_internal.h"

namespace p2g {

p2g_status cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();  // clear a sticky-free error so later calls can proceed
    if (e == cudaErrorMemoryAllocation)
        return set_error(P2G_ERR_OOM, "device allocation failed: %s (%s)", cudaGetErrorString(e), what);
    return set_error(P2G_ERR_CUDA, "CUDA error: %s (%s)", cudaGetErrorString(e), what);
}

static inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }
// One-launch upload of page-locked inputs: from this many files on, in
// segments of at most 4 MiB (a segment's zero pad, the tail of a file's last
// slice, is encoded in 24 bits; larger tails are memset apart).
constexpr uint32_t kGatherMinFiles = 8;
constexpr uint64_t kGatherSegBytes = 4ull << 20;

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(round_up(n, 1 << 20), 1 << 20);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};
// Grow-only pinned host buffer.
struct PinBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(round_up(n, 1 << 16), 1 << 16);
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// One per process.  Calls are serialised on `mu`; the device is the one
// current on the first calling thread (or P2G_DEVICE).
struct Context {
    std::recursive_mutex mu;
    int device = -1;
    bool ready = false;
    static constexpr int kStreams = 7;  // encode, files, slice md5, crc, hash_full, encode (odd bands), packet md5
    static constexpr int kBandEvents = 64;
    cudaStream_t st[kStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_h16k = nullptr, ev_join[kStreams] = {}, ev_band[kBandEvents] = {};
    // device-pointer encodes on the caller's stream share the scratch below:
    // each waits for the previous one's use of it
    cudaEvent_t ev_scratch = nullptr;
    bool scratch_pending = false;
    DevBuf src, src_al, rec, basis, checks, h16k, hfull, pkt, spans, err, tmp_in, tmp_out, md5_state;
    DevBuf aimg;       // A operand image of the tensor-core encode
    DevBuf gseg;       // segment table of the one-launch upload of page-locked inputs
    DevBuf persist;    // single-job persistent run: descriptor, items, chain state, tables
    PinBuf h_spans, h_h16k, h_err, h_stage, h_persist, h_gseg;
    PinBuf h_rec;   // host copy of the recovery rows (create calls)
    PinBuf h_prog;  // encode progress: the device queue head, read while a job runs
};
static Context& ctx() {
    static Context* c = new Context();  // never destroyed: the CUDA runtime may be gone at exit
    return *c;
}

static p2g_status ensure_ready(Context& c) {
    if (!c.ready) {
        int dev = 0;
        if (const char* e = getenv("P2G_DEVICE")) dev = atoi(e);
        else if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0)
            return set_error(P2G_ERR_CUDA, "no CUDA device available (%s)",
                             e != cudaSuccess ? cudaGetErrorString(e) : "device count 0");
        if (dev >= n) dev = 0;
        P2G_CU(cudaSetDevice(dev));
        cudaDeviceProp prop;
        P2G_CU(cudaGetDeviceProperties(&prop, dev));
        if (prop.major < 10)
            return set_error(P2G_ERR_CUDA, "device %d (%s, sm_%d%d) is not sm_100: this build targets B200 only", dev,
                             prop.name, prop.major, prop.minor);
        // st[0] carries the encode; the MD5/CRC streams get the higher
        // priority so their small, long-running blocks are dispatched ahead of
        // encode CTAs and share the SMs with them.
        int lo_pri = 0, hi_pri = 0;
        P2G_CU(cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
        for (int i = 0; i < Context::kStreams; ++i)
            P2G_CU(cudaStreamCreateWithPriority(&c.st[i], cudaStreamNonBlocking, (i == 0 || i == 5) ? lo_pri : hi_pri));
        P2G_CU(cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming));
        P2G_CU(cudaEventCreateWithFlags(&c.ev_scratch, cudaEventDisableTiming));
        P2G_CU(cudaEventCreateWithFlags(&c.ev_h16k, cudaEventDisableTiming));
        for (auto& ev : c.ev_join) P2G_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        for (auto& ev : c.ev_band) P2G_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        P2G_CU(upload_tables());
        P2G_CU(c.err.ensure(64));
        P2G_CU(c.h_err.ensure(64));
        c.device = dev;
        c.ready = true;
    }
    P2G_CU(cudaSetDevice(c.device));
    return P2G_OK;
}

// Optional stage timeline (P2G_TRACE=1): timing events recorded after each
// stage on its stream, printed to stderr relative to the job start when the
// job is joined.  Off by default; costs nothing when off.
p2g_status ensure_device_ready() {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    return ensure_ready(c);
}

struct Tracer {
    bool on = false;
    cudaEvent_t t0 = nullptr;
    std::vector<std::pair<std::string, cudaEvent_t>> marks;
    void start(cudaStream_t s) {
        on = getenv("P2G_TRACE") != nullptr;
        if (!on) return;
        cudaEventCreate(&t0);
        cudaEventRecord(t0, s);
    }
    void mark(const char* what, cudaStream_t s) {
        if (!on) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        marks.push_back({what, e});
    }
    void finish() {
        if (!on) return;
        for (auto& m : marks) {
            cudaEventSynchronize(m.second);
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, m.second);
            fprintf(stderr, "[p2g trace] %8.3f ms  %s\n", ms, m.first.c_str());
            cudaEventDestroy(m.second);
        }
        cudaEventDestroy(t0);
        marks.clear();
    }
};

// Fork the side streams off `caller`, join them back.
static p2g_status fork_from(Context& c, cudaStream_t caller) {
    P2G_CU(cudaEventRecord(c.ev_fork, caller));
    for (auto& s : c.st) P2G_CU(cudaStreamWaitEvent(s, c.ev_fork, 0));
    return P2G_OK;
}
static p2g_status join_into(Context& c, cudaStream_t caller) {
    for (int i = 0; i < Context::kStreams; ++i) {
        P2G_CU(cudaEventRecord(c.ev_join[i], c.st[i]));
        P2G_CU(cudaStreamWaitEvent(caller, c.ev_join[i], 0));
    }
    return P2G_OK;
}

// ---------------------------------------------------------------------------
// Whole-file MD5 placement.  A file hash is one serial MD5 chain: on the
// device each chain runs on one thread; on the host on one core.  AUTO picks
// the side with the smaller estimated finish time from measured chain rates
// (overridable with P2G_FILE_HASH=device|host).
// ---------------------------------------------------------------------------
// Coefficient basis of the encode: precomputed by its own kernel into a
// scratch buffer (S x row groups x 1 KiB) and loaded by TMA, unless
// P2G_ENCODE_BASIS=derive has the encode kernel derive it (no scratch, ~6%
// more encode time on B200: 512 extra lookups per slice in a loop that is
// close to its issue limit).
// Which encode kernel runs a job: the shared-memory lookup kernel or the
// tensor-core bit-sliced one.  P2G_ENCODE_LUT / P2G_ENCODE_TENSOR (or
// P2G_ENCODE_VARIANT=lut|tensor) force one; otherwise the planner's cost
// model picks by shape (prefer_mma).
static bool use_tensor_encode(uint32_t flags, uint32_t S, uint32_t R, uint64_t slice_size) {
    if (flags & P2G_ENCODE_TENSOR) return true;
    if (flags & P2G_ENCODE_LUT) return false;
    if (const char* e = getenv("P2G_ENCODE_VARIANT")) {
        if (!strcmp(e, "tensor")) return true;
        if (!strcmp(e, "lut")) return false;
    }
    return prefer_mma(slice_size, S, R);
}

static bool generate_basis() {
    const char* e = getenv("P2G_ENCODE_BASIS");
    return e && !strcmp(e, "derive");
}

enum class FileHashMode { Device, Host };
static double env_double(const char* name, double dflt) {
    const char* e = getenv(name);
    return e ? atof(e) : dflt;
}
static FileHashMode choose_file_hash_mode(const std::vector<uint64_t>& lens) {
    if (const char* e = getenv("P2G_FILE_HASH")) {
        if (!strcmp(e, "device")) return FileHashMode::Device;
        if (!strcmp(e, "host")) return FileHashMode::Host;
    }
    // chain rates in bytes/s: one device thread, one host core
    const double dev_rate = env_double("P2G_DEVICE_MD5_RATE", 1.2e8);
    const double host_rate = env_double("P2G_HOST_MD5_RATE", 8.0e8);
    uint64_t mx = 0, total = 0;
    for (uint64_t l : lens) {
        mx = std::max(mx, l);
        total += l;
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const double t_dev = (double)mx / dev_rate;
    const double t_host = std::max((double)mx / host_rate, (double)total / (host_rate * hw));
    return t_host < t_dev ? FileHashMode::Host : FileHashMode::Device;
}

// Runs fn() on up to n threads including the caller's; threads that cannot
// be started are simply not used (fn must share its work through a counter).
template <class F>
static void run_on_threads(unsigned n, F&& fn) {
    std::vector<std::thread> th;
    for (unsigned t = 1; t < n; ++t) {
        try {
            th.emplace_back(fn);
        } catch (const std::exception&) {
            break;
        }
    }
    fn();
    for (auto& t : th) t.join();
}

// Host-side whole-file MD5 of several buffers on a small thread pool.  The
// caller's own thread takes whatever is left when it joins, so every buffer
// is hashed even when no thread could be started.
struct HostHasher {
    std::vector<std::thread> th;
    const std::vector<const uint8_t*>* data = nullptr;
    const std::vector<uint64_t>* lens = nullptr;
    std::vector<Md5>* out = nullptr;
    std::shared_ptr<std::atomic<size_t>> next;
    void work() {
        for (size_t i = (*next)++; i < data->size(); i = (*next)++) (*out)[i] = md5_of((*data)[i], (*lens)[i]);
    }
    void start(const std::vector<const uint8_t*>& d, const std::vector<uint64_t>& l, std::vector<Md5>& o) {
        o.resize(d.size());
        data = &d;
        lens = &l;
        out = &o;
        next = std::make_shared<std::atomic<size_t>>(0);
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned nt = (unsigned)std::min<size_t>(hw, d.size());
        for (unsigned t = 0; t < nt; ++t) {
            try {
                th.emplace_back([this]() { work(); });
            } catch (const std::exception&) {
                break;
            }
        }
    }
    void join() {
        if (next) work();
        for (auto& t : th) t.join();
        th.clear();
        next.reset();
    }
    ~HostHasher() { join(); }
};

// ---------------------------------------------------------------------------
// Device job: everything between "source resident in HBM" and "recovery rows,
// checksums, file hashes and packet MD5s in HBM".
// ---------------------------------------------------------------------------
struct JobFile {
    uint64_t length;
    uint64_t first_slice;
    uint64_t slices;
    const uint8_t* name;
    size_t name_len;
};
struct DeviceJob {
    const uint8_t* d_src = nullptr;
    uint32_t S = 0;
    uint64_t slice = 0;
    uint32_t R = 0;
    uint32_t first_exp = 0;
    std::vector<JobFile> files;
    uint8_t* d_rec = nullptr;
    uint64_t rec_stride = 0;
    p2g_slice_checksum* d_checks = nullptr;  // null: skip slice checksums
    uint8_t* d_h16k = nullptr;
    uint8_t* d_hfull = nullptr;  // null: hash_full not on the device
    uint8_t* d_pkt = nullptr;    // null: skip packet MD5
    uint32_t variant = 0;        // P2G_ENCODE_LUT / P2G_ENCODE_TENSOR, or 0: by shape
    // filled
    std::vector<Md5> h16k, file_ids;
    Md5 set_id{};
    // set instead of computing from hash16k (run_create with scanned sources)
    bool have_set_id = false;
    // optional: called from the calling thread while the encode runs, with
    // input slices done (an estimate from the items the device has taken)
    std::function<void(uint64_t done, uint64_t total)> progress;
};

static p2g_status check_device_error(Context& c);

// Encode progress from the device's own counter: while the persistent launch
// runs, the queue head (items taken so far) is read back on a side stream
// every ~0.5 ms.  Items are queued set-id / file hashes / scans, then encode
// items, then CRC32, so the encode items taken give the fraction done.
// Reported as input slices, monotonic, below S until the launch ends (the
// caller reports S itself).
static p2g_status poll_progress(Context& c, DeviceJob& j, const SingleJobPlan& pl, const uint32_t* d_head,
                                cudaStream_t st) {
    uint64_t first_enc = 0, n_enc = 0;
    for (size_t i = 0; i < pl.items.size(); ++i)
        if ((pl.items[i].kind_rg & kItemKindMask) == kItemEncode ||
            (pl.items[i].kind_rg & kItemKindMask) == kItemEncodeMma) {
            if (!n_enc) first_enc = i;
            ++n_enc;
        }
    if (!n_enc) return P2G_OK;
    P2G_CU(c.h_prog.ensure(64));
    volatile uint32_t* head = c.h_prog.as<uint32_t>();
    cudaStream_t side = c.st[1];
    uint64_t last = 0;
    for (;;) {
        const cudaError_t q = cudaStreamQuery(st);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) P2G_CU(q);
        P2G_CU(cudaMemcpyAsync(c.h_prog.p, d_head, sizeof(uint32_t), cudaMemcpyDeviceToHost, side));
        P2G_CU(cudaStreamSynchronize(side));
        const uint64_t taken = *head;
        const uint64_t enc = taken > first_enc ? std::min<uint64_t>(taken - first_enc, n_enc) : 0;
        const uint64_t done = std::min<uint64_t>((uint64_t)j.S * enc / n_enc, j.S ? j.S - 1 : 0);
        if (done > last) {
            last = done;
            j.progress(done, j.S);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(500));
    }
    // "not ready" answers are status, not errors: keep them out of the
    // error state the launch wrappers read next
    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
    return P2G_OK;
}

// The device job through the persistent kernel (p2g_kernels.cu, batch_kernel)
// with this one job: slice MD5/CRC32 scan items and the set-id item first,
// then encode items band by band (folded tail, tiles sized to whole rounds of
// the SMs); each band's completion advances the recovery-packet MD5 chains.
// Items are dynamic and SM-exclusive, so the banded path's one-wave bands
// and its hash kernels sharing SMs with encode CTAs do not arise.
static p2g_status run_device_job_persistent(Context& c, DeviceJob& j, cudaStream_t st) {
    const uint32_t n = (uint32_t)j.files.size();
    const uint32_t RG = (j.R + kRowsPerGroup - 1) / kRowsPerGroup;
    const bool chains = j.R && j.S && j.d_pkt;
    const bool sid_item = !j.have_set_id;
    uint64_t max_len = 0;
    for (const auto& f : j.files) max_len = std::max(max_len, f.length);
    // the last bands' items may be cut into accumulating slice ranges (the
    // columns they write are zeroed below); P2G_TAIL_SPLIT=0 turns that off
    static const bool split_tail = [] {
        const char* e = getenv("P2G_TAIL_SPLIT");
        return !(e && !strcmp(e, "0"));
    }();
    const bool mma = j.R && j.S && use_tensor_encode(j.variant, j.S, j.R, j.slice);
    const SingleJobPlan pl = plan_single_job(j.slice, j.S, j.R && j.S ? j.R : 0, n, j.d_checks != nullptr, sid_item,
                                             chains, (uint32_t)device_sm_count(), j.d_hfull ? max_len : 0,
                                             split_tail, mma);
    const uint32_t nb = (uint32_t)pl.band_items.size();
    const uint32_t Q = (j.R + kChainRows - 1) / kChainRows;
    const uint64_t ctl_words = 1 + (chains ? nb + 2 * Q + 1 : 0) + 1;  // head, chain state, error word
    uint64_t names_bytes = 0;
    for (const auto& f : j.files) names_bytes += round_up(f.name_len, 4);
    size_t off = 0;
    auto take = [&](size_t b) {
        const size_t o = off;
        off = round_up(off + std::max<size_t>(b, 1), 256);
        return o;
    };
    const size_t o_desc = take(sizeof(BatchJob)), o_items = take(sizeof(BatchItem) * pl.items.size());
    const size_t o_ctl = take(4 * ctl_words), o_bands = take(4 * nb), o_chain = take(16ull * j.R);
    const size_t o_files = take(16ull * n), o_noff = take(8ull * n), o_names = take(names_bytes);
    const size_t o_scratch = take(32ull * n + 12), o_sid = take(16);
    const size_t host_bytes = o_ctl;  // descriptor and items staged together
    // the staging buffer may still feed the previous call's copies, and the
    // device scratch (descriptor, A image, bases) its kernels, on any stream
    if (c.scratch_pending) P2G_CU(cudaEventSynchronize(c.ev_scratch));
    P2G_CU(cudaStreamSynchronize(st));
    P2G_CU(c.persist.ensure(off));
    P2G_CU(c.h_persist.ensure(off));
    uint8_t* D = c.persist.as<uint8_t>();
    uint8_t* H = c.h_persist.as<uint8_t>();
    // basis (precomputed unless P2G_ENCODE_BASIS=derive) and 16-byte aligned slices
    const bool gen = generate_basis() || mma;  // the tensor-core items read their A image instead
    if (j.R && j.S && !gen) P2G_CU(c.basis.ensure(basis_bytes(j.S, RG)));
    if (mma) P2G_CU(c.aimg.ensure(mma_aimg_bytes(j.S, j.R)));
    const uint8_t* esrc = j.d_src;
    uint64_t estride = j.slice;
    if (j.R && j.S && j.slice % 16) {
        estride = round_up(j.slice, 16);
        P2G_CU(c.src_al.ensure((size_t)estride * j.S));
        esrc = c.src_al.as<uint8_t>();
    }
    BatchJob& d = *reinterpret_cast<BatchJob*>(H + o_desc);
    memset(&d, 0, sizeof d);
    d.src = j.d_src;
    d.esrc = esrc;
    d.basis = j.R && j.S && !gen ? c.basis.as<uint16_t>() : nullptr;
    d.rec = j.d_rec;
    d.checks = j.d_checks;
    d.h16k = j.d_h16k;
    d.pkt = j.d_pkt;
    d.set_id = D + o_sid;
    d.hfull = j.d_hfull;
    d.files = reinterpret_cast<const uint64_t*>(D + o_files);
    d.names = D + o_names;
    d.name_off = reinterpret_cast<const uint32_t*>(D + o_noff);
    d.scratch = D + o_scratch;
    d.bstate = chains ? reinterpret_cast<uint32_t*>(D + o_ctl) + 1 : nullptr;
    d.band_items = reinterpret_cast<const uint32_t*>(D + o_bands);
    d.chain = reinterpret_cast<uint32_t*>(D + o_chain);
    d.slice = j.slice;
    d.estride = estride;
    d.rec_stride = j.rec_stride;
    d.S = j.S;
    d.R = j.S ? j.R : 0;
    d.RG = RG;
    d.n_files = n;
    d.n_bands = chains ? nb : 0;
    d.band_syms = pl.band_syms;
    d.ts = pl.ts;
    d.first_exp = j.first_exp;
    d.vec = j.slice % 16 == 0 ? 1u : 0u;
    if (mma) {
        d.mma = 1;
        d.aimg = c.aimg.as<uint8_t>();
        d.Rpad = (j.R + kMmaTileRows - 1) / kMmaTileRows * kMmaTileRows;
        d.ksteps = mma_image_steps(j.S);
        P2G_CU(make_src_map(&d.src_map, esrc, estride, j.S, (uint32_t)(estride / 2)));
    }
    memcpy(H + o_items, pl.items.data(), sizeof(BatchItem) * pl.items.size());
    uint8_t* hb = H + o_ctl;  // band counts, file tables and names after the descriptor and items
    memcpy(hb + (o_bands - o_ctl), pl.band_items.data(), 4 * nb);
    uint64_t* hf = reinterpret_cast<uint64_t*>(hb + (o_files - o_ctl));
    uint32_t* hn = reinterpret_cast<uint32_t*>(hb + (o_noff - o_ctl));
    uint8_t* hs = hb + (o_names - o_ctl);
    uint64_t noff = 0;
    for (uint32_t f = 0; f < n; ++f) {
        hf[2 * f] = j.files[f].first_slice * j.slice;
        hf[2 * f + 1] = j.files[f].length;
        hn[2 * f] = (uint32_t)noff;
        hn[2 * f + 1] = (uint32_t)j.files[f].name_len;
        memcpy(hs + noff, j.files[f].name, j.files[f].name_len);
        noff += round_up(j.files[f].name_len, 4);
    }
    if (j.have_set_id) memcpy(H + o_sid, j.set_id.data(), 16);
    int* err = reinterpret_cast<int*>(D + o_ctl) + (ctl_words - 1);
    P2G_CU(cudaMemcpyAsync(D, H, host_bytes, cudaMemcpyHostToDevice, st));  // descriptor + items
    P2G_CU(cudaMemsetAsync(D + o_ctl, 0, 4 * ctl_words, st));
    P2G_CU(cudaMemcpyAsync(D + o_bands, H + o_bands, o_sid - o_bands, cudaMemcpyHostToDevice, st));
    if (j.have_set_id) {
        P2G_CU(cudaMemcpyAsync(D + o_sid, H + o_sid, 16, cudaMemcpyHostToDevice, st));
        if (chains) {  // the set id is given: chain segments may start at once
            static const uint32_t one = 1;
            P2G_CU(cudaMemcpyAsync(reinterpret_cast<uint32_t*>(D + o_ctl) + 1 + nb + 2 * Q, &one, 4,
                                   cudaMemcpyHostToDevice, st));
        }
    }
    const uint64_t np_bytes = round_up(j.slice, 16);
    if (j.R && j.S && 2ull * pl.zero_from_sym < np_bytes)
        P2G_CU(cudaMemset2DAsync(j.d_rec + 2ull * pl.zero_from_sym, j.rec_stride, 0,
                                 np_bytes - 2ull * pl.zero_from_sym, j.R, st));
    if (d.basis) P2G_CU(launch_basis(c.basis.as<uint16_t>(), j.S, RG, j.R, j.first_exp, st));
    if (mma)
        P2G_CU(launch_a_image_batch(reinterpret_cast<const BatchJob*>(D + o_desc), 1, mma_aimg_bytes(j.S, j.R), st));
    if (esrc != j.d_src) P2G_CU(launch_realign(j.d_src, j.slice, c.src_al.as<uint8_t>(), estride, j.S, j.slice, st));
    P2G_CU(launch_batch(reinterpret_cast<const BatchJob*>(D + o_desc), reinterpret_cast<const BatchItem*>(D + o_items),
                        (uint32_t)pl.items.size(), reinterpret_cast<uint32_t*>(D + o_ctl), err,
                        (uint32_t)device_sm_count(), st, mma));
    P2G_CU(cudaMemcpyAsync(c.h_err.p, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    P2G_CU(cudaEventRecord(c.ev_scratch, st));
    c.scratch_pending = true;
    if (j.progress && j.R && j.S) P2G_TRY(poll_progress(c, j, pl, reinterpret_cast<const uint32_t*>(D + o_ctl), st));
    if (!j.have_set_id) {
        // set id = MD5(main packet body) over the sorted file ids
        // (src/source.rs:303-309, src/packet/main_packet.rs:25-42); the
        // device derived the same value for the packet MD5s
        P2G_CU(c.h_h16k.ensure(16 * (size_t)n));
        P2G_CU(cudaMemcpyAsync(c.h_h16k.p, j.d_h16k, 16 * n, cudaMemcpyDeviceToHost, st));
        P2G_CU(cudaStreamSynchronize(st));
        P2G_TRY(check_device_error(c));  // the error word arrived with the hash16k values
        j.h16k.resize(n);
        j.file_ids.resize(n);
        for (uint32_t f = 0; f < n; ++f) {
            memcpy(j.h16k[f].data(), c.h_h16k.as<uint8_t>() + 16 * f, 16);
            j.file_ids[f] = file_id_of(j.h16k[f].data(), j.files[f].length, j.files[f].name, j.files[f].name_len);
        }
        std::vector<uint8_t> mp;
        j.set_id = build_main_packet(j.slice, j.file_ids, mp);
    }
    return P2G_OK;
}

// P2G_BANDED=1 selects the multi-stream banded pipeline below instead.
static p2g_status run_device_job(Context& c, DeviceJob& j, cudaStream_t caller) {
    if (!getenv("P2G_BANDED")) return run_device_job_persistent(c, j, caller);
    const uint32_t n = (uint32_t)j.files.size();
    const uint32_t RG = (j.R + kRowsPerGroup - 1) / kRowsPerGroup;
    P2G_TRY(fork_from(c, caller));
    Tracer tr;
    tr.start(caller);
    cudaStream_t s_enc = c.st[0], s_files = c.st[1], s_md5 = c.st[2], s_crc = c.st[3], s_full = c.st[4];
    P2G_CU(cudaMemsetAsync(c.err.p, 0, sizeof(int), s_enc));

    // per-file spans: [0, n) hash16k spans, [n, 2n) hash_full spans
    const bool need_files = j.d_h16k && n > 0;
    if (need_files) {
        P2G_CU(c.h_spans.ensure(sizeof(FileSpan) * 2 * n));
        P2G_CU(c.spans.ensure(sizeof(FileSpan) * 2 * n));
        FileSpan* hs = c.h_spans.as<FileSpan>();
        for (uint32_t f = 0; f < n; ++f) {
            hs[f] = {j.files[f].first_slice * j.slice, std::min<uint64_t>(j.files[f].length, P2G_HASH16K_LEN)};
            hs[n + f] = {j.files[f].first_slice * j.slice, j.files[f].length};
        }
        P2G_CU(cudaMemcpyAsync(c.spans.p, hs, sizeof(FileSpan) * 2 * n, cudaMemcpyHostToDevice, s_files));
        P2G_CU(launch_md5_files(j.d_src, c.spans.as<FileSpan>(), n, j.d_h16k, s_files));
        if (!j.have_set_id) {
            P2G_CU(c.h_h16k.ensure(16 * n));
            P2G_CU(cudaMemcpyAsync(c.h_h16k.p, j.d_h16k, 16 * n, cudaMemcpyDeviceToHost, s_files));
        }
        P2G_CU(cudaEventRecord(c.ev_h16k, s_files));
        tr.mark("hash16k + D2H", s_files);
        if (j.d_hfull) {
            P2G_CU(cudaStreamWaitEvent(s_full, c.ev_h16k, 0));  // spans uploaded
            P2G_CU(launch_md5_files(j.d_src, c.spans.as<FileSpan>() + n, n, j.d_hfull, s_full));
            tr.mark("hash_full", s_full);
        }
    }
    if (j.d_checks && j.S) {
        P2G_CU(launch_md5_slices(j.d_src, j.slice, j.S, j.slice, j.d_checks, s_md5));
        tr.mark("slice md5", s_md5);
        // CRC32 is light but shared-memory and ALU heavy: run it after the
        // last encode band (see below), alongside the final packet-MD5 step.
    }
    // Banded encode: band b covers a contiguous symbol range of every row, so
    // the recovery-packet MD5 chains (one per row, src/format.rs:33-54) can
    // follow band by band while later bands are still encoding.
    EncodePlan plan;
    cudaStream_t s_enc2 = c.st[5], s_pkt = c.st[6];
    const bool gen = generate_basis();
    if (j.R && j.S) {
        if (!gen) {
            P2G_CU(c.basis.ensure(basis_bytes(j.S, RG)));
            P2G_CU(launch_basis(c.basis.as<uint16_t>(), j.S, RG, j.R, j.first_exp, s_enc));
        }
        const uint8_t* esrc = j.d_src;
        uint64_t estride = j.slice;
        if (j.slice % 16) {  // the TMA tile loads need 16-byte aligned slice starts
            estride = round_up(j.slice, 16);
            P2G_CU(c.src_al.ensure((size_t)estride * j.S));
            P2G_CU(launch_realign(j.d_src, j.slice, c.src_al.as<uint8_t>(), estride, j.S, j.slice, s_enc));
            esrc = c.src_al.as<uint8_t>();
        }
        // slice-MD5 (and device whole-file MD5) blocks each hold an SM for
        // about chain-length x 0.72 us per 64-byte block
        uint32_t reserve = hash_blocks(j.d_checks ? j.S : 0) + hash_blocks(j.d_h16k ? n : 0);
        double reserve_ms = j.d_checks ? (double)(j.slice / 64) * 7.2e-4 : 0.0;
        if (j.d_hfull) {
            uint64_t mx = 0;
            for (const auto& f : j.files) mx = std::max(mx, f.length);
            reserve += hash_blocks(n);
            reserve_ms = std::max(reserve_ms, (double)(mx / 64) * 7.2e-4);
        }
        plan = plan_encode(j.slice, j.S, RG, j.d_pkt != nullptr, reserve, reserve_ms, tail_fold(j.R));
        if (plan.bands.size() > (size_t)Context::kBandEvents)
            plan = plan_encode(j.slice, j.S, RG, false, 0, 0.0, tail_fold(j.R));
        tr.mark("basis", s_enc);
        P2G_CU(cudaEventRecord(c.ev_band[0], s_enc));  // basis (and realign) done
        P2G_CU(cudaStreamWaitEvent(s_enc2, c.ev_band[0], 0));
        for (uint32_t b = 0; b < (uint32_t)plan.bands.size(); ++b) {
            // one stream: band b+1 starts when band b's wave drains, so bands
            // complete in order and each packet-MD5 step can start early
            cudaStream_t sb = s_enc;
            P2G_CU(launch_encode_band(plan, b, esrc, estride, j.S, gen ? nullptr : c.basis.as<uint16_t>(), RG, j.R,
                                      j.d_rec, j.rec_stride, c.err.as<int>(), sb, j.first_exp));
            P2G_CU(cudaEventRecord(c.ev_band[b], sb));
            tr.mark("encode band", sb);
        }
    }
    if (j.d_checks && j.S) {
        if (j.R) P2G_CU(cudaStreamWaitEvent(s_crc, c.ev_band[plan.bands.size() - 1], 0));
        P2G_CU(launch_crc_slices(j.d_src, j.slice, j.S, j.slice, j.d_checks, s_crc));
        tr.mark("slice crc32", s_crc);
    }
    if (!j.have_set_id) {
        // set id = MD5(main packet body) over the sorted file ids
        // (src/source.rs:303-309, src/packet/main_packet.rs:25-42)
        P2G_CU(cudaEventSynchronize(c.ev_h16k));
        j.h16k.resize(n);
        j.file_ids.resize(n);
        for (uint32_t f = 0; f < n; ++f) {
            memcpy(j.h16k[f].data(), c.h_h16k.as<uint8_t>() + 16 * f, 16);
            j.file_ids[f] = file_id_of(j.h16k[f].data(), j.files[f].length, j.files[f].name, j.files[f].name_len);
        }
        std::vector<uint8_t> mp;
        j.set_id = build_main_packet(j.slice, j.file_ids, mp);
    }
    if (j.R && j.S && j.d_pkt) {
        P2G_CU(c.md5_state.ensure(16 * (size_t)j.R));
        const uint64_t total = 36 + j.slice;
        const uint64_t nblocks = (total + 8) / 64 + 1;
        uint64_t done = 0;
        for (uint32_t b = 0; b < (uint32_t)plan.bands.size(); ++b) {
            P2G_CU(cudaStreamWaitEvent(s_pkt, c.ev_band[b], 0));
            const bool final = b + 1 == plan.bands.size();
            const uint64_t complete = std::min<uint64_t>(j.slice, 2ull * plan.bands[b].end);
            const uint64_t upto = final ? nblocks : (36 + complete) / 64;
            P2G_CU(launch_md5_recovery_range(j.d_rec, j.rec_stride, j.R, j.slice, j.set_id.data(), j.first_exp,
                                             c.md5_state.as<uint32_t>(), done, upto, final, j.d_pkt, s_pkt));
            tr.mark("packet md5 band", s_pkt);
            done = upto;
        }
    } else if (j.R && j.d_pkt) {  // S == 0: all-zero recovery rows
        P2G_CU(launch_md5_recovery(j.d_rec, j.rec_stride, j.R, j.slice, j.set_id.data(), j.first_exp, j.d_pkt, s_enc));
    }
    P2G_CU(cudaMemcpyAsync(c.h_err.p, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, s_enc));
    P2G_TRY(join_into(c, caller));
    tr.mark("joined", caller);
    tr.finish();
    return P2G_OK;
}

static p2g_status check_device_error(Context& c) {
    if (*c.h_err.as<int>() != 0)
        return set_error(P2G_ERR_TIMEOUT, "a bounded device wait gave up (TMA stage never completed)");
    return P2G_OK;
}

static void emit(p2g_progress_fn cb, void* user, p2g_progress_event ev) {
    if (cb) cb(&ev, user);
}
static p2g_progress_event mk(uint32_t kind) {
    p2g_progress_event e;
    memset(&e, 0, sizeof e);
    e.kind = kind;
    return e;
}

// ---------------------------------------------------------------------------
// Input files: mapped read-only (like scan_via_mmap, src/source.rs:145-232),
// so the whole-file hash threads start on the page cache at once and the
// upload copies from the mapping; no staging copy, no pinning of the input.
// Files that cannot be mapped are read into pinned memory instead.
// ---------------------------------------------------------------------------
struct HostFile {
    std::string path;
    uint64_t length = 0;
    uint8_t* data = nullptr;  // mapping, or pinned copy when !mapped
    size_t map_len = 0;
    bool mapped = false;
    ~HostFile() {
        if (data && mapped) munmap(data, map_len);
        else if (data) cudaFreeHost(data);
    }
};
static p2g_status stat_len(const char* path, uint64_t* len) {
    struct stat sb;
    if (stat(path, &sb) != 0) return set_error(P2G_ERR_IO, "I/O error: %s: %s", path, strerror(errno));
    *len = (uint64_t)sb.st_size;
    return P2G_OK;
}
static p2g_status read_file(HostFile& hf, uint64_t max_bytes) {
    const int fd = open(hf.path.c_str(), O_RDONLY | O_CLOEXEC);
    if (fd < 0) return set_error(P2G_ERR_IO, "I/O error: %s: %s", hf.path.c_str(), strerror(errno));
    struct stat sb;
    fstat(fd, &sb);
    hf.length = std::min<uint64_t>((uint64_t)sb.st_size, max_bytes);
    if (S_ISREG(sb.st_mode) && hf.length > 0 && !getenv("P2G_NO_MMAP")) {
        void* m = mmap(nullptr, hf.length, PROT_READ, MAP_PRIVATE, fd, 0);
        if (m != MAP_FAILED) {
            madvise(m, hf.length, MADV_SEQUENTIAL);
            close(fd);
            hf.data = static_cast<uint8_t*>(m);
            hf.map_len = hf.length;
            hf.mapped = true;
            return P2G_OK;
        }
    }
    if (cudaHostAlloc((void**)&hf.data, std::max<uint64_t>(hf.length, 1), cudaHostAllocDefault) != cudaSuccess) {
        close(fd);
        cudaGetLastError();
        return set_error(P2G_ERR_OOM, "pinned host allocation of %llu bytes failed", (unsigned long long)hf.length);
    }
    uint64_t got = 0;
    while (got < hf.length) {
        const ssize_t r = read(fd, hf.data + got, std::min<uint64_t>(hf.length - got, 1u << 30));
        if (r < 0) {
            if (errno == EINTR) continue;
            const int e = errno;
            close(fd);
            return set_error(P2G_ERR_IO, "I/O error: %s: %s", hf.path.c_str(), strerror(e));
        }
        if (r == 0) break;
        got += (uint64_t)r;
    }
    hf.length = got;
    close(fd);
    return P2G_OK;
}

// ---------------------------------------------------------------------------
// Core in-memory create: upload, device job, download, packet assembly.
// ---------------------------------------------------------------------------
struct CreateInput {
    const uint8_t* data;  // host
    uint64_t length;
    const uint8_t* name;
    size_t name_len;
    const char* path;  // for messages / events
};
struct CreateOutput {
    std::vector<uint8_t> critical;
    Md5 set_id;
    std::vector<uint32_t> vol_sizes;
    uint8_t* rec_host = nullptr;  // pinned, R*slice
    std::vector<uint8_t> pkt_md5;  // 16*R
    std::vector<p2g_source_file> sources;  // scanned records (owned here until handed out)
};

static void free_source(p2g_source_file& sf) {
    free(sf.name);
    free(sf.path);
    free(sf.slice_checksums);
    memset(&sf, 0, sizeof sf);
}

// Builds the critical packet block of run_create_with_progress
// (src/creator.rs:219-235).
static Md5 critical_packets(uint64_t slice, const p2g_source_file* src, uint32_t n, const char* const* comments,
                            uint32_t n_comments, std::vector<uint8_t>& out) {
    std::vector<Md5> ids(n);
    for (uint32_t f = 0; f < n; ++f) memcpy(ids[f].data(), src[f].file_id, 16);
    out.clear();
    const Md5 set_id = build_main_packet(slice, ids, out);
    for (uint32_t f = 0; f < n; ++f) {
        append_file_desc(out, set_id, ids[f], src[f].hash_full, src[f].hash16k, src[f].length, src[f].name,
                         src[f].name_len);
        append_file_verify(out, set_id, ids[f], src[f].slice_checksums, src[f].slice_count);
    }
    append_creator(out, set_id);
    for (uint32_t i = 0; i < n_comments; ++i) append_comments(out, set_id, comments[i]);
    return set_id;
}

// Byte length of the critical packet block of n inputs, before any of them
// is hashed: the packets' sizes depend on names, lengths and slice counts
// only, so zero hashes and checksums stand in.
static size_t critical_len_of(uint64_t slice, const CreateInput* in, uint32_t n, const char* const* comments,
                              uint32_t n_comments) {
    std::vector<p2g_source_file> src(n);
    uint64_t max_slices = 0;
    for (uint32_t f = 0; f < n; ++f) max_slices = std::max<uint64_t>(max_slices, (in[f].length + slice - 1) / slice);
    std::vector<p2g_slice_checksum> zero(std::max<uint64_t>(max_slices, 1));
    memset(zero.data(), 0, sizeof(p2g_slice_checksum) * zero.size());
    for (uint32_t f = 0; f < n; ++f) {
        memset(&src[f], 0, sizeof src[f]);
        src[f].name = const_cast<uint8_t*>(in[f].name);
        src[f].name_len = in[f].name_len;
        src[f].length = in[f].length;
        src[f].slice_count = (in[f].length + slice - 1) / slice;
        src[f].slice_checksums = zero.data();
    }
    std::vector<uint8_t> out;
    critical_packets(slice, src.data(), n, comments, n_comments, out);
    return out.size();
}

// Pinned host copy of a create call's recovery rows.  The context keeps the
// buffer for the next call (pinning ~100 MB takes tens of milliseconds)
// unless it grew past kRetainPinnedRec.
constexpr size_t kRetainPinnedRec = size_t(1) << 30;
struct PinnedRec {
    PinBuf& buf;
    uint8_t* p = nullptr;
    explicit PinnedRec(Context& c) : buf(c.h_rec) {}
    cudaError_t ensure(size_t n) {
        const cudaError_t e = buf.ensure(n);
        p = buf.as<uint8_t>();
        return e;
    }
    ~PinnedRec() {
        if (buf.cap > kRetainPinnedRec) {
            cudaFreeHost(buf.p);
            buf.p = nullptr;
            buf.cap = 0;
        }
    }
};

// Work a create call can do while the host is still hashing whole files:
// called with the device results (set id, packet MD5s, recovery rows) and
// the byte length the critical packet block will have.
using WhileHashing = std::function<void(const CreateOutput&, size_t critical_len)>;

// Scan (+ encode when R > 0) n in-memory inputs on the device.
// `src_known` (optional): already-scanned SourceFile records; then only the
// encode and the packet MD5s run and the critical packets use them.
static p2g_status device_create(Context& c, const CreateInput* in, uint32_t n, uint64_t slice, uint32_t R,
                                const p2g_source_file* src_known, const char* const* comments, uint32_t n_comments,
                                CreateOutput& out, PinnedRec& rec_host,
                                const WhileHashing* while_hashing = nullptr,
                                const std::function<void(uint64_t, uint64_t)>* progress = nullptr) {
    std::vector<JobFile> files(n);
    uint64_t S = 0;
    for (uint32_t f = 0; f < n; ++f) {
        const uint64_t slices = src_known ? src_known[f].slice_count : (in[f].length + slice - 1) / slice;
        files[f] = {in[f].length, S, slices, in[f].name, in[f].name_len};
        S += slices;
    }
    const uint64_t rec_stride = round_up(slice, 16);
    const size_t src_bytes = (size_t)S * slice;
    P2G_CU(c.src.ensure(src_bytes));
    if (R) {
        P2G_CU(c.rec.ensure((size_t)R * rec_stride));
        P2G_CU(c.pkt.ensure(16 * (size_t)R));
    }
    if (!src_known) {
        P2G_CU(c.checks.ensure(sizeof(p2g_slice_checksum) * std::max<uint64_t>(S, 1)));
        P2G_CU(c.hfull.ensure(16 * (size_t)n));
    }
    P2G_CU(c.h16k.ensure(16 * (size_t)n));

    // Whole-file MD5 placement and host-side hashing in the background.
    std::vector<uint64_t> lens(n);
    std::vector<const uint8_t*> ptrs(n);
    for (uint32_t f = 0; f < n; ++f) {
        lens[f] = in[f].length;
        ptrs[f] = in[f].data;
    }
    const FileHashMode fmode = src_known ? FileHashMode::Host : choose_file_hash_mode(lens);
    std::vector<Md5> host_full;  // declared before the hasher: its threads write here until joined
    HostHasher hh;
    if (!src_known && fmode == FileHashMode::Host) hh.start(ptrs, lens, host_full);

    // Upload: each file to its first slice, zero the tail of its last slice.
    // Many page-locked inputs go in one launch that reads them over the bus
    // (thousands of small copies and memsets cost more in calls than in
    // bytes); the rest, and a few large files, by cudaMemcpyAsync.
    cudaStream_t up = c.st[0];
    std::vector<uint8_t> pinned(n, 0);
    uint32_t n_pinned = 0;
    for (uint32_t f = 0; f < n && n >= kGatherMinFiles; ++f) {
        cudaPointerAttributes pa;
        if (in[f].length && cudaPointerGetAttributes(&pa, in[f].data) == cudaSuccess &&
            pa.type == cudaMemoryTypeHost && pa.devicePointer == in[f].data) {
            pinned[f] = 1;
            ++n_pinned;
        }
        cudaGetLastError();  // an unregistered pointer is not an error here
    }
    std::vector<uint64_t> seg;
    if (n_pinned >= kGatherMinFiles) seg.reserve(3 * (size_t)(n_pinned + src_bytes / kGatherSegBytes + 1));
    for (uint32_t f = 0; f < n; ++f) {
        uint8_t* dst = c.src.as<uint8_t>() + files[f].first_slice * slice;
        const uint64_t cap = files[f].slices * slice;
        const uint64_t cp = std::min(in[f].length, cap);
        if (n_pinned >= kGatherMinFiles && pinned[f]) {
            const bool pad_in_seg = cap - cp < (1ull << 24);
            if (!pad_in_seg) P2G_CU(cudaMemsetAsync(dst + cp, 0, cap - cp, up));
            for (uint64_t o = 0; o < cp; o += kGatherSegBytes) {
                const uint64_t len = std::min<uint64_t>(kGatherSegBytes, cp - o);
                const uint64_t pad = o + len == cp && pad_in_seg ? cap - cp : 0;
                seg.push_back((uint64_t)(uintptr_t)(in[f].data + o));
                seg.push_back((uint64_t)(uintptr_t)(dst + o));
                seg.push_back(len | (pad << 40));
            }
            continue;
        }
        if (cp) P2G_CU(cudaMemcpyAsync(dst, in[f].data, cp, cudaMemcpyHostToDevice, up));
        if (cap > cp) P2G_CU(cudaMemsetAsync(dst + cp, 0, cap - cp, up));
    }
    if (!seg.empty()) {
        const size_t bytes = 8 * seg.size();
        P2G_CU(c.h_gseg.ensure(bytes));
        P2G_CU(c.gseg.ensure(bytes));
        memcpy(c.h_gseg.p, seg.data(), bytes);
        P2G_CU(cudaMemcpyAsync(c.gseg.p, c.h_gseg.p, bytes, cudaMemcpyHostToDevice, up));
        P2G_CU(launch_gather_host(c.gseg.as<uint64_t>(), (uint32_t)(seg.size() / 3), up));
    }
    P2G_CU(cudaStreamSynchronize(up));

    DeviceJob j;
    j.d_src = c.src.as<uint8_t>();
    j.S = (uint32_t)S;
    j.slice = slice;
    j.R = R;
    j.first_exp = 0;
    j.files = files;
    j.d_rec = c.rec.as<uint8_t>();
    j.rec_stride = rec_stride;
    j.d_checks = src_known ? nullptr : c.checks.as<p2g_slice_checksum>();
    j.d_h16k = src_known ? nullptr : c.h16k.as<uint8_t>();
    j.d_hfull = (!src_known && fmode == FileHashMode::Device) ? c.hfull.as<uint8_t>() : nullptr;
    j.d_pkt = R ? c.pkt.as<uint8_t>() : nullptr;
    std::vector<uint8_t> crit;
    std::vector<p2g_source_file> scanned;
    if (src_known) {
        j.set_id = critical_packets(slice, src_known, n, comments, n_comments, crit);
        j.have_set_id = true;
    }
    cudaStream_t main = c.st[0];
    if (progress) j.progress = *progress;
    P2G_TRY(run_device_job(c, j, main));

    // Downloads
    if (R) {
        P2G_CU(rec_host.ensure((size_t)R * slice));
        P2G_CU(cudaMemcpy2DAsync(rec_host.p, slice, c.rec.p, rec_stride, slice, R, cudaMemcpyDeviceToHost, main));
        out.pkt_md5.resize(16 * (size_t)R);
        P2G_CU(c.h_stage.ensure(16 * (size_t)R));
        P2G_CU(cudaMemcpyAsync(c.h_stage.p, c.pkt.p, 16 * (size_t)R, cudaMemcpyDeviceToHost, main));
    }
    std::vector<p2g_slice_checksum> checks;
    std::vector<uint8_t> hfull_dev;
    if (!src_known) {
        checks.resize(S);
        if (S) P2G_CU(cudaMemcpyAsync(checks.data(), c.checks.p, sizeof(p2g_slice_checksum) * S,
                                      cudaMemcpyDeviceToHost, main));
        if (fmode == FileHashMode::Device) {
            hfull_dev.resize(16 * (size_t)n);
            P2G_CU(cudaMemcpyAsync(hfull_dev.data(), c.hfull.p, 16 * (size_t)n, cudaMemcpyDeviceToHost, main));
        }
    }
    P2G_CU(cudaStreamSynchronize(main));
    P2G_TRY(check_device_error(c));
    if (R) memcpy(out.pkt_md5.data(), c.h_stage.p, 16 * (size_t)R);
    out.set_id = j.set_id;
    out.rec_host = rec_host.p;

    if (!src_known) {
        scanned.resize(n);
        for (uint32_t f = 0; f < n; ++f) {
            p2g_source_file& sf = scanned[f];
            memset(&sf, 0, sizeof sf);
            sf.name = (uint8_t*)malloc(std::max<size_t>(in[f].name_len, 1));
            memcpy(sf.name, in[f].name, in[f].name_len);
            sf.name_len = in[f].name_len;
            const char* pth = in[f].path ? in[f].path : "";
            sf.path = strdup(pth);
            sf.length = in[f].length;
            memcpy(sf.hash16k, j.h16k[f].data(), 16);
            memcpy(sf.file_id, j.file_ids[f].data(), 16);
            if (fmode == FileHashMode::Device) memcpy(sf.hash_full, hfull_dev.data() + 16 * f, 16);
            sf.slice_count = files[f].slices;
            sf.slice_checksums = (p2g_slice_checksum*)malloc(sizeof(p2g_slice_checksum) * std::max<uint64_t>(1, sf.slice_count));
            memcpy(sf.slice_checksums, checks.data() + files[f].first_slice, sizeof(p2g_slice_checksum) * sf.slice_count);
        }
    }
    if (while_hashing) {
        // the critical block's length does not depend on the whole-file hashes
        size_t crit_len = crit.size();
        if (!src_known) {
            std::vector<uint8_t> probe;
            critical_packets(slice, scanned.data(), n, comments, n_comments, probe);
            crit_len = probe.size();
        }
        (*while_hashing)(out, crit_len);
    }
    hh.join();

    if (!src_known) {
        if (fmode == FileHashMode::Host)
            for (uint32_t f = 0; f < n; ++f) memcpy(scanned[f].hash_full, host_full[f].data(), 16);
        const Md5 sid = critical_packets(slice, scanned.data(), n, comments, n_comments, crit);
        if (sid != j.set_id) {
            for (auto& sf : scanned) free_source(sf);
            return set_error(P2G_ERR_CUDA, "internal: set id mismatch between device job and packet assembly");
        }
    }
    out.critical = std::move(crit);
    out.sources = std::move(scanned);
    return P2G_OK;
}

// Byte pieces of one volume file: critical ‖ recovery packets ‖ critical
// (build_volume_packet, src/creator.rs:1025-1042).
static void volume_pieces_recovery(const CreateOutput& o, uint64_t slice, uint32_t first, uint32_t count,
                                   std::vector<uint8_t>& headers,
                                   std::vector<std::pair<const uint8_t*, size_t>>& pieces) {
    headers.assign(68 * (size_t)count, 0);
    pieces.clear();
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t e = first + k;
        recovery_packet_header(headers.data() + 68 * (size_t)k, o.set_id, o.pkt_md5.data() + 16 * (size_t)e, slice, e);
        pieces.push_back({headers.data() + 68 * (size_t)k, 68});
        pieces.push_back({o.rec_host + (size_t)e * slice, (size_t)slice});
    }
}
static void volume_pieces(const CreateOutput& o, uint64_t slice, uint32_t first, uint32_t count,
                          std::vector<uint8_t>& headers, std::vector<std::pair<const uint8_t*, size_t>>& pieces) {
    std::vector<std::pair<const uint8_t*, size_t>> mid;
    volume_pieces_recovery(o, slice, first, count, headers, mid);
    pieces.clear();
    pieces.push_back({o.critical.data(), o.critical.size()});
    pieces.insert(pieces.end(), mid.begin(), mid.end());
    pieces.push_back({o.critical.data(), o.critical.size()});
}

static char* dupstr(const std::string& s) {
    char* r = (char*)malloc(s.size() + 1);
    memcpy(r, s.c_str(), s.size() + 1);
    return r;
}

static void fill_path_list(p2g_path_list* out, const std::vector<std::string>& v) {
    if (!out) return;
    out->count = (uint32_t)v.size();
    out->paths = (char**)calloc(std::max<size_t>(v.size(), 1), sizeof(char*));
    for (size_t i = 0; i < v.size(); ++i) out->paths[i] = dupstr(v[i]);
}

}  // namespace p2g

using namespace p2g;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" uint64_t p2g_kernel_launch_count(void) { return launch_count(); }

extern "C" p2g_status p2g_device_info(char* buf, size_t cap) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    P2G_TRY(ensure_ready(c));
    cudaDeviceProp prop;
    P2G_CU(cudaGetDeviceProperties(&prop, c.device));
    if (buf && cap) snprintf(buf, cap, "%s sm_%d%d SMs=%d mem=%zuMiB", prop.name, prop.major, prop.minor,
                             prop.multiProcessorCount, prop.totalGlobalMem >> 20);
    return P2G_OK;
}

extern "C" void p2g_source_file_free(p2g_source_file* sf) {
    if (sf) free_source(*sf);
}
extern "C" void p2g_path_list_free(p2g_path_list* pl) {
    if (!pl) return;
    for (uint32_t i = 0; i < pl->count; ++i) free(pl->paths[i]);
    free(pl->paths);
    pl->paths = nullptr;
    pl->count = 0;
}
extern "C" void p2g_string_free(char* s) { free(s); }
extern "C" void p2g_output_set_free(p2g_output_set* os) {
    if (!os) return;
    for (uint32_t i = 0; i < os->count; ++i) {
        free(os->files[i].name);
        free(os->files[i].data);
    }
    free(os->files);
    os->files = nullptr;
    os->count = 0;
}

extern "C" p2g_status p2g_check_bounded_wait(uint32_t polls) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (polls == 0 || polls > (1u << 24)) return set_error(P2G_ERR_INVALID_ARGUMENT, "polls must be in [1, 2^24]");
    P2G_TRY(ensure_ready(c));
    cudaStream_t s = c.st[0];
    P2G_CU(c.err.ensure(sizeof(int)));
    P2G_CU(cudaMemsetAsync(c.err.p, 0, sizeof(int), s));
    P2G_CU(launch_bounded_wait_probe(c.err.as<int>(), polls, s));
    int gave_up = 0;
    P2G_CU(cudaMemcpyAsync(&gave_up, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaStreamSynchronize(s));
    if (gave_up) return set_error(P2G_ERR_TIMEOUT, "a bounded device wait gave up (diagnostic barrier never completes)");
    return P2G_OK;
}

// ---- seams ----------------------------------------------------------------
extern "C" p2g_status p2g_gf_mul_xor(uint16_t coeff, const uint8_t* input, uint8_t* output, size_t len,
                                     uint32_t flags, void* stream) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (len % 2) return set_error(P2G_ERR_INVALID_ARGUMENT, "buffer length must be even (16-bit symbols)");
    if (len && (!input || !output)) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL buffer");
    P2G_TRY(ensure_ready(c));
    if (!len) return P2G_OK;
    if (flags & P2G_DEVICE_POINTERS) {
        P2G_CU(launch_gf_mul_xor(coeff, input, output, len, (cudaStream_t)stream));
        return P2G_OK;
    }
    P2G_CU(c.tmp_in.ensure(len));
    P2G_CU(c.tmp_out.ensure(len));
    cudaStream_t s = c.st[0];
    P2G_CU(cudaMemcpyAsync(c.tmp_in.p, input, len, cudaMemcpyHostToDevice, s));
    P2G_CU(cudaMemcpyAsync(c.tmp_out.p, output, len, cudaMemcpyHostToDevice, s));
    P2G_CU(launch_gf_mul_xor(coeff, c.tmp_in.as<uint8_t>(), c.tmp_out.as<uint8_t>(), len, s));
    P2G_CU(cudaMemcpyAsync(output, c.tmp_out.p, len, cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaStreamSynchronize(s));
    return P2G_OK;
}

extern "C" p2g_status p2g_encode(const p2g_encode_job* job) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (!job) return set_error(P2G_ERR_INVALID_ARGUMENT, "job is NULL");
    const p2g_encode_job& jb = *job;
    if (jb.slice_size == 0 || jb.slice_size % 4)
        return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size %llu: must be > 0 and a multiple of 4",
                         (unsigned long long)jb.slice_size);
    if (jb.input_count > P2G_MAX_INPUT_BLOCKS)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "input_count %u exceeds 32768", jb.input_count);
    if ((uint64_t)jb.first_exponent + jb.recovery_count > 65536ull)
        return set_error(P2G_ERR_TOO_MANY_RECOVERY_BLOCKS, "recovery exponents exceed 65535");
    if (jb.src_stride < jb.slice_size || jb.recovery_stride < jb.slice_size)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "stride smaller than slice_size");
    P2G_TRY(ensure_ready(c));
    const uint32_t S = jb.input_count, R = jb.recovery_count;
    if (!R) return P2G_OK;
    const uint32_t RG = (R + kRowsPerGroup - 1) / kRowsPerGroup;
    if (jb.flags & P2G_DEVICE_POINTERS) {
        if (((uintptr_t)jb.src | (uintptr_t)jb.recovery) % 16 || jb.src_stride % 16 || jb.recovery_stride % 16)
            return set_error(P2G_ERR_INVALID_ARGUMENT,
                             "device encode needs 16-byte aligned pointers and strides that are multiples of 16");
        if (jb.recovery_stride < round_up(jb.slice_size, 16))
            return set_error(P2G_ERR_INVALID_ARGUMENT, "recovery_stride must be >= slice_size rounded up to 16");
        cudaStream_t s = (cudaStream_t)jb.stream;
        if (!S) {
            P2G_CU(cudaMemset2DAsync(jb.recovery, jb.recovery_stride, 0, jb.slice_size, R, s));
            return P2G_OK;
        }
        // the error word, bases and A image are the library's: a call on
        // another stream must not overwrite them while an earlier call reads
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        P2G_CU(cudaStreamIsCapturing(s, &cap));
        const bool order = cap == cudaStreamCaptureStatusNone;  // no outside event inside a capture
        if (order && c.scratch_pending) P2G_CU(cudaStreamWaitEvent(s, c.ev_scratch, 0));
        P2G_CU(cudaMemsetAsync(c.err.p, 0, sizeof(int), s));
        if (use_tensor_encode(jb.flags, S, R, jb.slice_size)) {
            P2G_CU(c.aimg.ensure(mma_aimg_bytes(S, R)));
            P2G_CU(launch_encode_mma(jb.src, jb.src_stride, S, jb.slice_size, R, jb.first_exponent,
                                     c.aimg.as<uint8_t>(), jb.recovery, jb.recovery_stride, c.err.as<int>(), s));
        } else {
            const bool gen = generate_basis();
            if (!gen) {
                P2G_CU(c.basis.ensure(basis_bytes(S, RG)));
                P2G_CU(launch_basis(c.basis.as<uint16_t>(), S, RG, R, jb.first_exponent, s));
            }
            P2G_CU(launch_encode(jb.src, jb.src_stride, S, gen ? nullptr : c.basis.as<uint16_t>(), RG, R,
                                 jb.slice_size, jb.recovery, jb.recovery_stride, c.err.as<int>(), s, jb.first_exponent));
        }
        if (order) {
            P2G_CU(cudaEventRecord(c.ev_scratch, s));
            c.scratch_pending = true;
        }
        if (jb.flags & P2G_ENCODE_WAIT) {
            P2G_CU(cudaMemcpyAsync(c.h_err.p, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            P2G_CU(cudaStreamSynchronize(s));
            return check_device_error(c);
        }
        return P2G_OK;
    }
    // host pointers: stage through device buffers (after any earlier call's
    // use of the shared scratch, whatever its stream)
    const uint64_t stride = round_up(jb.slice_size, 16);
    cudaStream_t s = c.st[0];
    if (c.scratch_pending) P2G_CU(cudaStreamWaitEvent(s, c.ev_scratch, 0));
    P2G_CU(c.src.ensure((size_t)stride * std::max<uint32_t>(S, 1)));
    P2G_CU(c.rec.ensure((size_t)stride * R));
    P2G_CU(cudaMemsetAsync(c.err.p, 0, sizeof(int), s));
    if (S) {
        P2G_CU(cudaMemcpy2DAsync(c.src.p, stride, jb.src, jb.src_stride, jb.slice_size, S, cudaMemcpyHostToDevice, s));
        if (stride != jb.slice_size)  // the 16-byte padding of each row is read: zero it
            P2G_CU(cudaMemset2DAsync(c.src.as<uint8_t>() + jb.slice_size, stride, 0, stride - jb.slice_size, S, s));
        if (use_tensor_encode(jb.flags, S, R, jb.slice_size)) {
            P2G_CU(c.aimg.ensure(mma_aimg_bytes(S, R)));
            P2G_CU(launch_encode_mma(c.src.as<uint8_t>(), stride, S, jb.slice_size, R, jb.first_exponent,
                                     c.aimg.as<uint8_t>(), c.rec.as<uint8_t>(), stride, c.err.as<int>(), s));
        } else {
            const bool gen = generate_basis();
            if (!gen) {
                P2G_CU(c.basis.ensure(basis_bytes(S, RG)));
                P2G_CU(launch_basis(c.basis.as<uint16_t>(), S, RG, R, jb.first_exponent, s));
            }
            P2G_CU(launch_encode(c.src.as<uint8_t>(), stride, S, gen ? nullptr : c.basis.as<uint16_t>(), RG, R,
                                 jb.slice_size, c.rec.as<uint8_t>(), stride, c.err.as<int>(), s, jb.first_exponent));
        }
    } else {
        P2G_CU(cudaMemsetAsync(c.rec.p, 0, (size_t)stride * R, s));
    }
    P2G_CU(cudaMemcpy2DAsync(jb.recovery, jb.recovery_stride, c.rec.p, stride, jb.slice_size, R,
                             cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaMemcpyAsync(c.h_err.p, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaStreamSynchronize(s));
    c.scratch_pending = false;  // all of it is done
    return check_device_error(c);
}

extern "C" p2g_status p2g_slice_checksums(const uint8_t* src, uint64_t src_stride, uint32_t count,
                                          uint64_t slice_size, p2g_slice_checksum* out, uint32_t flags,
                                          void* stream) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (slice_size == 0 || slice_size % 4)
        return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size %llu: must be > 0 and a multiple of 4",
                         (unsigned long long)slice_size);
    if (src_stride < slice_size || src_stride % 4 || (uintptr_t)src % 4)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "src must be 4-byte aligned with stride >= slice_size, multiple of 4");
    P2G_TRY(ensure_ready(c));
    if (!count) return P2G_OK;
    if (flags & P2G_DEVICE_POINTERS) {
        cudaStream_t s = (cudaStream_t)stream;
        P2G_CU(launch_md5_slices(src, src_stride, count, slice_size, out, s));
        P2G_CU(launch_crc_slices(src, src_stride, count, slice_size, out, s));
        return P2G_OK;
    }
    cudaStream_t s = c.st[0];
    P2G_CU(c.src.ensure((size_t)slice_size * count));
    P2G_CU(c.checks.ensure(sizeof(p2g_slice_checksum) * count));
    P2G_CU(cudaMemcpy2DAsync(c.src.p, slice_size, src, src_stride, slice_size, count, cudaMemcpyHostToDevice, s));
    P2G_CU(launch_md5_slices(c.src.as<uint8_t>(), slice_size, count, slice_size, c.checks.as<p2g_slice_checksum>(), s));
    P2G_CU(launch_crc_slices(c.src.as<uint8_t>(), slice_size, count, slice_size, c.checks.as<p2g_slice_checksum>(), s));
    P2G_CU(cudaMemcpyAsync(out, c.checks.p, sizeof(p2g_slice_checksum) * count, cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaStreamSynchronize(s));
    return P2G_OK;
}

extern "C" p2g_status p2g_file_hashes(const uint8_t* const* data, const uint64_t* lengths, uint32_t n,
                                      uint8_t* hash_full_out, uint8_t* hash16k_out, uint32_t flags, void* stream) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (n && (!data || !lengths)) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL arrays");
    P2G_TRY(ensure_ready(c));
    if (!n) return P2G_OK;
    for (uint32_t f = 0; f < n; ++f)
        if ((uintptr_t)data[f] % 4) return set_error(P2G_ERR_INVALID_ARGUMENT, "file %u data not 4-byte aligned", f);
    // Spans are offsets from a common base: the lowest pointer.
    const uint8_t* base = data[0];
    for (uint32_t f = 1; f < n; ++f) base = std::min(base, data[f]);
    P2G_CU(c.h_spans.ensure(sizeof(FileSpan) * 2 * n));
    P2G_CU(c.spans.ensure(sizeof(FileSpan) * 2 * n));
    FileSpan* hs = c.h_spans.as<FileSpan>();
    uint64_t total = 0;
    for (uint32_t f = 0; f < n; ++f) total += lengths[f];
    if (flags & P2G_DEVICE_POINTERS) {
        cudaStream_t s = (cudaStream_t)stream;
        for (uint32_t f = 0; f < n; ++f) {
            hs[f] = {(uint64_t)(data[f] - base), std::min<uint64_t>(lengths[f], P2G_HASH16K_LEN)};
            hs[n + f] = {(uint64_t)(data[f] - base), lengths[f]};
        }
        P2G_CU(cudaMemcpyAsync(c.spans.p, hs, sizeof(FileSpan) * 2 * n, cudaMemcpyHostToDevice, s));
        if (hash16k_out) P2G_CU(launch_md5_files(base, c.spans.as<FileSpan>(), n, hash16k_out, s));
        if (hash_full_out) P2G_CU(launch_md5_files(base, c.spans.as<FileSpan>() + n, n, hash_full_out, s));
        P2G_CU(cudaStreamSynchronize(s));  // h_spans is reused by the next call
        return P2G_OK;
    }
    cudaStream_t s = c.st[0];
    P2G_CU(c.src.ensure(std::max<uint64_t>(total + 16 * n, 16)));
    uint64_t off = 0;
    for (uint32_t f = 0; f < n; ++f) {
        hs[f] = {off, std::min<uint64_t>(lengths[f], P2G_HASH16K_LEN)};
        hs[n + f] = {off, lengths[f]};
        if (lengths[f]) P2G_CU(cudaMemcpyAsync(c.src.as<uint8_t>() + off, data[f], lengths[f], cudaMemcpyHostToDevice, s));
        off = round_up(off + lengths[f], 16);
    }
    P2G_CU(c.hfull.ensure(32 * (size_t)n));
    uint8_t* d16 = c.hfull.as<uint8_t>();
    uint8_t* dfull = d16 + 16 * (size_t)n;
    P2G_CU(cudaMemcpyAsync(c.spans.p, hs, sizeof(FileSpan) * 2 * n, cudaMemcpyHostToDevice, s));
    P2G_CU(launch_md5_files(c.src.as<uint8_t>(), c.spans.as<FileSpan>(), n, d16, s));
    P2G_CU(launch_md5_files(c.src.as<uint8_t>(), c.spans.as<FileSpan>() + n, n, dfull, s));
    if (hash16k_out) P2G_CU(cudaMemcpyAsync(hash16k_out, d16, 16 * (size_t)n, cudaMemcpyDeviceToHost, s));
    if (hash_full_out) P2G_CU(cudaMemcpyAsync(hash_full_out, dfull, 16 * (size_t)n, cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaStreamSynchronize(s));
    return P2G_OK;
}

extern "C" p2g_status p2g_recovery_packet_md5(const uint8_t set_id[16], const uint8_t* recovery,
                                              uint64_t recovery_stride, uint32_t count, uint64_t slice_size,
                                              uint16_t first_exponent, uint8_t* md5_out, uint32_t flags,
                                              void* stream) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (slice_size == 0 || slice_size % 4)
        return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size %llu", (unsigned long long)slice_size);
    if (recovery_stride < slice_size || recovery_stride % 4 || (uintptr_t)recovery % 4)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "recovery must be 4-byte aligned, stride >= slice_size");
    P2G_TRY(ensure_ready(c));
    if (!count) return P2G_OK;
    if (flags & P2G_DEVICE_POINTERS) {
        P2G_CU(launch_md5_recovery(recovery, recovery_stride, count, slice_size, set_id, first_exponent, md5_out,
                                   (cudaStream_t)stream));
        return P2G_OK;
    }
    cudaStream_t s = c.st[0];
    P2G_CU(c.rec.ensure((size_t)slice_size * count));
    P2G_CU(c.pkt.ensure(16 * (size_t)count));
    P2G_CU(cudaMemcpy2DAsync(c.rec.p, slice_size, recovery, recovery_stride, slice_size, count, cudaMemcpyHostToDevice, s));
    P2G_CU(launch_md5_recovery(c.rec.as<uint8_t>(), slice_size, count, slice_size, set_id, first_exponent,
                               c.pkt.as<uint8_t>(), s));
    P2G_CU(cudaMemcpyAsync(md5_out, c.pkt.p, 16 * (size_t)count, cudaMemcpyDeviceToHost, s));
    P2G_CU(cudaStreamSynchronize(s));
    return P2G_OK;
}

extern "C" p2g_status p2g_run_device_job(p2g_device_job* job) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (!job) return set_error(P2G_ERR_INVALID_ARGUMENT, "job is NULL");
    p2g_device_job& jb = *job;
    P2G_TRY(check_common(jb.file_count, jb.recovery_count, jb.slice_size));
    if (!jb.src || (uintptr_t)jb.src % 16 || (jb.recovery_count && ((uintptr_t)jb.recovery % 16 || jb.recovery_stride % 16 ||
                                                                    jb.recovery_stride < round_up(jb.slice_size, 16))))
        return set_error(P2G_ERR_INVALID_ARGUMENT,
                         "device job needs 16-byte aligned src/recovery and recovery_stride >= round_up(slice,16)");
    P2G_TRY(ensure_ready(c));
    DeviceJob j;
    uint64_t S = 0, total = 0;
    for (uint32_t f = 0; f < jb.file_count; ++f) {
        P2G_TRY(check_name(jb.names[f], jb.name_lens[f], ""));
        if (jb.file_lengths[f] == 0) return set_error(P2G_ERR_EMPTY_FILE, "input file %u is empty", f);
        const uint64_t sl = (jb.file_lengths[f] + jb.slice_size - 1) / jb.slice_size;
        j.files.push_back({jb.file_lengths[f], S, sl, jb.names[f], jb.name_lens[f]});
        S += sl;
        total += jb.file_lengths[f];
    }
    P2G_TRY(check_total_blocks(S, total, jb.slice_size));
    j.d_src = jb.src;
    j.S = (uint32_t)S;
    j.slice = jb.slice_size;
    j.R = jb.recovery_count;
    j.d_rec = jb.recovery;
    j.rec_stride = jb.recovery_stride;
    j.d_checks = jb.checksums;
    j.d_h16k = jb.hash16k;
    j.d_hfull = (jb.flags & P2G_JOB_SKIP_HASH_FULL) ? nullptr : jb.hash_full;
    j.variant = jb.flags & (P2G_ENCODE_LUT | P2G_ENCODE_TENSOR);
    j.d_pkt = jb.packet_md5;
    if (!j.d_h16k) return set_error(P2G_ERR_INVALID_ARGUMENT, "hash16k output is required (it derives the set id)");
    P2G_TRY(run_device_job(c, j, (cudaStream_t)jb.stream));
    memcpy(jb.set_id_out, j.set_id.data(), 16);
    return P2G_OK;
}

// ---- create pipeline ----------------------------------------------------
static p2g_status scan_impl(const char* path, const uint8_t* name, size_t name_len, uint64_t slice,
                            p2g_progress_fn cb, void* user, p2g_source_file* out) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (!path || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL argument");
    P2G_TRY(check_name(name, name_len, path));
    if (slice == 0 || slice % 4)
        return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size %llu: must be > 0 and a multiple of 4",
                         (unsigned long long)slice);
    uint64_t len = 0;
    P2G_TRY(stat_len(path, &len));
    if (len == 0) return set_error(P2G_ERR_EMPTY_FILE, "input file \"%s\" is empty; PAR2 requires non-empty files", path);
    const uint64_t total_slices = (len + slice - 1) / slice;
    p2g_progress_event ev = mk(P2G_EV_SCAN_STARTED);
    ev.path = path;
    ev.total_slices = total_slices;
    emit(cb, user, ev);
    P2G_TRY(ensure_ready(c));
    HostFile hf;
    hf.path = path;
    P2G_TRY(read_file(hf, len));
    if (hf.length == 0) return set_error(P2G_ERR_EMPTY_FILE, "input file \"%s\" is empty; PAR2 requires non-empty files", path);
    CreateInput in = {hf.data, hf.length, name, name_len, path};
    CreateOutput o;
    PinnedRec rec(c);
    P2G_TRY(device_create(c, &in, 1, slice, 0, nullptr, nullptr, 0, o, rec));
    const uint64_t done = o.sources[0].slice_count;
    ev = mk(P2G_EV_SCAN_PROGRESS);
    ev.path = path;
    ev.slices_done = done;
    ev.total_slices = done;
    emit(cb, user, ev);
    ev = mk(P2G_EV_SCAN_COMPLETED);
    ev.path = path;
    emit(cb, user, ev);
    *out = o.sources[0];
    o.sources.clear();
    return P2G_OK;
}

extern "C" p2g_status p2g_scan(const char* path, const uint8_t* display_name, size_t name_len, uint64_t slice_size,
                               p2g_source_file* out) {
    return scan_impl(path, display_name, name_len, slice_size, nullptr, nullptr, out);
}
extern "C" p2g_status p2g_scan_with_progress(const char* path, const uint8_t* display_name, size_t name_len,
                                             uint64_t slice_size, p2g_progress_fn cb, void* user,
                                             p2g_source_file* out) {
    return scan_impl(path, display_name, name_len, slice_size, cb, user, out);
}

// Writes the volume files of an already computed set on up to 8 threads (the
// reference writes volumes in parallel too, src/creator.rs:296-314); events
// follow in volume order.  On failure the volumes before the first failing
// one are reported written and its error is returned.
static p2g_status write_volumes(const std::string& output, const CreateOutput& co, uint64_t slice,
                                p2g_progress_fn cb, void* user, std::vector<std::string>& written) {
    const size_t nv = co.vol_sizes.size();
    std::vector<std::string> paths(nv);
    std::vector<uint32_t> firsts(nv);
    uint32_t first = 0;
    for (size_t v = 0; v < nv; ++v) {
        firsts[v] = first;
        paths[v] = volume_filename(output, (uint16_t)first, co.vol_sizes[v]);
        first += co.vol_sizes[v];
    }
    std::vector<p2g_status> st(nv, P2G_OK);
    std::vector<std::string> msg(nv);
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        std::vector<uint8_t> headers;
        std::vector<std::pair<const uint8_t*, size_t>> pieces;
        for (size_t v = next++; v < nv; v = next++) {
            volume_pieces(co, slice, firsts[v], co.vol_sizes[v], headers, pieces);
            st[v] = write_atomic(paths[v], pieces);
            if (st[v] != P2G_OK) msg[v] = p2g_last_error_message();
        }
    };
    run_on_threads((unsigned)std::min<size_t>(std::min(8u, std::max(1u, std::thread::hardware_concurrency())), nv),
                   worker);
    for (size_t v = 0; v < nv; ++v) {
        if (st[v] != P2G_OK) return set_error(st[v], "%s", msg[v].c_str());
        p2g_progress_event ev = mk(P2G_EV_VOLUME_WRITTEN);
        ev.path = paths[v].c_str();
        emit(cb, user, ev);
        written.push_back(paths[v]);
    }
    return P2G_OK;
}

// Volume files written in two passes around the host's whole-file hashes.
// While the files still hash, each volume's recovery packets (which need only
// the device results) go into its temporary file after room for the critical
// block.  Once the hashes are done, the critical block goes in at both ends,
// then fsync and rename as in write_atomic (src/creator.rs:1070-1087).
// Volumes are written on up to 8 threads; temp files are removed on failure.
struct StagedVolumes {
    std::vector<std::string> paths, tmps;
    std::vector<int> fds;
    std::vector<uint64_t> mid;  // recovery-packet bytes per volume
    size_t crit_len = 0;
    bool active = false;
    ~StagedVolumes() { discard(); }
    void discard() {
        for (size_t v = 0; v < fds.size(); ++v) {
            if (fds[v] >= 0) close(fds[v]);
            fds[v] = -1;
            if (!tmps[v].empty()) unlink(tmps[v].c_str());
        }
        active = false;
    }
    static p2g_status pwrite_all(int fd, const uint8_t* p, size_t n, uint64_t off, const std::string& path) {
        while (n) {
            const ssize_t w = pwrite(fd, p, n > (1u << 30) ? (1u << 30) : n, (off_t)off);
            if (w < 0) {
                if (errno == EINTR) continue;
                return set_error(P2G_ERR_IO, "I/O error: %s: %s", path.c_str(), strerror(errno));
            }
            p += w;
            n -= (size_t)w;
            off += (uint64_t)w;
        }
        return P2G_OK;
    }
    // runs fn(v) for every volume on a few threads; the first failure (in
    // volume order) is returned with its message
    template <class F>
    p2g_status each(F&& fn) {
        const size_t nv = paths.size();
        std::vector<p2g_status> st(nv, P2G_OK);
        std::vector<std::string> msg(nv);
        std::atomic<size_t> next{0};
        run_on_threads((unsigned)std::min<size_t>(std::min(8u, std::max(1u, std::thread::hardware_concurrency())),
                                                  std::max<size_t>(nv, 1)),
                       [&]() {
                           for (size_t v = next++; v < nv; v = next++) {
                               st[v] = fn(v);
                               if (st[v] != P2G_OK) msg[v] = p2g_last_error_message();
                           }
                       });
        for (size_t v = 0; v < nv; ++v)
            if (st[v] != P2G_OK) return set_error(st[v], "%s", msg[v].c_str());
        return P2G_OK;
    }
    p2g_status write_recovery(const std::string& output, const CreateOutput& o, uint64_t slice,
                              const std::vector<uint32_t>& vs, size_t clen) {
        const size_t nv = vs.size();
        paths.assign(nv, "");
        tmps.assign(nv, "");
        fds.assign(nv, -1);
        mid.assign(nv, 0);
        crit_len = clen;
        active = true;
        std::vector<uint32_t> firsts(nv);
        uint32_t first = 0;
        for (size_t v = 0; v < nv; ++v) {
            firsts[v] = first;
            paths[v] = volume_filename(output, (uint16_t)first, vs[v]);
            tmps[v] = paths[v] + ".par2rust.tmp";
            first += vs[v];
        }
        return each([&](size_t v) -> p2g_status {
            const int fd = open(tmps[v].c_str(), O_WRONLY | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
            if (fd < 0) return set_error(P2G_ERR_IO, "I/O error: %s: %s", tmps[v].c_str(), strerror(errno));
            fds[v] = fd;
            std::vector<uint8_t> headers;
            std::vector<std::pair<const uint8_t*, size_t>> pieces;
            volume_pieces_recovery(o, slice, firsts[v], vs[v], headers, pieces);
            uint64_t at = clen;
            for (auto& pc : pieces) {
                P2G_TRY(pwrite_all(fd, pc.first, pc.second, at, tmps[v]));
                at += pc.second;
            }
            mid[v] = at - clen;
            return P2G_OK;
        });
    }
    p2g_status finish(const std::vector<uint8_t>& critical, p2g_progress_fn cb, void* user,
                      std::vector<std::string>& written) {
        P2G_TRY(each([&](size_t v) -> p2g_status {
            P2G_TRY(pwrite_all(fds[v], critical.data(), critical.size(), 0, tmps[v]));
            P2G_TRY(pwrite_all(fds[v], critical.data(), critical.size(), crit_len + mid[v], tmps[v]));
            if (fsync(fds[v]) != 0) return set_error(P2G_ERR_IO, "I/O error: %s: %s", tmps[v].c_str(), strerror(errno));
            const int fd = fds[v];
            fds[v] = -1;
            if (close(fd) != 0) return set_error(P2G_ERR_IO, "I/O error: %s: %s", tmps[v].c_str(), strerror(errno));
            if (rename(tmps[v].c_str(), paths[v].c_str()) != 0)
                return set_error(P2G_ERR_IO, "I/O error: %s: %s", paths[v].c_str(), strerror(errno));
            tmps[v].clear();  // renamed: nothing to remove any more
            return P2G_OK;
        }));
        for (size_t v = 0; v < paths.size(); ++v) {
            p2g_progress_event ev = mk(P2G_EV_VOLUME_WRITTEN);
            ev.path = paths[v].c_str();
            emit(cb, user, ev);
            written.push_back(paths[v]);
        }
        active = false;
        return P2G_OK;
    }
};

// Writes the index and (if R > 0) volume files of an already computed set.
static p2g_status write_outputs(const p2g_create_options& o, const CreateOutput& co, uint32_t R, uint64_t slice,
                                p2g_progress_fn cb, void* user, std::vector<std::string>& written) {
    std::vector<std::pair<const uint8_t*, size_t>> pieces = {{co.critical.data(), co.critical.size()}};
    P2G_TRY(write_atomic(o.output, pieces));
    p2g_progress_event ev = mk(P2G_EV_INDEX_WRITTEN);
    ev.path = o.output;
    emit(cb, user, ev);
    written.push_back(o.output);
    if (!R) return P2G_OK;
    return write_volumes(o.output, co, slice, cb, user, written);
}

static void emit_encode_events(p2g_progress_fn cb, void* user, uint64_t S, uint32_t R, bool completed) {
    if (!completed) {
        p2g_progress_event ev = mk(P2G_EV_ENCODE_STARTED);
        ev.volume_index = 0;
        ev.total_volumes = 1;
        ev.input_blocks = S;
        ev.recovery_blocks = R;
        emit(cb, user, ev);
        return;
    }
    p2g_progress_event ev = mk(P2G_EV_ENCODE_PROGRESS);
    ev.input_block_done = S;
    ev.input_blocks = S;
    emit(cb, user, ev);
    ev = mk(P2G_EV_ENCODE_COMPLETED);
    emit(cb, user, ev);
}

static p2g_status run_create_impl(const p2g_create_options* opts, const p2g_source_file* sources, uint32_t n,
                                  p2g_progress_fn cb, void* user, p2g_path_list* out) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (!opts || !opts->output) return set_error(P2G_ERR_INVALID_ARGUMENT, "options/output is NULL");
    const uint32_t R = opts->recovery_block_count;
    const uint64_t slice = opts->slice_size;
    P2G_TRY(check_common(n, R, slice));
    uint64_t S = 0, total_bytes = 0;
    for (uint32_t f = 0; f < n; ++f) {
        S += sources[f].slice_count;
        total_bytes += sources[f].length;
    }
    P2G_TRY(check_total_blocks(S, total_bytes, slice));

    CreateOutput co;
    co.set_id = critical_packets(slice, sources, n, opts->comments, opts->comment_count, co.critical);
    std::vector<std::string> written;
    {  // index first (src/creator.rs:237-241)
        std::vector<std::pair<const uint8_t*, size_t>> pieces = {{co.critical.data(), co.critical.size()}};
        P2G_TRY(write_atomic(opts->output, pieces));
        p2g_progress_event ev = mk(P2G_EV_INDEX_WRITTEN);
        ev.path = opts->output;
        emit(cb, user, ev);
        written.push_back(opts->output);
    }
    if (R > 0) {
        P2G_TRY(resolve_volume_sizes(opts->volume_scheme, R, co.vol_sizes));
        P2G_TRY(ensure_ready(c));
        emit_encode_events(cb, user, S, R, false);
        // Re-read the sources (SourceReader, src/creator.rs:63-86): exactly the
        // slices listed in each SourceFile, zero-padded.
        std::vector<std::unique_ptr<HostFile>> hfs(n);
        std::vector<CreateInput> ins(n);
        for (uint32_t f = 0; f < n; ++f) {
            hfs[f].reset(new HostFile());
            hfs[f]->path = sources[f].path ? sources[f].path : "";
            P2G_TRY(read_file(*hfs[f], sources[f].slice_count * slice));
            ins[f] = {hfs[f]->data, hfs[f]->length, sources[f].name, sources[f].name_len, sources[f].path};
        }
        CreateOutput enc;
        PinnedRec rec(c);
        // encode progress from the device's item counter while it runs
        const std::function<void(uint64_t, uint64_t)> tick = [&](uint64_t done, uint64_t total) {
            p2g_progress_event ev = mk(P2G_EV_ENCODE_PROGRESS);
            ev.input_block_done = done;
            ev.input_blocks = total;
            emit(cb, user, ev);
        };
        P2G_TRY(device_create(c, ins.data(), n, slice, R, sources, opts->comments, opts->comment_count, enc, rec,
                              nullptr, cb ? &tick : nullptr));
        emit_encode_events(cb, user, S, R, true);
        co.rec_host = enc.rec_host;
        co.pkt_md5 = std::move(enc.pkt_md5);
        P2G_TRY(write_volumes(opts->output, co, slice, cb, user, written));
    }
    fill_path_list(out, written);
    return P2G_OK;
}

extern "C" p2g_status p2g_run_create(const p2g_create_options* opts, const p2g_source_file* sources, uint32_t n,
                                     p2g_path_list* out) {
    return run_create_impl(opts, sources, n, nullptr, nullptr, out);
}
extern "C" p2g_status p2g_run_create_with_progress(const p2g_create_options* opts, const p2g_source_file* sources,
                                                   uint32_t n, p2g_progress_fn cb, void* user, p2g_path_list* out) {
    return run_create_impl(opts, sources, n, cb, user, out);
}

extern "C" p2g_status p2g_write_index_file(const p2g_create_options* opts, const p2g_source_file* sources, uint32_t n,
                                           char** out_path) {
    if (!opts) return set_error(P2G_ERR_INVALID_ARGUMENT, "options is NULL");
    p2g_create_options o = *opts;
    o.recovery_block_count = 0;
    o.volume_scheme = p2g_volume_scheme{P2G_SCHEME_SINGLE, 0, 0, nullptr, nullptr, 0};
    p2g_path_list pl = {nullptr, 0};
    p2g_status st = run_create_impl(&o, sources, n, nullptr, nullptr, &pl);
    if (st != P2G_OK) return st;
    if (out_path) *out_path = dupstr(pl.paths[0]);
    p2g_path_list_free(&pl);
    return P2G_OK;
}

// Fused validation order, src/creator.rs:461-508.
static p2g_status fused_validate(uint32_t n, uint32_t R, uint64_t slice) { return check_common(n, R, slice); }

extern "C" p2g_status p2g_run_create_fused(const p2g_create_options* opts, const p2g_input* inputs, uint32_t n,
                                           p2g_progress_fn cb, void* user, p2g_path_list* out) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (!opts || !opts->output) return set_error(P2G_ERR_INVALID_ARGUMENT, "options/output is NULL");
    const uint32_t R = opts->recovery_block_count;
    const uint64_t slice = opts->slice_size;
    P2G_TRY(fused_validate(n, R, slice));
    std::vector<uint64_t> lens(n);
    uint64_t S = 0, total = 0;
    for (uint32_t f = 0; f < n; ++f) {
        P2G_TRY(check_name(inputs[f].display_name, inputs[f].name_len, inputs[f].path));
        P2G_TRY(stat_len(inputs[f].path, &lens[f]));
        if (lens[f] == 0)
            return set_error(P2G_ERR_EMPTY_FILE, "input file \"%s\" is empty; PAR2 requires non-empty files",
                             inputs[f].path);
        S += (lens[f] + slice - 1) / slice;
        total += lens[f];
    }
    P2G_TRY(check_total_blocks(S, total, slice));
    P2G_TRY(ensure_ready(c));
    if (R) emit_encode_events(cb, user, S, R, false);
    std::vector<std::unique_ptr<HostFile>> hfs(n);
    std::vector<CreateInput> ins(n);
    for (uint32_t f = 0; f < n; ++f) {
        p2g_progress_event ev = mk(P2G_EV_SCAN_STARTED);
        ev.path = inputs[f].path;
        ev.total_slices = (lens[f] + slice - 1) / slice;
        emit(cb, user, ev);
        hfs[f].reset(new HostFile());
        hfs[f]->path = inputs[f].path;
        P2G_TRY(read_file(*hfs[f], lens[f]));
        ins[f] = {hfs[f]->data, hfs[f]->length, inputs[f].display_name, inputs[f].name_len, inputs[f].path};
    }
    CreateOutput co;
    PinnedRec rec(c);
    // with a valid volume scheme, the volumes' recovery packets are written
    // while the whole files still hash (StagedVolumes)
    std::vector<uint32_t> early_vs;
    const bool stage = R && resolve_volume_sizes(opts->volume_scheme, R, early_vs) == P2G_OK;
    clear_error();
    StagedVolumes staged;
    p2g_status staged_st = P2G_OK;
    const WhileHashing write_early = [&](const CreateOutput& o, size_t clen) {
        staged_st = staged.write_recovery(opts->output, o, slice, early_vs, clen);
    };
    P2G_TRY(device_create(c, ins.data(), n, slice, R, nullptr, opts->comments, opts->comment_count, co, rec,
                          stage ? &write_early : nullptr));
    if (staged.active && (staged_st != P2G_OK || staged.crit_len != co.critical.size())) staged.discard();
    for (uint32_t f = 0; f < n; ++f) {
        p2g_progress_event ev = mk(P2G_EV_SCAN_PROGRESS);
        ev.path = inputs[f].path;
        ev.slices_done = ev.total_slices = co.sources[f].slice_count;
        emit(cb, user, ev);
        ev = mk(P2G_EV_SCAN_COMPLETED);
        ev.path = inputs[f].path;
        emit(cb, user, ev);
    }
    for (auto& sf : co.sources) free_source(sf);
    if (R) emit_encode_events(cb, user, S, R, true);
    if (R) {
        // the index is written before the scheme is resolved (src/creator.rs:237-244)
        std::vector<std::pair<const uint8_t*, size_t>> pieces = {{co.critical.data(), co.critical.size()}};
        std::vector<uint32_t> vs;
        p2g_status st = resolve_volume_sizes(opts->volume_scheme, R, vs);
        if (st != P2G_OK) {
            const std::string msg = p2g_last_error_message();
            P2G_TRY(write_atomic(opts->output, pieces));
            return set_error(st, "%s", msg.c_str());
        }
        co.vol_sizes = vs;
    }
    std::vector<std::string> written;
    if (staged.active) {
        std::vector<std::pair<const uint8_t*, size_t>> pieces = {{co.critical.data(), co.critical.size()}};
        P2G_TRY(write_atomic(opts->output, pieces));
        p2g_progress_event ev = mk(P2G_EV_INDEX_WRITTEN);
        ev.path = opts->output;
        emit(cb, user, ev);
        written.push_back(opts->output);
        P2G_TRY(staged.finish(co.critical, cb, user, written));
    } else {
        P2G_TRY(write_outputs(*opts, co, R, slice, cb, user, written));
    }
    fill_path_list(out, written);
    return P2G_OK;
}

extern "C" p2g_status p2g_create_in_memory(const p2g_create_options* opts, const p2g_buffer_input* inputs, uint32_t n,
                                           p2g_source_file* sources_out, p2g_output_set* out) {
    Context& c = ctx();
    std::lock_guard<std::recursive_mutex> lk(c.mu);
    clear_error();
    if (!opts || !out) return set_error(P2G_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint32_t R = opts->recovery_block_count;
    const uint64_t slice = opts->slice_size;
    P2G_TRY(fused_validate(n, R, slice));
    uint64_t S = 0, total = 0;
    std::vector<CreateInput> ins(n);
    for (uint32_t f = 0; f < n; ++f) {
        P2G_TRY(check_name(inputs[f].display_name, inputs[f].name_len, ""));
        if (inputs[f].length == 0) return set_error(P2G_ERR_EMPTY_FILE, "input file %u is empty; PAR2 requires non-empty files", f);
        S += (inputs[f].length + slice - 1) / slice;
        total += inputs[f].length;
        ins[f] = {inputs[f].data, inputs[f].length, inputs[f].display_name, inputs[f].name_len, nullptr};
    }
    P2G_TRY(check_total_blocks(S, total, slice));
    std::vector<uint32_t> vs;
    if (R) P2G_TRY(resolve_volume_sizes(opts->volume_scheme, R, vs));
    P2G_TRY(ensure_ready(c));
    CreateOutput co;
    PinnedRec rec(c);
    co.vol_sizes = vs;
    const std::string index = opts->output ? opts->output : "recovery.par2";
    // Volumes = critical | recovery packets | critical.  The recovery packets
    // only need the device results, so they are laid into the volume buffers
    // while the host still hashes whole files; the critical block (it holds
    // those hashes) fills both ends afterwards.
    std::vector<p2g_output_file> vols(vs.size());
    size_t crit_len = 0;
    bool vols_ok = true;
    // The volume buffers are allocated, and their pages touched, on a host
    // thread while the device works: with hundreds of MB of recovery
    // packets the first-touch page faults would otherwise fall between the
    // download and the return.
    std::vector<uint8_t*> pre(vs.size(), nullptr);
    size_t pre_clen = 0;
    std::thread prefault([&]() {
        pre_clen = critical_len_of(slice, ins.data(), n, opts->comments, opts->comment_count);
        for (size_t v = 0; v < vs.size(); ++v) {
            const size_t len = 2 * pre_clen + (size_t)vs[v] * (68 + slice);
            pre[v] = (uint8_t*)malloc(std::max<size_t>(len, 1));
            if (pre[v])
                for (size_t o = 0; o < len; o += 4096) pre[v][o] = 0;
        }
    });
    auto take_pre = [&]() {  // joins the thread; buffers not handed out are freed by the caller below
        if (prefault.joinable()) prefault.join();
    };
    auto free_vols = [&]() {
        for (auto& of : vols) {
            free(of.name);
            free(of.data);
            of = p2g_output_file{};
        }
    };
    const WhileHashing lay_out = [&](const CreateOutput& o, size_t clen) {
        crit_len = clen;
        take_pre();
        uint32_t first = 0;
        std::vector<std::vector<uint8_t>> headers(vs.size());
        std::vector<std::pair<const uint8_t*, size_t>> pieces;
        struct Copy {
            uint8_t* dst;
            const uint8_t* src;
            size_t len;
        };
        std::vector<Copy> copies;
        size_t bytes = 0;
        for (size_t v = 0; v < vs.size() && vols_ok; ++v) {
            volume_pieces_recovery(o, slice, first, vs[v], headers[v], pieces);
            size_t tot = 2 * clen;
            for (auto& p : pieces) tot += p.second;
            p2g_output_file& of = vols[v];
            of.name = dupstr(volume_filename(index, (uint16_t)first, vs[v]));
            of.length = tot;
            if (pre[v] && clen == pre_clen) {
                of.data = pre[v];  // prefaulted, the same size
                pre[v] = nullptr;
            } else {
                of.data = (uint8_t*)malloc(std::max<size_t>(tot, 1));
            }
            if (!of.name || !of.data) {
                vols_ok = false;
                break;
            }
            size_t at = clen;
            for (auto& p : pieces) {
                copies.push_back({of.data + at, p.first, p.second});
                at += p.second;
                bytes += p.second;
            }
            first += vs[v];
        }
        if (!vols_ok) return;
        // hundreds of MB for large recovery sets: copy in ~4 MB pieces on a
        // few threads (one core may still be hashing whole files)
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned nt = (unsigned)std::min<size_t>(std::min(8u, hw), std::max<size_t>(1, bytes >> 24));
        std::atomic<size_t> next{0};
        constexpr size_t kPiece = 4u << 20;
        auto worker = [&]() {
            for (size_t i = next++; i < copies.size(); i = next++) {
                const Copy& cp = copies[i];
                for (size_t off = 0; off < cp.len; off += kPiece)
                    memcpy(cp.dst + off, cp.src + off, std::min(kPiece, cp.len - off));
            }
        };
        run_on_threads(nt, worker);
    };
    const p2g_status st = device_create(c, ins.data(), n, slice, R, nullptr, opts->comments, opts->comment_count, co,
                                        rec, &lay_out);
    take_pre();
    for (uint8_t* b : pre) free(b);  // unused (a failed call, or a size that changed)
    if (st != P2G_OK || !vols_ok || co.critical.size() != crit_len) {
        free_vols();
        if (st != P2G_OK) return st;
        for (auto& sf : co.sources) free_source(sf);
        if (!vols_ok) return set_error(P2G_ERR_OOM, "out of host memory for the volume buffers");
        return set_error(P2G_ERR_CUDA, "internal: critical packet length changed after hashing");
    }
    out->count = 1 + (uint32_t)vs.size();
    out->files = (p2g_output_file*)calloc(out->count, sizeof(p2g_output_file));
    out->files[0].name = dupstr(index);
    out->files[0].length = co.critical.size();
    out->files[0].data = (uint8_t*)malloc(std::max<size_t>(co.critical.size(), 1));
    memcpy(out->files[0].data, co.critical.data(), co.critical.size());
    for (size_t v = 0; v < vs.size(); ++v) {
        p2g_output_file& of = vols[v];
        memcpy(of.data, co.critical.data(), crit_len);
        memcpy(of.data + of.length - crit_len, co.critical.data(), crit_len);
        out->files[1 + v] = of;
    }
    if (sources_out)
        for (uint32_t f = 0; f < n; ++f) sources_out[f] = co.sources[f];
    else
        for (auto& sf : co.sources) free_source(sf);
    return P2G_OK;
}
