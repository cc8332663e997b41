// p2g_noalloc.cu -- p2g_encode_noalloc: the Reed-Solomon encode without any
// memory allocation by the library.
//
// Who needs it: callers that own every byte of device memory themselves --
// a server or framework whose caching allocator or fixed memory pool must
// account for all device memory, a process running under a hard memory cap,
// or code on a latency-critical path where a cudaMalloc/cudaFree would
// implicitly synchronise the device and stall unrelated streams.  Such a
// caller cannot let the library call cudaMalloc behind its back, so this
// entry point uses a scratch buffer that lives in the library's own module
// instead.
//
// The scratch is the coefficient-basis matrix the encode kernel reads
// (1 KiB per input slice per group of 32 recovery rows), held in a
// file-scope __device__ array of kNoAllocBasisBytes.  Every GPU that loads
// libpar2gpu.so carries that array until the process exits.  In host code
// the array's name is only a host-side stand-in for the device symbol, so
// its device address is obtained once per device with cudaGetSymbolAddress
// and that pointer is what the kernels receive.
#include <mutex>

#include "p2g_host_util.h"
#include "p2g_internal.h"

namespace p2g {

// 8 MiB: enough for S * ceil(R/32) <= 8192, e.g. 1,027 slices with up to 224
// recovery rows, or 8,192 slices with up to 32.
constexpr size_t kNoAllocBasisBytes = 8u << 20;
constexpr uint64_t kNoAllocMaxGroups = kNoAllocBasisBytes / 1024;

static __device__ __align__(256) uint8_t g_noalloc_basis[kNoAllocBasisBytes];
static __device__ __align__(256) int g_noalloc_err[64];

namespace {
struct NoAllocDevice {
    bool ready = false;
    uint16_t* basis = nullptr;
    int* err = nullptr;
};
constexpr int kMaxDevices = 64;
NoAllocDevice g_dev[kMaxDevices];
std::mutex g_mu;

// Once per device, with that device current: upload the GF tables and look
// up the device addresses of the scratch arrays.
p2g_status noalloc_setup(int dev, NoAllocDevice** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    NoAllocDevice& d = g_dev[dev];
    if (!d.ready) {
        cudaError_t e = upload_tables_noheap();
        if (e != cudaSuccess)
            return set_error(P2G_ERR_CUDA, "CUDA error: %s (uploading GF tables)", cudaGetErrorString(e));
        void* p = nullptr;
        if ((e = cudaGetSymbolAddress(&p, g_noalloc_basis)) != cudaSuccess)
            return set_error(P2G_ERR_CUDA, "CUDA error: %s (scratch address)", cudaGetErrorString(e));
        d.basis = static_cast<uint16_t*>(p);
        if ((e = cudaGetSymbolAddress(&p, g_noalloc_err)) != cudaSuccess)
            return set_error(P2G_ERR_CUDA, "CUDA error: %s (error-flag address)", cudaGetErrorString(e));
        d.err = static_cast<int*>(p);
        d.ready = true;
    }
    *out = &d;
    return P2G_OK;
}
}  // namespace

}  // namespace p2g

using namespace p2g;

extern "C" p2g_status p2g_encode_noalloc(const p2g_encode_job* job) {
    clear_error();
    if (!job) return set_error(P2G_ERR_INVALID_ARGUMENT, "job is NULL");
    const p2g_encode_job& jb = *job;
    if (!(jb.flags & P2G_DEVICE_POINTERS))
        return set_error(P2G_ERR_INVALID_ARGUMENT,
                         "p2g_encode_noalloc takes device pointers only (host buffers would need staging memory)");
    if (jb.slice_size == 0 || jb.slice_size % 4)
        return set_error(P2G_ERR_INVALID_SLICE_SIZE, "invalid slice size %llu: must be > 0 and a multiple of 4",
                         (unsigned long long)jb.slice_size);
    if (jb.input_count > P2G_MAX_INPUT_BLOCKS)
        return set_error(P2G_ERR_INVALID_ARGUMENT, "input_count %u exceeds 32768", jb.input_count);
    if ((uint64_t)jb.first_exponent + jb.recovery_count > 65536ull)
        return set_error(P2G_ERR_TOO_MANY_RECOVERY_BLOCKS, "recovery exponents exceed 65535");
    if (((uintptr_t)jb.src | (uintptr_t)jb.recovery) % 16 || jb.src_stride % 16 || jb.recovery_stride % 16 ||
        jb.src_stride < jb.slice_size || jb.recovery_stride < ((jb.slice_size + 15) & ~15ull))
        return set_error(P2G_ERR_INVALID_ARGUMENT,
                         "needs 16-byte aligned pointers, strides that are multiples of 16, src_stride >= slice_size "
                         "and recovery_stride >= slice_size rounded up to 16");
    const uint32_t S = jb.input_count, R = jb.recovery_count;
    const uint32_t RG = (R + kRowsPerGroup - 1) / kRowsPerGroup;
    if ((uint64_t)S * RG > kNoAllocMaxGroups)
        return set_error(P2G_ERR_INVALID_ARGUMENT,
                         "p2g_encode_noalloc: %u input slices x %u row groups of 32 needs %llu KiB of scratch, "
                         "more than its fixed %llu KiB (input_count * ceil(recovery_count/32) must be <= %llu); "
                         "use p2g_encode",
                         S, RG, (unsigned long long)S * RG, (unsigned long long)(kNoAllocBasisBytes >> 10),
                         (unsigned long long)kNoAllocMaxGroups);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return set_error(P2G_ERR_CUDA, "no usable current CUDA device");
    NoAllocDevice* d = nullptr;
    p2g_status st = noalloc_setup(dev, &d);
    if (st != P2G_OK) return st;
    if (!R) return P2G_OK;
    cudaStream_t s = (cudaStream_t)jb.stream;
    if (!S) {
        e = cudaMemset2DAsync(jb.recovery, jb.recovery_stride, 0, jb.slice_size, R, s);
        return e == cudaSuccess ? P2G_OK : set_error(P2G_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(e));
    }
    // The scratch keeps the previous call's contents: the error flag must start at zero;
    // the basis matrix is fully rewritten by launch_basis before the encode reads it.
    if ((e = cudaMemsetAsync(d->err, 0, sizeof(int), s)) != cudaSuccess ||
        (e = launch_basis(d->basis, S, RG, R, jb.first_exponent, s)) != cudaSuccess ||
        (e = launch_encode_noheap(jb.src, jb.src_stride, S, d->basis, RG, R, jb.slice_size, jb.recovery,
                                  jb.recovery_stride, d->err, s)) != cudaSuccess)
        return set_error(P2G_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(e));
    if (jb.flags & P2G_ENCODE_WAIT) {
        // read the flag into a local: a pageable copy after the stream's work
        int flag = 0;
        if ((e = cudaMemcpyAsync(&flag, d->err, sizeof flag, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return set_error(P2G_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(e));
        if (flag)
            return set_error(P2G_ERR_TIMEOUT, "a bounded device wait gave up; the recovery rows are not valid");
    }
    return P2G_OK;
}
