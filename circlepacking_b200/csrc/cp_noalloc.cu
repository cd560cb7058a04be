// Box refinement that allocates no memory: cp_refine_boxes_static.
//
// Some callers cannot let a library call cudaMalloc: applications that hand all
// device memory to their own pool or caching allocator, and latency-critical
// loops where an allocation's implicit device synchronisation is not acceptable.
// For them this entry point runs the same refinement as cp_refine_boxes inside
// one fixed scratch array that is part of the library image
// (kStaticScratchBytes per device, held from the first use until the process
// exits).  The caller passes the seed boxes and receives the report.
//
// Every call on a device shares that array and leaves its contents behind;
// each call clears the parts that must start at zero.  Calls that overlap on
// the GPU (different streams or host threads at the same time) race on the
// array and must not be issued.  The first call on each device also performs
// the set-up (it resolves the array's device address and fills a
// single-placement table there with one kernel launch); make that first call
// before any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "cp_common.h"
#include "cp_engine.h"
#include "cp_worklist.cuh"

namespace {

// 32 MiB of device scratch: counters, the single-placement table, level buffers
constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr int kTableN = 1 << 16;  // the same grid as the handle's table (cp_create)
constexpr size_t kCounterBytes = 4096;
constexpr size_t kTableBytes = 2 * sizeof(double) * kTableN;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct DeviceSlot {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_static_scratch on this device
};
std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];

// Once per device, with that device current: the array's device address, and
// the single-placement table (a constant that no call overwrites).
cp_status setup(int dev, cudaStream_t st, unsigned char** base) {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceSlot& s = g_slots[dev];
    if (!s.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) return cp_record_cuda_error(e, CP_ERR_CUDA);
        unsigned char* b = (unsigned char*)p;
        double* t = (double*)(b + kCounterBytes);
        double* v = t + kTableN;
        const double h = (cpb::kLambdaMax - cpb::kLambdaMin) / (kTableN - 1);
        cp_status rc = cp_engine_launch_table(cpb::kLambdaMin, h, kTableN, t, v, st);
        if (rc != CP_OK) return rc;
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
        s.base = b;
        s.ready = true;
    }
    *base = s.base;
    return CP_OK;
}

}  // namespace

extern "C" cp_status cp_refine_boxes_static(int family, int precision, int policy, int max_depth, const double* lo,
                                            const double* hi, const uint8_t* depth, size_t n, cp_refine_report* report,
                                            void* stream) {
    if (family < 0 || family > 5 || (precision != CP_FP64 && precision != CP_FP32_PREFILTER) ||
        policy < CP_SPLIT_UNIFORM || policy > CP_SPLIT_WIDEST || !report || (n && (!lo || !hi)))
        return CP_ERR_INVALID;
    if (max_depth < 0 || max_depth > CP_STATIC_MAX_DEPTH || n > CP_STATIC_MAX_SEEDS) {
        return cp_fail(CP_ERR_CAPACITY, "cp_refine_boxes_static: at most %d seed boxes and max_depth %d (got %zu, %d)",
                       CP_STATIC_MAX_SEEDS, CP_STATIC_MAX_DEPTH, n, max_depth);
    }
    std::memset(report, 0, sizeof(*report));
    // the host mirror of the counter block below is a fixed-size local array
    const size_t words = cp_engine_counter_words();
    if (words > 128) return cp_fail(CP_ERR_INVALID, "cp_refine_boxes_static: counter block of %zu words", words);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return cp_record_cuda_error(e, CP_ERR_NO_DEVICE);
    cudaStream_t st = (cudaStream_t)stream;
    // the scratch array resolved below belongs to the current device: a stream
    // of another device would run kernels on memory it cannot address
    int stream_dev = dev;
    if ((e = cudaStreamGetDevice(st, &stream_dev)) != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    if (stream_dev != dev)
        return cp_fail(CP_ERR_INVALID, "cp_refine_boxes_static: the stream belongs to device %d, the current device is %d",
                       stream_dev, dev);
    unsigned char* base = nullptr;
    cp_status rc = setup(dev, st, &base);
    if (rc != CP_OK) return rc;

    // layout: counters | table | (max_depth + 1) level buffers of equal capacity
    unsigned long long* cnt = (unsigned long long*)base;
    const double* tab_t = (const double*)(base + kCounterBytes);
    const double* tab_v = tab_t + kTableN;
    const double tab_h = (cpb::kLambdaMax - cpb::kLambdaMin) / (kTableN - 1);
    const int D = cpb::family_dims(family);
    const int levels = max_depth + 1;
    const size_t per_box = (size_t)D * 2 * sizeof(double) + 1;
    const size_t avail = kStaticScratchBytes - kCounterBytes - kTableBytes;
    const size_t cap = ((avail / (size_t)levels) / per_box) & ~size_t(255);
    const int F = cpb::fanout(policy, D);
    if (cap < (size_t)F || n > cap) {
        return cp_fail(CP_ERR_CAPACITY, "cp_refine_boxes_static: %zu seed boxes exceed the %zu-box level capacity", n,
                       cap);
    }
    cpb::BoxList lv[CP_STATIC_MAX_DEPTH + 1];
    size_t cnt_in[CP_STATIC_MAX_DEPTH + 1];
    unsigned char* p = base + kCounterBytes + kTableBytes;
    for (int l = 0; l < levels; ++l) {
        const size_t bytes = ((cap * per_box) + 255) & ~size_t(255);
        lv[l].lo = (double*)p;
        lv[l].hi = lv[l].lo + (size_t)D * cap;
        lv[l].depth = (uint8_t*)(lv[l].hi + (size_t)D * cap);
        lv[l].cap = cap;
        lv[l].aux = nullptr;  // no lambda-independent terms in the fixed scratch
        cnt_in[l] = 0;
        p += bytes;
    }
    // the counters must start at zero; the level buffers are written before read
    if ((e = cudaMemsetAsync(cnt, 0, words * sizeof(unsigned long long), st)) != cudaSuccess)
        return cp_record_cuda_error(e, CP_ERR_CUDA);
    for (int d = 0; d < D && n; ++d) {
        if ((e = cudaMemcpyAsync(lv[0].lo + (size_t)d * cap, lo + (size_t)d * n, sizeof(double) * n,
                                 cudaMemcpyDeviceToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(lv[0].hi + (size_t)d * cap, hi + (size_t)d * n, sizeof(double) * n,
                                 cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
            return cp_record_cuda_error(e, CP_ERR_CUDA);
    }
    if (n) {
        e = depth ? cudaMemcpyAsync(lv[0].depth, depth, n, cudaMemcpyDeviceToDevice, st)
                  : cudaMemsetAsync(lv[0].depth, 0, n, st);
        if (e != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    }
    cnt_in[0] = n;
    unsigned long long h_cnt[128] = {0};
    // deepest non-empty level first, in chunks whose children fit the next level
    for (;;) {
        int l = -1;
        for (int k = levels - 1; k >= 0; --k)
            if (cnt_in[k] > 0) {
                l = k;
                break;
            }
        if (l < 0) break;
        const bool last = (l + 1 >= levels);
        size_t c = cnt_in[l];
        if (!last) c = std::min(c, (cap - cnt_in[l + 1]) / (size_t)F);
        if (c == 0) return CP_ERR_CAPACITY;
        const size_t begin = cnt_in[l] - c;
        rc = cp_engine_launch_level(family, precision, 0, lv[l], begin, c, last ? nullptr : &lv[l + 1],
                                    last ? 0ull : (unsigned long long)cnt_in[l + 1], cnt, tab_t, tab_v, kTableN,
                                    tab_h, policy, max_depth, st);
        if (rc != CP_OK) return rc;
        if ((e = cudaMemcpyAsync(h_cnt, cnt, words * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cp_record_cuda_error(e, CP_ERR_CUDA);
        if (cp_engine_overflowed(h_cnt)) return CP_ERR_CAPACITY;
        if (!last) cnt_in[l + 1] = (size_t)cp_engine_children(h_cnt);
        cnt_in[l] -= c;
        report->launches++;
    }
    cp_engine_fill_report(h_cnt, report);
    return CP_OK;
}
