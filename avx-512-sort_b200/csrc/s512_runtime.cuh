// s512_runtime.cuh -- host-side runtime shared by the C-ABI translation units:
// per-device context, grow-only scratch pool, persistent-grid sizing, error
// strings, statistics and the pointer-kind probe.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "sort512cuda.h"

namespace s512 {

// ---------------------------------------------------------------------------
// errors
void set_error(const char* fmt, ...);
#define S512_CUDA_TRY(expr)                                                            \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            ::s512::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_),  \
                              __FILE__, __LINE__);                                     \
            return e_ == cudaErrorMemoryAllocation ? S512_ERR_ALLOC : S512_ERR_CUDA;   \
        }                                                                              \
    } while (0)
#define S512_LAUNCH_CHECK() S512_CUDA_TRY(cudaGetLastError())
// return a non-zero status of a library routine
#define S512_TRY_RC(expr)          \
    do {                           \
        const int rc_ = (expr);    \
        if (rc_) return rc_;       \
    } while (0)

// ---------------------------------------------------------------------------
// configuration + statistics
s512_config& config();
s512_stats& thread_stats();

// Records CUDA events around phases when statistics are enabled.
class PhaseTimer {
  public:
    PhaseTimer(cudaStream_t st, bool on) : st_(st), on_(on) {}
    ~PhaseTimer();
    // marks the current position in the stream; returns an index
    int mark();
    // elapsed ms between two marks (synchronises on the later one)
    double ms(int a, int b);
    bool on() const { return on_; }

  private:
    cudaStream_t st_;
    bool on_;
    std::vector<cudaEvent_t> ev_;
};

// ---------------------------------------------------------------------------
// per-device state and per-stream scratch pools

// Kernel attributes of one device (shared by every stream's pool).
struct DevShared {
    int dev = -1;
    int sms = 0;
    size_t smem_optin = 0;
    std::mutex mu;
    std::map<const void*, int> occ;  // kernel -> resident blocks per SM
    std::map<const void*, size_t> smem_set;
};

// The scratch pool of the calls made on one stream of one device.  Calls on
// one stream are ordered by the stream, so a pool's buffers need no other
// ordering; calls on different streams use different pools and may overlap
// on the device (a host-pointer sort on one stream copies its result back
// while the next one, on another stream, copies its input in).
struct DevCtx {
    DevShared* sh = nullptr;
    int dev = -1;
    int sms = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;                   // one call at a time on this pool
    std::map<std::string, std::pair<void*, size_t>> bufs;
    void* pinned = nullptr;          // small pinned host buffer for read-backs
    size_t pinned_bytes = 0;
    void* stage[2] = {nullptr, nullptr};  // streamed sorts: page-locked staging arrays (grow-only)
    size_t stage_bytes[2] = {0, 0};
    cudaStream_t copy_stream = nullptr;  // host-pointer sorts: input copies beside the sort
    std::vector<cudaEvent_t> events;     // host-pointer sorts: chunk arrivals (+1: call start)

    // grow-only named scratch buffer
    void* get(const char* name, size_t bytes);
    void* host_pinned(size_t bytes);
    // page-locked staging array k (0 or 1) of at least `bytes`, kept for the
    // next call like the device scratch (page-locking is slow)
    void* stage_pinned(int k, size_t bytes);
    void release_all();
    // blocks for a persistent launch: SMs x resident blocks per SM
    int persistent_grid(const void* fn, int threads, size_t smem);
    // raise the dynamic shared memory limit of a kernel once
    cudaError_t prepare(const void* fn, size_t smem);
    // the copy stream and at least n events (created on first use)
    cudaError_t copy_resources(size_t n);
};

// The pool of stream `st` on the current device (created on first use).
DevCtx* current_ctx(int* status, cudaStream_t st);

// Serialises the library calls that use one pool (host-side state).
class CallGuard {
  public:
    CallGuard(DevCtx* c, cudaStream_t st);
    ~CallGuard();
    void finish() {}  // (calls on one pool are ordered by its stream)

  private:
    std::unique_lock<std::mutex> lk_;
};

// pointer kind: 1 pageable host memory, 3 page-locked host memory the device
// can address (cudaHostAlloc / cudaHostRegister), 2 device (or managed), 0
// memory of a device other than the current one (an error: the kernels run
// on the current device)
enum { PTR_OTHER_DEVICE = 0, PTR_PAGEABLE = 1, PTR_DEVICE_MEM = 2, PTR_PINNED = 3 };
int pointer_kind(const void* p, int flags);
// the device address of page-locked host memory (nullptr if it has none)
const void* mapped_host_address(const void* p);

// `var` = whether p is host memory and `var##_pinned` whether that host
// memory is page-locked; returns S512_ERR_ARG from the enclosing function
// when p belongs to another device
#define S512_HOST_PTR(var, p, flags)                                    \
    const int var##_kind_ = ::s512::pointer_kind((p), (flags));         \
    if (var##_kind_ == ::s512::PTR_OTHER_DEVICE) return S512_ERR_ARG;   \
    const bool var = var##_kind_ != ::s512::PTR_DEVICE_MEM;             \
    const bool var##_pinned = var##_kind_ == ::s512::PTR_PINNED;        \
    (void)var##_pinned

template <typename F>
inline cudaError_t launch_persistent(DevCtx& C, F fn, int threads, size_t smem, cudaStream_t st, int max_blocks,
                                     int* grid_out) {
    cudaError_t e = C.prepare((const void*)fn, smem);
    if (e != cudaSuccess) return e;
    int g = C.persistent_grid((const void*)fn, threads, smem);
    if (max_blocks > 0 && g > max_blocks) g = max_blocks;
    if (g < 1) g = 1;
    *grid_out = g;
    return cudaSuccess;
}

}  // namespace s512
