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
// per-device context

struct DevCtx {
    int dev = -1;
    int sms = 0;
    size_t smem_optin = 0;
    std::mutex mu;
    std::map<std::string, std::pair<void*, size_t>> bufs;
    std::map<const void*, int> occ;  // kernel -> resident blocks per SM
    std::map<const void*, size_t> smem_set;
    void* pinned = nullptr;          // small pinned host buffer for read-backs
    size_t pinned_bytes = 0;
    cudaEvent_t last_done = nullptr; // completion of the previous call

    // grow-only named scratch buffer
    void* get(const char* name, size_t bytes);
    void* host_pinned(size_t bytes);
    void release_all();
    // blocks for a persistent launch: SMs x resident blocks per SM
    int persistent_grid(const void* fn, int threads, size_t smem);
    // raise the dynamic shared memory limit of a kernel once
    cudaError_t prepare(const void* fn, size_t smem);
};

DevCtx* current_ctx(int* status);

// Serialises library calls on one device and orders the caller's stream after
// the previous call (the scratch pool is shared).
class CallGuard {
  public:
    CallGuard(DevCtx* c, cudaStream_t st);
    ~CallGuard();
    void finish();  // record completion on the stream

  private:
    DevCtx* c_;
    cudaStream_t st_;
    std::unique_lock<std::mutex> lk_;
};

// pointer kind: 1 host, 2 device (or managed), 0 memory of a device other
// than the current one (an error: the kernels run on the current device)
int pointer_kind(const void* p, int flags);

// `var` = whether p is host memory; returns S512_ERR_ARG from the enclosing
// function when p belongs to another device
#define S512_HOST_PTR(var, p, flags)                          \
    const int var##_kind_ = ::s512::pointer_kind((p), (flags)); \
    if (var##_kind_ == 0) return S512_ERR_ARG;                \
    const bool var = var##_kind_ == 1

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
