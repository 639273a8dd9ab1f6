// s512_noalloc.cu -- Partition512 for callers that cannot allocate memory.
//
// Some callers may not call cudaMalloc (or anything that allocates) at the
// moment they need a partition: code that runs while the device's memory is
// fully owned by another allocator (a framework's caching allocator that has
// reserved everything), real-time or embedded hosts that reserve all memory at
// start-up and forbid later allocations, and code paths where an allocation
// would synchronise the device or fail unpredictably under memory pressure.
// s512_partition_i32_noalloc serves them: it runs the same two-way partition
// kernel as s512_partition_i32, but its scratch lives in a fixed, file-scope
// device array that every GPU loading this library holds until the process
// exits.  The caller passes the data and receives the boundary as before.
//
// Limits and rules:
//   * at most S512_NOALLOC_MAX_ELEMS (2^20) elements per call; larger ranges
//     are rejected with S512_ERR_ARG and a message;
//   * the array is shared by every call on a device and keeps the last call's
//     contents; this file clears what must start at zero on every call, and
//     calls whose work overlaps on the GPU (different streams, or threads that
//     do not wait for each other) race on it;
//   * the first call on a device does the set-up: with that device current it
//     looks up the array's device address (cudaGetSymbolAddress) and the
//     kernel's occupancy.  CUDA loads modules lazily by default
//     (CUDA_MODULE_LOADING=LAZY), so that first call is also when the driver
//     loads this file's module and reserves the array's memory on the device.
//     Make it at start-up, before another allocator takes the device's memory
//     and before any stream capture; a call with an empty range (right < left)
//     does only this set-up;
//   * `data` must be memory of the current device (or managed memory);
//   * the partitioned range is copied back over the caller's data only when
//     the kernel reports no error, so a failed call leaves the data as it was.
#include <mutex>

#include "s512_partition2.cuh"
#include "s512_runtime.cuh"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_IPT = 16;
constexpr int NA_TILE = NA_THREADS * NA_IPT;
constexpr size_t NA_MAX = S512_NOALLOC_MAX_ELEMS;
constexpr size_t NA_TILES = (NA_MAX + NA_TILE - 1) / NA_TILE;
// [keys: NA_MAX ints][status: NA_TILES x 2 words][control block]
constexpr size_t NA_KEYS_BYTES = NA_MAX * sizeof(int);
constexpr size_t NA_STATUS_OFF = NA_KEYS_BYTES;
// (one spare pair of status words past the last tile: the failure-injection
// test waits on it, and nothing ever writes it)
constexpr size_t NA_STATUS_BYTES = (NA_TILES + 1) * 2 * sizeof(unsigned long long);
constexpr size_t NA_CTL_OFF = NA_STATUS_OFF + NA_STATUS_BYTES;
constexpr size_t NA_BYTES = NA_CTL_OFF + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mu;
unsigned char* g_na_ptr[NA_MAX_DEVICES] = {};
int g_na_grid[NA_MAX_DEVICES] = {};

// Device address of the scratch array and the grid size for this device,
// looked up once per device with that device current.
int noalloc_setup(int dev, unsigned char** ptr, int* grid) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            s512::set_error("cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
            return S512_ERR_CUDA;
        }
        int sms = 0, per_sm = 0;
        auto fn = s512::partition2_kernel<int, false, NA_THREADS, NA_IPT>;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NA_THREADS, 0) != cudaSuccess) {
            cudaGetLastError();
            s512::set_error("device query for the no-alloc partition failed");
            return S512_ERR_CUDA;
        }
        g_na_grid[dev] = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
        g_na_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *ptr = g_na_ptr[dev];
    *grid = g_na_grid[dev];
    return S512_OK;
}

#define NA_TRY(expr)                                                                                 \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            s512::set_error("%s failed: %s", #expr, cudaGetErrorString(e_));                         \
            return S512_ERR_CUDA;                                                                    \
        }                                                                                            \
    } while (0)

}  // namespace

extern "C" {

int s512_partition_i32_noalloc(int* data, size_t left, size_t right, int pivot, size_t* boundary, void* stream) {
    if (!boundary) return S512_ERR_ARG;
    int dev = 0;
    NA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) return S512_ERR_UNSUPPORTED;
    unsigned char* base = nullptr;
    int grid = 0;
    int rc = noalloc_setup(dev, &base, &grid);
    if (rc) return rc;
    if (right < left) {  // empty range: the set-up above is all there is to do
        *boundary = left;
        return S512_OK;
    }
    if (!data) return S512_ERR_ARG;
    const size_t n = right - left + 1;
    if (n > NA_MAX) {
        s512::set_error("s512_partition_i32_noalloc: %zu elements exceed the fixed scratch of %zu elements", n,
                        NA_MAX);
        return S512_ERR_ARG;
    }
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, data) != cudaSuccess ||
        (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        s512::set_error("s512_partition_i32_noalloc: data must be device memory");
        return S512_ERR_ARG;
    }
    if (at.type == cudaMemoryTypeDevice && at.device != dev) {
        s512::set_error("s512_partition_i32_noalloc: data is memory of device %d, the current device is %d",
                        at.device, dev);
        return S512_ERR_ARG;
    }

    cudaStream_t st = (cudaStream_t)stream;
    int* keys_out = reinterpret_cast<int*>(base);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(base + NA_STATUS_OFF);
    s512::Part2Ctl* ctl = reinterpret_cast<s512::Part2Ctl*>(base + NA_CTL_OFF);
    const uint32_t ntiles = (uint32_t)((n + NA_TILE - 1) / NA_TILE);
    // the look-back status words and the control block must start at zero
    NA_TRY(cudaMemsetAsync(status, 0, (size_t)(ntiles + 1) * 2 * sizeof(unsigned long long), st));
    NA_TRY(cudaMemsetAsync(ctl, 0, sizeof(s512::Part2Ctl), st));
    if (grid > (int)ntiles) grid = (int)ntiles;
    s512::partition2_kernel<int, false, NA_THREADS, NA_IPT>
        <<<grid, NA_THREADS, 0, st>>>(data + left, nullptr, keys_out, nullptr, (uint64_t)n, pivot, status, ctl,
                                      ntiles, (s512::config().fault_inject & S512_FAULT_TIMEOUT) ? ntiles
                                                                                                  : 0xFFFFFFFFu);
    NA_TRY(cudaGetLastError());
    s512::Part2Ctl h;
    NA_TRY(cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
    if (h.err) {
        // tiles that gave up wrote nothing: the scratch holds stale keys, so
        // the caller's range is left untouched
        s512::set_error("s512_partition_i32_noalloc: look-back wait timed out");
        return S512_ERR_TIMEOUT;
    }
    NA_TRY(cudaMemcpyAsync(data + left, keys_out, n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    NA_TRY(cudaStreamSynchronize(st));
    *boundary = left + (size_t)h.total_low;
    return S512_OK;
}

}  // extern "C"
