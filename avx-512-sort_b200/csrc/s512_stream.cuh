// s512_stream.cuh -- host arrays larger than the device budget: an external
// sort streamed through the device in two passes over PCIe.
//
// The reference sorts host memory of any size in place (Sort512::Sort on a
// host array; its benchmark goes to 2^30 keys, sort512perf.cpp:374; and
// Sort512kv::Sort on two host arrays, sort512kv.hpp:6133).  A host array (or
// key/value pair of arrays) whose sort would not fit the device budget (s512_config.device_budget,
// about six times the data for the array plus the level buffers) is sorted
// here as:
//   1. runs: consecutive pieces of m keys are copied in, sorted on the device
//      and copied out to a pinned staging array, three pieces in flight;
//   2. merge by exact rank: output piece j holds ranks [j*m, (j+1)*m).  For
//      each boundary rank the host finds the boundary key by bisection over
//      the encoded key range (counting keys <= a value with one binary search
//      per run) and splits ties between runs in run order, which gives every
//      run's cut exactly; piece j is then the runs' slices between two cuts,
//      gathered to the device, sorted there and copied to its final place in
//      the caller's array, again three pieces in flight.
// Every piece holds at most m keys whatever the data (ties included), so the
// device budget holds.  Keys cross PCIe twice each way.
#pragma once

#include <cstring>
#include <vector>

#include "s512_pipeline.cuh"

namespace s512 {

// Host-side order-preserving encodings, the same transforms as the device
// codecs (s512_common.cuh).
inline uint64_t host_key(int x) { return (uint32_t)x ^ 0x80000000u; }
inline uint64_t host_key(long long x) { return (uint64_t)x ^ 0x8000000000000000ull; }
inline uint64_t host_key(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

// How a streamed sort sees the caller's data: NARR host arrays of ESZ-byte
// elements, the encoded key of element i, and the device codec of a piece.
template <typename T> struct StreamTypes;
template <> struct StreamTypes<int> {
    using K = uint32_t;
    static constexpr int NARR = 1;
    static constexpr size_t ESZ = 4;
    static CodecI32 codec(void* const* d) { return CodecI32{(const int*)d[0], (int*)d[0]}; }
    static uint64_t key(void* const* h, size_t i) { return host_key(static_cast<const int*>(h[0])[i]); }
};
template <> struct StreamTypes<double> {
    using K = uint64_t;
    static constexpr int NARR = 1;
    static constexpr size_t ESZ = 8;
    static CodecF64 codec(void* const* d) {
        return CodecF64{(const unsigned long long*)d[0], (unsigned long long*)d[0]};
    }
    static uint64_t key(void* const* h, size_t i) { return host_key(static_cast<const double*>(h[0])[i]); }
};
template <> struct StreamTypes<long long> {
    using K = uint64_t;
    static constexpr int NARR = 1;
    static constexpr size_t ESZ = 8;
    static CodecI64 codec(void* const* d) {
        return CodecI64{(const unsigned long long*)d[0], (unsigned long long*)d[0]};
    }
    static uint64_t key(void* const* h, size_t i) { return host_key(static_cast<const long long*>(h[0])[i]); }
};
// int keys + int values in two arrays, ordered by (key, value) like the device codec
struct StreamKV {
    using K = uint64_t;
    static constexpr int NARR = 2;
    static constexpr size_t ESZ = 4;
    static CodecKV codec(void* const* d) {
        return CodecKV{(const int*)d[0], (const int*)d[1], (int*)d[0], (int*)d[1]};
    }
    static uint64_t key(void* const* h, size_t i) {
        return (host_key(static_cast<const int*>(h[0])[i]) << 32) | host_key(static_cast<const int*>(h[1])[i]);
    }
};

// Device bytes one host-pointer call may use.
inline size_t device_budget() {
    if (config().device_budget) return (size_t)config().device_budget;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return (size_t)1 << 34;
    }
    return free_b / 10 * 8;
}

// Keys per streamed piece: the piece, its level buffers and scratch in ~6x
// (esz: bytes of one element over all its arrays).
inline size_t stream_piece_keys(size_t esz) {
    size_t m = device_budget() / (6 * esz);
    m &= ~(size_t)4095;
    return m < 65536 ? 65536 : m;
}

// Whether a host array must be streamed.  Without a configured budget, a
// working set under 1 GiB never is (no free-memory query on small calls).
inline bool stream_needed(size_t n, size_t esz) {
    if (!config().device_budget && n * esz * 6 < ((size_t)1 << 30)) return false;
    return n > stream_piece_keys(esz);
}

// Number of elements of the sorted run [first, first+len) of the staging
// arrays whose encoded key is <= v (or < v).
template <typename ST>
static size_t count_le(void* const* stage, size_t first, size_t len, uint64_t v, bool strict) {
    size_t lo = 0, hi = len;
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        const uint64_t k = ST::key(stage, first + mid);
        if (strict ? k < v : k <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Pieces in flight: while one is sorted, the copies of the next ones in and of
// the previous ones out run in both directions of PCIe.  Each has its own
// stream and scratch pool (the caller's, then helper streams), and a piece
// buffer is reused three pieces later, after its copy out on the same stream.
constexpr int STREAM_INFLIGHT = 3;

template <typename ST>
static int stream_sort_arrays(DevCtx& C, void* const* host, size_t n, cudaStream_t st) {
    using K = typename ST::K;
    constexpr int NA = ST::NARR;
    constexpr int F = STREAM_INFLIGHT;
    const size_t esz = ST::ESZ;
    size_t m = stream_piece_keys(esz * NA) / F;
    m = m < 65536 ? 65536 : (m & ~(size_t)4095);
    const size_t nruns = (n + m - 1) / m;

    struct {
        void* p[2] = {nullptr, nullptr};
    } stage;  // the pool's page-locked staging arrays
    // streams and pools: S[0] the caller's (pool C, already held), S[1] and
    // S[2] the copy streams of the pools before them
    cudaStream_t S[F];
    DevCtx* P[F];
    S[0] = st;
    P[0] = &C;
    for (int b = 1; b < F; ++b) {
        S512_CUDA_TRY(P[b - 1]->copy_resources(1));
        S[b] = P[b - 1]->copy_stream;
        int rc = S512_OK;
        P[b] = current_ctx(&rc, S[b]);
        if (!P[b]) return rc;
    }
    static_assert(F == 3, "one guard per helper pool below");
    CallGuard g1(P[1], S[1]), g2(P[2], S[2]);
    // every return waits for all F streams first: their copies and sorts use
    // the pools' buffers and the staging arrays
    struct Drain {
        cudaStream_t* s;
        ~Drain() {
            for (int b = 0; b < F; ++b) cudaStreamSynchronize(s[b]);
        }
    } drain{S};
    void* d[F][2] = {};
    for (int k = 0; k < NA; ++k) {
        stage.p[k] = C.stage_pinned(k, n * esz);
        if (!stage.p[k]) return S512_ERR_ALLOC;
        for (int b = 0; b < F; ++b) {
            d[b][k] = P[b]->get(k ? "stream_piece1" : "stream_piece0", m * esz);
            if (!d[b][k]) return S512_ERR_ALLOC;
        }
    }
    auto at = [&](void* base, size_t i) { return static_cast<char*>(base) + i * esz; };
    auto piece_len = [&](size_t r) { return (n - r * m) < m ? (n - r * m) : m; };

    // 1. sorted runs of m elements into the staging arrays; the inputs of the
    //    next F-1 runs are queued before a run's sort (which waits on the host
    //    between its levels)
    auto run_in = [&](size_t r) -> int {
        const int b = (int)(r % F);
        for (int k = 0; k < NA; ++k)
            S512_CUDA_TRY(cudaMemcpyAsync(d[b][k], at(host[k], r * m), piece_len(r) * esz, cudaMemcpyHostToDevice,
                                          S[b]));
        return S512_OK;
    };
    for (size_t r = 0; r + 1 < F && r < nruns; ++r) S512_TRY_RC(run_in(r));
    for (size_t r = 0; r < nruns; ++r) {
        if (r + F - 1 < nruns) S512_TRY_RC(run_in(r + F - 1));
        const int b = (int)(r % F);
        int rc = sort_device<K>(*P[b], ST::codec(d[b]), ST::codec(d[b]), piece_len(r), S[b]);
        if (rc) return rc;
        for (int k = 0; k < NA; ++k)
            S512_CUDA_TRY(cudaMemcpyAsync(at(stage.p[k], r * m), d[b][k], piece_len(r) * esz,
                                          cudaMemcpyDeviceToHost, S[b]));
    }
    for (int b = 0; b < F; ++b) S512_CUDA_TRY(cudaStreamSynchronize(S[b]));

    auto run_len = [&](size_t r) { return (n - r * m) < m ? (n - r * m) : m; };

    // 2. cuts at ranks j*m: cut[j][r] = elements of run r that go before rank j*m
    std::vector<std::vector<size_t>> cut(nruns + 1, std::vector<size_t>(nruns, 0));
    for (size_t r = 0; r < nruns; ++r) cut[nruns][r] = run_len(r);
    uint64_t kmin = ~0ull, kmax = 0;
    for (size_t r = 0; r < nruns; ++r) {
        const uint64_t a = ST::key(stage.p, r * m), b = ST::key(stage.p, r * m + run_len(r) - 1);
        kmin = a < kmin ? a : kmin;
        kmax = b > kmax ? b : kmax;
    }
    for (size_t j = 1; j < nruns; ++j) {
        const size_t rank = j * m;
        // smallest encoded v with (elements <= v) >= rank
        uint64_t lo = kmin, hi = kmax;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            size_t c = 0;
            for (size_t r = 0; r < nruns; ++r) c += count_le<ST>(stage.p, r * m, run_len(r), mid, false);
            if (c >= rank) hi = mid; else lo = mid + 1;
        }
        const uint64_t v = lo;
        size_t below = 0;
        std::vector<size_t> lt(nruns), le(nruns);
        for (size_t r = 0; r < nruns; ++r) {
            lt[r] = count_le<ST>(stage.p, r * m, run_len(r), v, true);
            le[r] = count_le<ST>(stage.p, r * m, run_len(r), v, false);
            below += lt[r];
        }
        size_t need = rank - below;  // elements equal to v that go before the cut, taken in run order
        for (size_t r = 0; r < nruns; ++r) {
            const size_t take = (le[r] - lt[r]) < need ? (le[r] - lt[r]) : need;
            cut[j][r] = lt[r] + take;
            need -= take;
        }
    }

    // 3. each output piece: gather its slices, sort, copy to its final place
    //    (the gathers of the next F-1 pieces queued before a piece's sort)
    auto piece_in = [&](size_t j) -> int {
        const int b = (int)(j % F);
        size_t len = 0;
        for (size_t r = 0; r < nruns; ++r) {
            const size_t a = cut[j][r], e = cut[j + 1][r];
            if (e > a) {
                for (int k = 0; k < NA; ++k)
                    S512_CUDA_TRY(cudaMemcpyAsync(at(d[b][k], len), at(stage.p[k], r * m + a), (e - a) * esz,
                                                  cudaMemcpyHostToDevice, S[b]));
                len += e - a;
            }
        }
        if (len != run_len(j)) {
            set_error("streamed sort: piece %zu holds %zu keys, expected %zu", j, len, run_len(j));
            return S512_ERR_INTERNAL;
        }
        return S512_OK;
    };
    for (size_t j = 0; j + 1 < F && j < nruns; ++j) S512_TRY_RC(piece_in(j));
    for (size_t j = 0; j < nruns; ++j) {
        if (j + F - 1 < nruns) S512_TRY_RC(piece_in(j + F - 1));
        const int b = (int)(j % F);
        int rc = sort_device<K>(*P[b], ST::codec(d[b]), ST::codec(d[b]), run_len(j), S[b]);
        if (rc) return rc;
        for (int k = 0; k < NA; ++k)
            S512_CUDA_TRY(cudaMemcpyAsync(at(host[k], j * m), d[b][k], run_len(j) * esz, cudaMemcpyDeviceToHost,
                                          S[b]));
    }
    for (int b = 0; b < F; ++b) S512_CUDA_TRY(cudaStreamSynchronize(S[b]));
    return S512_OK;
}

template <typename T>
static int stream_sort(DevCtx& C, T* host, size_t n, cudaStream_t st) {
    void* h[1] = {host};
    return stream_sort_arrays<StreamTypes<T>>(C, h, n, st);
}

static inline int stream_sort_kv(DevCtx& C, int* keys, int* values, size_t n, cudaStream_t st) {
    void* h[2] = {keys, values};
    return stream_sort_arrays<StreamKV>(C, h, n, st);
}

}  // namespace s512
