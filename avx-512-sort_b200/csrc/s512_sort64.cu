// s512_sort64.cu -- the sort for 64-bit words that the reference's interface
// describes but does not implement: int64 keys, and int key/value pairs stored
// interleaved as int[2] (the reference's README speaks of sorting "int[2]";
// its kv interface, sort512kv.hpp:6133, takes two separate arrays).  Same
// pipeline as s512_sort.cu, through the CodecI64 / CodecKVPairs codecs.
#include "s512_pipeline.cuh"
#include "s512_stream.cuh"

#include <type_traits>

using namespace s512;

namespace s512 {

template <typename Codec, typename T>
static int sort_words(T* data, size_t n, int flags, void* stream) {
    if (n == 0) return S512_OK;
    if (!data) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    CallGuard guard(C, st);
    S512_HOST_PTR(host, data, flags);
    if constexpr (std::is_same<Codec, CodecI64>::value) {
        if (host && stream_needed(n, 8)) {  // larger than the device budget
            int rc = stream_sort<long long>(*C, data, n, st);
            if (rc) return rc;
            return finish_call(guard, st, flags, host);
        }
    }
    unsigned long long* d = (unsigned long long*)data;
    HostFeed feed;
    bool chunked = false;
    if (host) {
        d = (unsigned long long*)C->get("stage0", n * 8);
        if (!d) return S512_ERR_ALLOC;
        void* hp[1] = {data};
        void* dp[1] = {d};
        S512_TRY_RC(copy_in<uint64_t>(*C, 1, hp, dp, 8, n, host_pinned, st, &feed, &chunked));
    }
    int rc = sort_device<uint64_t>(*C, Codec{d, d}, Codec{d, d}, n, st, use_learned(flags), chunked ? &feed : nullptr);
    if (rc) return rc;
    if (host) S512_CUDA_TRY(cudaMemcpyAsync(data, d, n * 8, cudaMemcpyDeviceToHost, st));
    return finish_call(guard, st, flags, host, host_pinned);
}

}  // namespace s512

extern "C" {

int s512_sort_i64(long long* data, size_t n, int flags, void* stream) {
    return sort_words<CodecI64>(data, n, flags, stream);
}

int s512_sort_kv_pairs_i32(int* pairs, size_t n, int flags, void* stream) {
    return sort_words<CodecKVPairs>(reinterpret_cast<long long*>(pairs), n, flags, stream);
}

}  // extern "C"
