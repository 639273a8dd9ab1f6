// s512_learned.cu -- checking entry points of the learned splitter model: the
// root's forward/backward pass for given parameters (so its gradient can be
// compared with an independent computation) and a full fit on a given sorted
// sample with the model's losses and bucket balance.
#include "s512_pipeline.cuh"

namespace s512 {

template <typename K>
__global__ void __launch_bounds__(LR_THREADS) root_grad_kernel(const K* __restrict__ smp, uint32_t m,
                                                               const float* __restrict__ theta, float* __restrict__ out) {
    __shared__ double mom[LR_ROOT * RM_COUNT];
    __shared__ uint32_t pstart[LR_ROOT + 1];
    RootMap<K> rm;
    rm.init(smp[0], smp[m - 1]);
    root_moments<K>(smp, m, rm, pstart, mom);
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        float th[RP];
#pragma unroll
        for (int k = 0; k < RP; ++k) th[k] = theta[l * RP + k];
        double loss, g[RP];
        root_eval_warp(mom, m, th, &loss, g);
#pragma unroll
        for (int k = 0; k < RP; ++k) out[1 + l * RP + k] = (float)(g[k] * 2.0 * th[k]);
        if (l == 0) out[0] = (float)loss;
    }
}

template <typename K>
static int root_grad(const void* d_keys, uint32_t m, const float* theta, float* loss, float* grad, cudaStream_t st) {
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    CallGuard guard(C, st);
    float* buf = (float*)C->get("lr_diag", (2 * LR_ROOT + 1) * sizeof(float));
    if (!buf) return S512_ERR_ALLOC;
    S512_CUDA_TRY(cudaMemcpyAsync(buf + LR_ROOT + 1, theta, LR_ROOT * sizeof(float), cudaMemcpyHostToDevice, st));
    root_grad_kernel<K><<<1, LR_THREADS, 0, st>>>((const K*)d_keys, m, buf + LR_ROOT + 1, buf);
    S512_LAUNCH_CHECK();
    float h[LR_ROOT + 1];
    S512_CUDA_TRY(cudaMemcpyAsync(h, buf, sizeof(h), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    guard.finish();
    *loss = h[0];
    memcpy(grad, h + 1, LR_ROOT * sizeof(float));
    return S512_OK;
}

template <typename K>
__global__ void learned_hist_kernel(const K* __restrict__ smp, uint32_t m, const LearnedSet<K>* __restrict__ L,
                                    uint32_t* __restrict__ hist) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        atomicAdd(&hist[learned_bucket<K>(*L, smp[i])], 1u);
}

template <typename K>
static int fit(const void* d_keys, uint32_t m, uint64_t seg_count, uint32_t* d_hist, s512_learned_report* out,
               cudaStream_t st) {
    constexpr int KB = sizeof(K);
    if (m != sample_size(target_buckets(KB, seg_count))) {
        set_error("s512_learned_fit: a segment of %llu keys is modelled from %u sample keys, got %u",
                  (unsigned long long)seg_count, sample_size(target_buckets(KB, seg_count)), m);
        return S512_ERR_ARG;
    }
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    CallGuard guard(C, st);
    K* samples = (K*)C->get("lr_fit_samples", (size_t)SAMPLE_N * KB);
    SegDesc* seg = (SegDesc*)C->get("lr_fit_seg", sizeof(SegDesc));
    SplitSet<K>* ss = (SplitSet<K>*)C->get("lr_fit_split", sizeof(SplitSet<K>));
    LearnedSet<K>* ls = (LearnedSet<K>*)C->get("lr_fit_model", sizeof(LearnedSet<K>));
    if (!samples || !seg || !ss || !ls) return S512_ERR_ALLOC;
    SegDesc sd{0, seg_count, 0, 0, 0, 0};
    S512_CUDA_TRY(cudaMemcpyAsync(samples, d_keys, (size_t)m * KB, cudaMemcpyDeviceToDevice, st));
    S512_CUDA_TRY(cudaMemcpyAsync(seg, &sd, sizeof(sd), cudaMemcpyHostToDevice, st));
    splitter_kernel<K><<<1, NB, 0, st>>>(samples, seg, 1, ss, KB);
    S512_LAUNCH_CHECK();
    uint32_t* lfirst = (uint32_t*)C->get("lr_fit_first", (LR_LEAVES + 1) * sizeof(uint32_t));
    if (!lfirst) return S512_ERR_ALLOC;
    launch_learned_fit<K>(samples, seg, 1, ss, ls, lfirst, KB, (float)config().max_imbalance, st, 1);
    S512_LAUNCH_CHECK();
    if (d_hist) {
        S512_CUDA_TRY(cudaMemsetAsync(d_hist, 0, NB * sizeof(uint32_t), st));
        learned_hist_kernel<K><<<16, 256, 0, st>>>(samples, m, ls, d_hist);
        S512_LAUNCH_CHECK();
    }
    struct {
        float loss_init, loss_root, loss_final, max_over_mean;
        uint32_t nbuckets, nmodel, ok, balanced;
    } h;
    const LearnedSet<K>* lp = ls;
    S512_CUDA_TRY(cudaMemcpyAsync(&h.loss_init, &lp->loss_init, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaMemcpyAsync(&h.max_over_mean, &lp->max_over_mean, sizeof(float), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaMemcpyAsync(&h.nbuckets, &lp->nbuckets, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaMemcpyAsync(&h.nmodel, &lp->nmodel, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaMemcpyAsync(&h.ok, &lp->ok, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaMemcpyAsync(&h.balanced, &lp->balanced, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    guard.finish();
    out->loss_init = h.loss_init;
    out->loss_root = h.loss_root;
    out->loss_final = h.loss_final;
    out->max_over_mean = h.max_over_mean;
    out->nbuckets = h.nbuckets;
    out->nmodel = h.nmodel;
    out->ok = h.ok;
    out->balanced = h.balanced;
    return S512_OK;
}

}  // namespace s512

using namespace s512;

extern "C" {

int s512_learned_root_grad(int key_bytes, const void* d_sorted_keys, uint32_t m, const float* theta, float* loss,
                           float* grad, void* stream) {
    if (!d_sorted_keys || !theta || !loss || !grad || m < 2) return S512_ERR_ARG;
    if (key_bytes == 4) return root_grad<uint32_t>(d_sorted_keys, m, theta, loss, grad, (cudaStream_t)stream);
    if (key_bytes == 8) return root_grad<uint64_t>(d_sorted_keys, m, theta, loss, grad, (cudaStream_t)stream);
    return S512_ERR_ARG;
}

int s512_learned_fit(int key_bytes, const void* d_sorted_keys, uint32_t m, uint64_t seg_count,
                     uint32_t* d_bucket_hist, s512_learned_report* report, void* stream) {
    if (!d_sorted_keys || !report || m < 2) return S512_ERR_ARG;
    if (key_bytes == 4) return fit<uint32_t>(d_sorted_keys, m, seg_count, d_bucket_hist, report, (cudaStream_t)stream);
    if (key_bytes == 8) return fit<uint64_t>(d_sorted_keys, m, seg_count, d_bucket_hist, report, (cudaStream_t)stream);
    return S512_ERR_ARG;
}

}  // extern "C"
