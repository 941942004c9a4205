// gen.cu - device generator for synthetic inputs (rows computed independently, see brig_gen.cuh).
#include "brig_gen.cuh"
#include "launch.h"

namespace brig {

namespace {

__global__ void k_gen(GenParams g, uint32_t* __restrict__ rk, uint32_t* __restrict__ rv,
                      uint32_t* __restrict__ sk, uint32_t* __restrict__ sv) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.nr; i += stride) {
        if (rk) rk[i] = gen_r_key(g, i);
        if (rv) rv[i] = (uint32_t)i;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.ns; i += stride) {
        if (sk) sk[i] = gen_s_key(g, i);
        if (sv) sv[i] = (uint32_t)i;
    }
}

}  // namespace

cudaError_t enqueue_gen(uint64_t seed, int64_t n_r, int64_t n_s, double match_frac, double zipf_s,
                        uint32_t* r_key, uint32_t* r_val, uint32_t* s_key, uint32_t* s_val,
                        cudaStream_t stream) {
    const GenParams g = make_gen_params(seed, n_r, n_s, match_frac, zipf_s);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_gen<<<sms * 8, 256, 0, stream>>>(g, r_key, r_val, s_key, s_val);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace brig
