// peaks.cu - the random-read rate that bounds the level-2 Bloom probe.
//
// The level-2 Bloom pass reads one 8-byte word pair at a hashed position of its level-1
// partition's filter segments for every S key (1.57 MB of segments per partition at 640M keys, held
// in L2). Such loads each touch their own cache line, and the SM's L1/texture pipeline looks up one
// line per cycle, so that pipeline, not HBM, sets the pass's ceiling. k_gather_rate issues nothing
// but such loads, at positions drawn from a linear congruential sequence over a power-of-two table
// (also L2-resident), with eight loads in flight per thread and two 512-thread CTAs per SM as in the
// Bloom pass; the benchmark times it to report the Bloom pass as a fraction of that rate.
#include <algorithm>
#include <cstdint>
#include "../../include/brig_join.h"
#include "launch.h"

namespace brig {
namespace {

constexpr int kGatherThreads = 512;
constexpr int kGatherU = 8;  // loads in flight per thread

__global__ void __launch_bounds__(kGatherThreads, 2)
k_gather_rate(const uint2* __restrict__ table, uint32_t mask, int rounds, uint32_t* sink) {
    uint32_t h = (blockIdx.x * kGatherThreads + threadIdx.x) * 0x9E3779B9u + 0x7F4A7C15u;
    uint32_t acc = 0;
    for (int r = 0; r < rounds; ++r) {
        uint2 w[kGatherU];
#pragma unroll
        for (int u = 0; u < kGatherU; ++u) {
            h = h * 1664525u + 1013904223u;
            w[u] = __ldg(table + ((h >> 7) & mask));
        }
#pragma unroll
        for (int u = 0; u < kGatherU; ++u) acc ^= w[u].x + w[u].y;
    }
    if (acc == 0x5bd1e995u) atomicAdd(sink, 1u);  // a data dependence that keeps every load
}

}  // namespace
}  // namespace brig

extern "C" int brig_join_gather_rate(const void* table, int64_t table_bytes, int64_t loads, uint32_t* sink,
                                     int64_t* loads_issued, void* stream) {
    using namespace brig;
    if (!table || !sink || !loads_issued || loads <= 0 || table_bytes < 256 || (table_bytes & (table_bytes - 1)) ||
        table_bytes / 8 > (int64_t)UINT32_MAX + 1 || (reinterpret_cast<uintptr_t>(table) & 7))
        return BRIG_E_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BRIG_E_CUDA;
    const int64_t threads = (int64_t)sms * 2 * kGatherThreads;
    const int64_t rounds = std::max<int64_t>(1, loads / (threads * kGatherU));
    if (rounds > INT32_MAX) return BRIG_E_INVALID;
    k_gather_rate<<<sms * 2, kGatherThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const uint2*>(table), (uint32_t)(table_bytes / 8 - 1), (int)rounds, sink);
    note_launches(1);
    *loads_issued = threads * kGatherU * rounds;
    return cudaGetLastError() == cudaSuccess ? BRIG_OK : BRIG_E_CUDA;
}
