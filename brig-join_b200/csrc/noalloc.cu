// noalloc.cu - brig_join_run_noalloc: the join pipeline over a static device scratch array.
//
// Some callers cannot allocate device memory at the point where they join: host frameworks that
// own every byte of device memory through their own pool and forbid their operators to allocate
// outside it, and latency-critical callers for whom the device-wide synchronisation of
// cudaMalloc/cudaFree is not acceptable. For them this entry point runs the same kernels as
// brig_join_run, with every intermediate buffer (partitions, histograms, Bloom filter, task list,
// counters) carved out of one file-scope __device__ array instead of a handle's workspace. It calls
// no cudaMalloc, cudaFree, cudaMallocHost or other allocating routine, and needs no handle.
//
// Limits and sharing:
//   * at most BRIG_NOALLOC_MAX_TUPLES tuples per relation, and the join's layout must fit in
//     BRIG_NOALLOC_SCRATCH_BYTES; larger requests are rejected with BRIG_E_UNSUPPORTED;
//   * every GPU that loads the library holds the array until the process exits;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) and
//     sets the kernels' attributes on that device; the entry point refuses to run under stream
//     capture (BRIG_E_UNSUPPORTED): it uploads its descriptors from a stack buffer, which a
//     captured graph could not replay;
//   * a device-side consistency failure (a bounds check, a wait that gave up) writes -1 to
//     out->d_count instead of the count, since this entry point has no handle to report it through;
//   * all calls on a device share the one array and it keeps the last call's contents: the
//     pipeline clears what must start at zero (counters, queue words) and fully writes everything
//     else before reading it, but two calls whose work overlaps on the GPU race on the array, so
//     callers must order them (one stream, or events between streams).
#include <cstring>
#include <mutex>
#include "../../include/brig_join.h"
#include "engine.h"

namespace brig {
namespace {

static_assert(BRIG_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size");

// The scratch. In host code this name is only a stand-in for the symbol, not a device address;
// the address is looked up per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[BRIG_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up on the first call per device.
char* scratch_address(int dev) {
    if (dev < 0 || dev >= kMaxDevices) fail(BRIG_E_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            fail(BRIG_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<char*>(p);
    }
    return g_scratch_addr[dev];
}

}  // namespace
}  // namespace brig

extern "C" int brig_join_run_noalloc(const brig_join_config* cfg, const uint32_t* r_key, const uint32_t* r_val,
                                     int64_t n_r, const uint32_t* s_key, const uint32_t* s_val, int64_t n_s,
                                     const brig_join_output* out, void* stream) {
    using namespace brig;
    try {
        if (!cfg || !out) fail(BRIG_E_INVALID, "null argument");
        if (cfg->abi_version != BRIG_JOIN_ABI_VERSION) fail(BRIG_E_INVALID, "config ABI version mismatch");
        if (n_r < 0 || n_s < 0) fail(BRIG_E_INVALID, "negative size");
        if (n_r > BRIG_NOALLOC_MAX_TUPLES || n_s > BRIG_NOALLOC_MAX_TUPLES)
            fail(BRIG_E_UNSUPPORTED, "relation larger than BRIG_NOALLOC_MAX_TUPLES (262144 tuples): use "
                                     "brig_join_run, which allocates its workspace");
        if ((n_r > 0 && (!r_key || !r_val)) || (n_s > 0 && (!s_key || !s_val)))
            fail(BRIG_E_INVALID, "null input array");
        if (out->capacity < 0 || (out->capacity > 0 && (!out->r_val || !out->s_val)))
            fail(BRIG_E_INVALID, "bad output");
        if (!out->d_count) fail(BRIG_E_INVALID, "d_count is required: it is the only way the count comes back");
        if (cfg->device >= 0) cuda_check(cudaSetDevice(cfg->device), "cudaSetDevice");
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cuda_check(cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap), "cudaStreamIsCapturing");
        if (cap != cudaStreamCaptureStatusNone)
            fail(BRIG_E_UNSUPPORTED, "brig_join_run_noalloc cannot be captured into a CUDA graph (its descriptor "
                                     "upload reads a stack buffer); call it directly");
        int dev = 0, sms = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");

        brig_join_config c = *cfg;
        c.use_cuda_graph = 0;
        c.profile_stages = 0;
        const JoinPlan plan = plan_join(c, n_r, n_s);
        JoinOffs jo;
        Shape sh;
        layout_for(c, &plan, 1, sms, &jo, sh);
        if (sh.total > (size_t)BRIG_NOALLOC_SCRATCH_BYTES)
            fail(BRIG_E_UNSUPPORTED, "join layout (" + std::to_string(sh.total) +
                                         " bytes) exceeds BRIG_NOALLOC_SCRATCH_BYTES; lower the fan-outs "
                                         "or use brig_join_run");
        // one join: the descriptor image is one JoinDesc and five prefix arrays of two int64
        alignas(16) char meta[sizeof(JoinDesc) + 5 * 2 * sizeof(int64_t)];
        if (sh.meta_bytes > sizeof(meta)) fail(BRIG_E_INTERNAL, "descriptor image size");
        char* ws = scratch_address(dev);
        const JoinIO io{r_key, r_val, s_key, s_val, n_r, n_s, *out};
        PipelineArgs a{};
        fill_pipeline(c, &plan, &io, 1, sh, ws, meta, sms, a);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // From pageable memory the copy returns once `meta` has been staged, so the stack buffer
        // may go out of scope afterwards.
        cuda_check(cudaMemcpyAsync(ws + sh.meta, meta, sh.meta_bytes, cudaMemcpyHostToDevice, st),
                   "descriptor upload");
        cuda_check(cudaMemsetAsync(ws + sh.counters, 0, (size_t)kCntWords * 8, st), "counter reset");
        cuda_check(enqueue_pipeline(a, st), "pipeline launch");
        return BRIG_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.status;
    } catch (...) {
        set_last_error("unknown failure");
        return BRIG_E_INTERNAL;
    }
}
