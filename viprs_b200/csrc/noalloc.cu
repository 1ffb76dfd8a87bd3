// noalloc.cu -- viprs_reduce_noalloc: ReduceOp (PipelineBuilder::reduce) with
// no device allocation at all.
//
// Who needs it: a caller whose device memory is owned by someone else cannot
// call cudaMalloc (or cudaMallocAsync) for the library.  Examples are a host
// framework whose caching allocator has reserved the GPU's memory and hands
// the library only the input and output buffers, a plugin run inside another
// program's processing callback where allocating is not allowed, and
// latency-bound loops where cudaMalloc/cudaFree would synchronise the device.
// viprs_reduce allocates its coefficient and position tables (and, when the
// fused tile does not fit in shared memory, an intermediate plane) for every
// call; this variant puts them in one file-scope device array instead.
//
// The array (kScratchBytes = VIPRS_NOALLOC_SCRATCH_BYTES, 4 MiB) exists on
// every GPU that loads this library, for as long as the process runs.  Its
// device address is looked up once per device, on the first call made with
// that device current (cudaGetSymbolAddress); that first call may load this
// library's device code on the device.  Every call shares the array and it
// keeps the last call's contents:
// calls whose GPU work overlaps (different streams, or different host threads
// on one device, without ordering between them) race on it.  Nothing in it
// needs to start at zero: each call's host-to-device copy rewrites the tables
// before its kernel runs, and an intermediate plane is fully written by the
// first stage before the second reads it.
#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <mutex>

#include "chain.hpp"
#include "viprs_b200.h"

namespace {

constexpr size_t kScratchBytes = VIPRS_NOALLOC_SCRATCH_BYTES;
static_assert(kScratchBytes % 256 == 0, "scratch size must keep 256-byte alignment");

// The scratch.  In host code this name is only a host-side stand-in for the
// device variable: a kernel must be given the address from
// cudaGetSymbolAddress, never this symbol.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<uint8_t*> g_scratch_addr[kMaxDevices];
std::mutex g_setup_mutex;

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Device address of the scratch on the current device (set-up on first use).
int scratch_on_current_device(uint8_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return viprs::cuda_status(e);
    if (dev < 0 || dev >= kMaxDevices) return VIPRS_ERR_INVALID_ARGUMENT;
    uint8_t* p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        p = g_scratch_addr[dev].load(std::memory_order_relaxed);
        if (!p) {
            e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
            if (e != cudaSuccess) return viprs::cuda_status(e);
            g_scratch_addr[dev].store(p, std::memory_order_release);
        }
    }
    *out = p;
    return VIPRS_OK;
}

}  // namespace

extern "C" int32_t viprs_reduce_noalloc(const viprs_image* in, const viprs_image* out, double hfactor,
                                        double vfactor, int32_t kernel, void* stream) {
    using namespace viprs;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    PlanNode n;
    n.kind = NodeKind::Reduce;
    n.factor = hfactor;
    n.vfactor = vfactor;
    n.kernel = Kernel(kernel);
    viprs_plan plan;  // host-side tables and stage list only
    int st = plan_single_node(in, out, n, &plan);
    if (st) return st;
    const size_t tables = align256(plan.host_tables.size());
    if (tables > kScratchBytes || plan.work_bytes > kScratchBytes - tables) return VIPRS_ERR_SCRATCH_LIMIT;
    uint8_t* scratch = nullptr;
    st = scratch_on_current_device(&scratch);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The tables come from pageable host memory (the plan's vector, freed when
    // this call returns): the runtime stages a pageable host-to-device copy
    // before cudaMemcpyAsync returns, so the vector may go away afterwards.
    if (!plan.host_tables.empty()) {
        const cudaError_t e =
            cudaMemcpyAsync(scratch, plan.host_tables.data(), plan.host_tables.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    plan.d_tables = scratch;
    plan.d_work = plan.work_bytes ? scratch + tables : nullptr;
    st = execute_plan(&plan, in->data, out->data, s);
    plan.d_tables = nullptr;
    plan.d_work = nullptr;
    return st;
}
