// Throughput probe for the splat's roofline: the rate at which this GPU retires float4
// reductions (RED, `atomicAdd` of a float4 without a return value) at scattered rows of
// a table, the access the splat makes once per (point, remainder).  The splat is bound by
// these L2 atomics and by the latency of its probes, not by DRAM bandwidth, so its
// achieved RED rate is reported against this measured one.  Not a filtering path.
#include <cuda_runtime.h>

#include "engine.h"

namespace pgpu {
namespace {

constexpr int kProbeThreads = 256;

// Thread t adds `per_thread` float4 rows at pseudo-random rows of `rows` (a multiplicative
// walk), so the lanes of a warp hit different rows, as the splat's lanes mostly do.
__global__ void __launch_bounds__(kProbeThreads) red_probe_kernel(float4* table, uint32_t rows,
                                                                  int per_thread) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = t * 0x9E3779B1u + 0x7F4A7C15u;
    const float4 one = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    for (int k = 0; k < per_thread; ++k) {
        h = h * 0x85EBCA6Bu + 0xC2B2AE35u;
        atomicAdd(table + __umulhi(h, rows), one);
    }
}

}  // namespace
}  // namespace pgpu

using namespace pgpu;

extern "C" int pgpu_probe_red_rate(void* table, long long rows, int per_thread, int blocks,
                                   void* stream, double* reds_per_second) {
    clear_error();
    if (!table || rows < 1 || rows > 0xFFFFFFFFll || per_thread < 1 || blocks < 1 ||
        !reds_per_second)
        return fail(PGPU_ERR_ARGUMENT, "invalid probe arguments");
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    red_probe_kernel<<<blocks, kProbeThreads, 0, st>>>((float4*)table, (uint32_t)rows, per_thread);
    CUDA_TRY(cudaGetLastError());   // warm-up launch
    CUDA_TRY(cudaEventRecord(e0, st));
    red_probe_kernel<<<blocks, kProbeThreads, 0, st>>>((float4*)table, (uint32_t)rows, per_thread);
    CUDA_TRY(cudaEventRecord(e1, st));
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.0f;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *reds_per_second = (double)blocks * kProbeThreads * per_thread / (ms * 1e-3);
    return PGPU_OK;
}
