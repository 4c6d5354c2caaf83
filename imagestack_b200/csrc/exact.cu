// FP64 brute-force Gauss transform at sampled query points — the error oracle.
//
// out[i][c] = sum_j exp(-|q_i - p_j|^2 / 2) v_j[c] over every source point j, positions
// already divided by their sigmas: the kernel of GaussTransform::apply's EXACT method
// (src/GaussTransform.cpp:135-162), evaluated with an exact double-precision exponential
// instead of that method's 4096-entry table.  It states how far a lattice result is from
// the Gauss transform it approximates; it is not on the filtering path.
#include <cuda_runtime.h>

#include "engine.h"

namespace pgpu {
namespace {

constexpr int kExactThreads = 256;
constexpr int kExactMaxVd = 8;

// One block per query; its threads stride over the sources, then reduce in shared memory.
template <int D>
__global__ void __launch_bounds__(kExactThreads) exact_gt_kernel(int vd, const float* __restrict__ q, int n,
                                                                  const float* __restrict__ p,
                                                                  const float* __restrict__ v,
                                                                  double* __restrict__ out) {
    __shared__ double red[kExactThreads][kExactMaxVd];
    const int i = blockIdx.x;
    double qi[D];
#pragma unroll
    for (int c = 0; c < D; ++c) qi[c] = (double)__ldg(q + (size_t)i * D + c);
    double acc[kExactMaxVd];
#pragma unroll
    for (int c = 0; c < kExactMaxVd; ++c) acc[c] = 0.0;
    for (int j = threadIdx.x; j < n; j += kExactThreads) {
        double dist = 0.0;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double t = qi[c] - (double)__ldg(p + (size_t)j * D + c);
            dist += t * t;
        }
        // exp(-745) is the last non-zero double: farther sources add exactly nothing
        if (dist >= 1490.0) continue;
        const double w = exp(-0.5 * dist);
#pragma unroll
        for (int c = 0; c < kExactMaxVd; ++c)
            if (c < vd) acc[c] += w * (double)__ldg(v + (size_t)j * vd + c);
    }
#pragma unroll
    for (int c = 0; c < kExactMaxVd; ++c) red[threadIdx.x][c] = acc[c];
    __syncthreads();
    for (int s = kExactThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int c = 0; c < kExactMaxVd; ++c) red[threadIdx.x][c] += red[threadIdx.x + s][c];
        }
        __syncthreads();
    }
    if (threadIdx.x < vd) out[(size_t)i * vd + threadIdx.x] = red[0][threadIdx.x];
}

template <int D>
void launch_exact(int vd, int nq, const float* q, int n, const float* p, const float* v, double* out,
                  cudaStream_t st) {
    exact_gt_kernel<D><<<nq, kExactThreads, 0, st>>>(vd, q, n, p, v, out);
}

}  // namespace
}  // namespace pgpu

using namespace pgpu;

extern "C" int pgpu_exact_gauss_transform_f64(int d, int vd, int nq, const float* q, int n,
                                              const float* p, const float* v, double* out,
                                              void* stream) {
    clear_error();
    if (d < 1 || d > kMaxD || vd < 1 || vd > kExactMaxVd || nq < 0 || n < 0 ||
        (nq > 0 && (!q || !out)) || (n > 0 && (!p || !v)))
        return fail(PGPU_ERR_ARGUMENT, "invalid exact Gauss transform arguments");
    if (nq == 0) return PGPU_OK;
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(PGPU_ERR_NO_DEVICE, "no CUDA device (this library has no CPU path)");
    }
    cudaStream_t st = (cudaStream_t)stream;
    switch (d) {
#define PGPU_EXACT_CASE(k) \
    case k: launch_exact<k>(vd, nq, q, n, p, v, out, st); break;
        PGPU_EXACT_CASE(1) PGPU_EXACT_CASE(2) PGPU_EXACT_CASE(3) PGPU_EXACT_CASE(4)
        PGPU_EXACT_CASE(5) PGPU_EXACT_CASE(6) PGPU_EXACT_CASE(7) PGPU_EXACT_CASE(8)
        PGPU_EXACT_CASE(9) PGPU_EXACT_CASE(10) PGPU_EXACT_CASE(11) PGPU_EXACT_CASE(12)
        PGPU_EXACT_CASE(13) PGPU_EXACT_CASE(14) PGPU_EXACT_CASE(15) PGPU_EXACT_CASE(16)
#undef PGPU_EXACT_CASE
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(st));
    return PGPU_OK;
}
