// The bilateral grid on the GPU: the GRID branch of GaussTransform::apply
// (src/GaussTransform.cpp:227-290), which JointBilateral::apply picks by default for at
// most four position channels (:553-564), with the reference's DenseGrid
// (src/DenseGrid.h): a dense grid over the positions' bounding box, multilinear splatting
// into the 2^d corners of each point's cell, two [1 2 1]/4 passes per dimension (taps 5),
// and multilinear slicing.
//
//   preview  min and max of every scaled position coordinate (block reduction, then
//            order-preserving integer atomics: exact in any order)
//   splat    one thread per point; FP32 atomics into the corners (the reference adds in
//            point order, so sums agree to rounding)
//   blur     one launch per dimension, one thread per grid value: the reference's two
//            in-place passes (src/DenseGrid.h:199-236) evaluated out of place, cell by cell,
//            with their exact arithmetic, including the last cell's double-precision step
//   slice    one thread per point; the corners gathered in the reference's order
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "engine.h"

namespace pgpu {
namespace {

constexpr int kGridTaps = 5;        // GaussTransform::apply builds DenseGrid(d, vd, 5)
constexpr int kGridMaxD = 5;        // 2^d corners per point; the reference's AUTO uses d <= 4
constexpr int kGridMaxVd = 8;
constexpr int kGridThreads = 256;
constexpr long long kGridMaxCells = 1LL << 30;   // floats in the grid

struct GridArgs {
    int vd;
    float sf;                            // scaleFactor, the same in every dimension
    float minp[kGridMaxD];               // minPosition
    int sizes[kGridMaxD];
    long long stride[kGridMaxD + 1];     // stride[0] = vd
    float* grid;
};

// float <-> unsigned mapping that preserves order, for min/max by integer atomics
__device__ __forceinline__ unsigned ordered_bits(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
float unordered_float(unsigned u) {
    const unsigned b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

// DenseGrid::preview (src/DenseGrid.h:142-160): the bounding box of position * scaleFactor
template <int D>
__global__ void __launch_bounds__(kGridThreads) grid_minmax_kernel(PointSource src, uint32_t n, float sf,
                                                                   unsigned* mm) {
    __shared__ unsigned smin[D], smax[D];
    if (threadIdx.x < D) {
        smin[threadIdx.x] = 0xFFFFFFFFu;
        smax[threadIdx.x] = 0u;
    }
    __syncthreads();
    unsigned lo[D], hi[D];
#pragma unroll
    for (int c = 0; c < D; ++c) lo[c] = 0xFFFFFFFFu, hi[c] = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float p[D];
        load_position<D>(src, i, p);
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const unsigned o = ordered_bits(__fmul_rn(p[c], sf));
            lo[c] = min(lo[c], o);
            hi[c] = max(hi[c], o);
        }
    }
#pragma unroll
    for (int c = 0; c < D; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = min(lo[c], __shfl_xor_sync(0xFFFFFFFFu, lo[c], o));
            hi[c] = max(hi[c], __shfl_xor_sync(0xFFFFFFFFu, hi[c], o));
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicMin(&smin[c], lo[c]);
            atomicMax(&smax[c], hi[c]);
        }
    }
    __syncthreads();
    if (threadIdx.x < D) {
        atomicMin(&mm[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&mm[D + threadIdx.x], smax[threadIdx.x]);
    }
}

// DenseGrid::query (src/DenseGrid.h:240-285): integral cell and fractions of one point
template <int D>
__device__ __forceinline__ void grid_cell(const GridArgs& g, const float (&p)[D], int (&I)[D], float (&F)[D],
                                          float (&Fi)[D]) {
#pragma unroll
    for (int c = 0; c < D; ++c) {
        const float f = __fsub_rn(__fmul_rn(p[c], g.sf), g.minp[c]);
        I[c] = (int)(short)floorf(f);
        F[c] = __fsub_rn(f, (float)I[c]);
        Fi[c] = __fsub_rn(1.0f, F[c]);
    }
}

// The cell's base offset, and which of its upper corners lie inside the grid (bit j: the
// corners one step up along dimension j); false if the cell itself is outside.  A corner
// past the grid's last cell has weight exactly 0 (the point lies on the last plane) and is
// skipped, as DenseGrid::query's bounds checks do.
template <int D>
__device__ __forceinline__ bool grid_base(const GridArgs& g, const int (&I)[D], long long& base, unsigned& hi_ok) {
    base = 0;
    hi_ok = 0;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        ok = ok && I[j] >= 0 && I[j] < g.sizes[j];
        base += (long long)I[j] * g.stride[j];
        if (I[j] + 1 < g.sizes[j]) hi_ok |= 1u << j;
    }
    return ok;
}

// Corner `corner` of the cell (unrolled by the caller): its weight in the reference's
// product order and its offset from the cell's base.
template <int D>
__device__ __forceinline__ float grid_corner_weight(const GridArgs& g, const float (&F)[D], const float (&Fi)[D],
                                                    int corner, long long base, long long& off) {
    float w = 1.0f;
    off = base;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        const bool up = (corner >> j) & 1;
        w = __fmul_rn(w, up ? F[j] : Fi[j]);
        if (up) off += g.stride[j];
    }
    return w;
}

// Blocks of the splat and slice: tiles of (bw * kp) x (kGridThreads/bw) pixels of one frame
// (bw = 32 for images, kGridThreads for point lists of one row; kp consecutive pixels of a
// row per thread), so a thread finds its pixels without dividing.
struct PixelTiles {
    unsigned bw;
    dim3 grid;
};
PixelTiles pixel_tiles(const PointSource& s, unsigned kp) {
    PixelTiles t;
    t.bw = s.height == 1 ? (unsigned)kGridThreads : 32u;
    const unsigned bh = kGridThreads / t.bw, w = t.bw * kp;
    t.grid = dim3(((unsigned)s.width + w - 1) / w, ((unsigned)s.height + bh - 1) / bh, (unsigned)s.frames);
    return t;
}

// the splat's atomic of one corner: VD values of a cell are 8- or 16-byte aligned when VD is
// 2 or 4, so one vector atomic adds them; otherwise one float atomic per value
template <int VD>
__device__ __forceinline__ void grid_add(const GridArgs& g, long long off, const float* c) {
    if constexpr (VD == 2) {
        atomicAdd(reinterpret_cast<float2*>(g.grid + off), make_float2(c[0], c[1]));
    } else if constexpr (VD == 4) {
        atomicAdd(reinterpret_cast<float4*>(g.grid + off), make_float4(c[0], c[1], c[2], c[3]));
    } else {
#pragma unroll
        for (int k = 0; k < kGridMaxVd; ++k)
            if (k < g.vd) atomicAdd(g.grid + off + k, c[k]);
    }
}

// KP consecutive pixels of a row per thread.  With KP > 1 (small grids: the 2^D corners x
// VD values fit in registers) a run of pixels that fall into the same cell is summed in
// registers first and sent as one set of corner atomics: neighbouring pixels share cells,
// and the splat is bound by the atomics' rate (4K grey d=3: 66 M float2 atomics).  The sums
// differ from the reference's point-by-point additions only in rounding order.
template <int D, int VD, int KP>
__global__ void __launch_bounds__(kGridThreads) grid_splat_kernel(PointSource src, unsigned bw, GridArgs g) {
    constexpr int NC = 1 << D;
    constexpr int NV = VD > 0 ? VD : kGridMaxVd;
    const uint32_t x0 = (blockIdx.x * bw + threadIdx.x % bw) * KP;
    const uint32_t y = blockIdx.y * (kGridThreads / bw) + threadIdx.x / bw;
    if (x0 >= (uint32_t)src.width || y >= (uint32_t)src.height) return;
    float acc[KP > 1 ? NC : 1][NV];
    long long run_base = -1;
    unsigned run_hi = 0;
    auto flush = [&]() {
        if (run_base < 0) return;
#pragma unroll
        for (int corner = 0; corner < NC; ++corner) {
            if (corner & ~run_hi) continue;
            long long off = run_base;
#pragma unroll
            for (int j = 0; j < D; ++j)
                if ((corner >> j) & 1) off += g.stride[j];
            grid_add<VD>(g, off, acc[KP > 1 ? corner : 0]);
        }
    };
#pragma unroll
    for (int kp = 0; kp < KP; ++kp) {
        const uint32_t x = x0 + kp;
        if (x >= (uint32_t)src.width) break;
        float p[D], v[kGridMaxVd];
        load_point_xyt<D, kGridMaxVd>(src, x, y, blockIdx.z, p, v);
        int I[D];
        float F[D], Fi[D];
        grid_cell<D>(g, p, I, F, Fi);
        long long base;
        unsigned hi_ok;
        if (!grid_base<D>(g, I, base, hi_ok)) continue;
        if constexpr (KP > 1) {
            if (base != run_base) {   // a new cell: send the run so far, start a new one
                flush();
                run_base = base;
                run_hi = hi_ok;
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int k = 0; k < NV; ++k) acc[c][k] = 0.0f;
            }
#pragma unroll
            for (int corner = 0; corner < NC; ++corner) {
                long long off;
                const float w = grid_corner_weight<D>(g, F, Fi, corner, base, off);
#pragma unroll
                for (int k = 0; k < NV; ++k) acc[corner][k] = __fadd_rn(acc[corner][k], __fmul_rn(w, v[k]));
            }
        } else {
#pragma unroll
            for (int corner = 0; corner < NC; ++corner) {
                if (corner & ~hi_ok) continue;
                long long off;
                const float w = grid_corner_weight<D>(g, F, Fi, corner, base, off);
                float c[NV];
#pragma unroll
                for (int k = 0; k < NV; ++k) c[k] = __fmul_rn(w, v[k]);
                grid_add<VD>(g, off, c);
            }
        }
    }
    if constexpr (KP > 1) flush();
}

// The two [1 2 1]/4 passes of DenseGrid::blur_ (src/DenseGrid.h:186-238) along dimension j
// (taps 5: taps/2 passes).  The reference walks each row in place, but every value a pass
// writes depends only on values from before that pass (row[x] is overwritten after both
// row[x] and row[x+1] were read, and the running tmp carries 0.5*(old[x-1] + old[x])), so
// each cell is computed independently here, out of place, with the same single-precision
// operations in the same order:
//   x = 0:           0.5*(old[0]/2 + 0.5*(old[0] + old[1]))
//   0 < x < len-1:   0.5*(0.5*(old[x-1] + old[x]) + 0.5*(old[x] + old[x+1]))
//   x = len-1:       0.5*(tmp + 0.5*old[len-1]) in double (the reference's double literals),
//                    tmp = 0.5*(old[len-2] + old[len-1]) in single, or old[0]/2 when len == 1
// The second pass at x needs the first pass at x-1, x and x+1, which each thread evaluates
// from the five values around x.  One thread per grid value; consecutive threads are
// consecutive values, so every access is coalesced whatever the dimension.
__device__ __forceinline__ float grid_pass_value(float left, float here, float right, uint32_t x, uint32_t len) {
    const float t1 = x == 0 ? __fdiv_rn(here, 2.0f) : __fmul_rn(0.5f, __fadd_rn(left, here));
    if (x == len - 1) return (float)__dmul_rn(0.5, __dadd_rn((double)t1, __dmul_rn(0.5, (double)here)));
    return __fmul_rn(0.5f, __fadd_rn(t1, __fmul_rn(0.5f, __fadd_rn(here, right))));
}

__global__ void __launch_bounds__(kGridThreads) grid_blur_kernel(GridArgs g, int j, const float* src,
                                                                 float* dst, uint32_t total) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;   // grids hold < 2^30 values
    if (t >= total) return;
    const uint32_t s = (uint32_t)g.stride[j];
    const uint32_t len = (uint32_t)g.sizes[j];
    const uint32_t x = (t / s) % len;
    // old values at x-2 .. x+2 (those outside the row are never used)
    float o[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int xx = (int)x + k - 2;
        o[k] = (xx >= 0 && xx < (int)len) ? src[(int64_t)t + (int64_t)(k - 2) * s] : 0.0f;
    }
    // first pass at x-1, x, x+1, then the second pass at x
    float p1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int xx = (int)x + k - 1;
        p1[k] = (xx >= 0 && xx < (int)len) ? grid_pass_value(o[k], o[k + 1], o[k + 2], (uint32_t)xx, len) : 0.0f;
    }
    dst[t] = grid_pass_value(p1[0], p1[1], p1[2], x, len);
}

template <int D, int VD>
__global__ void __launch_bounds__(kGridThreads) grid_slice_kernel(PointSource src, unsigned bw, GridArgs g,
                                                                  OutView out) {
    const uint32_t x = blockIdx.x * bw + threadIdx.x % bw;
    const uint32_t y = blockIdx.y * (kGridThreads / bw) + threadIdx.x / bw;
    if (x >= (uint32_t)src.width || y >= (uint32_t)src.height) return;
    float p[D];
    load_position_xyt<D>(src, x, y, blockIdx.z, p);
    int I[D];
    float F[D], Fi[D];
    grid_cell<D>(g, p, I, F, Fi);
    float acc[kGridMaxVd];
#pragma unroll
    for (int k = 0; k < kGridMaxVd; ++k) acc[k] = 0.0f;
    long long base;
    unsigned hi_ok;
    const bool inside = grid_base<D>(g, I, base, hi_ok);
#pragma unroll
    for (int corner = 0; corner < (1 << D); ++corner) {
        if (!inside || (corner & ~hi_ok)) continue;
        long long off;
        const float w = grid_corner_weight<D>(g, F, Fi, corner, base, off);
        float c[kGridMaxVd];
        if constexpr (VD == 2) {
            const float2 q = __ldg(reinterpret_cast<const float2*>(g.grid + off));
            c[0] = q.x, c[1] = q.y;
        } else if constexpr (VD == 4) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(g.grid + off));
            c[0] = q.x, c[1] = q.y, c[2] = q.z, c[3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < kGridMaxVd; ++k) c[k] = k < g.vd ? g.grid[off + k] : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < kGridMaxVd; ++k)
            if (k < g.vd) acc[k] = __fadd_rn(acc[k], __fmul_rn(w, c[k]));
    }
    float* o = out.base + (long long)blockIdx.z * out.tstride + (long long)y * out.ystride + x;
    float wsum = acc[0];
#pragma unroll
    for (int k = 0; k < kGridMaxVd; ++k) if (k == g.vd - 1) wsum = acc[k];
#pragma unroll
    for (int k = 0; k < kGridMaxVd; ++k)
        if (k < out.channels) o[(long long)k * out.cstride] = out.normalize ? acc[k] / wsum : acc[k];
}

template <int D>
void launch_minmax(const PointSource& s, uint32_t n, float sf, unsigned* mm, int sms, cudaStream_t st) {
    uint64_t blocks = (n + kGridThreads - 1) / kGridThreads;
    if (blocks > (uint64_t)sms * 8) blocks = (uint64_t)sms * 8;
    if (blocks < 1) blocks = 1;
    grid_minmax_kernel<D><<<(unsigned)blocks, kGridThreads, 0, st>>>(s, n, sf, mm);
}
template <int D>
void launch_splat(const PointSource& s, uint32_t n, const GridArgs& g, cudaStream_t st) {
    if (!n) return;
    // runs of pixels summed in registers where the corner sums fit (2^d x vd <= 16)
    if (g.vd == 2 && D <= 3) {
        const PixelTiles t = pixel_tiles(s, 4);
        grid_splat_kernel<D, 2, 4><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g);
    } else if (g.vd == 4 && D <= 2) {
        const PixelTiles t = pixel_tiles(s, 4);
        grid_splat_kernel<D, 4, 4><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g);
    } else {
        const PixelTiles t = pixel_tiles(s, 1);
        if (g.vd == 2) grid_splat_kernel<D, 2, 1><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g);
        else if (g.vd == 4) grid_splat_kernel<D, 4, 1><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g);
        else grid_splat_kernel<D, 0, 1><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g);
    }
}
template <int D>
void launch_slice(const PointSource& s, uint32_t n, const GridArgs& g, const OutView& o, cudaStream_t st) {
    if (!n) return;
    const PixelTiles t = pixel_tiles(s, 1);
    if (g.vd == 2) grid_slice_kernel<D, 2><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g, o);
    else if (g.vd == 4) grid_slice_kernel<D, 4><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g, o);
    else grid_slice_kernel<D, 0><<<t.grid, kGridThreads, 0, st>>>(s, t.bw, g, o);
}

#define PGPU_GRID_DISPATCH(d, call)          \
    switch (d) {                             \
    case 1: { constexpr int DD = 1; call; } break; \
    case 2: { constexpr int DD = 2; call; } break; \
    case 3: { constexpr int DD = 3; call; } break; \
    case 4: { constexpr int DD = 4; call; } break; \
    case 5: { constexpr int DD = 5; call; } break; \
    }

}  // namespace

int run_grid(Engine& E, const LatticeJob& J, cudaStream_t st) {
    const int d = J.d, vd = J.vd;
    if (d < 1 || d > kGridMaxD)
        return fail(PGPU_ERR_UNSUPPORTED, "the grid method takes 1..%d position dimensions (got %d)",
                    kGridMaxD, d);
    if (vd < 1 || vd > kGridMaxVd) return fail(PGPU_ERR_UNSUPPORTED, "%d value channels", vd);
    if (J.payload != kPayloadF32) return fail(PGPU_ERR_UNSUPPORTED, "the grid method computes in FP32 only");
    for (const PointSource* ps : {&J.splat, &J.slice}) {   // the launches' grid dimensions
        if (ps == &J.slice && J.replay) continue;
        if (ps->frames > 65535 || (ps->height > 1 && ps->height > 65535 * (kGridThreads / 32)))
            return fail(PGPU_ERR_UNSUPPORTED, "the grid method takes at most 65535 frames and %d rows",
                        65535 * (kGridThreads / 32));
    }
    // DenseGrid's constructor (src/DenseGrid.h:111-127): sqrtf(1.0/3 + (taps-1)*0.25)
    const float sf = sqrtf((float)(1.0 / 3 + (kGridTaps - 1) * 0.25));
    const PointSource& sl = J.replay ? J.splat : J.slice;
    const uint32_t nsl = J.replay ? J.n : J.n_slice;
    int rc;
    if ((rc = E.meta.ensure(64))) return rc;
    unsigned* mm = (unsigned*)E.meta.p;
    CUDA_TRY(cudaEventRecord(E.ev[0], st));
    CUDA_TRY(cudaMemsetAsync(mm, 0xFF, sizeof(unsigned) * d, st));
    CUDA_TRY(cudaMemsetAsync(mm + d, 0, sizeof(unsigned) * d, st));
    PGPU_GRID_DISPATCH(d, launch_minmax<DD>(J.splat, J.n, sf, mm, E.sms, st));
    if (!J.replay) PGPU_GRID_DISPATCH(d, launch_minmax<DD>(sl, nsl, sf, mm, E.sms, st));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(E.hstat, mm, sizeof(unsigned) * 2 * d, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));

    GridArgs g;
    memset(&g, 0, sizeof(g));
    g.vd = vd;
    g.sf = sf;
    g.stride[0] = vd;
    for (int i = 0; i < d; ++i) {
        const float lo = unordered_float(E.hstat[i]), hi = unordered_float(E.hstat[d + i]);
        if (!std::isfinite(lo) || !std::isfinite(hi))
            return fail(PGPU_ERR_ARGUMENT, "positions are not finite");
        g.minp[i] = lo;
        const float span = hi - lo;   // float subtraction, as maxPosition[i] - minPosition[i]
        g.sizes[i] = (int)(std::ceil(span) + 1);
        g.stride[i + 1] = g.stride[i] * g.sizes[i];
        if (g.sizes[i] < 1 || g.stride[i + 1] > kGridMaxCells)
            return fail(PGPU_ERR_CAPACITY, "the grid would need more than %lld cells", kGridMaxCells);
    }
    const long long cells = g.stride[d];
    if ((rc = E.grid.ensure((size_t)cells * sizeof(float))) ||
        (rc = E.grid2.ensure((size_t)cells * sizeof(float))))
        return rc;
    g.grid = (float*)E.grid.p;
    CUDA_TRY(cudaMemsetAsync(g.grid, 0, (size_t)cells * sizeof(float), st));
    CUDA_TRY(cudaEventRecord(E.ev[1], st));
    PGPU_GRID_DISPATCH(d, launch_splat<DD>(J.splat, J.n, g, st));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(E.ev[3], st));
    // one launch per dimension (both of its passes), ping-ponging between the grid and a
    // second buffer
    static_assert(kGridTaps / 2 == 2, "grid_blur_kernel fuses exactly two passes");
    float* bufs[2] = {g.grid, (float*)E.grid2.p};
    int cur = 0;
    const unsigned blur_blocks = (unsigned)((cells + kGridThreads - 1) / kGridThreads);
    for (int j = 0; j < d; ++j, cur ^= 1)
        grid_blur_kernel<<<blur_blocks, kGridThreads, 0, st>>>(g, j, bufs[cur], bufs[cur ^ 1], (uint32_t)cells);
    g.grid = bufs[cur];
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(E.ev[4], st));
    PGPU_GRID_DISPATCH(d, launch_slice<DD>(sl, nsl, g, J.out, st));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(E.ev[5], st));
    CUDA_TRY(cudaStreamSynchronize(st));

    pgpu_stats s;
    memset(&s, 0, sizeof(s));
    s.points = J.n;
    s.vertices = cells / vd;        // grid cells
    s.capacity = cells / vd;
    s.d = d;
    s.vd = vd;
    s.payload = J.payload;
    cudaEventElapsedTime(&s.ms_splat, E.ev[1], E.ev[3]);
    cudaEventElapsedTime(&s.ms_compact, E.ev[0], E.ev[1]);   // the bounding-box preview
    cudaEventElapsedTime(&s.ms_blur, E.ev[3], E.ev[4]);
    cudaEventElapsedTime(&s.ms_slice, E.ev[4], E.ev[5]);
    cudaEventElapsedTime(&s.ms_total, E.ev[0], E.ev[5]);
    set_stats(s);
    return PGPU_OK;
}

}  // namespace pgpu
