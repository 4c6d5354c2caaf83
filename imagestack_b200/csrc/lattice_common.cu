// Kernels that do not depend on the number of position dimensions: first-touch
// marking, the prefix popcount that numbers the vertices, compaction and the blur.
#include <algorithm>

#include "lattice_ops.h"

// default tile splat tiles: PGPU_TILE_W pixels wide, kTilePixels / PGPU_TILE_W high (a
// power of two up to kTilePixels; the autotuner also tries 32x8)
#ifndef PGPU_TILE_W
#define PGPU_TILE_W 16u
#endif

namespace pgpu {

__global__ void mark_kernel(const uint32_t* __restrict__ ft, uint32_t cap, uint32_t* bitmap) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < cap; s += gridDim.x * blockDim.x) {
        const uint32_t f = ft[s];
        if (f != 0xFFFFFFFFu) atomicOr(bitmap + (f >> 5), 1u << (f & 31u));
    }
}

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= (unsigned)o) v += u;
    }
    return v;
}

// exclusive scan across the block; returns the block total through *total
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t inc = warp_inclusive(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t ws = (lane < blockDim.x / 32) ? warp_sums[lane] : 0u;
        const uint32_t wi = warp_inclusive(ws);
        warp_sums[lane] = wi - ws;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const uint32_t r = warp_sums[warp] + inc - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads)
scan_reduce_kernel(const uint32_t* __restrict__ bitmap, uint32_t nwords, uint32_t* partials) {
    const uint32_t base = blockIdx.x * (uint32_t)(kScanThreads * kScanItems);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t w = base + k * kScanThreads + threadIdx.x;
        if (w < nwords) s += __popc(bitmap[w]);
    }
    __shared__ uint32_t total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
scan_partials_kernel(uint32_t* partials, uint32_t nparts, uint32_t* total_out) {
    __shared__ uint32_t total;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nparts; base += kScanThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nparts ? partials[i] : 0u;
        const uint32_t ex = block_exclusive(v, &total);
        if (i < nparts) partials[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void __launch_bounds__(kScanThreads)
scan_down_kernel(const uint32_t* __restrict__ bitmap, uint32_t nwords,
                 const uint32_t* __restrict__ partials, uint32_t* offs) {
    const uint32_t base = blockIdx.x * (uint32_t)(kScanThreads * kScanItems) + threadIdx.x * kScanItems;
    uint32_t c[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        c[k] = (base + k < nwords) ? __popc(bitmap[base + k]) : 0u;
        s += c[k];
    }
    __shared__ uint32_t total;
    uint32_t ex = block_exclusive(s, &total) + partials[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < nwords) offs[base + k] = ex;
        ex += c[k];
    }
}

// Vertices of each segment of a batch: first touches are numbered segment after segment,
// so segment k owns the first-touch bits in [entry[k], entry[k+1]).
__device__ __forceinline__ uint32_t bits_before(const uint32_t* bitmap, const uint32_t* offs,
                                                uint32_t nwords, uint32_t total, uint32_t e) {
    const uint32_t w = e >> 5;
    if (w >= nwords) return total;
    return offs[w] + __popc(bitmap[w] & ((1u << (e & 31u)) - 1u));
}

__global__ void segment_counts_kernel(const uint32_t* bitmap, const uint32_t* offs, uint32_t nwords,
                                      const uint32_t* total, const uint32_t* entry, int nseg,
                                      uint32_t* counts) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nseg) return;
    const uint32_t t = *total;
    counts[k] = bits_before(bitmap, offs, nwords, t, entry[k + 1]) -
                bits_before(bitmap, offs, nwords, t, entry[k]);
}

void launch_segment_counts(const uint32_t* bitmap, const uint32_t* offs, uint32_t nwords,
                           const uint32_t* total, const uint32_t* entry, int nseg, uint32_t* counts,
                           cudaStream_t st) {
    segment_counts_kernel<<<(nseg + 127) / 128, 128, 0, st>>>(bitmap, offs, nwords, total, entry,
                                                              nseg, counts);
}

// ---------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------
static uint32_t pow2_at_least(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

void segment_geometry(Segment& s, const PointSource& slice_src, bool tiled, uint32_t* splat,
                      uint32_t* tile, uint32_t* slice, uint32_t tile_w) {
    const PointSource& q = s.src;
    s.src.pos_is_val = q.pos.base == q.val.base && q.pos.ystride == q.val.ystride &&
                       q.pos.tstride == q.val.tstride && q.pos.cstride == q.val.cstride &&
                       q.pos_channels == q.val_channels;
    const uint32_t W = (uint32_t)s.src.width, H = (uint32_t)s.src.height, F = (uint32_t)s.src.frames;
    const uint64_t n = (uint64_t)W * H * F;
    if (tiled) {
        // tile_w x (kTilePixels / tile_w) tiles (16x16 by default: a warp is two rows of
        // 16 pixels); a point list (one row) in runs of kTilePixels
        const uint32_t tw = tile_w ? tile_w : (uint32_t)PGPU_TILE_W;
        s.tile_w = (H == 1 && F == 1) ? (uint32_t)kTilePixels : std::min<uint32_t>(tw, pow2_at_least(W));
        s.tile_h = (uint32_t)kTilePixels / s.tile_w;
        s.tiles_x = (W + s.tile_w - 1) / s.tile_w;
        s.tiles_y = (H + s.tile_h - 1) / s.tile_h;
        *tile = s.tiles_x * s.tiles_y * F;
        *splat = 0;
    } else {
        s.tile_w = s.tile_h = s.tiles_x = s.tiles_y = 0;
        *tile = 0;
        *splat = (uint32_t)((n + kSplatThreads - 1) / kSplatThreads);
    }
    const uint32_t Ws = (uint32_t)slice_src.width, Hs = (uint32_t)slice_src.height,
                   Fs = (uint32_t)slice_src.frames;
    s.slice_tw = (Hs == 1 && Fs == 1) ? (uint32_t)kSliceThreads : std::min<uint32_t>(32u, pow2_at_least(Ws));
    s.slice_th = (uint32_t)kSliceThreads / s.slice_tw;
    s.stiles_x = (Ws + s.slice_tw - 1) / s.slice_tw;
    s.stiles_y = (Hs + s.slice_th - 1) / s.slice_th;
    *slice = s.stiles_x * s.stiles_y * Fs;
}
const DimOps* dim_ops(int d) {
    switch (d) {
    case 1: return dim_ops_1();
    case 2: return dim_ops_2();
    case 3: return dim_ops_3();
    case 4: return dim_ops_4();
    case 5: return dim_ops_5();
    case 6: return dim_ops_6();
    case 7: return dim_ops_7();
    case 8: return dim_ops_8();
    case 9: return dim_ops_9();
    case 10: return dim_ops_10();
    case 11: return dim_ops_11();
    case 12: return dim_ops_12();
    case 13: return dim_ops_13();
    case 14: return dim_ops_14();
    case 15: return dim_ops_15();
    case 16: return dim_ops_16();
    }
    return nullptr;
}

static int grid_for(uint64_t work, int threads, int sms) {
    uint64_t g = (work + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

void launch_mark(const uint32_t* ft, uint32_t cap, uint32_t* bitmap, int sms, cudaStream_t st) {
    mark_kernel<<<grid_for(cap, 256, sms), 256, 0, st>>>(ft, cap, bitmap);
}

uint32_t scan_parts(uint32_t nwords) {
    const uint32_t per = kScanThreads * kScanItems;
    return (nwords + per - 1) / per;
}

void launch_scan(const uint32_t* bitmap, uint32_t nwords, uint32_t* partials, uint32_t* offs,
                 uint32_t* total, cudaStream_t st) {
    const uint32_t parts = scan_parts(nwords);
    if (parts == 0) {
        cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
        return;
    }
    scan_reduce_kernel<<<parts, kScanThreads, 0, st>>>(bitmap, nwords, partials);
    scan_partials_kernel<<<1, kScanThreads, 0, st>>>(partials, parts, total);
    scan_down_kernel<<<parts, kScanThreads, 0, st>>>(bitmap, nwords, partials, offs);
}

template <int KW, int VDP, typename Acc, typename P, bool HOMOG>
static void assign_t(const CompactArgs& a, int sms, cudaStream_t st) {
    if (a.vlist)
        assign_list_kernel<KW, VDP, Acc, P, HOMOG><<<grid_for(a.table.cap, 256, sms), 256, 0, st>>>(a);
    else
        assign_kernel<KW, VDP, Acc, P, HOMOG><<<grid_for(a.table.cap, 256, sms), 256, 0, st>>>(a);
}

template <int KW, int VDP>
static bool assign_p(const CompactArgs& a, int payload, bool homog, int sms, cudaStream_t st) {
    if (homog) {   // 16-bit homogeneous lattices: FP32 normalised rows for the first blur pass
        if (payload != kPayloadF16 && payload != kPayloadBF16) return false;
        assign_t<KW, VDP, float, float, true>(a, sms, st);
        return true;
    }
    switch (payload) {
    case kPayloadF32: assign_t<KW, VDP, float, float, false>(a, sms, st); return true;
    case kPayloadF16: assign_t<KW, VDP, float, __half, false>(a, sms, st); return true;
    case kPayloadBF16: assign_t<KW, VDP, float, __nv_bfloat16, false>(a, sms, st); return true;
    case kPayloadF64: assign_t<KW, VDP, double, double, false>(a, sms, st); return true;
    }
    return false;
}

template <int KW>
static bool assign_v(const CompactArgs& a, int vdp, int payload, bool homog, int sms,
                     cudaStream_t st) {
    switch (vdp) {
    case 2: return assign_p<KW, 2>(a, payload, homog, sms, st);
    case 4: return assign_p<KW, 4>(a, payload, homog, sms, st);
    case 8: return assign_p<KW, 8>(a, payload, homog, sms, st);
    }
    return false;
}

bool launch_assign(const CompactArgs& a, int kw, int vdp, int payload, bool homog, int sms,
                   cudaStream_t st) {
    switch (kw) {
    case 1: return assign_v<1>(a, vdp, payload, homog, sms, st);
    case 2: return assign_v<2>(a, vdp, payload, homog, sms, st);
    case 3: return assign_v<3>(a, vdp, payload, homog, sms, st);
    }
    return false;
}

}  // namespace pgpu
