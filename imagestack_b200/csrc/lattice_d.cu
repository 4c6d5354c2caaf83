// Per-dimension instantiation of the splat, neighbour and slice kernels.  This file is
// compiled once for each d in 1..16 with -DPGPU_D=d, so the sixteen variants build in
// parallel and each keeps its per-point arrays in registers.
#include <atomic>

#include "lattice_ops.h"

#ifndef PGPU_D
#error "compile with -DPGPU_D=<number of position dimensions>"
#endif

namespace pgpu {
namespace {

constexpr int D = PGPU_D;

int grid_cap(uint64_t work, int threads, int sms) {
    uint64_t g = (work + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

template <int VDP, typename Acc>
void splat_t(const SplatArgs& a, cudaStream_t st) {
    if (a.blocks) splat_kernel<D, VDP, Acc><<<a.blocks, kSplatThreads, 0, st>>>(a);
}

bool splat(const SplatArgs& a, int vdp, int payload, cudaStream_t st) {
    const bool f64 = payload == kPayloadF64;
    switch (vdp) {
    case 2: f64 ? splat_t<2, double>(a, st) : splat_t<2, float>(a, st); return true;
    case 4: f64 ? splat_t<4, double>(a, st) : splat_t<4, float>(a, st); return true;
    case 8: f64 ? splat_t<8, double>(a, st) : splat_t<8, float>(a, st); return true;
    }
    return false;
}

// The tile splat's shared-memory limit is an attribute of each kernel on each device; it
// is set once per device (a bit per device ordinal), outside any stream capture.
std::atomic<uint64_t> g_tile_prepared{0};

template <int VDP>
bool prepare_tile_t() {
    if constexpr (key_words(D) == 1) {
        if (cudaFuncSetAttribute(splat_tile_kernel<D, VDP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_smem_bytes(D, VDP)) != cudaSuccess)
            return false;
        if constexpr (index_in_key(D))
            return cudaFuncSetAttribute(splat_tile_kernel<D, VDP, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tile_smem_bytes(D, VDP)) == cudaSuccess;
    }
    return true;
}

bool prepare() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const uint64_t bit = 1ull << (dev & 63);
    if (g_tile_prepared.load() & bit) return true;
    if (!prepare_tile_t<2>() || !prepare_tile_t<4>() || !prepare_tile_t<8>()) return false;
    g_tile_prepared.fetch_or(bit);
    return true;
}

template <int VDP>
bool splat_tile_t(const SplatArgs& a, cudaStream_t st) {
    if constexpr (key_words(D) == 1) {
        if (!a.tile_blocks) return true;
        if (a.vrows) {   // vertex-ordered rows: d <= 6 only
            if constexpr (index_in_key(D)) {
                splat_tile_kernel<D, VDP, true><<<a.tile_blocks, kTileThreads, tile_smem_bytes(D, VDP), st>>>(a);
                return true;
            }
            return false;
        }
        splat_tile_kernel<D, VDP, false><<<a.tile_blocks, kTileThreads, tile_smem_bytes(D, VDP), st>>>(a);
        return true;
    } else {
        return a.tile_blocks == 0;
    }
}

bool splat_tile(const SplatArgs& a, int vdp, int payload, cudaStream_t st) {
    if (payload == kPayloadF64) return a.tile_blocks == 0;
    switch (vdp) {
    case 2: return splat_tile_t<2>(a, st);
    case 4: return splat_tile_t<4>(a, st);
    case 8: return splat_tile_t<8>(a, st);
    }
    return false;
}

void neighbours(const NbrArgs& a, uint32_t vmax, int sms, cudaStream_t st) {
    neighbours_kernel<D><<<grid_cap(vmax, 256, sms), 256, 0, st>>>(a);
}

template <int VDP, typename A>
void slice_t(const SliceArgs& a, cudaStream_t st) {
    if (!a.blocks) return;
    if (a.rec_slot && a.rec_w_in && !a.rec_vtx)
        slice_replay_kernel<D, VDP, A><<<a.blocks, kSliceThreads, 0, st>>>(a);
    else
        slice_kernel<D, VDP, A><<<a.blocks, kSliceThreads, 0, st>>>(a);
}

// the slice reads the last blur pass's rows, plain (not homogeneous) products: FP64 for
// the FP64 lattice, FP32 otherwise; homogeneous lattices exist only for 16-bit payloads
template <int VDP>
bool slice_p(const SliceArgs& a, int payload, bool homog, cudaStream_t st) {
    switch (payload) {
    case kPayloadF32: slice_t<VDP, float>(a, st); return !homog;
    case kPayloadF16:
    case kPayloadBF16: slice_t<VDP, float>(a, st); return true;
    case kPayloadF64: slice_t<VDP, double>(a, st); return !homog;
    }
    return false;
}

bool slice(const SliceArgs& a, int vdp, int payload, bool homog, cudaStream_t st) {
    switch (vdp) {
    case 2: return slice_p<2>(a, payload, homog, st);
    case 4: return slice_p<4>(a, payload, homog, st);
    case 8: return slice_p<8>(a, payload, homog, st);
    }
    return false;
}

const DimOps kOps = {splat, splat_tile, prepare, neighbours, slice};

}  // namespace

#define PGPU_CAT2(a, b) a##b
#define PGPU_CAT(a, b) PGPU_CAT2(a, b)
const DimOps* PGPU_CAT(dim_ops_, PGPU_D)() { return &kOps; }

}  // namespace pgpu
