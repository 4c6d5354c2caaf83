// Launch interface between the host pipeline (engine.cu) and the kernels.
#pragma once

#include "lattice_kernels.cuh"

namespace pgpu {

enum PayloadKind { kPayloadF32 = 0, kPayloadF16 = 1, kPayloadBF16 = 2, kPayloadF64 = 3 };

inline int payload_bytes(int payload) {
    return payload == kPayloadF64 ? 8 : payload == kPayloadF32 ? 4 : 2;
}
// splat accumulators are FP32, or FP64 for the FP64 lattice
inline int accum_bytes(int payload) { return payload == kPayloadF64 ? 8 : 4; }

// kernels whose code depends on the number of position dimensions d
struct DimOps {
    bool (*splat)(const SplatArgs&, int vdp, int payload, cudaStream_t);
    // the tile splat over the segments with tile_w > 0 (a.tile_blocks blocks); false when
    // this d or payload has no tile splat (multi-word keys, FP64 accumulators)
    bool (*splat_tile)(const SplatArgs&, int vdp, int payload, cudaStream_t);
    // one-time per-device set-up of the tile splat's kernels (their shared-memory limit);
    // called outside any stream capture, before the first launch
    bool (*prepare)();
    void (*neighbours)(const NbrArgs&, uint32_t vmax, int sms, cudaStream_t);
    bool (*slice)(const SliceArgs&, int vdp, int payload, bool homog, cudaStream_t);
};

// one definition per d, in lattice_d.cu compiled once per d
#define PGPU_DECLARE_DIM(D) const DimOps* dim_ops_##D();
PGPU_DECLARE_DIM(1) PGPU_DECLARE_DIM(2) PGPU_DECLARE_DIM(3) PGPU_DECLARE_DIM(4)
PGPU_DECLARE_DIM(5) PGPU_DECLARE_DIM(6) PGPU_DECLARE_DIM(7) PGPU_DECLARE_DIM(8)
PGPU_DECLARE_DIM(9) PGPU_DECLARE_DIM(10) PGPU_DECLARE_DIM(11) PGPU_DECLARE_DIM(12)
PGPU_DECLARE_DIM(13) PGPU_DECLARE_DIM(14) PGPU_DECLARE_DIM(15) PGPU_DECLARE_DIM(16)
#undef PGPU_DECLARE_DIM

const DimOps* dim_ops(int d);

// Launch geometry of one segment (its src, the splat points, and slice_src, the points
// sliced, are set): the direct-splat blocks or, when `tiled`, the tile-splat tiles, and
// the slice tiles.  Returns the blocks of each launch through *splat, *tile and *slice.
void segment_geometry(Segment& s, const PointSource& slice_src, bool tiled, uint32_t* splat,
                      uint32_t* tile, uint32_t* slice, uint32_t tile_w = 0);

void launch_mark(const uint32_t* ft, uint32_t cap, uint32_t* bitmap, int sms, cudaStream_t st);
// per-segment vertex counts from the first-touch bitmap and its prefix popcount
void launch_segment_counts(const uint32_t* bitmap, const uint32_t* offs, uint32_t nwords,
                           const uint32_t* total, const uint32_t* entry, int nseg, uint32_t* counts,
                           cudaStream_t st);
uint32_t scan_parts(uint32_t nwords);
void launch_scan(const uint32_t* bitmap, uint32_t nwords, uint32_t* partials, uint32_t* offs,
                 uint32_t* total, cudaStream_t st);
// homog: rows normalised by the homogeneous weight, written as FP32 for the first blur pass
bool launch_assign(const CompactArgs& a, int kw, int vdp, int payload, bool homog, int sms,
                   cudaStream_t st);
// src_f32: the pass reads FP32 rows (first pass of a homogeneous 16-bit lattice);
// dst_acc: it writes rows of the arithmetic type (the last pass, for the slice);
// pair: it blurs along two consecutive axes
bool launch_blur(const BlurArgs& a, int blocks, int ilp, int vdp, int payload, bool homog,
                 bool src_f32, bool dst_acc, bool pair, cudaStream_t st);

// All d+1 blur axes in fused pairs; intermediate rows ping-pong between bufs[0] and
// bufs[1] (payload type); the last pass writes the arithmetic type into slot space
// through vtx2slot, where the slice reads it.
struct BlurPlan {
    int d, vdp, payload;
    bool homog, src_f32;
    const int2* nbr;       // (d+1) x nbr_stride neighbour pairs
    size_t nbr_stride;
    const uint32_t* nverts;
    uint32_t vmax;
    const void* src;       // the compaction's rows in vertex order
    void* bufs[2];
    void* f32buf = nullptr;   // FP32 rows (16-bit payloads, one axis per pass)
    void* sval;
    const uint32_t* vtx2slot;
    int wc, sms;
    bool pairs = true;     // fuse consecutive axes into one launch
    int grid = 0;          // 0: 16 blocks per SM striding over the vertices, 1: one vertex per
                           // thread, 2: as 0 with two vertices per iteration (one-axis passes)
};
int blur_all_axes(const BlurPlan& p, cudaStream_t st);   // 0 on success

}  // namespace pgpu
