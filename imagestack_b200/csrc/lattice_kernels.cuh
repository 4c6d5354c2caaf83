// Kernels of the permutohedral-lattice Gauss transform (sm_100a).
//
// Pipeline for one lattice (one image, or one segment of a batch):
//   splat      one thread per point: positions from the planar images, elevation and
//              simplex (src/Permutohedral.h:293-356), d+1 vertex keys, warp-aggregated
//              insert into the open-addressed table and vector atomics of the weighted
//              values into the slot's accumulator row; atomicMin of the first touch.
//   mark       one bit per (point, remainder) entry: the entry that first touched a
//              vertex gets its bit set.
//   scan       prefix popcount of that bitmap: the rank of a first-touch entry among
//              all first touches is the vertex index the reference assigns
//              (insertion order, src/Permutohedral.h:69-75).
//   assign     vertex index per slot, compacted keys and values in vertex order.
//   neighbours two neighbours per vertex and axis (src/Permutohedral.h:446-464).
//   blur       d+1 passes of [1 2 1]/4 over the compacted vertex list (:466-470).
//   slice      one thread per output point: the same simplex again, d+1 lookups,
//              barycentric interpolation (:418-427 / :405-407), optional normalisation
//              by the homogeneous channel (src/GaussTransform.cpp:673-676).
#pragma once

#include <type_traits>

#include "lattice_device.cuh"

namespace pgpu {

// A planar float32 image: element (x, y, t, c) at base + c*cstride + t*tstride + y*ystride + x
// (the addressing of ImageStack's Image, src/Image.h:57-67).
struct PlanarView {
    const float* base;
    long long ystride, tstride, cstride;
};

// Where the points of a lattice come from.  Point i is pixel (x, y, t) of a
// width x height x frames grid, i = (t*height + y)*width + x, the loop order of
// src/GaussTransform.cpp:173-185.  Position channel c (c < pos_channels) is
// view(c) * pos_scale[c]; then the enabled pixel coordinates follow, each multiplied by
// its scale (the X()/Y()/T() positions of src/GaussTransform.cpp:657-667).  Values are
// the val_channels of the value view, then a homogeneous 1 if `homogeneous`.
struct PointSource {
    int width, height, frames;
    PlanarView pos;
    int pos_channels;
    float pos_scale[kMaxD];
    int coord_mask;            // bit 0: x, bit 1: y, bit 2: t
    float coord_scale[3];
    PlanarView val;
    int val_channels;
    int homogeneous;
    int pos_is_val;            // the position channels are the value channels (bilateral)
};

struct OutView {
    float* base;
    long long ystride, tstride, cstride;
    int channels;     // channels written
    int normalize;    // 1: out[c] = acc[c] / acc[vd-1] (JointBilateral), 0: out[c] = acc[c]
};

// One lattice of a batch — one image; the single-image entry points run a batch of one.
// Each lattice owns a contiguous range of the shared hash-slot array and of the point
// numbering; its points are numbered after the previous lattice's, so first-touch order,
// and with it the vertex numbering, stays per-lattice insertion order.
//
// Blocks of three launches cover a segment, each launch with its own block numbering:
//   direct splat  kSplatThreads consecutive points per block (splat_base; no blocks when
//                 the segment uses the tile splat)
//   tile splat    one tile_w x tile_h tile of one frame per block, tiles_x x tiles_y tiles
//                 per frame (tile_base; no blocks when tile_w == 0)
//   slice         one slice_tw x slice_th tile of one frame per block (slice_tw * slice_th
//                 == kSliceThreads), stiles_x x stiles_y tiles per frame (block_base)
struct Segment {
    PointSource src;       // its points
    OutView out;           // where its slice goes
    uint32_t n;            // points
    uint32_t point_base;   // first point in the batch numbering
    uint32_t block_base;   // first block of the segment in the slice launch
    uint32_t slot_base;    // first slot in the shared hash-slot array
    uint32_t cap;          // slots
    uint32_t splat_base;   // first block in the direct splat launch
    uint32_t tile_base;    // first block in the tile splat launch
    uint32_t tile_w, tile_h, tiles_x, tiles_y;     // tile splat geometry (tile_w 0: direct)
    uint32_t slice_tw, slice_th, stiles_x, stiles_y;   // slice geometry
    uint32_t pad_;
};

// Segment of block b of a launch whose per-segment first blocks are the field Base: the
// last segment whose Base <= b (segments are in block order; a segment with no blocks in
// this launch shares its Base with the next one and is never picked for a block).
template <uint32_t Segment::*Base>
__device__ __forceinline__ int segment_by(const Segment* segs, int nseg, uint32_t b) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&(segs[mid].*Base)) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int segment_of_block(const Segment* segs, int nseg, uint32_t b) {
    return segment_by<&Segment::block_base>(segs, nseg, b);
}

// Segment of slot s: the last k with slot_base[k] <= s (slot_base has nseg + 1 entries).
__device__ __forceinline__ int segment_of_slot(const uint32_t* slot_base, int nseg, uint32_t s) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(slot_base + mid) <= s) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// the block's segment, copied into shared memory by the whole block (ends with a barrier)
__device__ __forceinline__ void load_segment(const Segment* g, Segment& s) {
    static_assert(sizeof(Segment) % 4 == 0, "Segment is copied as 32-bit words");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(g);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s);
    for (int t = threadIdx.x; t < (int)(sizeof(Segment) / 4); t += blockDim.x) dst[t] = __ldg(src + t);
    __syncthreads();
}

struct SplatArgs {
    const Segment* segs;
    int nseg;
    uint32_t n_total;      // points of the batch
    LatticeConsts lc;
    uint4* key0;           // the shared hash-slot array (cap_total slots)
    uint4* keyn;
    uint32_t cap_total;
    void* vals;            // cap_total * VDP accumulators (float or double), zeroed
    uint32_t* ft;          // cap_total first-touch entries, all ones; null: not tracked
    uint32_t* rec_slot;    // optional [r][n_total] slot of every (point, remainder)
    float* rec_w;          // optional [r][n_total] barycentric weight of every (point, remainder)
    unsigned* seg_status;  // one status word per segment
    uint32_t blocks;       // direct splat blocks of the batch
    uint32_t tile_blocks;  // tile splat blocks of the batch
    // optional vertex list: every slot the splat creates is appended to vlist (vcount
    // entries, zeroed), and counted in its segment's seg_counts entry (zeroed)
    uint32_t* vlist;
    uint32_t* vcount;
    uint32_t* seg_counts;
    // Vertex-ordered rows (the tile splat, d <= 6): with vrows set, the splat numbers each
    // vertex as it creates it (the position the vertex list would give it) and
    // accumulates every lane's row into vrows[v*VDP..] (FP32, zeroed before the launch);
    // the record holds vertex indices instead of slots; the creator writes the vertex's
    // key (vkey0), its slot (vtx2slot) and its index into the key word, where other blocks
    // read it.  No compaction is needed afterwards.
    void* vrows = nullptr;
    uint4* vkey0 = nullptr;
    uint32_t* vtx2slot = nullptr;
    // with vrows: the creator also marks its vertex's neighbour pairs (nbr_axes axes,
    // nbr_stride apart) absent, for a neighbour search that looks up one direction per axis
    int2* nbr_init = nullptr;
    uint32_t nbr_stride = 0;
    int nbr_axes = 0;
};

// Appends of one block to the batch's vertex list: slots go to the block's shared-memory
// list first; after a barrier one thread reserves the block's range of the global list
// with one atomic (and adds the count to the segment's), and the block copies its slots.
// A block that creates more than kBlockListCap slots appends the rest one by one.
constexpr uint32_t kBlockListCap = 512;
struct BlockList {
    uint32_t* slots;   // shared memory, kBlockListCap entries
    uint32_t* count;   // shared memory, zeroed before the block's first append
    uint32_t* base;    // shared memory
};
__device__ __forceinline__ void block_list_append(const BlockList& L, const SplatArgs& a, int kseg,
                                                  uint32_t slot) {
    const uint32_t j = atomicAdd(L.count, 1u);
    if (j < kBlockListCap) {
        L.slots[j] = slot;
    } else {
        a.vlist[atomicAdd(a.vcount, 1u)] = slot;
        atomicAdd(a.seg_counts + kseg, 1u);
    }
}
// called by the whole block, after a barrier that follows the last append
__device__ __forceinline__ void block_list_flush(const BlockList& L, const SplatArgs& a, int kseg) {
    const uint32_t n = min(*L.count, kBlockListCap);
    if (n == 0) return;
    if (threadIdx.x == 0) {
        *L.base = atomicAdd(a.vcount, n);
        atomicAdd(a.seg_counts + kseg, n);
    }
    __syncthreads();
    const uint32_t base = *L.base;
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) a.vlist[base + j] = L.slots[j];
}

struct CompactArgs {
    TableView table;
    const uint32_t* ft;
    uint32_t* bitmap;      // words covering n*(d+1) entries
    uint32_t nwords;
    const uint32_t* offs;  // exclusive prefix popcount per word
    uint32_t* slot2vtx;
    uint32_t* vtx2slot;
    uint4* vkey0;          // vertex keys, word 0 ...
    uint4* vkeyn;          // ... and later words, (KW-1) x vcap
    uint32_t vcap;
    const void* tvals;     // slot accumulators
    void* vvals;           // vertex values (payload type)
    int wc;                // homogeneous weight channel (homogeneous rows only)
    uint8_t* tags = nullptr;   // optional slot tags (zeroed), written for occupied slots
    const uint32_t* vlist = nullptr;    // the splat's vertex list (list order), or null:
    const uint32_t* nverts = nullptr;   // first-touch order through ft and the bitmap
    int index_in_key = 0;   // store each vertex's index in its key word (d <= 6)
    // optional: mark every vertex's neighbour pairs absent (nbr_axes axes, nbr_stride apart)
    // for the neighbour search that looks up one direction per axis
    int2* nbr_init = nullptr;
    uint32_t nbr_stride = 0;
    int nbr_axes = 0;
};

struct NbrArgs {
    uint4* key0;           // the shared hash-slot array
    uint4* keyn;
    uint32_t cap_total;
    const uint32_t* seg_slot_base;   // nseg + 1 slot boundaries
    int nseg;
    const uint32_t* vtx2slot;
    const uint32_t* slot2vtx;
    const uint4* vkey0;
    const uint4* vkeyn;
    uint32_t vcap;
    const uint32_t* nverts;
    int2* nbr;             // (d+1) x vcap pairs
    const uint8_t* tags = nullptr;   // slot tags of the compaction, or null: plain lookups
    const unsigned* seg_status = nullptr;   // the splat's per-segment status, or null
    // one lookup per axis: vertex v finds u = n1(v) and, as n2(u) = v, writes v into u's
    // pair too; every pair must hold (-1, -1) beforehand (written by the splat's creators
    // with vertex-ordered rows, by the compaction otherwise)
    int half = 0;
    // homogeneous FP32 rows the splat left as plain sums (w*m_0.., w), vertex-ordered:
    // each vertex's row is normalised here in place to (m_0.., w), as the compaction
    // would have stored it; null: nothing to do
    float* norm_rows = nullptr;
    int vdp = 0, wc = 0;
};

// One launch blurs along one axis (nbrA) or, fused, along two consecutive axes (nbrA then
// nbrB): the first axis's result stays in registers instead of being stored and reloaded.
struct BlurArgs {
    const int2* nbrA;           // neighbours along the first axis of the pass
    const int2* nbrB;           // neighbours along the second axis (fused passes)
    const uint32_t* nverts;
    const void* src;            // rows in vertex order
    void* dst;                  // rows in vertex order, or in slot space with dst_map
    const uint32_t* dst_map;    // row index of vertex v in dst (vertex -> slot); null: v
    int wc;                     // homogeneous weight channel (homogeneous rows only)
    int products = 0;           // homogeneous rows written as plain products (the last pass)
};

// Slice segments are the splat's for the replay slice; for a slice at other positions
// they carry those positions, with the same slot ranges.
struct SliceArgs {
    const Segment* segs;
    int nseg;
    uint32_t n_total;           // points of the batch (the record stride)
    LatticeConsts lc;
    uint4* key0;                // the shared hash-slot array
    uint4* keyn;
    uint32_t cap_total;
    const uint32_t* slot2vtx;   // parity dumps only
    const uint32_t* rec_slot;   // slots recorded by the splat, [r][n_total]; null: look up
    const float* rec_w_in;      // weights recorded by the splat, [r][n_total] (replay gather)
    const void* svals;          // filtered rows in slot space (float, or double)
    int vd;
    int* rec_vtx;               // optional (point, remainder) vertex indices (dumps)
    float* rec_w;               // optional weights
    unsigned* seg_status;
    uint32_t blocks;
};

// ---------------------------------------------------------------------------------
// point loading
// ---------------------------------------------------------------------------------
template <int D, int VDP>
__device__ __forceinline__ void load_point(const PointSource& s, uint32_t i, float (&p)[D],
                                           float (&v)[VDP]) {
    const uint32_t w = (uint32_t)s.width, h = (uint32_t)s.height;
    const uint32_t x = i % w;
    const uint32_t q = i / w;
    const uint32_t y = q % h;
    const uint32_t t = q / h;
    const long long off_p = (long long)t * s.pos.tstride + (long long)y * s.pos.ystride + x;
    int c = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        if (k < s.pos_channels) {
            p[k] = __fmul_rn(__ldg(s.pos.base + off_p + (long long)k * s.pos.cstride), s.pos_scale[k]);
        }
    }
    c = s.pos_channels;
    if (s.coord_mask & 1) { float f = __fmul_rn((float)x, s.coord_scale[0]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 2) { float f = __fmul_rn((float)y, s.coord_scale[1]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 4) { float f = __fmul_rn((float)t, s.coord_scale[2]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    const long long off_v = (long long)t * s.val.tstride + (long long)y * s.val.ystride + x;
#pragma unroll
    for (int k = 0; k < VDP; ++k) {
        float f = 0.0f;
        if (k < s.val_channels) f = __ldg(s.val.base + off_v + (long long)k * s.val.cstride);
        else if (k == s.val_channels && s.homogeneous) f = 1.0f;
        v[k] = f;
    }
}

template <int D>
__device__ __forceinline__ void load_position(const PointSource& s, uint32_t i, float (&p)[D]) {
    const uint32_t w = (uint32_t)s.width, h = (uint32_t)s.height;
    const uint32_t x = i % w;
    const uint32_t q = i / w;
    const uint32_t y = q % h;
    const uint32_t t = q / h;
    const long long off_p = (long long)t * s.pos.tstride + (long long)y * s.pos.ystride + x;
#pragma unroll
    for (int k = 0; k < D; ++k)
        if (k < s.pos_channels)
            p[k] = __fmul_rn(__ldg(s.pos.base + off_p + (long long)k * s.pos.cstride), s.pos_scale[k]);
    int c = s.pos_channels;
    if (s.coord_mask & 1) { float f = __fmul_rn((float)x, s.coord_scale[0]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 2) { float f = __fmul_rn((float)y, s.coord_scale[1]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 4) { float f = __fmul_rn((float)t, s.coord_scale[2]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
}

// positions of point (x, y, t) of a source, as load_position
template <int D>
__device__ __forceinline__ void load_position_xyt(const PointSource& s, uint32_t x, uint32_t y, uint32_t t,
                                                  float (&p)[D]) {
    const long long off_p = (long long)t * s.pos.tstride + (long long)y * s.pos.ystride + x;
#pragma unroll
    for (int k = 0; k < D; ++k)
        if (k < s.pos_channels)
            p[k] = __fmul_rn(__ldg(s.pos.base + off_p + (long long)k * s.pos.cstride), s.pos_scale[k]);
    int c = s.pos_channels;
    if (s.coord_mask & 1) { float f = __fmul_rn((float)x, s.coord_scale[0]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 2) { float f = __fmul_rn((float)y, s.coord_scale[1]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 4) { float f = __fmul_rn((float)t, s.coord_scale[2]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
}

// ---------------------------------------------------------------------------------
// accumulator rows
// ---------------------------------------------------------------------------------
template <int VDP>
__device__ __forceinline__ void atomic_add_row(float* dst, const float (&c)[VDP]) {
    if constexpr (VDP == 2) {
        atomicAdd(reinterpret_cast<float2*>(dst), make_float2(c[0], c[1]));
    } else {
#pragma unroll
        for (int k = 0; k < VDP; k += 4)
            atomicAdd(reinterpret_cast<float4*>(dst + k), make_float4(c[k], c[k + 1], c[k + 2], c[k + 3]));
    }
}
template <int VDP>
__device__ __forceinline__ void atomic_add_row(double* dst, const double (&c)[VDP]) {
#pragma unroll
    for (int k = 0; k < VDP; ++k) atomicAdd(dst + k, c[k]);
}

template <typename Acc> __device__ __forceinline__ Acc acc_mul(float a, float b);
template <> __device__ __forceinline__ float acc_mul<float>(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double acc_mul<double>(float a, float b) { return (double)a * (double)b; }
__device__ __forceinline__ float acc_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double acc_add(double a, double b) { return __dadd_rn(a, b); }

// ---------------------------------------------------------------------------------
// splat
// ---------------------------------------------------------------------------------
constexpr int kSplatThreads = 256;
// Tuning (measured on the 4K d=5 and d=3 bilaterals and the 2M-point d=16 transform): the
// splat is latency bound, so resident warps matter more than a few spilled registers —
// 6 blocks of 256 per SM up to d=5 (40 registers; 0.94 -> 0.77 ms at 4K d=5), 4 for d=6,
// fewer for the larger per-point state of higher d.  For 6 <= d <= PGPU_SPLAT_AHEAD_MAX_D
// the leaders issue the home-slot loads of all remainders before resolving any; up to
// d=5 the registers that takes cost more occupancy than the overlap gains.
#ifndef PGPU_SPLAT_AHEAD_MAX_D
#define PGPU_SPLAT_AHEAD_MAX_D 8
#endif
__host__ __device__ constexpr int splat_min_blocks(int d) { return d <= 5 ? 6 : d <= 6 ? 4 : d <= 8 ? 3 : 2; }

template <int D, int VDP, typename Acc>
__global__ void __launch_bounds__(kSplatThreads, splat_min_blocks(D)) splat_kernel(SplatArgs a) {
    constexpr int KW = key_words(D);
    // one-word keys of every remainder stay in shared memory for the leaders' inserts
    constexpr bool kKeysInSmem = KW == 1;
    __shared__ float s_delta[(D + 1) * kSplatThreads];
    __shared__ unsigned char s_coord[(D + 1) * kSplatThreads];
    __shared__ uint4 s_key[kKeysInSmem ? (D + 1) * kSplatThreads : 1];
    __shared__ uint32_t s_new[kBlockListCap];   // slots this block created
    __shared__ uint32_t s_new_count, s_new_base;
    __shared__ Segment sg;
    const int kseg = segment_by<&Segment::splat_base>(a.segs, a.nseg, blockIdx.x);
    if (threadIdx.x == 0) s_new_count = 0;
    load_segment(a.segs + kseg, sg);
    const BlockList blist{s_new, &s_new_count, &s_new_base};
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t i = (blockIdx.x - sg.splat_base) * (uint32_t)kSplatThreads + threadIdx.x;
    const bool valid = i < sg.n;
    const unsigned active = __ballot_sync(0xFFFFFFFFu, valid);
    if (valid) {
    unsigned* status = a.seg_status + kseg;
    const TableView table{a.key0 + sg.slot_base, a.keyn + sg.slot_base, sg.cap, a.cap_total};
    float p[D], v[VDP];
    load_point<D, VDP>(sg.src, i, p, v);
    Simplex<D> sx;
    const SimplexScratch scr{s_delta + threadIdx.x, s_coord + threadIdx.x, kSplatThreads};
    compute_simplex<D>(p, a.lc, sx, status, scr);
    const uint32_t gi = sg.point_base + i;   // point number in the batch
    const uint32_t e0 = gi * (uint32_t)(D + 1);
    Acc* vals = reinterpret_cast<Acc*>(a.vals) + (size_t)sg.slot_base * VDP;
    uint32_t* ft = a.ft ? a.ft + sg.slot_base : nullptr;

    // Phase 1: group the lanes that share each vertex key: lanes with equal hashes,
    // confirmed against the group leader's key (a hash collision inside the warp falls
    // back to matching all key words); each group's leader starts loading its home slot.  For d <= 8 the loads of all d+1
    // remainders are in flight together before any is needed.
    constexpr bool kAhead = D > 5 && D <= PGPU_SPLAT_AHEAD_MAX_D;
    unsigned peers[D + 1];
    uint32_t home[D + 1];
    uint4 first[D + 1];
    Key<KW> key;
    first_key<D>(sx, key);
#pragma unroll
    for (int r = 0; r <= D; ++r) {
        if (r > 0) key_step<D>(key, scr.coord[(D - (r - 1)) * scr.stride]);
        if (kKeysInSmem) s_key[r * kSplatThreads + threadIdx.x] = key.w[0];
        const uint32_t hk = key_hash<KW>(key);
        unsigned pr = __match_any_sync(active, hk);
        {
            const unsigned ld = __ffs(pr) - 1;
            bool same = true;
#pragma unroll
            for (int w = 0; w < KW; ++w) {
                same &= __shfl_sync(active, key.w[w].x, ld) == key.w[w].x;
                same &= __shfl_sync(active, key.w[w].y, ld) == key.w[w].y;
                same &= __shfl_sync(active, key.w[w].z, ld) == key.w[w].z;
                same &= __shfl_sync(active, key.w[w].w, ld) == key.w[w].w;
            }
            if (!__all_sync(active, same)) {
                pr = active;
#pragma unroll
                for (int w = 0; w < KW; ++w) {
                    pr &= __match_any_sync(active, ((unsigned long long)key.w[w].y << 32) | key.w[w].x);
                    pr &= __match_any_sync(active, ((unsigned long long)key.w[w].w << 32) | key.w[w].z);
                }
            }
        }
        peers[r] = pr;
        home[r] = home_slot(hk, table.cap);
        first[r] = make_uint4(0u, 0u, 0u, 0u);
        if (kAhead && lane == (unsigned)(__ffs(pr) - 1)) first[r] = __ldcg(&table.key0[home[r]]);
    }

    // Phase 2: per remainder, the group's leader finds or inserts the vertex and records
    // the first touch (a fire-and-forget atomicMin: the leader's entry is the group's
    // smallest); every lane then adds its own weighted values with one vector atomic.
    // Summing a group in registers first does not pay here: the lanes of a vertex are
    // rarely a run (on the 4K d=5 bilateral every warp has a vertex split over several
    // runs), and gathering them costs more instructions than the L2 atomics it saves.
    // Every lane records the slot for the slice.
#pragma unroll
    for (int r = 0; r <= D; ++r) {
        const unsigned pr = peers[r];
        const unsigned leader = __ffs(pr) - 1;
        Acc c[VDP];
#pragma unroll
        for (int k = 0; k < VDP; ++k) c[k] = acc_mul<Acc>(sx.bary[r], v[k]);
        int s = -1;
        if (lane == leader) {
            Key<KW> kr;
            if constexpr (kKeysInSmem) {
                kr.w[0] = s_key[r * kSplatThreads + threadIdx.x];
            } else {
                int kc[D];
                vertex_coords<D>(sx, r, kc);
                pack_key<D>(kc, kr);
            }
            const uint4 w0 = kAhead ? first[r] : __ldcg(&table.key0[home[r]]);
            bool created = false;
            s = table_insert<KW>(table, kr, home[r], w0, status, &created);
            if (s >= 0 && ft) atomicMin(&ft[s], e0 + (uint32_t)r);
            if (created && a.vlist) block_list_append(blist, a, kseg, sg.slot_base + (uint32_t)s);
        }
        s = __shfl_sync(active, s, leader);
        if (s >= 0) atomic_add_row<VDP>(vals + (size_t)s * VDP, c);
        if (a.rec_slot)
            a.rec_slot[(size_t)r * a.n_total + gi] = s >= 0 ? sg.slot_base + (uint32_t)s : 0xFFFFFFFFu;
        if (a.rec_w) a.rec_w[(size_t)r * a.n_total + gi] = sx.bary[r];
    }
    }
    if (!a.vlist) return;
    __syncthreads();
    block_list_flush(blist, a, kseg);
}

// ---------------------------------------------------------------------------------
// tile splat: one block per 2D tile of kTilePixels pixels of one frame
// ---------------------------------------------------------------------------------
// Neighbouring pixels land on the same lattice vertices (on the 4K d=5 bilateral a 16x16
// tile's 1536 (point, remainder) entries touch about 155 distinct vertices), while the
// direct splat pays one dependent probe of the global table, a trip to L2 or DRAM, per
// lane group.  The tile splat resolves every entry's key in a hash table of the block's
// own in shared memory instead (phase A), inserts each distinct vertex of the tile into
// the global table once (phase B), and then every lane adds its rows to the global slots
// with fire-and-forget vector reductions and writes its replay record (phase C).  A local
// slot's first touch is the smallest entry that reached it, so the global minimum over
// tiles is the reference's first insertion; the vertex set, keys and records equal the
// direct splat's, only the order of the FP32 additions differs.  An entry whose probe finds
// no free local slot within kTileProbe goes to the global table directly, so no tile can
// overflow.  One-word keys (d <= 7), FP32 accumulators.
constexpr int kTileThreads = 256;
constexpr int kTilePixels = 256;        // one pixel per thread
constexpr int kTileSlots = 1024;        // shared-memory hash slots per block
constexpr int kTileProbe = 64;
#ifndef PGPU_TILE_MIN_BLOCKS_D5
#define PGPU_TILE_MIN_BLOCKS_D5 5
#endif
__host__ __device__ constexpr int tile_min_blocks(int d) {
    return d <= 5 ? PGPU_TILE_MIN_BLOCKS_D5 : d <= 6 ? 4 : 3;
}

// dynamic shared memory of a tile splat block: keys, first touches (then global slots),
// the list of occupied slots, the slots the block creates, and the simplex scratch.  (The
// rows are not summed in shared memory: float atomics there are compare-and-swap loops,
// and a variant that summed each tile's rows before one global reduction per vertex took
// 2.1 ms per 4K frame against 0.73 ms.)
__host__ __device__ constexpr size_t tile_smem_bytes(int d, int vdp) {
    return (size_t)kTileSlots * 16 + (size_t)kTileSlots * 4 + (size_t)kTileSlots * 2 +
           (size_t)kBlockListCap * 4 + (size_t)kBlockListCap * 2 + (size_t)(d + 1) * kTileThreads * 4 +
           (size_t)(d + 1) * kTileThreads + 16 + 0 * (size_t)vdp;
}

// Home slot of a one-word key in a block's table: a cheap multiplicative mix of the three
// 32-bit words that carry coordinates 0..5 and the low half of the fourth (coordinate 6);
// the table is small and probing resolves its collisions, so the global hash (a 64-bit
// mix) is computed only once per distinct vertex, in phase B.
__device__ __forceinline__ uint32_t tile_home(const uint4& k) {
    const uint32_t h = k.x * 0x9E3779B1u + k.y * 0x85EBCA77u + k.z * 0xC2B2AE3Du + (k.w & 0xFFFFu) * 0x27D4EB2Fu;
    return (h ^ (h >> 15)) * 0x2C1B3C6Du >> (32 - 10);
}

// find-or-insert of a one-word key in the block's table; a new key's slot is appended to
// the block's list of occupied slots.  -1 when no slot within the probe limit is free (the
// caller then uses the global table).
__device__ __forceinline__ int tile_insert(uint4* t_key, uint16_t* t_list, uint32_t* t_count,
                                           const uint4& k) {
    const uint4 empty = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
    static_assert(kTileSlots == 1024, "the home slot has 10 bits");
    uint32_t l = tile_home(k);
#pragma unroll 1
    for (int probe = 0; probe < kTileProbe; ++probe) {
        uint4 w = t_key[l];
        if (is_empty_word(w)) {
            w = atomicCAS_block(&t_key[l], empty, k);
            if (is_empty_word(w)) {
                t_list[atomicAdd(t_count, 1u)] = (uint16_t)l;
                return (int)l;
            }
        }
        if (words_equal(w, k)) return (int)l;
        l = (l + 1) & (kTileSlots - 1);
    }
    return -1;
}

// point (x, y, t) of a source: positions and values as load_point
template <int D, int VDP>
__device__ __forceinline__ void load_point_xyt(const PointSource& s, uint32_t x, uint32_t y, uint32_t t,
                                               float (&p)[D], float (&v)[VDP]) {
    const long long off_v = (long long)t * s.val.tstride + (long long)y * s.val.ystride + x;
    if (s.pos_is_val) {   // one load per channel: the bilateral's guide is its image
#pragma unroll
        for (int k = 0; k < VDP; ++k) {
            float f = 0.0f;
            if (k < s.val_channels) f = __ldg(s.val.base + off_v + (long long)k * s.val.cstride);
            else if (k == s.val_channels && s.homogeneous) f = 1.0f;
            v[k] = f;
        }
#pragma unroll
        for (int k = 0; k < D && k < VDP; ++k)
            if (k < s.pos_channels) p[k] = __fmul_rn(v[k], s.pos_scale[k]);
    } else {
        const long long off_p = (long long)t * s.pos.tstride + (long long)y * s.pos.ystride + x;
#pragma unroll
        for (int k = 0; k < D; ++k)
            if (k < s.pos_channels)
                p[k] = __fmul_rn(__ldg(s.pos.base + off_p + (long long)k * s.pos.cstride), s.pos_scale[k]);
#pragma unroll
        for (int k = 0; k < VDP; ++k) {
            float f = 0.0f;
            if (k < s.val_channels) f = __ldg(s.val.base + off_v + (long long)k * s.val.cstride);
            else if (k == s.val_channels && s.homogeneous) f = 1.0f;
            v[k] = f;
        }
    }
    int c = s.pos_channels;
    if (s.coord_mask & 1) { float f = __fmul_rn((float)x, s.coord_scale[0]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 2) { float f = __fmul_rn((float)y, s.coord_scale[1]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
    if (s.coord_mask & 4) { float f = __fmul_rn((float)t, s.coord_scale[2]);
#pragma unroll
        for (int k = 0; k < D; ++k) if (k == c) p[k] = f;
        ++c; }
}

// Vertex v, created by this block in global slot s (batch numbering): its key and slot in
// vertex order (read by later kernels), then its index in the key word, which tells other
// blocks the vertex's number.  The rows were zeroed before the launch, so no fence is
// needed between the two: nothing a reader does with v depends on the creator's stores.
template <int VDP>
__device__ __forceinline__ void publish_vertex(const SplatArgs& a, uint32_t s, uint32_t v, uint4 key) {
    key.w = 0x00008000u;   // lane 6 = coordinate 0 (none for d <= 6), lane 7 = ready state
    a.vkey0[v] = key;
    a.vtx2slot[v] = s;
    if (a.nbr_init)
        for (int j = 0; j < a.nbr_axes; ++j) a.nbr_init[(size_t)j * a.nbr_stride + v] = make_int2(-1, -1);
    __stcg(reinterpret_cast<unsigned*>(a.key0 + s) + 3, enc_index(v));
}

// A vertex this block created in global slot gs (local slot l, or 0xFFFF for one placed in
// the global table directly): onto the block's list, numbered and published by the flush;
// when the list is full, numbered and published at once (returns its number then, else
// 0xFFFFFFFF).
template <int VDP>
__device__ __forceinline__ uint32_t list_new_vertex(const SplatArgs& a, int kseg, uint32_t* s_new,
                                                    uint16_t* s_new_l, uint32_t* s_new_count,
                                                    uint32_t gs, uint16_t l, const uint4& key) {
    const uint32_t jj = atomicAdd(s_new_count, 1u);
    if (jj < kBlockListCap) {
        s_new[jj] = gs;
        s_new_l[jj] = l;
        return 0xFFFFFFFFu;
    }
    const uint32_t v = atomicAdd(a.vcount, 1u);
    atomicAdd(a.seg_counts + kseg, 1u);
    publish_vertex<VDP>(a, gs, v, key);
    return v;
}

// t_ft marker of a vertex the block created and numbers in its flush (never a vertex index:
// indices stay below the 2^31 - 256 slots of a batch)
constexpr uint32_t kOwnPending = 0x7FFFFFFFu;

// the vertex index of global slot s, created by another block: wait (bounded) until its
// creator has published it, which takes the creator's global inserts and one atomic
// (microseconds); 0xFFFFFFFF with the spin-limit status bit if it is not published within
// kAwaitSpin polls, or at once when another wait of the lattice has given up already
constexpr int kAwaitSpin = 1 << 14;
__device__ __forceinline__ uint32_t await_vertex(const SplatArgs& a, uint32_t s, unsigned* status) {
    const unsigned* w = reinterpret_cast<const unsigned*>(a.key0 + s) + 3;
    for (int spin = 0; spin < kAwaitSpin; ++spin) {
        const unsigned x = __ldcg(w);
        if (has_index(x)) return dec_index(x);
        if ((spin & 63) == 63 && (__ldcg(status) & kStatusSpinLimit)) return 0xFFFFFFFFu;
        __nanosleep(64);
    }
    atomicOr(status, kStatusSpinLimit);
    return 0xFFFFFFFFu;
}

// One (point, remainder) entry of the tile splat's phase C: its weighted row into row s
// (VROWS: vertex s; otherwise segment slot s; 0xFFFFFFFF: not placed) and its record.
template <int D, int VDP, bool VROWS>
__device__ __forceinline__ void splat_entry(const SplatArgs& a, float* vals, uint32_t slot_base, uint32_t gi,
                                            int r, uint32_t s, float w, const float (&v)[VDP]) {
    if (s != 0xFFFFFFFFu) {
        float c[VDP];
#pragma unroll
        for (int q = 0; q < VDP; ++q) c[q] = __fmul_rn(w, v[q]);
        atomic_add_row<VDP>(vals + (size_t)s * VDP, c);
    }
    if (a.rec_slot)
        a.rec_slot[(size_t)r * a.n_total + gi] = s == 0xFFFFFFFFu ? 0xFFFFFFFFu : VROWS ? s : slot_base + s;
    if (a.rec_w) a.rec_w[(size_t)r * a.n_total + gi] = w;
}

// VROWS: number vertices as they are created and accumulate into vertex-ordered rows (the
// SplatArgs::vrows protocol, d <= 6, no first touches); otherwise rows in slot space.
template <int D, int VDP, bool VROWS>
__global__ void __launch_bounds__(kTileThreads, tile_min_blocks(D)) splat_tile_kernel(SplatArgs a) {
    static_assert(key_words(D) == 1, "the tile splat handles one-word keys (d <= 7)");
    static_assert(!VROWS || index_in_key(D), "vertex-ordered rows publish the index in the key word");
    extern __shared__ __align__(16) unsigned char tile_smem[];
    uint4* t_key = reinterpret_cast<uint4*>(tile_smem);
    uint32_t* t_ft = reinterpret_cast<uint32_t*>(t_key + kTileSlots);
    uint16_t* t_list = reinterpret_cast<uint16_t*>(t_ft + kTileSlots);
    uint32_t* s_new = reinterpret_cast<uint32_t*>(t_list + kTileSlots);
    uint16_t* s_new_l = reinterpret_cast<uint16_t*>(s_new + kBlockListCap);
    float* s_delta = reinterpret_cast<float*>(s_new_l + kBlockListCap);
    unsigned char* s_coord = reinterpret_cast<unsigned char*>(s_delta + (D + 1) * kTileThreads);
    __shared__ Segment sg;
    __shared__ uint32_t t_count, s_new_count, s_new_base;
    const int kseg = segment_by<&Segment::tile_base>(a.segs, a.nseg, blockIdx.x);
    for (int l = threadIdx.x; l < kTileSlots; l += kTileThreads) {
        t_key[l] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        t_ft[l] = 0xFFFFFFFFu;
    }
    if (threadIdx.x == 0) t_count = 0, s_new_count = 0;
    load_segment(a.segs + kseg, sg);   // ends with a barrier
    const BlockList blist{s_new, &s_new_count, &s_new_base};

    unsigned* status = a.seg_status + kseg;
    const TableView table{a.key0 + sg.slot_base, a.keyn + sg.slot_base, sg.cap, a.cap_total};
    float* vals = VROWS ? reinterpret_cast<float*>(a.vrows)
                        : reinterpret_cast<float*>(a.vals) + (size_t)sg.slot_base * VDP;
    uint32_t* ft = (!VROWS && a.ft) ? a.ft + sg.slot_base : nullptr;
    const uint32_t b = blockIdx.x - sg.tile_base;
    const uint32_t per_frame = sg.tiles_x * sg.tiles_y;
    const uint32_t f = b / per_frame, bt = b - f * per_frame;
    const uint32_t ty = bt / sg.tiles_x, tx = bt - ty * sg.tiles_x;
    const uint32_t px = tx * sg.tile_w + threadIdx.x % sg.tile_w;
    const uint32_t py = ty * sg.tile_h + threadIdx.x / sg.tile_w;
    const uint32_t W = (uint32_t)sg.src.width, H = (uint32_t)sg.src.height;
    const bool valid = px < W && py < H;
    const SimplexScratch scr{s_delta + threadIdx.x, s_coord + threadIdx.x, kTileThreads};

    // Phase A: this pixel's simplex and the local slot of each of its d+1 vertices.
    // loc[r] >= 0: local slot; -1: not placed; <= -2: global slot -(loc + 2), taken directly
    // because the local table was full around the key.
    float v[VDP];
    float bary[D + 1];
    int loc[D + 1];
    uint32_t gi = 0;
#pragma unroll
    for (int r = 0; r <= D; ++r) loc[r] = -1;
    if (valid) {
        float pp[D];
        load_point_xyt<D, VDP>(sg.src, px, py, f, pp, v);
        Simplex<D> sx;
        compute_simplex<D>(pp, a.lc, sx, status, scr);
        gi = sg.point_base + (f * H + py) * W + px;
        const uint32_t e0 = gi * (uint32_t)(D + 1);
        Key<1> key;
        first_key<D>(sx, key);
#pragma unroll
        for (int r = 0; r <= D; ++r) {
            if (r > 0) key_step<D>(key, scr.coord[(D - (r - 1)) * scr.stride]);
            bary[r] = sx.bary[r];
            const int l = tile_insert(t_key, t_list, &t_count, key.w[0]);
            if (l >= 0) {
                if (ft) atomicMin(&t_ft[l], e0 + (uint32_t)r);
                loc[r] = l;
            } else {
                const uint32_t home = home_slot(key_hash<1>(key), table.cap);
                bool created = false;
                const int s = table_insert<1, VROWS>(table, key, home, __ldcg(&table.key0[home]), status, &created);
                if (s >= 0) {
                    if constexpr (VROWS) {
                        // numbered by the flush (phase C reads the number from the key word)
                        if (created)
                            list_new_vertex<VDP>(a, kseg, s_new, s_new_l, &s_new_count,
                                                 sg.slot_base + (uint32_t)s, 0xFFFFu, key.w[0]);
                        loc[r] = -(s + 2);
                    } else {
                        if (ft) atomicMin(&ft[s], e0 + (uint32_t)r);
                        if (created && a.vlist) block_list_append(blist, a, kseg, sg.slot_base + (uint32_t)s);
                        loc[r] = -(s + 2);
                    }
                }
            }
        }
    }
    __syncthreads();

    // Phase B: each distinct vertex of the tile (the list of occupied local slots) into the
    // global table once
    const uint32_t count = t_count;
#pragma unroll 1
    for (uint32_t j = threadIdx.x; j < count; j += kTileThreads) {
        const int l = t_list[j];
        Key<1> kk;
        kk.w[0] = t_key[l];
        const uint32_t h = home_slot(key_hash<1>(kk), table.cap);
        bool created = false;
        uint4 seen = make_uint4(0u, 0u, 0u, 0u);
        const int s = table_insert<1, VROWS>(table, kk, h, __ldcg(&table.key0[h]), status, &created, &seen);
        if constexpr (VROWS) {
            // t_ft[l]: the vertex index; kOwnPending for a vertex this block numbers in its
            // flush; 0x80000000 | global slot while another block's vertex is not numbered
            uint32_t val = 0xFFFFFFFFu;
            if (s >= 0) {
                const uint32_t gs = sg.slot_base + (uint32_t)s;
                val = 0x80000000u | gs;
                if (created) {
                    const uint32_t vv = list_new_vertex<VDP>(a, kseg, s_new, s_new_l, &s_new_count, gs,
                                                             (uint16_t)l, kk.w[0]);
                    val = vv != 0xFFFFFFFFu ? vv : kOwnPending;
                } else if (has_index(seen.w)) {
                    val = dec_index(seen.w);
                }
            }
            t_ft[l] = val;
        } else {
            if (s >= 0 && ft) atomicMin(&ft[s], t_ft[l]);
            if (created && a.vlist) block_list_append(blist, a, kseg, sg.slot_base + (uint32_t)s);
            t_ft[l] = s >= 0 ? (uint32_t)s : 0xFFFFFFFFu;   // now the global slot (segment-relative)
        }
    }
    __syncthreads();
    if constexpr (VROWS) {
        // number the block's new vertices with one atomic and publish them; in the same
        // pass, learn (once per vertex) the numbers of the tile's vertices other blocks
        // created, which is faster than every lane waiting for its own entries in phase C
        const uint32_t n = min(s_new_count, kBlockListCap);
        if (n) {
            if (threadIdx.x == 0) {
                s_new_base = atomicAdd(a.vcount, n);
                atomicAdd(a.seg_counts + kseg, n);
            }
            __syncthreads();
        }
        const uint32_t base = s_new_base;
        for (uint32_t jj = threadIdx.x; jj < n; jj += kTileThreads) {
            const int l = s_new_l[jj];
            if (l != 0xFFFF) {
                publish_vertex<VDP>(a, s_new[jj], base + jj, t_key[l]);
                t_ft[l] = base + jj;
            } else {   // placed in the global table directly in phase A
                publish_vertex<VDP>(a, s_new[jj], base + jj, __ldcg(&a.key0[s_new[jj]]));
            }
        }
#pragma unroll 1
        for (uint32_t j = threadIdx.x; j < count; j += kTileThreads) {
            const int l = t_list[j];
            const uint32_t val = t_ft[l];
            if (val != 0xFFFFFFFFu && (val & 0x80000000u)) t_ft[l] = await_vertex(a, val & 0x7FFFFFFFu, status);
        }
        __syncthreads();
    } else {
        if (a.vlist) block_list_flush(blist, a, kseg);
    }

    // Phase C: every lane's rows into its vertices' global rows, and the replay record
    if (!valid) return;
#pragma unroll
    for (int r = 0; r <= D; ++r) {
        const int l = loc[r];
        uint32_t s;
        if (l >= 0) {
            s = t_ft[l];
        } else if (l <= -2) {
            s = (uint32_t)(-(l + 2));
            if constexpr (VROWS) s = await_vertex(a, sg.slot_base + s, status);
        } else {
            s = 0xFFFFFFFFu;
        }
        splat_entry<D, VDP, VROWS>(a, vals, sg.slot_base, gi, r, s, bary[r], v);
    }
}

// ---------------------------------------------------------------------------------
// compaction
// ---------------------------------------------------------------------------------
__global__ void mark_kernel(const uint32_t* __restrict__ ft, uint32_t cap, uint32_t* bitmap);

// exclusive prefix popcount over the bitmap words, three phases
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;    // words per thread
__global__ void scan_reduce_kernel(const uint32_t* __restrict__ bitmap, uint32_t nwords,
                                   uint32_t* partials);
__global__ void scan_partials_kernel(uint32_t* partials, uint32_t nparts, uint32_t* total);
__global__ void scan_down_kernel(const uint32_t* __restrict__ bitmap, uint32_t nwords,
                                 const uint32_t* __restrict__ partials, uint32_t* offs);

// HOMOG: the last value channel (index wc) is the homogeneous weight w; the vertex row is
// stored as (v_0/w, ..., v_{wc-1}/w, w) — homogeneous coordinates normalised by their own
// weight.  A filtered value is then a convex combination of stored values, so a 16-bit
// payload's rounding of w enters the normalised output only at second order.
template <int KW>
__device__ __forceinline__ void write_tag(const CompactArgs& a, uint32_t s) {
    Key<KW> k;
    k.w[0] = a.table.key0[s];
#pragma unroll
    for (int i = 1; i < KW; ++i) k.w[i] = a.table.keyn[(size_t)(i - 1) * a.table.stride + s];
    a.tags[s] = slot_tag(key_hash<KW>(k));
}

// vertex `vtx` of slot s: the index maps, its key and its row in vertex order
template <int KW, int VDP, typename Acc, typename P, bool HOMOG>
__device__ __forceinline__ void assign_vertex(const CompactArgs& a, uint32_t s, uint32_t vtx) {
    const Acc* tvals = reinterpret_cast<const Acc*>(a.tvals);
    P* vvals = reinterpret_cast<P*>(a.vvals);
    a.slot2vtx[s] = vtx;
    a.vtx2slot[vtx] = s;
    if (a.nbr_init)
        for (int j = 0; j < a.nbr_axes; ++j) a.nbr_init[(size_t)j * a.nbr_stride + vtx] = make_int2(-1, -1);
    const uint4 k0 = a.table.key0[s];
    a.vkey0[vtx] = k0;
    if (KW == 1 && a.index_in_key) a.table.key0[s] = make_uint4(k0.x, k0.y, k0.z, enc_index(vtx));
#pragma unroll
    for (int k = 1; k < KW; ++k)
        a.vkeyn[(size_t)(k - 1) * a.vcap + vtx] = a.table.keyn[(size_t)(k - 1) * a.table.stride + s];
    if (a.tags) write_tag<KW>(a, s);
    if constexpr (HOMOG) {
        Acc wt = tvals[(size_t)s * VDP];
#pragma unroll
        for (int k = 0; k < VDP; ++k) if (k == a.wc) wt = tvals[(size_t)s * VDP + k];
#pragma unroll
        for (int k = 0; k < VDP; ++k) {
            const Acc t = tvals[(size_t)s * VDP + k];
            const Acc m = (k == a.wc) ? wt : (k < a.wc && wt != (Acc)0) ? t / wt : (Acc)0;
            Payload<P>::store(vvals + (size_t)vtx * VDP + k, m);
        }
    } else {
#pragma unroll
        for (int k = 0; k < VDP; ++k)
            Payload<P>::store(vvals + (size_t)vtx * VDP + k, tvals[(size_t)s * VDP + k]);
    }
}

// Vertices in the reference's order (parity dumps): every occupied slot's index is the
// rank of its first touch among all first touches (the bitmap's prefix popcount).
template <int KW, int VDP, typename Acc, typename P, bool HOMOG>
__global__ void assign_kernel(CompactArgs a) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < a.table.cap;
         s += gridDim.x * blockDim.x) {
        const uint32_t f = a.ft[s];
        if (f == 0xFFFFFFFFu) continue;
        const uint32_t w = f >> 5;
        const uint32_t vtx = a.offs[w] + __popc(a.bitmap[w] & ((1u << (f & 31u)) - 1u));
        assign_vertex<KW, VDP, Acc, P, HOMOG>(a, s, vtx);
    }
}

// Vertices in the order the splat created them (its vertex list): the filtered values do
// not depend on how vertices are numbered, so lattices that need no dump skip the
// first-touch bookkeeping; the list keeps tiles' vertices together, as the reference's
// first-insertion order keeps a scanline's.
template <int KW, int VDP, typename Acc, typename P, bool HOMOG>
__global__ void assign_list_kernel(CompactArgs a) {
    const uint32_t m = *a.nverts;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x)
        assign_vertex<KW, VDP, Acc, P, HOMOG>(a, __ldg(a.vlist + v), v);
}

// ---------------------------------------------------------------------------------
// neighbours: n1 = key + 1 except n1[j] = key[j] - d; n2 = key - 1 except n2[j] = key[j] + d
// (for j == d every stored coordinate moves by one), src/Permutohedral.h:446-451.
// Both are formed in packed form: stored lanes are int16 + 0x8000 mod 2^16, so adding a
// per-lane 16-bit step (__vadd2) wraps exactly like the reference's short keys.
// ---------------------------------------------------------------------------------
// the packed step of axis j (sign +1: n1, -1: n2) for word w of a d-dimensional key
template <int D>
__device__ __forceinline__ uint32_t axis_step(int j, int sign, int w, int h) {
    uint32_t inc = 0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int lane = 2 * h + half;
        const int c = w == 0 ? lane : 7 + (w - 1) * 8 + lane;   // coordinate in this lane
        const bool stored = (w == 0 ? lane < 7 : true) && c < D;
        if (stored) {
            const int step = sign * ((c == j) ? -D : 1);
            inc |= ((uint32_t)(uint16_t)step) << (16 * half);
        }
    }
    return inc;
}

template <int D>
__device__ __forceinline__ void neighbour_key(const Key<key_words(D)>& k, int j, int sign,
                                              Key<key_words(D)>& out) {
    constexpr int KW = key_words(D);
#pragma unroll
    for (int w = 0; w < KW; ++w) {
        uint4 q = k.w[w];
        if (w == 0) q.w &= 0xFFFFu;   // a clean state lane (it may hold the vertex index)
        out.w[w].x = __vadd2(q.x, axis_step<D>(j, sign, w, 0));
        out.w[w].y = __vadd2(q.y, axis_step<D>(j, sign, w, 1));
        out.w[w].z = __vadd2(q.z, axis_step<D>(j, sign, w, 2));
        out.w[w].w = __vadd2(q.w, axis_step<D>(j, sign, w, 3));
    }
}

template <int D>
__device__ __forceinline__ int neighbour_index(const NbrArgs& a, const TableView& table, uint32_t base,
                                               const Key<key_words(D)>& k) {
    constexpr int KW = key_words(D);
    const uint32_t h = key_hash<KW>(k);
    if constexpr (index_in_key(D)) {
        return table_find_index<D>(table, k, h);
    } else {
        // tagged lookups exist for multi-word keys only (the host sets tags for those)
        const int s = (KW > 1 && a.tags) ? table_find_tagged<KW>(table, a.tags + base, k, h)
                                         : table_find<D>(table, k, h);
        return s >= 0 ? (int)__ldg(a.slot2vtx + base + s) : -1;
    }
}

template <int D>
__global__ void neighbours_kernel(NbrArgs a) {
    constexpr int KW = key_words(D);
    const uint32_t m = *a.nverts;
    for (uint32_t vtx = blockIdx.x * blockDim.x + threadIdx.x; vtx < m;
         vtx += gridDim.x * blockDim.x) {
        // neighbours are looked up in the vertex's own lattice only
        const int kseg = a.nseg > 1 ? segment_of_slot(a.seg_slot_base, a.nseg, __ldg(a.vtx2slot + vtx)) : 0;
        // a lattice whose splat overflowed is rerun by the host: its full table would make
        // every lookup of an absent key probe to the limit, so skip it
        if (a.seg_status && (__ldcg(a.seg_status + kseg) & (kStatusProbeLimit | kStatusSpinLimit))) {
            if (!a.half)
                for (int j = 0; j <= D; ++j) a.nbr[(size_t)j * a.vcap + vtx] = make_int2(-1, -1);
            continue;
        }
        if (a.norm_rows) {   // m = sum / w, 0 where w is 0 (the compaction's arithmetic)
            float* r = a.norm_rows + (size_t)vtx * a.vdp;
            const float w = r[a.wc];
            for (int k = 0; k < a.wc; ++k) r[k] = w != 0.0f ? r[k] / w : 0.0f;
            for (int k = a.wc + 1; k < a.vdp; ++k) r[k] = 0.0f;
        }
        const uint32_t base = __ldg(a.seg_slot_base + kseg);
        const TableView table{a.key0 + base, a.keyn + base, __ldg(a.seg_slot_base + kseg + 1) - base,
                              a.cap_total};
        Key<KW> key;
        key.w[0] = a.vkey0[vtx];
#pragma unroll
        for (int k = 1; k < KW; ++k) key.w[k] = a.vkeyn[(size_t)(k - 1) * a.vcap + vtx];
        if (a.half) {
            // n1 only: the key one step up along axis j; its vertex u has n2(u) = vtx
            // (axes unrolled for one-word keys, rolled for multi-word keys as below)
#pragma unroll (KW == 1 ? D + 1 : 1)
            for (int j = 0; j <= D; ++j) {
                Key<KW> k1;
                neighbour_key<D>(key, j, +1, k1);
                const int u1 = neighbour_index<D>(a, table, base, k1);
                int* pair = reinterpret_cast<int*>(a.nbr + (size_t)j * a.vcap);
                pair[2 * (size_t)vtx] = u1;
                if (u1 >= 0) pair[2 * (size_t)u1 + 1] = (int)vtx;
            }
            continue;
        }
        // one-word keys: the axes unrolled, so each axis's packed step is a constant;
        // multi-word keys: rolled (d=16, 2M points: 46.7 ms unrolled, 20.5 ms rolled)
#pragma unroll (KW == 1 ? D + 1 : 1)
        for (int j = 0; j <= D; ++j) {
            Key<KW> k1, k2;
            neighbour_key<D>(key, j, +1, k1);
            neighbour_key<D>(key, j, -1, k2);
            const int u1 = neighbour_index<D>(a, table, base, k1);
            const int u2 = neighbour_index<D>(a, table, base, k2);
            a.nbr[(size_t)j * a.vcap + vtx] = make_int2(u1, u2);
        }
    }
}

// ---------------------------------------------------------------------------------
// blur along one axis: new = 0.25*v(n1) + 0.5*old + 0.25*v(n2), absent neighbour = 0
// ---------------------------------------------------------------------------------
template <typename Acc> struct AccOf;   // arithmetic type of a payload
template <> struct AccOf<float> { using T = float; };
template <> struct AccOf<__half> { using T = float; };
template <> struct AccOf<__nv_bfloat16> { using T = float; };
template <> struct AccOf<double> { using T = double; };

__device__ __forceinline__ float blur3(float a, float b, float c) {
    return __fadd_rn(__fadd_rn(__fmul_rn(0.25f, a), __fmul_rn(0.5f, b)), __fmul_rn(0.25f, c));
}
__device__ __forceinline__ double blur3(double a, double b, double c) {
    return __dadd_rn(__dadd_rn(0.25 * a, 0.5 * b), 0.25 * c);
}

// Row of vertex u (zeros for an absent vertex, u < 0), in arithmetic type A.
template <int VDP, typename PS, typename A>
__device__ __forceinline__ void load_row(const PS* src, int u, A (&r)[VDP]) {
    // rows of 4 are read as one vector; an absent vertex (u < 0) reads vertex 0's row,
    // which exists whenever any vertex does, and is then replaced by zeros
    const size_t base = (size_t)(u >= 0 ? u : 0) * VDP;
    if constexpr (std::is_same<PS, float>::value && VDP % 4 == 0) {
#pragma unroll
        for (int k = 0; k < VDP; k += 4) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(src + base + k));
            r[k] = (A)q.x, r[k + 1] = (A)q.y, r[k + 2] = (A)q.z, r[k + 3] = (A)q.w;
        }
    } else if constexpr ((std::is_same<PS, __half>::value || std::is_same<PS, __nv_bfloat16>::value) &&
                         VDP % 4 == 0) {
#pragma unroll
        for (int k = 0; k < VDP; k += 4) {
            const uint2 q = __ldg(reinterpret_cast<const uint2*>(src + base + k));
            const PS* h = reinterpret_cast<const PS*>(&q);
#pragma unroll
            for (int j = 0; j < 4; ++j) r[k + j] = (A)Payload<PS>::load(h + j);
        }
    } else {
#pragma unroll
        for (int k = 0; k < VDP; ++k) r[k] = (A)Payload<PS>::load(src + base + k);
    }
    if (u < 0) {
#pragma unroll
        for (int k = 0; k < VDP; ++k) r[k] = (A)0;
    }
}

template <int VDP, typename PD, typename A>
__device__ __forceinline__ void store_row(PD* dst, size_t row, const A (&r)[VDP]) {
    if constexpr (std::is_same<PD, float>::value && VDP % 4 == 0) {
#pragma unroll
        for (int k = 0; k < VDP; k += 4)
            *reinterpret_cast<float4*>(dst + row * VDP + k) =
                make_float4((float)r[k], (float)r[k + 1], (float)r[k + 2], (float)r[k + 3]);
    } else if constexpr ((std::is_same<PD, __half>::value || std::is_same<PD, __nv_bfloat16>::value) &&
                         VDP % 4 == 0) {
#pragma unroll
        for (int k = 0; k < VDP; k += 4) {
            uint2 q;
            PD* h = reinterpret_cast<PD*>(&q);
#pragma unroll
            for (int j = 0; j < 4; ++j) Payload<PD>::store(h + j, (float)r[k + j]);
            *reinterpret_cast<uint2*>(dst + row * VDP + k) = q;
        }
    } else {
#pragma unroll
        for (int k = 0; k < VDP; ++k) Payload<PD>::store(dst + row * VDP + k, r[k]);
    }
}

// [1 2 1]/4 of three rows.  Homogeneous rows (m_0..m_{wc-1}, w): blur w and the products
// w*m, then renormalise, which is the same linear filter in homogeneous coordinates.
template <int VDP, typename A, bool HOMOG>
__device__ __forceinline__ void combine3(const A (&r1)[VDP], const A (&r0)[VDP], const A (&r2)[VDP],
                                         int wc, A (&out)[VDP]) {
    if constexpr (HOMOG) {
        A w1 = r1[0], w0 = r0[0], w2 = r2[0];
#pragma unroll
        for (int k = 0; k < VDP; ++k)
            if (k == wc) { w1 = r1[k]; w0 = r0[k]; w2 = r2[k]; }
        const A nw = blur3(w1, w0, w2);
        const A inv = nw != (A)0 ? (A)1 / nw : (A)0;
#pragma unroll
        for (int k = 0; k < VDP; ++k) {
            if (k == wc) out[k] = nw;
            else if (k < wc) out[k] = blur3(w1 * r1[k], w0 * r0[k], w2 * r2[k]) * inv;
            else out[k] = (A)0;
        }
    } else {
#pragma unroll
        for (int k = 0; k < VDP; ++k) out[k] = blur3(r1[k], r0[k], r2[k]);
    }
}

// the first-axis blur at vertex u (zeros when u is absent)
template <int VDP, typename PS, typename A, bool HOMOG>
__device__ __forceinline__ void blurred_row(const PS* src, const int2* nbr, int u, int wc,
                                            A (&out)[VDP]) {
    if (u < 0) {
#pragma unroll
        for (int k = 0; k < VDP; ++k) out[k] = (A)0;
        return;
    }
    const int2 nb = __ldg(nbr + u);
    A r1[VDP], r0[VDP], r2[VDP];
    load_row<VDP, PS, A>(src, nb.x, r1);
    load_row<VDP, PS, A>(src, u, r0);
    load_row<VDP, PS, A>(src, nb.y, r2);
    combine3<VDP, A, HOMOG>(r1, r0, r2, wc, out);
}

// PS/PD: row types read and written.  They differ for the first pass of a homogeneous
// 16-bit lattice (FP32 rows from the compaction) and for the last pass of a 16-bit
// lattice (FP32 rows in slot space for the slice).  A fused pair computes the first
// axis's rows in registers with the same arithmetic a separate pass would store, so in
// FP32 it is bit-identical to two passes.
// the last pass writes the slice's rows; homogeneous rows (m_0.., w) go back to plain
// products (w*m_0.., w), so the slice is the same kernel for every payload
template <int VDP, typename PD, typename A, bool HOMOG>
__device__ __forceinline__ void put_row(const BlurArgs& a, PD* dst, uint32_t vtx, A (&out)[VDP]) {
    if constexpr (HOMOG) {
        if (a.products) {
            A w = out[0];
#pragma unroll
            for (int k = 0; k < VDP; ++k) if (k == a.wc) w = out[k];
#pragma unroll
            for (int k = 0; k < VDP; ++k) if (k < a.wc) out[k] = out[k] * w;
        }
    }
    const size_t row = a.dst_map ? (size_t)__ldg(a.dst_map + vtx) : (size_t)vtx;
    store_row<VDP, PD, A>(dst, row, out);
}

// ILP: vertices per thread and iteration (one-axis passes): ILP = 2 issues both vertices'
// neighbour and row loads before either is combined, for twice the loads in flight.
template <int VDP, typename PS, typename PD, bool HOMOG, bool PAIR, int ILP>
__global__ void blur_kernel(BlurArgs a) {
    static_assert(ILP == 1 || (ILP == 2 && !PAIR), "two vertices per iteration in one-axis passes");
    using A = typename AccOf<PD>::T;
    const PS* src = reinterpret_cast<const PS*>(a.src);
    PD* dst = reinterpret_cast<PD*>(a.dst);
    const uint32_t m = *a.nverts;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t vtx = blockIdx.x * blockDim.x + threadIdx.x; vtx < m; vtx += stride * ILP) {
        A out[VDP];
        if constexpr (PAIR) {
            const int2 nb = __ldg(a.nbrB + vtx);
            A r1[VDP], r0[VDP], r2[VDP];
            blurred_row<VDP, PS, A, HOMOG>(src, a.nbrA, nb.x, a.wc, r1);
            blurred_row<VDP, PS, A, HOMOG>(src, a.nbrA, (int)vtx, a.wc, r0);
            blurred_row<VDP, PS, A, HOMOG>(src, a.nbrA, nb.y, a.wc, r2);
            combine3<VDP, A, HOMOG>(r1, r0, r2, a.wc, out);
            put_row<VDP, PD, A, HOMOG>(a, dst, vtx, out);
        } else if constexpr (ILP == 2) {
            const uint32_t v2 = vtx + stride;
            const bool two = v2 < m;
            const int2 na = __ldg(a.nbrA + vtx);
            const int2 nb = two ? __ldg(a.nbrA + v2) : make_int2(-1, -1);
            A p1[VDP], p0[VDP], p2[VDP], q1[VDP], q0[VDP], q2[VDP];
            load_row<VDP, PS, A>(src, na.x, p1);
            load_row<VDP, PS, A>(src, (int)vtx, p0);
            load_row<VDP, PS, A>(src, na.y, p2);
            load_row<VDP, PS, A>(src, nb.x, q1);
            load_row<VDP, PS, A>(src, two ? (int)v2 : -1, q0);
            load_row<VDP, PS, A>(src, nb.y, q2);
            combine3<VDP, A, HOMOG>(p1, p0, p2, a.wc, out);
            put_row<VDP, PD, A, HOMOG>(a, dst, vtx, out);
            if (two) {
                A out2[VDP];
                combine3<VDP, A, HOMOG>(q1, q0, q2, a.wc, out2);
                put_row<VDP, PD, A, HOMOG>(a, dst, v2, out2);
            }
        } else {
            blurred_row<VDP, PS, A, HOMOG>(src, a.nbrA, (int)vtx, a.wc, out);
            put_row<VDP, PD, A, HOMOG>(a, dst, vtx, out);
        }
    }
}

// ---------------------------------------------------------------------------------
// slice
// ---------------------------------------------------------------------------------
constexpr int kSliceThreads = 256;
// latency bound like the splat: 6 blocks of 256 per SM (40 registers) up to d=8
__host__ __device__ constexpr int slice_min_blocks(int d) { return d <= 8 ? 6 : 1; }

// A: arithmetic and storage type of the filtered rows (float, or double for the FP64
// lattice); rows live in slot space (svals[slot*VDP ..]).  With rec_slot the slots come
// from the splat's record of this very point (the reference's replay slice,
// src/Permutohedral.h:418-427); without it the keys are looked up (re-elevation slice at
// other positions, :405-407), and a vertex the splat never created contributes zero.
template <int D, int VDP, typename A>
__global__ void __launch_bounds__(kSliceThreads, slice_min_blocks(D)) slice_kernel(SliceArgs a) {
    constexpr int KW = key_words(D);
    __shared__ float s_delta[(D + 1) * kSliceThreads];
    __shared__ unsigned char s_coord[(D + 1) * kSliceThreads];
    __shared__ Segment sg;
    const int kseg = segment_of_block(a.segs, a.nseg, blockIdx.x);
    load_segment(a.segs + kseg, sg);
    // a block is a slice_tw x slice_th tile of one frame: neighbouring pixels gather the
    // same vertex rows, which then come from L1
    const uint32_t b = blockIdx.x - sg.block_base;
    const uint32_t per_frame = sg.stiles_x * sg.stiles_y;
    const uint32_t fr = b / per_frame, bt = b - fr * per_frame;
    const uint32_t ty = bt / sg.stiles_x, tx = bt - ty * sg.stiles_x;
    const uint32_t px = tx * sg.slice_tw + threadIdx.x % sg.slice_tw;
    const uint32_t py = ty * sg.slice_th + threadIdx.x / sg.slice_tw;
    if (px >= (uint32_t)sg.src.width || py >= (uint32_t)sg.src.height) return;
    const uint32_t i = (fr * (uint32_t)sg.src.height + py) * (uint32_t)sg.src.width + px;
    unsigned* status = a.seg_status + kseg;
    // A splat that overflowed the table is rerun by the host with more slots; its
    // output may be the caller's input image (in-place filtering), so write nothing.
    if (__ldcg(status) & (kStatusProbeLimit | kStatusSpinLimit | kStatusKeyRange)) return;
    const uint32_t gi = sg.point_base + i;
    float p[D];
    load_position<D>(sg.src, i, p);
    Simplex<D> sx;
    const SimplexScratch scr{s_delta + threadIdx.x, s_coord + threadIdx.x, kSliceThreads};
    compute_simplex<D>(p, a.lc, sx, status, scr);
    const A* sv = reinterpret_cast<const A*>(a.svals);
    A acc[VDP];
#pragma unroll
    for (int k = 0; k < VDP; ++k) acc[k] = (A)0;
    // Replay slice of small rows: the d+1 slots, then all d+1 rows in flight at once, as
    // one vector load each (a vertex the splat could not place loads row 0, unused).
    constexpr bool kGather = D <= 8 && VDP == 4 && sizeof(A) == 4;
    if (kGather && a.rec_slot && !a.rec_vtx) {
        int sl[D + 1];
#pragma unroll
        for (int r = 0; r <= D; ++r) sl[r] = (int)__ldg(a.rec_slot + (size_t)r * a.n_total + gi);
        float4 rows[D + 1];
#pragma unroll
        for (int r = 0; r <= D; ++r)
            rows[r] = __ldg(reinterpret_cast<const float4*>(sv) + (sl[r] >= 0 ? sl[r] : 0));
#pragma unroll
        for (int r = 0; r <= D; ++r) {
            if (sl[r] < 0) continue;
            const float w = sx.bary[r];
            const A row[4] = {rows[r].x, rows[r].y, rows[r].z, rows[r].w};
#pragma unroll
            for (int k = 0; k < VDP; ++k) acc[k] = acc_add(acc[k], (A)w * row[k]);
        }
    } else {
    Key<KW> key;
    if (!a.rec_slot) first_key<D>(sx, key);
#pragma unroll
    for (int r = 0; r <= D; ++r) {
        int s;   // slot in the shared array
        if (a.rec_slot) {
            s = (int)__ldg(a.rec_slot + (size_t)r * a.n_total + gi);
        } else {
            if (r > 0) key_step<D>(key, scr.coord[(D - (r - 1)) * scr.stride]);
            const TableView table{a.key0 + sg.slot_base, a.keyn + sg.slot_base, sg.cap, a.cap_total};
            const int ls = table_find<D>(table, key, key_hash<KW>(key));
            s = ls >= 0 ? (int)sg.slot_base + ls : -1;
        }
        const float w = sx.bary[r];
        if (a.rec_vtx) {
            a.rec_vtx[(size_t)gi * (D + 1) + r] = s >= 0 ? (int)__ldg(a.slot2vtx + s) : -1;
            a.rec_w[(size_t)gi * (D + 1) + r] = w;
        }
        if (s >= 0) {
            A row[VDP];
#pragma unroll
            for (int k = 0; k < VDP; ++k) row[k] = __ldg(sv + (size_t)s * VDP + k);
#pragma unroll
            for (int k = 0; k < VDP; ++k) acc[k] = acc_add(acc[k], (A)w * row[k]);
        }
    }
    }
    // write
    const uint32_t wdt = (uint32_t)sg.src.width, hgt = (uint32_t)sg.src.height;
    const uint32_t x = i % wdt, q = i / wdt, y = q % hgt, t = q / hgt;
    const OutView& ov = sg.out;
    float* o = ov.base + (long long)t * ov.tstride + (long long)y * ov.ystride + x;
    A wsum = acc[0];
#pragma unroll
    for (int j = 0; j < VDP; ++j) if (j == a.vd - 1) wsum = acc[j];
    // normalised per channel, as src/GaussTransform.cpp:673-676 divides
#pragma unroll
    for (int k = 0; k < VDP; ++k) {
        if (k < ov.channels) {
            const float r = ov.normalize ? (float)(acc[k] / wsum) : (float)acc[k];
            o[(long long)k * ov.cstride] = r;
        }
    }
}

// Replay slice from the splat's records of slots and weights (src/Permutohedral.h:418-427:
// the reference replays its recorded offsets and weights the same way): a gather of d+1 rows
// per point with no simplex to recompute.  A block is a slice_tw x slice_th tile of one frame.
template <int D, int VDP, typename A>
__global__ void __launch_bounds__(kSliceThreads) slice_replay_kernel(SliceArgs a) {
    __shared__ Segment sg;
    const int kseg = segment_of_block(a.segs, a.nseg, blockIdx.x);
    load_segment(a.segs + kseg, sg);
    const uint32_t b = blockIdx.x - sg.block_base;
    const uint32_t per_frame = sg.stiles_x * sg.stiles_y;
    const uint32_t fr = b / per_frame, bt = b - fr * per_frame;
    const uint32_t ty = bt / sg.stiles_x, tx = bt - ty * sg.stiles_x;
    const uint32_t px = tx * sg.slice_tw + threadIdx.x % sg.slice_tw;
    const uint32_t py = ty * sg.slice_th + threadIdx.x / sg.slice_tw;
    const uint32_t W = (uint32_t)sg.src.width, H = (uint32_t)sg.src.height;
    if (px >= W || py >= H) return;
    // an image whose splat overflowed its table is rerun by the host; write nothing
    if (__ldcg(a.seg_status + kseg) & (kStatusProbeLimit | kStatusSpinLimit | kStatusKeyRange)) return;
    const uint32_t gi = sg.point_base + (fr * H + py) * W + px;
    const A* sv = reinterpret_cast<const A*>(a.svals);
    int sl[D + 1];
    float w[D + 1];
#pragma unroll
    for (int r = 0; r <= D; ++r) {
        sl[r] = (int)__ldcs(a.rec_slot + (size_t)r * a.n_total + gi);
        w[r] = __ldcs(a.rec_w_in + (size_t)r * a.n_total + gi);
    }
    A acc[VDP];
#pragma unroll
    for (int k = 0; k < VDP; ++k) acc[k] = (A)0;
    if constexpr (VDP == 4 && sizeof(A) == 4) {
        float4 rows[D + 1];
#pragma unroll
        for (int r = 0; r <= D; ++r)   // a point the splat could not place reads row 0, unused
            rows[r] = __ldg(reinterpret_cast<const float4*>(sv) + (sl[r] >= 0 ? sl[r] : 0));
#pragma unroll
        for (int r = 0; r <= D; ++r) {
            if (sl[r] < 0) continue;
            acc[0] = acc_add(acc[0], w[r] * rows[r].x);
            acc[1] = acc_add(acc[1], w[r] * rows[r].y);
            acc[2] = acc_add(acc[2], w[r] * rows[r].z);
            acc[3] = acc_add(acc[3], w[r] * rows[r].w);
        }
    } else {
#pragma unroll
        for (int r = 0; r <= D; ++r) {
            if (sl[r] < 0) continue;
#pragma unroll
            for (int k = 0; k < VDP; ++k) acc[k] = acc_add(acc[k], (A)w[r] * __ldg(sv + (size_t)sl[r] * VDP + k));
        }
    }
    const OutView& ov = sg.out;
    float* o = ov.base + (long long)fr * ov.tstride + (long long)py * ov.ystride + px;
    A wsum = acc[0];
#pragma unroll
    for (int j = 0; j < VDP; ++j) if (j == a.vd - 1) wsum = acc[j];
#pragma unroll
    for (int k = 0; k < VDP; ++k) {
        if (k < ov.channels) {
            const float r = ov.normalize ? (float)(acc[k] / wsum) : (float)acc[k];
            __stcs(o + (long long)k * ov.cstride, r);
        }
    }
}

}  // namespace pgpu
