// The launch sequence of a batch of lattices — many images of one kind (same number of
// position dimensions, value channels and payload) per launch; a single image is a batch
// of one.  Every image owns a range of the shared hash-slot array sized from its learned
// vertices-per-pixel ratio; an image whose range overflows is rerun with a larger range.
// A batch can be captured as a CUDA graph and replayed for the next batch of the same
// shape: the per-image descriptors are data uploaded by the graph's first node, so only
// sizes are baked into it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace pgpu {

int Engine::ensure_hmeta(size_t bytes) {
    if (bytes <= hmeta_bytes) return PGPU_OK;
    if (hmeta) cudaFreeHost(hmeta);
    hmeta = nullptr;
    hmeta_bytes = 0;
    const size_t nb = std::max<size_t>(2 * bytes, 65536);
    if (cudaHostAlloc((void**)&hmeta, nb, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return fail(PGPU_ERR_MEMORY, "pinned allocation of %zu bytes failed", nb);
    }
    hmeta_bytes = nb;
    return PGPU_OK;
}

int Engine::ensure_copy_streams() {
    if (copy_in) return PGPU_OK;
    CUDA_TRY(cudaStreamCreateWithFlags(&copy_out, cudaStreamNonBlocking));
    for (auto& e : pipe_ev) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(cudaStreamCreateWithFlags(&copy_in, cudaStreamNonBlocking));
    return PGPU_OK;
}

void Engine::drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    graphs.clear();
}

void Engine::shutdown() {
    if (device >= 0) cudaSetDevice(device);
    drain_async(*this);
    for (auto& pb : pinned_free) cudaFreeHost(pb.first);
    pinned_free.clear();
    if (stream) cudaStreamSynchronize(stream);
    drop_graphs();
    for (auto& e : ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (cudaStream_t* cs : {&copy_in, &copy_out}) {
        if (*cs) cudaStreamSynchronize(*cs), cudaStreamDestroy(*cs);
        *cs = nullptr;
    }
    for (auto& e : pipe_ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (auto& e : join_ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    if (hstat) cudaFreeHost(hstat);
    hstat = nullptr;
    if (hmeta) cudaFreeHost(hmeta);
    hmeta = nullptr;
    hmeta_bytes = 0;
    for (DevBuf* b : {&key0, &keyn, &tvals, &ft, &slot2vtx, &bitmap, &offs, &partials, &vkey0, &vkeyn,
                      &vv0, &vv1, &nbr, &vf32, &vtx2slot, &sval, &rec, &recw, &grid, &grid2, &tags, &vlist, &dstat, &meta, &img_a, &img_b,
                      &img_c, &img_d})
        b->release();
}

namespace {

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Vertices per point learned from earlier lattices, shared by every engine of the process
// (the server's workers each have one): by image signature, and the latest batch's
// largest ratio per d as the guess for an unseen signature.  A guess that is too small
// makes the image overflow its hash range and run again.
std::mutex g_ratio_mu;
std::unordered_map<uint64_t, double> g_ratio_by_sig;
std::map<int, double> g_ratio;

inline uint64_t mix64(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h * 0xBF58476D1CE4E5B9ull;
}
inline uint64_t float_bits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

// an image's key for the learned vertex ratio: a 64-bit mix of its shape and position
// scales (a collision would only size a table from another image's ratio: at worst a rerun)
uint64_t item_signature(int d, const PointSource& s) {
    uint64_t h = mix64(0x51ED27B3ull, (uint64_t)d);
    h = mix64(h, ((uint64_t)(uint32_t)s.width << 32) | (uint32_t)s.height);
    h = mix64(h, ((uint64_t)(uint32_t)s.frames << 32) | (uint32_t)s.coord_mask);
    for (int c = 0; c < s.pos_channels && c < kMaxD; ++c) h = mix64(h, float_bits(s.pos_scale[c]));
    for (int c = 0; c < 3; ++c) h = mix64(h, float_bits(s.coord_scale[c]));
    return h;
}

// Each image's learned vertices-per-point ratio (by signature, else the latest batch's
// largest for d, else 1.0: a large table), and the density the splat choice goes by (the
// learned ratio, else the latest batch's for d, else 0: nothing known, the tile splat).
void learned_ratios(const BatchJob& B, std::vector<uint64_t>* sig, std::vector<double>* ratio,
                    std::vector<double>* density) {
    const int nseg = (int)B.items.size();
    sig->resize(nseg);
    ratio->resize(nseg);
    density->resize(nseg);
    std::lock_guard<std::mutex> lk(g_ratio_mu);
    const bool have_d = g_ratio.count(B.d) != 0;
    const double dflt = have_d ? g_ratio[B.d] : 1.0;
    for (int k = 0; k < nseg; ++k) {
        (*sig)[k] = item_signature(B.d, B.items[k].splat);
        auto it = g_ratio_by_sig.find((*sig)[k]);
        (*ratio)[k] = it != g_ratio_by_sig.end() ? it->second : dflt;
        (*density)[k] = it != g_ratio_by_sig.end() ? it->second : have_d ? dflt : 0.0;
    }
}

// Splat kernel per lattice: the tile splat (shared-memory table per 16x16 tile) where
// neighbouring points share vertices, which the learned vertices-per-point ratio tells
// (4K d=5 bilateral: 0.18; a 16x16 tile then holds about 155 of its 1536 entries'
// vertices); the direct splat for sparse lattices (ratio above kTileRatioMax: measured
// on the mixed batch, 1.5 beats 0.8 by 2 % and 0.4 by 3 %), multi-word keys and FP64
// accumulators.  With nothing learned yet for the image or its d, the tile splat.
// PGPU_SPLAT=direct or =tile in the environment overrides the choice where both exist
// (the parity tests compare the two).
#ifndef PGPU_TILE_RATIO_MAX
#define PGPU_TILE_RATIO_MAX 1.5
#endif
constexpr double kTileRatioMax = PGPU_TILE_RATIO_MAX;

int splat_forced() {
    const char* mode = std::getenv("PGPU_SPLAT");
    return !mode ? 0 : !strcmp(mode, "direct") ? 1 : !strcmp(mode, "tile") ? 2 : 0;
}

bool tile_splat_for(const BatchJob& B, int forced, double density, uint32_t n) {
    const bool tile_ok = key_words(B.d) == 1 && B.payload != kPayloadF64 && forced != 1 &&
                         (forced == 2 || B.splat == 0);
    return tile_ok && (forced == 2 || (density <= kTileRatioMax && n >= 256));
}

// the job asks for vertex-ordered rows (PGPU_ROWS=slot or =vertex in the environment
// overrides the job's choice; the parity tests compare both), where they can apply
bool vertex_rows_wanted(const BatchJob& B) {
    const char* rows_mode = std::getenv("PGPU_ROWS");
    const bool want = rows_mode && !strcmp(rows_mode, "vertex") ? true
                    : rows_mode && !strcmp(rows_mode, "slot")   ? false
                                                                : !B.slot_rows;
    const bool dumps = B.rec_vtx || B.dump_splat;
    return want && !dumps && B.replay && key_words(B.d) == 1 && index_in_key(B.d) &&
           B.payload != kPayloadF64;
}

// device (and pinned host) metadata of one batch
struct MetaLayout {
    size_t segstat, counts, slotbase, entry, segs, slsegs, total;
};

MetaLayout layout(int nseg, bool slice_segs) {
    MetaLayout L;
    // bytes [0, 64): [0] spare status word, [1] total vertices
    L.segstat = 64;
    L.counts = align16(L.segstat + 4 * (size_t)nseg);
    L.slotbase = align16(L.counts + 4 * (size_t)nseg);
    L.entry = align16(L.slotbase + 4 * (size_t)(nseg + 1));
    L.segs = align16(L.entry + 4 * (size_t)(nseg + 1));
    L.slsegs = align16(L.segs + sizeof(Segment) * nseg);
    L.total = align16(L.slsegs + (slice_segs ? sizeof(Segment) * nseg : 0));
    return L;
}

}  // namespace

size_t batch_meta_bytes(int nseg) { return layout(nseg, false).total; }

// Queue one pass over the batch on st, its metadata staged in the pinned buffer h (E.hmeta
// when null); *ps receives what finish_pass needs once the stream has run it.  timed: CUDA
// events around every stage (read by finish_pass).
static int enqueue_pass(Engine& E, const BatchJob& B, cudaStream_t st,
                        const std::vector<uint64_t>* cap_in, unsigned char* h_in, bool timed,
                        int pass, PassState* ps) {
    const int d = B.d, vd = B.vd;
    const int nseg = (int)B.items.size();
    if (nseg == 0) return PGPU_OK;
    const DimOps* ops = dim_ops(d);
    if (!ops) return fail(PGPU_ERR_UNSUPPORTED, "%d position dimensions (supported: 1..%d)", d, kMaxD);
    if (!ops->prepare())
        return fail(PGPU_ERR_CUDA, "tile splat set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    const int vdp = vdp_for(vd);
    if (!vdp) return fail(PGPU_ERR_UNSUPPORTED, "%d value channels (supported: 1..8)", vd);
    if (B.payload < 0 || B.payload > 3) return fail(PGPU_ERR_ARGUMENT, "unknown payload %d", B.payload);
    const int kw = key_words(d);
    // 16-bit payloads of lattices whose last value channel is the homogeneous weight keep
    // rows normalised by that weight (see assign_kernel)
    const bool homog = B.homog && (B.payload == kPayloadF16 || B.payload == kPayloadBF16);
    const float load = (B.load > 0.05f && B.load <= 0.9f) ? B.load : 0.5f;
    const size_t accb = accum_bytes(B.payload), payb = payload_bytes(B.payload);
    const LatticeConsts lc = make_consts(d);
    const bool dumps = B.rec_vtx || B.dump_splat;
    // Slot tags for the neighbour lookups pay for multi-word keys (d >= 8): those lattices
    // are sparse, most neighbours are absent, and the table is far larger than L2.  At
    // lower d most neighbours exist and the table fits in L2, where the tag is one more
    // dependent load (4K d=5: neighbours 0.18 -> 0.23 ms with tags; 2M points d=16:
    // 25.8 -> 20.5 ms).
    const bool use_tags = kw > 1;
    const bool graph = B.use_graph && !dumps;
    // Vertices are numbered in the reference's first-insertion order only for parity dumps
    // (first touches, a bitmap and its prefix popcount); otherwise in the order the splat
    // created them, which gives the same filtered values with less work.
    const bool exact_order = dumps;
    // The replay slice reads weights the splat recorded beside the slots, as the
    // reference's replay does, instead of recomputing every point's simplex (parity dumps
    // recompute them: they report the weights the slice sees).
    const bool replay_w = B.replay && !dumps;

    // points and first-touch entries, lattice after lattice
    uint64_t n_total = 0, ns_total = 0;
    std::vector<uint32_t> pbase(nseg), spbase(nseg);
    for (int k = 0; k < nseg; ++k) {
        const BatchItem& it = B.items[k];
        pbase[k] = (uint32_t)n_total;
        n_total += it.n;
        spbase[k] = (uint32_t)ns_total;
        ns_total += B.replay ? it.n : it.n_slice;
    }
    const uint64_t entries = n_total * (uint64_t)(d + 1);
    if (entries >= 0xFFFFFFFFull || ns_total * (uint64_t)(d + 1) >= 0xFFFFFFFFull)
        return fail(PGPU_ERR_UNSUPPORTED, "too many points for one batch (%llu)",
                    (unsigned long long)n_total);
    const uint32_t nwords = (uint32_t)((entries + 31) / 32);

    // slots per lattice: (learned vertices per point) x 1.3 x points / load
    std::vector<uint64_t> sig;
    std::vector<double> ratio, density;
    learned_ratios(B, &sig, &ratio, &density);
    std::vector<uint64_t> cap(nseg);
    for (int k = 0; k < nseg; ++k) {
        if (cap_in) {
            cap[k] = (*cap_in)[k];
            continue;
        }
        const uint64_t n = B.items[k].n;
        uint64_t est = (uint64_t)std::ceil(ratio[k] * 1.3 * (double)n) + 256;
        est = std::min<uint64_t>(est, n * (uint64_t)(d + 1) + 256);
        const uint64_t c = (uint64_t)std::ceil((double)est / load);
        cap[k] = std::max<uint64_t>((c + 31) & ~31ull, 256);
    }

    // splat kernel per lattice (tile_splat_for)
    const int forced = splat_forced();
    std::vector<Segment> segs(nseg), slsegs(B.replay ? 0 : nseg);
    uint64_t blocks = 0, tile_blocks = 0, slice_blocks = 0;
    int tiled_count = 0;
    for (int k = 0; k < nseg; ++k) {
        const BatchItem& it = B.items[k];
        Segment& sgm = segs[k];
        memset(&sgm, 0, sizeof(sgm));
        sgm.src = it.splat;
        sgm.out = it.out;
        sgm.n = it.n;
        sgm.point_base = pbase[k];
        const bool tiled = tile_splat_for(B, forced, density[k], it.n);
        uint32_t nb_splat = 0, nb_tile = 0, nb_slice = 0;
        segment_geometry(sgm, B.replay ? it.splat : it.slice, tiled, &nb_splat, &nb_tile, &nb_slice,
                         (uint32_t)B.tile_w);
        tiled_count += tiled ? 1 : 0;
        sgm.splat_base = (uint32_t)blocks;
        sgm.tile_base = (uint32_t)tile_blocks;
        sgm.block_base = (uint32_t)slice_blocks;
        blocks += nb_splat;
        tile_blocks += nb_tile;
        slice_blocks += nb_slice;
        if (!B.replay) {
            Segment& sl = slsegs[k];
            sl = sgm;
            sl.src = it.slice;
            sl.n = it.n_slice;
            sl.point_base = spbase[k];
        }
    }
    if (blocks >= 0x7FFFFFFFull || tile_blocks >= 0x7FFFFFFFull || slice_blocks >= 0x7FFFFFFFull)
        return fail(PGPU_ERR_UNSUPPORTED, "too many points for one batch (%llu)",
                    (unsigned long long)n_total);

    // Vertex-ordered rows: where every image takes the tile splat with one-word keys that
    // hold their vertex index (d <= 6) and the slice replays the splat points, the splat
    // numbers the vertices as it creates them and accumulates straight into
    // vertex-ordered FP32 rows, so no compaction runs; the first blur pass reads those
    // rows (16-bit payloads: FP32 rows, homogeneous ones normalised by the neighbour
    // search, once per vertex) and the slice reads rows by vertex index.
    const bool vrows = vertex_rows_wanted(B) && tiled_count == nseg;
    // PGPU_BLUR=pairs or =single in the environment overrides the blur pairing (tests)
    const char* blur_mode = std::getenv("PGPU_BLUR");
    const bool blur_pairs = blur_mode && !strcmp(blur_mode, "pairs") ? true
                          : blur_mode && !strcmp(blur_mode, "single") ? false
                                                                       : B.blur_pairs;
    // one neighbour lookup per axis (the splat's creators or the compaction mark the pairs
    // absent first); PGPU_NBR=half or =both in the environment overrides the job's choice
    const char* nbr_mode = std::getenv("PGPU_NBR");
    const bool nbr_half = nbr_mode && !strcmp(nbr_mode, "half") ? true
                        : nbr_mode && !strcmp(nbr_mode, "both") ? false
                                                                : B.nbr_half != 0;
    // 16-bit payloads accumulate in FP32 rows (vf32), which the first blur pass reads
    const bool f32_rows = vrows && (B.payload == kPayloadF16 || B.payload == kPayloadBF16);
    const MetaLayout L = layout(nseg, !B.replay);
    int rc;
    if ((!h_in && (rc = E.ensure_hmeta(L.total))) || (rc = E.meta.ensure(L.total))) return rc;
    if (h_in && !B.replay) return fail(PGPU_ERR_UNSUPPORTED, "queued passes replay the splat points");

    {
        std::vector<uint64_t> sbase(nseg + 1);
        uint64_t cap_total = 0;
        for (int k = 0; k < nseg; ++k) {
            sbase[k] = cap_total;
            cap_total += cap[k];
        }
        sbase[nseg] = cap_total;
        if (cap_total > 0x7FFFFF00ull) return fail(PGPU_ERR_CAPACITY, "batch needs more than 2^31 hash slots");

        if ((rc = E.key0.ensure(cap_total * 16)) || (rc = E.keyn.ensure((kw - 1) * cap_total * 16)) ||
            (rc = E.tvals.ensure(cap_total * vdp * accb)) ||
            (rc = E.slot2vtx.ensure(cap_total * 4)) ||
            (exact_order && (rc = E.ft.ensure(cap_total * 4))) ||
            (exact_order && (rc = E.bitmap.ensure((size_t)nwords * 4))) ||
            (exact_order && (rc = E.offs.ensure((size_t)nwords * 4))) ||
            (exact_order && (rc = E.partials.ensure((size_t)scan_parts(nwords) * 4 + 16))) ||
            (!exact_order && (rc = E.vlist.ensure(cap_total * 4))) ||
            (rc = E.vkey0.ensure(cap_total * 16)) || (rc = E.vkeyn.ensure((kw - 1) * cap_total * 16)) ||
            (rc = E.vv0.ensure(cap_total * vdp * payb)) || (rc = E.vv1.ensure(cap_total * vdp * payb)) ||
            (rc = E.nbr.ensure((size_t)(d + 1) * cap_total * 8)) ||
            ((homog || payb == 2) && (rc = E.vf32.ensure(cap_total * vdp * 4))) ||
            (rc = E.vtx2slot.ensure(cap_total * 4)) || (rc = E.sval.ensure(cap_total * vdp * accb)) ||
            (use_tags && (rc = E.tags.ensure(cap_total))) ||
            (B.replay && (rc = E.rec.ensure((size_t)entries * 4))) ||
            (replay_w && (rc = E.recw.ensure((size_t)entries * 4))))
            return rc;

        // per-lattice descriptors, staged in pinned memory and uploaded by the first copy
        unsigned char* h = h_in ? h_in : E.hmeta;
        uint32_t* hslot = (uint32_t*)(h + L.slotbase);
        uint32_t* hentry = (uint32_t*)(h + L.entry);
        Segment* hseg = (Segment*)(h + L.segs);
        Segment* hsl = (Segment*)(h + L.slsegs);
        for (int k = 0; k <= nseg; ++k) {
            hslot[k] = (uint32_t)sbase[k];
            hentry[k] = k < nseg ? pbase[k] * (uint32_t)(d + 1) : (uint32_t)entries;
        }
        for (int k = 0; k < nseg; ++k) {
            segs[k].slot_base = (uint32_t)sbase[k];
            segs[k].cap = (uint32_t)cap[k];
            hseg[k] = segs[k];
            if (!B.replay) {
                slsegs[k].slot_base = (uint32_t)sbase[k];
                slsegs[k].cap = (uint32_t)cap[k];
                hsl[k] = slsegs[k];
            }
        }

        unsigned char* dmeta = (unsigned char*)E.meta.p;
        uint32_t* dM = (uint32_t*)dmeta + 1;
        auto enqueue = [&](bool timed) -> int {
            // the lattice's time (and so the autotuner's) includes clearing its tables
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[6], st));
            CUDA_TRY(cudaMemcpyAsync(dmeta + L.slotbase, h + L.slotbase, L.total - L.slotbase,
                                     cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemsetAsync(dmeta, 0, L.slotbase, st));
            CUDA_TRY(cudaMemsetAsync(E.key0.p, 0xFF, cap_total * 16, st));
            if (!vrows) CUDA_TRY(cudaMemsetAsync(E.tvals.p, 0, cap_total * vdp * accb, st));
            else CUDA_TRY(cudaMemsetAsync((homog || f32_rows) ? E.vf32.p : E.vv0.p, 0, cap_total * vdp * 4, st));
            if (exact_order) {
                CUDA_TRY(cudaMemsetAsync(E.ft.p, 0xFF, cap_total * 4, st));
                CUDA_TRY(cudaMemsetAsync(E.bitmap.p, 0, (size_t)nwords * 4, st));
            }
            if (use_tags) CUDA_TRY(cudaMemsetAsync(E.tags.p, 0, cap_total, st));
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[0], st));

            SplatArgs sa;
            sa.segs = (const Segment*)(dmeta + L.segs);
            sa.nseg = nseg;
            sa.n_total = (uint32_t)n_total;
            sa.lc = lc;
            sa.key0 = (uint4*)E.key0.p;
            sa.keyn = (uint4*)E.keyn.p;
            sa.cap_total = (uint32_t)cap_total;
            sa.vals = E.tvals.p;
            sa.ft = exact_order ? (uint32_t*)E.ft.p : nullptr;
            sa.vlist = (exact_order || vrows) ? nullptr : (uint32_t*)E.vlist.p;
            if (vrows) {
                sa.vrows = (homog || f32_rows) ? E.vf32.p : E.vv0.p;
                sa.vkey0 = (uint4*)E.vkey0.p;
                sa.vtx2slot = (uint32_t*)E.vtx2slot.p;
                if (nbr_half) {
                    sa.nbr_init = (int2*)E.nbr.p;
                    sa.nbr_stride = (uint32_t)cap_total;
                    sa.nbr_axes = d + 1;
                }
            }
            sa.vcount = dM;
            sa.seg_counts = (uint32_t*)(dmeta + L.counts);
            sa.rec_slot = B.replay ? (uint32_t*)E.rec.p : nullptr;
            sa.rec_w = replay_w ? (float*)E.recw.p : nullptr;
            sa.seg_status = (unsigned*)(dmeta + L.segstat);
            sa.blocks = (uint32_t)blocks;
            sa.tile_blocks = (uint32_t)tile_blocks;
            if (!ops->splat(sa, vdp, B.payload, st)) return fail(PGPU_ERR_UNSUPPORTED, "splat variant");
            CUDA_TRY(cudaGetLastError());
            if (!ops->splat_tile(sa, vdp, B.payload, st)) return fail(PGPU_ERR_UNSUPPORTED, "tile splat variant");
            CUDA_TRY(cudaGetLastError());
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[1], st));

            if (exact_order) {
                launch_mark((const uint32_t*)E.ft.p, (uint32_t)cap_total, (uint32_t*)E.bitmap.p, E.sms, st);
                launch_scan((const uint32_t*)E.bitmap.p, nwords, (uint32_t*)E.partials.p,
                            (uint32_t*)E.offs.p, dM, st);
                launch_segment_counts((const uint32_t*)E.bitmap.p, (const uint32_t*)E.offs.p, nwords, dM,
                                      (const uint32_t*)(dmeta + L.entry), nseg,
                                      (uint32_t*)(dmeta + L.counts), st);
            }
            CompactArgs ca;
            memset(&ca, 0, sizeof(ca));
            if (!vrows) {
            ca.table = TableView{(uint4*)E.key0.p, (uint4*)E.keyn.p, (uint32_t)cap_total, (uint32_t)cap_total};
            ca.ft = (const uint32_t*)E.ft.p;
            ca.bitmap = (uint32_t*)E.bitmap.p;
            ca.nwords = nwords;
            ca.offs = (const uint32_t*)E.offs.p;
            ca.slot2vtx = (uint32_t*)E.slot2vtx.p;
            ca.vtx2slot = (uint32_t*)E.vtx2slot.p;
            ca.vkey0 = (uint4*)E.vkey0.p;
            ca.vkeyn = (uint4*)E.vkeyn.p;
            ca.vcap = (uint32_t)cap_total;
            ca.tvals = E.tvals.p;
            ca.vvals = homog ? E.vf32.p : E.vv0.p;
            ca.wc = vd - 1;
            ca.tags = use_tags ? (uint8_t*)E.tags.p : nullptr;
            ca.vlist = exact_order ? nullptr : (const uint32_t*)E.vlist.p;
            ca.nverts = dM;
            ca.index_in_key = index_in_key(d) ? 1 : 0;   // the neighbour lookups expect it
            if (nbr_half) {
                ca.nbr_init = (int2*)E.nbr.p;
                ca.nbr_stride = (uint32_t)cap_total;
                ca.nbr_axes = d + 1;
            }
            if (!launch_assign(ca, kw, vdp, B.payload, homog, E.sms, st))
                return fail(PGPU_ERR_UNSUPPORTED, "assign variant");
            CUDA_TRY(cudaGetLastError());
            }
            if (B.dump_splat)
                CUDA_TRY(cudaMemcpyAsync(B.dump_splat, E.vv0.p,
                                         std::min<size_t>(cap_total * vdp * payb, B.dump_bytes),
                                         cudaMemcpyDeviceToDevice, st));
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[2], st));

            NbrArgs na;
            na.key0 = (uint4*)E.key0.p;
            na.keyn = (uint4*)E.keyn.p;
            na.cap_total = (uint32_t)cap_total;
            na.seg_slot_base = (const uint32_t*)(dmeta + L.slotbase);
            na.nseg = nseg;
            na.vtx2slot = (const uint32_t*)E.vtx2slot.p;
            na.slot2vtx = (const uint32_t*)E.slot2vtx.p;
            na.vkey0 = (const uint4*)E.vkey0.p;
            na.vkeyn = (const uint4*)E.vkeyn.p;
            na.vcap = (uint32_t)cap_total;
            na.nverts = dM;
            na.nbr = (int2*)E.nbr.p;
            na.tags = use_tags ? (const uint8_t*)E.tags.p : nullptr;
            na.seg_status = (const unsigned*)(dmeta + L.segstat);
            na.half = nbr_half ? 1 : 0;
            if (vrows && homog) {   // the splat's sums, normalised once per vertex here
                na.norm_rows = (float*)E.vf32.p;
                na.vdp = vdp;
                na.wc = vd - 1;
            }
            ops->neighbours(na, (uint32_t)cap_total, E.sms, st);
            CUDA_TRY(cudaGetLastError());
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[3], st));

            BlurPlan bp;
            bp.d = d;
            bp.vdp = vdp;
            bp.payload = B.payload;
            bp.homog = homog;
            bp.src_f32 = homog || f32_rows;
            bp.nbr = (const int2*)E.nbr.p;
            bp.nbr_stride = cap_total;
            bp.nverts = dM;
            bp.vmax = (uint32_t)cap_total;
            bp.src = (homog || f32_rows) ? E.vf32.p : E.vv0.p;
            bp.bufs[0] = E.vv1.p;
            bp.bufs[1] = E.vv0.p;
            bp.sval = E.sval.p;
            bp.vtx2slot = vrows ? nullptr : (const uint32_t*)E.vtx2slot.p;   // null: vertex order
            bp.wc = vd - 1;
            bp.sms = E.sms;
            bp.pairs = blur_pairs;
            if (payb == 2) bp.f32buf = E.vf32.p;
            bp.grid = B.blur_grid;
            if (blur_all_axes(bp, st)) return fail(PGPU_ERR_UNSUPPORTED, "blur variant");
            CUDA_TRY(cudaGetLastError());
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[4], st));

            SliceArgs sl;
            sl.segs = (const Segment*)(dmeta + (B.replay ? L.segs : L.slsegs));
            sl.nseg = nseg;
            sl.n_total = (uint32_t)n_total;
            sl.lc = lc;
            sl.key0 = (uint4*)E.key0.p;
            sl.keyn = (uint4*)E.keyn.p;
            sl.cap_total = (uint32_t)cap_total;
            sl.slot2vtx = (const uint32_t*)E.slot2vtx.p;
            sl.rec_slot = B.replay ? (const uint32_t*)E.rec.p : nullptr;
            sl.rec_w_in = replay_w ? (const float*)E.recw.p : nullptr;
            sl.svals = E.sval.p;
            sl.vd = vd;
            sl.rec_vtx = B.rec_vtx;
            sl.rec_w = B.rec_w;
            sl.seg_status = (unsigned*)(dmeta + L.segstat);
            sl.blocks = (uint32_t)slice_blocks;
            if (!ops->slice(sl, vdp, B.payload, homog, st)) return fail(PGPU_ERR_UNSUPPORTED, "slice variant");
            CUDA_TRY(cudaGetLastError());
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[5], st));
            CUDA_TRY(cudaMemcpyAsync(h, dmeta, L.slotbase, cudaMemcpyDeviceToHost, st));
            return PGPU_OK;
        };

        if (graph) {
            // the graph bakes in sizes, settings and buffer addresses, so all of them key it
            std::vector<uint64_t> gk = {
                (uint64_t)d, (uint64_t)vd, (uint64_t)B.payload, (uint64_t)homog, (uint64_t)B.replay,
                (uint64_t)nseg, n_total, ns_total, cap_total, nwords, (uint64_t)blur_pairs,
                (uint64_t)B.blur_grid, blocks,
                tile_blocks, slice_blocks, (uint64_t)(uintptr_t)E.key0.p, (uint64_t)(uintptr_t)E.keyn.p,
                (uint64_t)(uintptr_t)E.tvals.p, (uint64_t)(uintptr_t)E.nbr.p, (uint64_t)(uintptr_t)E.rec.p,
                (uint64_t)(uintptr_t)E.recw.p, (uint64_t)(uintptr_t)E.meta.p, (uint64_t)(uintptr_t)h,
                (uint64_t)(uintptr_t)E.sval.p, (uint64_t)(uintptr_t)E.vlist.p, (uint64_t)(uintptr_t)E.vv0.p,
                (uint64_t)(uintptr_t)E.vv1.p, (uint64_t)(uintptr_t)E.vkey0.p, (uint64_t)(uintptr_t)E.vf32.p,
                (uint64_t)vrows, (uint64_t)(uintptr_t)E.vtx2slot.p, (uint64_t)nbr_half, (uint64_t)B.tile_w};
            gk.reserve(gk.size() + 2 * (size_t)nseg);
            for (int k = 0; k < nseg; ++k) {
                gk.push_back(cap[k]);
                gk.push_back(((uint64_t)B.items[k].n << 1) | (segs[k].tile_w ? 1u : 0u));
            }
            auto it = E.graphs.find(gk);
            if (it == E.graphs.end()) {
                if (E.graphs.size() >= 32) E.drop_graphs();
                cudaGraph_t g = nullptr;
                CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                const int erc = enqueue(false);
                const cudaError_t ce = cudaStreamEndCapture(st, &g);
                if (erc) {
                    if (g) cudaGraphDestroy(g);
                    return erc;
                }
                if (ce != cudaSuccess) return fail(PGPU_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
                cudaGraphExec_t ex = nullptr;
                const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) return fail(PGPU_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
                it = E.graphs.emplace(gk, ex).first;
            }
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[0], st));
            CUDA_TRY(cudaGraphLaunch(it->second, st));
            if (timed) CUDA_TRY(cudaEventRecord(E.ev[5], st));
        } else {
            if ((rc = enqueue(timed))) return rc;
        }
        ps->h = h;
        ps->segstat = L.segstat;
        ps->counts = L.counts;
        ps->cap = cap;
        ps->sig = sig;
        ps->load = load;
        ps->tiled = tiled_count;
        ps->pass = pass;
        ps->n_total = n_total;
        ps->cap_total = cap_total;
        ps->timed = timed ? (graph ? 2 : 1) : 0;
        ps->nbr_half = nbr_half ? 1 : 0;
        ps->vertex_rows = vrows ? 1 : 0;
        ps->blur_pairs = blur_pairs ? 1 : 0;
        ps->tile_w = B.tile_w ? B.tile_w : 16;
        return PGPU_OK;
    }
}

// The rest of a pass once st has run it: statuses, learned ratios, statistics.  Images
// whose range overflowed are listed in *failed, with the larger range to use in *cap_next
// (when given); their output is untouched (the slice skips them), while every other image
// of the pass is finished.
static int finish_pass(Engine& E, const BatchJob& B, const PassState& ps, std::vector<int>* failed,
                       std::vector<uint64_t>* cap_next) {
    const int d = B.d, nseg = (int)B.items.size();
    if (nseg == 0) return PGPU_OK;
    const unsigned char* h = ps.h;
    const uint32_t M = ((const uint32_t*)h)[1];
    const unsigned* segstat = (const unsigned*)(h + ps.segstat);
    const uint32_t* counts = (const uint32_t*)(h + ps.counts);
    bool retry = false;
    for (int k = 0; k < nseg; ++k) {
        if (segstat[k] & kStatusKeyRange)
            return fail(PGPU_ERR_ARGUMENT,
                        "image %d: positions leave the lattice's int16 key range (the reference's "
                        "keys wrap there and its rank indices leave [0, d]); scale them down", k);
        if (segstat[k] & (kStatusProbeLimit | kStatusSpinLimit)) {
            uint64_t c = std::max<uint64_t>((uint64_t)(ps.cap[k] * 2.5), (uint64_t)(counts[k] / ps.load * 2));
            failed->push_back(k);
            if (cap_next) cap_next->push_back((c + 31) & ~31ull);
            retry = true;
        }
    }

    double rmax = 0.0;
    uint64_t done_vertices = 0;
    size_t fi = 0;
    {
        std::lock_guard<std::mutex> lk(g_ratio_mu);
        if (g_ratio_by_sig.size() > 4096) g_ratio_by_sig.clear();
        for (int k = 0; k < nseg; ++k) {
            if (fi < failed->size() && (*failed)[fi] == k) {
                ++fi;
                continue;
            }
            done_vertices += counts[k];
            if (!B.items[k].n) continue;
            const double r = (double)counts[k] / (double)B.items[k].n;
            g_ratio_by_sig[ps.sig[k]] = r;
            rmax = std::max(rmax, r);
        }
        if (!retry) g_ratio[d] = rmax;
    }
    E.last_cap = ps.cap_total;
    if (B.vertices_out && !retry) B.vertices_out->assign(counts, counts + nseg);

    pgpu_stats s;
    memset(&s, 0, sizeof(s));
    s.points = (long long)ps.n_total;
    s.vertices = retry ? (long long)done_vertices : (long long)M;
    s.capacity = (long long)ps.cap_total;
    s.d = d;
    s.vd = B.vd;
    s.payload = B.payload;
    s.retries = ps.pass;
    s.load_factor = ps.load;
    s.blur_pairs = ps.blur_pairs;
    s.blur_grid = B.blur_grid;
    s.nbr_half = ps.nbr_half;
    s.vertex_rows = ps.vertex_rows;
    s.tile_w = ps.tile_w;
    s.tiled = ps.tiled;
    if (ps.timed == 1) {
        cudaEventElapsedTime(&s.ms_splat, E.ev[0], E.ev[1]);
        cudaEventElapsedTime(&s.ms_compact, E.ev[1], E.ev[2]);
        cudaEventElapsedTime(&s.ms_neighbours, E.ev[2], E.ev[3]);
        cudaEventElapsedTime(&s.ms_blur, E.ev[3], E.ev[4]);
        cudaEventElapsedTime(&s.ms_slice, E.ev[4], E.ev[5]);
        cudaEventElapsedTime(&s.ms_total, E.ev[6], E.ev[5]);
    } else if (ps.timed == 2) {
        cudaEventElapsedTime(&s.ms_total, E.ev[0], E.ev[5]);
    }
    set_stats(s);
    return PGPU_OK;
}

static int run_batch_pass(Engine& E, const BatchJob& B, cudaStream_t st,
                          const std::vector<uint64_t>* cap_in, std::vector<int>* failed,
                          std::vector<uint64_t>* cap_next, int pass) {
    if (B.items.empty()) return PGPU_OK;
    PassState ps;
    int rc;
    if ((rc = enqueue_pass(E, B, st, cap_in, nullptr, true, pass, &ps))) return rc;
    CUDA_TRY(cudaStreamSynchronize(st));
    return finish_pass(E, B, ps, failed, cap_next);
}

// Autotuner: coordinate descent over six knobs, starting from load 0.5, the tile splat,
// slot-space rows, two neighbour lookups, blur axes in pairs and the capped blur grid.
// Each knob's options are tried with the best setting found so far for the other knobs,
// each twice (the faster time counts: the first call of a shape also learns its vertex
// ratio), by the device time of what the knob changes (knob_time):
//   0. hash-table load factor 0.5 / 0.35 / 0.7;
//   1. splat: the tile splat wherever the learned vertex density allows it, or the direct
//      splat for every image;
//   2. rows: in slot space with a compaction into vertex order, or numbered by the tile
//      splat as it creates the vertices, in vertex order from the start (where every image
//      of the batch takes the tile splat);
//   3. neighbour search: one lookup per axis (n1), the other pair entry written by the
//      neighbour found (n2(n1(v)) = v), or two lookups per axis;
//   4. blur passes: axes fused in pairs, or one axis per pass (16-bit payloads: rows kept
//      in FP32 after every first axis of a would-be pair and rounded to 16 bits after the
//      second, as a pair rounds them, so the results are the same bit for bit);
//   5. blur grid: 16 blocks per SM striding over the vertices, one vertex per thread, or
//      (one-axis passes) 16 blocks per SM with two vertices per iteration;
//   6. tile splat tiles (the blocks per image): 16x16 or 32x8 pixels (splat time).
// Keys, vertex order and FP32/FP64 results do not depend on the choice.
constexpr float kTuneLoads[] = {0.5f, 0.35f, 0.7f};
constexpr int kTuneKnobs = 7;
constexpr int kTuneReps = 2;

// knobs in the order they are walked: 0 load, 1 splat kernel, 2 rows, 3 neighbour search,
// 4 blur pairing, 5 blur grid (the blur's best form depends on the row layout), 6 tiles
static int knob_options(int k) { return k == 0 || k == 5 ? 3 : 2; }

static Engine::Tuning::Setting with_option(Engine::Tuning::Setting s, int k, int o) {
    switch (k) {
    case 0: s.load = kTuneLoads[o]; break;
    case 1: s.splat = o; break;
    case 2: s.vertex_rows = o; break;
    case 3: s.nbr_half = o; break;
    case 4: s.pairs = o == 0; break;
    case 5: s.blur_grid = o; break;
    case 6: s.tile_w = o == 0 ? 16 : 32; break;
    }
    return s;
}

static bool same_setting(const Engine::Tuning::Setting& a, const Engine::Tuning::Setting& b) {
    return a.load == b.load && a.pairs == b.pairs && a.blur_grid == b.blur_grid && a.splat == b.splat &&
           a.vertex_rows == b.vertex_rows && a.nbr_half == b.nbr_half && a.tile_w == b.tile_w;
}

// the next setting to try (skipping options that are the best setting itself, already
// timed, and options the payload does not allow); false once every knob is done
static bool tune_next(Engine::Tuning& t, bool singles_ok, Engine::Tuning::Setting* out) {
    while (t.knob < kTuneKnobs) {
        if (t.option >= knob_options(t.knob)) {
            ++t.knob;
            t.option = 0;
            continue;
        }
        const Engine::Tuning::Setting c = with_option(t.best, t.knob, t.option);
        const bool timed_already = t.best_ms < 1e29f && same_setting(c, t.best);
        // two vertices per blur iteration exist for one-axis passes only
        if (timed_already || (!singles_ok && !c.pairs) || (c.pairs && c.blur_grid == 2)) {
            ++t.option;
            continue;
        }
        *out = c;
        return true;
    }
    t.done = true;
    return false;
}

// The time a knob is judged by: the blur's for the blur knobs, the splat's and the
// neighbour search's for the neighbour search (its pairs are marked absent by the splat),
// the whole lattice's for the others — a knob that changes one stage is judged without the
// other stages' noise.  Stage times exist for calls without a graph; with a graph every
// knob is judged by the whole lattice.
static float knob_time(int knob, float total, const float (&stage)[3]) {
    const bool staged = stage[0] > 0.0f && stage[0] < 1e29f;
    if (!staged) return total;
    if (knob == 4 || knob == 5) return stage[2];
    if (knob == 3) return stage[0] + stage[1];
    if (knob == 6) return stage[0];
    return total;
}

static void tune_record(Engine::Tuning& t, const Engine::Tuning::Setting& c, const pgpu_stats& s) {
    ++t.trials;
    const float st[3] = {s.ms_splat, s.ms_neighbours, s.ms_blur};
    t.cur_ms = std::min(t.cur_ms, s.ms_total);
    for (int i = 0; i < 3; ++i) t.cur_stage[i] = std::min(t.cur_stage[i], st[i]);
    if (++t.rep < kTuneReps) return;
    const bool first = t.best_ms >= 1e29f;
    if (first || knob_time(t.knob, t.cur_ms, t.cur_stage) < knob_time(t.knob, t.best_ms, t.best_stage)) {
        t.best_ms = t.cur_ms;
        for (int i = 0; i < 3; ++i) t.best_stage[i] = t.cur_stage[i];
        t.best = c;
    }
    t.cur_ms = 1e30f;
    for (float& x : t.cur_stage) x = 1e30f;
    t.rep = 0;
    ++t.option;
}

static std::string tune_key(const BatchJob& B) {
    uint64_t n = 0;
    for (const BatchItem& it : B.items) n += it.n;
    int lg = 0;
    while ((1ull << lg) < n) ++lg;
    char buf[96];
    snprintf(buf, sizeof(buf), "%d:%d:%d:%d:%d:%zu:%d", B.d, B.vd, B.payload, (int)B.homog,
             (int)B.replay, B.items.size(), lg);
    return buf;
}

static bool tunable(const BatchJob& B) { return B.autotune && !B.rec_vtx && !B.dump_splat; }
// 16-bit payloads blur one axis per pass with the pairs' rounding (bit-identical) from
// d = 2 up (three or more axes)
static bool singles_allowed(const BatchJob& B) {
    return (B.payload != kPayloadF16 && B.payload != kPayloadBF16) || B.d >= 2;
}
static void apply_setting(BatchJob& B, const Engine::Tuning::Setting& s) {
    B.load = s.load;
    B.blur_pairs = s.pairs;
    B.blur_grid = s.blur_grid;
    B.splat = s.splat;
    B.slot_rows = !s.vertex_rows;
    B.nbr_half = s.nbr_half;
    B.tile_w = s.tile_w;
}

bool tuned_settings(Engine& E, const BatchJob& B, BatchJob* out) {
    *out = B;
    if (!tunable(B)) return true;
    auto it = E.tuning.find(tune_key(B));
    if (it == E.tuning.end() || !it->second.done) return false;
    apply_setting(*out, it->second.best);
    return true;
}

int enqueue_batch(Engine& E, const BatchJob& B, cudaStream_t st, unsigned char* h, PassState* ps) {
    return enqueue_pass(E, B, st, nullptr, h, false, 0, ps);
}

int finish_batch(Engine& E, const BatchJob& B, const PassState& ps, std::vector<int>* failed) {
    return finish_pass(E, B, ps, failed, nullptr);
}

// The passes of one batch with fixed settings: images whose range overflowed go again,
// as a smaller batch with larger ranges.  *sum covers all passes.
static int run_passes(Engine& E, BatchJob cur, cudaStream_t st, pgpu_stats* sum) {
    const int d = cur.d, n0 = (int)cur.items.size();
    std::vector<uint64_t> caps;
    memset(sum, 0, sizeof(*sum));
    for (int pass = 0; pass < 6; ++pass) {
        std::vector<int> failed;
        std::vector<uint64_t> next;
        const int rc = run_batch_pass(E, cur, st, caps.empty() ? nullptr : &caps, &failed, &next, pass);
        if (rc) return rc;
        pgpu_stats s;
        if (get_stats(&s)) {
            if (pass == 0) sum->points = s.points, sum->d = s.d, sum->vd = s.vd, sum->payload = s.payload;
            sum->vertices += s.vertices;
            sum->capacity = std::max(sum->capacity, s.capacity);
            sum->retries = pass;
            sum->ms_splat += s.ms_splat, sum->ms_compact += s.ms_compact;
            sum->ms_neighbours += s.ms_neighbours, sum->ms_blur += s.ms_blur;
            sum->ms_slice += s.ms_slice, sum->ms_total += s.ms_total;
            if (pass == 0) sum->tiled = s.tiled;
        }
        if (failed.empty()) {
            sum->load_factor = s.load_factor;
            sum->blur_pairs = s.blur_pairs;
            sum->blur_grid = s.blur_grid;
            sum->nbr_half = s.nbr_half;
            sum->vertex_rows = s.vertex_rows;
            sum->tile_w = s.tile_w;
            return PGPU_OK;
        }
        BatchJob again = cur;
        again.items.clear();
        for (int k : failed) again.items.push_back(cur.items[k]);
        caps = next;
        cur = std::move(again);
    }
    return fail(PGPU_ERR_CAPACITY, "hash table overfull after retries (d=%d, %d images)", d, n0);
}

// Every image of a batch is filtered in place, so an image whose range overflowed cannot
// simply be rerun with its whole batch: the others are finished.  Only the overflowed
// ones go again (run_passes).  Vertex-ordered rows need every image of the launches on
// the tile splat; a batch that asks for them but has images for the direct splat runs as
// two, the tile-splat images with vertex-ordered rows, the others with slot-space rows.
int run_batch(Engine& E, const BatchJob& B, cudaStream_t st) {
    if (B.items.empty()) return PGPU_OK;
    BatchJob cur = B;
    Engine::Tuning* tune = nullptr;
    Engine::Tuning::Setting trial;
    if (tunable(B)) {
        if (E.tuning.size() > 1024) E.tuning.clear();
        Engine::Tuning& t = E.tuning[tune_key(B)];
        if (!t.done && tune_next(t, singles_allowed(B), &trial)) {
            tune = &t;
            apply_setting(cur, trial);
        } else {
            apply_setting(cur, t.best);
        }
    }
    const int nseg = (int)cur.items.size();
    std::vector<char> tiled(nseg, 0);
    int nt = 0;
    if (nseg > 1 && vertex_rows_wanted(cur)) {
        std::vector<uint64_t> sig;
        std::vector<double> ratio, density;
        learned_ratios(cur, &sig, &ratio, &density);
        const int forced = splat_forced();
        for (int k = 0; k < nseg; ++k) nt += (tiled[k] = tile_splat_for(cur, forced, density[k], cur.items[k].n)) ? 1 : 0;
    }
    pgpu_stats sum;
    int rc;
    if (nt > 0 && nt < nseg) {
        BatchJob a = cur, b = cur;
        a.items.clear();
        b.items.clear();
        b.slot_rows = true;
        for (int k = 0; k < nseg; ++k) (tiled[k] ? a : b).items.push_back(cur.items[k]);
        pgpu_stats sa, sb;
        if ((rc = run_passes(E, a, st, &sa)) || (rc = run_passes(E, b, st, &sb))) return rc;
        sum = sa;
        sum.points += sb.points, sum.vertices += sb.vertices;
        sum.capacity = std::max(sum.capacity, sb.capacity);
        sum.retries = std::max(sum.retries, sb.retries);
        sum.ms_splat += sb.ms_splat, sum.ms_compact += sb.ms_compact;
        sum.ms_neighbours += sb.ms_neighbours, sum.ms_blur += sb.ms_blur;
        sum.ms_slice += sb.ms_slice, sum.ms_total += sb.ms_total;
        sum.tiled += sb.tiled;
    } else if ((rc = run_passes(E, cur, st, &sum))) {
        return rc;
    }
    sum.tuned = tune ? 1 : tunable(B) ? 2 : 0;
    if (tune) tune_record(*tune, trial, sum);
    set_stats(sum);
    return PGPU_OK;
}

}  // namespace pgpu
