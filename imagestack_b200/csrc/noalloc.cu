// Bilateral filtering without any device allocation, for callers that cannot allocate.
//
// Some hosts own all device memory themselves: a render or video pipeline that reserved
// its pool at start-up, a plugin running inside another framework's allocator, or a
// latency-bound loop that must not stall the device (cudaMalloc and cudaFree synchronise
// it).  pgpu_bilateral_noalloc serves them: it runs the same lattice kernels as
// pgpu_bilateral, but every intermediate (hash table, vertex arrays, neighbours, the
// vertex numbering and the status word) lives in one file-scope device array of fixed
// size, so a call makes no cudaMalloc, cudaFree, cudaHostAlloc or other allocating call.
//
// Limits that follow from the fixed array: one frame, up to kNoAllocMaxPixels pixels and
// kNoAllocMaxChannels channels, FP32 values, and a lattice of at most kNoAllocSlots
// vertices' worth of hash slots (a frame that needs more is rejected, not truncated).
#include <cuda_runtime.h>

#include <cstring>

#include "engine.h"

namespace pgpu {
namespace {

constexpr int kNoAllocMaxPixels = 512 * 512;
constexpr int kNoAllocMaxChannels = 3;                 // d = channels + 2 <= 5, 4 values
constexpr int kNoAllocMaxD = kNoAllocMaxChannels + 2;
constexpr int kNoAllocVdp = 4;
constexpr uint32_t kNoAllocSlots = 3u << 17;           // hash slots (and vertex rows)
constexpr size_t kAlign = 256;

constexpr size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// layout of the scratch array
constexpr size_t kEntries = (size_t)kNoAllocMaxPixels * (kNoAllocMaxD + 1);
constexpr size_t kWords = (kEntries + 31) / 32;
constexpr size_t kParts = (kWords + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
constexpr size_t kOffStatus = 0;                                      // status, vertex count
constexpr size_t kOffSeg = align_up(kOffStatus + 64);                 // the image's descriptor
constexpr size_t kOffSlotBase = align_up(kOffSeg + sizeof(Segment));  // its slot range
constexpr size_t kOffKey0 = align_up(kOffSlotBase + 16);
constexpr size_t kOffTvals = align_up(kOffKey0 + (size_t)kNoAllocSlots * 16);
constexpr size_t kOffFt = align_up(kOffTvals + (size_t)kNoAllocSlots * kNoAllocVdp * 4);
constexpr size_t kOffSlot2Vtx = align_up(kOffFt + (size_t)kNoAllocSlots * 4);
constexpr size_t kOffBitmap = align_up(kOffSlot2Vtx + (size_t)kNoAllocSlots * 4);
constexpr size_t kOffOffs = align_up(kOffBitmap + kWords * 4);
constexpr size_t kOffParts = align_up(kOffOffs + kWords * 4);
constexpr size_t kOffVkey0 = align_up(kOffParts + kParts * 4 + 16);
constexpr size_t kOffVv0 = align_up(kOffVkey0 + (size_t)kNoAllocSlots * 16);
constexpr size_t kOffVv1 = align_up(kOffVv0 + (size_t)kNoAllocSlots * kNoAllocVdp * 4);
constexpr size_t kOffNbr = align_up(kOffVv1 + (size_t)kNoAllocSlots * kNoAllocVdp * 4);
constexpr size_t kOffVtx2Slot = align_up(kOffNbr + (size_t)(kNoAllocMaxD + 1) * kNoAllocSlots * 8);
constexpr size_t kOffSval = align_up(kOffVtx2Slot + (size_t)kNoAllocSlots * 4);
constexpr size_t kOffRec = align_up(kOffSval + (size_t)kNoAllocSlots * kNoAllocVdp * 4);
constexpr size_t kUsed = align_up(kOffRec + kEntries * 4);

// 72 MiB, held by every GPU that loads this part of the library until the process exits
constexpr size_t kScratchBytes = 72ull << 20;
static_assert(kUsed <= kScratchBytes, "no-alloc scratch layout does not fit");

// In host code this name is only a host-side stand-in for the device array: never pass
// it to a kernel; pass the address cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array in the current context.  Looked up on every call
// (the lookup allocates nothing): a cached address would go stale if the context were
// destroyed and recreated (cudaDeviceReset, a host that recreates its primary context),
// because the module, and with it the array, is then loaded again at a new address.
int scratch_address(int dev, unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(PGPU_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch) failed on device %d: %s",
                    dev, cudaGetErrorString(e));
    *out = (unsigned char*)p;
    return PGPU_OK;
}

}  // namespace
}  // namespace pgpu

using namespace pgpu;

extern "C" int pgpu_bilateral_noalloc(const float* d_in, float* d_out, int width, int height,
                                      int channels, float filter_width, float filter_height,
                                      float color_sigma, void* stream) {
    clear_error();
    if (!d_in || !d_out) return fail(PGPU_ERR_ARGUMENT, "null image pointer");
    if (width < 2 || height < 2 || channels < 1)
        return fail(PGPU_ERR_ARGUMENT, "image must be at least 2x2 with one channel");
    if ((long long)width * height > kNoAllocMaxPixels || channels > kNoAllocMaxChannels)
        return fail(PGPU_ERR_UNSUPPORTED,
                    "pgpu_bilateral_noalloc takes at most %d pixels and %d channels "
                    "(got %dx%d, %d channels); use pgpu_bilateral for larger images",
                    kNoAllocMaxPixels, kNoAllocMaxChannels, width, height, channels);
    if (!(filter_width > 0) || !(filter_height > 0) || !(color_sigma > 0) ||
        !(filter_width < 10 * width) || !(filter_height < 10 * height))
        return fail(PGPU_ERR_UNSUPPORTED,
                    "pgpu_bilateral_noalloc filters both pixel axes: it needs 0 < filter width "
                    "< 10 x width and 0 < filter height < 10 x height");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return fail(PGPU_ERR_NO_DEVICE, "no current CUDA device");
    }
    int major = 0, sms = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        major != 10)
        return fail(PGPU_ERR_NO_DEVICE, "device %d is not an sm_100 (B200) GPU", dev);
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t st = (cudaStream_t)stream;
    // The call waits for its stream and uploads its descriptor from the host stack, so it
    // cannot be recorded into a CUDA graph: refuse it while the stream is capturing.
    cudaStreamCaptureStatus cap_status = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(st, &cap_status));
    if (cap_status != cudaStreamCaptureStatusNone)
        return fail(PGPU_ERR_UNSUPPORTED,
                    "pgpu_bilateral_noalloc cannot run inside a stream capture (it waits for its "
                    "stream and uploads its descriptor from host memory)");
    unsigned char* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc) return rc;

    const int d = channels + 2;
    const int vd = channels + 1;
    const int vdp = vdp_for(vd);
    const uint32_t n = (uint32_t)(width * height);
    const uint32_t nwords = (uint32_t)(((uint64_t)n * (d + 1) + 31) / 32);
    const uint32_t cap = kNoAllocSlots;
    unsigned* dstatus = (unsigned*)(base + kOffStatus);
    uint32_t* dM = (uint32_t*)(base + kOffStatus) + 1;

    // every call starts from an empty table: the array keeps the previous call's contents
    CUDA_TRY(cudaMemsetAsync(base + kOffStatus, 0, 64, st));
    CUDA_TRY(cudaMemsetAsync(base + kOffKey0, 0xFF, (size_t)cap * 16, st));
    CUDA_TRY(cudaMemsetAsync(base + kOffTvals, 0, (size_t)cap * vdp * 4, st));
    CUDA_TRY(cudaMemsetAsync(base + kOffFt, 0xFF, (size_t)cap * 4, st));
    CUDA_TRY(cudaMemsetAsync(base + kOffBitmap, 0, (size_t)nwords * 4, st));

    // positions (c * 1/sigma_r ..., x * 1/sigma_s, y * 1/sigma_s), values (c ..., 1): the
    // single-frame JointBilateral::apply with the image as its own reference
    const long long plane = (long long)width * height;
    PointSource src;
    memset(&src, 0, sizeof(src));
    src.width = width;
    src.height = height;
    src.frames = 1;
    src.pos = PlanarView{d_in, width, plane, plane};
    src.pos_channels = channels;
    volatile float one = 1.0f;
    const float inv_r = one / color_sigma;
    for (int c = 0; c < channels; ++c) src.pos_scale[c] = inv_r;
    src.coord_mask = 3;
    src.coord_scale[0] = one / filter_width;
    src.coord_scale[1] = one / filter_height;
    src.val = PlanarView{d_in, width, plane, plane};
    src.val_channels = channels;
    src.homogeneous = 1;

    const DimOps* ops = dim_ops(d);
    const LatticeConsts lc = make_consts(d);

    // the image is a batch of one: its descriptor and slot range go to the array too
    Segment seg;
    memset(&seg, 0, sizeof(seg));
    seg.src = src;
    seg.out.base = d_out;
    seg.out.ystride = width;
    seg.out.tstride = plane;
    seg.out.cstride = plane;
    seg.out.channels = channels;
    seg.out.normalize = 1;
    seg.n = n;
    seg.cap = cap;
    uint32_t splat_blocks = 0, tile_blocks = 0, slice_blocks = 0;
    segment_geometry(seg, src, false, &splat_blocks, &tile_blocks, &slice_blocks);
    const uint32_t slot_bounds[2] = {0u, cap};
    CUDA_TRY(cudaMemcpyAsync(base + kOffSeg, &seg, sizeof(seg), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(base + kOffSlotBase, slot_bounds, sizeof(slot_bounds),
                             cudaMemcpyHostToDevice, st));
    const Segment* dseg = (const Segment*)(base + kOffSeg);
    uint4* key0 = (uint4*)(base + kOffKey0);

    SplatArgs sa;
    sa.segs = dseg;
    sa.nseg = 1;
    sa.n_total = n;
    sa.lc = lc;
    sa.key0 = key0;
    sa.keyn = key0;
    sa.cap_total = cap;
    sa.vals = base + kOffTvals;
    sa.ft = (uint32_t*)(base + kOffFt);
    sa.rec_slot = (uint32_t*)(base + kOffRec);
    sa.seg_status = dstatus;
    sa.blocks = splat_blocks;
    sa.tile_blocks = 0;
    sa.rec_w = nullptr;   // the slice recomputes the weights
    sa.vlist = nullptr;   // vertices numbered by first touch (mark, scan, assign below)
    sa.vcount = nullptr;
    sa.seg_counts = nullptr;
    if (!ops->splat(sa, vdp, kPayloadF32, st)) return fail(PGPU_ERR_UNSUPPORTED, "splat variant");
    CUDA_TRY(cudaGetLastError());

    launch_mark((const uint32_t*)(base + kOffFt), cap, (uint32_t*)(base + kOffBitmap), sms, st);
    launch_scan((const uint32_t*)(base + kOffBitmap), nwords, (uint32_t*)(base + kOffParts),
                (uint32_t*)(base + kOffOffs), dM, st);
    CompactArgs ca;
    memset(&ca, 0, sizeof(ca));
    ca.table = TableView{key0, key0, cap, cap};
    ca.ft = (const uint32_t*)(base + kOffFt);
    ca.bitmap = (uint32_t*)(base + kOffBitmap);
    ca.nwords = nwords;
    ca.offs = (const uint32_t*)(base + kOffOffs);
    ca.slot2vtx = (uint32_t*)(base + kOffSlot2Vtx);
    ca.vtx2slot = (uint32_t*)(base + kOffVtx2Slot);
    ca.vkey0 = (uint4*)(base + kOffVkey0);
    ca.vkeyn = (uint4*)(base + kOffVkey0);
    ca.vcap = cap;
    ca.tvals = base + kOffTvals;
    ca.vvals = base + kOffVv0;
    ca.wc = vd - 1;
    ca.index_in_key = index_in_key(d) ? 1 : 0;   // the neighbour lookups expect it
    if (!launch_assign(ca, 1, vdp, kPayloadF32, false, sms, st))
        return fail(PGPU_ERR_UNSUPPORTED, "assign variant");

    NbrArgs na;
    na.seg_status = dstatus;
    na.key0 = key0;
    na.keyn = key0;
    na.cap_total = cap;
    na.seg_slot_base = (const uint32_t*)(base + kOffSlotBase);
    na.nseg = 1;
    na.vtx2slot = (const uint32_t*)(base + kOffVtx2Slot);
    na.slot2vtx = (const uint32_t*)(base + kOffSlot2Vtx);
    na.vkey0 = (const uint4*)(base + kOffVkey0);
    na.vkeyn = (const uint4*)(base + kOffVkey0);
    na.vcap = cap;
    na.nverts = dM;
    na.nbr = (int2*)(base + kOffNbr);
    ops->neighbours(na, cap, sms, st);

    BlurPlan bp;
    bp.d = d;
    bp.vdp = vdp;
    bp.payload = kPayloadF32;
    bp.homog = false;
    bp.src_f32 = false;
    bp.nbr = (const int2*)(base + kOffNbr);
    bp.nbr_stride = cap;
    bp.nverts = dM;
    bp.vmax = cap;
    bp.src = base + kOffVv0;
    bp.bufs[0] = base + kOffVv1;
    bp.bufs[1] = base + kOffVv0;
    bp.sval = base + kOffSval;
    bp.vtx2slot = (const uint32_t*)(base + kOffVtx2Slot);
    bp.wc = vd - 1;
    bp.sms = sms;
    if (blur_all_axes(bp, st)) return fail(PGPU_ERR_UNSUPPORTED, "blur variant");

    SliceArgs sl;
    memset(&sl, 0, sizeof(sl));
    sl.segs = dseg;
    sl.nseg = 1;
    sl.n_total = n;
    sl.lc = lc;
    sl.key0 = key0;
    sl.keyn = key0;
    sl.cap_total = cap;
    sl.slot2vtx = (const uint32_t*)(base + kOffSlot2Vtx);
    sl.rec_slot = (const uint32_t*)(base + kOffRec);
    sl.svals = base + kOffSval;
    sl.vd = vd;
    sl.seg_status = dstatus;
    sl.blocks = slice_blocks;
    if (!ops->slice(sl, vdp, kPayloadF32, false, st)) return fail(PGPU_ERR_UNSUPPORTED, "slice variant");
    CUDA_TRY(cudaGetLastError());

    unsigned hstatus[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(hstatus, base + kOffStatus, sizeof(hstatus), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (hstatus[0] & kStatusKeyRange)
        return fail(PGPU_ERR_ARGUMENT, "positions leave the lattice's int16 key range");
    if (hstatus[0] & (kStatusProbeLimit | kStatusSpinLimit))
        return fail(PGPU_ERR_CAPACITY,
                    "the lattice of this image needs more than the %u hash slots of the fixed "
                    "no-alloc scratch; d_out was not written", cap);
    return PGPU_OK;
}
