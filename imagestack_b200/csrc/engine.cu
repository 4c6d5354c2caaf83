// Host side of the lattice: per-device workspace, the launch sequence of one lattice,
// the operation logic of ImageStack's GaussTransform / JointBilateral / Bilateral for
// the permutohedral method, and the C ABI declared in include/permgpu.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>

#include "engine.h"

namespace pgpu {

// ---------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------
static thread_local std::string t_error;
static thread_local pgpu_stats t_stats;
static thread_local bool t_have_stats = false;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_error = buf;
    return code;
}

void clear_error() { t_error.clear(); }
const char* last_error() { return t_error.c_str(); }
void set_stats(const pgpu_stats& s) { t_stats = s; t_have_stats = true; }
bool get_stats(pgpu_stats* s) { if (t_have_stats) *s = t_stats; return t_have_stats; }

// ---------------------------------------------------------------------------------
// buffers and engines
// ---------------------------------------------------------------------------------
static thread_local cudaStream_t t_call_stream = nullptr;
void set_call_stream(cudaStream_t st) { t_call_stream = st; }
cudaStream_t call_stream() { return t_call_stream; }

// The library's own stream-ordered memory pool of each device.  It keeps the memory that
// buffers give back (release threshold: unlimited), so a workspace that grows under load
// (the server's workers) is served from the pool instead of new driver allocations, and
// the device's default pool, which the host application may use, is left as it is.
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

static cudaMemPool_t device_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[dev] = pool;
    return pool;
}

// Make the library's pool on the current device hold `bytes` of device memory (at most
// half of what is free): one allocation of that size, freed at once, stays in the pool
// (its release threshold is unlimited), so buffers that grow later are served from memory
// the pool holds instead of mapping new memory while work is running.
int reserve_pool_memory(size_t bytes, cudaStream_t st) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return PGPU_OK;
    }
    bytes = std::min(bytes, free_b / 2);
    cudaMemPool_t pool = device_pool();
    if (!pool || bytes == 0) return PGPU_OK;
    size_t held = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &held) == cudaSuccess && held >= bytes)
        return PGPU_OK;
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes, pool, st) != cudaSuccess) {
        cudaGetLastError();   // a reservation that does not fit is skipped, not an error
        return PGPU_OK;
    }
    CUDA_TRY(cudaFreeAsync(p, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return PGPU_OK;
}

// Every call is synchronous, so when a buffer grows (at the start of a call) no earlier
// work still uses the old block, whichever stream it ran on.
int DevBuf::ensure(size_t need) {
    if (need == 0) need = 16;
    if (need <= bytes) return PGPU_OK;
    const cudaStream_t st = t_call_stream;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
    const size_t nb = need + need / 2;
    cudaMemPool_t pool = device_pool();
    const cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, nb, pool, st) : cudaMallocAsync(&p, nb, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return fail(PGPU_ERR_MEMORY, "device allocation of %zu bytes failed", nb);
    }
    bytes = nb;
    return PGPU_OK;
}

// released when no work uses the buffer any more (calls are synchronous); the free is
// queued on the legacy stream, which outlives every engine stream
void DevBuf::release() {
    if (p) cudaFreeAsync(p, cudaStreamLegacy);
    p = nullptr;
    bytes = 0;
}

DevBuf::~DevBuf() { release(); }

int device_count_sm100() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int good = 0;
    for (int i = 0; i < n; ++i) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, i) == cudaSuccess && p.major == 10) ++good;
    }
    return good;
}

int Engine::init(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || dev < 0 || dev >= n) {
        cudaGetLastError();
        return fail(PGPU_ERR_NO_DEVICE, "no CUDA device %d (this library has no CPU path)", dev);
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10)
        return fail(PGPU_ERR_NO_DEVICE, "device %d is not an sm_100 (B200) GPU", dev);
    CUDA_TRY(cudaSetDevice(dev));
    device = dev;
    sms = prop.multiProcessorCount;
    CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaHostAlloc((void**)&hstat, 64, cudaHostAllocDefault));
    for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
    for (auto& e : join_ev) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return PGPU_OK;
}

static std::mutex g_engines_mu;
static std::map<int, std::unique_ptr<Engine>> g_engines;

int get_engine(int dev, Engine** out) {
    std::lock_guard<std::mutex> lk(g_engines_mu);
    auto it = g_engines.find(dev);
    if (it != g_engines.end()) {
        *out = it->second.get();
        return PGPU_OK;
    }
    std::unique_ptr<Engine> e(new Engine());
    const int rc = e->init(dev);
    if (rc != PGPU_OK) return rc;
    *out = e.get();
    g_engines[dev] = std::move(e);
    return PGPU_OK;
}

// ---------------------------------------------------------------------------------
// lattice constants, computed in single precision in the order of the reference
// constructor (src/Permutohedral.h:257-274) and of `scale` (:301).  This file is
// compiled without fast-math and with -ffp-contract=off on the host side.
// ---------------------------------------------------------------------------------
LatticeConsts make_consts(int d) {
    LatticeConsts lc;
    memset(&lc, 0, sizeof(lc));
    for (int i = 0; i < d; i++) {
        volatile float s = 1.0f / (sqrtf((float)(i + 1) * (i + 2)));
        volatile float m = (float)(d + 1) * sqrtf((float)(2.0 / 3));
        lc.sf[i] = s * m;
    }
    volatile float one = 1.0f;
    lc.inv_d1 = one / (float)(d + 1);
    return lc;
}

int vdp_for(int vd) { return vd <= 2 ? 2 : vd <= 4 ? 4 : vd <= 8 ? 8 : 0; }

// ---------------------------------------------------------------------------------
// one lattice: splat, compact, neighbours, blur, slice
// ---------------------------------------------------------------------------------
int run_lattice(Engine& E, const LatticeJob& J, cudaStream_t st) {
    if (J.method == PGPU_METHOD_GRID) {
        if (J.rec_vtx || J.dump_splat) return fail(PGPU_ERR_UNSUPPORTED, "the grid method has no lattice dumps");
        return run_grid(E, J, st);
    }
    if (J.method != PGPU_METHOD_PERMUTOHEDRAL) return fail(PGPU_ERR_ARGUMENT, "unknown method %d", J.method);
    BatchJob B;
    B.d = J.d;
    B.vd = J.vd;
    B.payload = J.payload;
    B.load = J.load;
    B.homog = J.homog;
    B.replay = J.replay;
    BatchItem it;
    it.splat = J.splat;
    it.n = J.n;
    it.slice = J.slice;
    it.n_slice = J.n_slice;
    it.out = J.out;
    B.items.push_back(it);
    B.rec_vtx = J.rec_vtx;
    B.rec_w = J.rec_w;
    B.dump_splat = J.dump_splat;
    B.dump_bytes = J.dump_bytes;
    std::vector<uint32_t> counts;
    B.vertices_out = &counts;
    const int rc = run_batch(E, B, st);
    if (rc == PGPU_OK && J.vertices_out) *J.vertices_out = counts.empty() ? 0 : counts[0];
    return rc;
}

// ---------------------------------------------------------------------------------
// views and host staging
// ---------------------------------------------------------------------------------
bool view_ok(const pgpu_image* v) {
    return v && v->base && v->width > 0 && v->height > 0 && v->frames > 0 && v->channels > 0 &&
           v->ystride >= v->width && v->tstride >= 0 && v->cstride >= 0;
}

bool points_fit(const pgpu_image* v) {
    return (uint64_t)v->width * (uint64_t)v->height * (uint64_t)v->frames <= 0xFFFFFFFFull;
}

bool same_view(const pgpu_image& a, const pgpu_image& b) {
    return a.base == b.base && a.ystride == b.ystride && a.tstride == b.tstride &&
           a.cstride == b.cstride && a.width == b.width && a.height == b.height &&
           a.frames == b.frames && a.channels == b.channels;
}

bool is_dense(const pgpu_image& v) {
    return v.ystride == v.width && v.tstride == (long long)v.width * v.height &&
           (v.channels == 1 || v.cstride == (long long)v.width * v.height * v.frames);
}

pgpu_image dense_like(const pgpu_image& v, float* base, int channels) {
    pgpu_image d = v;
    d.base = base;
    d.channels = channels;
    d.ystride = v.width;
    d.tstride = (long long)v.width * v.height;
    d.cstride = (long long)v.width * v.height * v.frames;
    return d;
}

int copy_view(const pgpu_image& src, const pgpu_image& dst, int channels, cudaMemcpyKind kind,
              cudaStream_t st) {
    if (is_dense(src) && is_dense(dst)) {
        CUDA_TRY(cudaMemcpyAsync(dst.base, src.base,
                                 sizeof(float) * (size_t)src.width * src.height * src.frames * channels,
                                 kind, st));
        return PGPU_OK;
    }
    if (src.ystride == src.width && dst.ystride == dst.width) {
        // rows follow each other (a range of rows of a dense image): one plain copy per
        // channel and frame, which the copy engines move faster than a pitched copy
        const size_t plane = sizeof(float) * (size_t)src.width * src.height;
        for (int c = 0; c < channels; ++c)
            for (int t = 0; t < src.frames; ++t)
                CUDA_TRY(cudaMemcpyAsync(dst.base + c * dst.cstride + t * dst.tstride,
                                         src.base + c * src.cstride + t * src.tstride, plane, kind, st));
        return PGPU_OK;
    }
    for (int c = 0; c < channels; ++c)
        for (int t = 0; t < src.frames; ++t)
            CUDA_TRY(cudaMemcpy2DAsync(dst.base + c * dst.cstride + t * dst.tstride,
                                       sizeof(float) * dst.ystride,
                                       src.base + c * src.cstride + t * src.tstride,
                                       sizeof(float) * src.ystride, sizeof(float) * src.width,
                                       src.height, kind, st));
    return PGPU_OK;
}

int upload(Engine& E, DevBuf& buf, const pgpu_image& host, pgpu_image* dev, cudaStream_t st) {
    const size_t n = (size_t)host.width * host.height * host.frames * host.channels;
    int rc = buf.ensure(n * sizeof(float));
    if (rc) return rc;
    (void)E;
    *dev = dense_like(host, (float*)buf.p, host.channels);
    return copy_view(host, *dev, host.channels, cudaMemcpyHostToDevice, st);
}

int download(const pgpu_image& dev, const pgpu_image& host, int channels, cudaStream_t st) {
    return copy_view(dev, host, channels, cudaMemcpyDeviceToHost, st);
}

PlanarView planar(const pgpu_image& v) { return PlanarView{v.base, v.ystride, v.tstride, v.cstride}; }

OutView outview(const pgpu_image& v, int channels, int normalize) {
    OutView o;
    o.base = v.base;
    o.ystride = v.ystride;
    o.tstride = v.tstride;
    o.cstride = v.cstride;
    o.channels = channels;
    o.normalize = normalize;
    return o;
}

// ---------------------------------------------------------------------------------
// GaussTransform::apply, PERMUTOHEDRAL (src/GaussTransform.cpp:115-133, 163-226),
// on device views.
// ---------------------------------------------------------------------------------
int gauss_transform_device(Engine& E, const pgpu_image* slice, const pgpu_image& splat,
                           const pgpu_image& values, const float* sigmas, int n_sigmas,
                           const pgpu_image& out, int payload, float load, cudaStream_t st,
                           int method) {
    if (splat.width != values.width || splat.height != values.height || splat.frames != values.frames)
        return fail(PGPU_ERR_ARGUMENT, "Weights and locations of the Gaussians must be the same size");
    const bool replay = !slice || same_view(*slice, splat);
    if (!replay && slice->channels != splat.channels)
        return fail(PGPU_ERR_ARGUMENT,
                    "The evaluation locations and the locations of the Gaussians must have the same number of channels.");
    if (n_sigmas < splat.channels) return fail(PGPU_ERR_ARGUMENT, "need one sigma per position channel");
    const pgpu_image& sl = replay ? splat : *slice;
    if (out.width != sl.width || out.height != sl.height || out.frames != sl.frames ||
        out.channels < values.channels)
        return fail(PGPU_ERR_ARGUMENT, "output must have the slice positions' size and the values' channels");
    if (splat.channels > kMaxD) return fail(PGPU_ERR_UNSUPPORTED, "%d position dimensions (supported: 1..%d)", splat.channels, kMaxD);

    LatticeJob J;
    J.d = splat.channels;
    J.vd = values.channels;
    J.payload = payload;
    J.load = load;
    J.n = (uint32_t)((size_t)splat.width * splat.height * splat.frames);
    PointSource& s = J.splat;
    memset(&s, 0, sizeof(s));
    s.width = splat.width;
    s.height = splat.height;
    s.frames = splat.frames;
    s.pos = planar(splat);
    s.pos_channels = splat.channels;
    for (int c = 0; c < splat.channels; ++c) {
        volatile float one = 1.0f;
        s.pos_scale[c] = one / sigmas[c];   // invSigma (src/GaussTransform.cpp:131)
    }
    s.val = planar(values);
    s.val_channels = values.channels;
    s.homogeneous = 0;
    J.replay = replay;
    if (!replay) {
        J.slice = s;
        J.slice.width = sl.width;
        J.slice.height = sl.height;
        J.slice.frames = sl.frames;
        J.slice.pos = planar(sl);
        J.n_slice = (uint32_t)((size_t)sl.width * sl.height * sl.frames);
    }
    J.out = outview(out, values.channels, 0);
    J.method = method;
    return run_lattice(E, J, st);
}

// ---------------------------------------------------------------------------------
// JointBilateral::apply with the permutohedral method (src/GaussTransform.cpp:504-678)
// ---------------------------------------------------------------------------------
static pgpu_image region(const pgpu_image& v, int x, int y, int t, int w, int h, int f) {
    pgpu_image r = v;
    r.base = v.base + x + (long long)y * v.ystride + (long long)t * v.tstride;
    r.width = w;
    r.height = h;
    r.frames = f;
    return r;
}

int joint_bilateral_device(Engine& E, const pgpu_image& im, const pgpu_image& ref, float fw,
                           float fh, float ft, float cs, int payload, float load, cudaStream_t st,
                           int method) {
    if (im.width != ref.width || im.height != ref.height || im.frames != ref.frames)
        return fail(PGPU_ERR_ARGUMENT, "Image and reference must be the same size");
    if (im.width == 1) fw = 0;
    if (im.height == 1) fh = 0;
    if (im.frames == 1) ft = 0;
    if (im.width > 1 && fw == 0) {   // each column independently (:516-522)
        for (int x = 0; x < im.width; x++) {
            int rc = joint_bilateral_device(E, region(im, x, 0, 0, 1, im.height, im.frames),
                                            region(ref, x, 0, 0, 1, ref.height, ref.frames), 0, fh,
                                            ft, cs, payload, load, st, method);
            if (rc) return rc;
        }
        return PGPU_OK;
    }
    if (im.height > 1 && fh == 0) {   // each row independently (:524-530)
        for (int y = 0; y < im.height; y++) {
            int rc = joint_bilateral_device(E, region(im, 0, y, 0, im.width, 1, im.frames),
                                            region(ref, 0, y, 0, ref.width, 1, ref.frames), fw, 0,
                                            ft, cs, payload, load, st, method);
            if (rc) return rc;
        }
        return PGPU_OK;
    }
    if (im.frames > 1 && ft == 0) {   // each frame independently (:532-538)
        for (int t = 0; t < im.frames; t++) {
            int rc = joint_bilateral_device(E, region(im, 0, 0, t, im.width, im.height, 1),
                                            region(ref, 0, 0, t, ref.width, ref.height, 1), fw, fh,
                                            0, cs, payload, load, st, method);
            if (rc) return rc;
        }
        return PGPU_OK;
    }
    const bool fx = im.width > 1 && fw < 10 * im.width;
    const bool fy = im.height > 1 && fh < 10 * im.height;
    const bool fz = im.frames > 1 && ft < 10 * im.frames;
    const int d = ref.channels + (fx ? 1 : 0) + (fy ? 1 : 0) + (fz ? 1 : 0);
    if (d > kMaxD) return fail(PGPU_ERR_UNSUPPORTED, "%d position dimensions (supported: 1..%d)", d, kMaxD);
    if (im.channels + 1 > 8) return fail(PGPU_ERR_UNSUPPORTED, "%d image channels (supported: 1..7)", im.channels);

    LatticeJob J;
    J.d = d;
    J.vd = im.channels + 1;
    J.payload = payload;
    J.load = load;
    J.n = (uint32_t)((size_t)im.width * im.height * im.frames);
    PointSource& s = J.splat;
    memset(&s, 0, sizeof(s));
    s.width = im.width;
    s.height = im.height;
    s.frames = im.frames;
    s.pos = planar(ref);
    s.pos_channels = ref.channels;
    volatile float one = 1.0f;
    const float inv_r = one / cs;   // ref / colorSigma == ref * (1.0f/colorSigma) (src/Expr.h:2439-2443)
    for (int c = 0; c < ref.channels; ++c) s.pos_scale[c] = inv_r;
    s.coord_mask = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
    s.coord_scale[0] = fx ? one / fw : 0.0f;
    s.coord_scale[1] = fy ? one / fh : 0.0f;
    s.coord_scale[2] = fz ? one / ft : 0.0f;
    s.val = planar(im);
    s.val_channels = im.channels;
    s.homogeneous = 1;
    J.homog = true;
    J.replay = true;
    J.out = outview(im, im.channels, 1);
    J.method = method;
    return run_lattice(E, J, st);
}

}  // namespace pgpu

// =================================================================================
// C ABI
// =================================================================================
using namespace pgpu;

namespace {

struct ApiScope {
    Engine* E = nullptr;
    std::unique_lock<std::mutex> lock;
    cudaStream_t st = nullptr;
    int rc = PGPU_OK;
    // queue: a submission, which leaves the batches queued before it running
    ApiScope(const pgpu_options* opt, bool queue = false) {
        clear_error();
        const int dev = opt ? opt->device : 0;
        rc = get_engine(dev, &E);
        if (rc) return;
        lock = std::unique_lock<std::mutex>(E->mu);
        if (cudaSetDevice(dev) != cudaSuccess) {
            rc = fail(PGPU_ERR_CUDA, "cudaSetDevice(%d) failed", dev);
            return;
        }
        if (!queue && !E->async_q.empty()) {
            set_call_stream(E->stream);
            drain_async(*E);
            clear_error();
        }
        const bool device = opt && opt->memory == PGPU_MEM_DEVICE;
        st = (device && opt->stream) ? (cudaStream_t)opt->stream : E->stream;
        set_call_stream(st);
        // Device memory without a stream belongs to the legacy default stream (stream 0,
        // torch's default): the engine's own stream does not synchronise with it, so it
        // waits here for the work queued there before the call, and stream 0 waits on exit
        // for the call's work.
        if (device && !opt->stream) {
            if (cudaEventRecord(E->join_ev[0], cudaStreamLegacy) != cudaSuccess ||
                cudaStreamWaitEvent(E->stream, E->join_ev[0], 0) != cudaSuccess) {
                rc = fail(PGPU_ERR_CUDA, "ordering against the default stream failed: %s",
                          cudaGetErrorString(cudaGetLastError()));
                return;
            }
            joined = true;
        }
    }
    ~ApiScope() {
        if (joined && cudaEventRecord(E->join_ev[1], E->stream) == cudaSuccess)
            cudaStreamWaitEvent(cudaStreamLegacy, E->join_ev[1], 0);
        set_call_stream(nullptr);
    }
    bool joined = false;
};

pgpu_options opts_or_default(const pgpu_options* o) {
    pgpu_options d;
    pgpu_default_options(&d);
    return o ? *o : d;
}

// The batched bilateral lattice job over images [i0, i1) of dv (device views):
// JointBilateral::apply with each image as its own reference (src/GaussTransform.cpp:646-676).
void bilateral_job(const pgpu_image* dv, int i0, int i1, const float* filter_width,
                   const float* color_sigma, const pgpu_options& opt, BatchJob& B) {
    const int C = dv[i0].channels;
    B.d = C + 2;
    B.vd = C + 1;
    B.payload = opt.payload;
    B.load = opt.load_factor;
    B.homog = true;
    B.replay = true;
    B.use_graph = (opt.flags & PGPU_FLAG_GRAPH) != 0;
    B.autotune = (opt.flags & PGPU_FLAG_AUTOTUNE) != 0;
    B.items.resize(i1 - i0);
    volatile float one = 1.0f;
    for (int i = i0; i < i1; ++i) {
        BatchItem& it = B.items[i - i0];
        PointSource& s = it.splat;
        memset(&s, 0, sizeof(s));
        s.width = dv[i].width;
        s.height = dv[i].height;
        s.frames = 1;
        s.pos = planar(dv[i]);
        s.pos_channels = C;
        const float inv_r = one / color_sigma[i];
        for (int c = 0; c < C; ++c) s.pos_scale[c] = inv_r;
        s.coord_mask = 3;
        s.coord_scale[0] = one / filter_width[i];
        s.coord_scale[1] = one / filter_width[i];
        s.val = planar(dv[i]);
        s.val_channels = C;
        s.homogeneous = 1;
        it.n = (uint32_t)((size_t)dv[i].width * dv[i].height);
        it.out = outview(dv[i], C, 1);
    }
}

// Host-memory batches run in chunks of whole images of at least kChunkPixels pixels on three
// device slots in turn: while the lattices of chunk k run on the compute stream, chunk k+1
// is uploaded on one copy stream and chunk k-1 downloaded on the other, so with pinned host
// images the transfers hide behind the filtering.  (With two slots, the upload of chunk
// k+1 would wait for the download of chunk k-1 from the same slot.)  A batch smaller than two
// chunks is one chunk.  The reported statistics sum over the chunks.  The slots keep turning
// from one call to the next, so a queued batch (pgpu_bilateral_batch_submit) uploads its
// first chunks while the previous batch's last chunks are filtered and downloaded.
constexpr size_t kChunkPixels = size_t(1) << 22;

}  // namespace

namespace pgpu {
// One queued chunk of a submitted host batch: its lattice job (device slot views), the
// queued pass and the pinned buffer its metadata is staged in.
struct AsyncChunk {
    BatchJob job;
    PassState ps;
    unsigned char* h = nullptr;
    size_t h_bytes = 0;
    int i0 = 0, i1 = 0;
};

struct AsyncBatch {
    long long id = 0;
    std::vector<pgpu_image> in, out;
    std::vector<float> fw, cs;
    pgpu_options opt;
    std::vector<AsyncChunk> chunks;
    cudaEvent_t done = nullptr;   // on the download stream after the last download
};
}  // namespace pgpu

namespace {

unsigned char* pinned_get(Engine& E, size_t need, size_t* got) {
    for (size_t i = 0; i < E.pinned_free.size(); ++i) {
        if (E.pinned_free[i].second >= need) {
            unsigned char* p = E.pinned_free[i].first;
            *got = E.pinned_free[i].second;
            E.pinned_free.erase(E.pinned_free.begin() + i);
            return p;
        }
    }
    unsigned char* p = nullptr;
    const size_t nb = std::max<size_t>(need, 65536);
    if (cudaHostAlloc((void**)&p, nb, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *got = nb;
    return p;
}

void pinned_put(Engine& E, unsigned char* p, size_t bytes) {
    if (p) E.pinned_free.emplace_back(p, bytes);
}

int bilateral_batch_host(Engine& E, cudaStream_t st, const pgpu_image* ims, const pgpu_image* outs,
                         int count, const float* filter_width, const float* color_sigma,
                         const pgpu_options& opt, AsyncBatch* ab);

// Finish the oldest queued batch (its download stream has reached its event): statuses and
// learned ratios of every chunk; images whose hash range overflowed were left unfiltered
// and are filtered again here, synchronously, once every stream is idle.
void complete_oldest(Engine& E) {
    AsyncBatch* ab = E.async_q.front();
    E.async_q.pop_front();
    int rc = PGPU_OK;
    std::string msg;
    const cudaError_t ce = cudaEventSynchronize(ab->done);
    if (ce != cudaSuccess) {
        rc = fail(PGPU_ERR_CUDA, "queued batch: %s", cudaGetErrorString(ce));
        msg = last_error();
    }
    std::vector<int> again;
    pgpu_stats sum;
    memset(&sum, 0, sizeof(sum));
    for (AsyncChunk& c : ab->chunks) {
        if (rc) break;
        std::vector<int> failed;
        const int r = finish_batch(E, c.job, c.ps, &failed);
        if (r) {
            rc = r;
            msg = last_error();
            break;
        }
        pgpu_stats s;
        if (get_stats(&s)) {
            sum.points += s.points, sum.vertices += s.vertices;
            sum.capacity = std::max(sum.capacity, s.capacity);
            sum.d = s.d, sum.vd = s.vd, sum.payload = s.payload;
            sum.load_factor = s.load_factor, sum.blur_pairs = s.blur_pairs;
            sum.blur_grid = s.blur_grid;
            sum.nbr_half = s.nbr_half;
            sum.vertex_rows = s.vertex_rows;
            sum.tile_w = s.tile_w;
            sum.tuned = c.job.autotune ? 2 : 0;
            sum.tiled += s.tiled;
        }
        for (int k : failed) again.push_back(c.i0 + k);
    }
    if (!rc && !again.empty()) {
        // the slots may hold later batches' images: wait for everything queued
        cudaStreamSynchronize(E.copy_in);
        cudaStreamSynchronize(E.stream);
        cudaStreamSynchronize(E.copy_out);
        std::vector<pgpu_image> in, out;
        std::vector<float> fw, cs;
        for (int i : again) {
            in.push_back(ab->in[i]);
            out.push_back(ab->out[i]);
            fw.push_back(ab->fw[i]);
            cs.push_back(ab->cs[i]);
        }
        rc = bilateral_batch_host(E, E.stream, in.data(), out.data(), (int)in.size(), fw.data(), cs.data(),
                                  ab->opt, nullptr);
        if (rc) msg = last_error();
        else sum.retries = 1;
    }
    if (!rc) set_stats(sum);
    for (AsyncChunk& c : ab->chunks) pinned_put(E, c.h, c.h_bytes);
    if (ab->done) cudaEventDestroy(ab->done);
    E.async_done[ab->id] = std::make_pair(rc, msg);
    if (E.async_done.size() > 4096) E.async_done.erase(E.async_done.begin());
    delete ab;
}

}  // namespace

// Every call but a submission first finishes the queued batches: they share the device
// slots, the workspace and the copy streams.
void pgpu::drain_async(Engine& E) {
    while (!E.async_q.empty()) complete_oldest(E);
}

namespace {

int bilateral_batch_host(Engine& E, cudaStream_t st, const pgpu_image* ims, const pgpu_image* outs,
                         int count, const float* filter_width, const float* color_sigma,
                         const pgpu_options& opt, AsyncBatch* ab) {
    const int C = ims[0].channels;
    std::vector<int> cut{0};
    size_t acc = 0, slot_floats = 0, chunk_floats = 0;
    for (int i = 0; i < count; ++i) {
        const size_t px = (size_t)ims[i].width * ims[i].height;
        acc += px;
        chunk_floats += px * C;
        if ((acc >= kChunkPixels && i + 1 < count) || i + 1 == count) {
            cut.push_back(i + 1);
            slot_floats = std::max(slot_floats, chunk_floats);
            acc = chunk_floats = 0;
        }
    }
    const int nchunks = (int)cut.size() - 1;
    DevBuf* slots[3] = {&E.img_a, &E.img_b, &E.img_c};
    const size_t slot_bytes = slot_floats * sizeof(float);
    // a slot that must grow may still be read by queued batches: finish them first
    for (DevBuf* b : slots)
        if (b->bytes < slot_bytes && !E.async_q.empty()) drain_async(E);
    int rc;
    bool grown = false;
    for (DevBuf* b : slots) {
        const void* before = b->p;
        if ((rc = b->ensure(slot_bytes))) return rc;
        grown |= b->p != before;
    }
    const bool fresh_streams = !E.copy_in;
    if ((rc = E.ensure_copy_streams())) return rc;
    cudaStream_t cin = E.copy_in, cout = E.copy_out;
    // slots (re)allocated in order on the compute stream: the copy streams start after it.
    // Otherwise they do not wait for the compute stream, so a queued batch's uploads run
    // while the previous batch is still being filtered.
    if (grown || fresh_streams) {
        CUDA_TRY(cudaEventRecord(E.join_ev[0], st));
        CUDA_TRY(cudaStreamWaitEvent(cin, E.join_ev[0], 0));
        CUDA_TRY(cudaStreamWaitEvent(cout, E.join_ev[0], 0));
    }
    cudaEvent_t* uploaded = E.pipe_ev;
    cudaEvent_t* filtered = E.pipe_ev + 3;
    cudaEvent_t* downloaded = E.pipe_ev + 6;
    std::vector<int> slot_of(nchunks);
    for (int k = 0; k < nchunks; ++k) slot_of[k] = (E.slot_next + k) % 3;
    E.slot_next = (E.slot_next + nchunks) % 3;
    std::vector<pgpu_image> dv(ims, ims + count);

    auto upload = [&](int k) -> int {
        const int slot = slot_of[k];
        float* base = (float*)slots[slot]->p;
        if (E.slot_recorded[slot]) CUDA_TRY(cudaStreamWaitEvent(cin, downloaded[slot], 0));
        size_t off = 0;
        for (int i = cut[k]; i < cut[k + 1]; ++i) {
            dv[i] = dense_like(ims[i], base + off, C);
            off += (size_t)ims[i].width * ims[i].height * C;
            int r = copy_view(ims[i], dv[i], C, cudaMemcpyHostToDevice, cin);
            if (r) return r;
        }
        CUDA_TRY(cudaEventRecord(uploaded[slot], cin));
        return PGPU_OK;
    };
    auto download = [&](int k) -> int {
        const int slot = slot_of[k];
        CUDA_TRY(cudaEventRecord(filtered[slot], st));
        CUDA_TRY(cudaStreamWaitEvent(cout, filtered[slot], 0));
        for (int i = cut[k]; i < cut[k + 1]; ++i) {
            const int r = copy_view(dv[i], outs[i], C, cudaMemcpyDeviceToHost, cout);
            if (r) return r;
        }
        CUDA_TRY(cudaEventRecord(downloaded[slot], cout));
        E.slot_recorded[slot] = true;
        return PGPU_OK;
    };
    auto run = [&]() -> int {
        pgpu_stats sum;
        memset(&sum, 0, sizeof(sum));
        int r = upload(0);
        for (int k = 0; k < nchunks && !r; ++k) {
            if (k + 1 < nchunks && (r = upload(k + 1))) break;
            CUDA_TRY(cudaStreamWaitEvent(st, uploaded[slot_of[k]], 0));
            BatchJob B;
            bilateral_job(dv.data(), cut[k], cut[k + 1], filter_width, color_sigma, opt, B);
            if (ab) {
                // queued: the autotuner's choice, no host wait (checked when it completes)
                AsyncChunk c;
                c.i0 = cut[k];
                c.i1 = cut[k + 1];
                tuned_settings(E, B, &c.job);
                c.h = pinned_get(E, batch_meta_bytes((int)c.job.items.size()), &c.h_bytes);
                if (!c.h) return fail(PGPU_ERR_MEMORY, "pinned allocation for a queued batch failed");
                ab->chunks.push_back(std::move(c));
                AsyncChunk& q = ab->chunks.back();
                if ((r = enqueue_batch(E, q.job, st, q.h, &q.ps))) break;
            } else {
                if ((r = run_batch(E, B, st))) break;
                pgpu_stats s;
                if (get_stats(&s)) {
                    sum.points += s.points;
                    sum.vertices += s.vertices;
                    sum.capacity = std::max(sum.capacity, s.capacity);
                    sum.d = s.d, sum.vd = s.vd, sum.payload = s.payload;
                    sum.load_factor = s.load_factor, sum.blur_pairs = s.blur_pairs;
                    sum.blur_grid = s.blur_grid;
                    sum.nbr_half = s.nbr_half;
                    sum.vertex_rows = s.vertex_rows;
                    sum.tile_w = s.tile_w;
                    if (s.tuned == 1 || sum.tuned != 1) sum.tuned = s.tuned;   // 1 if any chunk was a trial
                    sum.tiled += s.tiled;
                    sum.retries += s.retries;
                    sum.ms_splat += s.ms_splat, sum.ms_compact += s.ms_compact;
                    sum.ms_neighbours += s.ms_neighbours, sum.ms_blur += s.ms_blur;
                    sum.ms_slice += s.ms_slice, sum.ms_total += s.ms_total;
                }
            }
            if ((r = download(k))) break;
        }
        if (!r && !ab) set_stats(sum);
        return r;
    };
    rc = run();
    if (ab && !rc) {
        CUDA_TRY(cudaEventCreateWithFlags(&ab->done, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(ab->done, cout));
        return PGPU_OK;
    }
    // the caller's host images are in use until every copy has landed, error or not
    const cudaError_t e1 = cudaStreamSynchronize(cin), e2 = cudaStreamSynchronize(cout);
    if (!rc && (e1 != cudaSuccess || e2 != cudaSuccess))
        return fail(PGPU_ERR_CUDA, "batch copies failed: %s",
                    cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    return rc;
}

}  // namespace

extern "C" {

void pgpu_default_options(pgpu_options* opt) {
    if (!opt) return;
    memset(opt, 0, sizeof(*opt));
    opt->payload = PGPU_PAYLOAD_FP32;
    opt->memory = PGPU_MEM_HOST;
    opt->device = 0;
    opt->stream = nullptr;
    opt->load_factor = 0.5f;
    opt->method = PGPU_METHOD_PERMUTOHEDRAL;
}

const char* pgpu_last_error(void) { return last_error(); }

int pgpu_version(void) { return 100; }

int pgpu_device_count(void) { return device_count_sm100(); }

int pgpu_last_stats(pgpu_stats* out) {
    if (!out) return fail(PGPU_ERR_ARGUMENT, "null stats pointer");
    if (!get_stats(out)) return fail(PGPU_ERR_ARGUMENT, "no lattice has run on this thread");
    return PGPU_OK;
}

int pgpu_gauss_transform(const pgpu_image* slice, const pgpu_image* splat, const pgpu_image* values,
                         const float* sigmas, int n_sigmas, pgpu_image* out,
                         const pgpu_options* opt_in) {
    const pgpu_options opt = opts_or_default(opt_in);
    if (!view_ok(splat) || !view_ok(values) || !view_ok(out) || (slice && !view_ok(slice)) || !sigmas)
        return fail(PGPU_ERR_ARGUMENT, "invalid image view or sigmas");
    if (!points_fit(splat) || (slice && !points_fit(slice)))
        return fail(PGPU_ERR_UNSUPPORTED, "more than 2^32 - 1 points in one lattice");
    ApiScope S(&opt);
    if (S.rc) return S.rc;
    Engine& E = *S.E;
    if (opt.memory == PGPU_MEM_DEVICE) {
        int rc = gauss_transform_device(E, slice, *splat, *values, sigmas, n_sigmas, *out,
                                        opt.payload, opt.load_factor, S.st, opt.method);
        return rc;
    }
    const bool replay = !slice || same_view(*slice, *splat);
    pgpu_image dsplat, dvals, dslice, dout;
    int rc;
    if ((rc = upload(E, E.img_a, *splat, &dsplat, S.st))) return rc;
    if ((rc = upload(E, E.img_b, *values, &dvals, S.st))) return rc;
    if (!replay && (rc = upload(E, E.img_c, *slice, &dslice, S.st))) return rc;
    const pgpu_image& sl = replay ? *splat : *slice;
    if ((rc = E.img_d.ensure(sizeof(float) * (size_t)sl.width * sl.height * sl.frames * values->channels)))
        return rc;
    dout = dense_like(sl, (float*)E.img_d.p, values->channels);
    rc = gauss_transform_device(E, replay ? nullptr : &dslice, dsplat, dvals, sigmas, n_sigmas, dout,
                                opt.payload, opt.load_factor, S.st, opt.method);
    if (rc) return rc;
    if ((rc = download(dout, *out, values->channels, S.st))) return rc;
    CUDA_TRY(cudaStreamSynchronize(S.st));
    return PGPU_OK;
}

int pgpu_joint_bilateral(pgpu_image* im, const pgpu_image* ref, float filter_width,
                         float filter_height, float filter_frames, float color_sigma,
                         const pgpu_options* opt_in) {
    const pgpu_options opt = opts_or_default(opt_in);
    if (!view_ok(im) || !view_ok(ref)) return fail(PGPU_ERR_ARGUMENT, "invalid image view");
    if (!points_fit(im)) return fail(PGPU_ERR_UNSUPPORTED, "more than 2^32 - 1 points in one lattice");
    ApiScope S(&opt);
    if (S.rc) return S.rc;
    Engine& E = *S.E;
    if (opt.memory == PGPU_MEM_DEVICE)
        return joint_bilateral_device(E, *im, *ref, filter_width, filter_height, filter_frames,
                                      color_sigma, opt.payload, opt.load_factor, S.st, opt.method);
    const bool same = same_view(*im, *ref);
    pgpu_image dim, dref;
    int rc;
    if ((rc = upload(E, E.img_a, *im, &dim, S.st))) return rc;
    if (same) dref = dim;
    else if ((rc = upload(E, E.img_b, *ref, &dref, S.st))) return rc;
    rc = joint_bilateral_device(E, dim, dref, filter_width, filter_height, filter_frames, color_sigma,
                                opt.payload, opt.load_factor, S.st, opt.method);
    if (rc) return rc;
    if ((rc = download(dim, *im, im->channels, S.st))) return rc;
    CUDA_TRY(cudaStreamSynchronize(S.st));
    return PGPU_OK;
}

int pgpu_bilateral(pgpu_image* im, float filter_width, float filter_height, float filter_frames,
                   float color_sigma, const pgpu_options* opt) {
    return pgpu_joint_bilateral(im, im, filter_width, filter_height, filter_frames, color_sigma, opt);
}

int pgpu_bilateral_batch(pgpu_image* ims, int count, const float* filter_width,
                         const float* color_sigma, const pgpu_options* opt_in) {
    const pgpu_options opt = opts_or_default(opt_in);
    if (count < 0 || (count > 0 && (!ims || !filter_width || !color_sigma)))
        return fail(PGPU_ERR_ARGUMENT, "invalid batch arguments");
    if (count == 0) return PGPU_OK;
    const int C = ims[0].channels;
    if (C + 1 > 8) return fail(PGPU_ERR_UNSUPPORTED, "%d image channels (supported: 1..7)", C);
    for (int i = 0; i < count; ++i) {
        const pgpu_image& v = ims[i];
        const float fw = filter_width[i];
        if (!view_ok(&v) || v.channels != C || v.frames != 1)
            return fail(PGPU_ERR_ARGUMENT, "batch image %d: single-frame images with %d channels expected", i, C);
        if (!points_fit(&v))
            return fail(PGPU_ERR_UNSUPPORTED, "batch image %d: more than 2^32 - 1 points", i);
        // every image must have both pixel axes as positions (d = C + 2), as
        // JointBilateral::apply makes them for fw < 10 x the size (src/GaussTransform.cpp:541-542)
        if (v.width < 2 || v.height < 2 || !(fw > 0) || !(fw < 10 * v.width) || !(fw < 10 * v.height) ||
            !(color_sigma[i] > 0))
            return fail(PGPU_ERR_UNSUPPORTED,
                        "batch image %d: needs width, height > 1 and 0 < filter width < 10 x its "
                        "width and height (filter it with pgpu_bilateral)", i);
    }
    ApiScope S(&opt);
    if (S.rc) return S.rc;
    Engine& E = *S.E;
    if (opt.memory == PGPU_MEM_DEVICE) {
        BatchJob B;
        bilateral_job(ims, 0, count, filter_width, color_sigma, opt, B);
        return run_batch(E, B, S.st);
    }
    return bilateral_batch_host(E, S.st, ims, ims, count, filter_width, color_sigma, opt, nullptr);
}

int pgpu_bilateral_batch_submit(const pgpu_image* in, pgpu_image* out, int count,
                                const float* filter_width, const float* color_sigma,
                                const pgpu_options* opt_in, long long* ticket) {
    const pgpu_options opt = opts_or_default(opt_in);
    if (!ticket || count < 1 || !in || !filter_width || !color_sigma)
        return fail(PGPU_ERR_ARGUMENT, "invalid batch arguments");
    if (opt.memory != PGPU_MEM_HOST) return fail(PGPU_ERR_ARGUMENT, "queued batches take host-memory images");
    if (opt.device < 0 || opt.device > 255) return fail(PGPU_ERR_ARGUMENT, "device %d", opt.device);
    *ticket = 0;
    const pgpu_image* outs = out ? out : in;
    const int C = in[0].channels;
    if (C + 1 > 8) return fail(PGPU_ERR_UNSUPPORTED, "%d image channels (supported: 1..7)", C);
    for (int i = 0; i < count; ++i) {
        const pgpu_image& v = in[i];
        const pgpu_image& o = outs[i];
        const float fw = filter_width[i];
        if (!view_ok(&v) || v.channels != C || v.frames != 1)
            return fail(PGPU_ERR_ARGUMENT, "batch image %d: single-frame images with %d channels expected", i, C);
        if (!points_fit(&v))
            return fail(PGPU_ERR_UNSUPPORTED, "batch image %d: more than 2^32 - 1 points", i);
        if (!view_ok(&o) || o.width != v.width || o.height != v.height || o.frames != 1 || o.channels != C)
            return fail(PGPU_ERR_ARGUMENT, "batch image %d: the output view differs in size from the input", i);
        if (v.width < 2 || v.height < 2 || !(fw > 0) || !(fw < 10 * v.width) || !(fw < 10 * v.height) ||
            !(color_sigma[i] > 0))
            return fail(PGPU_ERR_UNSUPPORTED,
                        "batch image %d: needs width, height > 1 and 0 < filter width < 10 x its "
                        "width and height (filter it with pgpu_bilateral)", i);
    }
    ApiScope S(&opt, true);
    if (S.rc) return S.rc;
    Engine& E = *S.E;
    const long long id = (++E.async_seq << 8) | opt.device;
    // a shape the autotuner is still timing runs now, as pgpu_bilateral_batch would
    bool queued = true;
    {
        std::vector<pgpu_image> probe(in, in + count);
        BatchJob T;
        // the chunks of one submission are cut by pixel count; each chunk is tuned by its
        // own shape, so check each
        size_t acc = 0;
        int i0 = 0;
        for (int i = 0; i < count && queued; ++i) {
            acc += (size_t)in[i].width * in[i].height;
            if ((acc >= kChunkPixels && i + 1 < count) || i + 1 == count) {
                BatchJob P;
                bilateral_job(probe.data(), i0, i + 1, filter_width, color_sigma, opt, P);
                queued = tuned_settings(E, P, &T);
                acc = 0;
                i0 = i + 1;
            }
        }
    }
    if (!queued) {
        drain_async(E);
        clear_error();
        const int rc = bilateral_batch_host(E, S.st, in, outs, count, filter_width, color_sigma, opt, nullptr);
        if (rc) return rc;
        E.async_done[id] = std::make_pair(PGPU_OK, std::string());
        *ticket = id;
        return PGPU_OK;
    }
    AsyncBatch* ab = new AsyncBatch();
    ab->id = id;
    ab->in.assign(in, in + count);
    ab->out.assign(outs, outs + count);
    ab->fw.assign(filter_width, filter_width + count);
    ab->cs.assign(color_sigma, color_sigma + count);
    ab->opt = opt;
    const int rc = bilateral_batch_host(E, S.st, in, outs, count, filter_width, color_sigma, opt, ab);
    if (rc) {
        // nothing of it may still run when the caller gets its buffers back
        cudaStreamSynchronize(E.copy_in);
        cudaStreamSynchronize(E.stream);
        cudaStreamSynchronize(E.copy_out);
        for (AsyncChunk& c : ab->chunks) pinned_put(E, c.h, c.h_bytes);
        if (ab->done) cudaEventDestroy(ab->done);
        delete ab;
        return rc;
    }
    E.async_q.push_back(ab);
    *ticket = id;
    return PGPU_OK;
}

int pgpu_batch_wait(long long ticket) {
    if (ticket <= 0) return fail(PGPU_ERR_ARGUMENT, "invalid ticket");
    pgpu_options opt;
    pgpu_default_options(&opt);
    opt.device = (int)(ticket & 0xFF);
    ApiScope S(&opt, true);
    if (S.rc) return S.rc;
    Engine& E = *S.E;
    for (;;) {
        auto it = E.async_done.find(ticket);
        if (it != E.async_done.end()) {
            const std::pair<int, std::string> r = it->second;
            E.async_done.erase(it);
            if (r.first) return fail(r.first, "%s", r.second.c_str());
            return PGPU_OK;
        }
        bool queued = false;
        for (AsyncBatch* a : E.async_q) queued |= a->id == ticket;
        if (!queued) return fail(PGPU_ERR_ARGUMENT, "unknown or already waited-for ticket");
        complete_oldest(E);
    }
}

int pgpu_lattice_dump(int d, int vd, int n, const float* pos, const float* val, int payload,
                      int* n_vertices, short* keys, int* replay_vtx, float* replay_w,
                      float* splat_vals, float* blur_vals, float* out) {
    if (d < 1 || d > kMaxD || vd < 1 || vd > 8 || n < 1 || !pos || !val)
        return fail(PGPU_ERR_ARGUMENT, "invalid dump arguments");
    pgpu_options opt;
    pgpu_default_options(&opt);
    opt.payload = payload;
    ApiScope S(&opt);
    if (S.rc) return S.rc;
    Engine& E = *S.E;
    cudaStream_t st = S.st;
    // planar (channel-major) copies of the interleaved points
    std::vector<float> hp((size_t)n * d), hv((size_t)n * vd);
    for (int i = 0; i < n; ++i) {
        for (int c = 0; c < d; ++c) hp[(size_t)c * n + i] = pos[(size_t)i * d + c];
        for (int c = 0; c < vd; ++c) hv[(size_t)c * n + i] = val[(size_t)i * vd + c];
    }
    const int vdp = vdp_for(vd);
    const size_t rows = (size_t)n * (d + 1);
    const size_t payb = payload_bytes(payload);
    DevBuf bp, bv, bo, brv, brw, bsv;
    int rc;
    if ((rc = bp.ensure(hp.size() * 4)) || (rc = bv.ensure(hv.size() * 4)) ||
        (rc = bo.ensure((size_t)n * vd * 4)) || (rc = brv.ensure(rows * 4)) ||
        (rc = brw.ensure(rows * 4)))
        return rc;
    // at most n*(d+1) vertices: the dumps copy that many rows of the vertex buffers
    const size_t dump_bytes = rows * vdp * payb;
    if ((rc = bsv.ensure(dump_bytes))) return rc;
    CUDA_TRY(cudaMemcpyAsync(bp.p, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(bv.p, hv.data(), hv.size() * 4, cudaMemcpyHostToDevice, st));
    pgpu_image vpos = {(float*)bp.p, n, 1, 1, d, n, n, n};
    pgpu_image vval = {(float*)bv.p, n, 1, 1, vd, n, n, n};
    pgpu_image vout = {(float*)bo.p, n, 1, 1, vd, n, n, n};
    LatticeJob J;
    J.d = d;
    J.vd = vd;
    J.payload = payload;
    J.load = 0.5f;
    J.n = (uint32_t)n;
    memset(&J.splat, 0, sizeof(J.splat));
    J.splat.width = n;
    J.splat.height = 1;
    J.splat.frames = 1;
    J.splat.pos = planar(vpos);
    J.splat.pos_channels = d;
    for (int c = 0; c < d; ++c) J.splat.pos_scale[c] = 1.0f;
    J.splat.val = planar(vval);
    J.splat.val_channels = vd;
    J.replay = true;
    J.out = outview(vout, vd, 0);
    J.rec_vtx = (int*)brv.p;
    J.rec_w = (float*)brw.p;
    J.dump_splat = bsv.p;
    J.dump_bytes = dump_bytes;
    uint32_t M = 0;
    J.vertices_out = &M;
    rc = run_lattice(E, J, st);
    if (rc) return rc;
    if (n_vertices) *n_vertices = (int)M;
    if (out) {   // the slice wrote channel-major; the dump is point-major
        std::vector<float> planar_out((size_t)n * vd);
        CUDA_TRY(cudaMemcpy(planar_out.data(), bo.p, planar_out.size() * 4, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < vd; ++c) out[(size_t)i * vd + c] = planar_out[(size_t)c * n + i];
    }
    if (replay_vtx) CUDA_TRY(cudaMemcpy(replay_vtx, brv.p, rows * 4, cudaMemcpyDeviceToHost));
    if (replay_w) CUDA_TRY(cudaMemcpy(replay_w, brw.p, rows * 4, cudaMemcpyDeviceToHost));
    const int kw = key_words(d);
    if (keys) {
        std::vector<uint4> k0(M), kn((size_t)(kw - 1) * M);
        const size_t vcap = E.last_cap;
        if (M) CUDA_TRY(cudaMemcpy(k0.data(), E.vkey0.p, (size_t)M * 16, cudaMemcpyDeviceToHost));
        for (int w = 1; w < kw; ++w)
            if (M) CUDA_TRY(cudaMemcpy(kn.data() + (size_t)(w - 1) * M, (uint4*)E.vkeyn.p + (size_t)(w - 1) * vcap,
                                      (size_t)M * 16, cudaMemcpyDeviceToHost));
        for (uint32_t v = 0; v < M; ++v) {
            for (int c = 0; c < d; ++c) {
                const int wi = lane_word(c), lp = lane_pos(c);
                const uint4 w = wi == 0 ? k0[v] : kn[(size_t)(wi - 1) * M + v];
                const uint32_t u = (lp >> 1) == 0 ? w.x : (lp >> 1) == 1 ? w.y : (lp >> 1) == 2 ? w.z : w.w;
                const uint32_t lane = (lp & 1) ? (u >> 16) : (u & 0xFFFFu);
                keys[(size_t)v * d + c] = (short)(uint16_t)(lane ^ 0x8000u);
            }
        }
    }
    auto conv = [&](void* dev, float* dst) -> int {
        if (!dst || !M) return PGPU_OK;
        std::vector<unsigned char> raw((size_t)M * vdp * payb);
        CUDA_TRY(cudaMemcpy(raw.data(), dev, raw.size(), cudaMemcpyDeviceToHost));
        for (uint32_t v = 0; v < M; ++v)
            for (int c = 0; c < vd; ++c) {
                const size_t idx = (size_t)v * vdp + c;
                float f;
                if (payload == kPayloadF32) f = ((float*)raw.data())[idx];
                else if (payload == kPayloadF64) f = (float)((double*)raw.data())[idx];
                else {
                    const uint16_t h = ((uint16_t*)raw.data())[idx];
                    f = payload == kPayloadF16 ? half_bits_to_float(h) : bf16_bits_to_float(h);
                }
                dst[(size_t)v * vd + c] = f;
            }
        return PGPU_OK;
    };
    if ((rc = conv(bsv.p, splat_vals))) return rc;
    if (blur_vals && M) {   // the filtered rows live in slot space, in the arithmetic type
        const size_t accb = accum_bytes(payload);
        std::vector<uint32_t> v2s(M);
        std::vector<unsigned char> rows((size_t)E.last_cap * vdp * accb);
        CUDA_TRY(cudaMemcpy(v2s.data(), E.vtx2slot.p, (size_t)M * 4, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(rows.data(), E.sval.p, rows.size(), cudaMemcpyDeviceToHost));
        for (uint32_t v = 0; v < M; ++v)
            for (int c = 0; c < vd; ++c) {
                const size_t idx = (size_t)v2s[v] * vdp + c;
                blur_vals[(size_t)v * vd + c] = accb == 8 ? (float)((double*)rows.data())[idx]
                                                          : ((float*)rows.data())[idx];
            }
    }
    return PGPU_OK;
}

}  // extern "C"
