// Host-side declarations shared by the C-ABI entry points, the batched pipeline and the
// request server.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/permgpu.h"
#include "lattice_ops.h"

namespace pgpu {

int fail(int code, const char* fmt, ...);
void clear_error();
const char* last_error();
void set_stats(const pgpu_stats& s);
bool get_stats(pgpu_stats* s);

#define CUDA_TRY(x)                                                                     \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess)                                                          \
            return ::pgpu::fail(PGPU_ERR_CUDA, "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), \
                                __FILE__, __LINE__);                                    \
    } while (0)

// The stream of the calling thread's current library call (the legacy default stream
// outside one): workspace buffers are allocated and freed in order on it.
void set_call_stream(cudaStream_t st);
cudaStream_t call_stream();

// Grow-only device buffer from the stream-ordered allocator: growing it frees the old
// block and allocates the new one on the call's stream, which — unlike cudaMalloc and
// cudaFree — does not synchronise the device, so engines on other streams (the server's
// workers) are not stalled.  Buffers grow by half again each time.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t need);
    void release();
    ~DevBuf();
};

struct AsyncBatch;   // a host-memory batch queued by pgpu_bilateral_batch_submit (engine.cu)

struct Engine {
    int device = -1;
    int sms = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    // hash table (slot space)
    DevBuf key0, keyn, tvals, ft, slot2vtx;
    // compaction
    DevBuf bitmap, offs, partials;
    // vertex space
    DevBuf vkey0, vkeyn, vv0, vv1, nbr;
    DevBuf vf32;   // FP32 normalised rows feeding the first blur pass (16-bit homogeneous)
    DevBuf vtx2slot;   // slot of each vertex
    DevBuf sval;       // filtered rows in slot space, arithmetic type, read by the slice
    DevBuf rec;        // slot of every (point, remainder), [r][n], recorded by the splat
    DevBuf recw;       // its barycentric weight, [r][n], recorded by the splat
    DevBuf grid, grid2;   // the dense grid of the grid method, and its blur's second buffer
    DevBuf tags;       // one tag byte per hash slot (compaction -> neighbour lookups)
    DevBuf vlist;      // slots in the order the splat created them (the vertex list)
    DevBuf dstat;
    // batch metadata: statuses, counts, segment tables (device copy of hmeta)
    DevBuf meta;
    unsigned char* hmeta = nullptr;   // pinned host mirror
    size_t hmeta_bytes = 0;
    // staging images for host-memory calls
    DevBuf img_a, img_b, img_c, img_d;
    unsigned* hstat = nullptr;
    cudaEvent_t ev[8] = {};
    cudaEvent_t join_ev[2] = {};   // ordering against the legacy default stream
    // host-memory batches: uploads and downloads overlap the lattices on these streams
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    cudaEvent_t pipe_ev[9] = {};   // per device slot (3): uploaded, filtered, downloaded
    int slot_next = 0;              // device slot of the next host chunk, in turn over 3
    bool slot_recorded[3] = {};     // the slot's download event has been recorded
    // queued host-memory batches (oldest first), the outcomes of finished ones that no
    // one has waited for yet (status, message), and pinned metadata buffers to reuse
    std::deque<AsyncBatch*> async_q;
    std::map<long long, std::pair<int, std::string>> async_done;
    long long async_seq = 0;
    std::vector<std::pair<unsigned char*, size_t>> pinned_free;
    // captured batch pipelines, keyed by everything a graph bakes in (sizes, buffer
    // addresses, settings, each image's points and slot range)
    std::map<std::vector<uint64_t>, cudaGraphExec_t> graphs;
    // autotuner state per batch shape (batch.cu): the knob and option being tried, the
    // repeats of that trial, the best setting so far and its time
    struct Tuning {
        struct Setting {
            float load = 0.5f;
            bool pairs = true;
            int blur_grid = 0;
            int splat = 0;
            int vertex_rows = 0;
            int nbr_half = 1;
            int tile_w = 16;
        };
        int knob = 0, option = 0, rep = 0, trials = 0;
        bool done = false;
        float best_ms = 1e30f;            // the best setting's whole-lattice time
        float best_stage[3] = {};         // and its splat, neighbours, blur times (0: untimed)
        float cur_ms = 1e30f, cur_stage[3] = {1e30f, 1e30f, 1e30f};
        Setting best;
    };
    std::map<std::string, Tuning> tuning;
    size_t last_cap = 0;
    uint64_t buffers_epoch = 0;   // bumped whenever a buffer moves (invalidates graphs)
    int init(int dev);
    int ensure_hmeta(size_t bytes);
    int ensure_copy_streams();
    void drop_graphs();
    void shutdown();   // release stream, events, pinned buffers and graphs
};

// image views and their staging (engine.cu)
bool view_ok(const pgpu_image* v);
// its pixels over all frames fit the lattice's 32-bit point numbering
bool points_fit(const pgpu_image* v);
bool same_view(const pgpu_image& a, const pgpu_image& b);
bool is_dense(const pgpu_image& v);
pgpu_image dense_like(const pgpu_image& v, float* base, int channels);
int copy_view(const pgpu_image& src, const pgpu_image& dst, int channels, cudaMemcpyKind kind,
              cudaStream_t st);
PlanarView planar(const pgpu_image& v);
OutView outview(const pgpu_image& v, int channels, int normalize);

int get_engine(int dev, Engine** out);
// hold `bytes` of device memory in the library's pool of the current device (engine.cu)
int reserve_pool_memory(size_t bytes, cudaStream_t st);
// finish every queued host batch of E (engine.cu); E.mu held
void drain_async(Engine& E);
int device_count_sm100();

// One image of a batch.
struct BatchItem {
    PointSource splat;     // its points
    uint32_t n = 0;
    PointSource slice;     // slice positions when the job does not replay
    uint32_t n_slice = 0;
    OutView out;
};

// Lattices that share d, value channels and payload, run by the same launches.
struct BatchJob {
    int d = 0, vd = 0, payload = 0;
    float load = 0.5f;
    bool homog = false;    // the last value channel is the homogeneous weight
    bool replay = true;    // slice at the splat points
    bool use_graph = false;   // capture / replay the launch sequence as a CUDA graph
    bool autotune = false;    // pick load factor and blur pairing per batch shape
    bool blur_pairs = true;   // blur two axes per launch
    int blur_grid = 0;        // 0: 16 blocks per SM striding over the vertices, 1: one vertex per
                              // thread, 2: as 0 with two vertices per iteration (one-axis passes)
    int splat = 0;            // 0: the tile splat where vertices are shared, 1: direct only
    bool slot_rows = true;    // rows in slot space with a compaction; false: the tile splat
                              // numbers vertices and fills vertex-ordered rows where it can
    int nbr_half = 1;         // one neighbour lookup per axis (1) or two (0)
    int tile_w = 0;           // tile splat tile width in pixels (0: the default, 16; height 256 / width)
    std::vector<BatchItem> items;
    // parity dumps (single-item jobs)
    int* rec_vtx = nullptr;
    float* rec_w = nullptr;
    void* dump_splat = nullptr;
    size_t dump_bytes = 0;
    // results
    std::vector<uint32_t>* vertices_out = nullptr;   // per item
};
int run_batch(Engine& E, const BatchJob& B, cudaStream_t st);

// A pass of a batch whose launches are queued on the stream but not read back yet: the
// pinned buffer its statuses and vertex counts land in, and what finishing it needs.
struct PassState {
    unsigned char* h = nullptr;
    size_t segstat = 0, counts = 0;   // offsets in h
    std::vector<uint64_t> cap, sig;
    float load = 0.5f;
    int tiled = 0, pass = 0;
    uint64_t n_total = 0, cap_total = 0;
    int timed = 0;   // 0: no events, 1: events around every stage, 2: around a graph
    int nbr_half = 0;   // the neighbour search looked up one direction per axis
    int vertex_rows = 0;   // the splat filled vertex-ordered rows (no compaction)
    int blur_pairs = 1;    // blur axes fused in pairs
    int tile_w = 16;       // tile splat tile width
};
// Bytes of pinned metadata a batch of nseg replayed lattices stages.
size_t batch_meta_bytes(int nseg);
// Settings the autotuner chose for B's shape; false while its trials are not finished
// (an untuned shape runs through run_batch, which times the trials).
bool tuned_settings(Engine& E, const BatchJob& B, BatchJob* out);
// Queue the first pass of B on st with its metadata staged in the pinned buffer h (at
// least batch_meta_bytes), without waiting for it.
int enqueue_batch(Engine& E, const BatchJob& B, cudaStream_t st, unsigned char* h, PassState* ps);
// Once st has run the pass: statuses, learned vertex ratios, statistics.  Images whose
// range overflowed (their output left as it was) are listed in *failed.
int finish_batch(Engine& E, const BatchJob& B, const PassState& ps, std::vector<int>* failed);

struct LatticeJob {
    int d = 0, vd = 0, payload = 0;
    float load = 0.5f;
    PointSource splat;
    uint32_t n = 0;
    bool replay = true;
    PointSource slice;
    uint32_t n_slice = 0;
    OutView out;
    int* rec_vtx = nullptr;
    float* rec_w = nullptr;
    void* dump_splat = nullptr;   // device copy of vertex values after the splat
    size_t dump_bytes = 0;
    uint32_t* vertices_out = nullptr;
    bool homog = false;   // the last value channel is the homogeneous weight
    int method = PGPU_METHOD_PERMUTOHEDRAL;   // or PGPU_METHOD_GRID (grid.cu)
};

LatticeConsts make_consts(int d);
int vdp_for(int vd);
int run_lattice(Engine& E, const LatticeJob& J, cudaStream_t st);
// the bilateral grid (GaussTransform::apply's GRID branch) over the same job description
int run_grid(Engine& E, const LatticeJob& J, cudaStream_t st);

inline float half_bits_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    const int exp = (h >> 10) & 0x1F;
    const uint32_t man = h & 0x3FF;
    uint32_t bits;
    if (exp == 0) {
        if (man == 0) {
            bits = sign;
        } else {   // subnormal: value = man * 2^-24
            float f = (float)man * (1.0f / 16777216.0f);
            uint32_t fb;
            memcpy(&fb, &f, 4);
            bits = sign | fb;
        }
    } else if (exp == 31) {
        bits = sign | 0x7F800000u | (man << 13);
    } else {
        bits = sign | ((uint32_t)(exp - 15 + 127) << 23) | (man << 13);
    }
    float out;
    memcpy(&out, &bits, 4);
    return out;
}

inline float bf16_bits_to_float(uint16_t h) {
    const uint32_t bits = (uint32_t)h << 16;
    float out;
    memcpy(&out, &bits, 4);
    return out;
}

}  // namespace pgpu
