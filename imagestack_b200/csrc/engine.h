// Host-side declarations shared by the C-ABI entry points, the batched pipeline and the
// request server.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
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
    // captured batch pipelines, keyed by everything a graph bakes in (sizes, buffer
    // addresses, settings, each image's points and slot range)
    std::map<std::vector<uint64_t>, cudaGraphExec_t> graphs;
    // autotuner state per batch shape: candidate trials so far, their times, the choice
    struct Tuning {
        int trials = 0;
        int count = 0;   // candidates this shape tries
        float ms[8] = {};
        int best = 0;
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
bool same_view(const pgpu_image& a, const pgpu_image& b);
bool is_dense(const pgpu_image& v);
pgpu_image dense_like(const pgpu_image& v, float* base, int channels);
int copy_view(const pgpu_image& src, const pgpu_image& dst, int channels, cudaMemcpyKind kind,
              cudaStream_t st);
PlanarView planar(const pgpu_image& v);
OutView outview(const pgpu_image& v, int channels, int normalize);

int get_engine(int dev, Engine** out);
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
    int splat = 0;            // 0: the tile splat where vertices are shared, 1: direct only
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
