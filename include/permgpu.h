/* permgpu.h — C ABI of the B200 (sm_100a) permutohedral-lattice Gauss transform.
 *
 * A drop-in GPU replacement for the PERMUTOHEDRAL method of ImageStack's Gauss
 * transform operations.  Every function takes plain pointers and sizes, returns a
 * status code (PGPU_OK == 0) and records a message for pgpu_last_error() on failure;
 * no C++ or CUDA type crosses this boundary.  Calls are synchronous: when one returns,
 * its output is in the caller's memory (pgpu_bilateral_batch_submit alone queues its work
 * and returns; pgpu_batch_wait finishes it).  There is no CPU fallback: without a usable
 * sm_100 device every compute call fails with PGPU_ERR_NO_DEVICE.
 *
 * Memory: image views point at HOST memory (ImageStack images, pageable or pinned) when
 * options.memory == PGPU_MEM_HOST, or at DEVICE memory when options.memory ==
 * PGPU_MEM_DEVICE.  The library never frees caller memory; it keeps its own device
 * workspace (hash table, vertex arrays, staging images) per device and reuses it.
 */
#ifndef PERMGPU_H
#define PERMGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* A planar float32 image view: element (x, y, t, c) lives at
 * base + c*cstride + t*tstride + y*ystride + x.
 * Mirrors ImageStack::Image (src/Image.h:26-27, element access src/Image.h:57-67);
 * a fresh Image has ystride = width, tstride = width*height,
 * cstride = width*height*frames. */
typedef struct pgpu_image {
    float *base;
    int width, height, frames, channels;
    long long ystride, tstride, cstride;
} pgpu_image;

/* status codes */
#define PGPU_OK 0
#define PGPU_ERR_ARGUMENT 1     /* bad sizes, mismatched images (the reference asserts) */
#define PGPU_ERR_UNSUPPORTED 2  /* position dimensions > 16, value channels > 8, or more than
                                 * 2^32 - 1 points (pixels x frames) in one lattice */
#define PGPU_ERR_CUDA 3         /* a CUDA call failed; see pgpu_last_error() */
#define PGPU_ERR_MEMORY 4       /* device or pinned allocation failed */
#define PGPU_ERR_CAPACITY 5     /* hash table still overfull after the retries */
#define PGPU_ERR_NO_DEVICE 7    /* no CUDA device with compute capability 10.x */
#define PGPU_ERR_ADMISSION 8    /* request larger than the serving memory budget */
#define PGPU_ERR_TIMEOUT 9      /* a bounded wait ran out */

/* value payload stored in the lattice (splat accumulation is always FP32, or FP64 for
 * PGPU_PAYLOAD_FP64) */
#define PGPU_PAYLOAD_FP32 0
#define PGPU_PAYLOAD_FP16 1
#define PGPU_PAYLOAD_BF16 2
#define PGPU_PAYLOAD_FP64 3

#define PGPU_MEM_HOST 0
#define PGPU_MEM_DEVICE 1

typedef struct pgpu_options {
    int payload;        /* PGPU_PAYLOAD_* (default FP32, the reference's arithmetic) */
    int memory;         /* PGPU_MEM_HOST or PGPU_MEM_DEVICE */
    int device;         /* CUDA device ordinal */
    void *stream;       /* cudaStream_t for PGPU_MEM_DEVICE calls; NULL: library stream */
    float load_factor;  /* hash-table target load in (0, 0.9]; 0: default 0.5 */
    int flags;          /* PGPU_FLAG_* (pgpu_bilateral_batch), else 0 */
    int method;         /* PGPU_METHOD_PERMUTOHEDRAL (default) or PGPU_METHOD_GRID */
} pgpu_options;

/* PGPU_METHOD_GRID: the bilateral grid, GaussTransform::apply's GRID branch
 * (src/GaussTransform.cpp:227-290, src/DenseGrid.h: multilinear splat and slice, two
 * [1 2 1]/4 passes per dimension), for gauss_transform and joint_bilateral/bilateral;
 * 1..5 position dimensions, FP32 only. */
#define PGPU_METHOD_PERMUTOHEDRAL 0
#define PGPU_METHOD_GRID 1

typedef struct pgpu_stats {
    long long points;      /* splatted points */
    long long vertices;    /* occupied lattice vertices M */
    long long capacity;    /* hash-table slots used */
    int d, vd, payload, retries;
    float ms_splat, ms_compact, ms_neighbours, ms_blur, ms_slice, ms_total;
    float load_factor;     /* hash-table load factor used */
    int blur_pairs;        /* 1: blur axes fused in pairs, 0: one axis per pass */
    int tiled;             /* images splatted by the tile splat (the others: direct) */
    int blur_grid;         /* blur launch: 0 16 blocks per SM striding over the vertices, 1 one
                              vertex per thread, 2 as 0 with two vertices per iteration */
    int tuned;             /* autotuner: 0 off, 1 this call was one of its trials, 2 its choice */
    int nbr_half;          /* 1: one neighbour lookup per axis (the other pair entry scattered) */
    int vertex_rows;       /* 1: the splat numbered vertices and filled vertex-ordered rows (no compaction) */
    int tile_w;            /* tile splat tile width in pixels (tiles of 256 pixels) */
} pgpu_stats;

/* Fill *opt with the defaults. */
void pgpu_default_options(pgpu_options *opt);

/* Message of the last failed call on this thread ("" if none). */
const char *pgpu_last_error(void);

/* Library version, major*10000 + minor*100 + patch. */
int pgpu_version(void);

/* Number of usable devices (compute capability 10.x); 0 when none. */
int pgpu_device_count(void);

/* GaussTransform::apply, PERMUTOHEDRAL branch (src/GaussTransform.cpp:115-133, 163-226).
 * Positions are splat(x,y,t,c) * (1/sigmas[c]); `out` (slice's width, height, frames and
 * values->channels channels, caller-allocated) receives the un-normalised transform.
 * When `slice` is NULL or describes exactly the same view as `splat` (the reference's
 * `slice == splat`, src/GaussTransform.cpp:196), the splat points are sliced; otherwise
 * the lattice is sliced at the slice positions, where vertices the splat never created
 * contribute zero (src/Permutohedral.h:405-407). */
int pgpu_gauss_transform(const pgpu_image *slice, const pgpu_image *splat,
                         const pgpu_image *values, const float *sigmas, int n_sigmas,
                         pgpu_image *out, const pgpu_options *opt);

/* JointBilateral::apply with the permutohedral method, in place on `im`
 * (src/GaussTransform.cpp:504-678): degenerate-axis recursion, positions
 * (ref*(1/color_sigma), x*(1/filter_width), y*(1/filter_height), t*(1/filter_frames)),
 * values (im, 1), normalisation by the homogeneous channel. */
int pgpu_joint_bilateral(pgpu_image *im, const pgpu_image *ref, float filter_width,
                         float filter_height, float filter_frames, float color_sigma,
                         const pgpu_options *opt);

/* Bilateral::apply with the permutohedral method (src/GaussTransform.cpp:730-734). */
int pgpu_bilateral(pgpu_image *im, float filter_width, float filter_height,
                   float filter_frames, float color_sigma, const pgpu_options *opt);

/* Many bilateral filters in one set of launches (no counterpart in the reference, which
 * filters one image per call; each image's result equals Bilateral::apply on it,
 * src/GaussTransform.cpp:730-734).  ims[i] is filtered in place with its own
 * filter_width[i] (= filter height) and color_sigma[i]; images may differ in size but
 * must share the channel count (1..7) and be single frames larger than 1x1 with
 * 0 < filter width < 10 x their width and height.  Every image keeps its own lattice
 * (its own hash-table range).  opt->flags & PGPU_FLAG_GRAPH captures the launch sequence
 * as a CUDA graph and replays it for later batches of the same shape.
 * opt->flags & PGPU_FLAG_AUTOTUNE lets the first calls of each batch shape (the number
 * of images, the point count to a power of two, d, the payload) try candidate settings
 * one knob at a time — hash-table load factor 0.5, 0.35 or 0.7, the tile splat where it
 * applies or the direct splat for every image, rows compacted from hash-slot space or
 * numbered in vertex order by the splat, one or two neighbour lookups per axis, blur axes
 * fused in pairs or one per pass, the blur's launch shape, 16x16 or 32x8 splat tiles —
 * and keeps the fastest for later calls of that shape (opt->load_factor is then unused);
 * results do not depend on the choice beyond the FP32 tolerance. */
#define PGPU_FLAG_GRAPH 1
#define PGPU_FLAG_AUTOTUNE 2
int pgpu_bilateral_batch(pgpu_image *ims, int count, const float *filter_width,
                         const float *color_sigma, const pgpu_options *opt);

/* Queued host-memory batches (no counterpart in the reference; each result equals
 * Bilateral::apply on the image, src/GaussTransform.cpp:730-734).  The batch of
 * pgpu_bilateral_batch over HOST images in[0..count), each result written to out[i] (same
 * size; out == NULL: in place), queued on the device and returned from at once: its
 * uploads, lattices and downloads run while the caller prepares or submits the next batch,
 * so the copies of consecutive batches overlap one another and the filtering.  Batches run
 * in submission order.  The in and out buffers must stay valid and untouched until
 * pgpu_batch_wait(*ticket) returns; pinned memory lets the copies run at full speed.  A
 * batch shape the autotuner (opt->flags & PGPU_FLAG_AUTOTUNE) is still timing runs before
 * the call returns.  Any other call on the same device first finishes the queued batches.
 * An image whose hash range overflows is filtered again when its batch is waited for. */
int pgpu_bilateral_batch_submit(const pgpu_image *in, pgpu_image *out, int count,
                                const float *filter_width, const float *color_sigma,
                                const pgpu_options *opt, long long *ticket);
/* Wait for a queued batch: its outputs are in place and its buffers free when this returns
 * PGPU_OK; its failure status otherwise.  Each ticket is waited for once; waiting for a
 * later ticket finishes the earlier ones too (their status is kept for their own wait). */
int pgpu_batch_wait(long long ticket);

/* ---- Request server (no counterpart in the reference, which runs one operation at a
 * time on the CPU).  A pool of worker threads, each with its own CUDA stream and lattice
 * workspace, takes queued requests in batches: compatible requests (same position
 * dimensions, value channels and kind) that fit the memory budget go into one batched
 * launch sequence; requests arriving while batches run are admitted as workers and
 * memory free up, and batches on different workers overlap on the device.  Images are
 * in host memory; each result goes to the request's `out`. ---- */
#define PGPU_REQ_BILATERAL 0        /* in: image; filtered into out (may be in) */
#define PGPU_REQ_JOINT_BILATERAL 1  /* in: image, ref: edge image; result into out */
#define PGPU_REQ_GAUSS_TRANSFORM 2  /* in: values, ref: positions, sigmas; un-normalised out */

typedef struct pgpu_server_config {
    int device;
    int workers;                 /* worker threads (streams); 0: 2 */
    int max_batch;               /* requests per batch; 0: 64 */
    int payload;                 /* PGPU_PAYLOAD_* of every lattice */
    float load_factor;           /* hash-table load; 0: 0.5 */
    long long memory_budget;     /* device bytes for images and lattices in flight; 0: 40 GiB */
} pgpu_server_config;

typedef struct pgpu_request {
    int kind;                    /* PGPU_REQ_* */
    pgpu_image in, ref, out;     /* host memory, single frames */
    float filter_width;          /* bilateral kinds: spatial sigma (width = height) */
    float color_sigma;
    const float *sigmas;         /* Gauss transform: one sigma per position channel */
    int n_sigmas;
} pgpu_request;

typedef struct pgpu_server_stats {
    long long submitted, completed, failed, rejected, queued, in_flight, batches;
    long long pixels;            /* points of completed requests */
    long long peak_bytes;        /* largest admitted footprint in flight */
    double seconds;              /* since the first submission */
    double p50_ms, p99_ms, mean_ms, max_ms;   /* submit -> done latency */
    double mpix_per_s, req_per_s;
} pgpu_server_stats;

int pgpu_server_create(const pgpu_server_config *cfg, void **server);
/* Queue a request (its images must stay valid until it completes); *ticket identifies it.
 * A request whose footprint alone exceeds the budget is refused with PGPU_ERR_ADMISSION. */
int pgpu_server_submit(void *server, const pgpu_request *req, long long *ticket);
/* Wait up to timeout_ms for a request; returns its status, or PGPU_ERR_TIMEOUT.  A request
 * is reported finished only after its worker's stream is idle, so its host buffers are
 * free to reuse when this returns, on success and on failure alike.  One thread waits per
 * ticket: a second concurrent wait on the same ticket returns PGPU_ERR_ARGUMENT. */
int pgpu_server_wait(void *server, long long ticket, int timeout_ms);
/* Wait up to timeout_ms until nothing is queued or running. */
int pgpu_server_drain(void *server, int timeout_ms);
int pgpu_server_get_stats(void *server, pgpu_server_stats *out);
/* Forget the latency record (start a new measurement window). */
int pgpu_server_reset_stats(void *server);
/* Stop the workers (after finishing what runs) and free everything. */
void pgpu_server_destroy(void *server);

/* Statistics of the last successful lattice run on this thread. */
int pgpu_last_stats(pgpu_stats *out);

/* Parity dump of one lattice over n interleaved points (pos n*d already scaled by
 * 1/sigma, val n*vd), host memory.  Outputs, each optional (NULL to skip):
 *   *n_vertices              M
 *   keys        [n*(d+1)*d]  vertex keys in vertex order (reference insertion order)
 *   replay_vtx  [n*(d+1)]    vertex index per (point, remainder)
 *   replay_w    [n*(d+1)]    barycentric weight per (point, remainder)
 *   splat_vals  [n*(d+1)*vd] vertex values after the splat
 *   blur_vals   [n*(d+1)*vd] vertex values after the blur
 *   out         [n*vd]       replay slice of the points
 * Buffers sized for the worst case M = n*(d+1); the first M rows are written.
 * Mirrors what src/Permutohedral.h computes: keys :365-369, replay :385-390,
 * values after splat :375-378 and blur :430-488, slice :418-427. */
int pgpu_lattice_dump(int d, int vd, int n, const float *pos, const float *val, int payload,
                      int *n_vertices, short *keys, int *replay_vtx, float *replay_w,
                      float *splat_vals, float *blur_vals, float *out);

/* Bilateral filtering that allocates nothing (no counterpart in the reference, which
 * only runs on the CPU).  For callers that cannot call cudaMalloc: hosts that own all
 * device memory through their own pool or allocator, and loops that must not stall the
 * device (cudaMalloc and cudaFree synchronise it).  Same result as pgpu_bilateral with
 * the permutohedral method on one frame with both pixel axes filtered, but every
 * intermediate lives in a fixed 72 MiB device array inside the library, which each GPU
 * that loads it keeps until the process exits.
 *   d_in, d_out  device memory, planar (channels, height, width) float32, dense; they may
 *                be the same buffer (in place)
 *   limits       width*height <= 262144 (512x512), channels 1..3,
 *                0 < filter_width < 10*width, 0 < filter_height < 10*height;
 *                anything else is rejected with PGPU_ERR_UNSUPPORTED before any work
 *   stream       cudaStream_t to run on (NULL: the legacy default stream); the call
 *                returns after that stream has finished the filter
 * Every call looks up the array's device address in the current context (a lookup, not
 * an allocation).  A call waits for its stream and uploads a small descriptor from host
 * memory, so it cannot be recorded into a CUDA graph: while `stream` is capturing, the
 * call returns PGPU_ERR_UNSUPPORTED without doing anything.  All calls on a device share
 * the one array, which keeps the last call's contents (each call clears what must start
 * at zero): calls that overlap on the GPU (other streams, other host threads) race and
 * corrupt each other, so serialise them.  A frame whose lattice needs more hash slots
 * than the array holds returns PGPU_ERR_CAPACITY and leaves d_out unwritten. */
int pgpu_bilateral_noalloc(const float *d_in, float *d_out, int width, int height,
                           int channels, float filter_width, float filter_height,
                           float color_sigma, void *stream);

/* FP64 brute-force Gauss transform at sampled queries, the error oracle for lattice
 * results: out[i][c] = sum_j exp(-|q_i - p_j|^2 / 2) v_j[c] over all n sources, positions
 * already divided by their sigmas.  It is the kernel of GaussTransform::apply's EXACT
 * method (src/GaussTransform.cpp:135-162) with an exact double exponential instead of its
 * table; not a filtering path.  Device memory, interleaved: q nq x d, p n x d and
 * v n x vd float32, out nq x vd double; d 1..16, vd 1..8.  Returns after `stream`
 * (cudaStream_t, NULL: the legacy default stream) has finished. */
int pgpu_exact_gauss_transform_f64(int d, int vd, int nq, const float *q, int n,
                                   const float *p, const float *v, double *out, void *stream);

/* Throughput probe (no counterpart in the reference): float4 reductions per second at
 * pseudo-random rows of `table` (device memory, rows x 16 bytes, contents changed), from
 * blocks x 256 threads adding per_thread rows each — the access the splat makes once per
 * (point, remainder); its measured rate is the splat's atomic roofline. */
int pgpu_probe_red_rate(void *table, long long rows, int per_thread, int blocks, void *stream,
                        double *reds_per_second);

#ifdef __cplusplus
}
#endif
#endif /* PERMGPU_H */
