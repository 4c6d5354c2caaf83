// Device-side building blocks of the permutohedral lattice for sm_100a.
//
// Each function here restates one step of ImageStack's src/Permutohedral.h for one
// point per thread.  Everything that determines the lattice keys follows the
// reference's single-precision evaluation order with explicitly rounded intrinsics
// (__fmul_rn / __fadd_rn / __fsub_rn), so the keys, the occupied vertex set and the
// per-point vertex indices are bit-exact with the reference's strict-IEEE build, and no
// compiler contraction into FMA can change them.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgpu {

constexpr int kMaxD = 16;      // position dimensions supported by the kernels
constexpr int kMaxProbe = 1 << 12;   // a probe this long means the table is full
constexpr int kMaxSpin = 1 << 20;

// status bits written by the kernels (atomicOr into the job's status word)
constexpr unsigned kStatusProbeLimit = 1u;   // hash table too full: rerun with more slots
constexpr unsigned kStatusSpinLimit = 2u;    // a pending slot never became ready
constexpr unsigned kStatusKeyRange = 4u;     // an elevated coordinate left the int16 range

// ---------------------------------------------------------------------------------
// Keys.  A vertex key is d int16 coordinates (the (d+1)-th is implied, the keys of
// src/Permutohedral.h:365-369).  On the device a key is KW 16-byte words:
//   word 0: coordinates 0..6 in lanes 0..6, slot state in lane 7;
//   word k>0: coordinates 7+8(k-1) .. 14+8(k-1).
// Coordinates are stored XOR 0x8000, so that a 32-bit half of a word is all ones only
// for the coordinate pair (32767, 32767); an all-ones word is how an empty slot looks.
// ---------------------------------------------------------------------------------
__host__ __device__ constexpr int key_words(int d) { return d <= 7 ? 1 : 1 + (d - 7 + 7) / 8; }

constexpr uint32_t kStateReady = 0x0000u;
constexpr uint32_t kStatePending = 0x0001u;
constexpr uint32_t kStateEmpty = 0xFFFFu;

template <int KW>
struct Key {
    uint4 w[KW];
};

__device__ __forceinline__ uint32_t enc_lane(int v) { return ((uint32_t)(uint16_t)(short)v) ^ 0x8000u; }
__device__ __forceinline__ int dec_lane(uint32_t e) { return (int)(short)(uint16_t)(e ^ 0x8000u); }

__device__ __forceinline__ uint32_t& word_u32(uint4& w, int i) {
    return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w;
}
__device__ __forceinline__ uint32_t word_u32(const uint4& w, int i) {
    return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w;
}

// Lane index of coordinate c inside the key words.
__host__ __device__ constexpr int lane_word(int c) { return c < 7 ? 0 : 1 + (c - 7) / 8; }
__host__ __device__ constexpr int lane_pos(int c) { return c < 7 ? c : (c - 7) % 8; }

template <int D>
__device__ __forceinline__ void pack_key(const int (&k)[D], Key<key_words(D)>& out) {
    constexpr int KW = key_words(D);
    uint32_t lanes[KW * 8];
#pragma unroll
    for (int i = 0; i < KW * 8; ++i) lanes[i] = enc_lane(0);
#pragma unroll
    for (int c = 0; c < D; ++c) lanes[lane_word(c) * 8 + lane_pos(c)] = enc_lane(k[c]);
    lanes[7] = kStateReady;
#pragma unroll
    for (int w = 0; w < KW; ++w) {
        out.w[w].x = lanes[w * 8 + 0] | (lanes[w * 8 + 1] << 16);
        out.w[w].y = lanes[w * 8 + 2] | (lanes[w * 8 + 3] << 16);
        out.w[w].z = lanes[w * 8 + 4] | (lanes[w * 8 + 5] << 16);
        out.w[w].w = lanes[w * 8 + 6] | (lanes[w * 8 + 7] << 16);
    }
}

template <int D>
__device__ __forceinline__ void unpack_key(const Key<key_words(D)>& in, int (&k)[D]) {
#pragma unroll
    for (int c = 0; c < D; ++c) {
        const uint4& w = in.w[lane_word(c)];
        int p = lane_pos(c);
        uint32_t u = word_u32(w, p >> 1);
        k[c] = dec_lane((p & 1) ? (u >> 16) : (u & 0xFFFFu));
    }
}

__device__ __forceinline__ uint32_t word_state(const uint4& w) { return w.w >> 16; }
__device__ __forceinline__ bool maybe_empty(const uint4& w) {
    return w.x == 0xFFFFFFFFu || w.y == 0xFFFFFFFFu || w.z == 0xFFFFFFFFu || w.w == 0xFFFFFFFFu;
}
__device__ __forceinline__ bool is_empty_word(const uint4& w) {
    return w.x == 0xFFFFFFFFu && w.y == 0xFFFFFFFFu && w.z == 0xFFFFFFFFu && w.w == 0xFFFFFFFFu;
}
__device__ __forceinline__ bool words_equal(const uint4& a, const uint4& b) {
    return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}
// equal in coordinates 0..6 (the state lane is ignored)
__device__ __forceinline__ bool prefix_equal(const uint4& a, const uint4& b) {
    return a.x == b.x && a.y == b.y && a.z == b.z && (a.w & 0xFFFFu) == (b.w & 0xFFFFu);
}
__device__ __forceinline__ uint4 with_state(uint4 w, uint32_t s) {
    w.w = (w.w & 0xFFFFu) | (s << 16);
    return w;
}

// Multiplicative hash over the key's 64-bit halves: each step multiplies by an odd
// constant, which carries every input bit into the high half; the final fold brings the
// high half down.  The slot is then taken from the top bits (home_slot).
template <int KW>
__device__ __forceinline__ uint32_t key_hash(const Key<KW>& k) {
    uint64_t h = 0x2545F4914F6CDD1Dull;
#pragma unroll
    for (int w = 0; w < KW; ++w) {
        uint4 q = k.w[w];
        if (w == 0) q.w &= 0xFFFFu;   // the state lane is not part of the key
        const uint64_t a = (uint64_t)q.x | ((uint64_t)q.y << 32);
        const uint64_t b = (uint64_t)q.z | ((uint64_t)q.w << 32);
        h = (h ^ a) * 0x9E3779B97F4A7C15ull;
        h = (h ^ b) * 0xC2B2AE3D27D4EB4Full;
    }
    h ^= h >> 29;
    return (uint32_t)(h >> 32) ^ (uint32_t)h;
}

// ---------------------------------------------------------------------------------
// Hash table: open addressing with linear probing over `cap` slots (any cap, mapped
// with a multiply-high).  key0[s] holds word 0, keyn[(w-1)*cap + s] the later words.
// The slot also owns an accumulator row vals[s*VDP..] and the first-touch entry ft[s]
// (smallest point*(d+1)+remainder that reached it), which later fixes the vertex's
// index: the reference numbers vertices in the order of their first insertion
// (src/Permutohedral.h:69-75).
// ---------------------------------------------------------------------------------
struct TableView {
    uint4* key0;       // word 0 of slot 0 of this table (a segment of a batch's slot array)
    uint4* keyn;       // word 1 of slot 0; word w at keyn[(w-1)*stride + s]
    uint32_t cap;      // slots of this table
    uint32_t stride;   // slots of the whole array
};

__device__ __forceinline__ uint32_t home_slot(uint32_t h, uint32_t cap) { return __umulhi(h, cap); }

// Insert-or-find during the splat, starting at slot `home` whose word 0 the caller has
// already loaded into `first` (so the loads of several keys can be in flight at once);
// returns the slot or -1 (status bit set).  *inserted, when given, is set when this call
// created the slot; *seen, when given, receives the word a found slot held.  XYZ: one-word
// keys of d <= 6 are compared on lanes 0..5 only, because a splat that numbers vertices as
// it creates them publishes each vertex's index in lanes 6-7 while others still insert.
template <int KW, bool XYZ = false>
__device__ int table_insert(const TableView& t, const Key<KW>& k, uint32_t home, uint4 first,
                            unsigned* status, bool* inserted = nullptr, uint4* seen = nullptr) {
    const uint4 empty = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
    uint32_t s = home;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        // A probe this long means a table (nearly) full: if the lattice has overflowed
        // already, give up at once, so a table sized too small fails fast and is rerun.
        if ((probe & 255) == 255 && (__ldcg(status) & kStatusProbeLimit)) return -1;
        uint4 w = probe == 0 ? first : __ldcg(&t.key0[s]);
        if (maybe_empty(w)) {
            // An empty slot, or a read that raced with the slot's one-time fill: the
            // compare-and-swap decides, and returns the slot's real contents.
            uint4 desired = (KW == 1) ? k.w[0] : with_state(k.w[0], kStatePending);
            w = atomicCAS(&t.key0[s], empty, desired);
            if (is_empty_word(w)) {
                if (inserted) *inserted = true;
                if (KW > 1) {
#pragma unroll
                    for (int i = 1; i < KW; ++i) __stcg(&t.keyn[(size_t)(i - 1) * t.stride + s], k.w[i]);
                    __threadfence();
                    atomicExch(&t.key0[s], k.w[0]);
                }
                return (int)s;
            }
        }
        if (KW == 1) {
            const bool eq = XYZ ? (w.x == k.w[0].x && w.y == k.w[0].y && w.z == k.w[0].z)
                                : words_equal(w, k.w[0]);
            if (eq) {
                if (seen) *seen = w;
                return (int)s;
            }
        } else if (prefix_equal(w, k.w[0])) {
            int spins = 0;
            while (word_state(w) == kStatePending) {
                if (++spins > kMaxSpin) {
                    atomicOr(status, kStatusSpinLimit);
                    return -1;
                }
                __nanosleep(64);
                w = __ldcg(&t.key0[s]);
            }
            __threadfence();
            bool same = true;
#pragma unroll
            for (int i = 1; i < KW; ++i)
                same = same && words_equal(__ldcg(&t.keyn[(size_t)(i - 1) * t.stride + s]), k.w[i]);
            if (same) return (int)s;
        }
        s = (s + 1 == t.cap) ? 0u : s + 1;
    }
    atomicOr(status, kStatusProbeLimit);
    return -1;
}

// For d <= 6 a one-word key leaves lanes 6 and 7 (the state lane) free of coordinates;
// the compaction (or the splat that numbers vertices as it creates them) stores the
// vertex's index there, so a neighbour lookup returns the index with the key.  Keys are
// then compared on lanes 0..5 only.  The index is stored as (v << 1) | 1: odd, so it never
// reads as the unnumbered word's lanes 6-7 (0x00008000) nor as an empty word's.
#ifndef PGPU_INDEX_IN_KEY_MAX_D
#define PGPU_INDEX_IN_KEY_MAX_D 6
#endif
__host__ __device__ constexpr bool index_in_key(int d) { return d <= PGPU_INDEX_IN_KEY_MAX_D; }
__device__ __forceinline__ uint32_t enc_index(uint32_t v) { return (v << 1) | 1u; }
__device__ __forceinline__ bool has_index(uint32_t w) { return (w & 1u) != 0; }
__device__ __forceinline__ uint32_t dec_index(uint32_t w) { return w >> 1; }

template <int D>
__device__ __forceinline__ bool key_match(const uint4& w, const uint4& k) {
    if constexpr (index_in_key(D)) return w.x == k.x && w.y == k.y && w.z == k.z;
    else return key_words(D) == 1 ? words_equal(w, k) : prefix_equal(w, k);
}

// Lookup in a table that no thread modifies any more (after the splat); -1 if absent.
template <int D>
__device__ __forceinline__ int table_find(const TableView& t, const Key<key_words(D)>& k, uint32_t h) {
    constexpr int KW = key_words(D);
    uint32_t s = home_slot(h, t.cap);
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        uint4 w = __ldg(&t.key0[s]);
        if (is_empty_word(w)) return -1;
        if (KW == 1) {
            if (key_match<D>(w, k.w[0])) return (int)s;
        } else if (prefix_equal(w, k.w[0])) {
            bool same = true;
#pragma unroll
            for (int i = 1; i < KW; ++i)
                same = same && words_equal(__ldg(&t.keyn[(size_t)(i - 1) * t.stride + s]), k.w[i]);
            if (same) return (int)s;
        }
        s = (s + 1 == t.cap) ? 0u : s + 1;
    }
    return -1;
}

// The vertex index of a key after the compaction, for d <= 6 (index_in_key); -1 if absent.
template <int D>
__device__ __forceinline__ int table_find_index(const TableView& t, const Key<1>& k, uint32_t h) {
    static_assert(index_in_key(D), "the vertex index lives in the key word for d <= 6 only");
    uint32_t s = home_slot(h, t.cap);
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        const uint4 w = __ldg(&t.key0[s]);
        if (is_empty_word(w)) return -1;
        if (key_match<D>(w, k.w[0])) return (int)dec_index(w.w);
        s = (s + 1 == t.cap) ? 0u : s + 1;
    }
    return -1;
}

// One byte per slot summarising its key (0: empty), written by the compaction: lookups of
// keys that are mostly absent (the blur's neighbours) read the small tag array, which
// stays in L2, and touch a slot's key only when its tag matches.
__device__ __forceinline__ uint8_t slot_tag(uint32_t h) { return (uint8_t)(h | 1u); }

template <int KW>
__device__ __forceinline__ int table_find_tagged(const TableView& t, const uint8_t* tags, const Key<KW>& k,
                                                 uint32_t h) {
    const uint8_t tag = slot_tag(h);
    uint32_t s = home_slot(h, t.cap);
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        const uint8_t g = __ldg(tags + s);
        if (g == 0) return -1;
        if (g == tag) {
            const uint4 w = __ldg(&t.key0[s]);
            bool same = KW == 1 ? words_equal(w, k.w[0]) : prefix_equal(w, k.w[0]);
#pragma unroll
            for (int i = 1; i < KW; ++i)
                same = same && words_equal(__ldg(&t.keyn[(size_t)(i - 1) * t.stride + s]), k.w[i]);
            if (same) return (int)s;
        }
        s = (s + 1 == t.cap) ? 0u : s + 1;
    }
    return -1;
}

// ---------------------------------------------------------------------------------
// The simplex that encloses one point: src/Permutohedral.h:293-356.
// ---------------------------------------------------------------------------------
struct LatticeConsts {
    float sf[kMaxD];   // scaleFactor[i] (src/Permutohedral.h:257-274), computed on the host
    float inv_d1;      // 1.0f/(d+1), computed on the host
};

template <int D>
struct Simplex {
    int g[D + 1];      // greedy[] after the hyperplane correction (int16 values)
    int rank[D + 1];
    float bary[D + 1]; // barycentric weight of remainder r
};

// Per-thread shared-memory column for compute_simplex: element k at col[k * stride].
struct SimplexScratch {
    float* delta;            // d+1 floats: delta of the coordinate of rank k
    unsigned char* coord;    // d+1 bytes: the coordinate of rank k
    int stride;
};

template <int D>
__device__ __forceinline__ void compute_simplex(const float (&p)[D], const LatticeConsts& lc,
                                                Simplex<D>& sx, unsigned* range_flag,
                                                const SimplexScratch& scr) {
    float e[D + 1];
    // elevated[d] = -d*position[d-1]*scaleFactor[d-1]
    e[D] = __fmul_rn(__fmul_rn((float)(-D), p[D - 1]), lc.sf[D - 1]);
#pragma unroll
    for (int i = D - 1; i > 0; --i) {
        float a = __fmul_rn(__fmul_rn((float)i, p[i - 1]), lc.sf[i - 1]);
        float c = __fmul_rn(__fmul_rn((float)(i + 2), p[i]), lc.sf[i]);
        e[i] = __fadd_rn(__fsub_rn(e[i + 1], a), c);
    }
    e[0] = __fadd_rn(e[1], __fmul_rn(__fmul_rn(2.0f, p[0]), lc.sf[0]));

    const float scale = lc.inv_d1;
    const float dp1 = (float)(D + 1);
    int sum = 0;
    bool out_of_range = false;
#pragma unroll
    for (int i = 0; i <= D; ++i) {
        float v = __fmul_rn(e[i], scale);
        // ceilf(v)*(d+1) is floorf(v)*(d+1) + (d+1) exactly (small integers times d+1)
        // unless v is an integer, where the reference's up == down; then down + (d+1) is
        // never the nearer one, so the pick is the same down
        float down = __fmul_rn(floorf(v), dp1);
        float up = __fadd_rn(down, dp1);
        float pick = (__fsub_rn(up, e[i]) < __fsub_rn(e[i], down)) ? up : down;
        out_of_range |= !(fabsf(pick) <= 32767.0f);
        // in range the reference's conversion (float -> int -> short) is the plain
        // truncating one; out of range the call fails (flagged below)
        int gi = __float2int_rz(pick);
        sx.g[i] = gi;
        sum += gi;
    }
    if (out_of_range && range_flag) atomicOr(range_flag, kStatusKeyRange);
    sum /= (D + 1);   // C division: truncation toward zero

    // rank differential; ties count for j (src/Permutohedral.h:321-324)
    float diff[D + 1];
#pragma unroll
    for (int i = 0; i <= D; ++i) {
        sx.rank[i] = 0;
        diff[i] = __fsub_rn(e[i], (float)sx.g[i]);
    }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = i + 1; j <= D; ++j) {
            if (diff[i] < diff[j]) sx.rank[i]++;
            else sx.rank[j]++;
        }

    // back onto the hyperplane (src/Permutohedral.h:326-348)
    if (sum > 0) {
#pragma unroll
        for (int i = 0; i <= D; ++i) {
            if (sx.rank[i] >= D + 1 - sum) {
                sx.g[i] = (int)(short)(sx.g[i] - (D + 1));
                sx.rank[i] += sum - (D + 1);
            } else {
                sx.rank[i] += sum;
            }
        }
    } else if (sum < 0) {
#pragma unroll
        for (int i = 0; i <= D; ++i) {
            if (sx.rank[i] < -sum) {
                sx.g[i] = (int)(short)(sx.g[i] + (D + 1));
                sx.rank[i] += (D + 1) + sum;
            } else {
                sx.rank[i] += sum;
            }
        }
    }

    // Barycentric weights (src/Permutohedral.h:351-356).  b[k] receives +delta of the
    // coordinate ranked d-k and -delta of the one ranked d+1-k; in IEEE arithmetic both
    // accumulation orders give delta_plus - delta_minus.  The ranks are a permutation of
    // 0..d, so the deltas are scattered by rank into this thread's shared-memory column
    // and read back in rank order (with the coordinate of each rank, for the key walk).
    // Ranks outside [0, d] only arise with keys outside int16, which is flagged above.
#pragma unroll
    for (int i = 0; i <= D; ++i) {
        const float delta = __fmul_rn(__fsub_rn(e[i], (float)sx.g[i]), scale);
        if ((unsigned)sx.rank[i] <= (unsigned)D) {
            scr.delta[sx.rank[i] * scr.stride] = delta;
            scr.coord[sx.rank[i] * scr.stride] = (unsigned char)i;
        }
    }
    float srt[D + 1];
#pragma unroll
    for (int k = 0; k <= D; ++k) srt[k] = scr.delta[k * scr.stride];
    // b[0] = delta(rank d) + (1 + b[d+1]),  b[d+1] = -delta(rank 0)
    sx.bary[0] = __fadd_rn(srt[D], __fadd_rn(1.0f, -srt[0]));
#pragma unroll
    for (int k = 1; k <= D; ++k) sx.bary[k] = __fsub_rn(srt[D - k], srt[D + 1 - k]);
}

// Key of remainder 0: the greedy point itself (canonical[0][j] = 0 for every j).
template <int D>
__device__ __forceinline__ void first_key(const Simplex<D>& sx, Key<key_words(D)>& k) {
    int kc[D];
#pragma unroll
    for (int i = 0; i < D; ++i) kc[i] = sx.g[i];
    pack_key<D>(kc, k);
}

// Key of remainder r+1 from that of r: with canonical[r][j] = r for j <= d-r, else r-(d+1)
// (src/Permutohedral.h:247-254), every stored coordinate grows by one except the one
// ranked d-r, which drops by d.  Stored lanes are int16 + 0x8000 mod 2^16, so the step is
// a per-lane 16-bit add (__vadd2) that wraps exactly like the reference's short keys.
// `coord` is the coordinate ranked d-r (d: the implied coordinate, no stored lane).
template <int D>
__device__ __forceinline__ void key_step(Key<key_words(D)>& k, int coord) {
    constexpr int KW = key_words(D);
#pragma unroll
    for (int w = 0; w < KW; ++w) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            uint32_t inc = 0;
            bool any = false;   // known at compile time once the loops are unrolled
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int lane = 2 * h + half;
                const int c = w == 0 ? lane : 7 + (w - 1) * 8 + lane;   // coordinate in this lane
                const bool stored = (w == 0 ? lane < 7 : true) && c < D;
                if (stored) {
                    const uint32_t step = coord == c ? (uint32_t)(uint16_t)(-D) : 1u;
                    inc |= step << (16 * half);
                    any = true;
                }
            }
            if (any) word_u32(k.w[w], h) = __vadd2(word_u32(k.w[w], h), inc);
        }
    }
}

// key of remainder r: greedy[i] + canonical[r*(d+1) + rank[i]] (src/Permutohedral.h:367-369),
// with canonical[r*(d+1)+j] = r for j <= d-r, else r-(d+1) (src/Permutohedral.h:247-254).
template <int D>
__device__ __forceinline__ void vertex_coords(const Simplex<D>& sx, int r, int (&k)[D]) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
        int c = (sx.rank[i] <= D - r) ? r : r - (D + 1);
        k[i] = (int)(short)(sx.g[i] + c);
    }
}

// ---------------------------------------------------------------------------------
// Payload (vertex value storage) conversions.
// ---------------------------------------------------------------------------------
template <typename P> struct Payload;
template <> struct Payload<float> {
    __device__ static float load(const float* p) { return *p; }
    __device__ static void store(float* p, float v) { *p = v; }
};
template <> struct Payload<double> {
    __device__ static double load(const double* p) { return *p; }
    __device__ static void store(double* p, double v) { *p = v; }
};
template <> struct Payload<__half> {
    __device__ static float load(const __half* p) { return __half2float(*p); }
    __device__ static void store(__half* p, float v) { *p = __float2half_rn(v); }
};
template <> struct Payload<__nv_bfloat16> {
    __device__ static float load(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ static void store(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

}  // namespace pgpu
