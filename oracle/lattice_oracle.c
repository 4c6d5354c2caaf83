/* CPU oracle for the permutohedral-lattice Gauss transform — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the algorithm of ImageStack's src/Permutohedral.h, written
 * for checking the CUDA path.  Only the tests, the smoke check and the benchmark's CPU
 * baseline leg load it.  Parity is pinned: its FP32 mode reproduces the reference
 * build (oracle/_ref, strict IEEE flags) bit-for-bit on keys, vertex order, replay
 * records and values, which the CPU tests check on every run where the reference build
 * is present, and against the committed golden fixtures everywhere.
 *
 * Compile with -ffp-contract=off and without -ffast-math: every float expression below
 * is written in the reference's evaluation order, and contraction into FMA or
 * reassociation would change the lattice keys.
 */
#include "lattice_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- scale factors: src/Permutohedral.h:257-274 ---------------------------------- */
void lo_scale_factors(int d, float *sf) {
    for (int i = 0; i < d; i++) {
        float s = 1.0f / (sqrtf((float)(i + 1) * (i + 2)));
        s *= (d + 1) * sqrtf((float)(2.0 / 3));
        sf[i] = s;
    }
}

/* ---- one point onto its simplex: src/Permutohedral.h:293-369 --------------------- *
 * keys: (d+1) x d int16 (remainder-major), bary: d+1 weights (bary[r] for remainder r).
 * Work arrays e, g, rk, b have d+2 entries.                                          */
static int simplex_point(int d, const float *sf, const float *p, float *e, short *g,
                         int *rk, float *b, short *keys, float *bary) {
    /* elevation (:293-298): e[d] = ((-d)*p[d-1])*sf[d-1];
     * e[i] = (e[i+1] - (i*p[i-1])*sf[i-1]) + ((i+2)*p[i])*sf[i];  e[0] = e[1] + (2*p[0])*sf[0] */
    e[d] = (float)(-d) * p[d - 1] * sf[d - 1];
    for (int i = d - 1; i > 0; i--) {
        float a = (float)i * p[i - 1] * sf[i - 1];
        float c = (float)(i + 2) * p[i] * sf[i];
        e[i] = e[i + 1] - a + c;
    }
    e[0] = e[1] + 2.0f * p[0] * sf[0];

    /* greedy rounding to the nearest multiple of d+1 (:301-317) */
    const float scale = 1.0f / (float)(d + 1);
    int sum = 0;
    for (int i = 0; i <= d; i++) {
        float v = e[i] * scale;
        float up = ceilf(v) * (float)(d + 1);
        float down = floorf(v) * (float)(d + 1);
        float pick = (up - e[i] < e[i] - down) ? up : down;
        /* Outside the int16 range the reference's (short) cast wraps, its rank indices
         * leave [0, d] and it writes out of bounds: refuse such points. */
        if (!(fabsf(pick) <= 32767.0f)) return 1;
        g[i] = (short)(int)pick;
        sum += g[i];
    }
    sum /= d + 1;

    /* rank by the differential (:321-324); ties count for j */
    for (int i = 0; i <= d; i++) rk[i] = 0;
    for (int i = 0; i < d; i++)
        for (int j = i + 1; j <= d; j++)
            if (e[i] - (float)g[i] < e[j] - (float)g[j]) rk[i]++;
            else rk[j]++;

    /* move back onto the hyperplane (:326-348) */
    if (sum > 0) {
        for (int i = 0; i <= d; i++) {
            if (rk[i] >= d + 1 - sum) {
                g[i] = (short)(g[i] - (d + 1));
                rk[i] += sum - (d + 1);
            } else {
                rk[i] += sum;
            }
        }
    } else if (sum < 0) {
        for (int i = 0; i <= d; i++) {
            if (rk[i] < -sum) {
                g[i] = (short)(g[i] + (d + 1));
                rk[i] += (d + 1) + sum;
            } else {
                rk[i] += sum;
            }
        }
    }

    /* barycentric coordinates (:351-356) */
    for (int i = 0; i < d + 2; i++) b[i] = 0.0f;
    for (int i = 0; i <= d; i++) {
        float delta = (e[i] - (float)g[i]) * scale;
        b[d - rk[i]] += delta;
        b[d + 1 - rk[i]] -= delta;
    }
    b[0] += 1.0f + b[d + 1];

    /* keys of the d+1 vertices (:365-369): canonical simplex entry for coordinate i of
     * remainder r is r when rank[i] <= d-r, else r-(d+1) (:247-254). */
    for (int r = 0; r <= d; r++) {
        for (int i = 0; i < d; i++) {
            int c = (rk[i] <= d - r) ? r : r - (d + 1);
            keys[r * d + i] = (short)(g[i] + c);
        }
        bary[r] = b[r];
    }
    return 0;
}

void lo_simplex(int d, int n, const float *pos, short *keys, float *bary) {
    float sf[64], e[66], b[66];
    short g[66];
    int rk[66];
    lo_scale_factors(d, sf);
    for (int i = 0; i < n; i++)
        if (simplex_point(d, sf, pos + (size_t)i * d, e, g, rk, b,
                          keys + (size_t)i * (d + 1) * d, bary + (size_t)i * (d + 1))) {
            memset(keys + (size_t)i * (d + 1) * d, 0, sizeof(short) * (d + 1) * d);
            memset(bary + (size_t)i * (d + 1), 0, sizeof(float) * (d + 1));
        }
}

/* ---- lattice: open-addressed map from key to vertex index in insertion order ------- */
struct lo_lattice {
    int d, vd, n, fp64;
    float sf[64];
    size_t cap;          /* slots, power of two */
    int *slot;           /* vertex index or -1 */
    size_t M, Mcap;      /* vertices, allocated vertices */
    short *keys;         /* Mcap*d */
    float *vf;           /* Mcap*vd (fp32 mode) */
    double *vdbl;        /* Mcap*vd (fp64 mode) */
    int *rvtx;           /* n*(d+1) */
    float *rw;           /* n*(d+1) */
    size_t nrec;
};

static uint64_t key_hash(const short *k, int d) {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < d; i++) {
        h ^= (uint16_t)k[i];
        h *= 0xFF51AFD7ED558CCDull;
        h ^= h >> 29;
    }
    return h;
}

static int find(const lo_lattice *L, const short *k) {
    size_t h = key_hash(k, L->d) & (L->cap - 1);
    for (;;) {
        int v = L->slot[h];
        if (v < 0) return -1;
        if (memcmp(L->keys + (size_t)v * L->d, k, sizeof(short) * L->d) == 0) return v;
        h = (h + 1) & (L->cap - 1);
    }
}

static int rehash(lo_lattice *L, size_t ncap) {
    int *ns = (int *)malloc(sizeof(int) * ncap);
    if (!ns) return -1;
    for (size_t i = 0; i < ncap; i++) ns[i] = -1;
    for (size_t v = 0; v < L->M; v++) {
        size_t h = key_hash(L->keys + v * L->d, L->d) & (ncap - 1);
        while (ns[h] >= 0) h = (h + 1) & (ncap - 1);
        ns[h] = (int)v;
    }
    free(L->slot);
    L->slot = ns;
    L->cap = ncap;
    return 0;
}

/* find or append a zero-valued vertex; returns its index or -1 on allocation failure */
static int find_or_insert(lo_lattice *L, const short *k) {
    if (2 * (L->M + 1) > L->cap && rehash(L, L->cap * 2)) return -1;
    if (L->M == L->Mcap) {
        size_t nm = L->Mcap * 2;
        short *nk = (short *)realloc(L->keys, sizeof(short) * nm * L->d);
        if (!nk) return -1;
        L->keys = nk;
        if (L->fp64) {
            double *nv = (double *)realloc(L->vdbl, sizeof(double) * nm * L->vd);
            if (!nv) return -1;
            L->vdbl = nv;
        } else {
            float *nv = (float *)realloc(L->vf, sizeof(float) * nm * L->vd);
            if (!nv) return -1;
            L->vf = nv;
        }
        L->Mcap = nm;
    }
    size_t h = key_hash(k, L->d) & (L->cap - 1);
    for (;;) {
        int v = L->slot[h];
        if (v < 0) break;
        if (memcmp(L->keys + (size_t)v * L->d, k, sizeof(short) * L->d) == 0) return v;
        h = (h + 1) & (L->cap - 1);
    }
    int v = (int)L->M++;
    L->slot[h] = v;
    memcpy(L->keys + (size_t)v * L->d, k, sizeof(short) * L->d);
    if (L->fp64) memset(L->vdbl + (size_t)v * L->vd, 0, sizeof(double) * L->vd);
    else memset(L->vf + (size_t)v * L->vd, 0, sizeof(float) * L->vd);
    return v;
}

lo_lattice *lo_create(int d, int vd, int n, int fp64) {
    if (d < 1 || d > 63 || vd < 1) return NULL;
    lo_lattice *L = (lo_lattice *)calloc(1, sizeof(lo_lattice));
    if (!L) return NULL;
    L->d = d; L->vd = vd; L->n = n; L->fp64 = fp64;
    lo_scale_factors(d, L->sf);
    L->cap = 1 << 12;
    L->slot = (int *)malloc(sizeof(int) * L->cap);
    for (size_t i = 0; i < L->cap; i++) L->slot[i] = -1;
    L->Mcap = 1 << 10;
    L->keys = (short *)malloc(sizeof(short) * L->Mcap * d);
    if (fp64) L->vdbl = (double *)malloc(sizeof(double) * L->Mcap * vd);
    else L->vf = (float *)malloc(sizeof(float) * L->Mcap * vd);
    L->rvtx = (int *)malloc(sizeof(int) * ((size_t)n * (d + 1) + 1));
    L->rw = (float *)malloc(sizeof(float) * ((size_t)n * (d + 1) + 1));
    if (!L->slot || !L->keys || !(L->vf || L->vdbl) || !L->rvtx || !L->rw) {
        lo_destroy(L);
        return NULL;
    }
    return L;
}

void lo_destroy(lo_lattice *L) {
    if (!L) return;
    free(L->slot); free(L->keys); free(L->vf); free(L->vdbl); free(L->rvtx); free(L->rw);
    free(L);
}

/* splat (src/Permutohedral.h:372-390, record=true) */
int lo_splat(lo_lattice *L, const float *pos, const float *val, int n) {
    const int d = L->d, vd = L->vd;
    float e[66], b[66], bary[65];
    short g[66];
    int rk[66];
    short *keys = (short *)malloc(sizeof(short) * (d + 1) * d);
    if (!keys) return -1;
    for (int i = 0; i < n; i++) {
        const float *p = pos + (size_t)i * d;
        const float *v = val + (size_t)i * vd;
        if (simplex_point(d, L->sf, p, e, g, rk, b, keys, bary)) { free(keys); return -2; }
        for (int r = 0; r <= d; r++) {
            int vx = find_or_insert(L, keys + r * d);
            if (vx < 0) { free(keys); return -1; }
            if (L->fp64) {
                double *dst = L->vdbl + (size_t)vx * vd;
                for (int k = 0; k < vd; k++) dst[k] += (double)bary[r] * (double)v[k];
            } else {
                float *dst = L->vf + (size_t)vx * vd;
                for (int k = 0; k < vd; k++) dst[k] += bary[r] * v[k];
            }
            if (L->nrec < (size_t)L->n * (d + 1)) {
                L->rvtx[L->nrec] = vx;
                L->rw[L->nrec] = bary[r];
                L->nrec++;
            }
        }
    }
    free(keys);
    return 0;
}

int lo_size(const lo_lattice *L) { return (int)L->M; }

void lo_keys(const lo_lattice *L, short *out) {
    memcpy(out, L->keys, sizeof(short) * L->M * L->d);
}

void lo_values_f32(const lo_lattice *L, float *out) {
    if (L->fp64) {
        for (size_t i = 0; i < L->M * L->vd; i++) out[i] = (float)L->vdbl[i];
    } else {
        memcpy(out, L->vf, sizeof(float) * L->M * L->vd);
    }
}

void lo_values_f64(const lo_lattice *L, double *out) {
    if (L->fp64) {
        memcpy(out, L->vdbl, sizeof(double) * L->M * L->vd);
    } else {
        for (size_t i = 0; i < L->M * L->vd; i++) out[i] = L->vf[i];
    }
}

void lo_replay(const lo_lattice *L, int *vtx, float *w) {
    memcpy(vtx, L->rvtx, sizeof(int) * L->nrec);
    memcpy(w, L->rw, sizeof(float) * L->nrec);
}

/* blur along the d+1 lattice axes (src/Permutohedral.h:430-488) */
void lo_blur(lo_lattice *L) {
    const int d = L->d, vd = L->vd;
    const size_t M = L->M;
    short n1[64], n2[64];
    int *nb1 = (int *)malloc(sizeof(int) * (M ? M : 1));
    int *nb2 = (int *)malloc(sizeof(int) * (M ? M : 1));
    void *tmp = malloc((L->fp64 ? sizeof(double) : sizeof(float)) * (M ? M : 1) * vd);
    if (!nb1 || !nb2 || !tmp) { free(nb1); free(nb2); free(tmp); return; }
    for (int j = 0; j <= d; j++) {
        for (size_t i = 0; i < M; i++) {
            const short *k = L->keys + i * d;
            for (int c = 0; c < d; c++) {
                n1[c] = (short)(k[c] + 1);
                n2[c] = (short)(k[c] - 1);
            }
            if (j < d) {
                n1[j] = (short)(k[j] - d);
                n2[j] = (short)(k[j] + d);
            }
            nb1[i] = find(L, n1);
            nb2[i] = find(L, n2);
        }
        if (L->fp64) {
            double *old = L->vdbl, *nw = (double *)tmp;
            for (size_t i = 0; i < M; i++)
                for (int c = 0; c < vd; c++) {
                    double a = nb1[i] >= 0 ? old[(size_t)nb1[i] * vd + c] : 0.0;
                    double z = nb2[i] >= 0 ? old[(size_t)nb2[i] * vd + c] : 0.0;
                    nw[i * vd + c] = 0.25 * a + 0.5 * old[i * vd + c] + 0.25 * z;
                }
            L->vdbl = nw;
            tmp = old;
        } else {
            float *old = L->vf, *nw = (float *)tmp;
            for (size_t i = 0; i < M; i++)
                for (int c = 0; c < vd; c++) {
                    float a = nb1[i] >= 0 ? old[(size_t)nb1[i] * vd + c] : 0.0f;
                    float z = nb2[i] >= 0 ? old[(size_t)nb2[i] * vd + c] : 0.0f;
                    nw[i * vd + c] = 0.25f * a + 0.5f * old[i * vd + c] + 0.25f * z;
                }
            L->vf = nw;
            tmp = old;
        }
    }
    /* the value arrays swapped d+1 times; both buffers are Mcap-sized only if the
     * current one is the original allocation, so keep capacity consistent */
    if (L->fp64) {
        double *nv = (double *)malloc(sizeof(double) * L->Mcap * vd);
        if (nv) { memcpy(nv, L->vdbl, sizeof(double) * M * vd); free(L->vdbl); L->vdbl = nv; }
    } else {
        float *nv = (float *)malloc(sizeof(float) * L->Mcap * vd);
        if (nv) { memcpy(nv, L->vf, sizeof(float) * M * vd); free(L->vf); L->vf = nv; }
    }
    free(tmp); free(nb1); free(nb2);
}

/* replay slice (src/Permutohedral.h:418-427) */
void lo_slice_replay_f32(const lo_lattice *L, float *out) {
    const int d = L->d, vd = L->vd;
    for (int i = 0; i < L->n; i++) {
        float *o = out + (size_t)i * vd;
        for (int c = 0; c < vd; c++) o[c] = 0.0f;
        for (int r = 0; r <= d; r++) {
            size_t rec = (size_t)i * (d + 1) + r;
            float w = L->rw[rec];
            for (int c = 0; c < vd; c++) {
                float v = L->fp64 ? (float)L->vdbl[(size_t)L->rvtx[rec] * vd + c]
                                  : L->vf[(size_t)L->rvtx[rec] * vd + c];
                o[c] += w * v;
            }
        }
    }
}

void lo_slice_replay_f64(const lo_lattice *L, double *out) {
    const int d = L->d, vd = L->vd;
    for (int i = 0; i < L->n; i++) {
        double *o = out + (size_t)i * vd;
        for (int c = 0; c < vd; c++) o[c] = 0.0;
        for (int r = 0; r <= d; r++) {
            size_t rec = (size_t)i * (d + 1) + r;
            double w = L->rw[rec];
            for (int c = 0; c < vd; c++) {
                double v = L->fp64 ? L->vdbl[(size_t)L->rvtx[rec] * vd + c]
                                   : (double)L->vf[(size_t)L->rvtx[rec] * vd + c];
                o[c] += w * v;
            }
        }
    }
}

/* re-elevation slice (src/Permutohedral.h:358-383 with splatting=false) */
static void slice_positions(const lo_lattice *L, const float *pos, int n, float *of,
                            double *od) {
    const int d = L->d, vd = L->vd;
    float e[66], b[66], bary[65];
    short g[66];
    int rk[66];
    short *keys = (short *)malloc(sizeof(short) * (d + 1) * d);
    if (!keys) return;
    for (int i = 0; i < n; i++) {
        if (simplex_point(d, L->sf, pos + (size_t)i * d, e, g, rk, b, keys, bary)) {
            if (of) for (int c = 0; c < vd; c++) of[(size_t)i * vd + c] = NAN;
            if (od) for (int c = 0; c < vd; c++) od[(size_t)i * vd + c] = NAN;
            continue;
        }
        if (of) for (int c = 0; c < vd; c++) of[(size_t)i * vd + c] = 0.0f;
        if (od) for (int c = 0; c < vd; c++) od[(size_t)i * vd + c] = 0.0;
        for (int r = 0; r <= d; r++) {
            int vx = find(L, keys + r * d);
            if (vx < 0) continue;
            for (int c = 0; c < vd; c++) {
                size_t s = (size_t)vx * vd + c;
                if (of) of[(size_t)i * vd + c] += bary[r] * (L->fp64 ? (float)L->vdbl[s] : L->vf[s]);
                if (od) od[(size_t)i * vd + c] += (double)bary[r] * (L->fp64 ? L->vdbl[s] : (double)L->vf[s]);
            }
        }
    }
    free(keys);
}

void lo_slice_positions_f32(const lo_lattice *L, const float *pos, int n, float *out) {
    slice_positions(L, pos, n, out, NULL);
}

void lo_slice_positions_f64(const lo_lattice *L, const float *pos, int n, double *out) {
    slice_positions(L, pos, n, NULL, out);
}

/* ---- FP64 brute force (the concept of src/GaussTransform.cpp:135-162, in double and
 * with the true exponential instead of the reference's lookup table) -------------- */
void lo_exact_gt_f64(int d, int vd, int nq, const float *q, int n, const float *p,
                     const float *v, double *out) {
    for (int i = 0; i < nq; i++) {
        double *o = out + (size_t)i * vd;
        for (int c = 0; c < vd; c++) o[c] = 0.0;
        const float *qi = q + (size_t)i * d;
        for (int j = 0; j < n; j++) {
            const float *pj = p + (size_t)j * d;
            double dist = 0.0;
            for (int c = 0; c < d; c++) {
                double t = (double)qi[c] - (double)pj[c];
                dist += t * t;
            }
            double w = exp(-0.5 * dist);
            for (int c = 0; c < vd; c++) o[c] += w * (double)v[(size_t)j * vd + c];
        }
    }
}
