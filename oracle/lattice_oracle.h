/* CPU oracle for the permutohedral-lattice Gauss transform (test infrastructure).
 *
 * A plain-C restatement of ImageStack's lattice (src/Permutohedral.h) used ONLY by the
 * tests, the smoke check and the CPU-baseline leg of the benchmark, as the checker.
 * It is never linked into the product library.  Its FP32 mode is pinned bit-exactly
 * against the reference build (oracle/_ref) and the committed golden fixtures.
 *
 * Points are interleaved: pos[i*d + k], val[i*vd + k]; positions are already scaled by
 * 1/sigma (src/GaussTransform.cpp:177).
 */
#ifndef LATTICE_ORACLE_H
#define LATTICE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lo_lattice lo_lattice;

/* scaleFactor table of the lattice constructor (src/Permutohedral.h:257-274). */
void lo_scale_factors(int d, float *sf);

/* Per point: the d+1 vertex keys (d int16 each, remainder order 0..d) and the
 * barycentric weights of those vertices (src/Permutohedral.h:293-369). */
void lo_simplex(int d, int n, const float *pos, short *keys, float *bary);

/* Lattice with FP32 (fp64 == 0, reference arithmetic) or FP64 (fp64 != 0) values. */
lo_lattice *lo_create(int d, int vd, int n, int fp64);
void lo_destroy(lo_lattice *L);
/* Splat n points with replay recording.  Returns 0, -1 on allocation failure, or -2 when
 * a point's elevated coordinates leave the int16 key range (the reference's behaviour is
 * undefined there: its rank indices leave [0, d]). */
int lo_splat(lo_lattice *L, const float *pos, const float *val, int n);
int lo_size(const lo_lattice *L);
void lo_keys(const lo_lattice *L, short *out);            /* M*d, insertion order */
void lo_values_f32(const lo_lattice *L, float *out);      /* M*vd (fp32 lattices) */
void lo_values_f64(const lo_lattice *L, double *out);     /* M*vd (either mode) */
void lo_replay(const lo_lattice *L, int *vtx, float *w);  /* n*(d+1) */
void lo_blur(lo_lattice *L);
/* Replay slice of the splatted points; out is n*vd. */
void lo_slice_replay_f32(const lo_lattice *L, float *out);
void lo_slice_replay_f64(const lo_lattice *L, double *out);
/* Re-elevation slice at other positions (missing vertices contribute zero). */
void lo_slice_positions_f32(const lo_lattice *L, const float *pos, int n, float *out);
void lo_slice_positions_f64(const lo_lattice *L, const float *pos, int n, double *out);

/* FP64 brute-force Gauss transform on selected queries:
 * out[i*vd+k] = sum_j exp(-0.5*|q_i - p_j|^2) * v[j*vd+k]. */
void lo_exact_gt_f64(int d, int vd, int nq, const float *q, int n, const float *p,
                     const float *v, double *out);

#ifdef __cplusplus
}
#endif
#endif
