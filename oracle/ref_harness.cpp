// Test-only harness around the reference ImageStack build (oracle/_ref).
//
// This file is part of the checker, not of the product.  It is compiled against the
// reference's own headers and linked with the reference library built from its own
// sources by oracle/Makefile; nothing of the reference is copied here.  It exposes a
// C ABI so that Python tests can
//   (1) drive the reference PermutohedralLattice directly (src/Permutohedral.h:172-508)
//       exactly the way GaussTransform::apply's PERMUTOHEDRAL branch does
//       (src/GaussTransform.cpp:163-226), and read back its private state: keys in
//       insertion order, the per-point replay records, values after splat and blur;
//   (2) call GaussTransform::apply, JointBilateral::apply and Bilateral::apply
//       (src/GaussTransform.cpp:115, 504, 730) on planar float images;
//   (3) run NLMeans3D::apply's steps (src/GaussTransform.cpp:934-941) and hand back the
//       PCA guide it filters against, which the reference computes from random patches.
// The replay record is private in the reference, so this harness opens the class with
// a preprocessor switch that only affects this translation unit.

#include <chrono>
#include <cstring>
#include <string>

#include "Arithmetic.h"
#include "Convolve.h"
#include "GaussTransform.h"
#include "Statistics.h"
#define private public
#include "Permutohedral.h"
#undef private

using namespace ImageStack;

namespace {

std::string g_error;

struct Handle {
    PermutohedralLattice lattice;
    int d, vd, n;
    Handle(int d_, int vd_, int n_) : lattice(d_, vd_, n_), d(d_), vd(vd_), n(n_) {}
};

// Planar dense image (x fastest, then y, t, c) -> Image, the layout of src/Image.h:34-43.
Image toImage(const float *src, int w, int h, int f, int c) {
    Image im(w, h, f, c);
    for (int ci = 0; ci < c; ci++) {
        for (int t = 0; t < f; t++) {
            for (int y = 0; y < h; y++) {
                memcpy(&im(0, y, t, ci), src + (((size_t)ci * f + t) * h + y) * w,
                       sizeof(float) * w);
            }
        }
    }
    return im;
}

void fromImage(const Image &im, float *dst) {
    for (int ci = 0; ci < im.channels; ci++) {
        for (int t = 0; t < im.frames; t++) {
            for (int y = 0; y < im.height; y++) {
                memcpy(dst + (((size_t)ci * im.frames + t) * im.height + y) * im.width,
                       &im(0, y, t, ci), sizeof(float) * im.width);
            }
        }
    }
}

GaussTransform::Method toMethod(int m) {
    switch (m) {
    case 1: return GaussTransform::EXACT;
    case 2: return GaussTransform::GRID;
    case 3: return GaussTransform::PERMUTOHEDRAL;
    case 4: return GaussTransform::GKDTREE;
    default: return GaussTransform::AUTO;
    }
}

}  // namespace

extern "C" {

const char *refh_last_error() { return g_error.c_str(); }

void *refh_lattice_create(int d, int vd, int n) { return new Handle(d, vd, n); }

void refh_lattice_destroy(void *h) { delete (Handle *)h; }

// Splat n points, interleaved pos[n*d] (already multiplied by 1/sigma) and val[n*vd],
// with replay recording, in the order GaussTransform.cpp:173-185 visits them.
void refh_lattice_splat(void *hp, const float *pos, const float *val, int n) {
    Handle *h = (Handle *)hp;
    std::vector<float> p(h->d), v(h->vd);
    for (int i = 0; i < n; i++) {
        memcpy(&p[0], pos + (size_t)i * h->d, sizeof(float) * h->d);
        memcpy(&v[0], val + (size_t)i * h->vd, sizeof(float) * h->vd);
        h->lattice.splat(&p[0], &v[0]);
    }
}

int refh_lattice_size(void *hp) { return ((Handle *)hp)->lattice.hashTable.size(); }

void refh_lattice_keys(void *hp, short *out) {
    Handle *h = (Handle *)hp;
    memcpy(out, h->lattice.hashTable.getKeys(),
           sizeof(short) * (size_t)h->d * h->lattice.hashTable.size());
}

void refh_lattice_values(void *hp, float *out) {
    Handle *h = (Handle *)hp;
    memcpy(out, h->lattice.hashTable.getValues(),
           sizeof(float) * (size_t)h->vd * h->lattice.hashTable.size());
}

// Replay records of the splat: vertex index (= value offset / vd) and weight, n*(d+1).
void refh_lattice_replay(void *hp, int *vtx, float *w) {
    Handle *h = (Handle *)hp;
    size_t cnt = (size_t)h->n * (h->d + 1);
    for (size_t i = 0; i < cnt; i++) {
        vtx[i] = h->lattice.replay[i].offset / h->vd;
        w[i] = h->lattice.replay[i].weight;
    }
}

void refh_lattice_blur(void *hp) { ((Handle *)hp)->lattice.blur(); }

// Replay slice of all n points (GaussTransform.cpp:196-207).
void refh_lattice_slice_replay(void *hp, float *out, int n) {
    Handle *h = (Handle *)hp;
    h->lattice.beginSlice();
    for (int i = 0; i < n; i++) h->lattice.slice(out + (size_t)i * h->vd);
}

// Re-elevation slice at distinct positions (GaussTransform.cpp:208-221).
void refh_lattice_slice_positions(void *hp, const float *pos, float *out, int n) {
    Handle *h = (Handle *)hp;
    std::vector<float> p(h->d);
    for (int i = 0; i < n; i++) {
        memcpy(&p[0], pos + (size_t)i * h->d, sizeof(float) * h->d);
        h->lattice.slice(&p[0], out + (size_t)i * h->vd);
    }
}

// GaussTransform::apply on planar images.  same != 0 passes one Image handle as both
// slice and splat, which selects the replay slice (GaussTransform.cpp:196).
// Returns elapsed seconds of the apply call, or -1 on an exception.
double refh_gauss_transform(const float *slice, const float *splat, int same,
                            const float *values, int w, int h, int f, int dpos, int vd,
                            const float *sigmas, int method, float *out) {
    try {
        Image sp = toImage(splat, w, h, f, dpos);
        Image sl = same ? sp : toImage(slice, w, h, f, dpos);
        Image va = toImage(values, w, h, f, vd);
        vector<float> sig(sigmas, sigmas + dpos);
        auto t0 = std::chrono::steady_clock::now();
        Image r = GaussTransform::apply(sl, sp, va, sig, toMethod(method));
        auto t1 = std::chrono::steady_clock::now();
        fromImage(r, out);
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (Exception &e) {
        g_error = e.message;
        return -1.0;
    }
}

// JointBilateral::apply, in place on im (GaussTransform.cpp:504-678).
double refh_joint_bilateral(float *im, const float *ref, int w, int h, int f, int cim,
                            int cref, float fw, float fh, float ft, float cs, int method) {
    try {
        Image a = toImage(im, w, h, f, cim);
        Image b = toImage(ref, w, h, f, cref);
        auto t0 = std::chrono::steady_clock::now();
        JointBilateral::apply(a, b, fw, fh, ft, cs, toMethod(method));
        auto t1 = std::chrono::steady_clock::now();
        fromImage(a, im);
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (Exception &e) {
        g_error = e.message;
        return -1.0;
    }
}

// Bilateral::apply, in place (GaussTransform.cpp:730-734).
double refh_bilateral(float *im, int w, int h, int f, int c, float fw, float fh, float ft,
                      float cs, int method) {
    try {
        Image a = toImage(im, w, h, f, c);
        auto t0 = std::chrono::steady_clock::now();
        Bilateral::apply(a, fw, fh, ft, cs, toMethod(method));
        auto t1 = std::chrono::steady_clock::now();
        fromImage(a, im);
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (Exception &e) {
        g_error = e.message;
        return -1.0;
    }
}

// NLMeans3D::apply, in place on im, with the three calls of its body
// (src/GaussTransform.cpp:934-941) made here so that the guide they produce can be
// returned: PatchPCA3D's filters (dims of them, drawn from random patches), the image
// convolved with them (Zero boundary, Inner product: dims channels), and the joint
// bilateral against that guide with frames INF.  guide receives dims planar channels.
double refh_nlmeans3d(float *im, float *guide, int w, int h, int f, int c, float patch,
                      int dims, float spatial, float patch_sigma, int method) {
    try {
        Image a = toImage(im, w, h, f, c);
        auto t0 = std::chrono::steady_clock::now();
        Image filters = PatchPCA3D::apply(a, patch, dims);
        Image pca = Convolve::apply(a, filters, Convolve::Zero, Multiply::Inner);
        fromImage(pca, guide);
        JointBilateral::apply(a, pca, spatial, spatial, INF, patch_sigma, toMethod(method));
        auto t1 = std::chrono::steady_clock::now();
        fromImage(a, im);
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (Exception &e) {
        g_error = e.message;
        return -1.0;
    }
}

}  // extern "C"
