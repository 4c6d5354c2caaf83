// ImageStack plugin: the `permutohedral_gpu` (lattice) and `grid_gpu` (bilateral grid)
// methods for -gausstransform, -jointbilateral and -bilateral, and for the operations that
// end in JointBilateral::apply: -nlmeans, -nlmeans3d, -chromablur and -bilateralsharpen.
//
//     ImageStack -plugin libpermgpu_imagestack.so -load im.tmp \
//                -bilateral 0.1 16 16 0 permutohedral_gpu -save out.tmp
//
// The reference loads plugins with dlopen and hands its operation map to
// init_imagestack_plugin (src/Plugin.cpp:27-36).  This plugin replaces the operations
// with subclasses whose parse() accepts the extra method token (same argument grammar as
// src/GaussTransform.cpp:79-113, 473-502, 699-728, 755, 785, 843-865, 908-930) and
// forwards every other argument list to the original operation, so the CPU methods keep
// working unchanged.  The reference's GaussTransform::Method enum cannot grow without
// editing the reference, so the method is selected here, in parse().  The callers' own
// steps around the filter (patch PCA and its convolution, the colour conversions, the
// sharpening mix) run on the host through the reference's functions, in the order of
// their apply() bodies; only the joint bilateral moves to the GPU.
//
// The GPU work goes through the C ABI of libpermgpu.so (include/permgpu.h) on the
// images' host memory; a failing call becomes panic(), the reference's error convention
// (src/Exception.cpp:18-33).  Built against the reference's headers; the ImageStack
// symbols resolve from the executable, which links with -rdynamic.
#include <string>
#include <vector>

#include "Arithmetic.h"
#include "Color.h"
#include "Convolve.h"
#include "GaussTransform.h"
#include "Statistics.h"
#include "permgpu.h"

using namespace ImageStack;

namespace {

// method tokens: the permutohedral lattice and the bilateral grid on the GPU
int method_code(const string& tok) {
    if (tok == "permutohedral_gpu") return PGPU_METHOD_PERMUTOHEDRAL;
    if (tok == "grid_gpu") return PGPU_METHOD_GRID;
    return -1;
}

pgpu_image view_of(const Image& im) {
    pgpu_image v;
    v.base = im.baseAddress();
    v.width = im.width;
    v.height = im.height;
    v.frames = im.frames;
    v.channels = im.channels;
    v.ystride = im.ystride;
    v.tstride = im.tstride;
    v.cstride = im.cstride;
    return v;
}

void check(int rc, int method) {
    if (rc != PGPU_OK)
        panic("%s: %s\n", method == PGPU_METHOD_GRID ? "grid_gpu" : "permutohedral_gpu", pgpu_last_error());
}

pgpu_options host_options(int method) {
    pgpu_options o;
    pgpu_default_options(&o);
    o.memory = PGPU_MEM_HOST;
    o.method = method;
    return o;
}

// GaussTransform::apply for the GPU method: a new un-normalised image with the slice
// positions' size and the values' channels (src/GaussTransform.cpp:194).
Image gauss_transform_gpu(Image slice, Image splat, Image values, const vector<float>& sigmas,
                          int method = PGPU_METHOD_PERMUTOHEDRAL) {
    assert(splat.width == values.width && splat.height == values.height &&
               splat.frames == values.frames,
           "Weights and locations of the Gaussians must be the same size\n");
    assert(slice.channels == splat.channels,
           "The evaluation locations and the locations of the Gaussians must have"
           " the same number of channels.\n");
    Image out(slice.width, slice.height, slice.frames, values.channels);
    pgpu_image s = view_of(slice), p = view_of(splat), v = view_of(values), o = view_of(out);
    const pgpu_options opt = host_options(method);
    check(pgpu_gauss_transform(slice == splat ? nullptr : &s, &p, &v, sigmas.data(),
                               (int)sigmas.size(), &o, &opt), method);
    return out;
}

void joint_bilateral_gpu(Image im, Image ref, float fw, float fh, float ft, float cs,
                         int method = PGPU_METHOD_PERMUTOHEDRAL) {
    pgpu_image a = view_of(im), b = view_of(ref);
    const pgpu_options opt = host_options(method);
    check(pgpu_joint_bilateral(&a, &b, fw, fh, ft, cs, &opt), method);
}

class GpuGaussTransform : public GaussTransform {
public:
    void help() {
        GaussTransform::help();
        pprintf("With -plugin libpermgpu_imagestack.so the method may also be"
                " permutohedral_gpu (the permutohedral lattice) or grid_gpu (the bilateral"
                " grid), on a B200 GPU.\n");
    }

    bool test() {
        if (!GaussTransform::test()) return false;
        // the GPU method against the CPU lattice on GaussTransform::test's shapes
        Image splat(56, 34, 2, 3), slice(56, 34, 2, 3), values(56, 34, 2, 2);
        Noise::apply(splat, 0, 1);
        Noise::apply(slice, 0, 1);
        Noise::apply(values, 0, 1);
        values.channel(1).set(1.0f);
        vector<float> sigma(3);
        sigma[0] = 0.2f;
        sigma[1] = 0.3f;
        sigma[2] = 0.4f;
        Image cpu = GaussTransform::apply(slice, splat, values, sigma, PERMUTOHEDRAL);
        Image gpu = gauss_transform_gpu(slice, splat, values, sigma);
        return nearlyEqual(gpu, cpu);
    }

    void parse(vector<string> args) {
        const int method = args.empty() ? -1 : method_code(args[0]);
        if (method < 0) {
            GaussTransform::parse(args);
            return;
        }
        vector<float> sigmas;   // src/GaussTransform.cpp:96-108
        if (args.size() == 1) {
            sigmas = vector<float>(stack(0).channels, 1.0f);
        } else if (args.size() == 2) {
            sigmas = vector<float>(stack(0).channels, readFloat(args[1]));
        } else if ((int)args.size() == 1 + stack(1).channels) {
            for (int i = 0; i < stack(0).channels; i++) sigmas.push_back(readFloat(args[i + 1]));
        } else {
            panic("-gausstransform takes one argument, two arguments, or one plus the"
                  " number of channels in the second image on the stack arguments\n");
        }
        Image im = gauss_transform_gpu(stack(0), stack(1), stack(2), sigmas, method);
        pop();
        push(im);
    }
};

// shared argument grammar of -jointbilateral and -bilateral (src/GaussTransform.cpp:473-499)
bool parse_bilateral_args(const vector<string>& args, const char* name, float* cs, float* fw,
                          float* fh, float* ft, int* method) {
    if (args.size() != 5 || (*method = method_code(args[4])) < 0) return false;
    *cs = readFloat(args[0]);
    *fw = *fh = readFloat(args[1]);
    *fh = readFloat(args[2]);
    *ft = readFloat(args[3]);
    (void)name;
    return true;
}

class GpuJointBilateral : public JointBilateral {
public:
    void help() {
        JointBilateral::help();
        pprintf("With -plugin libpermgpu_imagestack.so the method may also be"
                " permutohedral_gpu or grid_gpu.\n");
    }

    bool test() {
        if (!JointBilateral::test()) return false;
        Image im(60, 50, 3, 3), ref(60, 50, 3, 3);   // JointBilateral::test's shape
        Noise::apply(im, 0, 1);
        Noise::apply(ref, 0, 1);
        Image cpu = im.copy(), gpu = im.copy();
        JointBilateral::apply(cpu, ref, 3, 4, 1, 0.25, GaussTransform::PERMUTOHEDRAL);
        joint_bilateral_gpu(gpu, ref, 3, 4, 1, 0.25);
        return nearlyEqual(gpu, cpu);
    }

    void parse(vector<string> args) {
        float cs, fw, fh, ft;
        int method;
        if (!parse_bilateral_args(args, "-jointbilateral", &cs, &fw, &fh, &ft, &method)) {
            JointBilateral::parse(args);
            return;
        }
        joint_bilateral_gpu(stack(0), stack(1), fw, fh, ft, cs, method);
    }
};

class GpuBilateral : public Bilateral {
public:
    void help() {
        Bilateral::help();
        pprintf("With -plugin libpermgpu_imagestack.so the method may also be"
                " permutohedral_gpu or grid_gpu.\n");
    }

    bool test() {
        Image im(80, 60, 1, 3);
        Noise::apply(im, 0, 1);
        Image cpu = im.copy(), gpu = im.copy();
        Bilateral::apply(cpu, 4, 4, 0, 0.2, GaussTransform::PERMUTOHEDRAL);
        joint_bilateral_gpu(gpu, gpu, 4, 4, 0, 0.2);
        return nearlyEqual(gpu, cpu);
    }

    void parse(vector<string> args) {
        float cs, fw, fh, ft;
        int method;
        if (!parse_bilateral_args(args, "-bilateral", &cs, &fw, &fh, &ft, &method)) {
            Bilateral::parse(args);
            return;
        }
        Image im = stack(0);
        joint_bilateral_gpu(im, im, fw, fh, ft, cs, method);
    }
};

// ---------------------------------------------------------------------------------
// The callers of JointBilateral::apply (src/GaussTransform.cpp:739-941)
// ---------------------------------------------------------------------------------

// A smooth RGB test volume (gradients and a brighter rectangle) with uniform noise of
// +-noise, for the self-tests below (the reference's own tests load a JPEG).
Image test_volume(int w, int h, int f, float noise) {
    Image im(w, h, f, 3);
    for (int c = 0; c < 3; c++)
        for (int t = 0; t < f; t++)
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++) {
                    float v = 0.15f + 0.5f * (float)x / (float)w + 0.1f * (float)c + 0.02f * (float)t;
                    if (3 * x > w && 3 * x < 2 * w && 4 * y > h && 4 * y < 3 * h) v += 0.3f;
                    im(x, y, t, c) = v + (noise > 0 ? randomFloat(-noise, noise) : 0.0f);
                }
    return im;
}

// The patch-PCA guide of NLMeans::apply / NLMeans3D::apply (src/GaussTransform.cpp:
// 870-873, 937-940): the image convolved with its leading patch eigenvectors.  The
// reference's patch sampler draws patch centres at least half a patch from every border
// (src/Statistics.cpp:1712, 1732-1734, 1797, 1816-1818), which has no valid centre when
// an axis is shorter than a patch (the reference then samples out of bounds, and was seen
// to run for minutes on a one-frame -nlmeans3d); that is refused here.
Image pca_guide(Image im, float patch, int dims, bool volume) {
    const int side = ((int)(patch * 6 + 1)) | 1;
    assert(im.width >= side && im.height >= side && (!volume || im.frames >= side),
           "patches of %d pixels%s do not fit in a %dx%dx%d image\n", side,
           volume ? " (and frames)" : "", im.width, im.height, im.frames);
    Image filters = volume ? PatchPCA3D::apply(im, patch, dims) : PatchPCA::apply(im, patch, dims);
    return Convolve::apply(im, filters, Convolve::Zero, Multiply::Inner);
}

// -nlmeans / -nlmeans3d: four arguments and a method token (src/GaussTransform.cpp:843-865,
// 908-930).  The reference's apply ignores its method argument (its JointBilateral call
// takes AUTO, the lattice for the d = dims + 2 of these filters); the GPU token is honoured.
template <class Base, bool Volume>
class GpuNLMeansOp : public Base {
public:
    void help() {
        Base::help();
        pprintf("With -plugin libpermgpu_imagestack.so the fifth argument may also be"
                " permutohedral_gpu (the joint bilateral on a B200 GPU; the patch PCA stays"
                " on the host).\n");
    }

    bool test() {
        // the GPU filter against the reference's lattice on one PCA guide
        Image im = Volume ? test_volume(32, 24, 6, 0.2f) : test_volume(64, 48, 1, 0.2f);
        Image guide = pca_guide(im, Volume ? 0.5f : 1.0f, 6, Volume);
        Image cpu = im.copy(), gpu = im.copy();
        JointBilateral::apply(cpu, guide, 4, 4, INF, 0.4f, GaussTransform::PERMUTOHEDRAL);
        joint_bilateral_gpu(gpu, guide, 4, 4, INF, 0.4f);
        return nearlyEqual(gpu, cpu);
    }

    void parse(vector<string> args) {
        if (args.size() != 5 || method_code(args[4]) != PGPU_METHOD_PERMUTOHEDRAL) {
            Base::parse(args);
            return;
        }
        const float patch = readFloat(args[0]);
        const int dims = readInt(args[1]);
        const float spatial = readFloat(args[2]);
        const float patch_sigma = readFloat(args[3]);
        Image im = stack(0);
        Image guide = pca_guide(im, patch, dims, Volume);
        joint_bilateral_gpu(im, guide, spatial, spatial, INF, patch_sigma);
    }
};

// ChromaBlur::apply with the GPU filter (src/GaussTransform.cpp:792-804): the chrominance
// joint-bilateral filtered against the luminance, which is then put back.
Image chroma_blur_gpu(Image im, float spatial, float color, int method) {
    assert(im.channels == 3, "input must be a rgb image\n");
    Image yuv = ColorConvert::rgb2yuv(im);
    Image luminance = ColorConvert::rgb2y(im);
    joint_bilateral_gpu(yuv, luminance, spatial, spatial, 0, color, method);
    yuv.channel(0).set(luminance);
    return ColorConvert::yuv2rgb(yuv);
}

// -chromablur: two arguments, plus a method token here (src/GaussTransform.cpp:785-790).
class GpuChromaBlur : public ChromaBlur {
public:
    void help() {
        ChromaBlur::help();
        pprintf("With -plugin libpermgpu_imagestack.so a third argument permutohedral_gpu"
                " or grid_gpu runs the filter on a B200 GPU (the reference's AUTO choice for"
                " its three position channels is the grid).\n");
    }

    bool test() {
        Image im = test_volume(72, 56, 1, 0.05f);
        Image grid = ChromaBlur::apply(im, 2, 0.5);   // AUTO: the grid
        return nearlyEqual(chroma_blur_gpu(im, 2, 0.5, PGPU_METHOD_GRID), grid);
    }

    void parse(vector<string> args) {
        const int method = args.size() == 3 ? method_code(args[2]) : -1;
        if (method < 0) {
            ChromaBlur::parse(args);
            return;
        }
        Image im = chroma_blur_gpu(stack(0), readFloat(args[0]), readFloat(args[1]), method);
        pop();
        push(im);
    }
};

// -bilateralsharpen: three arguments, plus a method token here (src/GaussTransform.cpp:
// 755-766): im * (1 + sharpness) - bilateral(im) * sharpness.
class GpuBilateralSharpen : public BilateralSharpen {
public:
    void help() {
        BilateralSharpen::help();
        pprintf("With -plugin libpermgpu_imagestack.so a fourth argument permutohedral_gpu"
                " or grid_gpu runs the bilateral filter on a B200 GPU.\n");
    }

    static Image sharpen_gpu(Image im, float spatial, float color, float sharpness, int method) {
        Image out = im.copy();
        joint_bilateral_gpu(out, out, spatial, spatial, 0, color, method);
        return im * (1 + sharpness) - out * sharpness;
    }

    bool test() {
        Image im = test_volume(80, 60, 1, 0.05f);
        Image cpu = BilateralSharpen::apply(im, 8, 0.25, 0.5);   // AUTO: the lattice (d = 5)
        return nearlyEqual(sharpen_gpu(im, 8, 0.25, 0.5, PGPU_METHOD_PERMUTOHEDRAL), cpu);
    }

    void parse(vector<string> args) {
        const int method = args.size() == 4 ? method_code(args[3]) : -1;
        if (method < 0) {
            BilateralSharpen::parse(args);
            return;
        }
        Image im = sharpen_gpu(stack(0), readFloat(args[0]), readFloat(args[1]), readFloat(args[2]), method);
        pop();
        push(im);
    }
};

void install(map<string, Operation*>& ops, const char* name, Operation* op) {
    map<string, Operation*>::iterator it = ops.find(name);
    if (it != ops.end()) delete it->second;
    ops[name] = op;
}

}  // namespace

extern "C" void init_imagestack_plugin(map<string, Operation*>& operationMap) {
    install(operationMap, "-gausstransform", new GpuGaussTransform());
    install(operationMap, "-jointbilateral", new GpuJointBilateral());
    install(operationMap, "-bilateral", new GpuBilateral());
    install(operationMap, "-nlmeans", new GpuNLMeansOp<NLMeans, false>());
    install(operationMap, "-nlmeans3d", new GpuNLMeansOp<NLMeans3D, true>());
    install(operationMap, "-chromablur", new GpuChromaBlur());
    install(operationMap, "-bilateralsharpen", new GpuBilateralSharpen());
}
