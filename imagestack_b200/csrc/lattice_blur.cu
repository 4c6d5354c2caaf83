// Blur launchers: one or two axes per pass, every payload and row-type combination the
// pass plan uses (its own file so the variants compile in parallel with the rest).
#include "lattice_ops.h"

namespace pgpu {
namespace {

// blocks of 256 threads over `work` vertex slots: capped at 16 per SM (the kernels stride
// over the vertices; modes 0 and 2), or one vertex per thread (mode 1)
int grid_blur(uint64_t work, int sms, int mode) {
    uint64_t g = (work + 255) / 256;
    const uint64_t cap = mode == 1 ? 0x7FFFFFFFull : (uint64_t)sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

template <int VDP, typename PS, typename PD, bool HOMOG>
void blur_t(const BlurArgs& a, bool pair, int blocks, int ilp, cudaStream_t st) {
    if (pair) blur_kernel<VDP, PS, PD, HOMOG, true, 1><<<blocks, 256, 0, st>>>(a);
    else if (ilp == 2) blur_kernel<VDP, PS, PD, HOMOG, false, 2><<<blocks, 256, 0, st>>>(a);
    else blur_kernel<VDP, PS, PD, HOMOG, false, 1><<<blocks, 256, 0, st>>>(a);
}

// 16-bit payload P: rows are P between passes, FP32 when read from the compaction
// (homogeneous lattices) or written for the slice (last pass)
template <int VDP, typename P, bool HOMOG>
void blur_16(const BlurArgs& a, bool src_f32, bool dst_acc, bool pair, int blocks,
             int ilp, cudaStream_t st) {
    if (src_f32 && dst_acc) blur_t<VDP, float, float, HOMOG>(a, pair, blocks, ilp, st);
    else if (src_f32) blur_t<VDP, float, P, HOMOG>(a, pair, blocks, ilp, st);
    else if (dst_acc) blur_t<VDP, P, float, HOMOG>(a, pair, blocks, ilp, st);
    else blur_t<VDP, P, P, HOMOG>(a, pair, blocks, ilp, st);
}

template <int VDP>
bool blur_v(const BlurArgs& a, int payload, bool homog, bool src_f32, bool dst_acc, bool pair,
            int blocks, int ilp, cudaStream_t st) {
    switch (payload) {
    case kPayloadF32:
        if (homog) return false;
        blur_t<VDP, float, float, false>(a, pair, blocks, ilp, st);
        return true;
    case kPayloadF64:
        if (homog) return false;
        blur_t<VDP, double, double, false>(a, pair, blocks, ilp, st);
        return true;
    case kPayloadF16:
        if (homog) blur_16<VDP, __half, true>(a, src_f32, dst_acc, pair, blocks, ilp, st);
        else blur_16<VDP, __half, false>(a, src_f32, dst_acc, pair, blocks, ilp, st);
        return true;
    case kPayloadBF16:
        if (homog) blur_16<VDP, __nv_bfloat16, true>(a, src_f32, dst_acc, pair, blocks, ilp, st);
        else blur_16<VDP, __nv_bfloat16, false>(a, src_f32, dst_acc, pair, blocks, ilp, st);
        return true;
    }
    return false;
}

}  // namespace

bool launch_blur(const BlurArgs& a, int blocks, int ilp, int vdp, int payload, bool homog,
                 bool src_f32, bool dst_acc, bool pair, cudaStream_t st) {
    switch (vdp) {
    case 2: return blur_v<2>(a, payload, homog, src_f32, dst_acc, pair, blocks, ilp, st);
    case 4: return blur_v<4>(a, payload, homog, src_f32, dst_acc, pair, blocks, ilp, st);
    case 8: return blur_v<8>(a, payload, homog, src_f32, dst_acc, pair, blocks, ilp, st);
    }
    return false;
}

int blur_all_axes(const BlurPlan& p, cudaStream_t st) {
    const int axes = p.d + 1;
    const int blocks = grid_blur(p.vmax, p.sms, p.grid);
    const bool p16 = p.payload == kPayloadF16 || p.payload == kPayloadBF16;
    if (p16 && !p.pairs && p.f32buf && axes >= 3) {
        // One axis per pass for 16-bit rows, rounded to 16 bits after every second axis,
        // exactly where fused pairs round them, so the result is bit-identical to pairs:
        // even passes write FP32 rows, odd passes 16-bit rows, the last FP32 rows for the
        // slice.  FP32 rows alternate between f32buf and sval (never sval right before the
        // last pass, which writes it), 16-bit rows between the two payload buffers.
        const void* cur = p.src;
        bool cur_f32 = p.src_f32;
        int hflip = 0;
        for (int j = 0; j < axes; ++j) {
            const bool last = j + 1 == axes;
            const bool out_f32 = last || j % 2 == 0;
            void* dst;
            if (last) {
                dst = p.sval;
            } else if (out_f32) {
                dst = cur == p.f32buf ? p.sval : p.f32buf;
            } else {
                dst = p.bufs[hflip];
                if (dst == cur) dst = p.bufs[hflip ^= 1];
                hflip ^= 1;
            }
            BlurArgs ba;
            ba.nbrA = p.nbr + (size_t)j * p.nbr_stride;
            ba.nbrB = nullptr;
            ba.nverts = p.nverts;
            ba.src = cur;
            ba.dst = dst;
            ba.dst_map = last ? p.vtx2slot : nullptr;
            ba.wc = p.wc;
            ba.products = last ? 1 : 0;
            if (!launch_blur(ba, blocks, p.grid == 2 ? 2 : 1, p.vdp, p.payload, p.homog, cur_f32, out_f32,
                             false, st))
                return 1;
            cur = dst;
            cur_f32 = out_f32;
        }
        return 0;
    }
    const void* src = p.src;
    bool src_f32 = p.src_f32;
    int flip = 0;
    for (int j = 0; j < axes;) {
        // (16-bit rows always pair here: one axis per pass would round them between axes)
        const bool pair = (p.pairs || p16) && j + 1 < axes;
        const int step = pair ? 2 : 1;
        const bool last = j + step >= axes;
        BlurArgs ba;
        ba.nbrA = p.nbr + (size_t)j * p.nbr_stride;
        ba.nbrB = pair ? p.nbr + (size_t)(j + 1) * p.nbr_stride : nullptr;
        ba.nverts = p.nverts;
        ba.src = src;
        ba.dst = last ? p.sval : p.bufs[flip];
        ba.dst_map = last ? p.vtx2slot : nullptr;
        ba.wc = p.wc;
        ba.products = last ? 1 : 0;
        if (!launch_blur(ba, blocks, p.grid == 2 ? 2 : 1, p.vdp, p.payload, p.homog, src_f32, last, pair, st))
            return 1;
        src = p.bufs[flip];
        flip ^= 1;
        src_f32 = false;
        j += step;
    }
    return 0;
}

}  // namespace pgpu
