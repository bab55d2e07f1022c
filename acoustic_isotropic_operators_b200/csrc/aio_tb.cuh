// Shared definitions of the interval-blocked stepper (aio_tile.cuh): pass
// modes, stored-wavefield precision, the per-CTA sparse device entries and the
// per-shot descriptor of one launch.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace aio {

// TB_ADJR: the adjoint recursion of TB_ADJ writing the finished coarse receiver sample
// R(its+1) (and R(0) at its == 0) instead of forming the Born image (extended imaging
// is done on those samples by the coarse kernels).
// TB_SCATX: the scattered pass of TB_SCAT with precomputed secondary-source slices (time-lag
// extended forward: ss(t) = sum_e ext[e] W[t - 2(e-h)]) in ring slots rSlot / rSlot0 of W.
// TB_SCATW: forward pass driven by dense secondary sources read from slices rSlot / rSlot0 of W
// (times dm when the launch has one), storing its finished coarse samples (tomo / WEMVA legs):
// sample its to slice oA of rcoarse, and at its == nts-2 sample its+1 to slice oB.
// TB_ADJX: the adjoint recursion (U = v2 * S) driven by dense secondary sources from slices
// rSlot / rSlot0 of W (times dm when given) built from a U-form receiver wavefield, so no v2
// factor is applied at injection; stores R(its+1) to slice oB and, at its == 0, R(0) to oA.
enum TBMode { TB_SRC = 0, TB_NL = 1, TB_SCAT = 2, TB_ADJ = 3, TB_ADJR = 4, TB_SCATX = 5, TB_SCATW = 6, TB_ADJX = 7 };
// modes whose injection is a dense secondary source staged from W (no sparse injection)
__host__ __device__ constexpr bool tb_scatlike(int mode) {
    return mode == TB_SCAT || mode == TB_SCATX || mode == TB_SCATW || mode == TB_ADJX;
}
// dense-source modes that also store coarse samples of the propagated field
__host__ __device__ constexpr bool tb_dense_out(int mode) { return mode == TB_SCATW || mode == TB_ADJX; }
// Stored source wavefield: FP32, BF16, or FP16 scaled per coarse slice and shot (the scale
// maps the slice's max |W| to 2^15, computed exactly from the finished FP32 slice).
enum TBWfld { TBW_F32 = 0, TBW_BF16 = 1, TBW_F16 = 2 };

struct TBEnt {   // sparse device entry of one CTA, sorted by column
    int col;     // interior x
    int row;     // interior z
    int dev;     // trace index
    int pad;
};

struct TBShot {
    const float* cur;     // input levels (interior slices)
    const float* old;
    float* ncur;          // output levels
    float* nold;
    const float* injSig;  // sparse injection traces
    float* recSig;        // sparse recording traces
    const int4* entStart; // per CTA: {inj begin, inj end, rec begin, rec end} into ent
    const TBEnt* ent;
    void* W;              // stored coarse wavefield [nts] (SRC: out, SCAT/ADJ: in)
    const float* part;    // coarse partial sum carried in (SRC: W[its], ADJ: R(its+1))
    float* partOut;       // coarse partial sum carried out (SRC: W[its+1], ADJ: R(its))
    double* img;          // ADJ: image accumulator (FP64 imaging)
    float* imgF;          // ADJ: image accumulator (FP32 imaging, the reference's precision)
    int injLd, recLd;
    // FP16 stored wavefield only
    float* wscale;        // [nts] value of one FP16 unit of slice t
    float* wstage;        // [2][isz] FP32 slices its and its+1 being accumulated (SRC)
    unsigned* wmax;       // [nts] max |W| of slice t as float bits (SRC)
    unsigned* wover;      // set to 1 when a slice stored with a speculative scale overflowed FP16 (SRC)
    float* rcoarse;       // ADJR / SCATW / ADJX: slices of coarse samples written by the launch
};

// Coarse slice t of a stored wavefield of `stride` elements per slice.
template <int WPREC>
__host__ __device__ inline void* tb_wslice(void* W, long long stride, int t) {
    return (char*)W + (long long)t * stride * (WPREC == TBW_F32 ? 4 : 2);
}

}  // namespace aio
