// Tiled interval stepper: one launch advances every shot of a wave by one
// coarse interval (T = sub = 4 fine steps), on 2-D register micro-tiles.
//
// Each CTA owns an interior z-strip of HZ output rows (recomputing 5*T halo
// rows on each side: R = HZ + 10T rows, NQ = R/4 row quads) and an x-chunk of
// LX output columns, and marches along x in blocks of BX = 16 columns. At
// iteration k the input block starts at column B = xs + 16k and time level t
// (t = 1..T) is computed on the columns [B - 5t, B - 5t + 16): the blocks of
// consecutive levels are skewed by the stencil half-width, so level t only
// needs level t-1 columns that are already in shared memory. Every time level
// 0..T-1 lives in a shared ring of KT_CB = 32 columns; one barrier separates
// the levels of an iteration.
//
// A thread owns a 4 (z) x 2 (x) micro-tile: row quad q (rows 4q..4q+3 of the
// strip, one float4) in columns c0, c0+1. Per level it reads 5 quads of each of
// its two columns (z-stencil and centre) and one quad of each of the 10
// neighbouring columns (x-stencil) as float4 from the ring of level t-1.
//
// The scheme per fine step is the reference's (F/src/kernelsGpu.cu:202-219,
// 513-552): S_t = D * (v2 * L(S_{t-1}) + 2 S_{t-1} - D * S_{t-2} + injection),
// with the second damping of p_cur applied when the level is used as p_old,
// D = taper[min(dist_z, dist_x)] = min(Dz, Dx) (monotone taper) and D = 0
// outside the interior so the zero boundary stays zero. Adjoint passes use the
// same recursion on U = v2 * S (stepAdjGpu, :574-610, multiplied by v2
// point-wise).
//
// Per-interval products — the coarse source-wavefield sample, receiver data,
// the imaging condition — are formed from the T levels of each output point
// when level T is computed; level T itself is only written to global memory.
// State slices use the interior layout (pitch ip = round_up(nzi, 32)).
#pragma once
#include <cuda_bf16.h>

#include "aio_common.cuh"
#include "aio_tb.cuh"

namespace aio {

constexpr int KT_T = 4;        // fine steps per launch (sub)
constexpr int KT_BX = 16;      // block columns per iteration
constexpr int KT_CB = 32;      // ring depth in columns of levels 1..T-1 (>= BX + 5T - 5 + 1 for the output reads)
constexpr int KT_CB0 = 64;     // ring depth of level 0: the next input block lands while the current one is read
constexpr int KT_RINGCOLS = KT_CB0 + (KT_T - 1) * KT_CB;
constexpr int KT_PADQ = 2;     // zero quads above and below every ring column
constexpr int KT_MAXQ = 42;    // row quads per strip (R <= 168, HZ <= 128)
constexpr int KT_MAXQ_S = 26;  // short-strip variant (R <= 104, HZ <= 64): two CTAs per SM fit
constexpr int KT_MAXQ_M = 30;  // mid-strip variant (R <= 120, HZ <= 80): two CTAs per SM fit (light modes)
// Variants holding up to KT_MAXQ_M row quads run two CTAs per SM; they read v^2 of level 1
// through L1 like the later levels instead of staging it in shared memory.
__host__ __device__ constexpr bool kt_v2s(int maxq) { return maxq > KT_MAXQ_M; }
// floats per ring column (compile-time offsets) of a variant holding up to maxq row quads
__host__ __device__ constexpr int kt_rs(int maxq) { return (maxq + 2 * KT_PADQ) * 4; }
constexpr int KT_RS = kt_rs(KT_MAXQ);
constexpr int KT_MAXT = (8 * KT_MAXQ + 31) / 32 * 32;  // threads per CTA (8 column pairs per quad)
static_assert(KT_CB >= KT_BX + 5 * KT_T - 5 + 1, "output stage reads level 1 5(T-1) columns behind its block");
static_assert(KT_CB >= KT_BX + 10, "a level is read 10 columns behind its block");

struct KTArgs {
    Geom g;
    Coefs c;
    const float* v2;       // interior slice (pitch ip)
    const float* taper;    // minPad entries
    const float* dm;       // SCAT (and SCATW / ADJX when set): scaled model perturbation (interior slice)
    const TBShot* shots;
    float h[2 * (SUB_MAX + 1)];
    int its;               // coarse interval
    int HZ, LX;            // strip rows (multiple of 4) / chunk columns
    int nStrips, nChunks;
    int NQ;                // row quads per strip (HZ/4 + 10)
    int iters;             // iterations per CTA
    int maxEnt;            // shared entry capacity
    long long wStride;     // elements per stored coarse slice (= isz)
    int rSlot, rSlot0;     // ADJR: ring slots of R(its+1) and (its == 0) R(0);
                           // SCATX / SCATW / ADJX: slices of W holding the sources at its, its+1
    int oA, oB;            // SCATW / ADJX: slices of rcoarse receiving the samples its, its+1
    int f16spec;           // FP16 source pass: store slices with the speculative scale where allowed
    int wRing;             // SRC: W is a ring of wRing FP32 slices (slice t in slot t % wRing); 0: all nts
    int imgF32;            // ADJ: accumulate the image in FP32 (imgF) instead of FP64 (img)
    int relIter;           // iteration at whose start the stream's next launch may begin its prologue
                           // (0: right after the dependency wait; >= iters: when the CTA exits)
};

// Per-thread staging slots (16 bytes each) filled by asynchronous copies: level-1 operands
// of the next iteration (old level: slots 0-1; v^2: 2-3 when v2s) and the output operands of
// the current iteration from slot kt_so(v2s) on (partial sum: +0..1, stored wavefield: +2..3,
// image: +4..7 in FP64, +4 and +6 in FP32; the scattered passes' sources: +0..3).
__host__ __device__ constexpr int kt_so(bool v2s) { return v2s ? 4 : 2; }
__host__ __device__ constexpr int kt_slots(int mode, bool v2s = true) {
    return kt_so(v2s) +
           (mode == TB_ADJ ? 8 : ((mode == TB_SRC || mode == TB_ADJR) ? 2 : (tb_scatlike(mode) ? 4 : 0)));
}
// Ring columns: levels 0..T-1, plus (scattered pass) the secondary sources dm*W[its] and
// dm*W[its+1] of the last 32 level-1 columns, formed once at level 1 and read by levels 2..T.
__host__ __device__ constexpr int kt_ringcols(int mode) { return KT_RINGCOLS + (tb_scatlike(mode) ? 2 * KT_CB : 0); }
// rings, staging, column damping table, per-launch injection values (T per entry), entries
inline size_t kt_smem_bytes(int mode, int threads, int iters, int maxEnt, int rs = KT_RS, bool v2s = true) {
    return (size_t)kt_ringcols(mode) * rs * sizeof(float) + (size_t)kt_slots(mode, v2s) * threads * 16 +
           (3 * ((size_t)iters * KT_BX + 64) + (size_t)maxEnt * KT_T) * sizeof(float) + (size_t)maxEnt * sizeof(TBEnt);
}

// cp.async: 16 (or 8) bytes global -> shared, zero-filled when !ok (no bytes are read then).
__device__ __forceinline__ void kt_cp16(void* s, const void* g, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(g), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void kt_cp16_l1(void* s, const void* g, bool ok) {  // also allocates in L1
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(g), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void kt_cp8(void* s, const void* g, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(g), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void kt_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void kt_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
// Programmatic dependent launch: a launch made with programmatic stream serialization may start
// while the previous kernel of its stream still runs. kt_grid_wait returns once that kernel has
// finished and its writes are visible (at once when there is no such dependency); before it a
// kernel reads only what the host uploaded ahead of the pass and writes only shared memory.
// kt_grid_release lets the next launch of the stream start its own prologue.
__device__ __forceinline__ void kt_grid_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void kt_grid_release() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
// four stored-wavefield samples from a staging slot (FP32: 16 bytes, BF16 / FP16: the first 8)
template <int WPREC>
__device__ __forceinline__ float4 kt_wfrom(const float4& slot, float sc) {
    if (WPREC == TBW_F32) return slot;
    const uint2 r = *reinterpret_cast<const uint2*>(&slot);
    if (WPREC == TBW_BF16) {
        const float2 fa = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.x));
        const float2 fb = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.y));
        return make_float4(fa.x, fa.y, fb.x, fb.y);
    }
    const float2 fa = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    const float2 fb = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    return make_float4(fa.x * sc, fa.y * sc, fb.x * sc, fb.y * sc);
}

template <int WPREC>
__device__ __forceinline__ float4 kt_wload4(const void* W, long long idx, float sc) {
    if (WPREC == TBW_F32) return __ldg(reinterpret_cast<const float4*>((const float*)W + idx));
    const uint2 r = __ldg(reinterpret_cast<const uint2*>((const unsigned short*)W + idx));
    if (WPREC == TBW_BF16) {
        const float2 fa = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.x));
        const float2 fb = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.y));
        return make_float4(fa.x, fa.y, fb.x, fb.y);
    }
    const float2 fa = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    const float2 fb = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    return make_float4(fa.x * sc, fa.y * sc, fb.x * sc, fb.y * sc);
}

template <int WPREC>
__device__ __forceinline__ void kt_wstore4(void* W, long long idx, const float v[4]) {
    if (WPREC == TBW_F32) {
        *reinterpret_cast<float4*>((float*)W + idx) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        const __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]);
        const __nv_bfloat162 b = __floats2bfloat162_rn(v[2], v[3]);
        uint2 r;
        r.x = *reinterpret_cast<const unsigned*>(&a);
        r.y = *reinterpret_cast<const unsigned*>(&b);
        *reinterpret_cast<uint2*>((__nv_bfloat16*)W + idx) = r;
    }
}

// FP16 unit of a slice whose max |W| is m (0 for an all-zero slice): m / 2^15
__device__ __forceinline__ float kt_f16_scale(unsigned maxBits) {
    const float m = __uint_as_float(maxBits);
    return m > 0.f ? m * (1.f / 32768.f) : 1.f;
}
// Speculative FP16 unit of slice t from the finished slice t-1 (max bits prevBits): the power of
// two 2^(e - 11) for a previous max in [2^e, 2^(e+1)), which maps that max into [2^11, 2^12).
// FP16 keeps 11 significant bits over its whole normal range, so this scale loses no precision
// against the exact one; it leaves headroom for slice t to grow 16x (up to 65504) before an
// overflow, which the source pass flags so the pass is run again with exact scales. Usable when
// the previous max is a normal float of at least 2^-115 (then the unit is a normal float too).
__host__ __device__ __forceinline__ bool kt_f16_spec_ok(unsigned prevBits) {
    const unsigned e = (prevBits >> 23) & 0xffu;
    return e >= 12u && e < 255u;
}
__device__ __forceinline__ float kt_f16_spec_scale(unsigned prevBits) {
    return __uint_as_float((((prevBits >> 23) & 0xffu) - 11u) << 23);
}
// slice t of a source pass was stored directly with the speculative scale (else staged in FP32
// and quantized with its exact max); slice 0 and the last slice are always staged
__device__ __forceinline__ bool kt_f16_spec_slice(const unsigned* wmax, int t, int nts, int spec) {
    return spec && t >= 1 && t <= nts - 2 && kt_f16_spec_ok(wmax[t - 1]);
}
// quantize four FP32 samples to FP16 units of `sc`
__device__ __forceinline__ uint2 kt_f16_pack(const float4& v, float sc) {
    const float inv = 1.f / sc;
    const __half2 a = __floats2half2_rn(v.x * inv, v.y * inv);
    const __half2 b = __floats2half2_rn(v.z * inv, v.w * inv);
    uint2 r;
    r.x = *reinterpret_cast<const unsigned*>(&a);
    r.y = *reinterpret_cast<const unsigned*>(&b);
    return r;
}

// FP16 stored wavefield: quantize the finished FP32 slice t (staging buffer) over the
// region [z0, z1) x [x0, x1) (z0 multiple of 4) with its exact scale.
__device__ __forceinline__ void kt_f16_quantize(const TBShot& sh, long long wStride, int ip, int t, int z0, int z1,
                                                int x0, int x1, int tid, int nthr) {
    const float sc = kt_f16_scale(sh.wmax[t]);
    const float* src = sh.wstage + (long long)(t & 1) * wStride;
    unsigned short* dst = (unsigned short*)sh.W + (long long)t * wStride;
    const int nq = (z1 - z0 + 3) / 4, n = nq * (x1 - x0);
    for (int i = tid; i < n; i += nthr) {
        const int x = x0 + i / nq, z = z0 + 4 * (i % nq);
        const long long idx = (long long)x * ip + z;
        *reinterpret_cast<uint2*>(dst + idx) = kt_f16_pack(*reinterpret_cast<const float4*>(src + idx), sc);
    }
}

// Finishes the last two slices (nts-2, nts-1) of an FP16 source pass (those staged in FP32) and
// records every slice's scale: the speculative one where the slice was stored directly.
__global__ void k_f16_finish(const TBShot* shots, long long wStride, int ip, int nzi, int nxi, int nts, int spec) {
    const TBShot sh = shots[blockIdx.y];
    const int nthr = gridDim.x * blockDim.x, tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = nts - 2; t < nts; t++)
        if (!kt_f16_spec_slice(sh.wmax, t, nts, spec)) kt_f16_quantize(sh, wStride, ip, t, 0, nzi, 0, nxi, tid, nthr);
    if (tid == 0)
        for (int t = 0; t < nts; t++)
            sh.wscale[t] = kt_f16_spec_slice(sh.wmax, t, nts, spec) ? kt_f16_spec_scale(sh.wmax[t - 1])
                                                                    : kt_f16_scale(sh.wmax[t]);
}

__device__ __forceinline__ float4 kt_ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void kt_st4(float* p, const float v[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ float kt_el(const float4& v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}
// rows (2h, 2h+1) of a quad
__device__ __forceinline__ float2 kt_half(const float4& v, int h) {
    return h == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
}
// rows (r, r+1), r in [-8, 10], of the 20-row window held as quads Z[0..4] (rows -8..11)
__device__ __forceinline__ float2 kt_pair(const float4 (&Z)[5], int r) {
    const int i = r + 8;
    return make_float2(kt_el(Z[i >> 2], i & 3), kt_el(Z[(i + 1) >> 2], (i + 1) & 3));
}

// element idx (0..19) of the 20-row window held as quads Z[0..4]
__device__ __forceinline__ float kt_win(const float4 (&Z)[5], int idx) { return kt_el(Z[idx >> 2], idx & 3); }
// Free surface, forward modes (setFsConditionFwdGpu, F/src/kernelsGpu.cu:555-567): the stencil
// sees the current level with its top interior row zeroed and rows -1..-5 set to minus rows
// 1..5. Applied to the z-window (rows zq-8 .. zq+11) of the threads whose outputs read row 0
// or above: zq = 0 (rows 0..3) and zq = 4 (rows 4..7), in whichever strip computes them.
__device__ __forceinline__ void kt_fs_window(float4 (&Z)[5], int zq) {
    float w[20];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        w[4 * i] = Z[i].x;
        w[4 * i + 1] = Z[i].y;
        w[4 * i + 2] = Z[i].z;
        w[4 * i + 3] = Z[i].w;
    }
    if (zq == 0) {  // row r at index r + 8
        w[8] = 0.f;
#pragma unroll
        for (int r = 1; r <= 5; r++) w[8 - r] = -w[8 + r];
    } else {        // zq == 4: row r at index r + 4
        w[4] = 0.f;
#pragma unroll
        for (int r = 1; r <= 4; r++) w[4 - r] = -w[4 + r];
    }
#pragma unroll
    for (int i = 0; i < 5; i++) Z[i] = make_float4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}
// 16-bit source field of tomo / WEMVA: coarse d2/dt2 (srcWfldSecondTimeDerivative,
// F/src/kernelsGpu.cu:188-197, k_dt2's expression) of the slices [t0, t1] (at most KT_DT2_B) of a
// source wavefield held in an FP32 ring of `ring` slices (slice t in slot t % ring; zero outside
// [0, nts)). BF16 stores the result; FP16 stages it in FP32 (slot t - t0 of `stage`) and folds
// each slice's max |d| into wmax[t] (one atomic per warp and slice) for k_dt2_f16_pack. Four
// points per thread (interior slices are whole float4s: isz % 32 == 0).
constexpr int KT_DT2_B = 32;
template <int WP>
__global__ void k_dt2_block(const float* __restrict__ ring, long long ringSt, int ringLen, void* out, long long outSt,
                            float* stage, long long stageSt, unsigned* wmax, int nts, long long isz, int t0, int t1,
                            float cSide, float cCenter) {
    const int b = blockIdx.y;
    ring += b * ringSt;
    float mx[KT_DT2_B];
#pragma unroll
    for (int k = 0; k < KT_DT2_B; k++) mx[k] = 0.f;
    const long long n4 = isz / 4;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
        const long long i = 4 * q;
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 prev = t0 > 0 ? *reinterpret_cast<const float4*>(ring + (long long)((t0 - 1) % ringLen) * isz + i) : z4;
        float4 c = *reinterpret_cast<const float4*>(ring + (long long)(t0 % ringLen) * isz + i);
#pragma unroll
        for (int k = 0; k < KT_DT2_B; k++) {
            const int t = t0 + k;
            if (t > t1) break;
            const float4 nx =
                t + 1 < nts ? *reinterpret_cast<const float4*>(ring + (long long)((t + 1) % ringLen) * isz + i) : z4;
            float d[4] = {cSide * (prev.x + nx.x) + cCenter * c.x, cSide * (prev.y + nx.y) + cCenter * c.y,
                          cSide * (prev.z + nx.z) + cCenter * c.z, cSide * (prev.w + nx.w) + cCenter * c.w};
            if (WP == TBW_BF16) {
                kt_wstore4<TBW_BF16>((unsigned short*)out + b * outSt + (long long)t * isz, i, d);
            } else {
                kt_st4(stage + b * stageSt + (long long)k * isz + i, d);
                mx[k] = fmaxf(mx[k], fmaxf(fmaxf(fabsf(d[0]), fabsf(d[1])), fmaxf(fabsf(d[2]), fabsf(d[3]))));
            }
            prev = c;
            c = nx;
        }
    }
    if (WP == TBW_F16) {
        // non-negative floats order like their bit patterns: one warp max, one atomic per warp
#pragma unroll
        for (int k = 0; k < KT_DT2_B; k++) {
            const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(mx[k]));
            if ((threadIdx.x & 31) == 0 && m && t0 + k <= t1) atomicMax(wmax + (long long)b * nts + t0 + k, m);
        }
    }
}
// FP16: slices [t0, t1] staged by k_dt2_block, quantized with each slice's exact unit (max / 2^15,
// kt_f16_scale), and the units recorded in wscale.
__global__ void k_dt2_f16_pack(const float* __restrict__ stage, long long stageSt, void* out, long long outSt,
                               const unsigned* __restrict__ wmax, float* wscale, int nts, long long isz, int t0,
                               int t1) {
    const int b = blockIdx.y;
    const long long n4 = isz / 4, tot = (long long)(t1 - t0 + 1) * n4;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q / n4);
        const long long i = 4 * (q - k * n4);
        const float sc = kt_f16_scale(wmax[(long long)b * nts + t0 + k]);
        const float4 v = *reinterpret_cast<const float4*>(stage + b * stageSt + (long long)k * isz + i);
        *reinterpret_cast<uint2*>((unsigned short*)out + b * outSt + (long long)(t0 + k) * isz + i) = kt_f16_pack(v, sc);
        if (i == 0) wscale[(long long)b * nts + t0 + k] = sc;
    }
}

__host__ __device__ constexpr bool kt_adj(int mode) { return mode == TB_ADJ || mode == TB_ADJR || mode == TB_ADJX; }

// FS: free surface at the top interior row (runs on the large-strip variant only)
template <int MODE, int WPREC, int MAXQ = KT_MAXQ, bool FS = false>
__global__ void __launch_bounds__((8 * MAXQ + 31) / 32 * 32, kt_v2s(MAXQ) ? 1 : 2) k_tile(const KTArgs a) {
    constexpr int T = KT_T;
    extern __shared__ float4 kt_smem4[];
    const int NQ = a.NQ;
    constexpr int RS = kt_rs(MAXQ);
    constexpr bool V2S = kt_v2s(MAXQ);
    constexpr int SO = kt_so(V2S);  // first output-operand slot
    constexpr int NS = kt_slots(MODE, V2S);
    float* ring = reinterpret_cast<float*>(kt_smem4);         // level 0: [KT_CB0][RS], levels 1..T-1: [KT_CB][RS]
    float4* stg = reinterpret_cast<float4*>(ring + kt_ringcols(MODE) * RS);  // [NS][blockDim.x]
    float* dxt = reinterpret_cast<float*>(stg + NS * blockDim.x);      // column damping, columns xs-32 ...
    const int nDx = a.iters * KT_BX + 64;                       // columns xs-32 .. of the tables below
    int* injFirst = reinterpret_cast<int*>(dxt + nDx);          // first injection entry of a column, or -1
    int* recFirst = injFirst + nDx;                             // first recording entry of a column, or -1
    float* sInjV = reinterpret_cast<float*>(recFirst + nDx);    // [maxEnt][T] injection value per level
    TBEnt* sEnt = reinterpret_cast<TBEnt*>(sInjV + a.maxEnt * T);

    const Geom& g = a.g;
    const TBShot sh = a.shots[blockIdx.z];
    float* __restrict__ pNcur = sh.ncur;
    float* __restrict__ pNold = sh.nold;
    const float* __restrict__ pPart = sh.part;
    float* __restrict__ pPartOut = sh.partOut;
    double* __restrict__ pImg = sh.img;
    float* __restrict__ pImgF = sh.imgF;
    float* __restrict__ pRec = sh.recSig;
    const float* __restrict__ pInj = sh.injSig;
    const float* __restrict__ cur = sh.cur;
    const float* __restrict__ old = sh.old;
    const float* __restrict__ v2p = a.v2;
    const float* __restrict__ dmp = a.dm;
    const int injLd = sh.injLd, recLd = sh.recLd;
    const int strip = blockIdx.x, chunk = blockIdx.y;
    const int ip = g.ip, nxi = g.nxi, nzi = g.nzi, H = g.H, sub = g.sub, its = a.its;

    const int tid = threadIdx.x;
    const int cp = tid / NQ;              // column pair 0..7 (>= 8: idle thread)
    const int q = tid - cp * NQ;          // row quad
    const bool act = cp < KT_BX / 2;
    const int z0 = strip * a.HZ;
    const int zq = z0 - 5 * T + 4 * q;    // first row of the quad (multiple of 4)
    const int x0 = chunk * a.LX;
    const int x1 = min(x0 + a.LX, nxi);
    const int xs = x0 - 5 * T;

    // ---- per-thread constants
    float Dz[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int z = zq + i;
        float d = 0.f;
        if (z >= 0 && z < nzi) {
            const int dd = FS ? nzi - 1 - z : min(z, nzi - 1 - z);  // dampCosineEdgeFs: no top taper
            d = dd < g.minPad ? __ldg(a.taper + dd) : 1.f;
        }
        Dz[i] = d;
    }
    const bool zLoad = act && zq >= 0 && zq < nzi;        // quad holds interior rows
    const int zv = min(max(zq, 0), ip - 4);               // clamped quad for v2 / operand reads
    const bool zOut = act && q >= 5 * T / 4 && q < 5 * T / 4 + a.HZ / 4 && zq < nzi;
    float2 zc2[6], xc2[6];  // coefficients, duplicated for paired instructions
#pragma unroll
    for (int i = 0; i < 6; i++) {
        zc2[i] = make_float2(a.c.zc[i], a.c.zc[i]);
        xc2[i] = make_float2(a.c.xc[i], a.c.xc[i]);
    }
    float* const ringQ = ring + (KT_PADQ + q) * 4;  // quad q of ring column 0, level 0
    // quad q of column c of level t's ring
    auto col = [&](int t, int c) -> float* {
        return t == 0 ? ringQ + (c & (KT_CB0 - 1)) * RS : ringQ + (KT_CB0 + (t - 1) * KT_CB + (c & (KT_CB - 1))) * RS;
    };
    // secondary-source rings of the scattered pass (s = 0: dm*W[its], 1: dm*W[its+1])
    auto ssCol = [&](int sidx, int c) -> float* { return ringQ + (KT_RINGCOLS + sidx * KT_CB + (c & (KT_CB - 1))) * RS; };
    float4* const mySlot = stg + tid;  // slot i of this thread: mySlot[i * blockDim.x]
    const int bd = blockDim.x;

    // Input of iteration k, issued one iteration ahead: the level-0 block [B, B+16) straight
    // into its ring slots, and the level-1 operands of iteration k (old level and v^2 at the
    // level-1 columns) into this thread's staging slots 0-3.
    auto issue_input = [&](int k) {
        if (!act) return;
        const int B = xs + KT_BX * k;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int c = B + 2 * cp + j;
            const bool okc = zLoad && c >= 0 && c < nxi;
            kt_cp16(col(0, c), okc ? cur + (long long)c * ip + zq : cur, okc);
            const int co = B - 5 + 2 * cp + j;
            const bool oko = zLoad && co >= 0 && co < nxi;
            kt_cp16(mySlot + j * bd, oko ? old + (long long)co * ip + zq : old, oko);
            const long long ic = (long long)min(max(co, 0), nxi - 1) * ip + zv;
            if (V2S) kt_cp16_l1(mySlot + (2 + j) * bd, v2p + ic, true);
            if (tb_scatlike(MODE)) {  // stored wavefield (or secondary sources) at its, its+1 (slots 4-7)
                const void* wa = tb_wslice<WPREC>(sh.W, a.wStride, MODE == TB_SCAT ? its : a.rSlot);
                const void* wb = tb_wslice<WPREC>(sh.W, a.wStride, MODE == TB_SCAT ? its + 1 : a.rSlot0);
                if (WPREC == TBW_F32) {
                    kt_cp16(mySlot + (SO + j) * bd, (const float*)wa + ic, true);
                    kt_cp16(mySlot + (SO + 2 + j) * bd, (const float*)wb + ic, true);
                } else {
                    kt_cp8(mySlot + (SO + j) * bd, (const __nv_bfloat16*)wa + ic, true);
                    kt_cp8(mySlot + (SO + 2 + j) * bd, (const __nv_bfloat16*)wb + ic, true);
                }
            }
        }
    };
    // ---- shared set-up: zero rings, column damping table, sparse entries (descriptors, entries
    // and the taper are uploaded before the pass: read before the grid dependency wait)
    static_assert(RS % 4 == 0, "ring columns are whole float4s");
    const int nRing4 = kt_ringcols(MODE) * (RS / 4);
    for (int i = tid; i < nRing4; i += blockDim.x) kt_smem4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = tid; i < nDx; i += blockDim.x) {
        injFirst[i] = -1;
        recFirst[i] = -1;
        const int c = xs - 32 + i;
        float d = 0.f;
        if (c >= 0 && c < nxi) {
            const int dd = min(c, nxi - 1 - c);
            d = dd < g.minPad ? __ldg(a.taper + dd) : 1.f;
        }
        dxt[i] = d;
    }
    int nInj = 0, nRec = 0, recOff = 0;
    if (sh.entStart) {
        const int4 se = sh.entStart[strip * a.nChunks + chunk];
        const int n = min(se.w - se.x, a.maxEnt);
        for (int i = tid; i < n; i += blockDim.x) sEnt[i] = sh.ent[se.x + i];
        nInj = se.y - se.x;
        recOff = se.z - se.x;
        nRec = se.w - se.z;
    }
    // everything below reads what the previous launch of the stream wrote (state, partial sums,
    // stored slices and their scales, recordings)
    kt_grid_wait();
    if (a.relIter == 0) kt_grid_release();
    __syncthreads();
    // the rings are zeroed: the first input block's copies go out now, and land while the
    // per-launch tables below are built
    issue_input(0);
    kt_commit();
    // FP16 slice scales read by this launch (SCAT: its, its+1; ADJ: 0, its+1)
    // (SCATW reading a 16-bit stored field: its slices rSlot, rSlot0)
    const float scA = (WPREC == TBW_F16 && MODE == TB_SCAT)    ? sh.wscale[its]
                      : (WPREC == TBW_F16 && MODE == TB_SCATW) ? sh.wscale[a.rSlot]
                                                               : 1.f;
    const float scB = (WPREC == TBW_F16 && (MODE == TB_SCAT || MODE == TB_ADJ)) ? sh.wscale[its + 1]
                      : (WPREC == TBW_F16 && MODE == TB_SCATW)                 ? sh.wscale[a.rSlot0]
                                                                               : 1.f;
    const float sc0 = (WPREC == TBW_F16 && MODE == TB_ADJ) ? sh.wscale[0] : 1.f;
    // Injected values of this interval, one per entry and fine step, read once here
    // instead of inside the level loop (adjoint: the v2 factor is applied at use).
    if (!tb_scatlike(MODE)) {
        for (int i = tid; i < nInj * T; i += blockDim.x) {
            const int e = i / T, t = i - e * T + 1;
            const float* tr = pInj + (long long)sEnt[e].dev * injLd;
            float v;
            if (MODE == TB_ADJ || MODE == TB_ADJR) {
                const int it2 = sub - t;
                v = tr[its] * a.h[it2 + 1] + tr[its + 1] * a.h[H + it2 + 1];
            } else {
                v = tr[its * sub + t - 1];
            }
            sInjV[i] = v;
        }
    }
    // column -> first entry (entries are sorted by column; inside [xs - 32, xs - 32 + nDx))
    for (int e = tid; e < nInj; e += blockDim.x)
        if (e == 0 || sEnt[e - 1].col != sEnt[e].col) injFirst[sEnt[e].col - xs + 32] = e;
    for (int e = tid; e < nRec; e += blockDim.x)
        if (e == 0 || sEnt[recOff + e - 1].col != sEnt[recOff + e].col) recFirst[sEnt[recOff + e].col - xs + 32] = e;
    __syncthreads();
    // does any injection / recording point fall in this thread's row quad?
    bool qInj = false, qRec = false;
    for (int e = 0; e < nInj; e++) qInj |= (unsigned)(sEnt[e].row - zq) < 4u;
    for (int e = 0; e < nRec; e++) qRec |= (unsigned)(sEnt[recOff + e].row - zq) < 4u;

    // FP16 source pass: slice its is stored directly with the speculative scale of slice its-1's
    // max when that max allows it (the same decision in every CTA), else staged in FP32
    const bool f16Spec = WPREC == TBW_F16 && MODE == TB_SRC && kt_f16_spec_slice(sh.wmax, its, g.nts, a.f16spec);
    const float f16Sc = f16Spec ? kt_f16_spec_scale(sh.wmax[its - 1]) : 1.f;
    if (WPREC == TBW_F16 && MODE == TB_SRC && its > 0 && !kt_f16_spec_slice(sh.wmax, its - 1, g.nts, a.f16spec)) {
        // slice its-1 was staged and is complete (previous launch): quantize this CTA's output
        // region of it with its exact max
        kt_f16_quantize(sh, a.wStride, ip, its - 1, z0, min(z0 + a.HZ, nzi), x0, x1, tid, blockDim.x);
        __syncthreads();  // the region's staging slots are rewritten below (slice its+1 at the end)
    }
    kt_wait<0>();
    __syncthreads();
    // FP16 source pass: max |W| of this thread's points of slice its (and its+1 at the end),
    // folded into the slice maxima once per warp after the last iteration
    float wmaxA = 0.f, wmaxB = 0.f;

    for (int k = 0; k < a.iters; k++) {
        const int B = xs + KT_BX * k;
        if (k > 0 && k == a.relIter) kt_grid_release();
        // Output operands of this iteration's level-T columns, copied asynchronously into
        // this thread's staging slots (read at the output stage).
        if (MODE == TB_SRC || MODE == TB_ADJ || MODE == TB_ADJR) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int c = B - 5 * T + 2 * cp + j;
                if (zOut && c >= x0 && c < x1) {
                    const long long idx = (long long)c * ip + zq;
                    kt_cp16(mySlot + (SO + j) * bd, pPart + idx, true);
                    if (MODE == TB_ADJ) {
                        const void* w = tb_wslice<WPREC>(sh.W, a.wStride, its + 1);
                        if (WPREC == TBW_F32) kt_cp16(mySlot + (SO + 2 + j) * bd, (const float*)w + idx, true);
                        else kt_cp8(mySlot + (SO + 2 + j) * bd, (const __nv_bfloat16*)w + idx, true);
                        if (a.imgF32) {
                            kt_cp16(mySlot + (SO + 4 + 2 * j) * bd, pImgF + idx, true);
                        } else {
                            kt_cp16(mySlot + (SO + 4 + 2 * j) * bd, pImg + idx, true);
                            kt_cp16(mySlot + (SO + 5 + 2 * j) * bd, pImg + idx + 2, true);
                        }
                    }
                }
            }
        }
        kt_commit();

        float lvT[2][T + 1][4];  // levels 1..T at the output columns (T-1 from the rings)
#pragma unroll
        for (int t = 1; t <= T; t++) {
            const int c0 = B - 5 * t + 2 * cp;
            // level t is valid on columns >= xs + 5t and needed up to x1 - 1 + 5(T - t)
            const bool need = act && q >= (5 * t) / 4 && q < NQ - (5 * t) / 4 &&
                              c0 + 1 >= xs + 5 * t && c0 <= x1 - 1 + 5 * (T - t);
            float S[2][4];
            if (need) {
                float4 zq4[2][5];
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int d = 0; d < 5; d++) zq4[j][d] = kt_ld4(col(t - 1, c0 + j) + 4 * (d - 2));
                float4 xm[5], xp[5];  // columns c0-5..c0-1 and c0+2..c0+6
#pragma unroll
                for (int d = 0; d < 5; d++) {
                    xm[d] = kt_ld4(col(t - 1, c0 - 5 + d));
                    xp[d] = kt_ld4(col(t - 1, c0 + 2 + d));
                }
                float4 ol[2];
                if (t == 1) {
                    ol[0] = mySlot[0];
                    ol[1] = mySlot[bd];
                } else {
                    ol[0] = kt_ld4(col(t - 2, c0));
                    ol[1] = kt_ld4(col(t - 2, c0 + 1));
                }
                // free surface: forward modes see row 0 zeroed and rows above it mirrored (also
                // row 0 of the old level); adjoint modes are corrected below
                const bool fsTop = FS && (zq == 0 || zq == 4);  // quads of rows 0..3 and 4..7
                if (!kt_adj(MODE) && fsTop) {
#pragma unroll
                    for (int j = 0; j < 2; j++) kt_fs_window(zq4[j], zq);
                    if (zq == 0) {
#pragma unroll
                        for (int d = 0; d < 5; d++) {
                            xm[d].x = 0.f;
                            xp[d].x = 0.f;
                        }
                        ol[0].x = 0.f;
                        ol[1].x = 0.f;
                    }
                }
                float4 vq[2];
                float Dx[2];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int c = c0 + j;
                    // level 1 (large-strip variant): prefetched with the input; otherwise read
                    // from L1, where the lines of the previous levels' reads still are
                    vq[j] = (V2S && t == 1) ? mySlot[(2 + j) * bd]
                                     : __ldg(reinterpret_cast<const float4*>(v2p + (long long)min(max(c, 0), nxi - 1) * ip + zv));
                    Dx[j] = dxt[c - xs + 32];
                }
                float Dm[2][4];
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int i = 0; i < 4; i++) Dm[j][i] = fminf(Dz[i], Dx[j]);
                float4 sa[2], sb[2];
                if (tb_scatlike(MODE)) {
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        if (t == 1) {
                            // imagingFwdGpu (F/src/kernelsGpu.cu:309-316): dm * W, kept for levels 2..T
                            // (SCATX, and SCATW / ADJX without dm: the sources are staged as they are)
                            const float4 wa = kt_wfrom<WPREC>(mySlot[(SO + j) * bd], scA);
                            const float4 wb = kt_wfrom<WPREC>(mySlot[(SO + 2 + j) * bd], scB);
                            if (MODE == TB_SCATX || (tb_dense_out(MODE) && dmp == nullptr)) {
                                sa[j] = wa;
                                sb[j] = wb;
                            } else {
                                const long long idx = (long long)min(max(c0 + j, 0), nxi - 1) * ip + zv;
                                const float4 dmv = __ldg(reinterpret_cast<const float4*>(dmp + idx));
                                sa[j] = make_float4(dmv.x * wa.x, dmv.y * wa.y, dmv.z * wa.z, dmv.w * wa.w);
                                sb[j] = make_float4(dmv.x * wb.x, dmv.y * wb.y, dmv.z * wb.z, dmv.w * wb.w);
                            }
                            const float va[4] = {sa[j].x, sa[j].y, sa[j].z, sa[j].w};
                            const float vb[4] = {sb[j].x, sb[j].y, sb[j].z, sb[j].w};
                            kt_st4(ssCol(0, c0 + j), va);
                            kt_st4(ssCol(1, c0 + j), vb);
                        } else {
                            sa[j] = kt_ld4(ssCol(0, c0 + j));
                            sb[j] = kt_ld4(ssCol(1, c0 + j));
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    // x-neighbour columns of column c0+j: offsets -5..5 map to xm / xp / the other column
                    float4 xn[11];
#pragma unroll
                    for (int d = -5; d <= 5; d++) {
                        const int o = j + d;  // offset from c0
                        xn[d + 5] = o < 0 ? xm[o + 5] : (o == 0 ? zq4[0][2] : (o == 1 ? zq4[1][2] : xp[o - 2]));
                    }
                    // Two rows per paired FP32 instruction (f32x2): rows (2P, 2P+1) of the quad.
                    // z-neighbour pairs at even offsets are register pairs of the loaded quads;
                    // odd offsets pair rows of two quads (kt_pair builds them).
#pragma unroll
                    for (int P = 0; P < 2; P++) {
                        const int a0 = 2 * P;
                        const float2 ctr = kt_pair(zq4[j], a0);
                        float2 lz = __fmul2_rn(zc2[0], ctr);
#pragma unroll
                        for (int kk = 1; kk <= 5; kk++)
                            lz = __ffma2_rn(zc2[kk], __fadd2_rn(kt_pair(zq4[j], a0 + kk), kt_pair(zq4[j], a0 - kk)), lz);
                        if (kt_adj(MODE) && fsTop) {
                            // stepAdjFsGpu (F/src/kernelsGpu.cu:613-740), U-form: rows zi = 1..4 drop
                            // the mirror terms, lz(zi) -= sum_{k=zi+1..5} zc[k] U(k - zi)
                            if (zq == 0) {
#pragma unroll
                                for (int h = 0; h < 2; h++) {
                                    const int zi = a0 + h;  // window index of row r: r + 8
                                    if (zi >= 1 && zi <= 4) {
                                        float c = h ? lz.y : lz.x;
#pragma unroll
                                        for (int k = zi + 1; k <= 5; k++) c = c - a.c.zc[k] * kt_win(zq4[j], k - zi + 8);
                                        if (h) lz.y = c;
                                        else lz.x = c;
                                    }
                                }
                            } else if (P == 0) {  // zq == 4: row 4 (index 8), k = 5 reads row 1 (index 5)
                                lz.x = lz.x - a.c.zc[5] * kt_win(zq4[j], 5);
                            }
                        }
                        float2 lx = __fmul2_rn(xc2[0], ctr);
#pragma unroll
                        for (int kk = 1; kk <= 5; kk++)
                            lx = __ffma2_rn(xc2[kk], __fadd2_rn(kt_half(xn[5 + kk], P), kt_half(xn[5 - kk], P)), lx);
                        float2 n = __ffma2_rn(kt_half(vq[j], P), __fadd2_rn(lz, lx), ctr);
                        n = __fadd2_rn(n, ctr);
                        n = __ffma2_rn(make_float2(-Dm[j][a0], -Dm[j][a0 + 1]), kt_half(ol[j], P), n);
                        // free surface, adjoint modes: the top row keeps the old level (D o)
                        if (kt_adj(MODE) && fsTop && zq == 0 && P == 0) n.x = Dm[j][0] * ol[j].x;
                        if (tb_scatlike(MODE)) {
                            // injectSecondarySource (F/src/kernelsGpu.cu:102-107): forward fine step it2 = t
                            // weighs ss(its), ss(its+1) by h[it2-1], h[H+it2-1]; adjoint step it2 = T-t by
                            // h[it2+1], h[H+it2+1]
                            const int hi = MODE == TB_ADJX ? T - t + 1 : t - 1;
                            n = __fadd2_rn(n, __ffma2_rn(kt_half(sb[j], P), make_float2(a.h[H + hi], a.h[H + hi]),
                                                         __fmul2_rn(kt_half(sa[j], P), make_float2(a.h[hi], a.h[hi]))));
                        }
                        S[j][a0] = n.x;  // damped below, after injection
                        S[j][a0 + 1] = n.y;
                    }
                }
                // sparse injection into this micro-tile (entries sorted by column)
                if (!tb_scatlike(MODE) && qInj) {
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        for (int e = injFirst[c0 + j - xs + 32]; e >= 0 && e < nInj && sEnt[e].col == c0 + j; e++) {
                            const int rr = sEnt[e].row - zq;
                            if (rr >= 0 && rr < 4) {
                                float v = sInjV[e * T + t - 1];
                                if (MODE == TB_ADJ || MODE == TB_ADJR) v = kt_el(vq[j], rr) * v;
#pragma unroll
                                for (int i = 0; i < 4; i++)
                                    if (i == rr) S[j][i] = S[j][i] + v;
                            }
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int i = 0; i < 4; i++) S[j][i] = S[j][i] * Dm[j][i];
                if (t < T) {
#pragma unroll
                    for (int j = 0; j < 2; j++) kt_st4(col(t, c0 + j), S[j]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int i = 0; i < 4; i++) S[j][i] = 0.f;
            }
            if (t == 1) {
                // level-1 operands of this iteration are consumed: stage the next input
                issue_input(k + 1);
                kt_commit();
            }
            if (t == T) {
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int i = 0; i < 4; i++) lvT[j][T][i] = S[j][i];
            } else {
                __syncthreads();  // level t complete before level t+1 (and the outputs) read it
            }
        }
        kt_wait<1>();  // this iteration's output operands (the input group may still be in flight)

        // ---- outputs at the level-T columns [B - 5T, B - 5T + 16)
        {
            const int c0 = B - 5 * T + 2 * cp;
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int c = c0 + j;
#pragma unroll
                for (int l = 1; l < T; l++) {
                    const float4 v = kt_ld4(col(l, c));
                    lvT[j][l][0] = v.x; lvT[j][l][1] = v.y; lvT[j][l][2] = v.z; lvT[j][l][3] = v.w;
                }
                if (!(zOut && c >= x0 && c < x1)) continue;
                const long long idx = (long long)c * ip + zq;
                kt_st4(pNcur + idx, lvT[j][T]);
                kt_st4(pNold + idx, lvT[j][T - 1]);
                if (MODE == TB_SRC) {
                    float wa[4], wb[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        wa[i] = kt_el(mySlot[(SO + j) * bd], i);
                        wb[i] = 0.f;
#pragma unroll
                        for (int l = 1; l <= T; l++) {
                            wa[i] += lvT[j][l][i] * a.h[l];
                            wb[i] += lvT[j][l][i] * a.h[H + l];
                        }
                    }
                    kt_st4(pPartOut + idx, wb);
                    if (WPREC == TBW_F16) {
                        // slice its: FP16 with the speculative scale, or FP32 into the staging
                        // buffer (the next launch or k_f16_finish quantizes it with the slice's
                        // exact max); slice its+1 at the end is always staged
                        float m = fmaxf(fmaxf(fabsf(wa[0]), fabsf(wa[1])), fmaxf(fabsf(wa[2]), fabsf(wa[3])));
                        if (f16Spec) {
                            *reinterpret_cast<uint2*>((unsigned short*)sh.W + (long long)its * a.wStride + idx) =
                                kt_f16_pack(make_float4(wa[0], wa[1], wa[2], wa[3]), f16Sc);
                            if (m >= 65504.f * f16Sc) atomicOr(sh.wover, 1u);  // FP16 overflow: redo exactly
                        } else {
                            kt_st4(sh.wstage + (long long)(its & 1) * a.wStride + idx, wa);
                        }
                        wmaxA = fmaxf(wmaxA, m);
                        if (its == g.nts - 2) {
                            kt_st4(sh.wstage + (long long)((its + 1) & 1) * a.wStride + idx, wb);
                            m = fmaxf(fmaxf(fabsf(wb[0]), fabsf(wb[1])), fmaxf(fabsf(wb[2]), fabsf(wb[3])));
                            wmaxB = fmaxf(wmaxB, m);
                        }
                    } else {
                        const int sA = a.wRing ? its % a.wRing : its, sB = a.wRing ? (its + 1) % a.wRing : its + 1;
                        kt_wstore4<WPREC>(tb_wslice<WPREC>(sh.W, a.wStride, sA), idx, wa);
                        if (its == g.nts - 2) kt_wstore4<WPREC>(tb_wslice<WPREC>(sh.W, a.wStride, sB), idx, wb);
                    }
                } else if (MODE == TB_ADJ) {
                    float ra[4], rb[4];
                    const float4 oP = mySlot[(SO + j) * bd];
                    const float4 oW = kt_wfrom<WPREC>(mySlot[(SO + 2 + j) * bd], scB);
                    float4 w0 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (its == 0) w0 = kt_wload4<WPREC>(tb_wslice<WPREC>(sh.W, a.wStride, 0), idx, sc0);
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        ra[i] = 0.f;
                        rb[i] = kt_el(oP, i);
#pragma unroll
                        for (int l = 1; l <= T; l++) {
                            ra[i] += lvT[j][l][i] * a.h[sub - l];
                            rb[i] += lvT[j][l][i] * a.h[H + sub - l];
                        }
                    }
                    kt_st4(pPartOut + idx, ra);
                    if (a.imgF32) {
                        // imagingAdjGpu (F/src/kernelsGpu.cu:318-325): model += W * R in FP32,
                        // R(its+1) here and R(0) after it at its == 0, as the reference's loop
                        const float4 oI = mySlot[(SO + 4 + 2 * j) * bd];
                        float acc[4];
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            acc[i] = fmaf(kt_el(oW, i), rb[i], kt_el(oI, i));
                            if (its == 0) acc[i] = fmaf(kt_el(w0, i), ra[i], acc[i]);
                        }
                        kt_st4(pImgF + idx, acc);
                    } else {
                        const double2* oI = reinterpret_cast<const double2*>(&mySlot[(SO + 4 + 2 * j) * bd]);
                        const double2* oI2 = reinterpret_cast<const double2*>(&mySlot[(SO + 5 + 2 * j) * bd]);
                        const double oImg[4] = {oI->x, oI->y, oI2->x, oI2->y};
                        double acc[4];
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            acc[i] = oImg[i] + (double)(kt_el(oW, i) * rb[i]);
                            if (its == 0) acc[i] += (double)(kt_el(w0, i) * ra[i]);
                        }
                        *reinterpret_cast<double2*>(pImg + idx) = make_double2(acc[0], acc[1]);
                        *reinterpret_cast<double2*>(pImg + idx + 2) = make_double2(acc[2], acc[3]);
                    }
                } else if (MODE == TB_SCATW) {
                    // interpFineToCoarseSlice on the scattered field (F/src/kernelsGpu.cu:166-182); the
                    // partial sum is read directly (staging slots 4-7 hold the sources)
                    const float4 oP = __ldg(reinterpret_cast<const float4*>(pPart + idx));
                    float wa[4], wb[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        wa[i] = kt_el(oP, i);
                        wb[i] = 0.f;
#pragma unroll
                        for (int l = 1; l <= T; l++) {
                            wa[i] += lvT[j][l][i] * a.h[l];
                            wb[i] += lvT[j][l][i] * a.h[H + l];
                        }
                    }
                    kt_st4(pPartOut + idx, wb);
                    kt_st4(sh.rcoarse + (long long)a.oA * a.wStride + idx, wa);                          // its
                    if (its == g.nts - 2) kt_st4(sh.rcoarse + (long long)a.oB * a.wStride + idx, wb);   // its+1
                } else if (MODE == TB_ADJR || MODE == TB_ADJX) {
                    float ra[4], rb[4];
                    const float4 oP = MODE == TB_ADJX ? __ldg(reinterpret_cast<const float4*>(pPart + idx))
                                                      : mySlot[(SO + j) * bd];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        ra[i] = 0.f;
                        rb[i] = kt_el(oP, i);
#pragma unroll
                        for (int l = 1; l <= T; l++) {
                            ra[i] += lvT[j][l][i] * a.h[sub - l];
                            rb[i] += lvT[j][l][i] * a.h[H + sub - l];
                        }
                    }
                    kt_st4(pPartOut + idx, ra);
                    const int sB = MODE == TB_ADJX ? a.oB : a.rSlot, sA = MODE == TB_ADJX ? a.oA : a.rSlot0;
                    kt_st4(sh.rcoarse + (long long)sB * a.wStride + idx, rb);                  // R(its+1)
                    if (its == 0) kt_st4(sh.rcoarse + (long long)sA * a.wStride + idx, ra);  // R(0)
                } else if (qRec) {
                    for (int e = recFirst[c - xs + 32]; e >= 0 && e < nRec && sEnt[recOff + e].col == c; e++) {
                        const int rr = sEnt[recOff + e].row - zq;
                        if (rr >= 0 && rr < 4) {
                            float ra = 0.f, rb = 0.f;
#pragma unroll
                            for (int l = 1; l <= T; l++) {
#pragma unroll
                                for (int i = 0; i < 4; i++) {
                                    if (i == rr) {
                                        ra += lvT[j][l][i] * a.h[l];
                                        rb += lvT[j][l][i] * a.h[H + l];
                                    }
                                }
                            }
                            // one thread owns each receiver: the atomics are plain read-free adds
                            float* tr = pRec + (long long)sEnt[recOff + e].dev * recLd;
                            atomicAdd(tr + its, ra);
                            atomicAdd(tr + its + 1, rb);
                        }
                    }
                }
            }
        }
        kt_wait<0>();     // the next input block and level-1 operands have landed
        __syncthreads();  // ... for every thread; outputs done before level 1 reuses ring slots
    }
    if (WPREC == TBW_F16 && MODE == TB_SRC) {
        // non-negative floats order like their bit patterns: one warp max, one atomic per warp
        const unsigned ma = __reduce_max_sync(0xffffffffu, __float_as_uint(wmaxA));
        const unsigned mb = __reduce_max_sync(0xffffffffu, __float_as_uint(wmaxB));
        if ((tid & 31) == 0) {
            if (ma) atomicMax(sh.wmax + its, ma);
            if (mb) atomicMax(sh.wmax + its + 1, mb);
        }
    }
}

}  // namespace aio
