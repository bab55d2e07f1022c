// Device kernels of the B200 acoustic-isotropic engine.
//
// One fused kernel advances every shot of a batch by one fine time step
// (gridDim.z = shot): 10th-order stencil, damping of both time levels, sparse
// source/data injection, dense secondary-source injection, sparse receiver /
// source recording and fine->coarse accumulation all happen in the same pass
// over the grid. The reference runs each of these as a separate launch
// (F/src/kernelsGpu.cu:88-239,513-610) per step and per shot.
//
// Damping of the current level. The reference damps both p_new and p_cur after
// every step (dampCosineEdge, F/src/kernelsGpu.cu:202-219); the damped p_cur is
// only ever used again point-wise as next step's p_old. The stepper therefore
// stores each level once (damped once) and applies the second damping factor
// when it reads p_old, which produces the same values with one store per point.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "aio_common.cuh"
#include "aio_tb.cuh"

namespace aio {

__device__ __forceinline__ float v2_scaled(float v, const float* __restrict__ v2, const Geom& g, int z, int x) {
    // v is zero outside the interior (FAT ring / padding never written).
    if (z >= 0 && z < g.nzi && x >= 0 && x < g.nxi) v *= __ldg(v2 + (long long)x * g.ip + z);
    return v;
}

// ADJ=false: n = v2*L(c) + 2c - D*o    (stepFwdGpu,  F/src/kernelsGpu.cu:513-552)
// ADJ=true : n = L(v2*c) + 2c - D*o    (stepAdjGpu,  F/src/kernelsGpu.cu:574-610)
// then      S = D * (n + injection), written over o.
// Free surface (a.fs): forward steps see the current level with its top interior row zeroed
// and the rows above it mirrored with opposite sign (setFsConditionFwdGpu, :555-567, which
// the reference applies to the slice in memory before every step, so the old level's top row
// is zero too); adjoint steps leave the top row at the old value and drop the mirror terms
// from rows 1-4 (stepAdjFsGpu, :613-740); the taper ignores the top edge (dampCosineEdgeFs).
// INJ: 0 none, 1 sparse traces (injectSource / interpInjectData, :88-99),
//      2 dense secondary source ssA*hA + ssB*hB (injectSecondarySource, :102-107).
// REC: sparse recording of S (recordInterpData / recordSource, :113-127).
// ACC: accA += S*hA, accB += S*hB (interpWavefield / extractInterpAdjointWavefield /
//      interpFineToCoarseSlice, :132-182).
template <bool ADJ, int INJ, bool REC, bool ACC>
__global__ void __launch_bounds__(TZ* TY) k_step(const StepArgs a) {
    __shared__ float s[TX + 2 * FAT][TZ + 2 * FAT];
    const Geom& g = a.g;
    // Descriptor fields are read once into registers: stores below could
    // otherwise alias the descriptor and force reloads.
    const ShotDesc* sdp = a.shots + blockIdx.z;
    float* const p0 = sdp->p[0];
    float* const p1 = sdp->p[1];
    const SparseList injL = sdp->inj, recL = sdp->rec;
    const float* __restrict__ injSig = sdp->injSig;
    float* __restrict__ recSig = sdp->recSig;
    const int injLd = sdp->injLd, recLd = sdp->recLd;
    float* const ssBase = sdp->ss;
    float* const accBase = sdp->acc;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX;
    const float* __restrict__ cur = a.parity ? p1 : p0;
    float* __restrict__ old = a.parity ? p0 : p1;

    // Stage the current level (times v^2 dtw^2 for the adjoint) with its halo.
    const bool fsFwd = !ADJ && a.fs && z0 == 0;
    for (int r = ty; r < TX + 2 * FAT; r += TY) {
        const int x = x0 - FAT + r;
        const float* col = cur + (long long)(x + FAT) * g.hp + ZOFF;
        float v = col[z0 + lane];
        if (ADJ) v = v2_scaled(v, a.v2, g, z0 + lane, x);
        if (fsFwd && lane == 0) v = 0.f;
        s[r][FAT + lane] = v;
        if (lane < 2 * FAT) {
            const int zz = lane < FAT ? z0 - FAT + lane : z0 + TZ + (lane - FAT);
            float hv = col[zz];
            if (ADJ) hv = v2_scaled(hv, a.v2, g, zz, x);
            if (fsFwd && zz < 0) hv = -col[-zz];
            s[r][lane < FAT ? lane : TZ + lane] = hv;
        }
    }

    const int zi = z0 + lane;
    const int xb = x0 + ty * PX;
    const float* __restrict__ ssA = (INJ == 2) ? ssBase + a.ssOffA : nullptr;
    const float* __restrict__ ssB = (INJ == 2) ? ssBase + a.ssOffB : nullptr;
    float* __restrict__ accA = ACC ? accBase + a.accOffA : nullptr;
    float* __restrict__ accB = ACC ? accBase + a.accOffB : nullptr;

    // Point operands are loaded before the barrier so that their latency overlaps
    // the tile load (each point is read and written by this thread only).
    float ov[PX], pv[PX], sa[PX], sb[PX], aa[PX], ab[PX];
#pragma unroll
    for (int j = 0; j < PX; j++) {
        const int xi = xb + j;
        ov[j] = pv[j] = sa[j] = sb[j] = aa[j] = ab[j] = 0.f;
        if (zi < g.nzi && xi < g.nxi) {
            const long long hidx = (long long)(xi + FAT) * g.hp + ZOFF + zi;
            const long long iidx = (long long)xi * g.ip + zi;
            ov[j] = (fsFwd && zi == 0) ? 0.f : old[hidx];
            pv[j] = ADJ ? cur[hidx] : __ldg(a.v2 + iidx);
            if (INJ == 2) {
                sa[j] = ssA[iidx];
                sb[j] = ssB[iidx];
            }
            if (ACC) {
                aa[j] = accA[iidx];
                ab[j] = accB[iidx];
            }
        }
    }
    __syncthreads();
    float inj[PX];
#pragma unroll
    for (int j = 0; j < PX; j++) inj[j] = 0.f;

    const int tile = blockIdx.y * gridDim.x + blockIdx.x;
    if (INJ == 1 && injL.tileStart) {
        const int b = injL.tileStart[tile], e = injL.tileStart[tile + 1];
        for (int k = b; k < e; k++) {
            const int2 en = injL.ent[k];
            const int lz = en.x & (TZ - 1), lx = en.x / TZ;
            if (lz == lane && (lx / PX) == ty) {
                const float* tr = injSig + (long long)en.y * injLd;
                float v = a.injTB >= 0 ? tr[a.injTA] * a.injCA + tr[a.injTB] * a.injCB : tr[a.injTA];
#pragma unroll
                for (int j = 0; j < PX; j++)
                    if (j == (lx % PX)) inj[j] += v;
            }
        }
    }

    float w[PX + 2 * FAT];
#pragma unroll
    for (int k = 0; k < PX + 2 * FAT; k++) w[k] = s[ty * PX + k][FAT + lane];

    const int dzd = a.fs ? g.nzi - 1 - zi : min(zi, g.nzi - 1 - zi);
    float S[PX];
#pragma unroll
    for (int j = 0; j < PX; j++) {
        const int xi = xb + j;
        const float* row = s[FAT + ty * PX + j];
        const float c = w[FAT + j];
        float lap = a.c.zc[0] * c + a.c.zc[1] * (row[FAT + lane - 1] + row[FAT + lane + 1]) +
                    a.c.zc[2] * (row[FAT + lane - 2] + row[FAT + lane + 2]) +
                    a.c.zc[3] * (row[FAT + lane - 3] + row[FAT + lane + 3]) +
                    a.c.zc[4] * (row[FAT + lane - 4] + row[FAT + lane + 4]) +
                    a.c.zc[5] * (row[FAT + lane - 5] + row[FAT + lane + 5]);
        if (ADJ && a.fs && zi >= 1 && zi < FAT) {
            // rows 1-4: minus zc[k] * (row k - zi) for k = zi+1 .. 5
            for (int k = zi + 1; k <= 5; k++) lap = lap - a.c.zc[k] * row[FAT + lane + k - 2 * zi];
        }
        lap = lap + a.c.xc[0] * c +
                          a.c.xc[1] * (w[FAT + j + 1] + w[FAT + j - 1]) +
                          a.c.xc[2] * (w[FAT + j + 2] + w[FAT + j - 2]) +
                          a.c.xc[3] * (w[FAT + j + 3] + w[FAT + j - 3]) +
                          a.c.xc[4] * (w[FAT + j + 4] + w[FAT + j - 4]) +
                          a.c.xc[5] * (w[FAT + j + 5] + w[FAT + j - 5]);
        S[j] = 0.f;
        if (zi < g.nzi && xi < g.nxi) {
            const long long hidx = (long long)(xi + FAT) * g.hp + ZOFF + zi;
            const long long iidx = (long long)xi * g.ip + zi;
            const int d = min(dzd, min(xi, g.nxi - 1 - xi));
            const float D = d < g.minPad ? __ldg(a.taper + d) : 1.f;
            const float o = D * ov[j];
            float n;
            if (ADJ) {
                const float cr = pv[j];
                n = (a.fs && zi == 0) ? o : lap + cr + cr - o;
            } else {
                n = pv[j] * lap + c + c - o;
            }
            if (INJ == 1) n = n + inj[j];
            if (INJ == 2) n = n + (sa[j] * a.hInjA + sb[j] * a.hInjB);
            const float sv = n * D;
            S[j] = sv;
            old[hidx] = sv;
            if (ACC) {
                accA[iidx] = aa[j] + sv * a.hAccA;
                accB[iidx] = ab[j] + sv * a.hAccB;
            }
        }
    }

    if (REC && recL.tileStart) {
        const int b = recL.tileStart[tile], e = recL.tileStart[tile + 1];
        for (int k = b; k < e; k++) {
            const int2 en = recL.ent[k];
            const int lz = en.x & (TZ - 1), lx = en.x / TZ;
            if (lz == lane && (lx / PX) == ty) {
                float v = 0.f;
#pragma unroll
                for (int j = 0; j < PX; j++)
                    if (j == (lx % PX)) v = S[j];
                float* tr = recSig + (long long)en.y * recLd;
                tr[a.recTA] += v * a.recCA;
                if (a.recTB >= 0) tr[a.recTB] += v * a.recCB;
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Coarse-time kernels on interior slices. blockIdx.y = shot; `*St` are per-shot
// strides in floats (0 for arrays shared by every shot of the batch). Slices
// are swept whole (padding lanes are zero in every operand).
// ----------------------------------------------------------------------------
#define AIO_GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// imagingFwdGpu (F/src/kernelsGpu.cu:309-316): ss = m * W.
__global__ void k_img_fwd(float* ss, long long ssSt, const float* m, long long mSt, const float* W, long long WSt,
                          long long n) {
    const int b = blockIdx.y;
    ss += b * ssSt; m += b * mSt; W += b * WSt;
    AIO_GRID_STRIDE(i, n) ss[i] = m[i] * W[i];
}

// imagingAdjGpu (F/src/kernelsGpu.cu:318-325): m += W * r; optionally r = 0 afterwards.
template <typename Acc>
__global__ void k_img_adj(Acc* m, long long mSt, float* r, long long rSt, const float* W, long long WSt, long long n,
                          int zeroR) {
    const int b = blockIdx.y;
    m += b * mSt; r += b * rSt; W += b * WSt;
    AIO_GRID_STRIDE(i, n) {
        const float rv = r[i];
        m[i] += (Acc)(W[i] * rv);
        if (zeroR) r[i] = 0.f;
    }
}

// imagingTimeFwdGpu (:337-350): ss += sum_e ext[e] * W[t - 2(e-h)].
__global__ void k_img_time_fwd(float* ss, long long ssSt, const float* ext, long long extSt, const float* W,
                               long long WSt, long long isz, int t, int e0, int e1, int hExt) {
    const int b = blockIdx.y;
    ss += b * ssSt; ext += b * extSt; W += b * WSt;
    AIO_GRID_STRIDE(i, isz) {
        float acc = ss[i];
        for (int e = e0; e < e1; e++) acc += ext[(long long)e * isz + i] * W[(long long)(t - 2 * (e - hExt)) * isz + i];
        ss[i] = acc;
    }
}

// imagingTimeTomoAdjGpu (:445-458): ss += sum_e ext[e] * R[t + 2(e-h)].
__global__ void k_img_time_tomo_adj(float* ss, long long ssSt, const float* ext, long long extSt, const float* R,
                                    long long RSt, long long isz, int t, int e0, int e1, int hExt) {
    const int b = blockIdx.y;
    ss += b * ssSt; ext += b * extSt; R += b * RSt;
    AIO_GRID_STRIDE(i, isz) {
        float acc = ss[i];
        for (int e = e0; e < e1; e++) acc += ext[(long long)e * isz + i] * R[(long long)(t + 2 * (e - hExt)) * isz + i];
        ss[i] = acc;
    }
}

// imagingTimeAdjGpu (:352-364): m[e] += r * W[t - 2(e-h)]; sign=-1 gives
// imagingWemvaTimeAdjGpu (:366-378): m[e] += r * W[t + 2(e-h)]. Optionally r = 0.
template <typename Acc>
__global__ void k_img_time_adj(Acc* m, long long mSt, float* r, long long rSt, const float* W, long long WSt,
                               long long isz, int t, int e0, int e1, int hExt, int sign, int zeroR) {
    const int b = blockIdx.y;
    m += b * mSt; r += b * rSt; W += b * WSt;
    AIO_GRID_STRIDE(i, isz) {
        const float rv = r[i];
        for (int e = e0; e < e1; e++)
            m[(long long)e * isz + i] += (Acc)(rv * W[(long long)(t - sign * 2 * (e - hExt)) * isz + i]);
        if (zeroR) r[i] = 0.f;
    }
}

// recordScaleWavefield (F/src/kernelsGpu.cu:145-153): W += r * rs * v2 (one coarse slice); with
// rs null, scaleSecondarySourceFd then recordWavefield (:269-276, :138-143): W += r * v2.
__global__ void k_record_scale(float* W, const float* r, const float* rs, const float* v2, long long isz) {
    if (rs) AIO_GRID_STRIDE(i, isz) W[i] += r[i] * rs[i] * v2[i];
    else AIO_GRID_STRIDE(i, isz) W[i] += r[i] * v2[i];
}

// ---- subsurface (horizontal) offsets, interior-slice layout (x*ip + z), x in [0, nxi) ----
// imagingOffsetFwdGpu + scaleSecondarySourceFd (F/src/kernelsGpu.cu:381-395, 269-276):
//   ss(x) = v2(x) * (ss(x) + sum_s m_{s+h}(x-s) W(x-2s)) over the offsets whose model point x-s
//   lies in [h, nxi-h), s ascending.
__global__ void k_img_offset_fwd(float* ss, long long ssSt, const float* m, long long mSt, const float* W,
                                 long long WSt, const float* v2, long long isz, int ip, int nxi, int hExt) {
    const int b = blockIdx.y;
    ss += b * ssSt; m += b * mSt; W += b * WSt;
    AIO_GRID_STRIDE(i, isz) {
        const int x = (int)(i / ip);
        const int e0 = max(-hExt, x + 1 + hExt - nxi), e1 = min(x - hExt, hExt) + 1;
        float acc = ss[i];
        for (int s = e0; s < e1; s++) acc += m[(long long)(s + hExt) * isz + i - (long long)s * ip] * W[i - 2LL * s * ip];
        ss[i] = acc * v2[i];
    }
}
// imagingOffsetTomoAdjGpu (:460-476): ss(x) += sum_s m_{s+h}(x+s) R(x+2s) v2(x+2s) over the offsets
// whose model point x+s lies in [h, nxi-h). With v2Out (U-form receiver wavefield, R = v2 R_ref
// already, v2Rec = nullptr): ss(x) = v2(x) * (ss(x) + sum_s m_{s+h}(x+s) R(x+2s)).
__global__ void k_img_offset_tomo_adj(float* ss, long long ssSt, const float* m, long long mSt, const float* R,
                                      long long RSt, const float* v2Rec, const float* v2Out, long long isz, int ip,
                                      int nxi, int hExt) {
    const int b = blockIdx.y;
    ss += b * ssSt; m += b * mSt; R += b * RSt;
    AIO_GRID_STRIDE(i, isz) {
        const int x = (int)(i / ip);
        const int e0 = max(-hExt, hExt - x), e1 = min(nxi - 1 - x - hExt, hExt) + 1;
        float acc = ss[i];
        for (int s = e0; s < e1; s++) {
            const long long j = i + 2LL * s * ip;
            const float r = v2Rec ? R[j] * v2Rec[j] : R[j];
            acc += m[(long long)(s + hExt) * isz + i + (long long)s * ip] * r;
        }
        ss[i] = v2Out ? acc * v2Out[i] : acc;
    }
}
// Subsurface-offset imaging of a block of coarse samples tlo..thi: imagingOffsetAdjGpu
// (F/src/kernelsGpu.cu:397-411, img_e(x) += A(x+s) B(x-s), s = e-h, x in [h, nxi-h)) applied at
// every sample of the block. R holds the block's ring samples (slice t - tlo, stride isz), F the
// full coarse field (slice t).
//   Born form (wemvaForm = 0): img_e(x) += sum_t (R_t(x+s) v2(x+s)) F_t(x-s) — the receiver
//     sample scaled by scaleSecondarySourceFd (:269-276) before imagingOffsetAdjGpu;
//   WEMVA form (1): img_e(x) += sum_t (R_t(x-s) F_t(x+s)) v2(x+s) — imagingOffsetWemvaScaleFwdGpu
//     (:429-443) with F the receiver wavefield and R the scattered samples.
// Each term is the reference's per-sample float product; the block's terms are summed in the
// accumulator type and added to the image once per block instead of once per sample. v2 may be
// null (factor 1: receiver samples in U-form, v2 * S, carry it already).
constexpr int OFF_K = 32;
template <typename Acc>
__global__ void k_img_offset_block(Acc* img, long long mSt, const float* R, long long RSt, const float* F,
                                   long long FSt, const float* v2, int isz, int ip, int nxi, int hExt, int nExt,
                                   int tlo, int thi, int wemvaForm) {
    const int b = blockIdx.y;
    img += b * mSt;
    R += b * RSt;
    F += b * FSt + (long long)tlo * isz;
    const int nk = min(thi - tlo + 1, OFF_K);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < isz; i += gridDim.x * blockDim.x) {
        const int x = i / ip;
        if (x < hExt || x >= nxi - hExt) continue;
        for (int e = 0; e < nExt; e++) {
            const int s = e - hExt;
            const int ja = i + s * ip, jb = i - s * ip;
            const float sa = v2 ? __ldg(v2 + ja) : 1.f;
            // all of the block's operands are loaded before the first product (the kernel is
            // bound by load latency otherwise)
            const int jr = wemvaForm ? jb : ja, jf = wemvaForm ? ja : jb;
            float rv[OFF_K], fv[OFF_K];
#pragma unroll
            for (int k = 0; k < OFF_K; k++) {
                rv[k] = k < nk ? __ldg(R + (long long)k * isz + jr) : 0.f;
                fv[k] = k < nk ? __ldg(F + (long long)k * isz + jf) : 0.f;
            }
            Acc acc = 0;
#pragma unroll
            for (int k = 0; k < OFF_K; k++) {
                if (k < nk) {
                    float v;
                    if (wemvaForm) {
                        v = rv[k] * fv[k];
                        v = v * sa;
                    } else {
                        const float a = rv[k] * sa;
                        v = a * fv[k];
                    }
                    acc += (Acc)v;
                }
            }
            img[(long long)e * isz + i] += acc;
        }
    }
}

// Time-lag imaging of a block of at most LAG_K coarse samples (imagingTimeAdjGpu,
// F/src/kernelsGpu.cu:352-364, applied at every t of the block; sign = -1 gives
// imagingWemvaTimeAdjGpu, :366-378):
//   img[e] += sum_{t = tlo..thi} R(t) * W[t - sign 2(e-h)]   over 0 <= t - sign 2(e-h) < nts,
// the same (t, e) pairs as the reference's truncating-division lag bounds (nExt = 1, hExt = 0:
// the zero-lag imagingAdjGpu, :318-325). R(t) lives in a ring of rRing slices (slot t % rRing).
// Each thread owns one point: its R samples are held in registers and the W slices
// tlo-2h .. tlo+LAG_K-1+2h of the block in shared memory (own column only, no barrier; zero
// outside [0, nts), so every (t, e) term is formed without bounds tests and the terms outside
// the reference's bounds add exact zeros), so W is read once per block instead of once per lag,
// and the image once per block instead of once per sample. Global loads are issued in batches:
// the kernels are latency bound otherwise.
constexpr int LAG_K = 32;
constexpr int LAG_B = 8;
constexpr int LAG_NP = 128;  // threads per block (points), a compile-time shared-memory stride
__host__ __device__ constexpr int lag_window_len(int hExt) { return LAG_K + 4 * hExt; }
// Sample tau of a stored wavefield at element idx: FP32, BF16, or FP16 in units of the slice's
// scale sc[tau] (the stored source wavefield of aio_tb.cuh).
template <int WP>
__device__ __forceinline__ float lag_wsample(const void* __restrict__ W, long long idx, const float* __restrict__ sc,
                                             int tau) {
    if (WP == TBW_F32) return __ldg(reinterpret_cast<const float*>(W) + idx);
    const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(W) + idx);
    if (WP == TBW_BF16) return __bfloat162float(__ushort_as_bfloat16(u));
    return __half2float(__ushort_as_half(u)) * __ldg(sc + tau);
}
// W slices tlo-2h .. of point p into this thread's shared column, zero outside [0, nts). The
// column holds consecutive samples in pairs (one float2 per pair): every lag offset 2h - 2(e-h)
// is even, so sample pairs (k, k+1) of any lag are one aligned float2 and the inner products
// run on paired FP32 instructions. W is stored in FP32, BF16 or FP16 with per-slice scales sc.
//
// 16-bit samples: the two lanes of a point pair (p even, p + 1; slices are a whole number of
// warps, isz % 32 == 0, so both lanes always run) share 32-bit loads. For each sample pair
// (k, k+1) the even lane loads the pair's word of slice k, the odd lane the word of slice k+1,
// and one shuffle hands each lane the other word: every lane then holds its own point's two
// samples. Half the load instructions of one 16-bit load per sample, four bytes per lane.
template <int WP>
__device__ __forceinline__ float lag_half(unsigned word, bool high) {
    const unsigned short u = (unsigned short)(high ? (word >> 16) : (word & 0xffffu));
    if (WP == TBW_BF16) return __bfloat162float(__ushort_as_bfloat16(u));
    return __half2float(__ushort_as_half(u));
}
template <int WP = TBW_F32>
__device__ __forceinline__ void lag_window(float2* W2, const void* __restrict__ W, const float* __restrict__ sc,
                                           long long isz, long long p, int tlo, int hExt, int nts) {
    const int n = lag_window_len(hExt), t0 = tlo - 2 * hExt;
    if constexpr (WP == TBW_F32) {
        for (int k0 = 0; k0 < n; k0 += 2 * LAG_B) {
            float v[2 * LAG_B];
#pragma unroll
            for (int j = 0; j < 2 * LAG_B; j++) {
                const int tau = t0 + k0 + j;
                v[j] = (k0 + j < n && tau >= 0 && tau < nts) ? lag_wsample<WP>(W, (long long)tau * isz + p, sc, tau)
                                                             : 0.f;
            }
#pragma unroll
            for (int j = 0; j < 2 * LAG_B; j += 2)
                if (k0 + j < n) W2[((k0 + j) >> 1) * LAG_NP] = make_float2(v[j], v[j + 1]);
        }
    } else {
        const bool odd = (p & 1) != 0;
        const unsigned* __restrict__ W32 = reinterpret_cast<const unsigned*>(W);
        const long long iszw = isz >> 1, pw = p >> 1;
        for (int k0 = 0; k0 < n; k0 += 2 * LAG_B) {
            unsigned wv[LAG_B];
#pragma unroll
            for (int j = 0; j < LAG_B; j++) {
                const int k = k0 + 2 * j + (odd ? 1 : 0);  // the sample this lane loads
                const int tau = t0 + k;
                wv[j] = (k < n && tau >= 0 && tau < nts) ? __ldg(W32 + (long long)tau * iszw + pw) : 0u;
            }
#pragma unroll
            for (int j = 0; j < LAG_B; j++) {
                const unsigned other = __shfl_xor_sync(0xffffffffu, wv[j], 1);
                const int k = k0 + 2 * j;
                if (k < n) {
                    float va = lag_half<WP>(odd ? other : wv[j], odd);  // sample k of this point
                    float vb = lag_half<WP>(odd ? wv[j] : other, odd);  // sample k + 1
                    if (WP == TBW_F16) {
                        const int ta = t0 + k;
                        va *= (ta >= 0 && ta < nts) ? __ldg(sc + ta) : 0.f;
                        vb *= (ta + 1 >= 0 && ta + 1 < nts) ? __ldg(sc + ta + 1) : 0.f;
                    }
                    W2[(k >> 1) * LAG_NP] = make_float2(va, vb);
                }
            }
        }
    }
}
// W: stored wavefield of WSt elements per shot (FP32, or BF16 / FP16 with nts scales per shot
// in wsc when WP says so).
template <typename Acc, int WP = TBW_F32>
__global__ void __launch_bounds__(LAG_NP) k_img_lag_block(Acc* __restrict__ img, long long mSt, const float* __restrict__ R,
                                                          long long rSt, int rRing, const void* __restrict__ W,
                                                          long long WSt, long long isz, int tlo, int thi, int nts,
                                                          int hExt, int nExt, int sign,
                                                          const float* __restrict__ wsc = nullptr) {
    extern __shared__ float2 lag_smem2[];
    const int b = blockIdx.y, tid = threadIdx.x;
    const long long p = (long long)blockIdx.x * LAG_NP + tid;
    if (p >= isz) return;
    R += b * rSt;
    const void* Wb = reinterpret_cast<const char*>(W) + b * WSt * (WP == TBW_F32 ? 4 : 2);
    const float* scb = WP == TBW_F16 ? wsc + (long long)b * nts : nullptr;
    img += b * mSt;
    float2* W2 = lag_smem2 + tid;
    lag_window<WP>(W2, Wb, scb, isz, p, tlo, hExt, nts);
    float2 r2[LAG_K / 2];
    int slot = tlo % rRing;  // ring slot of sample tlo; the block's slots follow with one wrap at most
#pragma unroll
    for (int k = 0; k < LAG_K; k += 2) {
        const float ra = (tlo + k <= thi) ? __ldg(R + (long long)slot * isz + p) : 0.f;
        slot = slot + 1 == rRing ? 0 : slot + 1;
        const float rb = (tlo + k + 1 <= thi) ? __ldg(R + (long long)slot * isz + p) : 0.f;
        slot = slot + 1 == rRing ? 0 : slot + 1;
        r2[k >> 1] = make_float2(ra, rb);
    }
    for (int e0 = 0; e0 < nExt; e0 += LAG_B) {
        float acc[LAG_B];
#pragma unroll
        for (int j = 0; j < LAG_B; j++) {
            // W index of sample k at lag e: tlo + k - sign 2(e-h), window offset 2h - sign 2(e-h)
            const int e = min(e0 + j, nExt - 1);
            const float2* w = W2 + ((2 * hExt - sign * 2 * (e - hExt)) >> 1) * LAG_NP;
            float2 sum = make_float2(0.f, 0.f);  // even and odd samples of the block
#pragma unroll
            for (int kp = 0; kp < LAG_K / 2; kp++) sum = __ffma2_rn(r2[kp], w[kp * LAG_NP], sum);
            acc[j] = sum.x + sum.y;
        }
        Acc old[LAG_B];
#pragma unroll
        for (int j = 0; j < LAG_B; j++) old[j] = e0 + j < nExt ? img[(long long)(e0 + j) * isz + p] : (Acc)0;
#pragma unroll
        for (int j = 0; j < LAG_B; j++)
            if (e0 + j < nExt) img[(long long)(e0 + j) * isz + p] = old[j] + (Acc)acc[j];
    }
}

// Secondary sources of a block of coarse steps of the time-lag extended forward
// (imagingTimeFwdGpu, F/src/kernelsGpu.cu:337-350, at every t of the block; sign = -1 gives
// imagingTimeTomoAdjGpu, :445-458):
//   ss(t) = sum_e ext[e] * W[t - sign 2(e-h)]   over 0 <= t - sign 2(e-h) < nts,
// written to a ring of ring slices (slot t % ring). One thread per point; the W slices of
// the block live in shared memory (own column only, zero outside [0, nts)), so W is read once
// per block, and ext once per block (lags outer, the block's samples accumulated in registers,
// in lag order, two samples per paired instruction).
template <int WP = TBW_F32>
__global__ void __launch_bounds__(LAG_NP) k_ss_lag_block(float* __restrict__ ss, long long ssSt, int ring,
                                                         const float* __restrict__ ext, const void* __restrict__ W,
                                                         long long WSt, long long isz, int tlo, int thi, int nts,
                                                         int hExt, int nExt, int sign,
                                                         const float* __restrict__ wsc = nullptr) {
    extern __shared__ float2 lag_smem2[];
    const int b = blockIdx.y, tid = threadIdx.x;
    const long long p = (long long)blockIdx.x * LAG_NP + tid;
    if (p >= isz) return;
    ss += b * ssSt;
    const void* Wb = reinterpret_cast<const char*>(W) + b * WSt * (WP == TBW_F32 ? 4 : 2);
    const float* scb = WP == TBW_F16 ? wsc + (long long)b * nts : nullptr;
    float2* W2 = lag_smem2 + tid;
    lag_window<WP>(W2, Wb, scb, isz, p, tlo, hExt, nts);
    float2 acc[LAG_K / 2];
#pragma unroll
    for (int k = 0; k < LAG_K / 2; k++) acc[k] = make_float2(0.f, 0.f);
    for (int e0 = 0; e0 < nExt; e0 += LAG_B) {
        float x[LAG_B];
#pragma unroll
        for (int j = 0; j < LAG_B; j++) x[j] = e0 + j < nExt ? __ldg(ext + (long long)(e0 + j) * isz + p) : 0.f;
#pragma unroll
        for (int j = 0; j < LAG_B; j++) {
            if (e0 + j < nExt) {
                const int e = e0 + j;
                const float2* w = W2 + ((2 * hExt - sign * 2 * (e - hExt)) >> 1) * LAG_NP;
                const float2 xx = make_float2(x[j], x[j]);
#pragma unroll
                for (int kp = 0; kp < LAG_K / 2; kp++) acc[kp] = __ffma2_rn(xx, w[kp * LAG_NP], acc[kp]);
            }
        }
    }
    int slot = tlo % ring;  // ring slot of sample tlo; the block's slots follow with one wrap at most
#pragma unroll
    for (int k = 0; k < LAG_K; k += 2) {
        if (tlo + k <= thi) ss[(long long)slot * isz + p] = acc[k >> 1].x;
        slot = slot + 1 == ring ? 0 : slot + 1;
        if (tlo + k + 1 <= thi) ss[(long long)slot * isz + p] = acc[k >> 1].y;
        slot = slot + 1 == ring ? 0 : slot + 1;
    }
}

// Scalings (F/src/kernelsGpu.cu:246-252, 278-303). mode 0: m *= v2*rs;
// mode 1: m *= rs*v2 (extended); mode 2: m = -(m*v2) (sloth); on images of v2-weighted
// (adjoint U-form) wavefields: mode 3: m *= rs, mode 4: m = -m, mode 5: m *= (v2*rs) / v2
// (zero where v2 is zero: padding lanes).
__global__ void k_scale(float* m, long long mSt, int nSlices, const float* v2, const float* rs, long long isz,
                        int mode) {
    const int b = blockIdx.y;
    m += b * mSt;
    const long long n = (long long)nSlices * isz;
    AIO_GRID_STRIDE(k, n) {
        const long long i = k % isz;
        const float v = v2[i], r = rs[i];
        if (mode == 0) m[k] *= v * r;
        else if (mode == 1) m[k] *= r * v;
        else if (mode == 3) m[k] *= r;   // images of v2-weighted (adjoint U-form) wavefields
        else if (mode == 4) m[k] = -m[k];
        else if (mode == 5) m[k] = v != 0.f ? m[k] / v * (v * r) : 0.f;
        else m[k] = -(m[k] * v);
    }
}

// Coarse second time derivative in place along the slice stack, zero outside
// [0, nts): srcWfldSecondTimeDerivative (F/src/kernelsGpu.cu:188-197) applied at
// every coarse sample as computeTomoSrcWfldDt2 does (F/src/tomoExtShotsGpuFunctions.cu:1251-1361).
__global__ void k_dt2(float* W, long long WSt, long long isz, int nts, float cSide, float cCenter) {
    const int b = blockIdx.y;
    W += b * WSt;
    AIO_GRID_STRIDE(i, isz) {
        float prev = 0.f, c = W[i];
        for (int t = 0; t < nts; t++) {
            const float nx = (t + 1 < nts) ? W[(long long)(t + 1) * isz + i] : 0.f;
            W[(long long)t * isz + i] = cSide * (prev + nx) + cCenter * c;
            prev = c;
            c = nx;
        }
    }
}

// Sum of per-shot images into one output: out[i] (+)= sum_b in[b][i].
template <typename Acc>
__global__ void k_sum_shots(float* out, const Acc* in, long long inSt, int nShots, long long n, int add) {
    AIO_GRID_STRIDE(i, n) {
        Acc s = 0;
        for (int b = 0; b < nShots; b++) s += in[b * inSt + i];
        out[i] = add ? out[i] + (float)s : (float)s;
    }
}

// FP64 -> FP32 with scaling for per-shot images kept in FP64.
__global__ void k_scale_d(double* m, long long mSt, int nSlices, const float* v2, const float* rs, long long isz,
                          int mode) {
    const int b = blockIdx.y;
    m += b * mSt;
    const long long n = (long long)nSlices * isz;
    AIO_GRID_STRIDE(k, n) {
        const long long i = k % isz;
        const double v = v2[i], r = rs[i];
        if (mode == 0) m[k] *= (double)(float)(v * r);
        else if (mode == 1) m[k] *= (double)(float)(r * v);
        else if (mode == 3) m[k] *= r;   // images of v2-weighted (adjoint U-form) wavefields
        else if (mode == 4) m[k] = -m[k];  // sloth images of U-form wavefields
        else if (mode == 5) m[k] = v != 0.0 ? m[k] / v * (double)(float)(v * r) : 0.0;  // U-form, v2*rs scaling
        else m[k] = -(m[k] * v);
    }
}

}  // namespace aio
