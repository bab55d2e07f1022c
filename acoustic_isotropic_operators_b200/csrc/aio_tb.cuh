// Temporally blocked stepper: one launch advances every shot of a wave by one
// coarse interval (T = sub fine steps).
//
// Each CTA owns an interior z-strip of HZ output rows (plus 5*T halo rows on
// each side, recomputed) and an x-chunk of LX output columns, and marches along
// x. At iteration k it loads input column xin = xs + k and computes time level
// t (t = 1..T) at column c_t = xin - 5t - TBD (a wavefront; TBD iterations hide
// the input load latency). One thread owns one row:
//   * the x-stencil reads the thread's own register queue of level t-1
//     (the 11 columns c_t-5 .. c_t+5),
//   * the z-stencil reads a shared-memory ring holding recent level t-1 columns
//     (rows padded with zeros so no bounds tests are needed),
//   * v^2 dtw^2 comes from a shared ring filled from the input front,
//   * the older level needed by the leapfrog (p_old) is in the queue of level
//     t-2 (or, for t = 1, the input's previous level),
//   * per-interval products — the coarse wavefield sample, receiver data, the
//     imaging condition — are formed when level T leaves column c_T, from the
//     values of all T levels still held in the queues.
// The scheme per fine step is the reference's (F/src/kernelsGpu.cu:202-219,
// 513-552): S_t = D * (v2 * L(S_{t-1}) + 2 S_{t-1} - D * S_{t-2} + injection),
// with the second damping of p_cur applied when the level is used as p_old.
//
// Adjoint passes run the same recursion on U = v2 * S: from stepAdjGpu
// (F/src/kernelsGpu.cu:574-610), S_t = D * (L(v2 S_{t-1}) + 2 S_{t-1} -
// D S_{t-2} + inj); multiplying by v2 point-wise gives
// U_t = D * (v2 * L(U_{t-1}) + 2 U_{t-1} - D U_{t-2} + v2 * inj).
//
// State slices (p_cur, p_old) use the interior layout; points outside the
// interior are the zero FAT boundary and are never loaded or stored.
#pragma once
#include <cuda_bf16.h>

#include "aio_common.cuh"

namespace aio {

constexpr int TBQ = 16;        // register queue depth (unroll period)
constexpr int TBR = 8;         // level ring depth (columns)
constexpr int TBV = 32;        // v^2 ring depth (columns)
constexpr int TBD = 4;         // input prefetch distance (iterations)
constexpr int TBP = 4;         // output-operand prefetch distance (iterations)
constexpr int TB_MAXROWS = 192;  // threads (rows) per CTA
constexpr int TB_PAD = 8;        // zero rows above and below each ring column
constexpr int TB_RS = TB_MAXROWS + 2 * TB_PAD;  // ring column stride

enum TBMode { TB_SRC = 0, TB_NL = 1, TB_SCAT = 2, TB_ADJ = 3 };
enum TBWfld { TBW_F32 = 0, TBW_BF16 = 1 };

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
    double* img;          // ADJ: image accumulator
    int injLd, recLd;
};

struct TBArgs {
    Geom g;
    Coefs c;
    const float* v2;       // interior slice
    const float* taper;    // minPad entries
    const float* dm;       // SCAT: scaled model perturbation (interior slice, shared)
    const TBShot* shots;
    float h[2 * (SUB_MAX + 1)];
    int its;               // coarse interval
    int HZ, LX;            // strip rows / chunk columns
    int nStrips, nChunks;
    int iters;             // iterations per CTA (multiple of TBQ)
    int maxEnt;            // shared entry capacity
    long long wStride;     // elements per stored coarse slice (= isz)
};

template <int WPREC>
__device__ __forceinline__ float tb_wload(const void* W, int idx) {
    if (WPREC == TBW_F32) return __ldg((const float*)W + idx);
    return __bfloat162float(((const __nv_bfloat16*)W)[idx]);
}

template <int WPREC>
__device__ __forceinline__ void tb_wstore(void* W, int idx, float v) {
    if (WPREC == TBW_F32) ((float*)W)[idx] = v;
    else ((__nv_bfloat16*)W)[idx] = __float2bfloat16_rn(v);
}

template <int WPREC>
__device__ __forceinline__ void* tb_wslice(void* W, long long stride, int t) {
    return (char*)W + (long long)t * stride * (WPREC == TBW_F32 ? 4 : 2);
}

__host__ __device__ inline size_t tb_ring_floats(int T, int mode) {
    // level rings + v2 ring + (scattered pass) two secondary-source rings + damping table
    return ((size_t)T * TBR + TBV * (mode == TB_SCAT ? 3 : 1)) * TB_RS + TBV;
}
inline size_t tb_smem_bytes(int T, int mode, int maxEnt) {
    return tb_ring_floats(T, mode) * sizeof(float) + (size_t)maxEnt * sizeof(TBEnt);
}

template <int T, int MODE, int WPREC>
__global__ void __launch_bounds__(TB_MAXROWS, 2) k_interval(const TBArgs a) {
    extern __shared__ float4 tb_smem4[];
    float* ring = reinterpret_cast<float*>(tb_smem4);              // [T][TBR][TB_RS]
    float* vring = ring + T * TBR * TB_RS;                         // [TBV][TB_RS] v^2 dtw^2
    float* sLring = vring + TBV * TB_RS;                           // SCAT: [TBV][TB_RS] dm*W[its]
    float* sRring = sLring + (MODE == TB_SCAT ? TBV * TB_RS : 0);  // SCAT: [TBV][TB_RS] dm*W[its+1]
    float* dxr = sRring + (MODE == TB_SCAT ? TBV * TB_RS : 0);     // [TBV] column damping factor
    TBEnt* sEnt = reinterpret_cast<TBEnt*>(dxr + TBV);

    const Geom& g = a.g;
    // Descriptor fields are copied into registers once: global stores below could
    // otherwise alias the descriptor and force a reload after every store.
    const TBShot sh = a.shots[blockIdx.z];
    float* __restrict__ pNcur = sh.ncur;
    float* __restrict__ pNold = sh.nold;
    const float* __restrict__ pPart = sh.part;
    float* __restrict__ pPartOut = sh.partOut;
    double* __restrict__ pImg = sh.img;
    float* __restrict__ pRec = sh.recSig;
    const float* __restrict__ pInj = sh.injSig;
    const int injLd = sh.injLd, recLd = sh.recLd;
    const int strip = blockIdx.x, chunk = blockIdx.y;
    const int row = threadIdx.x;
    const int nrows = a.HZ + 10 * T;
    const int z0 = strip * a.HZ;
    const int z = z0 - 5 * T + row;
    const bool zin = row < nrows && z >= 0 && z < g.nzi;
    const bool zout = zin && z >= z0 && z < z0 + a.HZ;
    const int x0 = chunk * a.LX;
    const int x1 = min(x0 + a.LX, g.nxi);
    const int xs = x0 - 5 * T;
    const int ip = g.ip;
    const int nxi = g.nxi;
    const int H = g.H;
    const int sub = g.sub;
    const int its = a.its;
    const int minPad = g.minPad;

    int nInj = 0, nRec = 0, recOff = 0;
    if (sh.entStart) {
        const int4 se = sh.entStart[strip * a.nChunks + chunk];
        const int n = min(se.w - se.x, a.maxEnt);
        for (int i = threadIdx.x; i < n; i += blockDim.x) sEnt[i] = sh.ent[se.x + i];
        nInj = se.y - se.x;
        recOff = se.z - se.x;
        nRec = se.w - se.z;
    }
    const int nRing = (int)tb_ring_floats(T, MODE);
    for (int i = threadIdx.x; i < nRing; i += blockDim.x) ring[i] = 0.f;
    __syncthreads();

    const float* __restrict__ cur = sh.cur;
    const float* __restrict__ old = sh.old;
    const void* Wa = nullptr;
    const void* Wb = nullptr;
    if (MODE == TB_SCAT) {
        Wa = tb_wslice<WPREC>(sh.W, a.wStride, its);
        Wb = tb_wslice<WPREC>(sh.W, a.wStride, its + 1);
    } else if (MODE == TB_ADJ) {
        Wa = tb_wslice<WPREC>(sh.W, a.wStride, 0);
        Wb = tb_wslice<WPREC>(sh.W, a.wStride, its + 1);
    }
    void* Wo = (MODE == TB_SRC) ? tb_wslice<WPREC>(sh.W, a.wStride, its) : nullptr;
    const float* __restrict__ dmp = a.dm;
    const float* __restrict__ v2p = a.v2;

    float Q[T][TBQ];
    float Qold[TBQ];
    float Qv[8], Qdm[8], QWa[8], QWb[8];  // raw input loads, consumed TBD iterations later
    float Pp[8], Pw[8];                   // output operands prefetched TBP iterations ahead
    double Pi[8];
#pragma unroll
    for (int t = 0; t < T; t++)
#pragma unroll
        for (int i = 0; i < TBQ; i++) Q[t][i] = 0.f;
#pragma unroll
    for (int i = 0; i < TBQ; i++) Qold[i] = 0.f;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        Qv[i] = Qdm[i] = QWa[i] = QWb[i] = 0.f;
        Pp[i] = Pw[i] = 0.f;
        Pi[i] = 0.0;
    }

    // Damping D = taper[min(dist_z, dist_x)] = min(Dz, Dx) (the taper is monotone, <= 1);
    // zero outside the domain so out-of-range rows / columns stay at the zero boundary.
    float Dz = 0.f;
    if (zin) {
        const int dzd = min(z, g.nzi - 1 - z);
        Dz = dzd < minPad ? __ldg(a.taper + dzd) : 1.f;
    }
    int injPtr[T];
#pragma unroll
    for (int t = 0; t < T; t++) injPtr[t] = 0;
    int recPtr = 0;
    float* myRing = ring + TB_PAD + row;
    float* myV = vring + TB_PAD + row;
    float* mySL = sLring + TB_PAD + row;
    float* mySR = sRring + TB_PAD + row;

    for (int kb = 0; kb < a.iters; kb += TBQ) {
#pragma unroll
        for (int u = 0; u < TBQ; u++) {
            const int k = kb + u;
            // 1. input column xs+k: levels, v^2 and (scattered pass) the secondary sources;
            //    published to the shared rings TBD iterations later.
            {
                const int xin = xs + k;
                const bool xok = xin >= 0 && xin < nxi;
                float v0 = 0.f, vo = 0.f, vv = 0.f, dmv = 0.f, wa = 0.f, wb = 0.f;
                if (zin && xok) {
                    const int idx = xin * ip + z;
                    v0 = cur[idx];
                    vo = old[idx];
                    vv = __ldg(v2p + idx);
                    if (MODE == TB_SCAT) {
                        dmv = __ldg(dmp + idx);
                        wa = tb_wload<WPREC>(Wa, idx);
                        wb = tb_wload<WPREC>(Wb, idx);
                    }
                }
                Q[0][u] = v0;
                Qold[u] = vo;
                Qv[u & 7] = vv;
                const int sp = (k - TBD) & (TBV - 1);
                myRing[((u - TBD) & (TBR - 1)) * TB_RS] = Q[0][(u - TBD) & (TBQ - 1)];
                myV[sp * TB_RS] = Qv[(u - TBD) & 7];
                if (MODE == TB_SCAT) {
                    Qdm[u & 7] = dmv;
                    QWa[u & 7] = wa;
                    QWb[u & 7] = wb;
                    const float d0 = Qdm[(u - TBD) & 7];
                    mySL[sp * TB_RS] = d0 * QWa[(u - TBD) & 7];
                    mySR[sp * TB_RS] = d0 * QWb[(u - TBD) & 7];
                }
                // output operands for the output column of iteration k+TBP
                if (MODE == TB_SRC || MODE == TB_ADJ) {
                    const int cP = xs + k + TBP - 5 * T - TBD;
                    float pp = 0.f, pw = 0.f;
                    double pi = 0.0;
                    if (zout && cP >= x0 && cP < x1) {
                        const int idx = cP * ip + z;
                        pp = pPart[idx];
                        if (MODE == TB_ADJ) {
                            pw = tb_wload<WPREC>(Wb, idx);
                            pi = pImg[idx];
                        }
                    }
                    Pp[u & 7] = pp;
                    Pw[u & 7] = pw;
                    Pi[u & 7] = pi;
                }
                if (row == 0) {
                    float dx = 0.f;
                    if (xok) {
                        const int dd = min(xin, nxi - 1 - xin);
                        dx = dd < minPad ? __ldg(a.taper + dd) : 1.f;
                    }
                    dxr[k & (TBV - 1)] = dx;
                }
            }
            float lv[T + 1];
            float ST = 0.f;
#pragma unroll
            for (int t = 1; t <= T; t++) {
                const int sc = (k - 5 * t - TBD) & (TBV - 1);  // column slot of c_t in the column rings
                float xv[11];
#pragma unroll
                for (int j = -5; j <= 5; j++) {
                    const int it = (t == 1) ? (u - 5 - TBD + j) : (u - 5 + j);
                    xv[j + 5] = Q[t - 1][it & (TBQ - 1)];
                }
                const float ctr = xv[5];
                const float* rg = myRing + ((t - 1) * TBR + ((u - 5 * t - TBD) & (TBR - 1))) * TB_RS;
                float oldv;
                if (t == 1) oldv = Qold[(u - 5 - TBD) & (TBQ - 1)];
                else if (t == 2) oldv = Q[0][(u - 10 - TBD) & (TBQ - 1)];
                else oldv = Q[t - 2][(u - 10) & (TBQ - 1)];
                const float vv = myV[sc * TB_RS];
                const float Dm = fminf(Dz, dxr[sc]);

                const float lz = a.c.zc[0] * ctr + a.c.zc[1] * (rg[-1] + rg[1]) + a.c.zc[2] * (rg[-2] + rg[2]) +
                                 a.c.zc[3] * (rg[-3] + rg[3]) + a.c.zc[4] * (rg[-4] + rg[4]) +
                                 a.c.zc[5] * (rg[-5] + rg[5]);
                const float lx = a.c.xc[0] * ctr + a.c.xc[1] * (xv[6] + xv[4]) + a.c.xc[2] * (xv[7] + xv[3]) +
                                 a.c.xc[3] * (xv[8] + xv[2]) + a.c.xc[4] * (xv[9] + xv[1]) +
                                 a.c.xc[5] * (xv[10] + xv[0]);
                float n = vv * (lz + lx) + ctr + ctr - Dm * oldv;
                if (MODE == TB_SCAT) {
                    n = n + (mySL[sc * TB_RS] * a.h[t - 1] + mySR[sc * TB_RS] * a.h[H + t - 1]);
                } else if (nInj > 0) {
                    const int c = xs + k - 5 * t - TBD;
                    int p = injPtr[t - 1];
                    while (p < nInj && sEnt[p].col < c) p++;
                    injPtr[t - 1] = p;
                    for (int q = p; q < nInj && sEnt[q].col == c; q++) {
                        if (sEnt[q].row == z) {
                            const float* tr = pInj + (long long)sEnt[q].dev * injLd;
                            float v;
                            if (MODE == TB_ADJ) {
                                const int it2 = sub - t;
                                v = vv * (tr[its] * a.h[it2 + 1] + tr[its + 1] * a.h[H + it2 + 1]);
                            } else {
                                v = tr[its * sub + t - 1];
                            }
                            n = n + v;
                        }
                    }
                }
                const float S = n * Dm;
                if (t < T) {
                    Q[t][u] = S;
                    myRing[(t * TBR + ((u - 5 * t - TBD) & (TBR - 1))) * TB_RS] = S;
                    lv[t] = Q[t][(u - 5 * (T - t)) & (TBQ - 1)];
                } else {
                    ST = S;
                    lv[T] = S;
                }
            }

            // 2. outputs at column c_T
            const int cT = xs + k - 5 * T - TBD;
            if (zout && cT >= x0 && cT < x1) {
                const int idx = cT * ip + z;
                pNcur[idx] = ST;
                pNold[idx] = Q[T - 1][(u - 5) & (TBQ - 1)];
                if (MODE == TB_SRC) {
                    float wa = Pp[(u - TBP) & 7], wb = 0.f;
#pragma unroll
                    for (int l = 1; l <= T; l++) {
                        wa += lv[l] * a.h[l];
                        wb += lv[l] * a.h[H + l];
                    }
                    pPartOut[idx] = wb;
                    tb_wstore<WPREC>(Wo, idx, wa);
                    if (its == g.nts - 2) tb_wstore<WPREC>(tb_wslice<WPREC>(sh.W, a.wStride, its + 1), idx, wb);
                } else if (MODE == TB_ADJ) {
                    float ra = 0.f, rb = Pp[(u - TBP) & 7];
#pragma unroll
                    for (int l = 1; l <= T; l++) {
                        ra += lv[l] * a.h[sub - l];
                        rb += lv[l] * a.h[H + sub - l];
                    }
                    pPartOut[idx] = ra;
                    double acc = Pi[(u - TBP) & 7] + (double)(Pw[(u - TBP) & 7] * rb);
                    if (its == 0) acc += (double)(tb_wload<WPREC>(Wa, idx) * ra);
                    pImg[idx] = acc;
                } else if (nRec > 0) {
                    int p = recPtr;
                    while (p < nRec && sEnt[recOff + p].col < cT) p++;
                    recPtr = p;
                    for (int q = p; q < nRec && sEnt[recOff + q].col == cT; q++) {
                        if (sEnt[recOff + q].row == z) {
                            float ra = 0.f, rb = 0.f;
#pragma unroll
                            for (int l = 1; l <= T; l++) {
                                ra += lv[l] * a.h[l];
                                rb += lv[l] * a.h[H + l];
                            }
                            float* tr = pRec + (long long)sEnt[recOff + q].dev * recLd;
                            tr[its] += ra;
                            tr[its + 1] += rb;
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace aio
