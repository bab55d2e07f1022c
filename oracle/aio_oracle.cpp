// ============================================================================
// CPU ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement (templated on float / double) of the reference's
// 2-D acoustic isotropic finite-difference scheme and of its pass sequences
// for the nonlinear, Born, extended (time-lag) Born, extended tomo and
// extended WEMVA operators. It exists to check the CUDA path: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. The
// product library never links or calls it.
//
// Reference paths below are relative to the reference project root:
//   F/ = acoustic_iso_lib/acoustic_iso_float   (FP32, restated with T=float)
//   D/ = acoustic_iso_lib/acoustic_iso_double  (FP64 twin, T=double)
// The FP64 tree is a type-for-type copy of the FP32 tree, so every citation
// into F/ holds for D/ at the same line.
//
// Parity pin: the reference ships no golden vectors or known-answer tests;
// this restatement is pinned against the reference's own compiled GPU code
// (oracle/_ref, built from the reference sources by oracle/Makefile and run
// on a B200) through fixtures committed under tests/golden/, and by FP64
// dot-product tests of every forward/adjoint pair.
//
// Arrays use the reference's host layout: a 2-D slice is nz*nx with z
// fastest (index = ix*nz + iz); wavefields are [nts][nx][nz]; traces are
// [nDevice][nt] with time fastest.
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

constexpr int FAT = 5;        // F/include/varDeclare.h:8
constexpr int SUB_MAX = 100;  // F/include/varDeclare.h:12
constexpr int PAD_MAX = 200;  // F/include/varDeclare.h:11

// Scheme constants and precomputed fields for one operator instance.
template <class T>
struct Grid {
    int nz, nx, nts, sub, ntw, minPad, H, nExt, hExt;
    int fs = 0;  // free surface at the top interior row (the reference's freeSurface == 1)
    int offset = 0;  // extension axis: 0 time lags, 1 subsurface (horizontal) offsets
    T zc[6], xc[6];
    T h[2 * (SUB_MAX + 1)];
    T taper[PAD_MAX];
    T cSide, cCenter;
    std::vector<T> v2, rs;  // v^2*dtw^2 and 2/v^3, nz*nx
    size_t N() const { return (size_t)nz * nx; }
};

// Laplacian coefficients: F/src/nonlinearShotsGpuFunctions.cu:123-135.
// Interpolation filter: F/src/nonlinearShotsGpuFunctions.cu:139-155.
// Cosine taper: F/src/nonlinearShotsGpuFunctions.cu:162-170.
// v^2 dtw^2 and 2/v^3: F/src/fdParam.cpp:15-25, 124-139.
// d2/dt2 coefficients for tomo/WEMVA: F/src/tomoExtShotsGpuFunctions.cu:138-139.
template <class T>
static void make_grid(Grid<T>& g, int nz, int nx, int nts, T dts, int sub, int minPad, T alphaCos,
                      T dz, T dx, int nExt, const T* vel) {
    g.nz = nz; g.nx = nx; g.nts = nts; g.sub = sub; g.ntw = (nts - 1) * sub + 1;
    g.minPad = minPad; g.H = sub + 1; g.nExt = nExt; g.hExt = (nExt - 1) / 2;
    static const double C[6] = {-2.927222222, 1.666666667, -0.238095238,
                                0.039682539,  -0.004960317, 0.000317460};
    for (int k = 0; k < 6; k++) {
        g.zc[k] = (T)(C[k] / (double)(dz * dz));
        g.xc[k] = (T)(C[k] / (double)(dx * dx));
    }
    const int H = g.H;
    for (int i = 0; i < 2 * (SUB_MAX + 1); i++) g.h[i] = 0;
    T r = std::sqrt((T)g.ntw / (T)g.nts);
    double sc = 1.0 / (double)r;
    for (int i = 0; i < H; i++) {
        g.h[i] = (T)(1.0 - 1.0 * i / sub);
        g.h[i + H] = (T)(1.0 - (double)g.h[i]);
        g.h[i] = (T)((double)g.h[i] * sc);
        g.h[i + H] = (T)((double)g.h[i + H] * sc);
    }
    for (int i = 0; i < PAD_MAX; i++) g.taper[i] = 1;
    for (int i = 0; i < minPad; i++) {
        T a = (T)(M_PI / (1.0 * minPad) * 1.0 * (minPad - i));
        T c = std::cos(a);
        g.taper[i] = (T)((double)alphaCos + (1.0 - (double)alphaCos) * (double)c);
    }
    g.cSide = (T)(1.0 / (double)(dts * dts));
    g.cCenter = (T)(-2.0 / (double)(dts * dts));
    T dtw = dts / (T)sub;
    g.v2.resize(g.N());
    g.rs.resize(g.N());
    for (size_t i = 0; i < g.N(); i++) {
        T v = vel[i];
        g.v2[i] = v * v * dtw * dtw;
        g.rs[i] = (T)(2.0 / (double)(T)(v * v * v));
    }
}

// ----------------------------------------------------------------------------
// Per-step building blocks (F/src/kernelsGpu.cu), applied to interior points
// iz in [FAT, nz-FAT), ix in [FAT, nx-FAT).
// ----------------------------------------------------------------------------

// setFsConditionFwdGpu, F/src/kernelsGpu.cu:555-567: on every interior column the top
// interior row of the current slice is set to zero and the FAT rows above it to the negative
// mirror of the rows below it (applied to the slice in memory before each forward step).
template <class T>
static void set_fs_fwd(const Grid<T>& g, T* c) {
    const int nz = g.nz;
    for (int ix = FAT; ix < g.nx - FAT; ix++) {
        T* col = c + (size_t)ix * nz;
        col[FAT] = 0;
        for (int m = 1; m <= FAT; m++) col[FAT - m] = -col[FAT + m];
    }
}

// stepFwdGpu, F/src/kernelsGpu.cu:513-552: n = v2*L(c) + 2c - o (n may alias o); with a free
// surface the current slice first gets setFsConditionFwdGpu (the reference's drivers launch it
// before every forward step, e.g. F/src/nonlinearShotsGpuFunctions.cu:446-450).
template <class T>
static void step_fwd(const Grid<T>& g, T* o, T* c) {
    const int nz = g.nz;
    if (g.fs) set_fs_fwd(g, c);
#pragma omp parallel for schedule(static)
    for (int ix = FAT; ix < g.nx - FAT; ix++) {
        for (int iz = FAT; iz < nz - FAT; iz++) {
            size_t i = (size_t)ix * nz + iz;
            T lap = g.zc[0] * c[i] + g.zc[1] * (c[i - 1] + c[i + 1]) + g.zc[2] * (c[i - 2] + c[i + 2]) +
                    g.zc[3] * (c[i - 3] + c[i + 3]) + g.zc[4] * (c[i - 4] + c[i + 4]) +
                    g.zc[5] * (c[i - 5] + c[i + 5]) + g.xc[0] * c[i] +
                    g.xc[1] * (c[i + nz] + c[i - nz]) + g.xc[2] * (c[i + 2 * nz] + c[i - 2 * nz]) +
                    g.xc[3] * (c[i + 3 * nz] + c[i - 3 * nz]) + g.xc[4] * (c[i + 4 * nz] + c[i - 4 * nz]) +
                    g.xc[5] * (c[i + 5 * nz] + c[i - 5 * nz]);
            o[i] = g.v2[i] * lap + c[i] + c[i] - o[i];
        }
    }
}

// stepAdjGpu, F/src/kernelsGpu.cu:574-610: o = L(v2*c) + 2c - n (o may alias n).
// Free surface: stepAdjFsGpu, :613-740 — the top interior row is not updated (it keeps n) and
// the z-stencil of the next four rows loses the terms the forward mirror condition adds.
template <class T>
static void step_adj(const Grid<T>& g, T* o, const T* c, std::vector<T>& tmp) {
    const int nz = g.nz;
    tmp.assign(g.N(), 0);
#pragma omp parallel for schedule(static)
    for (int ix = 0; ix < g.nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            size_t i = (size_t)ix * nz + iz;
            tmp[i] = c[i] * g.v2[i];
        }
    const T* s = tmp.data();
#pragma omp parallel for schedule(static)
    for (int ix = FAT; ix < g.nx - FAT; ix++) {
        for (int iz = FAT; iz < nz - FAT; iz++) {
            size_t i = (size_t)ix * nz + iz;
            if (g.fs && iz == FAT) continue;
            T lap = g.zc[0] * s[i] + g.zc[1] * (s[i - 1] + s[i + 1]) + g.zc[2] * (s[i - 2] + s[i + 2]) +
                    g.zc[3] * (s[i - 3] + s[i + 3]) + g.zc[4] * (s[i - 4] + s[i + 4]) +
                    g.zc[5] * (s[i - 5] + s[i + 5]);
            if (g.fs && iz < 2 * FAT) {
                // row r = iz - FAT (1..4): minus zc[k] * s[row k - r] for k = r+1 .. 5
                const int r = iz - FAT;
                for (int k = r + 1; k <= 5; k++) lap = lap - g.zc[k] * s[i + (k - 2 * r)];
            }
            lap = lap + g.xc[0] * s[i] +
                    g.xc[1] * (s[i + nz] + s[i - nz]) + g.xc[2] * (s[i + 2 * nz] + s[i - 2 * nz]) +
                    g.xc[3] * (s[i + 3 * nz] + s[i - 3 * nz]) + g.xc[4] * (s[i + 4 * nz] + s[i - 4 * nz]) +
                    g.xc[5] * (s[i + 5 * nz] + s[i - 5 * nz]);
            o[i] = lap + c[i] + c[i] - o[i];
        }
    }
}

// dampCosineEdge, F/src/kernelsGpu.cu:202-219: both slices scaled within minPad of the interior edge
// (free surface: dampCosineEdgeFs, :221-239, without the top edge).
template <class T>
static void damp(const Grid<T>& g, T* a, T* b) {
    const int nz = g.nz, nx = g.nx;
#pragma omp parallel for schedule(static)
    for (int ix = FAT; ix < nx - FAT; ix++)
        for (int iz = FAT; iz < nz - FAT; iz++) {
            int d = std::min(ix - FAT, std::min(nz - iz - 1 - FAT, nx - ix - 1 - FAT));
            if (!g.fs) d = std::min(d, iz - FAT);
            if (d < g.minPad) {
                size_t i = (size_t)ix * nz + iz;
                a[i] *= g.taper[d];
                b[i] *= g.taper[d];
            }
        }
}

// injectSource, F/src/kernelsGpu.cu:88-91.
template <class T>
static void inject_source(const Grid<T>& g, const T* sig, T* p, int itw, const int* pos, int n) {
    for (int s = 0; s < n; s++) p[pos[s]] += sig[(size_t)s * g.ntw + itw];
}
// interpInjectData, F/src/kernelsGpu.cu:94-99.
template <class T>
static void inject_data(const Grid<T>& g, const T* d, T* p, int its, int it2, const int* pos, int n) {
    for (int r = 0; r < n; r++)
        p[pos[r]] += d[(size_t)g.nts * r + its] * g.h[it2 + 1] + d[(size_t)g.nts * r + its + 1] * g.h[g.H + it2 + 1];
}
// recordSource, F/src/kernelsGpu.cu:113-116.
template <class T>
static void record_source(const Grid<T>& g, const T* p, T* m, int itw, const int* pos, int n) {
    for (int s = 0; s < n; s++) m[(size_t)g.ntw * s + itw] += p[pos[s]];
}
// recordInterpData, F/src/kernelsGpu.cu:119-127.
template <class T>
static void record_data(const Grid<T>& g, const T* p, T* d, int its, int it2, const int* pos, int n) {
    for (int r = 0; r < n; r++) {
        d[(size_t)g.nts * r + its] += p[pos[r]] * g.h[it2];
        d[(size_t)g.nts * r + its + 1] += p[pos[r]] * g.h[g.H + it2];
    }
}

template <class F>
static void for_interior(int nz, int nx, F&& f) {
#pragma omp parallel for schedule(static)
    for (int ix = FAT; ix < nx - FAT; ix++)
        for (int iz = FAT; iz < nz - FAT; iz++) f((size_t)ix * nz + iz);
}

// interpWavefield, F/src/kernelsGpu.cu:132-141 (W[its] and W[its+1]).
template <class T>
static void interp_wavefield(const Grid<T>& g, T* W, const T* p, int its, int it2) {
    const size_t N = g.N();
    T* w0 = W + (size_t)its * N;
    T* w1 = w0 + N;
    const T a = g.h[it2], b = g.h[g.H + it2];
    for_interior(g.nz, g.nx, [&](size_t i) { w0[i] += p[i] * a; w1[i] += p[i] * b; });
}
// extractInterpAdjointWavefield / interpFineToCoarseSlice, F/src/kernelsGpu.cu:166-182.
template <class T>
static void fine_to_coarse(const Grid<T>& g, T* L, T* R, const T* p, int it2) {
    const T a = g.h[it2], b = g.h[g.H + it2];
    for_interior(g.nz, g.nx, [&](size_t i) { L[i] += p[i] * a; R[i] += p[i] * b; });
}
// injectSecondarySource, F/src/kernelsGpu.cu:102-107.
template <class T>
static void inject_secondary(const Grid<T>& g, const T* L, const T* R, T* p, int k) {
    const T a = g.h[k], b = g.h[g.H + k];
    for_interior(g.nz, g.nx, [&](size_t i) { p[i] += L[i] * a + R[i] * b; });
}
// scaleReflectivity, F/src/kernelsGpu.cu:246-252.
template <class T>
static void scale_refl(const Grid<T>& g, T* m) {
    for_interior(g.nz, g.nx, [&](size_t i) { m[i] *= g.v2[i] * g.rs[i]; });
}
// scaleReflectivityExt / scaleReflectivitySlothExt, F/src/kernelsGpu.cu:278-303.
template <class T>
static void scale_refl_ext(const Grid<T>& g, T* m, int sloth) {
    const size_t N = g.N();
    for (int e = 0; e < g.nExt; e++) {
        T* me = m + (size_t)e * N;
        if (sloth == 0)
            for_interior(g.nz, g.nx, [&](size_t i) { me[i] *= g.rs[i] * g.v2[i]; });
        else
            for_interior(g.nz, g.nx, [&](size_t i) { me[i] = (T)((double)me[i] * (-1.0 * (double)g.v2[i])); });
    }
}
// imagingFwdGpu, F/src/kernelsGpu.cu:309-316: ss = m * W[its].
template <class T>
static void imaging_fwd(const Grid<T>& g, const T* m, T* ss, int its, const T* W) {
    const T* w = W + (size_t)its * g.N();
    for_interior(g.nz, g.nx, [&](size_t i) { ss[i] = m[i] * w[i]; });
}
// imagingAdjGpu, F/src/kernelsGpu.cu:318-325: m += W[its] * ss.
template <class T>
static void imaging_adj(const Grid<T>& g, T* m, const T* ss, const T* W, int its) {
    const T* w = W + (size_t)its * g.N();
    for_interior(g.nz, g.nx, [&](size_t i) { m[i] += w[i] * ss[i]; });
}
// imagingTimeFwdGpu, F/src/kernelsGpu.cu:337-350.
template <class T>
static void imaging_time_fwd(const Grid<T>& g, const T* m, T* ss, const T* W, int its, int e0, int e1) {
    const size_t N = g.N();
    for_interior(g.nz, g.nx, [&](size_t i) {
        for (int e = e0; e < e1; e++)
            ss[i] += m[(size_t)e * N + i] * W[(size_t)(its - 2 * (e - g.hExt)) * N + i];
    });
}
// imagingTimeAdjGpu, F/src/kernelsGpu.cu:352-364.
template <class T>
static void imaging_time_adj(const Grid<T>& g, T* m, const T* r, const T* W, int its, int e0, int e1) {
    const size_t N = g.N();
    for_interior(g.nz, g.nx, [&](size_t i) {
        for (int e = e0; e < e1; e++)
            m[(size_t)e * N + i] += r[i] * W[(size_t)(its - 2 * (e - g.hExt)) * N + i];
    });
}
// imagingWemvaTimeAdjGpu, F/src/kernelsGpu.cu:366-378.
template <class T>
static void imaging_wemva_time_adj(const Grid<T>& g, T* m, const T* s, const T* R, int its, int e0, int e1) {
    const size_t N = g.N();
    for_interior(g.nz, g.nx, [&](size_t i) {
        for (int e = e0; e < e1; e++)
            m[(size_t)e * N + i] += s[i] * R[(size_t)(its + 2 * (e - g.hExt)) * N + i];
    });
}
// imagingTimeTomoAdjGpu, F/src/kernelsGpu.cu:445-458.
template <class T>
static void imaging_time_tomo_adj(const Grid<T>& g, const T* Win, T* ss, const T* ext, int its, int e0, int e1) {
    const size_t N = g.N();
    for_interior(g.nz, g.nx, [&](size_t i) {
        for (int e = e0; e < e1; e++)
            ss[i] += ext[(size_t)e * N + i] * Win[(size_t)(its + 2 * (e - g.hExt)) * N + i];
    });
}

// ---- subsurface-offset extension (F/src/kernelsGpu.cu:254-276, 381-441) ----
// scaleReflectivityLinExt, :256-267: every offset slice times 2/v^3.
template <class T>
static void scale_refl_lin_ext(const Grid<T>& g, T* m) {
    const size_t N = g.N();
    for (int e = 0; e < g.nExt; e++) {
        T* me = m + (size_t)e * N;
        for_interior(g.nz, g.nx, [&](size_t i) { me[i] *= g.rs[i]; });
    }
}
// scaleSecondarySourceFd, :270-276: a slice times v^2 dtw^2.
template <class T>
static void scale_ss_fd(const Grid<T>& g, T* ss) {
    for_interior(g.nz, g.nx, [&](size_t i) { ss[i] *= g.v2[i]; });
}
// imagingOffsetFwdGpu, :381-395: ss(x) += sum_s m_s(x-s) W_its(x-2s) over the offsets whose model
// point x-s lies in [FAT+h, nx-FAT-h).
template <class T>
static void imaging_offset_fwd(const Grid<T>& g, const T* m, T* ss, const T* W, int its) {
    const int nz = g.nz, nx = g.nx, h = g.hExt;
    const size_t N = g.N();
    const T* w = W + (size_t)its * N;
    for (int ix = FAT; ix < nx - FAT; ix++) {
        const int e0 = std::max(-h, ix + 1 + FAT + h - nx), e1 = std::min(ix - h - FAT, h) + 1;
        for (int iz = FAT; iz < nz - FAT; iz++) {
            const size_t i = (size_t)ix * nz + iz;
            for (int s = e0; s < e1; s++)
                ss[i] += m[(size_t)(s + h) * N + (size_t)(ix - s) * nz + iz] * w[(size_t)(ix - 2 * s) * nz + iz];
        }
    }
}
// imagingOffsetAdjGpu, :397-411: m_e(x) += r(x+s) W_its(x-s), s = e-h, x in [FAT+h, nx-FAT-h).
template <class T>
static void imaging_offset_adj(const Grid<T>& g, T* m, const T* r, const T* W, int its) {
    const int nz = g.nz, nx = g.nx, h = g.hExt;
    const size_t N = g.N();
    const T* w = W + (size_t)its * N;
    for (int e = 0; e < g.nExt; e++) {
        const int s = e - h;
        for (int ix = FAT + h; ix < nx - FAT - h; ix++)
            for (int iz = FAT; iz < nz - FAT; iz++)
                m[(size_t)e * N + (size_t)ix * nz + iz] += r[(size_t)(ix + s) * nz + iz] * w[(size_t)(ix - s) * nz + iz];
    }
}
// imagingOffsetWemvaScaleFwdGpu, :429-443: m_e(x) += c(x-s) R_its(x+s) v2(x+s).
template <class T>
static void imaging_offset_wemva_scale_fwd(const Grid<T>& g, T* m, const T* c, const T* R, int its) {
    const int nz = g.nz, nx = g.nx, h = g.hExt;
    const size_t N = g.N();
    const T* r = R + (size_t)its * N;
    for (int e = 0; e < g.nExt; e++) {
        const int s = e - h;
        for (int ix = FAT + h; ix < nx - FAT - h; ix++)
            for (int iz = FAT; iz < nz - FAT; iz++) {
                const size_t j = (size_t)(ix + s) * nz + iz;
                m[(size_t)e * N + (size_t)ix * nz + iz] += c[(size_t)(ix - s) * nz + iz] * r[j] * g.v2[j];
            }
    }
}
// imagingOffsetTomoAdjGpu, :460-476: ss(x) += sum_s m_s(x+s) R_its(x+2s) v2(x+2s) over the offsets
// whose model point x+s lies in [FAT+h, nx-FAT-h).
template <class T>
static void imaging_offset_tomo_adj(const Grid<T>& g, const T* R, T* ss, const T* m, int its) {
    const int nz = g.nz, nx = g.nx, h = g.hExt;
    const size_t N = g.N();
    const T* r = R + (size_t)its * N;
    for (int ix = FAT; ix < nx - FAT; ix++) {
        const int e0 = std::max(-h, FAT + h - ix), e1 = std::min(nx - 1 - FAT - ix - h, h) + 1;
        for (int iz = FAT; iz < nz - FAT; iz++) {
            const size_t i = (size_t)ix * nz + iz;
            for (int s = e0; s < e1; s++) {
                const size_t j = (size_t)(ix + 2 * s) * nz + iz;
                ss[i] += m[(size_t)(s + h) * N + (size_t)(ix + s) * nz + iz] * r[j] * g.v2[j];
            }
        }
    }
}

// Lag bounds with C truncating division, as in F/src/BornExtShotsGpuFunctions.cu:366-383
// ("source side": W index its-2*lag in [0,nts)) and
// F/src/tomoExtShotsGpuFunctions.cu:2631-2650 ("receiver side": index its+2*lag).
template <class T>
static void lag_bounds_src(const Grid<T>& g, int t, int& e0, int& e1) {
    e0 = std::max((t + 1 - g.nts) / 2, -g.hExt) + g.hExt;
    e1 = std::min(t / 2, g.hExt) + g.hExt + 1;
}
template <class T>
static void lag_bounds_rec(const Grid<T>& g, int t, int& e0, int& e1) {
    e0 = std::max((-t) / 2, -g.hExt) + g.hExt;
    e1 = std::min((g.nts - 1 - t) / 2, g.hExt) + g.hExt + 1;
}

template <class T>
struct Work {
    std::vector<T> p0, p1, a, b, c, d, tmp;
    explicit Work(size_t N) : p0(N, 0), p1(N, 0), a(N, 0), b(N, 0), c(N, 0), d(N, 0) {}
};
template <class T>
static void zero(std::vector<T>& v) { std::fill(v.begin(), v.end(), (T)0); }

// ----------------------------------------------------------------------------
// Source-side propagation shared by every operator: stepFwd, inject source
// at itw-1, damp, then a per-step hook (store W, record, ...).
// F/src/nonlinearShotsGpuFunctions.cu:269-295, F/src/BornShotsGpuFunctions.cu:297-321.
// ----------------------------------------------------------------------------
template <class T, class Hook>
static void src_pass(const Grid<T>& g, Work<T>& w, const T* sig, const int* pos, int n, Hook&& hook) {
    zero(w.p0); zero(w.p1);
    T* P0 = w.p0.data();
    T* P1 = w.p1.data();
    for (int its = 0; its < g.nts - 1; its++)
        for (int it2 = 1; it2 < g.sub + 1; it2++) {
            int itw = its * g.sub + it2;
            step_fwd(g, P0, P1);
            inject_source(g, sig, P0, itw - 1, pos, n);
            damp(g, P0, P1);
            hook(P0, its, it2);
            std::swap(P0, P1);
        }
}

// Receiver-side adjoint propagation: stepAdj, inject data, damp, hook.
// F/src/nonlinearShotsGpuFunctions.cu:616-641, F/src/BornShotsGpuFunctions.cu:906-927.
template <class T, class Hook>
static void rec_pass(const Grid<T>& g, Work<T>& w, const T* data, const int* pos, int n, Hook&& hook) {
    zero(w.p0); zero(w.p1);
    T* P0 = w.p0.data();
    T* P1 = w.p1.data();
    for (int its = g.nts - 2; its > -1; its--)
        for (int it2 = g.sub - 1; it2 > -1; it2--) {
            step_adj(g, P0, P1, w.tmp);
            inject_data(g, data, P0, its, it2, pos, n);
            damp(g, P0, P1);
            hook(P0, its, it2);
            std::swap(P0, P1);
        }
}

// Forward-time scattered propagation driven by coarse secondary sources.
// make_ss(its, ss) fills ss for coarse time its (ss is zero on entry when
// reset_ss), then per fine step: stepFwd, inject ss with h[it2-1], damp, hook;
// after each coarse interval post(its, L) runs with the accumulated fine->coarse
// slice for `its` when accumulate=true.
// F/src/BornShotsGpuFunctions.cu:342-374, F/src/tomoExtShotsGpuFunctions.cu:2460-2525.
template <class T, class MakeSS, class Hook, class Post>
static void scat_fwd_pass(const Grid<T>& g, Work<T>& w, MakeSS&& make_ss, bool reset_ss, Hook&& hook,
                          bool accumulate, Post&& post) {
    zero(w.p0); zero(w.p1); zero(w.a); zero(w.b); zero(w.c); zero(w.d);
    T *P0 = w.p0.data(), *P1 = w.p1.data();
    T *SL = w.a.data(), *SR = w.b.data();
    T *CL = w.c.data(), *CR = w.d.data();
    const size_t N = g.N();
    make_ss(0, SL);
    for (int its = 0; its < g.nts - 1; its++) {
        make_ss(its + 1, SR);
        for (int it2 = 1; it2 < g.sub + 1; it2++) {
            step_fwd(g, P0, P1);
            inject_secondary(g, SL, SR, P0, it2 - 1);
            damp(g, P0, P1);
            hook(P0, its, it2);
            if (accumulate) fine_to_coarse(g, CL, CR, P0, it2);
            std::swap(P0, P1);
        }
        if (accumulate) post(its, CL);
        std::swap(SL, SR);
        if (reset_ss) std::fill(SR, SR + N, (T)0);
        if (accumulate) {
            std::swap(CL, CR);
            std::fill(CR, CR + N, (T)0);
        }
    }
    if (accumulate) post(g.nts - 1, CL);
}

// Backward-time scattered propagation (adjoint stepper) driven by coarse secondary
// sources injected with h[it2+1]; accumulated slice for coarse time its+1 handed
// to post(). F/src/tomoExtShotsGpuFunctions.cu:2619-2700,
// F/src/wemvaExtShotsGpuFunctions.cu:1038-1121.
template <class T, class MakeSS, class Post>
static void scat_adj_pass(const Grid<T>& g, Work<T>& w, MakeSS&& make_ss, bool reset_ss, Post&& post) {
    zero(w.p0); zero(w.p1); zero(w.a); zero(w.b); zero(w.c); zero(w.d);
    T *P0 = w.p0.data(), *P1 = w.p1.data();
    T *SL = w.a.data(), *SR = w.b.data();
    T *CL = w.c.data(), *CR = w.d.data();
    const size_t N = g.N();
    make_ss(g.nts - 1, SR);
    for (int its = g.nts - 2; its > -1; its--) {
        make_ss(its, SL);
        for (int it2 = g.sub - 1; it2 > -1; it2--) {
            step_adj(g, P0, P1, w.tmp);
            inject_secondary(g, SL, SR, P0, it2 + 1);
            damp(g, P0, P1);
            fine_to_coarse(g, CL, CR, P0, it2);
            std::swap(P0, P1);
        }
        post(its + 1, CR);
        std::swap(SR, SL);
        if (reset_ss) std::fill(SL, SL + N, (T)0);
        std::swap(CR, CL);
        std::fill(CL, CL + N, (T)0);
    }
    post(0, CR);
}

// Coarse source wavefield W[nts][nx][nz]: F/src/BornShotsGpuFunctions.cu:297-321.
template <class T>
static void source_wavefield(const Grid<T>& g, Work<T>& w, const T* sig, const int* pos, int n, T* W) {
    std::fill(W, W + (size_t)g.nts * g.N(), (T)0);
    src_pass(g, w, sig, pos, n, [&](const T* p, int its, int it2) { interp_wavefield(g, W, p, its, it2); });
}

// Coarse second time derivative of the source wavefield (zero outside [0,nts)).
// Equivalent to computeTomoSrcWfldDt2, F/src/tomoExtShotsGpuFunctions.cu:1251-1361:
// the coarse samples come from the same fine->coarse spreading and
// srcWfldSecondTimeDerivative (F/src/kernelsGpu.cu:188-197) is applied per sample.
template <class T>
static void source_wavefield_dt2(const Grid<T>& g, Work<T>& w, const T* sig, const int* pos, int n, T* W2) {
    const size_t N = g.N();
    std::vector<T> W((size_t)g.nts * N);
    source_wavefield(g, w, sig, pos, n, W.data());
    std::fill(W2, W2 + (size_t)g.nts * N, (T)0);
    for (int its = 0; its < g.nts; its++) {
        const T* s1 = W.data() + (size_t)its * N;
        const T* s0 = its > 0 ? s1 - N : nullptr;
        const T* s2 = its < g.nts - 1 ? s1 + N : nullptr;
        T* o = W2 + (size_t)its * N;
        for_interior(g.nz, g.nx, [&](size_t i) {
            T a = s0 ? s0[i] : (T)0;
            T b = s2 ? s2[i] : (T)0;
            o[i] = g.cSide * (a + b) + g.cCenter * s1[i];
        });
    }
}

// Receiver wavefield (adjoint propagation of data, stored coarse):
// computeTomoRecWfld, F/src/tomoExtShotsGpuFunctions.cu:1481-1515.
template <class T>
static void receiver_wavefield(const Grid<T>& g, Work<T>& w, const T* data, const int* pos, int n, T* R) {
    std::fill(R, R + (size_t)g.nts * g.N(), (T)0);
    rec_pass(g, w, data, pos, n, [&](const T* p, int its, int it2) { interp_wavefield(g, R, p, its, it2); });
}

// Saved wavefields (saveWavefield = 1): copy a whole [nts][nx][nz] field, or one coarse slice t.
template <class T>
static void copy_out(const Grid<T>& g, const std::vector<T>& W, T* out) {
    if (out) std::copy(W.begin(), W.begin() + (size_t)g.nts * g.N(), out);
}
template <class T>
static void save_slice(const Grid<T>& g, T* out, const T* C, int t) {
    if (out) std::copy(C, C + g.N(), out + (size_t)t * g.N());
}

// ============================ operators =====================================

// Nonlinear forward, F/src/nonlinearShotsGpuFunctions.cu:227-309 (and :310-395 with W).
template <class T>
static void nl_fwd(const Grid<T>& g, const T* model, const int* sp, int ns, const int* rp, int nr, T* data, T* W) {
    Work<T> w(g.N());
    std::fill(data, data + (size_t)nr * g.nts, (T)0);
    if (W) std::fill(W, W + (size_t)g.nts * g.N(), (T)0);
    src_pass(g, w, model, sp, ns, [&](const T* p, int its, int it2) {
        if (W) interp_wavefield(g, W, p, its, it2);
        record_data(g, p, data, its, it2, rp, nr);
    });
}

// Nonlinear adjoint, F/src/nonlinearShotsGpuFunctions.cu:579-652 (and :653-737 with W).
template <class T>
static void nl_adj(const Grid<T>& g, T* model, const int* sp, int ns, const int* rp, int nr, const T* data, T* W) {
    Work<T> w(g.N());
    std::fill(model, model + (size_t)ns * g.ntw, (T)0);
    if (W) std::fill(W, W + (size_t)g.nts * g.N(), (T)0);
    rec_pass(g, w, data, rp, nr, [&](const T* p, int its, int it2) {
        if (W) interp_wavefield(g, W, p, its, it2);
        record_source(g, p, model, its * g.sub + it2, sp, ns);
    });
}

// Born forward, F/src/BornShotsGpuFunctions.cu:260-388.
template <class T>
// Wsec (optional): the coarse scattered wavefield (BornShotsFwdGpuWavefield,
// F/src/BornShotsGpuFunctions.cu:390-535, interpWavefield of the scattered pass).
static void born_fwd(const Grid<T>& g, const T* model, const T* sig, const int* sp, int ns, const int* rp, int nr,
                     T* data, T* Wsrc, T* Wsec = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> Wloc;
    T* W = Wsrc;
    if (!W) { Wloc.resize((size_t)g.nts * N); W = Wloc.data(); }
    source_wavefield(g, w, sig, sp, ns, W);
    std::vector<T> dm(model, model + N);
    scale_refl(g, dm.data());
    std::fill(data, data + (size_t)nr * g.nts, (T)0);
    if (Wsec) std::fill(Wsec, Wsec + (size_t)g.nts * N, (T)0);
    scat_fwd_pass(
        g, w, [&](int t, T* ss) { imaging_fwd(g, dm.data(), ss, t, W); }, true,
        [&](const T* p, int its, int it2) {
            if (Wsec) interp_wavefield(g, Wsec, p, its, it2);
            record_data(g, p, data, its, it2, rp, nr);
        },
        false, [](int, T*) {});
}

// recordScaleWavefield, F/src/kernelsGpu.cu:145-153: W[its] += r * rs * v2.
template <class T>
static void record_scale_wavefield(const Grid<T>& g, T* W, const T* r, int its) {
    T* w = W + (size_t)its * g.N();
    for_interior(g.nz, g.nx, [&](size_t i) { w[i] += r[i] * g.rs[i] * g.v2[i]; });
}

// Born adjoint, F/src/BornShotsGpuFunctions.cu:829-957.
template <class T>
// Wrec (optional): the coarse receiver wavefield scaled by 2/v^3 * v^2 dtw^2 (recordScaleWavefield,
// F/src/kernelsGpu.cu:145-153, in BornShotsAdjGpuWavefield, F/src/BornShotsGpuFunctions.cu:959-1103).
static void born_adj(const Grid<T>& g, T* model, const T* sig, const int* sp, int ns, const int* rp, int nr,
                     const T* data, T* Wsrc, T* Wrec = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> Wloc;
    T* W = Wsrc;
    if (!W) { Wloc.resize((size_t)g.nts * N); W = Wloc.data(); }
    source_wavefield(g, w, sig, sp, ns, W);
    std::fill(model, model + N, (T)0);
    // receiver pass with fine->coarse spreading into L/R and imaging at its+1.
    std::vector<T> L(N, 0), R(N, 0);
    T *pL = L.data(), *pR = R.data();
    zero(w.p0); zero(w.p1);
    T *P0 = w.p0.data(), *P1 = w.p1.data();
    for (int its = g.nts - 2; its > -1; its--) {
        for (int it2 = g.sub - 1; it2 > -1; it2--) {
            step_adj(g, P0, P1, w.tmp);
            inject_data(g, data, P0, its, it2, rp, nr);
            damp(g, P0, P1);
            fine_to_coarse(g, pL, pR, P0, it2);
            std::swap(P0, P1);
        }
        imaging_adj(g, model, pR, W, its + 1);
        if (Wrec) record_scale_wavefield(g, Wrec, pR, its + 1);
        std::swap(pR, pL);
        std::fill(pL, pL + N, (T)0);
    }
    if (Wrec) record_scale_wavefield(g, Wrec, pR, 0);
    imaging_adj(g, model, pR, W, 0);
    scale_refl(g, model);
}

// Extended (time-lag) Born forward, F/src/BornExtShotsGpuFunctions.cu:269-419.
// Wsrc / Wsec (optional): the coarse source and scattered wavefields (BornTimeShotsFwdGpuWavefield,
// :420-580, and BornOffsetShotsFwdGpuWavefield, :726-884: interpWavefield of the scattered pass;
// those drivers take no sloth flag).
template <class T>
static void bornext_fwd(const Grid<T>& g, const T* model, const T* sig, const int* sp, int ns, const int* rp,
                        int nr, T* data, int sloth, T* Wsrc = nullptr, T* Wsec = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> Wloc;
    T* Wp = Wsrc;
    if (!Wp) { Wloc.resize((size_t)g.nts * N); Wp = Wloc.data(); }
    source_wavefield(g, w, sig, sp, ns, Wp);
    if (Wsec) std::fill(Wsec, Wsec + (size_t)g.nts * N, (T)0);
    std::vector<T> dm(model, model + (size_t)g.nExt * N);
    // subsurface offsets: BornOffsetShotsFwdGpu, F/src/BornExtShotsGpuFunctions.cu:582-724
    if (g.offset) scale_refl_lin_ext(g, dm.data());
    else scale_refl_ext(g, dm.data(), sloth);
    std::fill(data, data + (size_t)nr * g.nts, (T)0);
    scat_fwd_pass(
        g, w,
        [&](int t, T* ss) {
            if (g.offset) {
                imaging_offset_fwd(g, dm.data(), ss, Wp, t);
                scale_ss_fd(g, ss);
                return;
            }
            int e0, e1;
            lag_bounds_src(g, t, e0, e1);
            imaging_time_fwd(g, dm.data(), ss, Wp, t, e0, e1);
        },
        true,
        [&](const T* p, int its, int it2) {
            if (Wsec) interp_wavefield(g, Wsec, p, its, it2);
            record_data(g, p, data, its, it2, rp, nr);
        },
        false, [](int, T*) {});
}

// recordWavefield (F/src/kernelsGpu.cu:138-143): W[its] += r.
template <class T>
static void record_wavefield(const Grid<T>& g, T* W, const T* r, int its) {
    T* w = W + (size_t)its * g.N();
    for_interior(g.nz, g.nx, [&](size_t i) { w[i] += r[i]; });
}

// Extended (time-lag) Born adjoint, F/src/BornExtShotsGpuFunctions.cu:1525-1675.
// Wsrc / Wrec (optional): the coarse source wavefield and the receiver wavefield
// (BornTimeShotsAdjGpuWavefield, :1680-1847: recordScaleWavefield before each imaging step;
// BornOffsetShotsAdjGpuWavefield, :1991-2151: recordWavefield of the v2-scaled sample).
template <class T>
static void bornext_adj(const Grid<T>& g, T* model, const T* sig, const int* sp, int ns, const int* rp, int nr,
                        const T* data, int sloth, T* Wsrc = nullptr, T* Wrec = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> Wloc;
    T* Wp = Wsrc;
    if (!Wp) { Wloc.resize((size_t)g.nts * N); Wp = Wloc.data(); }
    source_wavefield(g, w, sig, sp, ns, Wp);
    if (Wrec) std::fill(Wrec, Wrec + (size_t)g.nts * N, (T)0);
    std::fill(model, model + (size_t)g.nExt * N, (T)0);
    std::vector<T> L(N, 0), R(N, 0);
    T *pL = L.data(), *pR = R.data();
    zero(w.p0); zero(w.p1);
    T *P0 = w.p0.data(), *P1 = w.p1.data();
    int e0, e1;
    for (int its = g.nts - 2; its > -1; its--) {
        for (int it2 = g.sub - 1; it2 > -1; it2--) {
            step_adj(g, P0, P1, w.tmp);
            inject_data(g, data, P0, its, it2, rp, nr);
            damp(g, P0, P1);
            fine_to_coarse(g, pL, pR, P0, it2);
            std::swap(P0, P1);
        }
        if (g.offset) {  // BornOffsetShotsAdjGpu, F/src/BornExtShotsGpuFunctions.cu:1848-1990
            scale_ss_fd(g, pR);
            if (Wrec) record_wavefield(g, Wrec, pR, its + 1);
            imaging_offset_adj(g, model, pR, Wp, its + 1);
        } else {
            if (Wrec) record_scale_wavefield(g, Wrec, pR, its + 1);
            lag_bounds_src(g, its + 1, e0, e1);
            imaging_time_adj(g, model, pR, Wp, its + 1, e0, e1);
        }
        std::swap(pR, pL);
        std::fill(pL, pL + N, (T)0);
    }
    if (g.offset) {
        scale_ss_fd(g, pR);
        if (Wrec) record_wavefield(g, Wrec, pR, 0);
        imaging_offset_adj(g, model, pR, Wp, 0);
        scale_refl_lin_ext(g, model);
        return;
    }
    if (Wrec) record_scale_wavefield(g, Wrec, pR, 0);
    lag_bounds_src(g, 0, e0, e1);
    imaging_time_adj(g, model, pR, Wp, 0, e0, e1);
    scale_refl_ext(g, model, sloth);
}

// Extended tomo forward, F/src/tomoExtShotsGpuFunctions.cu:355-465 with
// legs :1554-1656 (s->i->m->d) and :1782-1881 (s->m->i->d).
template <class T>
//
// Saved wavefields (non-null Wsrc, Wsec1, Wsec2: the drivers' saveWavefield = 1): d2/dt2 of the
// source wavefield; the last leg's first scattered wavefield (tomoSecWavefield1, :429-432);
// the last leg's recorded scattered wavefield, accumulated per leg from zero
// (tomoSecWavefield2, :1615-1641, :1839-1871).
static void tomo_fwd(const Grid<T>& g, const T* model, const T* extRefl, const T* sig, const int* sp, int ns,
                     const int* rp, int nr, T* data, int sloth, int leg1, int leg2, T* Wsrc = nullptr,
                     T* Wsec1 = nullptr, T* Wsec2 = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> W2((size_t)g.nts * N), W1((size_t)g.nts * N);
    source_wavefield_dt2(g, w, sig, sp, ns, W2.data());
    std::vector<T> dm(model, model + N);
    scale_refl(g, dm.data());
    std::vector<T> ext(extRefl, extRefl + (size_t)g.nExt * N);
    // subsurface offsets: tomoOffsetShotsFwdGpu, F/src/tomoExtShotsGpuFunctions.cu:467-575, legs :2005-2105, :2227-2323
    if (g.offset) scale_refl_lin_ext(g, ext.data());
    else scale_refl_ext(g, ext.data(), sloth);
    std::fill(data, data + (size_t)nr * g.nts, (T)0);
    auto ext_src = [&](const T* Win) {
        return [&, Win](int t, T* ss) {
            if (g.offset) {
                imaging_offset_fwd(g, ext.data(), ss, Win, t);
                scale_ss_fd(g, ss);
                return;
            }
            int e0, e1;
            lag_bounds_src(g, t, e0, e1);
            imaging_time_fwd(g, ext.data(), ss, Win, t, e0, e1);
        };
    };
    auto store_W1 = [&](const T* p, int its, int it2) { interp_wavefield(g, W1.data(), p, its, it2); };
    auto rec = [&](const T* p, int its, int it2) {
        if (Wsec2) interp_wavefield(g, Wsec2, p, its, it2);
        record_data(g, p, data, its, it2, rp, nr);
    };
    auto nop = [](int, T*) {};
    copy_out(g, W2, Wsrc);
    auto clear_sec2 = [&] {
        if (Wsec2) std::fill(Wsec2, Wsec2 + (size_t)g.nts * N, (T)0);
    };
    if (leg1) {
        std::fill(W1.begin(), W1.end(), (T)0);
        scat_fwd_pass(g, w, ext_src(W2.data()), true, store_W1, false, nop);
        clear_sec2();
        scat_fwd_pass(g, w, [&](int t, T* ss) { imaging_fwd(g, dm.data(), ss, t, W1.data()); }, false, rec,
                      false, nop);
    }
    if (leg2) {
        std::fill(W1.begin(), W1.end(), (T)0);
        scat_fwd_pass(g, w, [&](int t, T* ss) { imaging_fwd(g, dm.data(), ss, t, W2.data()); }, false, store_W1,
                      false, nop);
        clear_sec2();
        scat_fwd_pass(g, w, ext_src(W1.data()), true, rec, false, nop);
    }
    copy_out(g, W1, Wsec1);
}

// Extended tomo adjoint, F/src/tomoExtShotsGpuFunctions.cu:797-910 with legs
// :2442-2527 (leg 1) and :2619-2701 (leg 2).
template <class T>
//
// Saved wavefields: d2/dt2 of the source wavefield, the receiver wavefield (tomoSecWavefield1,
// :850) and the coarse samples of the last leg's scattered wavefield, taken as they are imaged
// (tomoSecWavefield2, :2507-2525, :2680-2700).
static void tomo_adj(const Grid<T>& g, T* model, const T* extRefl, const T* sig, const int* sp, int ns,
                     const int* rp, int nr, const T* data, int sloth, int leg1, int leg2, T* Wsrc = nullptr,
                     T* Wsec1 = nullptr, T* Wsec2 = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> W2((size_t)g.nts * N), R((size_t)g.nts * N);
    source_wavefield_dt2(g, w, sig, sp, ns, W2.data());
    receiver_wavefield(g, w, data, rp, nr, R.data());
    copy_out(g, W2, Wsrc);
    copy_out(g, R, Wsec1);
    std::vector<T> ext(extRefl, extRefl + (size_t)g.nExt * N);
    // subsurface offsets: tomoOffsetShotsAdjGpu, F/src/tomoExtShotsGpuFunctions.cu:912-1023, legs :2788-2866, :2949-3021
    if (g.offset) scale_refl_lin_ext(g, ext.data());
    else scale_refl_ext(g, ext.data(), sloth);
    std::fill(model, model + N, (T)0);
    if (leg1) {
        scat_fwd_pass(
            g, w,
            [&](int t, T* ss) {
                if (g.offset) {
                    imaging_offset_fwd(g, ext.data(), ss, W2.data(), t);
                    scale_ss_fd(g, ss);
                    return;
                }
                int e0, e1;
                lag_bounds_src(g, t, e0, e1);
                imaging_time_fwd(g, ext.data(), ss, W2.data(), t, e0, e1);
            },
            true, [](const T*, int, int) {}, true,
            [&](int t, T* C) {
                save_slice(g, Wsec2, C, t);
                imaging_adj(g, model, C, R.data(), t);
            });
    }
    if (leg2) {
        scat_adj_pass(
            g, w,
            [&](int t, T* ss) {
                if (g.offset) {
                    imaging_offset_tomo_adj(g, R.data(), ss, ext.data(), t);
                    return;
                }
                int e0, e1;
                lag_bounds_rec(g, t, e0, e1);
                imaging_time_tomo_adj(g, R.data(), ss, ext.data(), t, e0, e1);
            },
            true, [&](int t, T* C) {
                save_slice(g, Wsec2, C, t);
                imaging_adj(g, model, C, W2.data(), t);
            });
    }
    scale_refl(g, model);
}

// Extended WEMVA forward, F/src/wemvaExtShotsGpuFunctions.cu:344-456 with legs
// :961-1037 (s->m->i<-d) and :1038-1122 (s->i<-m<-d). `rdata` is the regular-grid
// WEMVA data that drives the receiver wavefield.
template <class T>
//
// Saved wavefields: d2/dt2 of the source wavefield, the receiver wavefield (wemvaSecWavefield1,
// :55) and the coarse samples of the last leg's scattered wavefield as they are imaged
// (wemvaSecWavefield2, :1009, :1033, :1091, :1117; the offset second leg saves them after the
// v^2 dtw^2 scaling, :1232-1239).
static void wemva_fwd(const Grid<T>& g, const T* model, const T* sig, const int* sp, int ns, const int* rp, int nr,
                      const T* rdata, T* image, int leg1, int leg2, T* Wsrc = nullptr, T* Wsec1 = nullptr,
                      T* Wsec2 = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> W2((size_t)g.nts * N), R((size_t)g.nts * N);
    source_wavefield_dt2(g, w, sig, sp, ns, W2.data());
    receiver_wavefield(g, w, rdata, rp, nr, R.data());
    copy_out(g, W2, Wsrc);
    copy_out(g, R, Wsec1);
    std::vector<T> dm(model, model + N);
    scale_refl(g, dm.data());
    std::fill(image, image + (size_t)g.nExt * N, (T)0);
    if (leg1) {
        scat_fwd_pass(
            g, w, [&](int t, T* ss) { imaging_fwd(g, dm.data(), ss, t, W2.data()); }, false,
            [](const T*, int, int) {}, true, [&](int t, T* C) {
                save_slice(g, Wsec2, C, t);
                if (g.offset) {  // wemvaOffsetShotsFwdGpu (:458-574) legs, F/src/wemvaExtShotsGpuFunctions.cu:1123-1269
                    imaging_offset_wemva_scale_fwd(g, image, C, R.data(), t);
                    return;
                }
                int e0, e1;
                lag_bounds_rec(g, t, e0, e1);
                imaging_wemva_time_adj(g, image, C, R.data(), t, e0, e1);
            });
    }
    if (leg2) {
        scat_adj_pass(
            g, w, [&](int t, T* ss) { imaging_fwd(g, dm.data(), ss, t, R.data()); }, false, [&](int t, T* C) {
                if (g.offset) {
                    scale_ss_fd(g, C);
                    save_slice(g, Wsec2, C, t);
                    imaging_offset_adj(g, image, C, W2.data(), t);
                    return;
                }
                save_slice(g, Wsec2, C, t);
                int e0, e1;
                lag_bounds_src(g, t, e0, e1);
                imaging_time_adj(g, image, C, W2.data(), t, e0, e1);
            });
    }
    if (g.offset) scale_refl_lin_ext(g, image);
    else scale_refl_ext(g, image, 0);
}

// Extended WEMVA adjoint, F/src/wemvaExtShotsGpuFunctions.cu:575-688 with legs
// :1270-1350 (leg 1) and :1352-1426 (leg 2).
template <class T>
//
// Saved wavefields: as wemva_fwd (wemvaSecWavefield2 from :1325, :1347, :1401, :1422).
static void wemva_adj(const Grid<T>& g, T* model, const T* sig, const int* sp, int ns, const int* rp, int nr,
                      const T* rdata, const T* imageIn, int leg1, int leg2, T* Wsrc = nullptr, T* Wsec1 = nullptr,
                      T* Wsec2 = nullptr) {
    Work<T> w(g.N());
    const size_t N = g.N();
    std::vector<T> W2((size_t)g.nts * N), R((size_t)g.nts * N);
    source_wavefield_dt2(g, w, sig, sp, ns, W2.data());
    receiver_wavefield(g, w, rdata, rp, nr, R.data());
    copy_out(g, W2, Wsrc);
    copy_out(g, R, Wsec1);
    std::vector<T> img(imageIn, imageIn + (size_t)g.nExt * N);
    // subsurface offsets: wemvaOffsetShotsAdjGpu, F/src/wemvaExtShotsGpuFunctions.cu:689-810, legs :1428-1580
    if (g.offset) scale_refl_lin_ext(g, img.data());
    else scale_refl_ext(g, img.data(), 0);
    std::fill(model, model + N, (T)0);
    if (leg1) {
        scat_adj_pass(
            g, w,
            [&](int t, T* ss) {
                if (g.offset) {
                    imaging_offset_tomo_adj(g, R.data(), ss, img.data(), t);
                    return;
                }
                int e0, e1;
                lag_bounds_rec(g, t, e0, e1);
                imaging_time_tomo_adj(g, R.data(), ss, img.data(), t, e0, e1);
            },
            true, [&](int t, T* C) {
                save_slice(g, Wsec2, C, t);
                imaging_adj(g, model, C, W2.data(), t);
            });
    }
    if (leg2) {
        scat_fwd_pass(
            g, w,
            [&](int t, T* ss) {
                if (g.offset) {
                    imaging_offset_fwd(g, img.data(), ss, W2.data(), t);
                    scale_ss_fd(g, ss);
                    return;
                }
                int e0, e1;
                lag_bounds_src(g, t, e0, e1);
                imaging_time_fwd(g, img.data(), ss, W2.data(), t, e0, e1);
            },
            true, [](const T*, int, int) {}, true, [&](int t, T* C) {
                save_slice(g, Wsec2, C, t);
                imaging_adj(g, model, C, R.data(), t);
            });
    }
    scale_refl(g, model);
}

// ======================= host-side preparation ==============================

// interpTimeLinTbb::forward/adjoint, F/src/interpTimeLinTbb.cpp:26-102.
template <class T>
static void time_interp_fwd(int nts, T dts, T ots, int sub, int nDev, const T* m, T* d) {
    int ntw = (nts - 1) * sub + 1;
    T dtw = dts / sub;
    T otw = ots;
    T sc = (T)ntw / (T)nts;
    sc = (T)(1.0 / (double)std::sqrt(sc));
    std::fill(d, d + (size_t)nDev * ntw, (T)0);
    for (int k = 0; k < nDev; k++) {
        const T* mk = m + (size_t)k * nts;
        T* dk = d + (size_t)k * ntw;
        for (int itw = 0; itw < ntw - 1; itw++) {
            T tw = otw + itw * dtw;
            T weight = (tw - ots) / dts;
            int inf = (int)weight;
            weight = weight - inf;
            dk[itw] += (mk[inf] * (1.0 - weight) + mk[inf + 1] * weight) * sc;
        }
        dk[ntw - 1] += sc * mk[nts - 1];
    }
}
template <class T>
static void time_interp_adj(int nts, T dts, T ots, int sub, int nDev, T* m, const T* d) {
    int ntw = (nts - 1) * sub + 1;
    T dtw = dts / sub;
    T otw = ots;
    T sc = (T)ntw / (T)nts;
    sc = (T)(1.0 / (double)std::sqrt(sc));
    std::fill(m, m + (size_t)nDev * nts, (T)0);
    for (int k = 0; k < nDev; k++) {
        T* mk = m + (size_t)k * nts;
        const T* dk = d + (size_t)k * ntw;
        for (int itw = 0; itw < ntw - 1; itw++) {
            T tw = otw + itw * dtw;
            T weight = (tw - ots) / dts;
            int inf = (int)weight;
            weight = weight - inf;
            mk[inf] += sc * dk[itw] * (1.0 - weight);
            mk[inf + 1] += sc * dk[itw] * weight;
        }
        mk[nts - 1] += sc * dk[ntw - 1];
    }
}
// secondTimeDerivative::forward, F/src/secondTimeDerivative.cpp:14-26 (self-adjoint stencil).
template <class T>
static void second_deriv(int nt, T dt, int nDev, const T* m, T* d) {
    T dt2 = (T)(1.0 / (double)(dt * dt));
    std::fill(d, d + (size_t)nDev * nt, (T)0);
    for (int k = 0; k < nDev; k++) {
        const T* mk = m + (size_t)k * nt;
        T* dk = d + (size_t)k * nt;
        dk[0] += dt2 * (mk[1] - 2.0 * mk[0]);
        for (int it = 1; it < nt - 1; it++) dk[it] += dt2 * (mk[it + 1] - 2.0 * mk[it] + mk[it - 1]);
        dk[nt - 1] += dt2 * (mk[nt - 2] - 2.0 * mk[nt - 1]);
    }
}

}  // namespace orc

// ============================ C ABI for ctypes ===============================
using namespace orc;

struct OrcParams {
    int nz, nx, nts, sub, minPad, nExt;
    double dz, dx, dts, alphaCos;
    int freeSurface;
    int extension;  // 0 time lags, 1 subsurface offsets
};

template <class T>
static Grid<T> grid_from(const OrcParams* p, const T* vel) {
    Grid<T> g;
    make_grid<T>(g, p->nz, p->nx, p->nts, (T)p->dts, p->sub, p->minPad, (T)p->alphaCos, (T)p->dz, (T)p->dx,
                 p->nExt, vel);
    g.fs = p->freeSurface;
    g.offset = p->extension;
    return g;
}

#define ORC_EXPORT extern "C" __attribute__((visibility("default")))

#define ORC_DEFINE(SUF, T)                                                                                        \
    ORC_EXPORT void orc_constants_##SUF(const OrcParams* p, const T* vel, T* zc, T* xc, T* h, T* taper, T* v2,   \
                                        T* rs) {                                                                  \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        for (int k = 0; k < 6; k++) { zc[k] = g.zc[k]; xc[k] = g.xc[k]; }                                         \
        for (int k = 0; k < 2 * g.H; k++) h[k] = g.h[k];                                                          \
        for (int k = 0; k < g.minPad; k++) taper[k] = g.taper[k];                                                 \
        std::copy(g.v2.begin(), g.v2.end(), v2);                                                                  \
        std::copy(g.rs.begin(), g.rs.end(), rs);                                                                  \
    }                                                                                                             \
    ORC_EXPORT void orc_nl_fwd_##SUF(const OrcParams* p, const T* vel, const T* model, const int* sp, int ns,      \
                                     const int* rp, int nr, T* data, T* W) {                                      \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        nl_fwd<T>(g, model, sp, ns, rp, nr, data, W);                                                             \
    }                                                                                                             \
    ORC_EXPORT void orc_nl_adj_##SUF(const OrcParams* p, const T* vel, T* model, const int* sp, int ns,            \
                                     const int* rp, int nr, const T* data, T* W) {                                \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        nl_adj<T>(g, model, sp, ns, rp, nr, data, W);                                                             \
    }                                                                                                             \
    ORC_EXPORT void orc_born_fwd_##SUF(const OrcParams* p, const T* vel, const T* model, const T* sig,            \
                                       const int* sp, int ns, const int* rp, int nr, T* data, T* W, T* S) {       \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        born_fwd<T>(g, model, sig, sp, ns, rp, nr, data, W, S);                                                   \
    }                                                                                                             \
    ORC_EXPORT void orc_born_adj_##SUF(const OrcParams* p, const T* vel, T* model, const T* sig, const int* sp,   \
                                       int ns, const int* rp, int nr, const T* data, T* W, T* R) {                \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        born_adj<T>(g, model, sig, sp, ns, rp, nr, data, W, R);                                                   \
    }                                                                                                             \
    ORC_EXPORT void orc_bornext_fwd_##SUF(const OrcParams* p, const T* vel, const T* model, const T* sig,         \
                                          const int* sp, int ns, const int* rp, int nr, T* data, int sloth) {     \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        bornext_fwd<T>(g, model, sig, sp, ns, rp, nr, data, sloth);                                               \
    }                                                                                                             \
    ORC_EXPORT void orc_bornext_adj_##SUF(const OrcParams* p, const T* vel, T* model, const T* sig,               \
                                          const int* sp, int ns, const int* rp, int nr, const T* data,            \
                                          int sloth) {                                                            \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        bornext_adj<T>(g, model, sig, sp, ns, rp, nr, data, sloth);                                               \
    }                                                                                                             \
    ORC_EXPORT void orc_bornext_fwd_wfld_##SUF(const OrcParams* p, const T* vel, const T* model, const T* sig,    \
                                               const int* sp, int ns, const int* rp, int nr, T* data, T* W,       \
                                               T* S) {                                                            \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        bornext_fwd<T>(g, model, sig, sp, ns, rp, nr, data, 0, W, S);                                             \
    }                                                                                                             \
    ORC_EXPORT void orc_bornext_adj_wfld_##SUF(const OrcParams* p, const T* vel, T* model, const T* sig,          \
                                               const int* sp, int ns, const int* rp, int nr, const T* data, T* W, \
                                               T* R) {                                                            \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        bornext_adj<T>(g, model, sig, sp, ns, rp, nr, data, 0, W, R);                                             \
    }                                                                                                             \
    ORC_EXPORT void orc_tomo_fwd_##SUF(const OrcParams* p, const T* vel, const T* model, const T* ext,            \
                                       const T* sig, const int* sp, int ns, const int* rp, int nr, T* data,       \
                                       int sloth, int leg1, int leg2, T* W0, T* W1, T* W2) {                      \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        tomo_fwd<T>(g, model, ext, sig, sp, ns, rp, nr, data, sloth, leg1, leg2, W0, W1, W2);                     \
    }                                                                                                             \
    ORC_EXPORT void orc_tomo_adj_##SUF(const OrcParams* p, const T* vel, T* model, const T* ext, const T* sig,    \
                                       const int* sp, int ns, const int* rp, int nr, const T* data, int sloth,    \
                                       int leg1, int leg2, T* W0, T* W1, T* W2) {                                 \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        tomo_adj<T>(g, model, ext, sig, sp, ns, rp, nr, data, sloth, leg1, leg2, W0, W1, W2);                     \
    }                                                                                                             \
    ORC_EXPORT void orc_wemva_fwd_##SUF(const OrcParams* p, const T* vel, const T* model, const T* sig,           \
                                        const int* sp, int ns, const int* rp, int nr, const T* rdata, T* image,   \
                                        int leg1, int leg2, T* W0, T* W1, T* W2) {                                \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        wemva_fwd<T>(g, model, sig, sp, ns, rp, nr, rdata, image, leg1, leg2, W0, W1, W2);                        \
    }                                                                                                             \
    ORC_EXPORT void orc_wemva_adj_##SUF(const OrcParams* p, const T* vel, T* model, const T* sig, const int* sp,  \
                                        int ns, const int* rp, int nr, const T* rdata, const T* image, int leg1,  \
                                        int leg2, T* W0, T* W1, T* W2) {                                          \
        Grid<T> g = grid_from<T>(p, vel);                                                                         \
        wemva_adj<T>(g, model, sig, sp, ns, rp, nr, rdata, image, leg1, leg2, W0, W1, W2);                        \
    }                                                                                                             \
    ORC_EXPORT void orc_time_interp_fwd_##SUF(int nts, double dts, double ots, int sub, int nDev, const T* m,      \
                                              T* d) {                                                             \
        time_interp_fwd<T>(nts, (T)dts, (T)ots, sub, nDev, m, d);                                                 \
    }                                                                                                             \
    ORC_EXPORT void orc_time_interp_adj_##SUF(int nts, double dts, double ots, int sub, int nDev, T* m,            \
                                              const T* d) {                                                       \
        time_interp_adj<T>(nts, (T)dts, (T)ots, sub, nDev, m, d);                                                 \
    }                                                                                                             \
    ORC_EXPORT void orc_second_deriv_##SUF(int nt, double dt, int nDev, const T* m, T* d) {                       \
        second_deriv<T>(nt, (T)dt, nDev, m, d);                                                                   \
    }

ORC_DEFINE(f32, float)
ORC_DEFINE(f64, double)
