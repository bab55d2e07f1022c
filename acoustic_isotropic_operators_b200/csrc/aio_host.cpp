// Host-side preparation of the reference's per-shot operators, in C++ with the
// reference's FP32 expressions (results feed the GPU seam unchanged):
//   * fdParam precompute of v^2 dtw^2 and 2/v^3   (F/src/fdParam.cpp:15-25, 124-139)
//   * linear coarse<->fine time interpolation      (F/src/interpTimeLinTbb.cpp:9-102)
//   * coarse second time derivative                (F/src/secondTimeDerivative.cpp:9-39)
//   * dtw^2 v^2 source scaling                     (F/include/seismicOperator2D.cpp:72-86)
//   * device spread / gather on unique grid points (F/src/deviceGpu.cpp:201-261)
//   * the Born-family source preparation chain     (F/include/seismicOperator2D.cpp:10-39)
// OpenMP replaces the reference's TBB parallel_for.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "aio_b200.h"

#define AIO_API extern "C" __attribute__((visibility("default")))

AIO_API int aio_fd_precompute(int nz, int nx, float dts, int sub, const float* vel, float* vel2Dtw2,
                              float* reflectivityScale) {
    if (nz <= 0 || nx <= 0 || sub <= 0 || !vel) return AIO_ERR_ARGUMENT;
    const float dtw = dts / float(sub);
#pragma omp parallel for schedule(static)
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            const long long i = (long long)ix * nz + iz;
            const float v = vel[i];
            if (vel2Dtw2) vel2Dtw2[i] = v * v * dtw * dtw;
            if (reflectivityScale) reflectivityScale[i] = (float)(2.0 / (double)(v * v * v));
        }
    return AIO_OK;
}

AIO_API int aio_time_interp_forward(int add, int nts, float dts, float ots, int sub, int nDev, const float* coarse,
                                    float* fine) {
    if (nts < 2 || sub < 1) return AIO_ERR_ARGUMENT;
    const int ntw = (nts - 1) * sub + 1;
    const float dtw = dts / sub;
    const float otw = ots;
    float sc = float(ntw) / float(nts);
    sc = 1.0 / std::sqrt(sc);
    if (!add) std::memset(fine, 0, sizeof(float) * (size_t)nDev * ntw);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nDev; k++) {
        const float* m = coarse + (size_t)k * nts;
        float* d = fine + (size_t)k * ntw;
        for (int itw = 0; itw < ntw - 1; itw++) {
            const float tw = otw + itw * dtw;
            float weight = (tw - ots) / dts;
            const int inf = weight;
            weight = weight - inf;
            d[itw] += (m[inf] * (1.0 - weight) + m[inf + 1] * weight) * sc;
        }
        d[ntw - 1] += sc * m[nts - 1];
    }
    return AIO_OK;
}

AIO_API int aio_time_interp_adjoint(int add, int nts, float dts, float ots, int sub, int nDev, float* coarse,
                                    const float* fine) {
    if (nts < 2 || sub < 1) return AIO_ERR_ARGUMENT;
    const int ntw = (nts - 1) * sub + 1;
    const float dtw = dts / sub;
    const float otw = ots;
    float sc = float(ntw) / float(nts);
    sc = 1.0 / std::sqrt(sc);
    if (!add) std::memset(coarse, 0, sizeof(float) * (size_t)nDev * nts);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nDev; k++) {
        float* m = coarse + (size_t)k * nts;
        const float* d = fine + (size_t)k * ntw;
        for (int itw = 0; itw < ntw - 1; itw++) {
            const float tw = otw + itw * dtw;
            float weight = (tw - ots) / dts;
            const int inf = weight;
            weight = weight - inf;
            m[inf] += sc * d[itw] * (1.0 - weight);
            m[inf + 1] += sc * d[itw] * weight;
        }
        m[nts - 1] += sc * d[ntw - 1];
    }
    return AIO_OK;
}

// The reference stencil is symmetric, so forward and adjoint are the same map.
AIO_API int aio_second_time_derivative(int add, int nt, float dt, int nDev, const float* in, float* out) {
    if (nt < 2) return AIO_ERR_ARGUMENT;
    const float dt2 = 1.0 / (dt * dt);
    if (!add) std::memset(out, 0, sizeof(float) * (size_t)nDev * nt);
    for (int k = 0; k < nDev; k++) {
        const float* m = in + (size_t)k * nt;
        float* d = out + (size_t)k * nt;
        d[0] += dt2 * (m[1] - 2.0 * m[0]);
        for (int it = 1; it < nt - 1; it++) d[it] += dt2 * (m[it + 1] - 2.0 * m[it] + m[it - 1]);
        d[nt - 1] += dt2 * (m[nt - 2] - 2.0 * m[nt - 1]);
    }
    return AIO_OK;
}

AIO_API int aio_scale_seismic_source(int nDevReg, const int* posReg, int nt, float dts, int sub, const float* vel,
                                     float* signal) {
    const float dtw = dts / float(sub);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nDevReg; k++) {
        const float scale = dtw * dtw * vel[posReg[k]] * vel[posReg[k]];
        for (int it = 0; it < nt; it++) signal[(size_t)k * nt + it] = signal[(size_t)k * nt + it] * scale;
    }
    return AIO_OK;
}

// cornerIdx[nDevIrreg*nCorner] indexes the unique regular list; weights alike.
AIO_API int aio_device_spread(int add, int nDevIrreg, int nCorner, const int* cornerIdx, const float* weights,
                              int nDevReg, int nt, const float* irreg, float* reg) {
    if (!add) std::memset(reg, 0, sizeof(float) * (size_t)nDevReg * nt);
    for (int d = 0; d < nDevIrreg; d++)
        for (int c = 0; c < nCorner; c++) {
            const int i1 = d * nCorner + c;
            const int i2 = cornerIdx[i1];
            if (i2 < 0 || i2 >= nDevReg) return AIO_ERR_ARGUMENT;
            for (int it = 0; it < nt; it++) reg[(size_t)i2 * nt + it] += weights[i1] * irreg[(size_t)d * nt + it];
        }
    return AIO_OK;
}

AIO_API int aio_device_gather(int add, int nDevIrreg, int nCorner, const int* cornerIdx, const float* weights,
                              int nDevReg, int nt, const float* reg, float* irreg) {
    if (!add) std::memset(irreg, 0, sizeof(float) * (size_t)nDevIrreg * nt);
    for (int d = 0; d < nDevIrreg; d++)
        for (int c = 0; c < nCorner; c++) {
            const int i1 = d * nCorner + c;
            const int i2 = cornerIdx[i1];
            if (i2 < 0 || i2 >= nDevReg) return AIO_ERR_ARGUMENT;
            for (int it = 0; it < nt; it++) irreg[(size_t)d * nt + it] += weights[i1] * reg[(size_t)i2 * nt + it];
        }
    return AIO_OK;
}

// Born / tomo / WEMVA source chain (seismicOperator2D::setSources): spread the
// irregular wavelets to the unique grid points, d2/dt2 on the coarse grid,
// dtw^2 v^2 scaling, linear interpolation to the fine grid. Output
// [nDevReg][ntw]. With secondDerivative=0 it is the nonlinear chain
// (F/src/nonlinearPropGpu.cpp:44-51).
AIO_API int aio_prepare_source(int secondDerivative, int nDevIrreg, int nCorner, const int* cornerIdx,
                               const float* weights, int nDevReg, const int* posReg, int nts, float dts, int sub,
                               const float* vel, const float* wavelets, float* out) {
    std::vector<float> reg((size_t)nDevReg * nts), d2((size_t)nDevReg * nts);
    int rc = aio_device_spread(0, nDevIrreg, nCorner, cornerIdx, weights, nDevReg, nts, wavelets, reg.data());
    if (rc) return rc;
    float* cur = reg.data();
    if (secondDerivative) {
        rc = aio_second_time_derivative(0, nts, dts, nDevReg, reg.data(), d2.data());
        if (rc) return rc;
        cur = d2.data();
    }
    rc = aio_scale_seismic_source(nDevReg, posReg, nts, dts, sub, vel, cur);
    if (rc) return rc;
    return aio_time_interp_forward(0, nts, dts, 0.f, sub, nDevReg, cur, out);
}
