// C++ shims with the reference's own names for its GPU seam
// (F/include/{nonlinear,Born,BornExt,tomoExt,wemvaExt}ShotsGpuFunctions.h): each forwards
// to the aio_ C function of the same name and, where the reference would print and
// throw std::runtime_error or exit(-1), throws std::runtime_error with the library's
// message. Include this header instead of the reference's *ShotsGpuFunctions.h and
// link libaio_b200.so.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "aio_b200.h"

namespace aio_seam_detail {
inline void ck(int rc) {
    if (rc != AIO_OK) throw std::runtime_error(std::string("acoustic_isotropic_operators_b200: ") + aio_last_error());
}
}  // namespace aio_seam_detail

// F/src/nonlinearShotsGpuFunctions.cu:18-84 (true when every listed GPU exists)
inline bool getGpuInfo(std::vector<int> gpuList, int info, int deviceNumberInfo) {
    return aio_getGpuInfo(gpuList.data(), (int)gpuList.size(), info, deviceNumberInfo) == AIO_OK;
}

inline void initNonlinearGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc) { aio_seam_detail::ck(aio_initNonlinearGpu(dz, dx, nz, nx, nts, dts, sub, minPad, blockSize, alphaCos, nGpu, iGpuId, iGpuAlloc)); }
inline void allocateNonlinearGpu(float* vel2Dtw2, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_allocateNonlinearGpu(vel2Dtw2, iGpu, iGpuId)); }
inline void deallocateNonlinearGpu(int iGpu, int iGpuId) { aio_seam_detail::ck(aio_deallocateNonlinearGpu(iGpu, iGpuId)); }
inline void propShotsFwdGpu(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_propShotsFwdGpu(modelRegDtw, dataRegDts, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, wavefieldDts, iGpu, iGpuId)); }
inline void propShotsFwdGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_propShotsFwdGpuWavefield(modelRegDtw, dataRegDts, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, wavefieldDts, iGpu, iGpuId)); }
inline void propShotsAdjGpu(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_propShotsAdjGpu(modelRegDtw, dataRegDts, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, wavefieldDts, iGpu, iGpuId)); }
inline void propShotsAdjGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_propShotsAdjGpuWavefield(modelRegDtw, dataRegDts, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, wavefieldDts, iGpu, iGpuId)); }
inline void initBornGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc) { aio_seam_detail::ck(aio_initBornGpu(dz, dx, nz, nx, nts, dts, sub, minPad, blockSize, alphaCos, nGpu, iGpuId, iGpuAlloc)); }
inline void allocateBornShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_allocateBornShotsGpu(vel2Dtw2, reflectivityScale, iGpu, iGpuId)); }
inline void deallocateBornShotsGpu(int iGpu, int iGpuId) { aio_seam_detail::ck(aio_deallocateBornShotsGpu(iGpu, iGpuId)); }
inline void BornShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield, float* scatWavefield, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_BornShotsFwdGpu(model, dataRegDts, sourcesSignals, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, srcWavefield, scatWavefield, iGpu, iGpuId)); }
inline void BornShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield, float* recWavefield, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_BornShotsAdjGpu(model, dataRegDts, sourcesSignals, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, srcWavefield, recWavefield, iGpu, iGpuId)); }
inline void initBornExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize, float alphaCos, int nExt, int nGpu, int iGpuId, int iGpuAlloc) { aio_seam_detail::ck(aio_initBornExtGpu(dz, dx, nz, nx, nts, dts, sub, minPad, blockSize, alphaCos, nExt, nGpu, iGpuId, iGpuAlloc)); }
inline void allocateBornExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_allocateBornExtShotsGpu(vel2Dtw2, reflectivityScale, iGpu, iGpuId)); }
inline void deallocateBornExtShotsGpu(int iGpu, int iGpuId) { aio_seam_detail::ck(aio_deallocateBornExtShotsGpu(iGpu, iGpuId)); }
inline void BornTimeShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield, float* scatWavefield, int sloth, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_BornTimeShotsFwdGpu(model, dataRegDts, sourcesSignals, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, srcWavefield, scatWavefield, sloth, iGpu, iGpuId)); }
inline void BornTimeShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield, float* recWavefield, int sloth, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_BornTimeShotsAdjGpu(model, dataRegDts, sourcesSignals, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, srcWavefield, recWavefield, sloth, iGpu, iGpuId)); }
inline void initTomoExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize, float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId, int iGpuAlloc) { aio_seam_detail::ck(aio_initTomoExtGpu(dz, dx, nz, nx, nts, dts, sub, minPad, blockSize, alphaCos, nExt, leg1, leg2, nGpu, iGpuId, iGpuAlloc)); }
inline void allocateTomoExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_allocateTomoExtShotsGpu(vel2Dtw2, reflectivityScale, iGpu, iGpuId)); }
inline void deallocateTomoExtShotsGpu(int iGpu, int iGpuId) { aio_seam_detail::ck(aio_deallocateTomoExtShotsGpu(iGpu, iGpuId)); }
inline void tomoTimeShotsFwdGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2, int sloth, int iGpu, int iGpuId, int saveWavefield) { aio_seam_detail::ck(aio_tomoTimeShotsFwdGpu(model, dataRegDts, extReflectivity, sourcesSignals, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, tomoSrcWavefieldDt2, tomoSecWavefield1, tomoSecWavefield2, sloth, iGpu, iGpuId, saveWavefield)); }
inline void tomoTimeShotsAdjGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2, int sloth, int iGpu, int iGpuId, int saveWavefield) { aio_seam_detail::ck(aio_tomoTimeShotsAdjGpu(model, dataRegDts, extReflectivity, sourcesSignals, sourcesPositionReg, nSourcesReg, receiversPositionReg, nReceiversReg, tomoSrcWavefieldDt2, tomoSecWavefield1, tomoSecWavefield2, sloth, iGpu, iGpuId, saveWavefield)); }
inline void initWemvaExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize, float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId, int iGpuAlloc) { aio_seam_detail::ck(aio_initWemvaExtGpu(dz, dx, nz, nx, nts, dts, sub, minPad, blockSize, alphaCos, nExt, leg1, leg2, nGpu, iGpuId, iGpuAlloc)); }
inline void allocateWemvaExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) { aio_seam_detail::ck(aio_allocateWemvaExtShotsGpu(vel2Dtw2, reflectivityScale, iGpu, iGpuId)); }
inline void deallocateWemvaExtShotsGpu(int iGpu, int iGpuId) { aio_seam_detail::ck(aio_deallocateWemvaExtShotsGpu(iGpu, iGpuId)); }
inline void wemvaTimeShotsFwdGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, float* wemvaDataRegDts, int* receiversPositionReg, int nReceiversReg, float* wemvaSrcWavefieldDt2, float* wemvaSecWavefield1, float* wemvaSecWavefield2, int iGpu, int iGpuId, int saveWavefield) { aio_seam_detail::ck(aio_wemvaTimeShotsFwdGpu(model, wemvaExtImage, sourcesSignals, sourcesPositionReg, nSourcesReg, wemvaDataRegDts, receiversPositionReg, nReceiversReg, wemvaSrcWavefieldDt2, wemvaSecWavefield1, wemvaSecWavefield2, iGpu, iGpuId, saveWavefield)); }
inline void wemvaTimeShotsAdjGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sourcesPositionReg, int nSourcesReg, float* wemvaDataRegDts, int* receiversPositionReg, int nReceiversReg, float* wemvaSrcWavefieldDt2, float* wemvaSecWavefield1, float* wemvaSecWavefield2, int iGpu, int iGpuId, int saveWavefield) { aio_seam_detail::ck(aio_wemvaTimeShotsAdjGpu(model, wemvaExtImage, sourcesSignals, sourcesPositionReg, nSourcesReg, wemvaDataRegDts, receiversPositionReg, nReceiversReg, wemvaSrcWavefieldDt2, wemvaSecWavefield1, wemvaSecWavefield2, iGpu, iGpuId, saveWavefield)); }
