// ============================================================================
// Reference-code harness — TEST INFRASTRUCTURE ONLY.
//
// Linked (by oracle/Makefile) with ONE of the reference's own GPU driver
// translation units, compiled for sm_100a from the reference tree where it
// lies. It exposes that driver's free functions (C++ linkage, declared in the
// reference's own headers) under extern "C" names so the parity tests can run
// the reference itself on a B200 and compare. Nothing here implements any of
// the scheme; it only forwards arguments and turns the reference's thrown
// std::runtime_error into a return code.
//
// REF_REAL is float (acoustic_iso_float) or double (acoustic_iso_double).
// ============================================================================
#include <stdexcept>
#include <vector>

#if defined(REF_FAMILY_NL)
#include "nonlinearShotsGpuFunctions.h"
#elif defined(REF_FAMILY_BORN)
#include "BornShotsGpuFunctions.h"
#elif defined(REF_FAMILY_BORNEXT)
#include "BornExtShotsGpuFunctions.h"
#elif defined(REF_FAMILY_TOMO)
#include "tomoExtShotsGpuFunctions.h"
#elif defined(REF_FAMILY_WEMVA)
#include "wemvaExtShotsGpuFunctions.h"
#endif

typedef REF_REAL R;
#define REF_EXPORT extern "C" __attribute__((visibility("default")))
#define GUARD(expr)       \
    try {                 \
        expr;             \
    } catch (...) {       \
        return -1;        \
    }                     \
    return 0;

// Single-GPU use: nGpu=1, iGpu=0, iGpuAlloc=iGpuId=device.
#if defined(REF_FAMILY_NL)
// F/include/nonlinearShotsGpuFunctions.h:7-24
REF_EXPORT int ref_init(R dz, R dx, int nz, int nx, int nts, R dts, int sub, int minPad, R alphaCos, int nExt,
                        int leg1, int leg2, int dev) {
    (void)nExt; (void)leg1; (void)leg2;
    GUARD(initNonlinearGpu(dz, dx, nz, nx, nts, dts, sub, minPad, 16, alphaCos, 1, dev, dev))
}
REF_EXPORT int ref_allocate(R* v2, R* rs, int dev) { (void)rs; GUARD(allocateNonlinearGpu(v2, 0, dev)) }
REF_EXPORT int ref_deallocate(int dev) { GUARD(deallocateNonlinearGpu(0, dev)) }
REF_EXPORT int ref_nl_fwd(R* modelDtw, R* data, int* sp, int ns, int* rp, int nr, R* W, int dev) {
    if (W) { GUARD(propShotsFwdGpuWavefield(modelDtw, data, sp, ns, rp, nr, W, 0, dev)) }
    GUARD(propShotsFwdGpu(modelDtw, data, sp, ns, rp, nr, W, 0, dev))
}
REF_EXPORT int ref_nl_adj(R* modelDtw, R* data, int* sp, int ns, int* rp, int nr, R* W, int dev) {
    if (W) { GUARD(propShotsAdjGpuWavefield(modelDtw, data, sp, ns, rp, nr, W, 0, dev)) }
    GUARD(propShotsAdjGpu(modelDtw, data, sp, ns, rp, nr, W, 0, dev))
}
// free-surface drivers (F/include/nonlinearShotsGpuFunctions.h:15,23)
REF_EXPORT int ref_nl_fwd_fs(R* modelDtw, R* data, int* sp, int ns, int* rp, int nr, R* W, int dev) {
    GUARD(propShotsFwdFsGpu(modelDtw, data, sp, ns, rp, nr, W, 0, dev))
}
REF_EXPORT int ref_nl_adj_fs(R* modelDtw, R* data, int* sp, int ns, int* rp, int nr, R* W, int dev) {
    GUARD(propShotsAdjFsGpu(modelDtw, data, sp, ns, rp, nr, W, 0, dev))
}
#elif defined(REF_FAMILY_BORN)
// F/include/BornShotsGpuFunctions.h:7-33
REF_EXPORT int ref_init(R dz, R dx, int nz, int nx, int nts, R dts, int sub, int minPad, R alphaCos, int nExt,
                        int leg1, int leg2, int dev) {
    (void)nExt; (void)leg1; (void)leg2;
    GUARD(initBornGpu(dz, dx, nz, nx, nts, dts, sub, minPad, 16, alphaCos, 1, dev, dev))
}
REF_EXPORT int ref_allocate(R* v2, R* rs, int dev) { GUARD(allocateBornShotsGpu(v2, rs, 0, dev)) }
REF_EXPORT int ref_deallocate(int dev) { GUARD(deallocateBornShotsGpu(0, dev)) }
REF_EXPORT int ref_born_fwd(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornShotsFwdGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
REF_EXPORT int ref_born_adj(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornShotsAdjGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
// wavefield drivers (F/include/BornShotsGpuFunctions.h:17,29): coarse [nts][nx][nz] wavefields out
REF_EXPORT int ref_born_fwd_wfld(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, R* srcW, R* secW,
                                 int dev) {
    GUARD(BornShotsFwdGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, secW, 0, dev))
}
REF_EXPORT int ref_born_adj_wfld(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, R* srcW, R* recW,
                                 int dev) {
    GUARD(BornShotsAdjGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, recW, 0, dev))
}
// free-surface drivers (F/include/BornShotsGpuFunctions.h:20,32)
REF_EXPORT int ref_born_fwd_fs(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornShotsFwdFsGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
REF_EXPORT int ref_born_adj_fs(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornShotsAdjFsGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
#elif defined(REF_FAMILY_BORNEXT)
// F/include/BornExtShotsGpuFunctions.h:6-54
REF_EXPORT int ref_init(R dz, R dx, int nz, int nx, int nts, R dts, int sub, int minPad, R alphaCos, int nExt,
                        int leg1, int leg2, int dev) {
    (void)leg1; (void)leg2;
    GUARD(initBornExtGpu(dz, dx, nz, nx, nts, dts, sub, minPad, 16, alphaCos, nExt, 1, dev, dev))
}
REF_EXPORT int ref_allocate(R* v2, R* rs, int dev) { GUARD(allocateBornExtShotsGpu(v2, rs, 0, dev)) }
REF_EXPORT int ref_deallocate(int dev) { GUARD(deallocateBornExtShotsGpu(0, dev)) }
REF_EXPORT int ref_bornext_fwd(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int sloth, int dev) {
    GUARD(BornTimeShotsFwdGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, sloth, 0, dev))
}
REF_EXPORT int ref_bornext_adj(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int sloth, int dev) {
    GUARD(BornTimeShotsAdjGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, sloth, 0, dev))
}
// subsurface-offset drivers (F/include/BornExtShotsGpuFunctions.h:22,44)
REF_EXPORT int ref_bornext_fwd_off(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornOffsetShotsFwdGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
REF_EXPORT int ref_bornext_adj_off(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornOffsetShotsAdjGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
// free-surface drivers (F/include/BornExtShotsGpuFunctions.h:27,49; no sloth flag)
REF_EXPORT int ref_bornext_fwd_fs(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornTimeShotsFwdFsGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
REF_EXPORT int ref_bornext_adj_fs(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(BornTimeShotsAdjFsGpu(model, data, sig, sp, ns, rp, nr, nullptr, nullptr, 0, dev))
}
// wavefield drivers (F/include/BornExtShotsGpuFunctions.h:19,23,28,32 forward; :41,45,50,54 adjoint):
// coarse [nts][nx][nz] wavefields out; off / fs select the offset and free-surface forms
REF_EXPORT int ref_bornext_fwd_wfld(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, R* srcW, R* secW,
                                    int off, int fs, int dev) {
    if (off && fs) { GUARD(BornOffsetShotsFwdFsGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, secW, 0, dev)) }
    if (off) { GUARD(BornOffsetShotsFwdGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, secW, 0, dev)) }
    if (fs) { GUARD(BornTimeShotsFwdFsGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, secW, 0, dev)) }
    GUARD(BornTimeShotsFwdGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, secW, 0, dev))
}
REF_EXPORT int ref_bornext_adj_wfld(R* model, R* data, R* sig, int* sp, int ns, int* rp, int nr, R* srcW, R* recW,
                                    int off, int fs, int dev) {
    if (off && fs) { GUARD(BornOffsetShotsAdjFsGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, recW, 0, dev)) }
    if (off) { GUARD(BornOffsetShotsAdjGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, recW, 0, dev)) }
    if (fs) { GUARD(BornTimeShotsAdjFsGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, recW, 0, dev)) }
    GUARD(BornTimeShotsAdjGpuWavefield(model, data, sig, sp, ns, rp, nr, srcW, recW, 0, dev))
}
#elif defined(REF_FAMILY_TOMO)
// F/include/tomoExtShotsGpuFunctions.h:6-33
REF_EXPORT int ref_init(R dz, R dx, int nz, int nx, int nts, R dts, int sub, int minPad, R alphaCos, int nExt,
                        int leg1, int leg2, int dev) {
    GUARD(initTomoExtGpu(dz, dx, nz, nx, nts, dts, sub, minPad, 16, alphaCos, nExt, leg1, leg2, 1, dev, dev))
}
REF_EXPORT int ref_allocate(R* v2, R* rs, int dev) { GUARD(allocateTomoExtShotsGpu(v2, rs, 0, dev)) }
REF_EXPORT int ref_deallocate(int dev) { GUARD(deallocateTomoExtShotsGpu(0, dev)) }
REF_EXPORT int ref_tomo_fwd(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, int sloth,
                            int dev) {
    GUARD(tomoTimeShotsFwdGpu(model, data, ext, sig, sp, ns, rp, nr, nullptr, nullptr, nullptr, sloth, 0, dev, 0))
}
REF_EXPORT int ref_tomo_adj(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, int sloth,
                            int dev) {
    GUARD(tomoTimeShotsAdjGpu(model, data, ext, sig, sp, ns, rp, nr, nullptr, nullptr, nullptr, sloth, 0, dev, 0))
}
// subsurface-offset drivers (F/include/tomoExtShotsGpuFunctions.h:17,29)
REF_EXPORT int ref_tomo_fwd_off(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(tomoOffsetShotsFwdGpu(model, data, ext, sig, sp, ns, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
REF_EXPORT int ref_tomo_adj_off(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(tomoOffsetShotsAdjGpu(model, data, ext, sig, sp, ns, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
// free-surface drivers (F/include/tomoExtShotsGpuFunctions.h:20,32; no sloth flag)
REF_EXPORT int ref_tomo_fwd_fs(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(tomoTimeShotsFwdFsGpu(model, data, ext, sig, sp, ns, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
REF_EXPORT int ref_tomo_adj_fs(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, int dev) {
    GUARD(tomoTimeShotsAdjFsGpu(model, data, ext, sig, sp, ns, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
// saveWavefield = 1: source d2/dt2 and the two secondary wavefields out ([nts][nx][nz] each);
// off / fs select the offset and free-surface drivers (sloth applies to the plain time-lag one)
REF_EXPORT int ref_tomo_fwd_wfld(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, R* W0, R* W1,
                                 R* W2, int off, int fs, int sloth, int dev) {
    if (off && fs) { GUARD(tomoOffsetShotsFwdFsGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, 0, dev, 1)) }
    if (off) { GUARD(tomoOffsetShotsFwdGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, 0, dev, 1)) }
    if (fs) { GUARD(tomoTimeShotsFwdFsGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, 0, dev, 1)) }
    GUARD(tomoTimeShotsFwdGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, sloth, 0, dev, 1))
}
REF_EXPORT int ref_tomo_adj_wfld(R* model, R* data, R* ext, R* sig, int* sp, int ns, int* rp, int nr, R* W0, R* W1,
                                 R* W2, int off, int fs, int sloth, int dev) {
    if (off && fs) { GUARD(tomoOffsetShotsAdjFsGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, 0, dev, 1)) }
    if (off) { GUARD(tomoOffsetShotsAdjGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, 0, dev, 1)) }
    if (fs) { GUARD(tomoTimeShotsAdjFsGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, 0, dev, 1)) }
    GUARD(tomoTimeShotsAdjGpu(model, data, ext, sig, sp, ns, rp, nr, W0, W1, W2, sloth, 0, dev, 1))
}
#elif defined(REF_FAMILY_WEMVA)
// F/include/wemvaExtShotsGpuFunctions.h:6-17
REF_EXPORT int ref_init(R dz, R dx, int nz, int nx, int nts, R dts, int sub, int minPad, R alphaCos, int nExt,
                        int leg1, int leg2, int dev) {
    GUARD(initWemvaExtGpu(dz, dx, nz, nx, nts, dts, sub, minPad, 16, alphaCos, nExt, leg1, leg2, 1, dev, dev))
}
REF_EXPORT int ref_allocate(R* v2, R* rs, int dev) { GUARD(allocateWemvaExtShotsGpu(v2, rs, 0, dev)) }
REF_EXPORT int ref_deallocate(int dev) { GUARD(deallocateWemvaExtShotsGpu(0, dev)) }
REF_EXPORT int ref_wemva_fwd(R* model, R* image, R* sig, int* sp, int ns, R* rdata, int* rp, int nr, int dev) {
    GUARD(wemvaTimeShotsFwdGpu(model, image, sig, sp, ns, rdata, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
REF_EXPORT int ref_wemva_adj(R* model, R* image, R* sig, int* sp, int ns, R* rdata, int* rp, int nr, int dev) {
    GUARD(wemvaTimeShotsAdjGpu(model, image, sig, sp, ns, rdata, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
// subsurface-offset drivers (F/include/wemvaExtShotsGpuFunctions.h:13,17)
REF_EXPORT int ref_wemva_fwd_off(R* model, R* image, R* sig, int* sp, int ns, R* rdata, int* rp, int nr, int dev) {
    GUARD(wemvaOffsetShotsFwdGpu(model, image, sig, sp, ns, rdata, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
REF_EXPORT int ref_wemva_adj_off(R* model, R* image, R* sig, int* sp, int ns, R* rdata, int* rp, int nr, int dev) {
    GUARD(wemvaOffsetShotsAdjGpu(model, image, sig, sp, ns, rdata, rp, nr, nullptr, nullptr, nullptr, 0, dev, 0))
}
// saveWavefield = 1: source d2/dt2 and the two secondary wavefields out; off selects the offset drivers
REF_EXPORT int ref_wemva_fwd_wfld(R* model, R* image, R* sig, int* sp, int ns, R* rdata, int* rp, int nr, R* W0,
                                  R* W1, R* W2, int off, int dev) {
    if (off) { GUARD(wemvaOffsetShotsFwdGpu(model, image, sig, sp, ns, rdata, rp, nr, W0, W1, W2, 0, dev, 1)) }
    GUARD(wemvaTimeShotsFwdGpu(model, image, sig, sp, ns, rdata, rp, nr, W0, W1, W2, 0, dev, 1))
}
REF_EXPORT int ref_wemva_adj_wfld(R* model, R* image, R* sig, int* sp, int ns, R* rdata, int* rp, int nr, R* W0,
                                  R* W1, R* W2, int off, int dev) {
    if (off) { GUARD(wemvaOffsetShotsAdjGpu(model, image, sig, sp, ns, rdata, rp, nr, W0, W1, W2, 0, dev, 1)) }
    GUARD(wemvaTimeShotsAdjGpu(model, image, sig, sp, ns, rdata, rp, nr, W0, W1, W2, 0, dev, 1))
}
#endif
