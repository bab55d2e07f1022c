/*
 * aio_b200.h — C ABI of the B200 (sm_100a) acoustic isotropic operators.
 *
 * Two layers, both plain C (pointers, sizes, int status codes; 0 = success):
 *
 *  1. Reference seam. Drop-in replacements for the free functions the
 *     reference's per-shot operators call (F/include/*ShotsGpuFunctions.h,
 *     F = acoustic_iso_lib/acoustic_iso_float), same argument lists, prefixed
 *     `aio_`, returning a status instead of throwing / exit(-1). Each family
 *     keeps its own state per iGpu slot, so the families are re-entrant with
 *     respect to one another (the reference shares one set of globals).
 *
 *  2. Batched API. An `aio_context` holds one operator instance (one grid,
 *     velocity and device). Every call takes a whole batch of shots and runs
 *     them together: one fused stepper launch advances every shot of a wave by
 *     one fine step. `memSpace` says whether the per-shot trace / model arrays
 *     are host (AIO_MEM_HOST) or device (AIO_MEM_DEVICE) pointers; device
 *     position arrays are always host arrays.
 *
 * Conventions (identical to the reference): slices are nz*nx floats with z
 * fastest (index ix*nz+iz, FAT=5 ring included); device positions are such
 * linear indices ("regular" grid points, unique per list); traces are
 * [nDevice][nt] with time fastest; fine time has ntw=(nts-1)*sub+1 samples.
 * Source / receiver positions must lie inside the interior
 * [5,nz-5) x [5,nx-5); other positions return AIO_ERR_ARGUMENT.
 */
#ifndef AIO_B200_H
#define AIO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AIO_OK 0
#define AIO_ERR_ARGUMENT 1   /* invalid parameter / geometry (reference: std::runtime_error) */
#define AIO_ERR_CUDA 2       /* CUDA runtime error (reference: exit(-1)) */
#define AIO_ERR_MEMORY 3     /* device allocation failed */
#define AIO_ERR_STATE 4      /* call order (e.g. shot call before allocate) */

#define AIO_MEM_HOST 0
#define AIO_MEM_DEVICE 1

#define AIO_NONLINEAR 0
#define AIO_BORN 1
#define AIO_BORN_EXT 2
#define AIO_TOMO_EXT 3
#define AIO_WEMVA_EXT 4

#define AIO_WFLD_FP32 0  /* stored source wavefield in FP32 (reference behaviour) */
#define AIO_WFLD_BF16 1  /* BF16 (no scale: BF16 keeps FP32's exponent range) */
#define AIO_WFLD_FP16 2  /* FP16 with a per-time-slice FP32 scale */
/* Compressed settings apply on the interval-blocked stepper to the Born source wavefield, the
 * extended Born (time lags) source wavefield, and the tomo / WEMVA source field d2/dt2 (their
 * second stored field stays FP32); the subsurface-offset extension and the per-fine-step paths
 * refuse them with AIO_ERR_ARGUMENT. */

typedef struct aio_context aio_context;

typedef struct {
    int nz, nx;          /* padded grid including FAT (reference par nz, nx) */
    int nts, sub;        /* coarse samples, fine sub-steps per coarse step */
    int minPad;          /* sponge width, min(zPad, xPad) (F/src/fdParam.cpp:93) */
    int nExt;            /* extension length (odd), 1 for non-extended operators */
    float dz, dx, dts;   /* spacings (m) and coarse sampling (s) */
    float alphaCos;      /* taper floor, reference default 0.99 */
    int leg1, leg2;      /* tomo / WEMVA legs (reference par leg1, leg2) */
    int sloth;           /* extended Born / tomo: slowness-squared perturbation */
    int wavefieldPrecision;  /* AIO_WFLD_* for the stored source wavefield */
    int imageFp64;       /* 1: accumulate imaging conditions in FP64 on the GPU; 0: in FP32, as the
                            reference's imaging kernels do */
    int device;          /* CUDA device ordinal */
    long long memBudgetBytes; /* cap on device memory for shot buffers; 0 = 93% of free */
    int stepper;         /* AIO_STEPPER_*: how Born / nonlinear passes advance time */
    int chunkColumns;    /* blocked stepper x-chunk width: 0 = autotuned (measured once per wave size),
                            > 0 = fixed width (strips of at most 128 rows) */
    int freeSurface;     /* 1: free surface at the top interior row (reference par freeSurface;
                            the *FsGpu drivers); both steppers */
    int extension;       /* AIO_EXT_*: extension axis of the extended Born / tomo / WEMVA operators
                            (reference par extension "time" / "offset") */
} aio_params;

#define AIO_EXT_TIME 0      /* time lags (the *TimeShots* drivers) */
#define AIO_EXT_OFFSET 1    /* horizontal subsurface offsets (the *OffsetShots* drivers; per-fine-step stepper) */

#define AIO_STEPPER_AUTO 0      /* interval-blocked where available (sub == 4), else per fine step */
#define AIO_STEPPER_FINE 1      /* one fused launch per fine step (the reference's schedule) */
#define AIO_STEPPER_BLOCKED 2   /* one launch per coarse interval, 2-D register tiles (requires sub == 4) */

typedef struct {
    const int* sourcesPositionReg;   /* host array, nSourcesReg */
    int nSourcesReg;
    const int* receiversPositionReg; /* host array, nReceiversReg */
    int nReceiversReg;
    const float* sourcesSignals;     /* [nSourcesReg][ntw]: Born-family d2/dt2-scaled-interpolated
                                        wavelet; nonlinear forward: the model traces */
    float* data;                     /* [nReceiversReg][nts]: output (forward) / input (adjoint) */
    const float* wemvaData;          /* WEMVA only: [nReceiversReg][nts] data driving the receiver wavefield */
    float* sourcesOut;               /* nonlinear adjoint only: [nSourcesReg][ntw] output traces */
} aio_shot;

/* ---------------------------------------------------------------- batched API */
int aio_context_create(const aio_params* params, const float* vel2Dtw2, const float* reflectivityScale,
                       aio_context** out);
int aio_context_destroy(aio_context* ctx);
/* Replace the velocity-derived fields (reference setVel + fdParam precompute). */
int aio_context_set_velocity(aio_context* ctx, const float* vel2Dtw2, const float* reflectivityScale);
/* Device-memory budget for the context's shot buffers from now on (bytes; <= 0: 93 % of the
 * device's free memory, sampled now). A server that admits work by its own HBM budget hands each
 * context the bytes it reserved for that context's batch, so both plan with the same number. */
int aio_context_set_budget(aio_context* ctx, long long bytes);
/* Maximum number of shots one wave can hold for operator `family` under the memory budget. */
int aio_context_wave_capacity(aio_context* ctx, int family);
/* Number of stepper launches issued by the most recent operator call. */
long long aio_context_last_launches(aio_context* ctx);
const char* aio_last_error(void);
/* The CUDA stream (cudaStream_t) every kernel of this context runs on. */
void* aio_context_stream(aio_context* ctx);
/* Blocked-stepper plan for a wave of nShots shots (nShots <= 0: the plan of the most recent
 * blocked launch): plan[0..3] = strip rows, strips, chunk columns, chunks (the autotuned plan
 * once a Born source pass of that wave size has run). */
int aio_context_blocked_plan(aio_context* ctx, int nShots, int* plan);
/* Live stepper timing: bracket every sampleEvery-th stepper launch with CUDA events (0 = off). */
int aio_context_profile(aio_context* ctx, int sampleEvery);
/* Kernels launched, and timed-stepper totals (milliseconds, launches, interior
 * point-updates of those launches) since the last reset. */
int aio_context_stats(aio_context* ctx, long long* kernels, double* stepperMs, long long* stepperTimed,
                      double* stepperPoints);
int aio_context_reset_stats(aio_context* ctx);
/* Interval loops replayed from CUDA graphs since the context was created. A blocked pass's
 * per-interval launches run directly the first time a (plan, buffers) key is seen, are captured
 * into a CUDA graph the second time and replayed from it afterwards; AIO_GRAPHS=0 in the
 * environment (read at context creation) and live stepper timing (aio_context_profile) keep the
 * direct launches. */
long long aio_context_graph_replays(aio_context* ctx);
/* Device bytes the context holds: velocity constants plus its per-call buffers, which grow to the
 * largest wave the context has run and stay allocated between calls. */
long long aio_context_device_bytes(aio_context* ctx);
/* Frees the context's per-call buffers (the next call allocates them again) and its captured
 * CUDA graphs; waits for the context's stream first. For servers that plan the memory of many
 * contexts on one device. */
int aio_context_release_buffers(aio_context* ctx);

/* Nonlinear: model = source traces (sourcesSignals), data per shot. */
int aio_nonlinear_forward(aio_context* ctx, int nShots, const aio_shot* shots, int memSpace);
int aio_nonlinear_adjoint(aio_context* ctx, int nShots, const aio_shot* shots, int memSpace);
/* One shot with its coarse wavefield [nts][nx][nz] (host) written out: nonlinear forward
 * (F/src/nonlinearShotsGpuFunctions.cu:310-395, propShotsFwdGpuWavefield) and adjoint
 * (:653-739, propShotsAdjGpuWavefield; unscaled, the caller applies dtw^2 v^2). */
int aio_nonlinear_forward_wavefield(aio_context* ctx, const aio_shot* shot, int memSpace, float* wavefield);
int aio_nonlinear_adjoint_wavefield(aio_context* ctx, const aio_shot* shot, int memSpace, float* wavefield);
/* Born: model nz*nx (shared by all shots). adjoint: add=0 overwrites, add=1 accumulates. */
int aio_born_forward(aio_context* ctx, const float* model, int nShots, const aio_shot* shots, int memSpace);
int aio_born_adjoint(aio_context* ctx, float* model, int add, int nShots, const aio_shot* shots, int memSpace);
/* Born adjoint returning each shot's own image: images[s] (nz*nx, overwritten, host or device
 * per memSpace). The shots still run together; used to batch independent requests. */
int aio_born_adjoint_shots(aio_context* ctx, float* const* images, int nShots, const aio_shot* shots, int memSpace);
/* Born of one shot with its coarse wavefields, [nts][nx][nz] each with a zero FAT ring (the
 * reference's forwardWavefield / adjointWavefield, getSrcWfld / getSecWfld): forward returns the
 * source and scattered wavefields (F/src/BornShotsGpuFunctions.cu:390-535), adjoint the receiver
 * wavefield scaled by 2/v^3 v^2 dtw^2 (:959-1103) and, when srcWavefield is not NULL, the source
 * wavefield. Per-fine-step stepper. */
int aio_born_forward_wavefield(aio_context* ctx, const float* model, const aio_shot* shot, int memSpace,
                               float* srcWavefield, float* secWavefield);
int aio_born_adjoint_wavefield(aio_context* ctx, float* model, int add, const aio_shot* shot, int memSpace,
                               float* srcWavefield, float* recWavefield);
/* Extended Born of one shot with saved wavefields (the reference's *Wavefield drivers of
 * F/src/BornExtShotsGpuFunctions.cu, :420-580 forward, :1680-1847 adjoint): forward returns the
 * source and scattered wavefields; adjoint the receiver wavefield (time lags: scaled by
 * 2/v^3 v^2 dtw^2; offsets: by v^2 dtw^2) and, when srcWavefield is not NULL, the source
 * wavefield. Per-fine-step stepper; non-sloth time-lag scaling. */
int aio_born_ext_forward_wavefield(aio_context* ctx, const float* model, const aio_shot* shot, int memSpace,
                                   float* srcWavefield, float* secWavefield);
int aio_born_ext_adjoint_wavefield(aio_context* ctx, float* model, int add, const aio_shot* shot, int memSpace,
                                   float* srcWavefield, float* recWavefield);
/* Extended (time-lag) Born: model nExt*nz*nx. */
int aio_born_ext_forward(aio_context* ctx, const float* model, int nShots, const aio_shot* shots, int memSpace);
int aio_born_ext_adjoint(aio_context* ctx, float* model, int add, int nShots, const aio_shot* shots, int memSpace);
/* Extended tomo: model nz*nx, background extended reflectivity nExt*nz*nx. */
int aio_tomo_ext_forward(aio_context* ctx, const float* model, const float* extReflectivity, int nShots,
                         const aio_shot* shots, int memSpace);
int aio_tomo_ext_adjoint(aio_context* ctx, float* model, int add, const float* extReflectivity, int nShots,
                         const aio_shot* shots, int memSpace);
/* Extended WEMVA: model nz*nx, data = extended image nExt*nz*nx. */
int aio_wemva_ext_forward(aio_context* ctx, const float* model, float* image, int add, int nShots,
                          const aio_shot* shots, int memSpace);
int aio_wemva_ext_adjoint(aio_context* ctx, float* model, int add, const float* image, int nShots,
                          const aio_shot* shots, int memSpace);
/* Tomo and WEMVA of one shot with the saved wavefields of the reference's saveWavefield = 1
 * drivers, each [nts][nx][nz] with a zero FAT ring: srcDt2 = d2/dt2 of the source wavefield.
 * Tomo forward (F/src/tomoExtShotsGpuFunctions.cu:355-465): sec1 = the last leg's first
 * scattered wavefield, sec2 = its second (recorded) scattered wavefield. Tomo adjoint
 * (:797-910) and WEMVA forward / adjoint (F/src/wemvaExtShotsGpuFunctions.cu:344-456, :575-688):
 * sec1 = the receiver wavefield, sec2 = the coarse samples of the last leg's scattered
 * wavefield. Per-fine-step stepper, FP32 fields (wavefieldPrecision AIO_WFLD_FP32). */
int aio_tomo_ext_forward_wavefield(aio_context* ctx, const float* model, const float* extReflectivity,
                                   const aio_shot* shot, int memSpace, float* srcDt2, float* sec1, float* sec2);
int aio_tomo_ext_adjoint_wavefield(aio_context* ctx, float* model, int add, const float* extReflectivity,
                                   const aio_shot* shot, int memSpace, float* srcDt2, float* sec1, float* sec2);
int aio_wemva_ext_forward_wavefield(aio_context* ctx, const float* model, float* image, int add,
                                    const aio_shot* shot, int memSpace, float* srcDt2, float* sec1, float* sec2);
int aio_wemva_ext_adjoint_wavefield(aio_context* ctx, float* model, int add, const float* image,
                                    const aio_shot* shot, int memSpace, float* srcDt2, float* sec1, float* sec2);

/* ------------------------------------------------------------ host preparation
 * The reference's host-side numerics, FP32 expressions unchanged; arrays are
 * host memory. add=0 overwrites the output, add=1 accumulates.
 */
/* fdParam: v^2*dtw^2 and 2/v^3 over the padded grid (F/src/fdParam.cpp:124-139). Either output may be NULL. */
int aio_fd_precompute(int nz, int nx, float dts, int sub, const float* vel, float* vel2Dtw2, float* reflectivityScale);
/* interpTimeLinTbb forward / adjoint: coarse [nDev][nts] <-> fine [nDev][ntw] (F/src/interpTimeLinTbb.cpp:26-102). */
int aio_time_interp_forward(int add, int nts, float dts, float ots, int sub, int nDev, const float* coarse, float* fine);
int aio_time_interp_adjoint(int add, int nts, float dts, float ots, int sub, int nDev, float* coarse, const float* fine);
/* secondTimeDerivative forward (= adjoint), [nDev][nt] (F/src/secondTimeDerivative.cpp:14-39). */
int aio_second_time_derivative(int add, int nt, float dt, int nDev, const float* in, float* out);
/* seismicOperator2D::scaleSeismicSource: signal[k][:] *= dtw^2 v(pos[k])^2 (F/include/seismicOperator2D.cpp:72-86). */
int aio_scale_seismic_source(int nDevReg, const int* posReg, int nt, float dts, int sub, const float* vel, float* signal);
/* deviceGpu adjoint / forward on unique grid points (F/src/deviceGpu.cpp:227-261). */
int aio_device_spread(int add, int nDevIrreg, int nCorner, const int* cornerIdx, const float* weights, int nDevReg,
                      int nt, const float* irreg, float* reg);
int aio_device_gather(int add, int nDevIrreg, int nCorner, const int* cornerIdx, const float* weights, int nDevReg,
                      int nt, const float* reg, float* irreg);
/* seismicOperator2D::setSources chain: spread, [d2/dt2], dtw^2 v^2 scale, interpolate to fine time
 * (F/include/seismicOperator2D.cpp:10-39; secondDerivative=0 gives F/src/nonlinearPropGpu.cpp:44-51). */
int aio_prepare_source(int secondDerivative, int nDevIrreg, int nCorner, const int* cornerIdx, const float* weights,
                       int nDevReg, const int* posReg, int nts, float dts, int sub, const float* vel,
                       const float* wavelets, float* out);

/* -------------------------------------------------------------- reference seam
 * Each replaces the reference function of the same name without the prefix;
 * blockSize is accepted and ignored (the reference requires 16; tiles here are
 * fixed by the kernels). nGpu / iGpuAlloc are accepted for signature parity.
 */
/* F/include/nonlinearShotsGpuFunctions.h:7-24 */
int aio_initNonlinearGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize,
                         float alphaCos, int nGpu, int iGpuId, int iGpuAlloc);
int aio_allocateNonlinearGpu(float* vel2Dtw2, int iGpu, int iGpuId);
int aio_deallocateNonlinearGpu(int iGpu, int iGpuId);
int aio_propShotsFwdGpu(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                        int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId);
int aio_propShotsFwdGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                                 int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu,
                                 int iGpuId);
int aio_propShotsAdjGpu(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                        int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId);
int aio_propShotsAdjGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                                 int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu,
                                 int iGpuId);
/* F/include/BornShotsGpuFunctions.h:7-33 */
int aio_initBornGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize,
                    float alphaCos, int nGpu, int iGpuId, int iGpuAlloc);
int aio_allocateBornShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId);
int aio_deallocateBornShotsGpu(int iGpu, int iGpuId);
int aio_BornShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                        int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                        float* scatWavefield, int iGpu, int iGpuId);
int aio_BornShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                        int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                        float* recWavefield, int iGpu, int iGpuId);
/* F/include/BornShotsGpuFunctions.h:17 (coarse source and scattered wavefields out, [nts][nx][nz]) */
int aio_BornShotsFwdGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                 int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                                 float* scatWavefield, int iGpu, int iGpuId);
/* F/include/BornShotsGpuFunctions.h:29 (scaled coarse receiver wavefield out; srcWavefield untouched, as in
 * the reference) */
int aio_BornShotsAdjGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                 int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                                 float* recWavefield, int iGpu, int iGpuId);
/* F/include/BornExtShotsGpuFunctions.h:6-54 (time-lag extension) */
int aio_initBornExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize,
                       float alphaCos, int nExt, int nGpu, int iGpuId, int iGpuAlloc);
int aio_allocateBornExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId);
int aio_deallocateBornExtShotsGpu(int iGpu, int iGpuId);
int aio_BornTimeShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                            int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                            float* scatWavefield, int sloth, int iGpu, int iGpuId);
int aio_BornTimeShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                            int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                            float* recWavefield, int sloth, int iGpu, int iGpuId);
/* F/include/tomoExtShotsGpuFunctions.h:6-33 (time-lag extension). saveWavefield = 1 fills the three
 * wavefield arrays of the call as aio_tomo_ext_{forward,adjoint}_wavefield describe; the WEMVA
 * calls below do the same with aio_wemva_ext_{forward,adjoint}_wavefield's fields. */
int aio_initTomoExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize,
                       float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId, int iGpuAlloc);
int aio_allocateTomoExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId);
int aio_deallocateTomoExtShotsGpu(int iGpu, int iGpuId);
int aio_tomoTimeShotsFwdGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                            int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                            float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                            int sloth, int iGpu, int iGpuId, int saveWavefield);
int aio_tomoTimeShotsAdjGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                            int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                            float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                            int sloth, int iGpu, int iGpuId, int saveWavefield);
/* Free-surface drivers (reference freeSurface == 1): same arguments as the plain calls of the family,
 * with the top interior row as a pressure-free surface. */
/* F/include/nonlinearShotsGpuFunctions.h:15 */
int aio_propShotsFwdFsGpu(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                          int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId);
/* F/include/nonlinearShotsGpuFunctions.h:16 */
int aio_propShotsFwdFsGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                                   int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu,
                                   int iGpuId);
/* F/include/nonlinearShotsGpuFunctions.h:23 */
int aio_propShotsAdjFsGpu(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                          int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu, int iGpuId);
/* F/include/nonlinearShotsGpuFunctions.h:24 */
int aio_propShotsAdjFsGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sourcesPositionReg, int nSourcesReg,
                                   int* receiversPositionReg, int nReceiversReg, float* wavefieldDts, int iGpu,
                                   int iGpuId);
/* F/include/BornShotsGpuFunctions.h:20 */
int aio_BornShotsFwdFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                          int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                          float* scatWavefield, int iGpu, int iGpuId);
/* F/include/BornShotsGpuFunctions.h:32 */
int aio_BornShotsAdjFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                          int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                          float* recWavefield, int iGpu, int iGpuId);
/* F/include/BornExtShotsGpuFunctions.h:27 */
int aio_BornTimeShotsFwdFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                              int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                              float* scatWavefield, int iGpu, int iGpuId);
/* F/include/BornExtShotsGpuFunctions.h:49 */
int aio_BornTimeShotsAdjFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                              int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                              float* recWavefield, int iGpu, int iGpuId);
/* F/include/tomoExtShotsGpuFunctions.h:20 */
int aio_tomoTimeShotsFwdFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                              int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                              float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                              int iGpu, int iGpuId, int saveWavefield);
/* F/include/tomoExtShotsGpuFunctions.h:32 */
int aio_tomoTimeShotsAdjFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                              int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                              float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                              int iGpu, int iGpuId, int saveWavefield);
/* Subsurface-offset drivers (reference extension "offset"): same arguments as the time-lag calls without
 * sloth; they run on the per-fine-step stepper. */
/* F/include/BornExtShotsGpuFunctions.h:22 */
int aio_BornOffsetShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                              int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                              float* scatWavefield, int iGpu, int iGpuId);
/* F/include/BornExtShotsGpuFunctions.h:44 */
int aio_BornOffsetShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                              int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                              float* recWavefield, int iGpu, int iGpuId);
/* F/include/BornExtShotsGpuFunctions.h:31 */
int aio_BornOffsetShotsFwdFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                                float* scatWavefield, int iGpu, int iGpuId);
/* F/include/BornExtShotsGpuFunctions.h:53 */
int aio_BornOffsetShotsAdjFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                int nSourcesReg, int* receiversPositionReg, int nReceiversReg, float* srcWavefield,
                                float* recWavefield, int iGpu, int iGpuId);
/* Extended Born with saved wavefields, [nts][nx][nz] with a zero FAT ring (per-fine-step stepper; the
 * time-lag scaling is the non-sloth one, as in the reference's drivers). Forward: coarse source and
 * scattered wavefields; adjoint: coarse source wavefield and receiver wavefield (time lags: scaled by
 * 2/v^3 v^2 dtw^2; offsets: by v^2 dtw^2). F/include/BornExtShotsGpuFunctions.h:19, 23, 28, 32, 41, 45,
 * 50, 54 in the order below. */
int aio_BornTimeShotsFwdGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                     int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                     float* srcWavefield, float* scatWavefield, int iGpu, int iGpuId);
int aio_BornOffsetShotsFwdGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                       int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                       float* srcWavefield, float* scatWavefield, int iGpu, int iGpuId);
int aio_BornTimeShotsFwdFsGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                       int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                       float* srcWavefield, float* scatWavefield, int iGpu, int iGpuId);
int aio_BornOffsetShotsFwdFsGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals,
                                         int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg,
                                         int nReceiversReg, float* srcWavefield, float* scatWavefield, int iGpu,
                                         int iGpuId);
int aio_BornTimeShotsAdjGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                     int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                     float* srcWavefield, float* recWavefield, int iGpu, int iGpuId);
int aio_BornOffsetShotsAdjGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                       int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                       float* srcWavefield, float* recWavefield, int iGpu, int iGpuId);
int aio_BornTimeShotsAdjFsGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sourcesPositionReg,
                                       int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                       float* srcWavefield, float* recWavefield, int iGpu, int iGpuId);
int aio_BornOffsetShotsAdjFsGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals,
                                         int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg,
                                         int nReceiversReg, float* srcWavefield, float* recWavefield, int iGpu,
                                         int iGpuId);
/* F/include/tomoExtShotsGpuFunctions.h:17 */
int aio_tomoOffsetShotsFwdGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                              int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                              float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                              int iGpu, int iGpuId, int saveWavefield);
/* F/include/tomoExtShotsGpuFunctions.h:29 */
int aio_tomoOffsetShotsAdjGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                              int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                              float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                              int iGpu, int iGpuId, int saveWavefield);
/* F/include/tomoExtShotsGpuFunctions.h:21 */
int aio_tomoOffsetShotsFwdFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                                int iGpu, int iGpuId, int saveWavefield);
/* F/include/tomoExtShotsGpuFunctions.h:33 */
int aio_tomoOffsetShotsAdjFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                int* sourcesPositionReg, int nSourcesReg, int* receiversPositionReg, int nReceiversReg,
                                float* tomoSrcWavefieldDt2, float* tomoSecWavefield1, float* tomoSecWavefield2,
                                int iGpu, int iGpuId, int saveWavefield);
/* F/include/wemvaExtShotsGpuFunctions.h:13 */
int aio_wemvaOffsetShotsFwdGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sourcesPositionReg,
                               int nSourcesReg, float* wemvaDataRegDts, int* receiversPositionReg, int nReceiversReg,
                               float* wemvaSrcWavefieldDt2, float* wemvaSecWavefield1, float* wemvaSecWavefield2,
                               int iGpu, int iGpuId, int saveWavefield);
/* F/include/wemvaExtShotsGpuFunctions.h:17 */
int aio_wemvaOffsetShotsAdjGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sourcesPositionReg,
                               int nSourcesReg, float* wemvaDataRegDts, int* receiversPositionReg, int nReceiversReg,
                               float* wemvaSrcWavefieldDt2, float* wemvaSecWavefield1, float* wemvaSecWavefield2,
                               int iGpu, int iGpuId, int saveWavefield);
/* F/include/wemvaExtShotsGpuFunctions.h:6-17 (time-lag extension) */
int aio_initWemvaExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize,
                        float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId, int iGpuAlloc);
int aio_allocateWemvaExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId);
int aio_deallocateWemvaExtShotsGpu(int iGpu, int iGpuId);
int aio_wemvaTimeShotsFwdGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sourcesPositionReg,
                             int nSourcesReg, float* wemvaDataRegDts, int* receiversPositionReg, int nReceiversReg,
                             float* wemvaSrcWavefieldDt2, float* wemvaSecWavefield1, float* wemvaSecWavefield2,
                             int iGpu, int iGpuId, int saveWavefield);
int aio_wemvaTimeShotsAdjGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sourcesPositionReg,
                             int nSourcesReg, float* wemvaDataRegDts, int* receiversPositionReg, int nReceiversReg,
                             float* wemvaSrcWavefieldDt2, float* wemvaSecWavefield1, float* wemvaSecWavefield2,
                             int iGpu, int iGpuId, int saveWavefield);
/* Allocation-free nonlinear forward of one shot. No counterpart in the reference.
 * For callers that cannot let a library allocate device memory: services that
 * plan all device memory ahead and forbid allocation on the request path, and
 * hosts whose own allocator owns the device heap. Inputs and output are
 * device pointers (vel2Dtw2: nz*nx; modelRegDtw: [nSourcesReg][ntw]; dataRegDts:
 * [nReceiversReg][nts], overwritten); positions are host arrays; work is queued
 * on `stream` (a cudaStream_t, NULL = default stream) and not waited for.
 * Every temporary lives in one fixed 48 MiB __device__ array that each GPU
 * loading the library holds until exit; grids needing more return
 * AIO_ERR_ARGUMENT. The first call on a device looks up that array's device
 * address (make it before any stream capture). All calls share the array:
 * calls whose GPU work overlaps race and must be serialised by the caller.
 * Errors are returned as codes and described on stderr. */
int aio_propShotsFwdGpu_noalloc(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad,
                                float alphaCos, const float* vel2Dtw2, const float* modelRegDtw,
                                const int* sourcesPositionReg, int nSourcesReg, const int* receiversPositionReg,
                                int nReceiversReg, float* dataRegDts, void* stream);
/* FP64 inner product sum(a[i]*b[i]) of two FP32 arrays of n elements, reduced on GPU `device`
 * (host arrays are copied there first when memSpace is AIO_MEM_HOST): the reduction of the
 * dot-product test, F/include/operator.h:50-88 (which takes SEP vector dot products). Products are
 * exact in FP64 and summed in a fixed order, so the result is reproducible. */
int aio_dot_f64(int device, int memSpace, long long n, const float* a, const float* b, double* result);
/* F/src/nonlinearShotsGpuFunctions.cu:18-84: validates a GPU id list (info printing dropped). */
int aio_getGpuInfo(const int* gpuList, int nGpuList, int info, int deviceNumberInfo);

#ifdef __cplusplus
}
#endif
#endif /* AIO_B200_H */
