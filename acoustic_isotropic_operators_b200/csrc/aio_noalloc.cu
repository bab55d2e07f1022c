// Allocation-free nonlinear forward propagation of one shot.
//
// Some callers cannot let a library allocate device memory: services that
// pre-plan every byte of device memory up front and forbid allocations on the
// request path (an allocation there can stall on the device or fail under
// fragmentation), and hosts whose own allocator owns the device heap (a second
// allocator beside it would take memory it has already counted as free). This
// entry point serves them: the caller passes its inputs
// and output as device pointers and a stream, and every temporary the stepper
// needs (the two fine time levels, the interior copy of v^2 dtw^2, the damping
// table, the shot descriptor and the sparse device lists) lives in one
// file-scope __device__ array of fixed size. Nothing here calls cudaMalloc,
// cudaFree or any other allocating routine.
//
// The kernel is the engine's fused stepper (aio_kernels.cuh) instantiated for
// the nonlinear forward pass: stencil + source injection + damping + receiver
// recording per fine step, the pass sequence of the reference's
// propShotsFwdGpu.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "aio_b200.h"

// The engine's kernels, given internal linkage in this translation unit so the
// library links them once per unit without symbol clashes.
namespace {
#include "aio_kernels.cuh"
}

// Fixed scratch: 48 MiB. Every GPU that loads this library holds it until exit.
// In host code `g_scratch` is only a stand-in for the symbol, not a device
// address: the address comes from cudaGetSymbolAddress below.
static constexpr size_t kScratchBytes = size_t(48) << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

namespace {
namespace noalloc {
using namespace aio;

constexpr int kMaxDevices = 64;
static void* g_scratchAddr[kMaxDevices] = {};  // device address of g_scratch per device
static std::mutex g_mu;

// Host-side staging for the sparse lists and the descriptor (static: no heap).
constexpr int kMaxListWords = 1 << 20;
static int g_words[kMaxListWords];
static int g_tileCount[kMaxListWords];

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Sparse CSR over stepper tiles written into words[off...]; returns words used or -1.
static long long build_list(const Geom& g, const int* pos, int n, int* words, long long off, long long cap) {
    const int nT = g.tilesZ * g.tilesX;
    const int startWords = (nT + 1 + 1) & ~1;
    if (off + startWords + 2LL * n > cap || nT + 1 > kMaxListWords) return -1;
    int* start = words + off;
    int* ent = start + startWords;
    for (int t = 0; t <= nT; t++) g_tileCount[t] = 0;
    for (int k = 0; k < n; k++) {
        const long long p = pos[k];
        const int iz = (int)(p % g.nz), ix = (int)(p / g.nz);
        if (p < 0 || ix >= g.nx || iz < FAT || iz >= g.nz - FAT || ix < FAT || ix >= g.nx - FAT) return -2;
        const int z = iz - FAT, x = ix - FAT;
        g_tileCount[(x / TX) * g.tilesZ + z / TZ + 1]++;
    }
    for (int t = 0; t < nT; t++) g_tileCount[t + 1] += g_tileCount[t];
    for (int t = 0; t <= nT; t++) start[t] = g_tileCount[t];
    for (int k = 0; k < n; k++) {
        const long long p = pos[k];
        const int z = (int)(p % g.nz) - FAT, x = (int)(p / g.nz) - FAT;
        const int tile = (x / TX) * g.tilesZ + z / TZ;
        const int slot = g_tileCount[tile]++;
        ent[2 * slot] = (x % TX) * TZ + (z % TZ);
        ent[2 * slot + 1] = k;
    }
    return startWords + 2LL * n;
}

// Errors are reported on stderr (no allocation) and through the return code.
static int fail(int code, const char* msg, unsigned long long a = 0, unsigned long long b = 0) {
    std::fprintf(stderr, "aio_propShotsFwdGpu_noalloc: ");
    std::fprintf(stderr, msg, a, b);
    std::fprintf(stderr, "\n");
    return code;
}

}  // namespace noalloc
}  // namespace

using namespace aio;
using namespace noalloc;

extern "C" __attribute__((visibility("default"))) int aio_propShotsFwdGpu_noalloc(
    float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, float alphaCos,
    const float* vel2Dtw2, const float* modelRegDtw, const int* sourcesPositionReg, int nSourcesReg,
    const int* receiversPositionReg, int nReceiversReg, float* dataRegDts, void* stream) {
    if (nz <= 2 * FAT || nx <= 2 * FAT || nts < 2 || sub < 1 || sub >= SUB_MAX || minPad < 0 || minPad >= PAD_MAX)
        return fail(AIO_ERR_ARGUMENT, "invalid grid / time parameters");
    if (!vel2Dtw2 || !dataRegDts || (nSourcesReg > 0 && (!modelRegDtw || !sourcesPositionReg)) ||
        (nReceiversReg > 0 && !receiversPositionReg) || nSourcesReg < 0 || nReceiversReg < 0)
        return fail(AIO_ERR_ARGUMENT, "null input / output pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const Geom g = make_geom(nz, nx, nts, sub, minPad, 1);

    // Scratch layout: descriptor | taper | v2 (interior slice) | two halo slices | device lists.
    const size_t offDesc = 0;
    const size_t offTaper = align256(offDesc + sizeof(ShotDesc));
    const size_t offV2 = align256(offTaper + PAD_MAX * sizeof(float));
    const size_t offP = align256(offV2 + (size_t)g.isz * sizeof(float));
    const size_t offLists = align256(offP + 2 * (size_t)g.hsz * sizeof(float));
    const int nT = g.tilesZ * g.tilesX;
    const long long listWords = 2LL * (((nT + 2) & ~1) + 0) + 2LL * ((long long)nSourcesReg + nReceiversReg);
    const size_t need = align256(offLists + (size_t)listWords * sizeof(int));
    if (need > kScratchBytes)
        return fail(AIO_ERR_ARGUMENT, "grid needs %llu bytes of scratch; the fixed maximum is %llu bytes (48 MiB)",
                    (unsigned long long)need, (unsigned long long)kScratchBytes);

    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return fail(AIO_ERR_CUDA, "no usable current device");
    // One-time set-up per device, with that device current: the scratch array's
    // device address (the host-side symbol is not a device address).
    if (!g_scratchAddr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) return fail(AIO_ERR_CUDA, "cudaGetSymbolAddress failed (error %llu)", e);
        g_scratchAddr[dev] = p;
    }
    unsigned char* base = (unsigned char*)g_scratchAddr[dev];
    ShotDesc* dDesc = (ShotDesc*)(base + offDesc);
    float* dTaper = (float*)(base + offTaper);
    float* dV2 = (float*)(base + offV2);
    float* dP = (float*)(base + offP);
    int* dLists = (int*)(base + offLists);

    // Scheme constants with the reference's FP32 expressions
    // (F/src/nonlinearShotsGpuFunctions.cu:123-170).
    Coefs cf;
    static const double C[6] = {-2.927222222, 1.666666667, -0.238095238, 0.039682539, -0.004960317, 0.000317460};
    for (int i = 0; i < 6; i++) {
        cf.zc[i] = (float)(C[i] / (double)(dz * dz));
        cf.xc[i] = (float)(C[i] / (double)(dx * dx));
    }
    const int ntw = g.ntw, H = g.H;
    float h[2 * (SUB_MAX + 1)] = {};
    const float r = std::sqrt((float)ntw / (float)nts);
    const double sc = 1.0 / (double)r;
    for (int i = 0; i < H; i++) {
        h[i] = (float)(1.0 - 1.0 * i / sub);
        h[i + H] = (float)(1.0 - (double)h[i]);
        h[i] = (float)((double)h[i] * sc);
        h[i + H] = (float)((double)h[i + H] * sc);
    }
    static float taper[PAD_MAX];
    for (int i = 0; i < PAD_MAX; i++) taper[i] = 1.f;
    for (int i = 0; i < minPad; i++) {
        const float a = (float)(M_PI / (1.0 * minPad) * 1.0 * (minPad - i));
        taper[i] = (float)((double)alphaCos + (1.0 - (double)alphaCos) * (double)std::cos(a));
    }

    // Sparse lists (sources inject, receivers record).
    long long off = 0;
    const long long ws = build_list(g, sourcesPositionReg, nSourcesReg, g_words, off, kMaxListWords);
    if (ws < 0) return fail(AIO_ERR_ARGUMENT, "a source position lies outside the interior grid");
    const long long srcOff = off;
    off += ws;
    const long long wr = build_list(g, receiversPositionReg, nReceiversReg, g_words, off, kMaxListWords);
    if (wr < 0) return fail(AIO_ERR_ARGUMENT, "a receiver position lies outside the interior grid");
    const long long recOff = off;
    off += wr;
    const int startWords = (nT + 1 + 1) & ~1;

    ShotDesc d;
    std::memset(&d, 0, sizeof(d));
    d.p[0] = dP;
    d.p[1] = dP + g.hsz;
    d.inj = nSourcesReg > 0 ? SparseList{dLists + srcOff, (const int2*)(dLists + srcOff + startWords)}
                            : SparseList{nullptr, nullptr};
    d.injSig = modelRegDtw;
    d.injLd = ntw;
    d.rec = nReceiversReg > 0 ? SparseList{dLists + recOff, (const int2*)(dLists + recOff + startWords)}
                              : SparseList{nullptr, nullptr};
    d.recSig = dataRegDts;
    d.recLd = nts;

#define NA_CK(x)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) return fail(AIO_ERR_CUDA, "CUDA error %llu at line %llu", e_, __LINE__); \
    } while (0)
    // The scratch keeps the previous call's contents: clear what must start at zero.
    NA_CK(cudaMemsetAsync(dP, 0, 2 * (size_t)g.hsz * sizeof(float), st));
    NA_CK(cudaMemsetAsync(dV2, 0, (size_t)g.isz * sizeof(float), st));
    NA_CK(cudaMemsetAsync(dataRegDts, 0, (size_t)nReceiversReg * nts * sizeof(float), st));
    NA_CK(cudaMemcpy2DAsync(dV2, (size_t)g.ip * 4, vel2Dtw2 + (long long)FAT * nz + FAT, (size_t)nz * 4,
                            (size_t)g.nzi * 4, g.nxi, cudaMemcpyDeviceToDevice, st));
    NA_CK(cudaMemcpyAsync(dTaper, taper, PAD_MAX * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(dDesc, &d, sizeof(d), cudaMemcpyHostToDevice, st));
    if (off > 0) NA_CK(cudaMemcpyAsync(dLists, g_words, (size_t)off * sizeof(int), cudaMemcpyHostToDevice, st));

    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = g;
    a.c = cf;
    a.v2 = dV2;
    a.taper = dTaper;
    a.shots = dDesc;
    a.injTB = -1;
    dim3 grid(g.tilesZ, g.tilesX, 1), block(TZ, TY);
    int parity = 0;
    for (int its = 0; its < nts - 1; its++)
        for (int it2 = 1; it2 < sub + 1; it2++) {
            a.parity = parity;
            a.injTA = its * sub + it2 - 1;
            a.recTA = its;
            a.recTB = its + 1;
            a.recCA = h[it2];
            a.recCB = h[H + it2];
            k_step<false, 1, true, false><<<grid, block, 0, st>>>(a);
            NA_CK(cudaGetLastError());
            parity ^= 1;
        }
#undef NA_CK
    return AIO_OK;
}
