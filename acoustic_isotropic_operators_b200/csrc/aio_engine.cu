// B200 engine for the 2-D acoustic isotropic operators: operator contexts,
// batched pass drivers and the C ABI declared in include/aio_b200.h.
//
// A context owns the velocity-derived fields of one operator instance and
// reusable per-wave buffers. An operator call splits its shots into waves that
// fit the device-memory budget; inside a wave every shot advances together,
// one fused stepper launch per fine step (gridDim.z = shot), one element-wise
// launch per coarse step for imaging. The pass sequences follow the reference
// drivers (F/src/*ShotsGpuFunctions.cu), cited at each pass.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "aio_b200.h"
#include "aio_kernels.cuh"
#include "aio_tile.cuh"

namespace aio {

static thread_local std::string g_err;

struct Error {
    int code;
    std::string msg;
};

#define AIO_CK(x)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess)                                                                      \
            throw Error{AIO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_) + " (line " + \
                                          std::to_string(__LINE__) + ")"};                          \
    } while (0)

static void require(bool ok, const std::string& msg) {
    if (!ok) throw Error{AIO_ERR_ARGUMENT, msg};
}

template <class F>
static int guard(F&& f) {
    try {
        f();
        return AIO_OK;
    } catch (const Error& e) {
        g_err = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return AIO_ERR_ARGUMENT;
    }
}

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t b) {
        if (b <= bytes) return;
        release();
        if (b == 0) return;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            bytes = 0;
            throw Error{AIO_ERR_MEMORY, "cudaMalloc of " + std::to_string(b) + " bytes failed"};
        }
        bytes = b;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    ~DevMem() { release(); }
    template <class T>
    T* as() const { return (T*)p; }
};

// Host copies of the scheme constants, computed with the reference's own
// expressions and FP32 rounding (F/src/nonlinearShotsGpuFunctions.cu:123-170,
// F/src/tomoExtShotsGpuFunctions.cu:138-139).
struct HostConsts {
    Coefs c;
    float h[2 * (SUB_MAX + 1)];
    float taper[PAD_MAX];
    float cSide, cCenter;
};

static HostConsts make_consts(const aio_params& P) {
    HostConsts k;
    static const double C[6] = {-2.927222222, 1.666666667, -0.238095238, 0.039682539, -0.004960317, 0.000317460};
    for (int i = 0; i < 6; i++) {
        k.c.zc[i] = (float)(C[i] / (double)(P.dz * P.dz));
        k.c.xc[i] = (float)(C[i] / (double)(P.dx * P.dx));
    }
    const int ntw = (P.nts - 1) * P.sub + 1, H = P.sub + 1;
    std::fill(k.h, k.h + 2 * (SUB_MAX + 1), 0.f);
    const float r = std::sqrt((float)ntw / (float)P.nts);
    const double sc = 1.0 / (double)r;
    for (int i = 0; i < H; i++) {
        k.h[i] = (float)(1.0 - 1.0 * i / P.sub);
        k.h[i + H] = (float)(1.0 - (double)k.h[i]);
        k.h[i] = (float)((double)k.h[i] * sc);
        k.h[i + H] = (float)((double)k.h[i + H] * sc);
    }
    std::fill(k.taper, k.taper + PAD_MAX, 1.f);
    for (int i = 0; i < P.minPad; i++) {
        const float a = (float)(M_PI / (1.0 * P.minPad) * 1.0 * (P.minPad - i));
        const float cs = std::cos(a);
        k.taper[i] = (float)((double)P.alphaCos + (1.0 - (double)P.alphaCos) * (double)cs);
    }
    k.cSide = (float)(1.0 / (double)(P.dts * P.dts));
    k.cCenter = (float)(-2.0 / (double)(P.dts * P.dts));
    return k;
}

// Sparse device lists of one wave: per shot a CSR over stepper tiles.
struct WaveLists {
    std::vector<int> words;             // concatenated [start (nT+1, padded even)] [entries int2]
    std::vector<long long> srcOff, recOff;  // word offsets of each shot's src / rec list (-1: empty)
};

static void append_list(const Geom& g, const int* pos, int n, std::vector<int>& words, long long& off,
                        const char* what) {
    if (n <= 0 || !pos) {
        off = -1;
        return;
    }
    const int nT = g.tilesZ * g.tilesX;
    std::vector<int> tileOf(n), local(n), cnt(nT + 1, 0);
    for (int k = 0; k < n; k++) {
        const long long p = pos[k];
        const int iz = (int)(p % g.nz), ix = (int)(p / g.nz);
        require(p >= 0 && ix < g.nx && iz >= FAT && iz < g.nz - FAT && ix >= FAT && ix < g.nx - FAT,
                std::string(what) + " position " + std::to_string(p) + " is outside the interior grid");
        const int z = iz - FAT, x = ix - FAT;
        tileOf[k] = (x / TX) * g.tilesZ + z / TZ;
        local[k] = (x % TX) * TZ + (z % TZ);
        cnt[tileOf[k] + 1]++;
    }
    for (int t = 0; t < nT; t++) cnt[t + 1] += cnt[t];
    const int startWords = (nT + 1 + 1) & ~1;  // keep the entries 8-byte aligned
    off = (long long)words.size();
    words.resize(words.size() + startWords + 2 * (size_t)n, 0);
    int* start = words.data() + off;
    for (int t = 0; t <= nT; t++) start[t] = cnt[t];
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    int* ent = start + startWords;
    for (int k = 0; k < n; k++) {
        const int slot = fill[tileOf[k]]++;
        ent[2 * slot] = local[k];
        ent[2 * slot + 1] = k;
    }
}

enum AccMode { ACC_NONE = 0, ACC_FULL = 1, ACC_RING = 2 };

struct Context {
    aio_params P;
    Geom g;
    HostConsts k;
    int dev = 0;
    int smCount = 148;  // streaming multiprocessors of `dev`
    cudaStream_t st = nullptr;
    DevMem v2, rs, taper;
    // per-wave buffers
    DevMem pbuf, ringb, ssb, wf1, wf2, wf3, img, lists, desc, sig, dat, aux, model, ext, outv;
    std::vector<ShotDesc> hdesc;
    long long launches = 0;      // stepper launches of the last operator call
    long long kernels = 0;       // every kernel launched since the last stats reset
    long long budget = 0;
    // Live stepper timing: every profEvery-th stepper launch is bracketed by a
    // pair of CUDA events on the engine stream; pairs are read back at sync().
    int profEvery = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evFree, evBusy;
    std::vector<long long> evPoints;   // interior points advanced by each timed launch
    double stepMs = 0.0;
    long long stepTimed = 0;
    double stepPoints = 0.0;

    // ------------------------------------------------------------- set-up
    void init(const aio_params& p, const float* vel2Dtw2, const float* reflScale) {
        P = p;
        require(p.nz > 2 * FAT && p.nx > 2 * FAT, "nz and nx must exceed 2*FAT");
        require(p.nts >= 2, "nts must be >= 2");
        require(p.sub >= 1 && p.sub < SUB_MAX, "sub must be in [1, 100)");
        require(p.minPad >= 0 && p.minPad < PAD_MAX, "minPad must be in [0, 200)");
        require(p.nExt >= 1 && (p.nExt % 2) == 1, "nExt must be a positive odd number");
        require(p.wavefieldPrecision == AIO_WFLD_FP32 || p.wavefieldPrecision == AIO_WFLD_BF16 ||
                    p.wavefieldPrecision == AIO_WFLD_FP16,
                "stored wavefield precision must be AIO_WFLD_FP32, AIO_WFLD_BF16 or AIO_WFLD_FP16");
        require(p.stepper >= AIO_STEPPER_AUTO && p.stepper <= AIO_STEPPER_BLOCKED, "unknown stepper");
        require(p.stepper < AIO_STEPPER_BLOCKED || p.sub == 4, "the interval-blocked steppers require sub == 4");
        require(p.freeSurface == 0 || p.freeSurface == 1, "freeSurface must be 0 or 1");
        require(p.extension == AIO_EXT_TIME || p.extension == AIO_EXT_OFFSET,
                "extension must be AIO_EXT_TIME or AIO_EXT_OFFSET");
        require(p.extension != AIO_EXT_OFFSET || 2 * ((p.nExt - 1) / 2) < p.nx - 2 * FAT,
                "subsurface offsets longer than the interior width");
        require(p.wavefieldPrecision == AIO_WFLD_FP32 || (p.stepper != AIO_STEPPER_FINE && p.sub == 4),
                "compressed stored wavefields need the interval-blocked stepper (sub == 4)");
        g = make_geom(p.nz, p.nx, p.nts, p.sub, p.minPad, p.nExt);
        k = make_consts(p);
        // the blocked stepper evaluates taper[min(a, b)] as min(taper[a], taper[b])
        for (int i = 1; i < p.minPad; i++)
            require(k.taper[i] >= k.taper[i - 1] && k.taper[i] <= 1.f, "cosine taper must be monotone and <= 1");
        dev = p.device;
        AIO_CK(cudaSetDevice(dev));
        AIO_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        AIO_CK(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, dev));
        v2.ensure(g.isz * 4);
        rs.ensure(g.isz * 4);
        taper.ensure(PAD_MAX * 4);
        AIO_CK(cudaMemcpyAsync(taper.p, k.taper, PAD_MAX * 4, cudaMemcpyHostToDevice, st));
        set_velocity(vel2Dtw2, reflScale);
        size_t fr = 0, tot = 0;
        AIO_CK(cudaMemGetInfo(&fr, &tot));
        budget = p.memBudgetBytes > 0 ? p.memBudgetBytes : (long long)(0.93 * (double)fr);
        const char* gEnv = std::getenv("AIO_GRAPHS");  // AIO_GRAPHS=0: launch every interval directly
        graphsOn = !(gEnv && gEnv[0] == '0');
        // AIO_PDL=0: no programmatic dependent launches; 1: the next launch may start as soon as
        // every CTA has passed its dependency wait; 2: once every CTA has begun its last iteration
        const char* pEnv = std::getenv("AIO_PDL");
        if (pEnv && pEnv[0] >= '0' && pEnv[0] <= '2') pdlMode = pEnv[0] - '0';
        live_contexts()[dev & 63]++;
        counted = true;
    }
    // contexts alive per device (process-wide): the launch overlap policy depends on it
    static std::atomic<int>* live_contexts() {
        static std::atomic<int> n[64];
        return n;
    }
    bool counted = false;
    // Effective overlap mode of this context's stepper launches. Alone on its device, a launch
    // lets the next one start right after its dependency wait (the next launch's CTAs fill the SMs
    // its own leave free and finish their prologue early). Beside other contexts, whose streams
    // run kernels at the same time, CTAs waiting that long would hold SM resources those kernels
    // could use, so the release moves to the last iteration.
    int pdl_mode() const {
        if (pdlMode != 3) return pdlMode;
        return live_contexts()[dev & 63].load() > 1 ? 2 : 1;
    }

    void set_velocity(const float* vel2Dtw2, const float* reflScale) {
        AIO_CK(cudaSetDevice(dev));
        AIO_CK(cudaMemsetAsync(v2.p, 0, g.isz * 4, st));
        AIO_CK(cudaMemsetAsync(rs.p, 0, g.isz * 4, st));
        if (vel2Dtw2) to_interior(v2.as<float>(), vel2Dtw2, 1, AIO_MEM_HOST);
        if (reflScale) to_interior(rs.as<float>(), reflScale, 1, AIO_MEM_HOST);
        AIO_CK(cudaStreamSynchronize(st));
    }

    void destroy() {
        if (counted) live_contexts()[dev & 63]--;
        counted = false;
        drop_graphs();
        for (auto& e : evFree) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
        for (auto& e : evBusy) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
        evFree.clear();
        evBusy.clear();
        if (st) cudaStreamDestroy(st);
        st = nullptr;
    }
    void kcheck() {
        AIO_CK(cudaGetLastError());
        kernels++;
    }

    // ------------------------------------------------------------- graph-captured time loops
    // A pass's per-interval launches (one blocked-stepper launch per coarse interval, ~2000 per
    // pass) are a fixed sequence once the pass's key is fixed: plan, entry capacity and the device
    // addresses baked into the launch arguments (descriptors, stored wavefield, model). The first
    // run of a key launches directly; the second is captured into a CUDA graph, which this and
    // every later run with the same key replay with one cudaGraphLaunch. Off while live stepper
    // timing brackets single launches with events, and with AIO_GRAPHS=0.
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        long long launches = 0, kernels = 0;
    };
    std::map<std::vector<long long>, GraphEntry> graphs;
    std::map<std::vector<long long>, int> graphRuns;
    bool graphsOn = true;
    // blocked-stepper launches may start their prologue (ring zeroing, tables, entries) while the
    // previous launch of the stream still runs; the kernel waits for it before reading its output
    int pdlMode = 3;  // 0 off, 1 early release, 2 release at the last iteration, 3 by live contexts
    long long graphReplays = 0;

    void drop_graphs() {
        for (auto& e : graphs)
            if (e.second.exec) cudaGraphExecDestroy(e.second.exec);
        graphs.clear();
        graphRuns.clear();
    }
    // key: the pass's own fields; the settings that select kernel variants (free surface,
    // stored precision) are appended here so no pass can replay another variant's graph
    template <class Body>
    void graph_loop(std::vector<long long> key, Body&& body) {
        if (!graphsOn || profEvery > 0) {
            body();
            return;
        }
        key.insert(key.end(), {P.freeSurface, P.wavefieldPrecision, P.extension, P.sloth, P.stepper, pdl_mode()});
        auto it = graphs.find(key);
        if (it != graphs.end()) {
            AIO_CK(cudaGraphLaunch(it->second.exec, st));
            launches += it->second.launches;
            kernels += it->second.kernels;
            graphReplays++;
            return;
        }
        if (graphRuns[key]++ == 0) {  // first run: direct launches (also sets kernel attributes)
            body();
            return;
        }
        if (graphs.size() >= 64) drop_graphs();
        const long long l0 = launches, k0 = kernels;
        AIO_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t gph = nullptr;
        try {
            body();
        } catch (...) {
            cudaStreamEndCapture(st, &gph);
            if (gph) cudaGraphDestroy(gph);
            throw;
        }
        AIO_CK(cudaStreamEndCapture(st, &gph));
        cudaGraphExec_t ex = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ex, gph, 0);
        cudaGraphDestroy(gph);
        AIO_CK(e);
        graphs[key] = GraphEntry{ex, launches - l0, kernels - k0};
        AIO_CK(cudaGraphLaunch(ex, st));
    }

    // full nz*nx (per slice) <-> interior pitched slices
    void to_interior(float* dst, const float* src, int nSlices, int mem) {
        const cudaMemcpyKind kind = mem == AIO_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        for (int e = 0; e < nSlices; e++)
            AIO_CK(cudaMemcpy2DAsync(dst + (long long)e * g.isz, (size_t)g.ip * 4,
                                     src + (long long)e * g.nz * g.nx + (long long)FAT * g.nz + FAT, (size_t)g.nz * 4,
                                     (size_t)g.nzi * 4, g.nxi, kind, st));
    }
    void from_interior(float* dst, const float* src, int nSlices, int mem) {
        const cudaMemcpyKind kind = mem == AIO_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        for (int e = 0; e < nSlices; e++)
            AIO_CK(cudaMemcpy2DAsync(dst + (long long)e * g.nz * g.nx + (long long)FAT * g.nz + FAT, (size_t)g.nz * 4,
                                     src + (long long)e * g.isz, (size_t)g.ip * 4, (size_t)g.nzi * 4, g.nxi, kind, st));
    }

    // ------------------------------------------------------------- waves
    struct Needs {
        int nWavefields = 0;  // full coarse wavefields per shot (FP32)
        int nImg = 0;         // per-shot image slices
        bool ss = false;
    };

    long long per_shot_bytes(const Needs& n, int maxSrc, int maxRec) const {
        long long b = 2 * g.hsz * 4 + 2 * g.isz * 4;  // fine levels + accumulation ring
        if (n.ss) b += 2 * g.isz * 4;
        b += (long long)n.nWavefields * g.nts * g.isz * 4;
        b += (long long)n.nImg * g.isz * (P.imageFp64 ? 8 : 4);
        if (offsets()) b += (long long)OFF_K * g.isz * 4;  // block of ring samples (img_offset_adj_block)
        b += (long long)maxSrc * g.ntw * 4 + 2LL * maxRec * g.nts * 4;
        b += 16LL * (g.tilesZ * g.tilesX + 2) + 16LL * (maxSrc + maxRec);
        return b;
    }

    int capacity(const Needs& n, int maxSrc, int maxRec) const {
        long long shared = 2 * g.isz * 4 + (long long)g.nExt * g.isz * 4 * 2 + (long long)g.nExt * g.isz * 8;
        long long avail = budget - shared;
        long long per = per_shot_bytes(n, maxSrc, maxRec);
        long long c = avail / per;
        return (int)std::max(0LL, std::min(c, 4096LL));
    }

    int wave_size(const Needs& n, int nShots, const aio_shot* shots) {
        int maxSrc = 1, maxRec = 1;
        for (int s = 0; s < nShots; s++) {
            maxSrc = std::max(maxSrc, shots[s].nSourcesReg);
            maxRec = std::max(maxRec, shots[s].nReceiversReg);
        }
        int cap = capacity(n, maxSrc, maxRec);
        require(cap >= 1, "device memory budget cannot hold one shot for this operator");
        return balanced_wave(cap, nShots);
    }
    // Waves of (nearly) equal size: ceil(nShots / cap) waves rather than full waves and a
    // small remainder, whose launches would use the GPU poorly.
    static int balanced_wave(long long cap, int nShots) {
        if (nShots <= cap) return nShots;
        const long long waves = (nShots + cap - 1) / cap;
        return (int)((nShots + waves - 1) / waves);
    }

    // Allocate wave buffers for nb shots and fill descriptors; traces are staged
    // (host mode) or referenced in place (device mode).
    void setup_wave(const Needs& n, int nb, const aio_shot* shots, int mem, bool dataIsInput, bool needWemvaData) {
        int maxSrc = 1, maxRec = 1;
        for (int s = 0; s < nb; s++) {
            maxSrc = std::max(maxSrc, shots[s].nSourcesReg);
            maxRec = std::max(maxRec, shots[s].nReceiversReg);
        }
        pbuf.ensure((size_t)nb * 2 * g.hsz * 4);
        ringb.ensure((size_t)nb * 2 * g.isz * 4);
        if (n.ss) ssb.ensure((size_t)nb * 2 * g.isz * 4);
        if (n.nWavefields >= 1) wf1.ensure((size_t)nb * g.nts * g.isz * 4);
        if (n.nWavefields >= 2) wf2.ensure((size_t)nb * g.nts * g.isz * 4);
        if (n.nWavefields >= 3) wf3.ensure((size_t)nb * g.nts * g.isz * 4);
        if (n.nImg) img.ensure((size_t)nb * n.nImg * g.isz * (P.imageFp64 ? 8 : 4));
        AIO_CK(cudaMemsetAsync(pbuf.p, 0, (size_t)nb * 2 * g.hsz * 4, st));
        AIO_CK(cudaMemsetAsync(ringb.p, 0, (size_t)nb * 2 * g.isz * 4, st));

        WaveLists L;
        L.srcOff.resize(nb);
        L.recOff.resize(nb);
        for (int s = 0; s < nb; s++) {
            append_list(g, shots[s].sourcesPositionReg, shots[s].nSourcesReg, L.words, L.srcOff[s], "source");
            append_list(g, shots[s].receiversPositionReg, shots[s].nReceiversReg, L.words, L.recOff[s], "receiver");
        }
        lists.ensure(std::max<size_t>(L.words.size(), 2) * 4);
        if (!L.words.empty())
            AIO_CK(cudaMemcpyAsync(lists.p, L.words.data(), L.words.size() * 4, cudaMemcpyHostToDevice, st));

        if (mem == AIO_MEM_HOST) {
            sig.ensure((size_t)nb * maxSrc * g.ntw * 4);
            dat.ensure((size_t)nb * maxRec * g.nts * 4);
            if (needWemvaData) aux.ensure((size_t)nb * maxRec * g.nts * 4);
        }
        hdesc.assign(nb, ShotDesc{});
        const int nT = g.tilesZ * g.tilesX;
        const int startWords = (nT + 1 + 1) & ~1;
        srcLists.assign(nb, SparseList{nullptr, nullptr});
        recLists.assign(nb, SparseList{nullptr, nullptr});
        srcSig.assign(nb, nullptr);
        dataPtr.assign(nb, nullptr);
        wdataPtr.assign(nb, nullptr);
        for (int s = 0; s < nb; s++) {
            ShotDesc& d = hdesc[s];
            d.p[0] = pbuf.as<float>() + (long long)s * 2 * g.hsz;
            d.p[1] = d.p[0] + g.hsz;
            d.ss = n.ss ? ssb.as<float>() + (long long)s * 2 * g.isz : nullptr;
            d.acc = ringb.as<float>() + (long long)s * 2 * g.isz;
            if (L.srcOff[s] >= 0) {
                const int* base = lists.as<int>() + L.srcOff[s];
                srcLists[s] = SparseList{base, (const int2*)(base + startWords)};
            }
            if (L.recOff[s] >= 0) {
                const int* base = lists.as<int>() + L.recOff[s];
                recLists[s] = SparseList{base, (const int2*)(base + startWords)};
            }
            const aio_shot& sh = shots[s];
            if (mem == AIO_MEM_HOST) {
                float* sp = sig.as<float>() + (long long)s * maxSrc * g.ntw;
                float* dp = dat.as<float>() + (long long)s * maxRec * g.nts;
                if (sh.sourcesSignals && sh.nSourcesReg > 0)
                    AIO_CK(cudaMemcpyAsync(sp, sh.sourcesSignals, (size_t)sh.nSourcesReg * g.ntw * 4,
                                           cudaMemcpyHostToDevice, st));
                if (dataIsInput) {
                    require(sh.data != nullptr || sh.nReceiversReg == 0, "adjoint input data missing");
                    if (sh.nReceiversReg > 0)
                        AIO_CK(cudaMemcpyAsync(dp, sh.data, (size_t)sh.nReceiversReg * g.nts * 4,
                                               cudaMemcpyHostToDevice, st));
                } else {
                    AIO_CK(cudaMemsetAsync(dp, 0, (size_t)std::max(sh.nReceiversReg, 0) * g.nts * 4, st));
                }
                srcSig[s] = sp;
                dataPtr[s] = dp;
                if (needWemvaData) {
                    float* wp = aux.as<float>() + (long long)s * maxRec * g.nts;
                    require(sh.wemvaData != nullptr, "WEMVA data missing");
                    AIO_CK(cudaMemcpyAsync(wp, sh.wemvaData, (size_t)sh.nReceiversReg * g.nts * 4,
                                           cudaMemcpyHostToDevice, st));
                    wdataPtr[s] = wp;
                }
            } else {
                srcSig[s] = sh.sourcesSignals;
                dataPtr[s] = sh.data;
                if (!dataIsInput && sh.data && sh.nReceiversReg > 0)
                    AIO_CK(cudaMemsetAsync(sh.data, 0, (size_t)sh.nReceiversReg * g.nts * 4, st));
                if (needWemvaData) wdataPtr[s] = sh.wemvaData;
            }
        }
        desc.ensure((size_t)nb * sizeof(ShotDesc));
    }
    std::vector<SparseList> srcLists, recLists;
    std::vector<const float*> srcSig, wdataPtr;
    std::vector<float*> dataPtr;

    void upload_desc(int nb) {
        AIO_CK(cudaMemcpyAsync(desc.p, hdesc.data(), (size_t)nb * sizeof(ShotDesc), cudaMemcpyHostToDevice, st));
    }

    // Copy forward-modelled data of a wave back to the caller (host mode).
    void download_data(int nb, const aio_shot* shots, int mem) {
        if (mem != AIO_MEM_HOST) return;
        for (int s = 0; s < nb; s++)
            if (shots[s].nReceiversReg > 0 && shots[s].data)
                AIO_CK(cudaMemcpyAsync(shots[s].data, dataPtr[s], (size_t)shots[s].nReceiversReg * g.nts * 4,
                                       cudaMemcpyDeviceToHost, st));
    }

    // ------------------------------------------------------------- stepper
    StepArgs base_args() const {
        StepArgs a;
        std::memset(&a, 0, sizeof(a));
        a.g = g;
        a.c = k.c;
        a.v2 = v2.as<float>();
        a.taper = taper.as<float>();
        a.shots = desc.as<ShotDesc>();
        a.injTB = -1;
        a.recTB = -1;
        a.fs = P.freeSurface ? 1 : 0;
        return a;
    }

    std::pair<cudaEvent_t, cudaEvent_t> take_events() {
        if (evFree.empty()) {
            cudaEvent_t a, b;
            AIO_CK(cudaEventCreate(&a));
            AIO_CK(cudaEventCreate(&b));
            evFree.push_back({a, b});
        }
        auto e = evFree.back();
        evFree.pop_back();
        return e;
    }
    void collect_events() {
        for (size_t i = 0; i < evBusy.size(); i++) {
            auto& e = evBusy[i];
            float ms = 0.f;
            AIO_CK(cudaEventElapsedTime(&ms, e.first, e.second));
            stepMs += ms;
            stepTimed++;
            stepPoints += (double)evPoints[i];
            evFree.push_back(e);
        }
        evBusy.clear();
        evPoints.clear();
    }

    void launch(int nb, bool adj, int inj, bool rec, bool acc, const StepArgs& a) {
        const bool timed = profEvery > 0 && (launches % profEvery) == 0;
        std::pair<cudaEvent_t, cudaEvent_t> ev{};
        if (timed) {
            ev = take_events();
            AIO_CK(cudaEventRecord(ev.first, st));
        }
        dim3 grid(g.tilesZ, g.tilesX, nb), block(TZ, TY);
        const int key = (adj ? 1 : 0) | (inj << 1) | ((rec ? 1 : 0) << 3) | ((acc ? 1 : 0) << 4);
        switch (key) {
#define AIO_CASE(A, I, R, C) \
    case ((A) | ((I) << 1) | ((R) << 3) | ((C) << 4)): k_step<(A) != 0, (I), (R) != 0, (C) != 0><<<grid, block, 0, st>>>(a); break;
            AIO_CASE(0, 0, 0, 0) AIO_CASE(1, 0, 0, 0) AIO_CASE(0, 1, 0, 0) AIO_CASE(1, 1, 0, 0)
            AIO_CASE(0, 2, 0, 0) AIO_CASE(1, 2, 0, 0) AIO_CASE(0, 0, 1, 0) AIO_CASE(1, 0, 1, 0)
            AIO_CASE(0, 1, 1, 0) AIO_CASE(1, 1, 1, 0) AIO_CASE(0, 2, 1, 0) AIO_CASE(1, 2, 1, 0)
            AIO_CASE(0, 0, 0, 1) AIO_CASE(1, 0, 0, 1) AIO_CASE(0, 1, 0, 1) AIO_CASE(1, 1, 0, 1)
            AIO_CASE(0, 2, 0, 1) AIO_CASE(1, 2, 0, 1) AIO_CASE(0, 0, 1, 1) AIO_CASE(1, 0, 1, 1)
            AIO_CASE(0, 1, 1, 1) AIO_CASE(1, 1, 1, 1) AIO_CASE(0, 2, 1, 1) AIO_CASE(1, 2, 1, 1)
#undef AIO_CASE
            default: throw Error{AIO_ERR_ARGUMENT, "unsupported stepper variant"};
        }
        AIO_CK(cudaGetLastError());
        if (timed) {
            AIO_CK(cudaEventRecord(ev.second, st));
            evBusy.push_back(ev);
            evPoints.push_back((long long)nb * g.nzi * g.nxi);
        }
        launches++;
        kernels++;
    }

    float hf(int i) const { return k.h[i]; }

    // Sets injection from sources (fine traces) and recording into receivers.
    void desc_sources_in(int nb, bool recordData) {
        for (int s = 0; s < nb; s++) {
            ShotDesc& d = hdesc[s];
            d.inj = srcLists[s];
            d.injSig = srcSig[s];
            d.injLd = g.ntw;
            d.rec = recordData ? recLists[s] : SparseList{nullptr, nullptr};
            d.recSig = recordData ? dataPtr[s] : nullptr;
            d.recLd = g.nts;
        }
    }
    // Sets injection of receiver data (coarse traces) and optional recording at sources.
    void desc_data_in(int nb, const std::vector<const float*>& data, const std::vector<float*>* srcOut) {
        for (int s = 0; s < nb; s++) {
            ShotDesc& d = hdesc[s];
            d.inj = recLists[s];
            d.injSig = data[s];
            d.injLd = g.nts;
            d.rec = srcOut ? srcLists[s] : SparseList{nullptr, nullptr};
            d.recSig = srcOut ? (*srcOut)[s] : nullptr;
            d.recLd = g.ntw;
        }
    }
    void desc_acc(int nb, DevMem* full) {
        for (int s = 0; s < nb; s++)
            hdesc[s].acc = full ? full->as<float>() + (long long)s * g.nts * g.isz
                                : ringb.as<float>() + (long long)s * 2 * g.isz;
    }
    void desc_dense(int nb, bool recordData) {
        for (int s = 0; s < nb; s++) {
            ShotDesc& d = hdesc[s];
            d.inj = SparseList{nullptr, nullptr};
            d.injSig = nullptr;
            d.rec = recordData ? recLists[s] : SparseList{nullptr, nullptr};
            d.recSig = recordData ? dataPtr[s] : nullptr;
            d.recLd = g.nts;
        }
    }

    void zero_levels(int nb) { AIO_CK(cudaMemsetAsync(pbuf.p, 0, (size_t)nb * 2 * g.hsz * 4, st)); }
    void zero_ring(int nb) { AIO_CK(cudaMemsetAsync(ringb.p, 0, (size_t)nb * 2 * g.isz * 4, st)); }
    void zero_ss(int nb) { AIO_CK(cudaMemsetAsync(ssb.p, 0, (size_t)nb * 2 * g.isz * 4, st)); }

    // Forward-time propagation of sparse injected traces (sources), optional
    // receiver recording and optional accumulation into a full coarse wavefield.
    // F/src/nonlinearShotsGpuFunctions.cu:269-295 and :351-380,
    // F/src/BornShotsGpuFunctions.cu:297-321.
    void fwd_sparse_pass(int nb, bool recordData, DevMem* wfld) {
        desc_sources_in(nb, recordData);
        desc_acc(nb, wfld);
        upload_desc(nb);
        zero_levels(nb);
        if (wfld) AIO_CK(cudaMemsetAsync(wfld->p, 0, (size_t)nb * g.nts * g.isz * 4, st));
        StepArgs a = base_args();
        int parity = 0;
        for (int its = 0; its < g.nts - 1; its++)
            for (int it2 = 1; it2 < g.sub + 1; it2++) {
                a.parity = parity;
                a.injTA = its * g.sub + it2 - 1;
                a.injTB = -1;
                a.recTA = its; a.recTB = its + 1; a.recCA = hf(it2); a.recCB = hf(g.H + it2);
                a.accOffA = (long long)its * g.isz; a.accOffB = (long long)(its + 1) * g.isz;
                a.hAccA = hf(it2); a.hAccB = hf(g.H + it2);
                launch(nb, false, 1, recordData, wfld != nullptr, a);
                parity ^= 1;
            }
    }

    // Adjoint-time propagation of injected receiver data with optional source
    // recording and accumulation (full wavefield or a 2-slice ring whose complete
    // coarse sample t is handed to post(t, slotOffset)).
    // F/src/nonlinearShotsGpuFunctions.cu:616-641, F/src/BornShotsGpuFunctions.cu:906-937,
    // F/src/tomoExtShotsGpuFunctions.cu:1481-1515.
    void adj_sparse_pass(int nb, const std::vector<const float*>& data, const std::vector<float*>* srcOut, AccMode am,
                         DevMem* wfld, const std::function<void(int, long long)>& post) {
        desc_data_in(nb, data, srcOut);
        desc_acc(nb, am == ACC_FULL ? wfld : nullptr);
        upload_desc(nb);
        zero_levels(nb);
        if (am == ACC_FULL) AIO_CK(cudaMemsetAsync(wfld->p, 0, (size_t)nb * g.nts * g.isz * 4, st));
        if (am == ACC_RING) zero_ring(nb);
        StepArgs a = base_args();
        int parity = 0;
        for (int its = g.nts - 2; its > -1; its--) {
            for (int it2 = g.sub - 1; it2 > -1; it2--) {
                a.parity = parity;
                a.injTA = its; a.injTB = its + 1; a.injCA = hf(it2 + 1); a.injCB = hf(g.H + it2 + 1);
                a.recTA = its * g.sub + it2; a.recTB = -1; a.recCA = 1.f;
                if (am == ACC_FULL) {
                    a.accOffA = (long long)its * g.isz; a.accOffB = (long long)(its + 1) * g.isz;
                } else {
                    a.accOffA = (long long)(its % 2) * g.isz; a.accOffB = (long long)((its + 1) % 2) * g.isz;
                }
                a.hAccA = hf(it2); a.hAccB = hf(g.H + it2);
                launch(nb, true, 1, srcOut != nullptr, am != ACC_NONE, a);
                parity ^= 1;
            }
            if (am == ACC_RING) post(its + 1, (long long)((its + 1) % 2) * g.isz);
        }
        if (am == ACC_RING) post(0, 0);
    }

    // Forward-time scattered propagation driven by a coarse secondary-source ring
    // (make_ss(t, slotOffset) fills slot t%2); optional data recording and
    // accumulation (full wavefield, or ring with post(t, slotOffset)).
    // F/src/BornShotsGpuFunctions.cu:342-374, F/src/tomoExtShotsGpuFunctions.cu:1554-1656,2442-2527.
    void fwd_dense_pass(int nb, const std::function<void(int, long long)>& make_ss, bool resetSS, bool recordData,
                        AccMode am, DevMem* wfld, const std::function<void(int, long long)>& post) {
        desc_dense(nb, recordData);
        desc_acc(nb, am == ACC_FULL ? wfld : nullptr);
        upload_desc(nb);
        zero_levels(nb);
        zero_ss(nb);
        if (am == ACC_FULL) AIO_CK(cudaMemsetAsync(wfld->p, 0, (size_t)nb * g.nts * g.isz * 4, st));
        if (am == ACC_RING) zero_ring(nb);
        StepArgs a = base_args();
        int parity = 0;
        make_ss(0, 0);
        for (int its = 0; its < g.nts - 1; its++) {
            const long long sL = (long long)(its % 2) * g.isz, sR = (long long)((its + 1) % 2) * g.isz;
            make_ss(its + 1, sR);
            for (int it2 = 1; it2 < g.sub + 1; it2++) {
                a.parity = parity;
                a.ssOffA = sL; a.ssOffB = sR; a.hInjA = hf(it2 - 1); a.hInjB = hf(g.H + it2 - 1);
                a.recTA = its; a.recTB = its + 1; a.recCA = hf(it2); a.recCB = hf(g.H + it2);
                if (am == ACC_FULL) {
                    a.accOffA = (long long)its * g.isz; a.accOffB = (long long)(its + 1) * g.isz;
                } else {
                    a.accOffA = sL; a.accOffB = sR;
                }
                a.hAccA = hf(it2); a.hAccB = hf(g.H + it2);
                launch(nb, false, 2, recordData, am != ACC_NONE, a);
                parity ^= 1;
            }
            if (am == ACC_RING) post(its, sL);
            if (resetSS) zero_slot(ssb, nb, sL);
        }
        if (am == ACC_RING) post(g.nts - 1, (long long)((g.nts - 1) % 2) * g.isz);
    }

    // Adjoint-time scattered propagation driven by a coarse secondary-source ring,
    // injected with h[it2+1]; the completed ring slot of coarse time t goes to post.
    // F/src/tomoExtShotsGpuFunctions.cu:2619-2700, F/src/wemvaExtShotsGpuFunctions.cu:1038-1121.
    void adj_dense_pass(int nb, const std::function<void(int, long long)>& make_ss, bool resetSS,
                        const std::function<void(int, long long)>& post) {
        desc_dense(nb, false);
        desc_acc(nb, nullptr);
        upload_desc(nb);
        zero_levels(nb);
        zero_ss(nb);
        zero_ring(nb);
        StepArgs a = base_args();
        int parity = 0;
        make_ss(g.nts - 1, (long long)((g.nts - 1) % 2) * g.isz);
        for (int its = g.nts - 2; its > -1; its--) {
            const long long sL = (long long)(its % 2) * g.isz, sR = (long long)((its + 1) % 2) * g.isz;
            make_ss(its, sL);
            for (int it2 = g.sub - 1; it2 > -1; it2--) {
                a.parity = parity;
                a.ssOffA = sL; a.ssOffB = sR; a.hInjA = hf(it2 + 1); a.hInjB = hf(g.H + it2 + 1);
                a.accOffA = sL; a.accOffB = sR; a.hAccA = hf(it2); a.hAccB = hf(g.H + it2);
                launch(nb, true, 2, false, true, a);
                parity ^= 1;
            }
            post(its + 1, sR);
            if (resetSS) zero_slot(ssb, nb, sR);
        }
        post(0, 0);
    }

    void zero_slot(DevMem& ring, int nb, long long off) {
        AIO_CK(cudaMemset2DAsync(ring.as<float>() + off, (size_t)2 * g.isz * 4, 0, (size_t)g.isz * 4, nb, st));
    }

    // ------------------------------------------------------------- coarse ops
    dim3 ew_grid(int nb, long long n) const {
        long long blocks = (n + 255) / 256;
        blocks = std::min<long long>(blocks, 1184);
        return dim3((unsigned)std::max<long long>(blocks, 1), nb, 1);
    }
    float* ss_ptr(long long off) { return ssb.as<float>() + off; }
    float* ring_ptr(long long off) { return ringb.as<float>() + off; }
    long long pairSt() const { return 2 * g.isz; }
    long long wfSt() const { return (long long)g.nts * g.isz; }

    // ss[slot] = m * W[t]  (imagingFwdGpu)
    void img_fwd(int nb, long long slot, const float* m, long long mSt, const float* W, int t) {
        k_img_fwd<<<ew_grid(nb, g.isz), 256, 0, st>>>(ss_ptr(slot), pairSt(), m, mSt, W + (long long)t * g.isz,
                                                       wfSt(), g.isz);
        kcheck();
    }
    // image += W[t] * ring[slot]; ring[slot] = 0  (imagingAdjGpu)
    void img_adj(int nb, long long slot, const float* W, int t) {
        if (P.imageFp64)
            k_img_adj<double><<<ew_grid(nb, g.isz), 256, 0, st>>>(img.as<double>(), g.isz, ring_ptr(slot), pairSt(),
                                                                  W + (long long)t * g.isz, wfSt(), g.isz, 1);
        else
            k_img_adj<float><<<ew_grid(nb, g.isz), 256, 0, st>>>(img.as<float>(), g.isz, ring_ptr(slot), pairSt(),
                                                                 W + (long long)t * g.isz, wfSt(), g.isz, 1);
        kcheck();
    }
    // Lag bounds with C truncating division (F/src/BornExtShotsGpuFunctions.cu:366-383;
    // F/src/tomoExtShotsGpuFunctions.cu:2631-2650).
    void bounds_src(int t, int& e0, int& e1) const {
        e0 = std::max((t + 1 - g.nts) / 2, -g.hExt) + g.hExt;
        e1 = std::min(t / 2, g.hExt) + g.hExt + 1;
    }
    void bounds_rec(int t, int& e0, int& e1) const {
        e0 = std::max((-t) / 2, -g.hExt) + g.hExt;
        e1 = std::min((g.nts - 1 - t) / 2, g.hExt) + g.hExt + 1;
    }
    // ss[slot] += sum_e ext[e] W[t-2(e-h)]  (imagingTimeFwdGpu)
    void img_time_fwd(int nb, long long slot, const float* ext, const float* W, int t) {
        int e0, e1;
        bounds_src(t, e0, e1);
        k_img_time_fwd<<<ew_grid(nb, g.isz), 256, 0, st>>>(ss_ptr(slot), pairSt(), ext, 0, W, wfSt(), g.isz, t, e0,
                                                            e1, g.hExt);
        kcheck();
    }
    // ss[slot] += sum_e ext[e] R[t+2(e-h)]  (imagingTimeTomoAdjGpu)
    void img_time_tomo_adj(int nb, long long slot, const float* ext, const float* R, int t) {
        int e0, e1;
        bounds_rec(t, e0, e1);
        k_img_time_tomo_adj<<<ew_grid(nb, g.isz), 256, 0, st>>>(ss_ptr(slot), pairSt(), ext, 0, R, wfSt(), g.isz, t,
                                                                 e0, e1, g.hExt);
        kcheck();
    }
    // image[e] += ring[slot] * W[t -/+ 2(e-h)]; ring[slot] = 0
    //   sign=+1: imagingTimeAdjGpu (source side); sign=-1: imagingWemvaTimeAdjGpu.
    void img_time_adj(int nb, long long slot, const float* W, int t, int sign) {
        int e0, e1;
        if (sign > 0) bounds_src(t, e0, e1);
        else bounds_rec(t, e0, e1);
        const long long mSt = (long long)g.nExt * g.isz;
        if (P.imageFp64)
            k_img_time_adj<double><<<ew_grid(nb, g.isz), 256, 0, st>>>(img.as<double>(), mSt, ring_ptr(slot), pairSt(),
                                                                       W, wfSt(), g.isz, t, e0, e1, g.hExt, sign, 1);
        else
            k_img_time_adj<float><<<ew_grid(nb, g.isz), 256, 0, st>>>(img.as<float>(), mSt, ring_ptr(slot), pairSt(),
                                                                      W, wfSt(), g.isz, t, e0, e1, g.hExt, sign, 1);
        kcheck();
    }

    // ---- subsurface offsets (interior-slice kernels in aio_kernels.cuh)
    bool offsets() const { return P.extension == AIO_EXT_OFFSET; }
    // ss[slot] = v2 * (ss[slot] + sum_s m_s(x-s) F_t(x-2s))  (imagingOffsetFwdGpu + scaleSecondarySourceFd)
    void img_offset_fwd(int nb, long long slot, const float* m, const float* F, int t) {
        k_img_offset_fwd<<<ew_grid(nb, g.isz), 256, 0, st>>>(ss_ptr(slot), pairSt(), m, 0, F + (long long)t * g.isz,
                                                              wfSt(), v2.as<float>(), g.isz, g.ip, g.nxi, g.hExt);
        kcheck();
    }
    // ss[slot] += sum_s m_s(x+s) R_t(x+2s) v2(x+2s)  (imagingOffsetTomoAdjGpu)
    void img_offset_tomo_adj(int nb, long long slot, const float* m, const float* R, int t) {
        k_img_offset_tomo_adj<<<ew_grid(nb, g.isz), 256, 0, st>>>(ss_ptr(slot), pairSt(), m, 0,
                                                                   R + (long long)t * g.isz, wfSt(), v2.as<float>(),
                                                                   nullptr, g.isz, g.ip, g.nxi, g.hExt);
        kcheck();
    }
    // Subsurface-offset imaging in blocks of OFF_K coarse samples: the ring slot of sample t is
    // copied into slice t % OFF_K of offBuf and zeroed; once the block holding t is complete
    // (passes running backward in time: t % OFF_K == 0; forward: t % OFF_K == OFF_K - 1 or
    // t == nts - 1), k_img_offset_block images all of its samples, reading and writing the image
    // once per block.
    DevMem offBuf;
    void img_offset_adj_block(int nb, long long slot, const float* F, int t, bool wemvaForm, bool backward) {
        offBuf.ensure((size_t)nb * OFF_K * g.isz * 4);
        AIO_CK(cudaMemcpy2DAsync(offBuf.as<float>() + (long long)(t % OFF_K) * g.isz, (size_t)OFF_K * g.isz * 4,
                                 ring_ptr(slot), (size_t)pairSt() * 4, (size_t)g.isz * 4, nb,
                                 cudaMemcpyDeviceToDevice, st));
        zero_slot(ringb, nb, slot);
        const bool done = backward ? (t % OFF_K == 0) : (t % OFF_K == OFF_K - 1 || t == g.nts - 1);
        if (!done) return;
        const int tlo = t - t % OFF_K, thi = std::min(tlo + OFF_K - 1, g.nts - 1);
        const long long mSt = (long long)g.nExt * g.isz, RSt = (long long)OFF_K * g.isz;
        if (P.imageFp64)
            k_img_offset_block<double><<<ew_grid(nb, g.isz), 256, 0, st>>>(
                img.as<double>(), mSt, offBuf.as<float>(), RSt, F, wfSt(), v2.as<float>(), (int)g.isz, g.ip, g.nxi,
                g.hExt, g.nExt, tlo, thi, wemvaForm ? 1 : 0);
        else
            k_img_offset_block<float><<<ew_grid(nb, g.isz), 256, 0, st>>>(
                img.as<float>(), mSt, offBuf.as<float>(), RSt, F, wfSt(), v2.as<float>(), (int)g.isz, g.ip, g.nxi,
                g.hExt, g.nExt, tlo, thi, wemvaForm ? 1 : 0);
        kcheck();
    }

    void scale_shared(float* m, int nSlices, int mode) {
        k_scale<<<ew_grid(1, (long long)nSlices * g.isz), 256, 0, st>>>(m, 0, nSlices, v2.as<float>(), rs.as<float>(),
                                                                         g.isz, mode);
        kcheck();
    }

    // Scale per-shot images (reference scales each shot's model before the host
    // stack, F/src/BornShotsGpu.cpp:325-332) and sum them into out (interior slices).
    void reduce_images(int nb, int nSlices, int mode, float* out, bool add) {
        const long long n = (long long)nSlices * g.isz;
        if (P.imageFp64) {
            k_scale_d<<<ew_grid(nb, n), 256, 0, st>>>(img.as<double>(), n, nSlices, v2.as<float>(), rs.as<float>(),
                                                      g.isz, mode);
            kcheck();
            k_sum_shots<double><<<ew_grid(1, n), 256, 0, st>>>(out, img.as<double>(), n, nb, n, add ? 1 : 0);
        } else {
            k_scale<<<ew_grid(nb, n), 256, 0, st>>>(img.as<float>(), n, nSlices, v2.as<float>(), rs.as<float>(), g.isz,
                                                    mode);
            kcheck();
            k_sum_shots<float><<<ew_grid(1, n), 256, 0, st>>>(out, img.as<float>(), n, nb, n, add ? 1 : 0);
        }
        kcheck();
    }
    void zero_images(int nb, int nSlices) {
        AIO_CK(cudaMemsetAsync(img.p, 0, (size_t)nb * nSlices * g.isz * (P.imageFp64 ? 8 : 4), st));
    }

    // Model staging: shared interior slices for models, extended reflectivity
    // and the summed output.
    float* stage_model(const float* m, int nSlices, int mem, DevMem& buf) {
        buf.ensure((size_t)nSlices * g.isz * 4);
        AIO_CK(cudaMemsetAsync(buf.p, 0, (size_t)nSlices * g.isz * 4, st));
        to_interior(buf.as<float>(), m, nSlices, mem);
        return buf.as<float>();
    }
    void write_model(float* dst, int nSlices, int add, int mem, float* outInterior) {
        // outInterior already holds (add ? dst + result : result) on interior points.
        if (!add) {
            if (mem == AIO_MEM_HOST) std::memset(dst, 0, (size_t)nSlices * g.nz * g.nx * 4);
            else AIO_CK(cudaMemsetAsync(dst, 0, (size_t)nSlices * g.nz * g.nx * 4, st));
        }
        from_interior(dst, outInterior, nSlices, mem);
    }
    void sync() {
        AIO_CK(cudaStreamSynchronize(st));
        collect_events();
    }

    void begin_call() {
        AIO_CK(cudaSetDevice(dev));
        launches = 0;
    }


    // ============================================================ blocked stepper
    // One launch per coarse interval (aio_tb.cuh). State, partial sums and
    // images use interior slices; the stored wavefield is FP32 or BF16.
    DevMem tbState, tbPart, tbImg, tbW, tbEnt, tbStart, tbDesc, shotImg;
    DevMem tbWscale, tbWmax, tbWstage;  // FP16 stored wavefield: per-slice scales, max |W|, FP32 staging
    DevMem tbWover;                     // FP16 stored wavefield: overflow flag of the speculative scales
    DevMem tbR;                         // extended adjoint: coarse receiver samples [shot][LAG_K][isz]
    DevMem tbSS;                        // extended forward: secondary sources [shot][2 LAG_K][isz]
    DevMem tbF2;                        // tomo / WEMVA: second full coarse field [shot][nts][isz]

    // Per-call buffers: every device allocation of the context but the velocity constants. They
    // grow to the largest wave seen and are kept between calls; a request server that plans the
    // device memory of several contexts counts them (device_bytes) and frees those of an idle
    // context when another needs the room (release_buffers).
    std::vector<DevMem*> call_buffers() {
        return {&pbuf,  &ringb,    &ssb,    &wf1,      &wf2,     &wf3,     &img,     &lists,   &desc,
                &sig,   &dat,      &aux,    &model,    &ext,     &outv,    &offBuf,  &tbState, &tbPart,
                &tbImg, &tbW,      &tbEnt,  &tbStart,  &tbDesc,  &shotImg, &tbWscale, &tbWmax, &tbWstage,
                &tbWover, &tbR,    &tbSS,   &tbF2};
    }
    long long device_bytes() {
        long long b = (long long)(v2.bytes + rs.bytes + taper.bytes);
        for (DevMem* m : call_buffers()) b += (long long)m->bytes;
        return b;
    }
    // Frees the per-call buffers (and the captured graphs, whose launches hold their addresses).
    void release_buffers() {
        AIO_CK(cudaSetDevice(dev));
        AIO_CK(cudaStreamSynchronize(st));
        drop_graphs();
        for (DevMem* m : call_buffers()) m->release();
    }
    // k_tile plan: strips of HZ (multiple of 4) output rows, NQ = HZ/4 + 10 row quads,
    // 8 column pairs per quad, x-chunks of LX columns marched in blocks of 16.
    struct TBPlan {
        int T = KT_T, HZ = 0, nStrips = 0, LX = 0, nChunks = 0, iters = 0, threads = 0, NQ = 0;
    };

    bool tb_enabled() const { return P.stepper != AIO_STEPPER_FINE && g.sub == KT_T; }
    int wbytes() const { return P.wavefieldPrecision == AIO_WFLD_FP32 ? 4 : 2; }
    bool f16() const { return P.wavefieldPrecision == AIO_WFLD_FP16; }

    // nb: shots of the wave (one CTA column per shot)
    // Plan of a wave of nb shots: the autotuned plan when one was measured, else the model's.
    // Plans are tuned per wave size and kernel class: light modes (SRC, NL, ADJR: at most 6
    // staging slots, no secondary-source rings), heavy modes (SCAT, SCATX, SCATW, ADJX), whose
    // larger shared-memory footprint changes how many CTAs an SM holds, and the Born receiver
    // pass (ADJ: 12 staging slots, FP64 image read-modify-write, receivers injected).
    // The nonlinear forward (NL: sources in, receivers recorded, no stored wavefield) is tuned as
    // its own class: its single-shot calls are the small, latency-bound waves.
    enum TBClass { TB_LIGHT = 0, TB_HEAVY = 1, TB_RECV = 2, TB_NLC = 3 };
    TBPlan tb_plan(int nb, bool heavy = false) const { return tb_plan_c(nb, heavy ? TB_HEAVY : TB_LIGHT); }
    TBPlan tb_plan_c(int nb, int cls) const {
        auto it = tbTuned.find(4 * nb + cls);
        if (it != tbTuned.end()) return it->second;
        return tb_model_plan(nb, 4 * (KT_MAXQ - 10), P.chunkColumns > 0 ? P.chunkColumns : 0);
    }

    // Strips of at most maxHZ rows; x-chunks of about chunkColumns columns, or (0) the chunk
    // count minimising the modelled time: whole CTA waves over the SMs (one resident CTA per
    // SM) times the iterations of one CTA (each chunk recomputes 10T warm-up columns), at
    // least 4 waves preferred so that CTAs of uneven cost (strips holding sources or
    // receivers) balance out.
    // minWaves: smallest number of CTA waves (of one CTA per SM) the chunk count is chosen from
    TBPlan tb_model_plan(int nb, int maxHZ, int chunkColumns, int forceChunks = 0, int minWaves = 4) const {
        TBPlan pl;
        pl.nStrips = (g.nzi + maxHZ - 1) / maxHZ;
        pl.HZ = round_up((g.nzi + pl.nStrips - 1) / pl.nStrips, 4);
        pl.NQ = pl.HZ / 4 + 10;
        pl.threads = round_up(8 * pl.NQ, 32);
        if (forceChunks > 0) {
            pl.nChunks = std::min(forceChunks, g.nxi);
        } else if (chunkColumns > 0) {
            pl.nChunks = std::max(1, (g.nxi + chunkColumns / 2) / chunkColumns);
        } else {
            double best = 1e300, bestAny = 1e300;
            int ncAny = 1;
            pl.nChunks = 0;
            for (int nc = 1; nc <= std::max(1, g.nxi / 48); nc++) {
                const int lx = (g.nxi + nc - 1) / nc;
                const long long ctas = (long long)pl.nStrips * nc * nb;
                const double cost = (double)((ctas + smCount - 1) / smCount) * ((lx + 10 * pl.T + KT_BX - 1) / KT_BX);
                if (cost < bestAny * 0.999) {
                    bestAny = cost;
                    ncAny = nc;
                }
                if (ctas >= (long long)minWaves * smCount && cost < best * 0.999) {
                    best = cost;
                    pl.nChunks = nc;
                }
            }
            if (pl.nChunks == 0) pl.nChunks = ncAny;
        }
        pl.LX = (g.nxi + pl.nChunks - 1) / pl.nChunks;
        pl.iters = (pl.LX + 10 * pl.T + KT_BX - 1) / KT_BX;
        return pl;
    }

    // Measured autotuning of the blocked stepper's plan for waves of nb shots (chunkColumns
    // == 0): strip heights {128, 112, 96, 80, 64} rows x chunk counts around the model's choices
    // (at least 4 waves of CTAs, and the cheapest count for any number of waves) are each timed
    // on the source-pass launch of interval 0 (idempotent: it reads one state set and
    // overwrites the other, the stored slice 0 and the partial sums), the fastest is cached
    // for the context. The state is zeroed again afterwards.
    std::map<int, TBPlan> tbTuned;
    TBPlan tbLast;  // plan of the most recent blocked launch

    // Plans measured by any context of the process, shared by the contexts of the same device,
    // interior size, free-surface setting and stored precision: a new context (a request server
    // opens one per grid and velocity model) takes them instead of timing the candidates again.
    // The velocity model does not enter a launch's duration.
    static std::map<std::vector<int>, TBPlan>& shared_plans() {
        static std::map<std::vector<int>, TBPlan> m;
        return m;
    }
    static std::mutex& shared_plans_mu() {
        static std::mutex mu;
        return mu;
    }
    std::vector<int> shared_plan_key(int k) const {
        return {dev, g.nzi, g.nxi, k, P.freeSurface, P.wavefieldPrecision};
    }
    // The shared plans of waves of nb shots, when every class has one that fits these shots.
    bool tb_take_shared(int nb, const aio_shot* shots, bool nonlinear) {
        const std::vector<int> classes = nonlinear ? std::vector<int>{TB_NLC} : std::vector<int>{TB_LIGHT, TB_HEAVY, TB_RECV};
        std::vector<TBPlan> got;
        {
            std::lock_guard<std::mutex> lk(shared_plans_mu());
            for (int c : classes) {
                auto it = shared_plans().find(shared_plan_key(4 * nb + c));
                if (it == shared_plans().end()) return false;
                got.push_back(it->second);
            }
        }
        for (const TBPlan& pl : got)
            if (!tb_plan_fits(pl, tb_max_entries(pl, nb, shots))) return false;
        for (size_t i = 0; i < classes.size(); i++) tbTuned[4 * nb + classes[i]] = got[i];
        return true;
    }

    // Largest sparse-entry counts one CTA of plan pl holds, per kind of pass: sources injected
    // over the halo region plus receivers recorded in the output region (SRC, NL), receivers
    // recorded (SCAT, SCATX), receivers injected over the halo region plus sources recorded
    // (ADJ, ADJR).
    struct TBEntries {
        int fwd = 1, scat = 1, adj = 1;
    };
    TBEntries tb_max_entries(const TBPlan& pl, int nb, const aio_shot* shots) const {
        const int h = 5 * (pl.T - 1);
        const size_t nCTA = (size_t)pl.nStrips * pl.nChunks;
        std::vector<int> srcHalo(nCTA), srcOut(nCTA), recHalo(nCTA), recOut(nCTA);
        TBEntries m;
        for (int s = 0; s < nb; s++) {
            for (auto* v : {&srcHalo, &srcOut, &recHalo, &recOut}) std::fill(v->begin(), v->end(), 0);
            auto add = [&](const int* pos, int n, std::vector<int>& halo, std::vector<int>& out) {
                for (int k2 = 0; k2 < n; k2++) {
                    const int iz = (int)(pos[k2] % g.nz) - FAT, ix = (int)(pos[k2] / g.nz) - FAT;
                    for (int st2 = std::max(0, (iz - h) / pl.HZ - 1); st2 <= std::min(pl.nStrips - 1, (iz + h) / pl.HZ + 1); st2++) {
                        const int z0 = st2 * pl.HZ, z1 = std::min(z0 + pl.HZ, g.nzi);
                        if (iz < z0 - h || iz >= z1 + h) continue;
                        for (int ch = std::max(0, (ix - h) / pl.LX - 1); ch <= std::min(pl.nChunks - 1, (ix + h) / pl.LX + 1); ch++) {
                            const int x0 = ch * pl.LX, x1 = std::min(x0 + pl.LX, g.nxi);
                            if (ix < x0 - h || ix >= x1 + h) continue;
                            const size_t c = (size_t)st2 * pl.nChunks + ch;
                            halo[c]++;
                            if (ix >= x0 && ix < x1 && iz >= z0 && iz < z1) out[c]++;
                        }
                    }
                }
            };
            add(shots[s].sourcesPositionReg, shots[s].nSourcesReg, srcHalo, srcOut);
            add(shots[s].receiversPositionReg, shots[s].nReceiversReg, recHalo, recOut);
            for (size_t c = 0; c < nCTA; c++) {
                m.fwd = std::max(m.fwd, srcHalo[c] + recOut[c]);
                m.scat = std::max(m.scat, recOut[c]);
                m.adj = std::max(m.adj, recHalo[c] + srcOut[c]);
            }
        }
        return m;
    }
    // row quads of the k_tile variant a strip of NQ row quads runs on (the free surface: the
    // large-strip variant only)
    int tb_variant(int NQ) const {
        if (P.freeSurface) return KT_MAXQ;
        return NQ <= KT_MAXQ_S ? KT_MAXQ_S : (NQ <= KT_MAXQ_M ? KT_MAXQ_M : KT_MAXQ);
    }
    // plan pl fits in shared memory in every mode
    bool tb_plan_fits(const TBPlan& pl, const TBEntries& e) const {
        int smemMax = 0;
        if (cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
        const int mq = tb_variant(pl.NQ);
        const std::pair<int, int> need[] = {{TB_SRC, e.fwd}, {TB_SCAT, e.scat}, {TB_ADJ, e.adj}, {TB_SCATW, 1}};
        for (const auto& mn : need)
            if (kt_smem_bytes(mn.first, pl.threads, pl.iters, mn.second, kt_rs(mq), kt_v2s(mq)) > (size_t)smemMax)
                return false;
        return true;
    }

    // Candidates: strip heights {128 .. 64} rows (and, for waves too small to fill the GPU with
    // 128-row strips, 48 and 32 rows) x chunk counts around the model's choices; for those small
    // waves also the chunk counts that give one or two CTAs per SM, with chunks down to 16
    // columns. nonlinear: the NL class alone is timed (its launch with recording off).
    void tb_autotune(int nb, const aio_shot* shots, bool nonlinear = false) {
        if (P.chunkColumns != 0 || tbTuned.count(4 * nb + (nonlinear ? TB_NLC : TB_LIGHT))) return;
        if (tb_take_shared(nb, shots, nonlinear)) return;
        const bool small = (long long)tb_model_plan(nb, 128, 0, 0, 1).nStrips * std::max(1, g.nxi / 48) * nb <
                           2LL * smCount;
        std::vector<int> heights = {128, 112, 96, 80, 64};
        if (small) heights.insert(heights.end(), {48, 32});
        const int maxChunks = std::max(1, g.nxi / (small ? 16 : 32));
        std::vector<TBPlan> cand;
        for (int maxHZ : heights)
            for (int minWaves : {4, 1, 0}) {
                TBPlan m;
                if (minWaves > 0) {
                    m = tb_model_plan(nb, maxHZ, 0, 0, minWaves);
                } else {  // small waves: about one and two CTAs per SM
                    if (!small) continue;
                    m = tb_model_plan(nb, maxHZ, 0, 1);
                    m.nChunks = std::max(1, (int)(smCount / std::max(1LL, (long long)m.nStrips * nb)));
                }
                for (int d : {-2, -1, 0, 1, 2, minWaves == 0 ? m.nChunks : 0}) {
                    const int nc = m.nChunks + d;
                    if (nc < 1 || nc > maxChunks) continue;
                    TBPlan c = tb_model_plan(nb, maxHZ, 0, nc);
                    bool dup = false;
                    for (auto& o : cand) dup |= (o.HZ == c.HZ && o.nChunks == c.nChunks);
                    if (!dup && c.threads <= KT_MAXT && c.NQ <= KT_MAXQ &&
                        tb_plan_fits(c, tb_max_entries(c, nb, shots)))
                        cand.push_back(c);
                }
            }
        if (cand.empty()) return;  // the model's plan (tb_plan) then stands
        cudaEvent_t e0, e1;
        AIO_CK(cudaEventCreate(&e0));
        AIO_CK(cudaEventCreate(&e1));
        float bestMs = 1e30f, bestHeavyMs = 1e30f, bestRecvMs = 1e30f;
        TBPlan best = cand.front(), bestHeavy = cand.front(), bestRecv = cand.front();
        const long long saveLaunches = launches, saveKernels = kernels;
        const int saveProf = profEvery;
        const char* logEnv = std::getenv("AIO_AUTOTUNE_LOG");  // print every candidate's timings
        const bool logTune = logEnv && *logEnv && *logEnv != '0';
        profEvery = 0;
        // Per-launch time: the fastest of three timings of n back-to-back launches (after a timed
        // warm-up launch: smem carve-out, caches), so that a disturbed timing does not decide the
        // plan; n makes a timing span >= 0.1 ms (at most 8 launches), which for single-shot
        // launches of ~20 us keeps event and clock jitter from deciding it while keeping the
        // tuning of a new wave size short (serving tunes one per grid and wave size).
        auto timeMin = [&](auto launch) {
            AIO_CK(cudaEventRecord(e0, st));
            launch();
            AIO_CK(cudaEventRecord(e1, st));
            AIO_CK(cudaEventSynchronize(e1));
            float t1 = 0.f;
            AIO_CK(cudaEventElapsedTime(&t1, e0, e1));
            const int n = std::min(8, std::max(2, (int)std::ceil(0.1f / std::max(t1, 1e-3f))));
            float best2 = 1e30f;
            for (int rep = 0; rep < 3; rep++) {
                AIO_CK(cudaEventRecord(e0, st));
                for (int i = 0; i < n; i++) launch();
                AIO_CK(cudaEventRecord(e1, st));
                AIO_CK(cudaEventSynchronize(e1));
                float t = 0.f;
                AIO_CK(cudaEventElapsedTime(&t, e0, e1));
                best2 = std::min(best2, t / n);
            }
            return best2;
        };
        for (const TBPlan& pl : cand) {
            const int maxEnt = tb_lists(pl, nb, shots, 1, false);
            tb_zero(nb, false);
            tb_desc(pl, nb, true, false, false, nonlinear ? nullptr : tbW.p, false);
            KTArgs a = tb_args(pl, maxEnt, nullptr);
            a.its = 0;
            if (nonlinear) {  // NL class: the launch without recording (the data stay untouched)
                const float ms = timeMin([&] { tb_launch<TB_NL>(pl, nb, a, 0); });
                if (ms < bestMs) {
                    bestMs = ms;
                    best = pl;
                }
                if (logTune)
                    std::fprintf(stderr, "aio autotune (NL): shots %d strip %d x %d chunk %d x %d threads %d: %.3f ms\n",
                                 nb, pl.HZ, pl.nStrips, pl.LX, pl.nChunks, pl.threads, ms);
                continue;
            }
            if (f16()) AIO_CK(cudaMemsetAsync(tbWmax.p, 0, (size_t)nb * g.nts * 4, st));
            float ms = timeMin([&] { tb_launch<TB_SRC>(pl, nb, a, 0); });
            if (ms < bestMs) {
                bestMs = ms;
                best = pl;
            }
            const float lightMs = ms;
            // heavy class: the time-lag scattered pass (reads W slices 0, 1 as its sources;
            // writes only the other state set)
            const int maxEntH = tb_lists(pl, nb, shots, 0, false);  // before tb_desc: it may move the lists
            tb_desc(pl, nb, false, false, false, tbW.p, false);
            a = tb_args(pl, maxEntH, nullptr);
            a.its = 0;
            a.rSlot = 0;
            a.rSlot0 = 1;
            ms = timeMin([&] { tb_launch<TB_SCATX>(pl, nb, a, 0); });
            if (ms < bestHeavyMs) {
                bestHeavyMs = ms;
                bestHeavy = pl;
            }
            const float heavyMs = ms;
            // receiver class: the Born receiver pass at the last interval (reads state set 0 and
            // W[nts-1], writes the other state set and partial sums; its image accumulation is
            // discarded: the pass zeroes the image first)
            tbImg.ensure((size_t)nb * g.isz * 8);
            const int maxEntR = tb_lists(pl, nb, shots, 2, false);
            tb_desc(pl, nb, false, true, false, tbW.p, false);
            a = tb_args(pl, maxEntR, nullptr);
            a.its = g.nts - 2;
            ms = timeMin([&] { tb_launch<TB_ADJ>(pl, nb, a, 0); });
            if (ms < bestRecvMs) {
                bestRecvMs = ms;
                bestRecv = pl;
            }
            if (logTune)
                std::fprintf(stderr,
                             "aio autotune: shots %d strip %d x %d chunk %d x %d threads %d: light %.3f ms heavy %.3f ms "
                             "receiver %.3f ms\n",
                             nb, pl.HZ, pl.nStrips, pl.LX, pl.nChunks, pl.threads, lightMs, heavyMs, ms);
        }
        AIO_CK(cudaEventDestroy(e0));
        AIO_CK(cudaEventDestroy(e1));
        launches = saveLaunches;
        kernels = saveKernels;
        profEvery = saveProf;
        if (nonlinear) {
            tbTuned[4 * nb + TB_NLC] = best;
        } else {
            tbTuned[4 * nb + TB_LIGHT] = best;
            tbTuned[4 * nb + TB_HEAVY] = bestHeavy;
            tbTuned[4 * nb + TB_RECV] = bestRecv;
        }
        std::lock_guard<std::mutex> lk(shared_plans_mu());
        for (int c : nonlinear ? std::vector<int>{TB_NLC} : std::vector<int>{TB_LIGHT, TB_HEAVY, TB_RECV})
            shared_plans()[shared_plan_key(4 * nb + c)] = tbTuned[4 * nb + c];
    }

    // Per-CTA sparse lists of every shot of a wave. inj: 0 none, 1 sources, 2 receivers
    // (over the CTA's recomputed halo region); rec: record receivers (output region).
    int tb_lists(const TBPlan& pl, int nb, const aio_shot* shots, int inj, bool rec) {
        std::vector<TBEnt> ents;
        std::vector<int4> starts((size_t)nb * pl.nStrips * pl.nChunks);
        const int h = 5 * (pl.T - 1);
        int maxEnt = 1;
        for (int s = 0; s < nb; s++) {
            std::vector<std::pair<int, int>> ipos, rpos;  // (interior x, interior z) per device
            auto collect = [&](const int* pos, int n, std::vector<std::pair<int, int>>& out, const char* what) {
                out.resize(n);
                for (int k2 = 0; k2 < n; k2++) {
                    const long long p = pos[k2];
                    const int iz = (int)(p % g.nz), ix = (int)(p / g.nz);
                    require(p >= 0 && ix < g.nx && iz >= FAT && iz < g.nz - FAT && ix >= FAT && ix < g.nx - FAT,
                            std::string(what) + " position " + std::to_string(p) + " is outside the interior grid");
                    out[k2] = {ix - FAT, iz - FAT};
                }
            };
            if (inj == 1) collect(shots[s].sourcesPositionReg, shots[s].nSourcesReg, ipos, "source");
            if (inj == 2) collect(shots[s].receiversPositionReg, shots[s].nReceiversReg, ipos, "receiver");
            if (rec) collect(shots[s].receiversPositionReg, shots[s].nReceiversReg, rpos, "receiver");
            for (int st2 = 0; st2 < pl.nStrips; st2++)
                for (int ch = 0; ch < pl.nChunks; ch++) {
                    const int z0 = st2 * pl.HZ, z1 = std::min(z0 + pl.HZ, g.nzi);
                    const int x0 = ch * pl.LX, x1 = std::min(x0 + pl.LX, g.nxi);
                    std::vector<TBEnt> a1, a2;
                    for (size_t d = 0; d < ipos.size(); d++) {
                        const int x = ipos[d].first, z = ipos[d].second;
                        if (x >= x0 - h && x < x1 + h && z >= z0 - h && z < z1 + h) a1.push_back(TBEnt{x, z, (int)d, 0});
                    }
                    for (size_t d = 0; d < rpos.size(); d++) {
                        const int x = rpos[d].first, z = rpos[d].second;
                        if (x >= x0 && x < x1 && z >= z0 && z < z1) a2.push_back(TBEnt{x, z, (int)d, 0});
                    }
                    auto byCol = [](const TBEnt& A, const TBEnt& B) { return A.col < B.col || (A.col == B.col && A.row < B.row); };
                    std::sort(a1.begin(), a1.end(), byCol);
                    std::sort(a2.begin(), a2.end(), byCol);
                    int4 se;
                    se.x = (int)ents.size();
                    ents.insert(ents.end(), a1.begin(), a1.end());
                    se.y = (int)ents.size();
                    se.z = se.y;
                    ents.insert(ents.end(), a2.begin(), a2.end());
                    se.w = (int)ents.size();
                    starts[((size_t)s * pl.nStrips + st2) * pl.nChunks + ch] = se;
                    maxEnt = std::max(maxEnt, se.w - se.x);
                }
        }
        require(maxEnt <= 4096, "too many sparse devices inside one blocked-stepper tile");
        tbEnt.ensure(std::max<size_t>(ents.size(), 1) * sizeof(TBEnt));
        tbStart.ensure(starts.size() * sizeof(int4));
        if (!ents.empty())
            AIO_CK(cudaMemcpyAsync(tbEnt.p, ents.data(), ents.size() * sizeof(TBEnt), cudaMemcpyHostToDevice, st));
        AIO_CK(cudaMemcpyAsync(tbStart.p, starts.data(), starts.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
        return maxEnt;
    }

    void tb_alloc(int nb, bool needImg) {
        require(g.isz < (1LL << 31), "interior slice too large for 32-bit in-slice offsets");
        tbState.ensure((size_t)nb * 4 * g.isz * 4);
        tbPart.ensure((size_t)nb * 2 * g.isz * 4);
        if (needImg) tbImg.ensure((size_t)nb * g.isz * 8);
        tbDesc.ensure((size_t)2 * nb * sizeof(TBShot));
        if (f16()) {
            tbWscale.ensure((size_t)nb * g.nts * 4);
            tbWmax.ensure((size_t)nb * g.nts * 4);
            tbWstage.ensure((size_t)nb * 2 * g.isz * 4);
            tbWover.ensure(4);
        }
    }

    // Descriptor pairs: version v reads state/part set v and writes set 1-v
    // (partSwap=true: the ADJ part ordering, see tb_adj_pass).
    // wSlices: coarse slices per shot in W (the stored wavefield: nts; a secondary-source ring: its length)
    // out / outSlices: per-shot slices written by ADJR / SCATW / ADJX (default: the LAG_K ring tbR)
    // dataIn: traces injected when injData (default: the wave's data)
    // W: the stored source wavefield (elements of wbytes()) or, with wSlices > 0, an FP32 ring of
    // wSlices secondary-source slices
    void tb_desc(const TBPlan& pl, int nb, bool injSources, bool injData, bool recData, void* W, bool partFlip,
                 int wSlices = 0, float* out = nullptr, int outSlices = 0, const float* const* dataIn = nullptr) {
        const int wElem = wSlices > 0 ? 4 : wbytes();
        if (wSlices <= 0) wSlices = g.nts;
        if (!out && tbR.p) {
            out = tbR.as<float>();
            outSlices = LAG_K;
        }
        std::vector<TBShot> d(2 * (size_t)nb);
        const int nCTA = pl.nStrips * pl.nChunks;
        for (int v = 0; v < 2; v++)
            for (int s = 0; s < nb; s++) {
                TBShot& t = d[(size_t)v * nb + s];
                std::memset(&t, 0, sizeof(t));
                float* base = tbState.as<float>() + (size_t)s * 4 * g.isz;
                t.cur = base + (size_t)(2 * v) * g.isz;
                t.old = base + (size_t)(2 * v + 1) * g.isz;
                t.ncur = base + (size_t)(2 * (1 - v)) * g.isz;
                t.nold = base + (size_t)(2 * (1 - v) + 1) * g.isz;
                float* pb = tbPart.as<float>() + (size_t)s * 2 * g.isz;
                const int vin = partFlip ? (v ^ 1) : v;
                t.part = pb + (size_t)vin * g.isz;
                t.partOut = pb + (size_t)(1 - vin) * g.isz;
                t.injSig = injSources ? srcSig[s] : (injData ? (dataIn ? dataIn[s] : dataPtr[s]) : nullptr);
                t.injLd = injSources ? g.ntw : g.nts;
                t.recSig = recData ? dataPtr[s] : nullptr;
                t.recLd = g.nts;
                t.entStart = tbStart.as<int4>() + (size_t)s * nCTA;
                t.ent = tbEnt.as<TBEnt>();
                t.W = W ? (void*)((char*)W + (size_t)s * wSlices * g.isz * wElem) : nullptr;
                t.img = tbImg.p ? tbImg.as<double>() + (size_t)s * g.isz : nullptr;
                t.imgF = tbImg.p ? tbImg.as<float>() + (size_t)s * g.isz : nullptr;
                t.rcoarse = out ? out + (size_t)s * outSlices * g.isz : nullptr;
                if (f16()) {
                    t.wscale = tbWscale.as<float>() + (size_t)s * g.nts;
                    t.wmax = tbWmax.as<unsigned>() + (size_t)s * g.nts;
                    t.wstage = tbWstage.as<float>() + (size_t)s * 2 * g.isz;
                    t.wover = tbWover.as<unsigned>();
                }
            }
        AIO_CK(cudaMemcpyAsync(tbDesc.p, d.data(), d.size() * sizeof(TBShot), cudaMemcpyHostToDevice, st));
    }

    KTArgs tb_args(const TBPlan& pl, int maxEnt, const float* dm) const {
        KTArgs a;
        std::memset(&a, 0, sizeof(a));
        a.g = g;
        a.c = k.c;
        a.v2 = v2.as<float>();
        a.taper = taper.as<float>();
        a.dm = dm;
        std::copy(k.h, k.h + 2 * (SUB_MAX + 1), a.h);
        a.HZ = pl.HZ;
        a.LX = pl.LX;
        a.nStrips = pl.nStrips;
        a.nChunks = pl.nChunks;
        a.NQ = pl.NQ;
        a.iters = pl.iters;
        a.maxEnt = maxEnt;
        a.wStride = g.isz;
        a.imgF32 = P.imageFp64 ? 0 : 1;
        return a;
    }

    template <int MODE, int WP, int MAXQ, bool FS = false>
    void tb_launch_q(const TBPlan& pl, int nb, KTArgs& a, int v) {
        const size_t smem = kt_smem_bytes(MODE, pl.threads, pl.iters, a.maxEnt, kt_rs(MAXQ), kt_v2s(MAXQ));
        static int attrDev = -1;
        static int smemMax = 0;
        if (attrDev != dev) {
            AIO_CK(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            AIO_CK(cudaFuncSetAttribute(k_tile<MODE, WP, MAXQ, FS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smemMax));
            attrDev = dev;
        }
        require(smem <= (size_t)smemMax, "blocked stepper: shared memory plan of " + std::to_string(smem) +
                                             " bytes exceeds the device limit (too many devices per tile)");
        require(pl.NQ <= MAXQ && pl.threads <= (8 * MAXQ + 31) / 32 * 32, "blocked stepper: strip taller than the ring");
        a.shots = tbDesc.as<TBShot>() + (size_t)v * nb;
        tbLast = pl;
        const bool timed = profEvery > 0 && (launches % profEvery) == 0;
        std::pair<cudaEvent_t, cudaEvent_t> ev{};
        if (timed) {
            ev = take_events();
            AIO_CK(cudaEventRecord(ev.first, st));
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(pl.nStrips, pl.nChunks, nb);
        cfg.blockDim = dim3(pl.threads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        const int pm = pdl_mode();
        cfg.numAttrs = pm ? 1 : 0;
        a.relIter = pm == 1 ? 0 : pl.iters - 1;
        AIO_CK(cudaLaunchKernelEx(&cfg, k_tile<MODE, WP, MAXQ, FS>, a));
        if (timed) {
            AIO_CK(cudaEventRecord(ev.second, st));
            evBusy.push_back(ev);
            evPoints.push_back((long long)nb * g.nzi * g.nxi * pl.T);
        }
        launches++;
        kernels++;
    }
    // Short strips (<= 64 rows) and mid strips (<= 80 rows) use the variants with narrower
    // rings (two CTAs per SM); taller strips the large one.
    template <int MODE, int WP>
    void tb_launch_t(const TBPlan& pl, int nb, KTArgs& a, int v) {
        if (P.freeSurface) tb_launch_q<MODE, WP, KT_MAXQ, true>(pl, nb, a, v);
        else if (pl.NQ <= KT_MAXQ_S) tb_launch_q<MODE, WP, KT_MAXQ_S>(pl, nb, a, v);
        else if (pl.NQ <= KT_MAXQ_M) tb_launch_q<MODE, WP, KT_MAXQ_M>(pl, nb, a, v);
        else tb_launch_q<MODE, WP, KT_MAXQ>(pl, nb, a, v);
    }
    template <int MODE>
    void tb_launch(const TBPlan& pl, int nb, KTArgs& a, int v) {
        // the dense-source modes read FP32 rings of secondary sources, and the receiver-sample
        // pass reads no stored wavefield: those run on FP32 whatever the stored precision
        if (MODE == TB_SCATX || MODE == TB_SCATW || MODE == TB_ADJX || MODE == TB_ADJR) tb_launch_t<MODE, TBW_F32>(pl, nb, a, v);
        else if (P.wavefieldPrecision == AIO_WFLD_BF16) tb_launch_t<MODE, TBW_BF16>(pl, nb, a, v);
        else if (P.wavefieldPrecision == AIO_WFLD_FP16) tb_launch_t<MODE, TBW_F16>(pl, nb, a, v);
        else tb_launch_t<MODE, TBW_F32>(pl, nb, a, v);
    }

    void tb_zero(int nb, bool img) {
        AIO_CK(cudaMemsetAsync(tbState.p, 0, (size_t)nb * 4 * g.isz * 4, st));
        AIO_CK(cudaMemsetAsync(tbPart.p, 0, (size_t)nb * 2 * g.isz * 4, st));
        if (img) AIO_CK(cudaMemsetAsync(tbImg.p, 0, (size_t)nb * g.isz * 8, st));
    }

    // Source pass storing W[nts] (F/src/BornShotsGpuFunctions.cu:297-321), or the
    // nonlinear forward when recordData (F/src/nonlinearShotsGpuFunctions.cu:269-295).
    // FP16 stored wavefield: slices are stored with speculative power-of-two scales from the
    // previous slice's max (kt_f16_spec_scale); if any slice outgrew its scale's headroom the
    // pass is run again with every slice staged in FP32 and quantized with its exact max.
    void tb_src_pass(int nb, const aio_shot* shots, bool nonlinear, bool exactF16 = false) {
        tb_autotune(nb, shots, nonlinear);
        const TBPlan pl = nonlinear ? tb_plan_c(nb, TB_NLC) : tb_plan(nb);
        const int maxEnt = tb_lists(pl, nb, shots, 1, nonlinear);
        tb_zero(nb, false);
        tb_desc(pl, nb, true, false, nonlinear, nonlinear ? nullptr : tbW.p, false);
        KTArgs a = tb_args(pl, maxEnt, nullptr);
        const bool spec = !nonlinear && f16() && !exactF16;
        a.f16spec = spec ? 1 : 0;
        if (!nonlinear && f16()) AIO_CK(cudaMemsetAsync(tbWmax.p, 0, (size_t)nb * g.nts * 4, st));
        if (spec) AIO_CK(cudaMemsetAsync(tbWover.p, 0, 4, st));
        tbLast = pl;
        graph_loop({1, nonlinear, nb, pl.HZ, pl.nStrips, pl.LX, pl.nChunks, maxEnt, (long long)tbDesc.p,
                    (long long)tbW.p, a.f16spec, P.wavefieldPrecision},
                   [&] {
                       for (int its = 0; its < g.nts - 1; its++) {
                           a.its = its;
                           if (nonlinear) tb_launch<TB_NL>(pl, nb, a, its & 1);
                           else tb_launch<TB_SRC>(pl, nb, a, its & 1);
                       }
                   });
        if (!nonlinear && f16()) {  // last two slices and the per-slice scales
            k_f16_finish<<<dim3(std::max(1, smCount), nb), 256, 0, st>>>(tbDesc.as<TBShot>(), g.isz, g.ip, g.nzi,
                                                                          g.nxi, g.nts, a.f16spec);
            kcheck();
        }
        if (spec) {
            unsigned over = 0;
            AIO_CK(cudaMemcpyAsync(&over, tbWover.p, 4, cudaMemcpyDeviceToHost, st));
            AIO_CK(cudaStreamSynchronize(st));
            f16Reruns += over ? 1 : 0;
            if (over) tb_src_pass(nb, shots, nonlinear, true);
        }
    }
    long long f16Reruns = 0;  // FP16 source passes run again with exact scales (speculative overflow)

    // Scattered pass with data recording (F/src/BornShotsGpuFunctions.cu:323-376); W: the stored
    // field the secondary sources dm * W come from (default: the source wavefield tbW).
    // A caller's W (the tomo forward's scattered field) is FP32 whatever the stored precision.
    void tb_scat_pass(int nb, const aio_shot* shots, const float* dm, const float* W = nullptr) {
        const TBPlan pl = tb_plan(nb, true);
        const int maxEnt = tb_lists(pl, nb, shots, 0, true);
        tb_zero(nb, false);
        tb_desc(pl, nb, false, false, true, W ? (void*)W : tbW.p, false, W ? g.nts : 0);
        KTArgs a = tb_args(pl, maxEnt, dm);
        tbLast = pl;
        graph_loop({2, nb, pl.HZ, pl.nStrips, pl.LX, pl.nChunks, maxEnt, (long long)tbDesc.p, (long long)dm,
                    (long long)(W ? (const void*)W : tbW.p), P.wavefieldPrecision},
                   [&] {
                       for (int its = 0; its < g.nts - 1; its++) {
                           a.its = its;
                           if (W) tb_launch_t<TB_SCAT, TBW_F32>(pl, nb, a, its & 1);
                           else tb_launch<TB_SCAT>(pl, nb, a, its & 1);
                       }
                   });
    }

    // Receiver pass with imaging (F/src/BornShotsGpuFunctions.cu:880-950), on U = v2*p.
    // Launch L handles interval its = nts-2-L: it reads the partial R(its+1) written by
    // launch L-1 and writes R(its); state ping-pongs with L.
    void tb_adj_pass(int nb, const aio_shot* shots) {
        const TBPlan pl = tb_plan_c(nb, TB_RECV);
        const int maxEnt = tb_lists(pl, nb, shots, 2, false);
        tb_zero(nb, true);
        tb_desc(pl, nb, false, true, false, tbW.p, false);
        KTArgs a = tb_args(pl, maxEnt, nullptr);
        tbLast = pl;
        graph_loop({3, nb, pl.HZ, pl.nStrips, pl.LX, pl.nChunks, maxEnt, (long long)tbDesc.p, (long long)tbW.p,
                    P.wavefieldPrecision},
                   [&] {
                       for (int L = 0; L < g.nts - 1; L++) {
                           a.its = g.nts - 2 - L;
                           tb_launch<TB_ADJ>(pl, nb, a, L & 1);
                       }
                   });
    }

    // Receiver pass of the extended (time-lag) adjoint (F/src/BornExtShotsGpuFunctions.cu:1525-1675)
    // on the blocked stepper: launch L (interval its = nts-2-L) finishes the coarse receiver
    // sample R(its+1) (and R(0) at its == 0) into a ring of LAG_K slices; each time the lowest
    // sample of a block [bK, bK+K) has arrived, k_img_lag_block correlates the block with the
    // stored wavefield (imagingTimeAdjGpu, F/src/kernelsGpu.cu:352-364, for every t of it), or
    // with subsurface offsets k_img_offset_block (imagingOffsetAdjGpu, :397-411).
    void tb_adjx_pass(int nb, const aio_shot* shots) {
        const TBPlan pl = tb_plan(nb);
        const int maxEnt = tb_lists(pl, nb, shots, 2, false);
        tb_zero(nb, false);
        tb_desc(pl, nb, false, true, false, tbW.p, false);
        KTArgs a = tb_args(pl, maxEnt, nullptr);
        const long long mSt = (long long)g.nExt * g.isz;
        const int nP = LAG_NP;
        const size_t lagSmem = (size_t)lag_window_len(g.hExt) * nP * 4;
        static int lagAttr = -1;
        if (lagAttr != dev) {
            AIO_CK(cudaFuncSetAttribute(k_img_lag_block<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_img_lag_block<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_img_lag_block<double, TBW_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_img_lag_block<float, TBW_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_img_lag_block<double, TBW_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_img_lag_block<float, TBW_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            lagAttr = dev;
        }
        require(offsets() || lagSmem <= 200 * 1024, "extension too long for the blocked lag imaging");
        auto image = [&](int tlo, int thi) {
            if (offsets()) {
                // subsurface offsets (BornOffsetShotsAdjGpu, F/src/BornExtShotsGpuFunctions.cu:1848-1990):
                // U-form samples carry the v2 of scaleSecondarySourceFd already
                const long long RSt = (long long)LAG_K * g.isz;
                if (P.imageFp64)
                    k_img_offset_block<double><<<ew_grid(nb, g.isz), 256, 0, st>>>(
                        img.as<double>(), mSt, tbR.as<float>(), RSt, tbW.as<float>(), wfSt(), nullptr, (int)g.isz,
                        g.ip, g.nxi, g.hExt, g.nExt, tlo, thi, 0);
                else
                    k_img_offset_block<float><<<ew_grid(nb, g.isz), 256, 0, st>>>(
                        img.as<float>(), mSt, tbR.as<float>(), RSt, tbW.as<float>(), wfSt(), nullptr, (int)g.isz,
                        g.ip, g.nxi, g.hExt, g.nExt, tlo, thi, 0);
                kcheck();
                return;
            }
            const dim3 grid((unsigned)((g.isz + nP - 1) / nP), nb);
            const long long rSt = (long long)LAG_K * g.isz;
            const float* sc = f16() ? tbWscale.as<float>() : nullptr;
#define AIO_LAG_IMG(ACC, WP)                                                                                          \
    k_img_lag_block<ACC, WP><<<grid, nP, lagSmem, st>>>(img.as<ACC>(), mSt, tbR.as<float>(), rSt, LAG_K, tbW.p, wfSt(), \
                                                        g.isz, tlo, thi, g.nts, g.hExt, g.nExt, 1, sc)
            if (P.wavefieldPrecision == AIO_WFLD_BF16) {
                if (P.imageFp64) AIO_LAG_IMG(double, TBW_BF16);
                else AIO_LAG_IMG(float, TBW_BF16);
            } else if (f16()) {
                if (P.imageFp64) AIO_LAG_IMG(double, TBW_F16);
                else AIO_LAG_IMG(float, TBW_F16);
            } else {
                if (P.imageFp64) AIO_LAG_IMG(double, TBW_F32);
                else AIO_LAG_IMG(float, TBW_F32);
            }
#undef AIO_LAG_IMG
            kcheck();
        };
        for (int L = 0; L < g.nts - 1; L++) {
            a.its = g.nts - 2 - L;
            const int t = a.its + 1;
            a.rSlot = t % LAG_K;
            a.rSlot0 = 0;
            tb_launch<TB_ADJR>(pl, nb, a, L & 1);
            if (a.its == 0) image(0, std::min(LAG_K - 1, g.nts - 1));
            else if (t % LAG_K == 0) image(t, std::min(t + LAG_K - 1, g.nts - 1));
        }
    }

    // Scattered pass of the extended (time-lag) forward (F/src/BornExtShotsGpuFunctions.cu:269-419)
    // on the blocked stepper: the secondary sources ss(t) = sum_e ext[e] W[t - 2(e-h)] are formed
    // for blocks of LAG_K coarse steps ahead of use (k_ss_lag_block) into a ring of 2 LAG_K slices,
    // read by TB_SCATX at slots its and its+1.
    void tb_scatx_pass(int nb, const aio_shot* shots, const float* ext, const float* F = nullptr) {
        const int ring = 2 * LAG_K;
        const TBPlan pl = tb_plan(nb, true);
        const int maxEnt = tb_lists(pl, nb, shots, 0, true);
        tb_zero(nb, false);
        tb_desc(pl, nb, false, false, true, tbSS.p, false, ring);
        KTArgs a = tb_args(pl, maxEnt, nullptr);
        const int nP = LAG_NP;
        const size_t lagSmem = (size_t)lag_window_len(g.hExt) * nP * 4;
        static int ssAttr = -1;
        if (ssAttr != dev) {
            AIO_CK(cudaFuncSetAttribute(k_ss_lag_block<TBW_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_ss_lag_block<TBW_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            AIO_CK(cudaFuncSetAttribute(k_ss_lag_block<TBW_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            ssAttr = dev;
        }
        require(offsets() || lagSmem <= 200 * 1024, "extension too long for the blocked lag imaging");
        auto sources = [&](int tlo) {
            const int thi = std::min(tlo + LAG_K - 1, g.nts - 1);
            if (offsets()) {
                // subsurface offsets (imagingOffsetFwdGpu + scaleSecondarySourceFd): one slice per
                // sample, formed into the zeroed ring slots of the block
                const long long rSt = (long long)ring * g.isz;
                AIO_CK(cudaMemset2DAsync(tbSS.as<float>() + (long long)(tlo % ring) * g.isz, (size_t)rSt * 4, 0,
                                         (size_t)(thi - tlo + 1) * g.isz * 4, nb, st));
                const float* Fs = F ? F : tbW.as<float>();
                for (int t = tlo; t <= thi; t++)
                    k_img_offset_fwd<<<ew_grid(nb, g.isz), 256, 0, st>>>(
                        tbSS.as<float>() + (long long)(t % ring) * g.isz, rSt, ext, 0, Fs + (long long)t * g.isz,
                        wfSt(), v2.as<float>(), g.isz, g.ip, g.nxi, g.hExt);
                kcheck();
                return;
            }
            const dim3 grid((unsigned)((g.isz + nP - 1) / nP), nb);
            // F (a caller's FP32 field) or the stored source wavefield in its precision
            const int wp = F ? AIO_WFLD_FP32 : P.wavefieldPrecision;
            const void* Ws = F ? (const void*)F : tbW.p;
            const float* sc = (!F && f16()) ? tbWscale.as<float>() : nullptr;
            if (wp == AIO_WFLD_BF16)
                k_ss_lag_block<TBW_BF16><<<grid, nP, lagSmem, st>>>(tbSS.as<float>(), (long long)ring * g.isz, ring, ext,
                                                                    Ws, wfSt(), g.isz, tlo, thi, g.nts, g.hExt, g.nExt,
                                                                    1, sc);
            else if (wp == AIO_WFLD_FP16)
                k_ss_lag_block<TBW_F16><<<grid, nP, lagSmem, st>>>(tbSS.as<float>(), (long long)ring * g.isz, ring, ext,
                                                                   Ws, wfSt(), g.isz, tlo, thi, g.nts, g.hExt, g.nExt,
                                                                   1, sc);
            else
                k_ss_lag_block<TBW_F32><<<grid, nP, lagSmem, st>>>(tbSS.as<float>(), (long long)ring * g.isz, ring, ext,
                                                                   Ws, wfSt(), g.isz, tlo, thi, g.nts, g.hExt, g.nExt,
                                                                   1, sc);
            kcheck();
        };
        for (int its = 0; its < g.nts - 1; its++) {
            if (its == 0) sources(0);
            if ((its + 1) % LAG_K == 0) sources(its + 1);  // next block, before ss(its+1) is read
            a.its = its;
            a.rSlot = its % ring;
            a.rSlot0 = (its + 1) % ring;
            tb_launch<TB_SCATX>(pl, nb, a, its & 1);
        }
    }

    void born_ext_forward_tb(const float* model, int nShots, const aio_shot* shots, int mem) {
        float* ext = stage_model(model, g.nExt, mem, this->model);
        // subsurface offsets: 2/v^3 only, v^2 applied to each secondary-source slice
        scale_shared(ext, g.nExt, offsets() ? 3 : (P.sloth ? 2 : 1));
        Needs n;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_wave_size(nShots - s0, shots + s0, true, false);
            setup_wave(n, nb, shots + s0, mem, false, false);
            tb_alloc(nb, false);
            tbW.ensure((size_t)nb * g.nts * g.isz * wbytes());
            tbSS.ensure((size_t)nb * 2 * LAG_K * g.isz * 4);
            tb_src_pass(nb, shots + s0, false);
            tb_scatx_pass(nb, shots + s0, ext);
            download_data(nb, shots + s0, mem);
            sync();
            s0 += nb;
        }
    }

    void born_ext_adjoint_tb(float* modelOut, int add, int nShots, const aio_shot* shots, int mem) {
        require(P.wavefieldPrecision == AIO_WFLD_FP32 || !offsets(),
                "the subsurface-offset extension keeps the stored wavefield in FP32 (wavefieldPrecision)");
        Needs n;
        n.nImg = g.nExt;
        float* out = stage_out(modelOut, g.nExt, add, mem);
        for (int s0 = 0; s0 < nShots;) {
            int nb = tb_wave_size(nShots - s0, shots + s0, true, false);
            // extended images: nExt slices per shot
            const long long perImg = (long long)g.nExt * g.isz * (P.imageFp64 ? 8 : 4) + (long long)LAG_K * g.isz * 4;
            nb = std::max(1, std::min<int>(nb, (int)std::max<long long>(1, (budget / 2) / perImg)));
            setup_wave(n, nb, shots + s0, mem, true, false);
            tb_alloc(nb, false);
            tbW.ensure((size_t)nb * g.nts * g.isz * wbytes());
            tbR.ensure((size_t)nb * LAG_K * g.isz * 4);
            tb_src_pass(nb, shots + s0, false);
            zero_images(nb, g.nExt);
            tb_adjx_pass(nb, shots + s0);
            // images of U = v2 * receiver wavefield: the reference's rs*v2 scaling reduces to rs,
            // the sloth scaling -(m*v2) to a sign change; subsurface offsets: rs (2/v^3) only, the
            // v2 of their scaleSecondarySourceFd being the one U carries
            reduce_images(nb, g.nExt, (P.sloth && !offsets()) ? 4 : 3, out, true);
            sync();
            s0 += nb;
        }
        write_model(modelOut, g.nExt, add, mem, out);
        sync();
    }

    // ------------------------------------------- tomo / WEMVA on the blocked stepper
    // Every leg is one blocked pass. Receiver-side fields are kept in U-form (U = v2 * S, the
    // adjoint recursion of TB_ADJR / TB_ADJX), so secondary sources built from them already
    // carry the v2 of U-form injection and every image term (one source-side factor, one
    // receiver-side factor) carries v2 once: reduce_images divides it out (scaling mode 5).
    static constexpr int TB_RING = 2 * LAG_K;  // source and sample rings: two blocks of LAG_K

    struct TBSrc {                // dense secondary sources of a pass
        const void* F = nullptr;    // full coarse field [shot][nts][isz], precision wp
        const float* ext = nullptr; // lag sources ss(t) = sum_e ext[e] F[t - sign 2(e-h)]; null: F (times dm)
        const float* dm = nullptr;  // zero-lag sources: dm * F(t) (null: F(t))
        int sign = 1;
        int wp = TBW_F32;           // F's precision: FP32, or the 16-bit source field (tbW, scales tbWscale)
    };
    struct TBOut {                // what a pass does with its coarse samples
        float* full = nullptr;      // store all of them [shot][nts][isz]
        const void* imgF = nullptr; // else image them against this full field (ring of TB_RING samples)
        bool lag = false;           // time-lag image (nExt slices) or zero-lag (one slice)
        int sign = 1;
        int wp = TBW_F32;           // imgF's precision (as TBSrc::wp)
    };
    // precision of the tomo / WEMVA source field d2/dt2 (tbW) on the blocked stepper: the stored
    // precision (16-bit with per-slice scales for FP16)
    int src_wp() const {
        return P.wavefieldPrecision == AIO_WFLD_BF16 ? TBW_BF16 : (P.wavefieldPrecision == AIO_WFLD_FP16 ? TBW_F16 : TBW_F32);
    }

    void tb_lag_attr() {
        static int lagDev = -1;
        if (lagDev == dev) return;
        const int b = 200 * 1024;
        AIO_CK(cudaFuncSetAttribute(k_img_lag_block<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_img_lag_block<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_img_lag_block<double, TBW_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_img_lag_block<float, TBW_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_img_lag_block<double, TBW_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_img_lag_block<float, TBW_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_ss_lag_block<TBW_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_ss_lag_block<TBW_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        AIO_CK(cudaFuncSetAttribute(k_ss_lag_block<TBW_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
        lagDev = dev;
    }
    size_t tb_lag_smem(int hExt) const {
        const size_t b = (size_t)lag_window_len(hExt) * LAG_NP * 4;
        require(b <= 200 * 1024, "extension too long for the blocked lag imaging");
        return b;
    }
    // secondary sources of the coarse steps [tlo, thi] into the ring tbSS
    void tb_ss_block(int nb, const TBSrc& src, int tlo, int thi) {
        tb_lag_attr();
        const int nP = LAG_NP;
        const dim3 grid((unsigned)((g.isz + nP - 1) / nP), nb);
        const size_t sm = tb_lag_smem(g.hExt);
        const long long rSt = (long long)TB_RING * g.isz;
        float* ss = tbSS.as<float>();
        if (src.wp == TBW_BF16)
            k_ss_lag_block<TBW_BF16><<<grid, nP, sm, st>>>(ss, rSt, TB_RING, src.ext, src.F, wfSt(), g.isz, tlo, thi,
                                                           g.nts, g.hExt, g.nExt, src.sign);
        else if (src.wp == TBW_F16)
            k_ss_lag_block<TBW_F16><<<grid, nP, sm, st>>>(ss, rSt, TB_RING, src.ext, src.F, wfSt(), g.isz, tlo, thi,
                                                          g.nts, g.hExt, g.nExt, src.sign, tbWscale.as<float>());
        else
            k_ss_lag_block<TBW_F32><<<grid, nP, sm, st>>>(ss, rSt, TB_RING, src.ext, src.F, wfSt(), g.isz, tlo, thi,
                                                          g.nts, g.hExt, g.nExt, src.sign);
        kcheck();
    }
    // image the samples [tlo, thi] of the ring tbR against out.imgF
    void tb_img_block(int nb, const TBOut& out, int tlo, int thi) {
        tb_lag_attr();
        const int nP = LAG_NP, nE = out.lag ? g.nExt : 1, hE = out.lag ? g.hExt : 0;
        const dim3 grid((unsigned)((g.isz + nP - 1) / nP), nb);
        const long long mSt = (long long)nE * g.isz, rSt = (long long)TB_RING * g.isz;
        const size_t sm = tb_lag_smem(hE);
        const float* R = tbR.as<float>();
        const float* sc = out.wp == TBW_F16 ? tbWscale.as<float>() : nullptr;
#define AIO_TB_IMG(ACC, WP)                                                                                         \
    k_img_lag_block<ACC, WP><<<grid, nP, sm, st>>>(img.as<ACC>(), mSt, R, rSt, TB_RING, out.imgF, wfSt(), g.isz, tlo, \
                                                   thi, g.nts, hE, nE, out.sign, sc)
        if (P.imageFp64) {
            if (out.wp == TBW_BF16) AIO_TB_IMG(double, TBW_BF16);
            else if (out.wp == TBW_F16) AIO_TB_IMG(double, TBW_F16);
            else AIO_TB_IMG(double, TBW_F32);
        } else {
            if (out.wp == TBW_BF16) AIO_TB_IMG(float, TBW_BF16);
            else if (out.wp == TBW_F16) AIO_TB_IMG(float, TBW_F16);
            else AIO_TB_IMG(float, TBW_F32);
        }
#undef AIO_TB_IMG
        kcheck();
    }

    // Forward-time dense pass (fwd_dense_pass on the blocked stepper, TB_SCATW):
    // F/src/tomoExtShotsGpuFunctions.cu:1554-1656,2442-2527, F/src/wemvaExtShotsGpuFunctions.cu:961-1037.
    // Lag sources are formed a block of LAG_K steps ahead; sample rings are imaged per block.
    void tb_dense_fwd(int nb, const aio_shot* shots, const TBSrc& src, const TBOut& out) {
        const TBPlan pl = tb_plan(nb, true);
        const int maxEnt = tb_lists(pl, nb, shots, 0, false);
        tb_zero(nb, false);
        const bool lagSrc = src.ext != nullptr;
        // zero-lag sources straight from a 16-bit source field: W is that field (wSlices 0: the
        // stored precision's element size), read with its per-slice scales
        const int wp = lagSrc ? TBW_F32 : src.wp;
        tb_desc(pl, nb, false, false, false, lagSrc ? tbSS.p : const_cast<void*>(src.F), false,
                lagSrc ? TB_RING : (wp == TBW_F32 ? g.nts : 0), out.full ? out.full : tbR.as<float>(),
                out.full ? g.nts : TB_RING);
        KTArgs a = tb_args(pl, maxEnt, lagSrc ? nullptr : src.dm);
        int lo = 0;  // lowest sample not yet imaged
        for (int its = 0; its < g.nts - 1; its++) {
            if (lagSrc) {
                if (its == 0) tb_ss_block(nb, src, 0, std::min(LAG_K - 1, g.nts - 1));
                if ((its + 1) % LAG_K == 0) tb_ss_block(nb, src, its + 1, std::min(its + LAG_K, g.nts - 1));
                a.rSlot = its % TB_RING;
                a.rSlot0 = (its + 1) % TB_RING;
            } else {
                a.rSlot = its;
                a.rSlot0 = its + 1;
            }
            a.oA = out.full ? its : its % TB_RING;
            a.oB = out.full ? its + 1 : (its + 1) % TB_RING;
            a.its = its;
            if (wp == TBW_BF16) tb_launch_t<TB_SCATW, TBW_BF16>(pl, nb, a, its & 1);
            else if (wp == TBW_F16) tb_launch_t<TB_SCATW, TBW_F16>(pl, nb, a, its & 1);
            else tb_launch_t<TB_SCATW, TBW_F32>(pl, nb, a, its & 1);
            if (!out.full) {
                if ((its + 1) % LAG_K == 0) {
                    tb_img_block(nb, out, lo, its);
                    lo = its + 1;
                }
                if (its == g.nts - 2) tb_img_block(nb, out, lo, g.nts - 1);
            }
        }
    }

    // Adjoint-time dense pass (adj_dense_pass on the blocked stepper, TB_ADJX) on U-form sources:
    // F/src/tomoExtShotsGpuFunctions.cu:2619-2700, F/src/wemvaExtShotsGpuFunctions.cu:1038-1121.
    void tb_dense_adj(int nb, const aio_shot* shots, const TBSrc& src, const TBOut& out) {
        const TBPlan pl = tb_plan(nb, true);
        const int maxEnt = tb_lists(pl, nb, shots, 0, false);
        tb_zero(nb, false);
        const bool lagSrc = src.ext != nullptr;
        require(lagSrc || src.wp == TBW_F32, "adjoint dense pass: zero-lag sources come from an FP32 field");
        tb_desc(pl, nb, false, false, false, lagSrc ? tbSS.p : const_cast<void*>(src.F), false,
                lagSrc ? TB_RING : g.nts, out.full ? out.full : tbR.as<float>(), out.full ? g.nts : TB_RING);
        KTArgs a = tb_args(pl, maxEnt, lagSrc ? nullptr : src.dm);
        int srcLo = g.nts;   // lowest source sample in the ring
        int hi = g.nts - 1;  // highest sample not yet imaged
        for (int L = 0; L < g.nts - 1; L++) {
            const int its = g.nts - 2 - L;
            if (lagSrc) {
                while (srcLo > its) {  // the blocks holding ss(its) and ss(its+1)
                    const int b = (srcLo - 1) / LAG_K * LAG_K;
                    tb_ss_block(nb, src, b, srcLo - 1);
                    srcLo = b;
                }
                a.rSlot = its % TB_RING;
                a.rSlot0 = (its + 1) % TB_RING;
            } else {
                a.rSlot = its;
                a.rSlot0 = its + 1;
            }
            a.oA = 0;
            a.oB = out.full ? its + 1 : (its + 1) % TB_RING;
            a.its = its;
            tb_launch_t<TB_ADJX, TBW_F32>(pl, nb, a, L & 1);
            if (!out.full) {
                const int t = its + 1;
                if (t % LAG_K == 0) {
                    tb_img_block(nb, out, t, hi);
                    hi = t - 1;
                }
                if (its == 0) tb_img_block(nb, out, 0, hi);
            }
        }
    }

    // Receiver wavefield in U-form, every coarse sample stored (computeTomoRecWfld,
    // F/src/tomoExtShotsGpuFunctions.cu:1481-1515, on TB_ADJR).
    void tb_rec_full(int nb, const aio_shot* shots, const float* const* data, float* R) {
        const TBPlan pl = tb_plan(nb);
        const int maxEnt = tb_lists(pl, nb, shots, 2, false);
        tb_zero(nb, false);
        tb_desc(pl, nb, false, true, false, nullptr, false, 0, R, g.nts, data);
        KTArgs a = tb_args(pl, maxEnt, nullptr);
        for (int L = 0; L < g.nts - 1; L++) {
            a.its = g.nts - 2 - L;
            a.rSlot = a.its + 1;
            a.rSlot0 = 0;
            tb_launch_t<TB_ADJR, TBW_F32>(pl, nb, a, L & 1);
        }
    }

    // Source wavefield and its second time derivative (computeTomoSrcWfldDt2,
    // F/src/tomoExtShotsGpuFunctions.cu:1251-1361) into tbW, in the stored precision.
    void tb_src_dt2(int nb, const aio_shot* shots) {
        if (src_wp() != TBW_F32) return tb_src_dt2_16(nb, shots);
        tb_src_pass(nb, shots, false);
        k_dt2<<<ew_grid(nb, g.isz), 256, 0, st>>>(tbW.as<float>(), wfSt(), g.isz, g.nts, k.cSide, k.cCenter);
        kcheck();
    }
    // 16-bit source field: the source pass stores W in an FP32 ring of TB_RING slices (tbSS, which
    // the legs use only later), and once a block of KT_DT2_B slices of d2/dt2 can be formed
    // (W one slice past it is final) k_dt2_block forms it with k_dt2's expression: BF16 stored
    // directly; FP16 staged in FP32 (tbR, also free until the legs) and quantized with each
    // slice's exact unit (max / 2^15). The FP32 field of nts slices is never held.
    void tb_src_dt2_16(int nb, const aio_shot* shots) {
        static_assert(TB_RING >= 2 * KT_DT2_B, "the block reads the slice before it and the slice after it");
        tb_autotune(nb, shots, false);
        const TBPlan pl = tb_plan(nb);
        const int maxEnt = tb_lists(pl, nb, shots, 1, false);
        tb_zero(nb, false);
        tb_desc(pl, nb, true, false, false, tbSS.p, false, TB_RING);
        KTArgs a = tb_args(pl, maxEnt, nullptr);
        a.wRing = TB_RING;
        const int wp = src_wp();
        if (wp == TBW_F16) AIO_CK(cudaMemsetAsync(tbWmax.p, 0, (size_t)nb * g.nts * 4, st));
        const long long rSt = (long long)TB_RING * g.isz;
        const dim3 grid((unsigned)std::max(1, 2 * smCount), nb);
        auto block = [&](int t0, int t1) {
            if (wp == TBW_BF16) {
                k_dt2_block<TBW_BF16><<<grid, 256, 0, st>>>(tbSS.as<float>(), rSt, TB_RING, tbW.p, wfSt(), nullptr, 0,
                                                            nullptr, g.nts, g.isz, t0, t1, k.cSide, k.cCenter);
                kcheck();
                return;
            }
            k_dt2_block<TBW_F16><<<grid, 256, 0, st>>>(tbSS.as<float>(), rSt, TB_RING, tbW.p, wfSt(), tbR.as<float>(),
                                                       rSt, tbWmax.as<unsigned>(), g.nts, g.isz, t0, t1, k.cSide,
                                                       k.cCenter);
            kcheck();
            k_dt2_f16_pack<<<grid, 256, 0, st>>>(tbR.as<float>(), rSt, tbW.p, wfSt(), tbWmax.as<unsigned>(),
                                                 tbWscale.as<float>(), g.nts, g.isz, t0, t1);
            kcheck();
        };
        tbLast = pl;
        graph_loop({11, nb, pl.HZ, pl.nStrips, pl.LX, pl.nChunks, maxEnt, (long long)tbDesc.p, (long long)tbSS.p,
                    (long long)tbW.p, (long long)tbR.p, wp},
                   [&] {
                       int lo = 0;  // first slice of d2/dt2 not yet formed
                       for (int its = 0; its < g.nts - 1; its++) {
                           a.its = its;
                           tb_launch_t<TB_SRC, TBW_F32>(pl, nb, a, its & 1);
                           // W[its] is final (and W[nts-1] after the last launch): d2/dt2 of the
                           // slices up to `ready` can be formed
                           const bool last = its == g.nts - 2;
                           const int ready = last ? g.nts - 1 : its - 1;
                           while (ready - lo + 1 >= KT_DT2_B || (last && lo <= ready)) {
                               const int t1 = std::min(lo + KT_DT2_B - 1, ready);
                               block(lo, t1);
                               lo = t1 + 1;
                           }
                       }
                   });
    }

    // Shots per wave with two full coarse fields, the rings and imgSlices image slices per shot.
    int tb_fields_wave(int nShots, const aio_shot* shots, int imgSlices) {
        int maxSrc = 1, maxRec = 1;
        for (int s = 0; s < nShots; s++) {
            maxSrc = std::max(maxSrc, shots[s].nSourcesReg);
            maxRec = std::max(maxRec, shots[s].nReceiversReg);
        }
        // the source field in the stored precision (16-bit with nts FP32 scales and maxima), the
        // second field in FP32
        const long long wsrc = (long long)g.nts * g.isz * (src_wp() == TBW_F32 ? 4 : 2) + 8LL * g.nts;
        const long long per = 6LL * g.isz * 4 + wsrc + (long long)g.nts * g.isz * 4 + 2LL * TB_RING * g.isz * 4 +
                              (long long)imgSlices * g.isz * (P.imageFp64 ? 8 : 4) + (long long)maxSrc * g.ntw * 4 +
                              2LL * maxRec * g.nts * 4 + 2 * g.hsz * 4 + 2 * g.isz * 4 + (1 << 16);
        const long long shared = (4LL + 2 * g.nExt) * g.isz * 4 + (64LL << 20);
        const long long cap = (budget - shared) / per;
        require(cap >= 1, "device memory budget cannot hold one shot for this operator");
        return balanced_wave(cap, nShots);
    }
    void tb_fields_alloc(int nb) {
        tb_alloc(nb, false);
        tbW.ensure((size_t)nb * g.nts * g.isz * (src_wp() == TBW_F32 ? 4 : 2));
        tbF2.ensure((size_t)nb * g.nts * g.isz * 4);
        tbSS.ensure((size_t)nb * TB_RING * g.isz * 4);
        tbR.ensure((size_t)nb * TB_RING * g.isz * 4);
    }

    // Extended tomo forward (F/src/tomoExtShotsGpuFunctions.cu:355-465, legs :1554-1881).
    void tomo_forward_tb(const float* dm, const float* ex, int nShots, const aio_shot* shots, int mem) {
        Needs n;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_fields_wave(nShots - s0, shots + s0, 0);
            setup_wave(n, nb, shots + s0, mem, false, false);
            tb_fields_alloc(nb);
            tb_src_dt2(nb, shots + s0);
            const void* W2 = tbW.p;  // d2/dt2 of the source wavefield, stored precision wp
            const int wp = src_wp();
            float* W1 = tbF2.as<float>();
            if (P.leg1) {
                tb_dense_fwd(nb, shots + s0, TBSrc{W2, ex, nullptr, 1, wp}, TBOut{W1});
                tb_scat_pass(nb, shots + s0, dm, W1);
            }
            if (P.leg2) {
                tb_dense_fwd(nb, shots + s0, TBSrc{W2, nullptr, dm, 1, wp}, TBOut{W1});
                tb_scatx_pass(nb, shots + s0, ex, W1);
            }
            download_data(nb, shots + s0, mem);
            sync();
            s0 += nb;
        }
    }

    // Extended tomo adjoint (F/src/tomoExtShotsGpuFunctions.cu:797-910, legs :2442-2701).
    void tomo_adjoint_tb(float* out, const float* ex, int nShots, const aio_shot* shots, int mem) {
        Needs n;
        n.nImg = 1;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_fields_wave(nShots - s0, shots + s0, 1);
            setup_wave(n, nb, shots + s0, mem, true, false);
            tb_fields_alloc(nb);
            tb_src_dt2(nb, shots + s0);
            const void* W2 = tbW.p;
            const int wp = src_wp();
            float* R = tbF2.as<float>();
            std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
            tb_rec_full(nb, shots + s0, din.data(), R);
            zero_images(nb, 1);
            if (P.leg1) tb_dense_fwd(nb, shots + s0, TBSrc{W2, ex, nullptr, 1, wp}, TBOut{nullptr, R, false, 1});
            if (P.leg2) tb_dense_adj(nb, shots + s0, TBSrc{R, ex, nullptr, -1}, TBOut{nullptr, W2, false, 1, wp});
            reduce_images(nb, 1, 5, out, true);
            sync();
            s0 += nb;
        }
    }

    // Extended WEMVA forward (F/src/wemvaExtShotsGpuFunctions.cu:344-456, legs :961-1122).
    void wemva_forward_tb(const float* dm, float* out, int nShots, const aio_shot* shots, int mem) {
        Needs n;
        n.nImg = g.nExt;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_fields_wave(nShots - s0, shots + s0, g.nExt);
            setup_wave(n, nb, shots + s0, mem, false, true);
            tb_fields_alloc(nb);
            tb_src_dt2(nb, shots + s0);
            const void* W2 = tbW.p;
            const int wp = src_wp();
            float* R = tbF2.as<float>();
            tb_rec_full(nb, shots + s0, wdataPtr.data(), R);
            zero_images(nb, g.nExt);
            if (P.leg1) tb_dense_fwd(nb, shots + s0, TBSrc{W2, nullptr, dm, 1, wp}, TBOut{nullptr, R, true, -1});
            if (P.leg2) tb_dense_adj(nb, shots + s0, TBSrc{R, nullptr, dm, 1}, TBOut{nullptr, W2, true, 1, wp});
            reduce_images(nb, g.nExt, 5, out, true);
            sync();
            s0 += nb;
        }
    }

    // Extended WEMVA adjoint (F/src/wemvaExtShotsGpuFunctions.cu:575-688, legs :1270-1426).
    void wemva_adjoint_tb(float* out, const float* im, int nShots, const aio_shot* shots, int mem) {
        Needs n;
        n.nImg = 1;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_fields_wave(nShots - s0, shots + s0, 1);
            setup_wave(n, nb, shots + s0, mem, false, true);
            tb_fields_alloc(nb);
            tb_src_dt2(nb, shots + s0);
            const void* W2 = tbW.p;
            const int wp = src_wp();
            float* R = tbF2.as<float>();
            tb_rec_full(nb, shots + s0, wdataPtr.data(), R);
            zero_images(nb, 1);
            if (P.leg1) tb_dense_adj(nb, shots + s0, TBSrc{R, im, nullptr, -1}, TBOut{nullptr, W2, false, 1, wp});
            if (P.leg2) tb_dense_fwd(nb, shots + s0, TBSrc{W2, im, nullptr, 1, wp}, TBOut{nullptr, R, false, 1});
            reduce_images(nb, 1, 5, out, true);
            sync();
            s0 += nb;
        }
    }

    // ============================================================ operators

    // Nonlinear forward (F/src/nonlinearShotsGpuFunctions.cu:227-309; with a
    // wavefield, :310-395 — only a batch of one shot returns it).
    void nonlinear_forward(int nShots, const aio_shot* shots, int mem, float* wavefieldOut) {
        begin_call();
        if (tb_enabled() && !wavefieldOut) return nonlinear_forward_tb(nShots, shots, mem);
        Needs n;
        n.nWavefields = wavefieldOut ? 1 : 0;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, false, false);
            fwd_sparse_pass(nb, true, wavefieldOut ? &wf1 : nullptr);
            download_data(nb, shots + s0, mem);
            if (wavefieldOut) download_wavefield(wavefieldOut, wf1.as<float>());
            sync();
            s0 += nb;
        }
    }

    // Nonlinear adjoint (F/src/nonlinearShotsGpuFunctions.cu:579-652 / :653-737).
    void nonlinear_adjoint(int nShots, const aio_shot* shots, int mem, float* wavefieldOut) {
        begin_call();
        Needs n;
        n.nWavefields = wavefieldOut ? 1 : 0;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, true, false);
            std::vector<float*> srcOut(nb);
            std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
            // source traces output: staged in the `sig` buffer (host) or caller memory (device)
            for (int s = 0; s < nb; s++) {
                const aio_shot& sh = shots[s0 + s];
                float* o = mem == AIO_MEM_HOST ? const_cast<float*>(srcSig[s]) : sh.sourcesOut;
                require(o != nullptr || sh.nSourcesReg == 0, "nonlinear adjoint output traces missing");
                if (sh.nSourcesReg > 0) AIO_CK(cudaMemsetAsync(o, 0, (size_t)sh.nSourcesReg * g.ntw * 4, st));
                srcOut[s] = o;
            }
            adj_sparse_pass(nb, din, &srcOut, wavefieldOut ? ACC_FULL : ACC_NONE, wavefieldOut ? &wf1 : nullptr,
                            [](int, long long) {});
            if (mem == AIO_MEM_HOST)
                for (int s = 0; s < nb; s++) {
                    const aio_shot& sh = shots[s0 + s];
                    if (sh.nSourcesReg > 0)
                        AIO_CK(cudaMemcpyAsync(sh.sourcesOut, srcOut[s], (size_t)sh.nSourcesReg * g.ntw * 4,
                                               cudaMemcpyDeviceToHost, st));
                }
            if (wavefieldOut) download_wavefield(wavefieldOut, wf1.as<float>());
            sync();
            s0 += nb;
        }
    }

    void download_wavefield(float* host, const float* dev) {
        // interior pitched [nts] slices -> full [nts][nx][nz] host array (zero outside interior)
        std::memset(host, 0, (size_t)g.nts * g.nz * g.nx * 4);
        for (int t = 0; t < g.nts; t++)
            AIO_CK(cudaMemcpy2DAsync(host + (long long)t * g.nz * g.nx + (long long)FAT * g.nz + FAT, (size_t)g.nz * 4,
                                     dev + (long long)t * g.isz, (size_t)g.ip * 4, (size_t)g.nzi * 4, g.nxi,
                                     cudaMemcpyDeviceToHost, st));
    }


    // Wave sizing for the blocked stepper: per shot 4 state + 2 partial slices,
    // the stored wavefield, an FP64 image, traces.
    int tb_wave_size(int nShots, const aio_shot* shots, bool wavefield, bool image) {
        int maxSrc = 1, maxRec = 1;
        for (int s = 0; s < nShots; s++) {
            maxSrc = std::max(maxSrc, shots[s].nSourcesReg);
            maxRec = std::max(maxRec, shots[s].nReceiversReg);
        }
        long long per = 6LL * g.isz * 4 + (wavefield ? (long long)g.nts * g.isz * wbytes() : 0) +
                        (wavefield && f16() ? 2LL * g.isz * 4 + 8LL * g.nts : 0) +
                        (image ? g.isz * 8LL : 0) + (long long)maxSrc * g.ntw * 4 + 2LL * maxRec * g.nts * 4 +
                        2 * g.hsz * 4 + 2 * g.isz * 4 + (1 << 16);
        long long shared = 4LL * g.isz * 4 + (64LL << 20);
        long long cap = (budget - shared) / per;
        require(cap >= 1, "device memory budget cannot hold one shot for this operator");
        return balanced_wave(cap, nShots);
    }

    void born_forward_tb(const float* model, int nShots, const aio_shot* shots, int mem) {
        float* dm = stage_model(model, 1, mem, this->model);
        scale_shared(dm, 1, 0);
        Needs n;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_wave_size(nShots - s0, shots + s0, true, false);
            setup_wave(n, nb, shots + s0, mem, false, false);
            tb_alloc(nb, false);
            tbW.ensure((size_t)nb * g.nts * g.isz * wbytes());
            tb_src_pass(nb, shots + s0, false);
            tb_scat_pass(nb, shots + s0, dm);
            download_data(nb, shots + s0, mem);
            sync();
            s0 += nb;
        }
    }

    // perShot: if non-null, perShot[s] receives shot s's own image (overwritten) and
    // modelOut may be null.
    void born_adjoint_tb(float* modelOut, int add, int nShots, const aio_shot* shots, int mem,
                         float* const* perShot = nullptr) {
        float* out = modelOut ? stage_out(modelOut, 1, add, mem) : nullptr;
        Needs n;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_wave_size(nShots - s0, shots + s0, true, true);
            setup_wave(n, nb, shots + s0, mem, true, false);
            tb_alloc(nb, true);
            tbW.ensure((size_t)nb * g.nts * g.isz * wbytes());
            tb_src_pass(nb, shots + s0, false);
            tb_adj_pass(nb, shots + s0);
            // images of U = v2*p: the reference's v2*(2/v^3) scaling reduces to 2/v^3
            // (FP32 images when imageFp64 = 0: accumulated in the receiver pass as the reference does)
            const long long nI = g.isz;
            if (P.imageFp64)
                k_scale_d<<<ew_grid(nb, nI), 256, 0, st>>>(tbImg.as<double>(), nI, 1, v2.as<float>(), rs.as<float>(),
                                                           g.isz, 3);
            else
                k_scale<<<ew_grid(nb, nI), 256, 0, st>>>(tbImg.as<float>(), nI, 1, v2.as<float>(), rs.as<float>(),
                                                         g.isz, 3);
            kcheck();
            auto sum = [&](float* dst, int s, int n, int add) {
                if (P.imageFp64)
                    k_sum_shots<double><<<ew_grid(1, nI), 256, 0, st>>>(dst, tbImg.as<double>() + s * nI, nI, n, nI, add);
                else
                    k_sum_shots<float><<<ew_grid(1, nI), 256, 0, st>>>(dst, tbImg.as<float>() + s * nI, nI, n, nI, add);
                kcheck();
            };
            if (out) sum(out, 0, nb, 1);
            if (perShot) {
                shotImg.ensure((size_t)g.isz * 4);
                for (int s = 0; s < nb; s++) {
                    sum(shotImg.as<float>(), s, 1, 0);
                    write_model(perShot[s0 + s], 1, 0, mem, shotImg.as<float>());
                }
            }
            sync();
            s0 += nb;
        }
        if (out) write_model(modelOut, 1, add, mem, out);
        sync();
    }

    // Born adjoint with one image per shot. Blocked stepper: all shots in the same
    // launches; per-fine-step stepper: one shot per call.
    void born_adjoint_shots(float* const* images, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        for (int s = 0; s < nShots; s++) require(images && images[s], "per-shot image output is NULL");
        if (tb_enabled()) return born_adjoint_tb(nullptr, 0, nShots, shots, mem, images);
        for (int s = 0; s < nShots; s++) born_adjoint(images[s], 0, 1, shots + s, mem);
    }

    void nonlinear_forward_tb(int nShots, const aio_shot* shots, int mem) {
        Needs n;
        for (int s0 = 0; s0 < nShots;) {
            const int nb = tb_wave_size(nShots - s0, shots + s0, false, false);
            setup_wave(n, nb, shots + s0, mem, false, false);
            tb_alloc(nb, false);
            tb_src_pass(nb, shots + s0, true);
            download_data(nb, shots + s0, mem);
            sync();
            s0 += nb;
        }
    }

    // Source pass storing the coarse source wavefield W[nts] of every shot of the wave.
    // F/src/BornShotsGpuFunctions.cu:297-321.
    void source_wavefield(int nb, DevMem& W) { fwd_sparse_pass(nb, false, &W); }

    // Born forward (F/src/BornShotsGpuFunctions.cu:260-388).
    void born_forward(const float* model, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        if (tb_enabled()) return born_forward_tb(model, nShots, shots, mem);
        Needs n;
        n.nWavefields = 1;
        n.ss = true;
        float* dm = stage_model(model, 1, mem, this->model);
        scale_shared(dm, 1, 0);
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, false, false);
            source_wavefield(nb, wf1);
            const float* W = wf1.as<float>();
            fwd_dense_pass(
                nb, [&](int t, long long slot) { img_fwd(nb, slot, dm, 0, W, t); }, false, true, ACC_NONE, nullptr,
                [](int, long long) {});
            download_data(nb, shots + s0, mem);
            sync();
            s0 += nb;
        }
    }

    // Born adjoint (F/src/BornShotsGpuFunctions.cu:829-957), per-shot images
    // summed on the device.
    void born_adjoint(float* modelOut, int add, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        if (tb_enabled()) return born_adjoint_tb(modelOut, add, nShots, shots, mem);
        Needs n;
        n.nWavefields = 1;
        n.nImg = 1;
        float* out = stage_out(modelOut, 1, add, mem);
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, true, false);
            source_wavefield(nb, wf1);
            zero_images(nb, 1);
            const float* W = wf1.as<float>();
            std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
            adj_sparse_pass(nb, din, nullptr, ACC_RING, nullptr,
                            [&](int t, long long slot) { img_adj(nb, slot, W, t); });
            reduce_images(nb, 1, 0, out, true);
            sync();
            s0 += nb;
        }
        write_model(modelOut, 1, add, mem, out);
        sync();
    }

    float* stage_out(float* dst, int nSlices, int add, int mem) {
        outv.ensure((size_t)nSlices * g.isz * 4);
        AIO_CK(cudaMemsetAsync(outv.p, 0, (size_t)nSlices * g.isz * 4, st));
        if (add) to_interior(outv.as<float>(), dst, nSlices, mem);
        return outv.as<float>();
    }

    // Operators whose stored fields stay in FP32 refuse a compressed stored-wavefield setting
    // instead of running with FP32 fields under it.
    void require_fp32_fields(const char* what) {
        require(P.wavefieldPrecision == AIO_WFLD_FP32,
                std::string(what) + " keep their stored wavefields in FP32 (wavefieldPrecision must be AIO_WFLD_FP32)");
    }

    // Extended (time-lag) Born forward (F/src/BornExtShotsGpuFunctions.cu:269-419).
    void born_ext_forward(const float* model, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        require(P.wavefieldPrecision == AIO_WFLD_FP32 || !offsets(),
                "the subsurface-offset extension keeps the stored wavefield in FP32 (wavefieldPrecision)");
        if (tb_enabled()) return born_ext_forward_tb(model, nShots, shots, mem);
        Needs n;
        n.nWavefields = 1;
        n.ss = true;
        float* dm = stage_model(model, g.nExt, mem, this->model);
        // subsurface offsets (BornOffsetShotsFwdGpu, F/src/BornExtShotsGpuFunctions.cu:582-724): 2/v^3 only,
        // v^2 dtw^2 applied to each secondary-source slice
        scale_shared(dm, g.nExt, offsets() ? 3 : (P.sloth ? 2 : 1));
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, false, false);
            source_wavefield(nb, wf1);
            const float* W = wf1.as<float>();
            fwd_dense_pass(
                nb,
                [&](int t, long long slot) {
                    if (offsets()) img_offset_fwd(nb, slot, dm, W, t);
                    else img_time_fwd(nb, slot, dm, W, t);
                },
                true, true, ACC_NONE, nullptr, [](int, long long) {});
            download_data(nb, shots + s0, mem);
            sync();
            s0 += nb;
        }
    }

    // Full padded-grid wavefield output [nts][nx][nz] (zero FAT ring) from interior slices.
    void wavefield_out(float* dst, const DevMem& src, int mem) {
        const size_t bytes = (size_t)g.nts * g.nz * g.nx * 4;
        if (mem == AIO_MEM_HOST) std::memset(dst, 0, bytes);
        else AIO_CK(cudaMemsetAsync(dst, 0, bytes, st));
        from_interior(dst, src.as<float>(), g.nts, mem);
    }

    // Born forward of one shot with its coarse source and scattered wavefields
    // (BornShotsFwdGpuWavefield, F/src/BornShotsGpuFunctions.cu:390-535), per-fine-step stepper.
    void born_forward_wavefield(const float* model, const aio_shot* shot, int mem, float* srcW, float* secW) {
        begin_call();
        require(srcW && secW, "wavefield output is NULL");
        float* dm = stage_model(model, 1, mem, this->model);
        scale_shared(dm, 1, 0);
        Needs n;
        n.nWavefields = 2;
        n.ss = true;
        require(wave_size(n, 1, shot) >= 1, "device memory budget cannot hold the wavefields of one shot");
        setup_wave(n, 1, shot, mem, false, false);
        source_wavefield(1, wf1);
        const float* W = wf1.as<float>();
        fwd_dense_pass(
            1, [&](int t, long long slot) { img_fwd(1, slot, dm, 0, W, t); }, false, true, ACC_FULL, &wf2,
            [](int, long long) {});
        download_data(1, shot, mem);
        wavefield_out(srcW, wf1, mem);
        wavefield_out(secW, wf2, mem);
        sync();
    }

    // Born adjoint of one shot with its receiver wavefield scaled by 2/v^3 v^2 dtw^2
    // (BornShotsAdjGpuWavefield, F/src/BornShotsGpuFunctions.cu:959-1103, which returns only that
    // one) and, when srcW is not null, its coarse source wavefield.
    void born_adjoint_wavefield(float* modelOut, int add, const aio_shot* shot, int mem, float* srcW, float* recW) {
        begin_call();
        require(recW != nullptr, "wavefield output is NULL");
        Needs n;
        n.nWavefields = 2;
        n.nImg = 1;
        require(wave_size(n, 1, shot) >= 1, "device memory budget cannot hold the wavefields of one shot");
        float* out = stage_out(modelOut, 1, add, mem);
        setup_wave(n, 1, shot, mem, true, false);
        source_wavefield(1, wf1);
        zero_images(1, 1);
        AIO_CK(cudaMemsetAsync(wf2.p, 0, (size_t)g.nts * g.isz * 4, st));
        const float* W = wf1.as<float>();
        std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
        adj_sparse_pass(1, din, nullptr, ACC_RING, nullptr, [&](int t, long long slot) {
            k_record_scale<<<ew_grid(1, g.isz), 256, 0, st>>>(wf2.as<float>() + (long long)t * g.isz, ring_ptr(slot),
                                                               rs.as<float>(), v2.as<float>(), g.isz);
            kcheck();
            img_adj(1, slot, W, t);
        });
        reduce_images(1, 1, 0, out, true);
        write_model(modelOut, 1, add, mem, out);
        if (srcW) wavefield_out(srcW, wf1, mem);
        wavefield_out(recW, wf2, mem);
        sync();
    }

    // Extended Born forward of one shot with its coarse source and scattered wavefields
    // (BornTimeShotsFwdGpuWavefield, F/src/BornExtShotsGpuFunctions.cu:420-580; offsets :726-884;
    // free surface :1038-1205, :1356-1524), per-fine-step stepper. Like those drivers, the
    // time-lag model scaling is the non-sloth one.
    void born_ext_forward_wavefield(const float* model, const aio_shot* shot, int mem, float* srcW, float* secW) {
        begin_call();
        require(srcW && secW, "wavefield output is NULL");
        float* dm = stage_model(model, g.nExt, mem, this->model);
        scale_shared(dm, g.nExt, offsets() ? 3 : 1);
        Needs n;
        n.nWavefields = 2;
        n.ss = true;
        require(wave_size(n, 1, shot) >= 1, "device memory budget cannot hold the wavefields of one shot");
        setup_wave(n, 1, shot, mem, false, false);
        source_wavefield(1, wf1);
        const float* W = wf1.as<float>();
        fwd_dense_pass(
            1,
            [&](int t, long long slot) {
                if (offsets()) img_offset_fwd(1, slot, dm, W, t);
                else img_time_fwd(1, slot, dm, W, t);
            },
            true, true, ACC_FULL, &wf2, [](int, long long) {});
        download_data(1, shot, mem);
        wavefield_out(srcW, wf1, mem);
        wavefield_out(secW, wf2, mem);
        sync();
    }
    // Extended Born adjoint of one shot with its coarse source wavefield and receiver wavefield
    // (BornTimeShotsAdjGpuWavefield, F/src/BornExtShotsGpuFunctions.cu:1680-1847: the receiver
    // samples scaled by 2/v^3 v^2 dtw^2; offsets :1991-2151: by v^2 dtw^2 only; free surface
    // :2306-2476, :2623-2783), per-fine-step stepper, non-sloth time-lag scaling.
    void born_ext_adjoint_wavefield(float* modelOut, int add, const aio_shot* shot, int mem, float* srcW,
                                    float* recW) {
        begin_call();
        require(recW != nullptr, "wavefield output is NULL");
        Needs n;
        n.nWavefields = 2;
        n.nImg = g.nExt;
        require(wave_size(n, 1, shot) >= 1, "device memory budget cannot hold the wavefields of one shot");
        float* out = stage_out(modelOut, g.nExt, add, mem);
        setup_wave(n, 1, shot, mem, true, false);
        source_wavefield(1, wf1);
        zero_images(1, g.nExt);
        AIO_CK(cudaMemsetAsync(wf2.p, 0, (size_t)g.nts * g.isz * 4, st));
        const float* W = wf1.as<float>();
        std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
        adj_sparse_pass(1, din, nullptr, ACC_RING, nullptr, [&](int t, long long slot) {
            k_record_scale<<<ew_grid(1, g.isz), 256, 0, st>>>(wf2.as<float>() + (long long)t * g.isz, ring_ptr(slot),
                                                               offsets() ? nullptr : rs.as<float>(), v2.as<float>(),
                                                               g.isz);
            kcheck();
            if (offsets()) img_offset_adj_block(1, slot, W, t, false, true);
            else img_time_adj(1, slot, W, t, +1);
        });
        reduce_images(1, g.nExt, offsets() ? 3 : 1, out, true);
        write_model(modelOut, g.nExt, add, mem, out);
        if (srcW) wavefield_out(srcW, wf1, mem);
        wavefield_out(recW, wf2, mem);
        sync();
    }

    // Extended (time-lag) Born adjoint (F/src/BornExtShotsGpuFunctions.cu:1525-1675).
    void born_ext_adjoint(float* modelOut, int add, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        require(P.wavefieldPrecision == AIO_WFLD_FP32 || !offsets(),
                "the subsurface-offset extension keeps the stored wavefield in FP32 (wavefieldPrecision)");
        if (tb_enabled()) return born_ext_adjoint_tb(modelOut, add, nShots, shots, mem);
        Needs n;
        n.nWavefields = 1;
        n.nImg = g.nExt;
        float* out = stage_out(modelOut, g.nExt, add, mem);
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, true, false);
            source_wavefield(nb, wf1);
            zero_images(nb, g.nExt);
            const float* W = wf1.as<float>();
            std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
            // subsurface offsets: BornOffsetShotsAdjGpu, F/src/BornExtShotsGpuFunctions.cu:1848-1990
            adj_sparse_pass(nb, din, nullptr, ACC_RING, nullptr, [&](int t, long long slot) {
                if (offsets()) img_offset_adj_block(nb, slot, W, t, false, true);
                else img_time_adj(nb, slot, W, t, +1);
            });
            reduce_images(nb, g.nExt, offsets() ? 3 : (P.sloth ? 2 : 1), out, true);
            sync();
            s0 += nb;
        }
        write_model(modelOut, g.nExt, add, mem, out);
        sync();
    }

    // Saved wavefields of one tomo / WEMVA shot (the reference drivers' saveWavefield = 1):
    // d2/dt2 of the source wavefield, and two secondary fields, each [nts][nx][nz]. While `save`
    // is set the four operators run one shot on the per-fine-step stepper with a third full
    // wavefield (wf3) for the second secondary field.
    struct SaveOut {
        float* src;
        float* sec1;
        float* sec2;
    };
    const SaveOut* save = nullptr;
    struct SaveScope {
        Context* c;
        SaveScope(Context* x, const SaveOut* o) : c(x) { c->save = o; }
        ~SaveScope() { c->save = nullptr; }
    };
    // Coarse sample t of a scattered field, taken from its ring slot before the imaging call that
    // clears the slot (the drivers' per-sample cudaMemcpy of scatLeft / scatRight). `scaled`
    // stores it times v^2 dtw^2: the subsurface-offset WEMVA forward saves its second-leg samples
    // after scaleSecondarySourceFd (F/src/wemvaExtShotsGpuFunctions.cu:1232-1239).
    void keep(int t, long long slot, bool scaled = false) {
        if (!save) return;
        float* dst = wf3.as<float>() + (long long)t * g.isz;
        if (scaled) {
            AIO_CK(cudaMemsetAsync(dst, 0, (size_t)g.isz * 4, st));
            k_record_scale<<<ew_grid(1, g.isz), 256, 0, st>>>(dst, ring_ptr(slot), nullptr, v2.as<float>(), g.isz);
            kcheck();
        } else {
            AIO_CK(cudaMemcpyAsync(dst, ring_ptr(slot), (size_t)g.isz * 4, cudaMemcpyDeviceToDevice, st));
        }
    }
    // The three saved fields of the shot to the caller: source d2/dt2 (wf2), first secondary
    // field (wf1: the receiver wavefield, or the tomo forward's first scattered field), second
    // secondary field (wf3).
    void save_out(int mem) {
        if (!save) return;
        wavefield_out(save->src, wf2, mem);
        wavefield_out(save->sec1, wf1, mem);
        wavefield_out(save->sec2, wf3, mem);
    }
    int fields_needed() const { return save ? 3 : 2; }
    void one_shot_saving(int nShots) {
        if (save) require(nShots == 1, "saved wavefields are returned for one shot per call");
    }
    void tomo_forward_wavefield(const float* model, const float* extRefl, const aio_shot* shot, int mem, float* w0,
                                float* w1, float* w2) {
        require(w0 && w1 && w2, "wavefield output is NULL");
        const SaveOut o{w0, w1, w2};
        SaveScope sc(this, &o);
        tomo_forward(model, extRefl, 1, shot, mem);
    }
    void tomo_adjoint_wavefield(float* modelOut, int add, const float* extRefl, const aio_shot* shot, int mem,
                                float* w0, float* w1, float* w2) {
        require(w0 && w1 && w2, "wavefield output is NULL");
        const SaveOut o{w0, w1, w2};
        SaveScope sc(this, &o);
        tomo_adjoint(modelOut, add, extRefl, 1, shot, mem);
    }
    void wemva_forward_wavefield(const float* model, float* imageOut, int add, const aio_shot* shot, int mem,
                                 float* w0, float* w1, float* w2) {
        require(w0 && w1 && w2, "wavefield output is NULL");
        const SaveOut o{w0, w1, w2};
        SaveScope sc(this, &o);
        wemva_forward(model, imageOut, add, 1, shot, mem);
    }
    void wemva_adjoint_wavefield(float* modelOut, int add, const float* image, const aio_shot* shot, int mem,
                                 float* w0, float* w1, float* w2) {
        require(w0 && w1 && w2, "wavefield output is NULL");
        const SaveOut o{w0, w1, w2};
        SaveScope sc(this, &o);
        wemva_adjoint(modelOut, add, image, 1, shot, mem);
    }

    // Source wavefield with coarse second time derivative (computeTomoSrcWfldDt2,
    // F/src/tomoExtShotsGpuFunctions.cu:1251-1361).
    void source_wavefield_dt2(int nb, DevMem& W) {
        fwd_sparse_pass(nb, false, &W);
        k_dt2<<<ew_grid(nb, g.isz), 256, 0, st>>>(W.as<float>(), wfSt(), g.isz, g.nts, k.cSide, k.cCenter);
        kcheck();
    }
    // Receiver wavefield (computeTomoRecWfld, F/src/tomoExtShotsGpuFunctions.cu:1481-1515).
    void receiver_wavefield(int nb, const std::vector<const float*>& data, DevMem& R) {
        adj_sparse_pass(nb, data, nullptr, ACC_FULL, &R, [](int, long long) {});
    }

    // Extended tomo forward (F/src/tomoExtShotsGpuFunctions.cu:355-465, legs :1554-1881).
    void tomo_forward(const float* model, const float* extRefl, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        if (!(tb_enabled() && !offsets() && !save)) require_fp32_fields("tomo and WEMVA off the blocked stepper");
        one_shot_saving(nShots);
        Needs n;
        n.nWavefields = fields_needed();
        n.ss = true;
        float* dm = stage_model(model, 1, mem, this->model);
        scale_shared(dm, 1, 0);
        float* ex = stage_model(extRefl, g.nExt, mem, this->ext);
        // subsurface offsets (tomoOffsetShotsFwdGpu, F/src/tomoExtShotsGpuFunctions.cu:467-575): 2/v^3 only
        scale_shared(ex, g.nExt, offsets() ? 3 : (P.sloth ? 2 : 1));
        if (tb_enabled() && !offsets() && !save)
            return tomo_forward_tb(dm, ex, nShots, shots, mem);
        // saving: the recorded (second) pass of each leg also accumulates its coarse field into wf3
        // (interpWavefield into tomoSecWavefield2, F/src/tomoExtShotsGpuFunctions.cu:1640-1641)
        const AccMode secondAcc = save ? ACC_FULL : ACC_NONE;
        DevMem* second = save ? &wf3 : nullptr;
        auto ext_src = [&](int nb, long long slot, const float* F, int t) {
            if (offsets()) img_offset_fwd(nb, slot, ex, F, t);
            else img_time_fwd(nb, slot, ex, F, t);
        };
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, false, false);
            source_wavefield_dt2(nb, wf2);
            const float* W2 = wf2.as<float>();
            const float* W1 = wf1.as<float>();
            auto nop = [](int, long long) {};
            if (P.leg1) {
                fwd_dense_pass(
                    nb, [&](int t, long long slot) { ext_src(nb, slot, W2, t); }, true, false, ACC_FULL, &wf1, nop);
                fwd_dense_pass(
                    nb, [&](int t, long long slot) { img_fwd(nb, slot, dm, 0, W1, t); }, false, true, secondAcc,
                    second, nop);
            }
            if (P.leg2) {
                fwd_dense_pass(
                    nb, [&](int t, long long slot) { img_fwd(nb, slot, dm, 0, W2, t); }, false, false, ACC_FULL, &wf1,
                    nop);
                fwd_dense_pass(
                    nb, [&](int t, long long slot) { ext_src(nb, slot, W1, t); }, true, true, secondAcc, second, nop);
            }
            download_data(nb, shots + s0, mem);
            save_out(mem);
            sync();
            s0 += nb;
        }
    }

    // Extended tomo adjoint (F/src/tomoExtShotsGpuFunctions.cu:797-910, legs :2442-2701).
    void tomo_adjoint(float* modelOut, int add, const float* extRefl, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        if (!(tb_enabled() && !offsets() && !save)) require_fp32_fields("tomo and WEMVA off the blocked stepper");
        one_shot_saving(nShots);
        Needs n;
        n.nWavefields = fields_needed();
        n.ss = true;
        n.nImg = 1;
        float* ex = stage_model(extRefl, g.nExt, mem, this->ext);
        // subsurface offsets (tomoOffsetShotsAdjGpu, F/src/tomoExtShotsGpuFunctions.cu:912-1023): 2/v^3 only
        scale_shared(ex, g.nExt, offsets() ? 3 : (P.sloth ? 2 : 1));
        float* out = stage_out(modelOut, 1, add, mem);
        if (tb_enabled() && !offsets() && !save) {
            tomo_adjoint_tb(out, ex, nShots, shots, mem);
            write_model(modelOut, 1, add, mem, out);
            sync();
            return;
        }
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, true, false);
            source_wavefield_dt2(nb, wf2);
            std::vector<const float*> din(dataPtr.begin(), dataPtr.end());
            receiver_wavefield(nb, din, wf1);
            zero_images(nb, 1);
            const float* W2 = wf2.as<float>();
            const float* R = wf1.as<float>();
            if (P.leg1)
                fwd_dense_pass(
                    nb,
                    [&](int t, long long slot) {
                        if (offsets()) img_offset_fwd(nb, slot, ex, W2, t);
                        else img_time_fwd(nb, slot, ex, W2, t);
                    },
                    true, false, ACC_RING, nullptr, [&](int t, long long slot) {
                        keep(t, slot);
                        img_adj(nb, slot, R, t);
                    });
            if (P.leg2)
                adj_dense_pass(
                    nb,
                    [&](int t, long long slot) {
                        if (offsets()) img_offset_tomo_adj(nb, slot, ex, R, t);
                        else img_time_tomo_adj(nb, slot, ex, R, t);
                    },
                    true, [&](int t, long long slot) {
                        keep(t, slot);
                        img_adj(nb, slot, W2, t);
                    });
            reduce_images(nb, 1, 0, out, true);
            save_out(mem);
            sync();
            s0 += nb;
        }
        write_model(modelOut, 1, add, mem, out);
        sync();
    }

    // Extended WEMVA forward (F/src/wemvaExtShotsGpuFunctions.cu:344-456, legs :961-1122).
    void wemva_forward(const float* model, float* imageOut, int add, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        if (!(tb_enabled() && !offsets() && !save)) require_fp32_fields("tomo and WEMVA off the blocked stepper");
        one_shot_saving(nShots);
        Needs n;
        n.nWavefields = fields_needed();
        n.ss = true;
        n.nImg = g.nExt;
        float* dm = stage_model(model, 1, mem, this->model);
        scale_shared(dm, 1, 0);
        float* out = stage_out(imageOut, g.nExt, add, mem);
        if (tb_enabled() && !offsets() && !save) {
            wemva_forward_tb(dm, out, nShots, shots, mem);
            write_model(imageOut, g.nExt, add, mem, out);
            sync();
            return;
        }
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, false, true);
            source_wavefield_dt2(nb, wf2);
            receiver_wavefield(nb, wdataPtr, wf1);
            zero_images(nb, g.nExt);
            const float* W2 = wf2.as<float>();
            const float* R = wf1.as<float>();
            // subsurface offsets: wemvaOffsetShotsFwdGpu, F/src/wemvaExtShotsGpuFunctions.cu:458-574
            if (P.leg1)
                fwd_dense_pass(
                    nb, [&](int t, long long slot) { img_fwd(nb, slot, dm, 0, W2, t); }, false, false, ACC_RING,
                    nullptr, [&](int t, long long slot) {
                        keep(t, slot);
                        if (offsets()) img_offset_adj_block(nb, slot, R, t, true, false);
                        else img_time_adj(nb, slot, R, t, -1);
                    });
            if (P.leg2)
                adj_dense_pass(
                    nb, [&](int t, long long slot) { img_fwd(nb, slot, dm, 0, R, t); }, false,
                    [&](int t, long long slot) {
                        keep(t, slot, offsets());
                        if (offsets()) img_offset_adj_block(nb, slot, W2, t, false, true);
                        else img_time_adj(nb, slot, W2, t, +1);
                    });
            reduce_images(nb, g.nExt, offsets() ? 3 : 1, out, true);
            save_out(mem);
            sync();
            s0 += nb;
        }
        write_model(imageOut, g.nExt, add, mem, out);
        sync();
    }

    // Extended WEMVA adjoint (F/src/wemvaExtShotsGpuFunctions.cu:575-688, legs :1270-1426).
    void wemva_adjoint(float* modelOut, int add, const float* image, int nShots, const aio_shot* shots, int mem) {
        begin_call();
        if (!(tb_enabled() && !offsets() && !save)) require_fp32_fields("tomo and WEMVA off the blocked stepper");
        one_shot_saving(nShots);
        Needs n;
        n.nWavefields = fields_needed();
        n.ss = true;
        n.nImg = 1;
        float* im = stage_model(image, g.nExt, mem, this->ext);
        // subsurface offsets (wemvaOffsetShotsAdjGpu, F/src/wemvaExtShotsGpuFunctions.cu:689-810): 2/v^3 only
        scale_shared(im, g.nExt, offsets() ? 3 : 1);
        float* out = stage_out(modelOut, 1, add, mem);
        if (tb_enabled() && !offsets() && !save) {
            wemva_adjoint_tb(out, im, nShots, shots, mem);
            write_model(modelOut, 1, add, mem, out);
            sync();
            return;
        }
        for (int s0 = 0; s0 < nShots;) {
            const int nb = wave_size(n, nShots - s0, shots + s0);
            setup_wave(n, nb, shots + s0, mem, false, true);
            source_wavefield_dt2(nb, wf2);
            receiver_wavefield(nb, wdataPtr, wf1);
            zero_images(nb, 1);
            const float* W2 = wf2.as<float>();
            const float* R = wf1.as<float>();
            if (P.leg1)
                adj_dense_pass(
                    nb,
                    [&](int t, long long slot) {
                        if (offsets()) img_offset_tomo_adj(nb, slot, im, R, t);
                        else img_time_tomo_adj(nb, slot, im, R, t);
                    },
                    true, [&](int t, long long slot) {
                        keep(t, slot);
                        img_adj(nb, slot, W2, t);
                    });
            if (P.leg2)
                fwd_dense_pass(
                    nb,
                    [&](int t, long long slot) {
                        if (offsets()) img_offset_fwd(nb, slot, im, W2, t);
                        else img_time_fwd(nb, slot, im, W2, t);
                    },
                    true, false, ACC_RING, nullptr, [&](int t, long long slot) {
                        keep(t, slot);
                        img_adj(nb, slot, R, t);
                    });
            reduce_images(nb, 1, 0, out, true);
            save_out(mem);
            sync();
            s0 += nb;
        }
        write_model(modelOut, 1, add, mem, out);
        sync();
    }
};

// ----------------------------------------------------------------------------
// Reference-seam state: one parameter block and one context per (family, iGpu)
// slot, the counterpart of the reference's per-translation-unit globals
// (F/include/varDeclare.h:22-93).
// ----------------------------------------------------------------------------
struct SeamSlot {
    aio_params P{};
    bool inited = false;
    Context* ctx = nullptr;
};
static std::mutex g_seam_mu;
static std::map<std::pair<int, int>, SeamSlot> g_seam;

static SeamSlot& seam(int family, int iGpu) { return g_seam[{family, iGpu}]; }

static void seam_init(int family, float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad,
                      float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId) {
    require(nGpu >= 1, "nGpu must be >= 1");
    std::lock_guard<std::mutex> lk(g_seam_mu);
    aio_params P{};
    P.nz = nz; P.nx = nx; P.nts = nts; P.sub = sub; P.minPad = minPad; P.nExt = nExt;
    P.dz = dz; P.dx = dx; P.dts = dts; P.alphaCos = alphaCos; P.leg1 = leg1; P.leg2 = leg2;
    P.wavefieldPrecision = AIO_WFLD_FP32; P.imageFp64 = 0; P.device = iGpuId;
    // The reference's slot index is iGpu (0..nGpu-1) while init is called per
    // device id; the parameters are identical for every slot of a family.
    for (int i = 0; i < nGpu; i++) {
        SeamSlot& s = seam(family, i);
        s.P = P;
        s.inited = true;
    }
}

static void seam_allocate(int family, float* vel2Dtw2, float* reflScale, int iGpu, int iGpuId) {
    std::lock_guard<std::mutex> lk(g_seam_mu);
    SeamSlot& s = seam(family, iGpu);
    if (!s.inited) throw Error{AIO_ERR_STATE, "allocate called before init"};
    if (s.ctx) {
        s.ctx->destroy();
        delete s.ctx;
        s.ctx = nullptr;
    }
    s.P.device = iGpuId;
    Context* c = new Context();
    try {
        c->init(s.P, vel2Dtw2, reflScale);
    } catch (...) {
        delete c;
        throw;
    }
    s.ctx = c;
}

static void seam_deallocate(int family, int iGpu) {
    std::lock_guard<std::mutex> lk(g_seam_mu);
    SeamSlot& s = seam(family, iGpu);
    if (s.ctx) {
        s.ctx->destroy();
        delete s.ctx;
    }
    s.ctx = nullptr;
}

static Context& seam_ctx(int family, int iGpu) {
    std::lock_guard<std::mutex> lk(g_seam_mu);
    SeamSlot& s = seam(family, iGpu);
    if (!s.ctx) throw Error{AIO_ERR_STATE, "operator call before allocate"};
    return *s.ctx;
}

static aio_shot one_shot(float* sig, int* sp, int ns, int* rp, int nr, float* data) {
    aio_shot s{};
    s.sourcesPositionReg = sp; s.nSourcesReg = ns;
    s.receiversPositionReg = rp; s.nReceiversReg = nr;
    s.sourcesSignals = sig; s.data = data;
    return s;
}

}  // namespace aio

using namespace aio;

struct aio_context {
    Context c;
};

#define AIO_API extern "C" __attribute__((visibility("default")))

AIO_API const char* aio_last_error(void) { return g_err.c_str(); }

AIO_API int aio_context_create(const aio_params* params, const float* vel2Dtw2, const float* reflectivityScale,
                               aio_context** out) {
    return guard([&] {
        require(params && out, "null argument");
        aio_context* c = new aio_context();
        try {
            c->c.init(*params, vel2Dtw2, reflectivityScale);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}
AIO_API int aio_context_destroy(aio_context* ctx) {
    return guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->c.dev);
        ctx->c.destroy();
        delete ctx;
    });
}
AIO_API int aio_context_set_velocity(aio_context* ctx, const float* vel2Dtw2, const float* reflectivityScale) {
    return guard([&] { ctx->c.set_velocity(vel2Dtw2, reflectivityScale); });
}
AIO_API int aio_context_wave_capacity(aio_context* ctx, int family) {
    Context::Needs n;
    switch (family) {
        case AIO_NONLINEAR: break;
        case AIO_BORN: n.nWavefields = 1; n.ss = true; n.nImg = 1; break;
        case AIO_BORN_EXT: n.nWavefields = 1; n.ss = true; n.nImg = ctx->c.g.nExt; break;
        default: n.nWavefields = 2; n.ss = true; n.nImg = ctx->c.g.nExt; break;
    }
    return ctx->c.capacity(n, 4, 4096);
}
AIO_API long long aio_context_last_launches(aio_context* ctx) { return ctx->c.launches; }
AIO_API void* aio_context_stream(aio_context* ctx) { return (void*)ctx->c.st; }
AIO_API int aio_context_profile(aio_context* ctx, int sampleEvery) {
    return guard([&] {
        require(sampleEvery >= 0, "sampleEvery must be >= 0");
        ctx->c.profEvery = sampleEvery;
    });
}
AIO_API int aio_context_stats(aio_context* ctx, long long* kernels, double* stepperMs, long long* stepperTimed,
                              double* stepperPoints) {
    if (kernels) *kernels = ctx->c.kernels;
    if (stepperMs) *stepperMs = ctx->c.stepMs;
    if (stepperTimed) *stepperTimed = ctx->c.stepTimed;
    if (stepperPoints) *stepperPoints = ctx->c.stepPoints;
    return AIO_OK;
}
AIO_API long long aio_context_graph_replays(aio_context* ctx) { return ctx ? ctx->c.graphReplays : 0; }
AIO_API long long aio_context_device_bytes(aio_context* ctx) { return ctx ? ctx->c.device_bytes() : 0; }
AIO_API int aio_context_release_buffers(aio_context* ctx) {
    return guard([&] {
        require(ctx != nullptr, "context is NULL");
        ctx->c.release_buffers();
    });
}
AIO_API int aio_context_set_budget(aio_context* ctx, long long bytes) {
    return guard([&] {
        require(ctx != nullptr, "context is NULL");
        Context& c = ctx->c;
        AIO_CK(cudaSetDevice(c.dev));
        if (bytes > 0) {
            c.budget = bytes;
        } else {
            size_t fr = 0, tot = 0;
            AIO_CK(cudaMemGetInfo(&fr, &tot));
            c.budget = (long long)(0.93 * (double)fr);
        }
        c.P.memBudgetBytes = bytes > 0 ? bytes : 0;
    });
}
AIO_API int aio_context_reset_stats(aio_context* ctx) {
    ctx->c.kernels = 0;
    ctx->c.stepMs = 0.0;
    ctx->c.stepTimed = 0;
    ctx->c.stepPoints = 0.0;
    return AIO_OK;
}

AIO_API int aio_nonlinear_forward(aio_context* ctx, int nShots, const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.nonlinear_forward(nShots, shots, memSpace, nullptr); });
}
AIO_API int aio_nonlinear_adjoint(aio_context* ctx, int nShots, const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.nonlinear_adjoint(nShots, shots, memSpace, nullptr); });
}
AIO_API int aio_nonlinear_forward_wavefield(aio_context* ctx, const aio_shot* shot, int memSpace, float* wavefield) {
    return guard([&] {
        require(wavefield != nullptr, "wavefield output is NULL");
        ctx->c.nonlinear_forward(1, shot, memSpace, wavefield);
    });
}
AIO_API int aio_nonlinear_adjoint_wavefield(aio_context* ctx, const aio_shot* shot, int memSpace, float* wavefield) {
    return guard([&] {
        require(wavefield != nullptr, "wavefield output is NULL");
        ctx->c.nonlinear_adjoint(1, shot, memSpace, wavefield);
    });
}
AIO_API int aio_born_forward(aio_context* ctx, const float* model, int nShots, const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.born_forward(model, nShots, shots, memSpace); });
}
AIO_API int aio_born_adjoint(aio_context* ctx, float* model, int add, int nShots, const aio_shot* shots,
                             int memSpace) {
    return guard([&] { ctx->c.born_adjoint(model, add, nShots, shots, memSpace); });
}
AIO_API int aio_context_blocked_plan(aio_context* ctx, int nShots, int* plan) {
    return guard([&] {
        require(plan != nullptr, "plan output is NULL");
        const auto pl = nShots >= 1 ? ctx->c.tb_plan(nShots) : ctx->c.tbLast;
        plan[0] = pl.HZ;
        plan[1] = pl.nStrips;
        plan[2] = pl.LX;
        plan[3] = pl.nChunks;
    });
}
AIO_API int aio_born_forward_wavefield(aio_context* ctx, const float* model, const aio_shot* shot, int memSpace,
                                       float* srcWavefield, float* secWavefield) {
    return guard([&] {
        require(shot != nullptr, "shot is NULL");
        ctx->c.born_forward_wavefield(model, shot, memSpace, srcWavefield, secWavefield);
    });
}
AIO_API int aio_born_adjoint_wavefield(aio_context* ctx, float* modelOut, int add, const aio_shot* shot, int memSpace,
                                       float* srcWavefield, float* recWavefield) {
    return guard([&] {
        require(shot != nullptr, "shot is NULL");
        ctx->c.born_adjoint_wavefield(modelOut, add, shot, memSpace, srcWavefield, recWavefield);
    });
}
AIO_API int aio_born_ext_forward_wavefield(aio_context* ctx, const float* model, const aio_shot* shot, int memSpace,
                                           float* srcWavefield, float* secWavefield) {
    return guard([&] {
        require(shot != nullptr, "shot is NULL");
        ctx->c.born_ext_forward_wavefield(model, shot, memSpace, srcWavefield, secWavefield);
    });
}
AIO_API int aio_born_ext_adjoint_wavefield(aio_context* ctx, float* modelOut, int add, const aio_shot* shot,
                                           int memSpace, float* srcWavefield, float* recWavefield) {
    return guard([&] {
        require(shot != nullptr, "shot is NULL");
        ctx->c.born_ext_adjoint_wavefield(modelOut, add, shot, memSpace, srcWavefield, recWavefield);
    });
}
AIO_API int aio_born_adjoint_shots(aio_context* ctx, float* const* images, int nShots, const aio_shot* shots,
                                   int memSpace) {
    return guard([&] { ctx->c.born_adjoint_shots(images, nShots, shots, memSpace); });
}
AIO_API int aio_born_ext_forward(aio_context* ctx, const float* model, int nShots, const aio_shot* shots,
                                 int memSpace) {
    return guard([&] { ctx->c.born_ext_forward(model, nShots, shots, memSpace); });
}
AIO_API int aio_born_ext_adjoint(aio_context* ctx, float* model, int add, int nShots, const aio_shot* shots,
                                 int memSpace) {
    return guard([&] { ctx->c.born_ext_adjoint(model, add, nShots, shots, memSpace); });
}
AIO_API int aio_tomo_ext_forward(aio_context* ctx, const float* model, const float* extReflectivity, int nShots,
                                 const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.tomo_forward(model, extReflectivity, nShots, shots, memSpace); });
}
AIO_API int aio_tomo_ext_adjoint(aio_context* ctx, float* model, int add, const float* extReflectivity, int nShots,
                                 const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.tomo_adjoint(model, add, extReflectivity, nShots, shots, memSpace); });
}
AIO_API int aio_wemva_ext_forward(aio_context* ctx, const float* model, float* image, int add, int nShots,
                                  const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.wemva_forward(model, image, add, nShots, shots, memSpace); });
}
AIO_API int aio_tomo_ext_forward_wavefield(aio_context* ctx, const float* model, const float* extReflectivity,
                                           const aio_shot* shot, int memSpace, float* srcDt2, float* sec1,
                                           float* sec2) {
    return guard([&] { ctx->c.tomo_forward_wavefield(model, extReflectivity, shot, memSpace, srcDt2, sec1, sec2); });
}
AIO_API int aio_tomo_ext_adjoint_wavefield(aio_context* ctx, float* model, int add, const float* extReflectivity,
                                           const aio_shot* shot, int memSpace, float* srcDt2, float* sec1,
                                           float* sec2) {
    return guard([&] {
        ctx->c.tomo_adjoint_wavefield(model, add, extReflectivity, shot, memSpace, srcDt2, sec1, sec2);
    });
}
AIO_API int aio_wemva_ext_forward_wavefield(aio_context* ctx, const float* model, float* image, int add,
                                            const aio_shot* shot, int memSpace, float* srcDt2, float* sec1,
                                            float* sec2) {
    return guard([&] { ctx->c.wemva_forward_wavefield(model, image, add, shot, memSpace, srcDt2, sec1, sec2); });
}
AIO_API int aio_wemva_ext_adjoint_wavefield(aio_context* ctx, float* model, int add, const float* image,
                                            const aio_shot* shot, int memSpace, float* srcDt2, float* sec1,
                                            float* sec2) {
    return guard([&] { ctx->c.wemva_adjoint_wavefield(model, add, image, shot, memSpace, srcDt2, sec1, sec2); });
}
AIO_API int aio_wemva_ext_adjoint(aio_context* ctx, float* model, int add, const float* image, int nShots,
                                  const aio_shot* shots, int memSpace) {
    return guard([&] { ctx->c.wemva_adjoint(model, add, image, nShots, shots, memSpace); });
}

// ------------------------------------------------------------ reference seam
AIO_API int aio_getGpuInfo(const int* gpuList, int nGpuList, int info, int deviceNumberInfo) {
    (void)info; (void)deviceNumberInfo;
    return guard([&] {
        int nDev = 0;
        AIO_CK(cudaGetDeviceCount(&nDev));
        require(nGpuList <= nDev, "number of requested GPUs greater than available GPUs");
        for (int i = 0; i < nGpuList; i++)
            require(gpuList[i] >= 0 && gpuList[i] < nDev, "GPU id list holds an invalid id");
    });
}

AIO_API int aio_initNonlinearGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad,
                                 int blockSize, float alphaCos, int nGpu, int iGpuId, int iGpuAlloc) {
    (void)blockSize; (void)iGpuAlloc;
    return guard([&] { seam_init(AIO_NONLINEAR, dz, dx, nz, nx, nts, dts, sub, minPad, alphaCos, 1, 1, 1, nGpu, iGpuId); });
}
AIO_API int aio_allocateNonlinearGpu(float* vel2Dtw2, int iGpu, int iGpuId) {
    return guard([&] { seam_allocate(AIO_NONLINEAR, vel2Dtw2, nullptr, iGpu, iGpuId); });
}
AIO_API int aio_deallocateNonlinearGpu(int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] { seam_deallocate(AIO_NONLINEAR, iGpu); });
}
AIO_API int aio_propShotsFwdGpu(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                float* wavefieldDts, int iGpu, int iGpuId) {
    (void)wavefieldDts; (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(modelRegDtw, sp, ns, rp, nr, dataRegDts);
        seam_ctx(AIO_NONLINEAR, iGpu).nonlinear_forward(1, &s, AIO_MEM_HOST, nullptr);
    });
}
AIO_API int aio_propShotsFwdGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                         float* wavefieldDts, int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(modelRegDtw, sp, ns, rp, nr, dataRegDts);
        seam_ctx(AIO_NONLINEAR, iGpu).nonlinear_forward(1, &s, AIO_MEM_HOST, wavefieldDts);
    });
}
AIO_API int aio_propShotsAdjGpu(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                float* wavefieldDts, int iGpu, int iGpuId) {
    (void)wavefieldDts; (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(nullptr, sp, ns, rp, nr, dataRegDts);
        s.sourcesOut = modelRegDtw;
        seam_ctx(AIO_NONLINEAR, iGpu).nonlinear_adjoint(1, &s, AIO_MEM_HOST, nullptr);
    });
}
AIO_API int aio_propShotsAdjGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                         float* wavefieldDts, int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(nullptr, sp, ns, rp, nr, dataRegDts);
        s.sourcesOut = modelRegDtw;
        seam_ctx(AIO_NONLINEAR, iGpu).nonlinear_adjoint(1, &s, AIO_MEM_HOST, wavefieldDts);
    });
}

AIO_API int aio_initBornGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad, int blockSize,
                            float alphaCos, int nGpu, int iGpuId, int iGpuAlloc) {
    (void)blockSize; (void)iGpuAlloc;
    return guard([&] { seam_init(AIO_BORN, dz, dx, nz, nx, nts, dts, sub, minPad, alphaCos, 1, 1, 1, nGpu, iGpuId); });
}
AIO_API int aio_allocateBornShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) {
    return guard([&] { seam_allocate(AIO_BORN, vel2Dtw2, reflectivityScale, iGpu, iGpuId); });
}
AIO_API int aio_deallocateBornShotsGpu(int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] { seam_deallocate(AIO_BORN, iGpu); });
}
AIO_API int aio_BornShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp,
                                int nr, float* srcWavefield, float* scatWavefield, int iGpu, int iGpuId) {
    (void)srcWavefield; (void)scatWavefield; (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        seam_ctx(AIO_BORN, iGpu).born_forward(model, 1, &s, AIO_MEM_HOST);
    });
}
AIO_API int aio_BornShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp,
                                int nr, float* srcWavefield, float* recWavefield, int iGpu, int iGpuId) {
    (void)srcWavefield; (void)recWavefield; (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        seam_ctx(AIO_BORN, iGpu).born_adjoint(model, 0, 1, &s, AIO_MEM_HOST);
    });
}

AIO_API int aio_BornShotsFwdGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                         int* rp, int nr, float* srcWavefield, float* scatWavefield, int iGpu,
                                         int iGpuId) {
    (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        seam_ctx(AIO_BORN, iGpu).born_forward_wavefield(model, &s, AIO_MEM_HOST, srcWavefield, scatWavefield);
    });
}
AIO_API int aio_BornShotsAdjGpuWavefield(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                         int* rp, int nr, float* srcWavefield, float* recWavefield, int iGpu,
                                         int iGpuId) {
    (void)iGpuId;
    return guard([&] {
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        (void)srcWavefield;  // the reference's driver returns the receiver wavefield only
        seam_ctx(AIO_BORN, iGpu).born_adjoint_wavefield(model, 0, &s, AIO_MEM_HOST, nullptr, recWavefield);
    });
}

AIO_API int aio_initBornExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad,
                               int blockSize, float alphaCos, int nExt, int nGpu, int iGpuId, int iGpuAlloc) {
    (void)blockSize; (void)iGpuAlloc;
    return guard(
        [&] { seam_init(AIO_BORN_EXT, dz, dx, nz, nx, nts, dts, sub, minPad, alphaCos, nExt, 1, 1, nGpu, iGpuId); });
}
AIO_API int aio_allocateBornExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) {
    return guard([&] { seam_allocate(AIO_BORN_EXT, vel2Dtw2, reflectivityScale, iGpu, iGpuId); });
}
AIO_API int aio_deallocateBornExtShotsGpu(int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] { seam_deallocate(AIO_BORN_EXT, iGpu); });
}
AIO_API int aio_BornTimeShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp,
                                    int nr, float* srcWavefield, float* scatWavefield, int sloth, int iGpu,
                                    int iGpuId) {
    (void)srcWavefield; (void)scatWavefield; (void)iGpuId;
    return guard([&] {
        Context& c = seam_ctx(AIO_BORN_EXT, iGpu);
        c.P.sloth = sloth;
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        c.born_ext_forward(model, 1, &s, AIO_MEM_HOST);
    });
}
AIO_API int aio_BornTimeShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp,
                                    int nr, float* srcWavefield, float* recWavefield, int sloth, int iGpu,
                                    int iGpuId) {
    (void)srcWavefield; (void)recWavefield; (void)iGpuId;
    return guard([&] {
        Context& c = seam_ctx(AIO_BORN_EXT, iGpu);
        c.P.sloth = sloth;
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        c.born_ext_adjoint(model, 0, 1, &s, AIO_MEM_HOST);
    });
}

AIO_API int aio_initTomoExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad,
                               int blockSize, float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId,
                               int iGpuAlloc) {
    (void)blockSize; (void)iGpuAlloc;
    return guard([&] {
        seam_init(AIO_TOMO_EXT, dz, dx, nz, nx, nts, dts, sub, minPad, alphaCos, nExt, leg1, leg2, nGpu, iGpuId);
    });
}
AIO_API int aio_allocateTomoExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) {
    return guard([&] { seam_allocate(AIO_TOMO_EXT, vel2Dtw2, reflectivityScale, iGpu, iGpuId); });
}
AIO_API int aio_deallocateTomoExtShotsGpu(int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] { seam_deallocate(AIO_TOMO_EXT, iGpu); });
}
// saveWavefield = 1 (the reference drivers' flag): the call also returns, for its one shot, d2/dt2
// of the source wavefield in w0 and the two secondary wavefields in w1 and w2, each
// [nts][nx][nz] (F/src/tomoExtShotsGpuFunctions.cu:396,429-432,843-850,877;
// F/src/wemvaExtShotsGpuFunctions.cu:46,55,78-80). Any other value returns none of them.
static void seam_tomo(Context& c, bool adjoint, float* model, float* data, float* ext, float* sig, int* sp, int ns,
                      int* rp, int nr, float* w0, float* w1, float* w2, int saveWavefield) {
    aio_shot s = one_shot(sig, sp, ns, rp, nr, data);
    if (saveWavefield == 1) {
        if (adjoint) c.tomo_adjoint_wavefield(model, 0, ext, &s, AIO_MEM_HOST, w0, w1, w2);
        else c.tomo_forward_wavefield(model, ext, &s, AIO_MEM_HOST, w0, w1, w2);
    } else if (adjoint) {
        c.tomo_adjoint(model, 0, ext, 1, &s, AIO_MEM_HOST);
    } else {
        c.tomo_forward(model, ext, 1, &s, AIO_MEM_HOST);
    }
}
static void seam_wemva(Context& c, bool adjoint, float* model, float* image, float* sig, int* sp, int ns,
                       float* wemvaData, int* rp, int nr, float* w0, float* w1, float* w2, int saveWavefield) {
    aio_shot s = one_shot(sig, sp, ns, rp, nr, nullptr);
    s.wemvaData = wemvaData;
    if (saveWavefield == 1) {
        if (adjoint) c.wemva_adjoint_wavefield(model, 0, image, &s, AIO_MEM_HOST, w0, w1, w2);
        else c.wemva_forward_wavefield(model, image, 0, &s, AIO_MEM_HOST, w0, w1, w2);
    } else if (adjoint) {
        c.wemva_adjoint(model, 0, image, 1, &s, AIO_MEM_HOST);
    } else {
        c.wemva_forward(model, image, 0, 1, &s, AIO_MEM_HOST);
    }
}
AIO_API int aio_tomoTimeShotsFwdGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                    int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int sloth,
                                    int iGpu, int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        Context& c = seam_ctx(AIO_TOMO_EXT, iGpu);
        c.P.sloth = sloth;
        seam_tomo(c, false, model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, w0, w1, w2,
                  saveWavefield);
    });
}
AIO_API int aio_tomoTimeShotsAdjGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                    int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int sloth,
                                    int iGpu, int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        Context& c = seam_ctx(AIO_TOMO_EXT, iGpu);
        c.P.sloth = sloth;
        seam_tomo(c, true, model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, w0, w1, w2,
                  saveWavefield);
    });
}

// Free-surface seam calls (the reference's *FsGpu drivers): the slot's context runs the call
// with the free surface on and, as those drivers take no sloth flag, without sloth.
struct SeamFs {
    Context& c;
    int fs, sloth;
    explicit SeamFs(Context& cc) : c(cc), fs(cc.P.freeSurface), sloth(cc.P.sloth) {
        c.P.freeSurface = 1;
        c.P.sloth = 0;
    }
    ~SeamFs() {
        c.P.freeSurface = fs;
        c.P.sloth = sloth;
    }
};
AIO_API int aio_propShotsFwdFsGpu(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                  float* wavefieldDts, int iGpu, int iGpuId) {
    (void)wavefieldDts; (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_NONLINEAR, iGpu));
        aio_shot s = one_shot(modelRegDtw, sp, ns, rp, nr, dataRegDts);
        fs.c.nonlinear_forward(1, &s, AIO_MEM_HOST, nullptr);
    });
}
AIO_API int aio_propShotsFwdFsGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                           float* wavefieldDts, int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_NONLINEAR, iGpu));
        aio_shot s = one_shot(modelRegDtw, sp, ns, rp, nr, dataRegDts);
        fs.c.nonlinear_forward(1, &s, AIO_MEM_HOST, wavefieldDts);
    });
}
AIO_API int aio_propShotsAdjFsGpu(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                  float* wavefieldDts, int iGpu, int iGpuId) {
    (void)wavefieldDts; (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_NONLINEAR, iGpu));
        aio_shot s = one_shot(nullptr, sp, ns, rp, nr, dataRegDts);
        s.sourcesOut = modelRegDtw;
        fs.c.nonlinear_adjoint(1, &s, AIO_MEM_HOST, nullptr);
    });
}
AIO_API int aio_propShotsAdjFsGpuWavefield(float* modelRegDtw, float* dataRegDts, int* sp, int ns, int* rp, int nr,
                                           float* wavefieldDts, int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_NONLINEAR, iGpu));
        aio_shot s = one_shot(nullptr, sp, ns, rp, nr, dataRegDts);
        s.sourcesOut = modelRegDtw;
        fs.c.nonlinear_adjoint(1, &s, AIO_MEM_HOST, wavefieldDts);
    });
}
AIO_API int aio_BornShotsFwdFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp,
                                  int nr, float* srcWavefield, float* scatWavefield, int iGpu, int iGpuId) {
    (void)srcWavefield; (void)scatWavefield; (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_BORN, iGpu));
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        fs.c.born_forward(model, 1, &s, AIO_MEM_HOST);
    });
}
AIO_API int aio_BornShotsAdjFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp,
                                  int nr, float* srcWavefield, float* recWavefield, int iGpu, int iGpuId) {
    (void)srcWavefield; (void)recWavefield; (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_BORN, iGpu));
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        fs.c.born_adjoint(model, 0, 1, &s, AIO_MEM_HOST);
    });
}
AIO_API int aio_BornTimeShotsFwdFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                      int* rp, int nr, float* srcWavefield, float* scatWavefield, int iGpu,
                                      int iGpuId) {
    (void)srcWavefield; (void)scatWavefield; (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_BORN_EXT, iGpu));
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        fs.c.born_ext_forward(model, 1, &s, AIO_MEM_HOST);
    });
}
AIO_API int aio_BornTimeShotsAdjFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                      int* rp, int nr, float* srcWavefield, float* recWavefield, int iGpu,
                                      int iGpuId) {
    (void)srcWavefield; (void)recWavefield; (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_BORN_EXT, iGpu));
        aio_shot s = one_shot(sourcesSignals, sp, ns, rp, nr, dataRegDts);
        fs.c.born_ext_adjoint(model, 0, 1, &s, AIO_MEM_HOST);
    });
}
AIO_API int aio_tomoTimeShotsFwdFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                      int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int iGpu,
                                      int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_TOMO_EXT, iGpu));
        seam_tomo(fs.c, false, model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, w0, w1, w2,
                  saveWavefield);
    });
}
AIO_API int aio_tomoTimeShotsAdjFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                      int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int iGpu,
                                      int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        SeamFs fs(seam_ctx(AIO_TOMO_EXT, iGpu));
        seam_tomo(fs.c, true, model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, w0, w1, w2,
                  saveWavefield);
    });
}

// Subsurface-offset seam calls (the reference's *OffsetShots* drivers, optionally free-surface):
// the slot's context runs the call with the offset axis on.
struct SeamExt {
    Context& c;
    int ext, fs;
    SeamExt(Context& cc, bool freeSurface) : c(cc), ext(cc.P.extension), fs(cc.P.freeSurface) {
        c.P.extension = AIO_EXT_OFFSET;
        c.P.freeSurface = freeSurface ? 1 : 0;
    }
    ~SeamExt() {
        c.P.extension = ext;
        c.P.freeSurface = fs;
    }
};
static void seam_born_offset(float* model, float* dataRegDts, float* sig, int* sp, int ns, int* rp, int nr, int iGpu,
                             bool adjoint, bool fs) {
    SeamExt x(seam_ctx(AIO_BORN_EXT, iGpu), fs);
    aio_shot s = one_shot(sig, sp, ns, rp, nr, dataRegDts);
    if (adjoint) x.c.born_ext_adjoint(model, 0, 1, &s, AIO_MEM_HOST);
    else x.c.born_ext_forward(model, 1, &s, AIO_MEM_HOST);
}
AIO_API int aio_BornOffsetShotsFwdGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                      int* rp, int nr, float* srcWavefield, float* scatWavefield, int iGpu,
                                      int iGpuId) {
    (void)srcWavefield; (void)scatWavefield; (void)iGpuId;
    return guard([&] { seam_born_offset(model, dataRegDts, sourcesSignals, sp, ns, rp, nr, iGpu, false, false); });
}
AIO_API int aio_BornOffsetShotsAdjGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                      int* rp, int nr, float* srcWavefield, float* recWavefield, int iGpu,
                                      int iGpuId) {
    (void)srcWavefield; (void)recWavefield; (void)iGpuId;
    return guard([&] { seam_born_offset(model, dataRegDts, sourcesSignals, sp, ns, rp, nr, iGpu, true, false); });
}
AIO_API int aio_BornOffsetShotsFwdFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                        int* rp, int nr, float* srcWavefield, float* scatWavefield, int iGpu,
                                        int iGpuId) {
    (void)srcWavefield; (void)scatWavefield; (void)iGpuId;
    return guard([&] { seam_born_offset(model, dataRegDts, sourcesSignals, sp, ns, rp, nr, iGpu, false, true); });
}
AIO_API int aio_BornOffsetShotsAdjFsGpu(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns,
                                        int* rp, int nr, float* srcWavefield, float* recWavefield, int iGpu,
                                        int iGpuId) {
    (void)srcWavefield; (void)recWavefield; (void)iGpuId;
    return guard([&] { seam_born_offset(model, dataRegDts, sourcesSignals, sp, ns, rp, nr, iGpu, true, true); });
}
// Extended Born with saved wavefields (the reference's *Wavefield drivers): offsets / free surface as named.
static void seam_born_ext_wfld(float* model, float* dataRegDts, float* sig, int* sp, int ns, int* rp, int nr, int iGpu,
                               bool adjoint, bool offset, bool fs, float* srcW, float* secW) {
    Context& c = seam_ctx(AIO_BORN_EXT, iGpu);
    const int ext = c.P.extension, fs0 = c.P.freeSurface;
    c.P.extension = offset ? AIO_EXT_OFFSET : AIO_EXT_TIME;
    c.P.freeSurface = fs ? 1 : 0;
    aio_shot s = one_shot(sig, sp, ns, rp, nr, dataRegDts);
    try {
        if (adjoint) c.born_ext_adjoint_wavefield(model, 0, &s, AIO_MEM_HOST, srcW, secW);
        else c.born_ext_forward_wavefield(model, &s, AIO_MEM_HOST, srcW, secW);
    } catch (...) {
        c.P.extension = ext;
        c.P.freeSurface = fs0;
        throw;
    }
    c.P.extension = ext;
    c.P.freeSurface = fs0;
}
#define AIO_BORN_EXT_WFLD(NAME, ADJ, OFF, FS)                                                                   \
    AIO_API int NAME(float* model, float* dataRegDts, float* sourcesSignals, int* sp, int ns, int* rp, int nr,  \
                     float* srcWavefield, float* secWavefield, int iGpu, int iGpuId) {                          \
        (void)iGpuId;                                                                                           \
        return guard([&] {                                                                                      \
            seam_born_ext_wfld(model, dataRegDts, sourcesSignals, sp, ns, rp, nr, iGpu, ADJ, OFF, FS,           \
                               srcWavefield, secWavefield);                                                    \
        });                                                                                                     \
    }
AIO_BORN_EXT_WFLD(aio_BornTimeShotsFwdGpuWavefield, false, false, false)
AIO_BORN_EXT_WFLD(aio_BornOffsetShotsFwdGpuWavefield, false, true, false)
AIO_BORN_EXT_WFLD(aio_BornTimeShotsFwdFsGpuWavefield, false, false, true)
AIO_BORN_EXT_WFLD(aio_BornOffsetShotsFwdFsGpuWavefield, false, true, true)
AIO_BORN_EXT_WFLD(aio_BornTimeShotsAdjGpuWavefield, true, false, false)
AIO_BORN_EXT_WFLD(aio_BornOffsetShotsAdjGpuWavefield, true, true, false)
AIO_BORN_EXT_WFLD(aio_BornTimeShotsAdjFsGpuWavefield, true, false, true)
AIO_BORN_EXT_WFLD(aio_BornOffsetShotsAdjFsGpuWavefield, true, true, true)
#undef AIO_BORN_EXT_WFLD

static void seam_tomo_offset(float* model, float* dataRegDts, float* ext, float* sig, int* sp, int ns, int* rp, int nr,
                             int iGpu, float* w0, float* w1, float* w2, int saveWavefield, bool adjoint, bool fs) {
    SeamExt x(seam_ctx(AIO_TOMO_EXT, iGpu), fs);
    seam_tomo(x.c, adjoint, model, dataRegDts, ext, sig, sp, ns, rp, nr, w0, w1, w2, saveWavefield);
}
AIO_API int aio_tomoOffsetShotsFwdGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                      int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int iGpu,
                                      int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        seam_tomo_offset(model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, iGpu, w0, w1, w2,
                         saveWavefield,
                         false, false);
    });
}
AIO_API int aio_tomoOffsetShotsAdjGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                      int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int iGpu,
                                      int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        seam_tomo_offset(model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, iGpu, w0, w1, w2,
                         saveWavefield,
                         true, false);
    });
}
AIO_API int aio_tomoOffsetShotsFwdFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                        int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int iGpu,
                                        int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        seam_tomo_offset(model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, iGpu, w0, w1, w2,
                         saveWavefield,
                         false, true);
    });
}
AIO_API int aio_tomoOffsetShotsAdjFsGpu(float* model, float* dataRegDts, float* extReflectivity, float* sourcesSignals,
                                        int* sp, int ns, int* rp, int nr, float* w0, float* w1, float* w2, int iGpu,
                                        int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        seam_tomo_offset(model, dataRegDts, extReflectivity, sourcesSignals, sp, ns, rp, nr, iGpu, w0, w1, w2,
                         saveWavefield,
                         true, true);
    });
}

AIO_API int aio_initWemvaExtGpu(float dz, float dx, int nz, int nx, int nts, float dts, int sub, int minPad,
                                int blockSize, float alphaCos, int nExt, int leg1, int leg2, int nGpu, int iGpuId,
                                int iGpuAlloc) {
    (void)blockSize; (void)iGpuAlloc;
    return guard([&] {
        seam_init(AIO_WEMVA_EXT, dz, dx, nz, nx, nts, dts, sub, minPad, alphaCos, nExt, leg1, leg2, nGpu, iGpuId);
    });
}
AIO_API int aio_allocateWemvaExtShotsGpu(float* vel2Dtw2, float* reflectivityScale, int iGpu, int iGpuId) {
    return guard([&] { seam_allocate(AIO_WEMVA_EXT, vel2Dtw2, reflectivityScale, iGpu, iGpuId); });
}
AIO_API int aio_deallocateWemvaExtShotsGpu(int iGpu, int iGpuId) {
    (void)iGpuId;
    return guard([&] { seam_deallocate(AIO_WEMVA_EXT, iGpu); });
}
AIO_API int aio_wemvaTimeShotsFwdGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sp, int ns,
                                     float* wemvaDataRegDts, int* rp, int nr, float* w0, float* w1, float* w2,
                                     int iGpu, int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        seam_wemva(seam_ctx(AIO_WEMVA_EXT, iGpu), false, model, wemvaExtImage, sourcesSignals, sp, ns,
                   wemvaDataRegDts, rp, nr, w0, w1, w2, saveWavefield);
    });
}
AIO_API int aio_wemvaOffsetShotsFwdGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sp, int ns,
                                       float* wemvaDataRegDts, int* rp, int nr, float* w0, float* w1, float* w2,
                                       int iGpu, int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        SeamExt x(seam_ctx(AIO_WEMVA_EXT, iGpu), false);
        seam_wemva(x.c, false, model, wemvaExtImage, sourcesSignals, sp, ns, wemvaDataRegDts, rp, nr, w0, w1, w2,
                   saveWavefield);
    });
}
AIO_API int aio_wemvaOffsetShotsAdjGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sp, int ns,
                                       float* wemvaDataRegDts, int* rp, int nr, float* w0, float* w1, float* w2,
                                       int iGpu, int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        SeamExt x(seam_ctx(AIO_WEMVA_EXT, iGpu), false);
        seam_wemva(x.c, true, model, wemvaExtImage, sourcesSignals, sp, ns, wemvaDataRegDts, rp, nr, w0, w1, w2,
                   saveWavefield);
    });
}
AIO_API int aio_wemvaTimeShotsAdjGpu(float* model, float* wemvaExtImage, float* sourcesSignals, int* sp, int ns,
                                     float* wemvaDataRegDts, int* rp, int nr, float* w0, float* w1, float* w2,
                                     int iGpu, int iGpuId, int saveWavefield) {
    (void)iGpuId;
    return guard([&] {
        seam_wemva(seam_ctx(AIO_WEMVA_EXT, iGpu), true, model, wemvaExtImage, sourcesSignals, sp, ns,
                   wemvaDataRegDts, rp, nr, w0, w1, w2, saveWavefield);
    });
}
