// Shared definitions for the B200 acoustic-isotropic engine: grid geometry,
// device memory layouts, per-shot descriptors and launch argument blocks.
//
// Device layouts (all FP32 unless stated):
//   * halo slice  — the two time levels of the fine-time stepper. Column-major
//     in x with pitch `hp` floats; interior point (z, x) (0-based interior
//     coordinates, z fastest) lives at (x + 5) * hp + 32 + z. The 5-point ring
//     around the interior and all padding stay zero, which is the reference's
//     zero Dirichlet FAT boundary (F/src/kernelsGpu.cu:513-552 only writes the
//     interior). Interior rows start 128-byte aligned.
//   * interior slice — everything that lives on interior points only (v^2 dtw^2,
//     2/v^3, models, images, coarse wavefield samples): (z, x) at x * ip + z,
//     ip = round_up(nzi, 32). Padding lanes stay zero so element-wise kernels may
//     sweep whole pitched slices.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace aio {

constexpr int FAT = 5;        // stencil half-width (10th order), F/include/varDeclare.h:8
constexpr int SUB_MAX = 100;  // F/include/varDeclare.h:12
constexpr int PAD_MAX = 200;  // F/include/varDeclare.h:11
constexpr int TZ = 32;        // stepper tile along z (one warp)
constexpr int TX = 32;        // stepper tile along x
constexpr int TY = 8;         // warps per stepper CTA; each thread owns TX/TY x-points
constexpr int PX = TX / TY;   // x-points per thread
constexpr int ZOFF = 32;      // offset of interior z=0 inside a halo column

inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

struct Geom {
    int nz, nx;        // full grid including the FAT ring (reference nz, nx)
    int nzi, nxi;      // interior extent nz-2*FAT, nx-2*FAT
    int hp, hcols;     // halo slice pitch (floats) and column count
    int ip;            // interior slice pitch (floats)
    long long hsz;     // floats per halo slice
    long long isz;     // floats per interior slice
    int nts, sub, ntw; // coarse samples, sub-stepping, fine samples
    int minPad, nExt, hExt, H;  // sponge width, extension length/half, filter half-length
    int tilesZ, tilesX;
};

inline Geom make_geom(int nz, int nx, int nts, int sub, int minPad, int nExt) {
    Geom g;
    g.nz = nz; g.nx = nx;
    g.nzi = nz - 2 * FAT; g.nxi = nx - 2 * FAT;
    g.hp = ZOFF + round_up(g.nzi, TZ) + 32;
    g.hcols = round_up(g.nxi, TX) + 2 * FAT;
    g.ip = round_up(g.nzi, 32);
    g.hsz = (long long)g.hp * g.hcols;
    g.isz = (long long)g.ip * g.nxi;
    g.nts = nts; g.sub = sub; g.ntw = (nts - 1) * sub + 1;
    g.minPad = minPad; g.nExt = nExt; g.hExt = (nExt - 1) / 2; g.H = sub + 1;
    g.tilesZ = (g.nzi + TZ - 1) / TZ;
    g.tilesX = (g.nxi + TX - 1) / TX;
    return g;
}

// Sparse device list for one shot: CSR over stepper tiles. Entry .x packs the
// point's position inside its tile (lx * TZ + lz); .y is the regular-device index.
struct SparseList {
    const int* tileStart;  // tilesZ*tilesX + 1 offsets (nullptr = no devices)
    const int2* ent;
};

// Per-shot state used by the fused stepper. All pointers are device pointers.
struct ShotDesc {
    float* p[2];              // halo slices; p[parity] is the current level
    float* ss;                // secondary-source ring (interior slices)
    float* acc;               // accumulation target ring / wavefield (interior slices)
    SparseList inj;           // injection points
    const float* injSig;      // injected traces [nDev][injLd]
    SparseList rec;           // recording points
    float* recSig;            // recorded traces [nDev][recLd]
    int injLd, recLd;
};

// Scheme constants shared by every launch of one operator instance.
struct Coefs {
    float zc[6], xc[6];
};

// Uniform arguments of one fused fine-step launch.
struct StepArgs {
    Geom g;
    Coefs c;
    const float* v2;        // v^2 dtw^2, interior slice
    const float* taper;     // cosine taper, minPad entries
    const ShotDesc* shots;  // gridDim.z entries
    int parity;
    long long ssOffA, ssOffB;    // dense injection slices (offsets into ss)
    float hInjA, hInjB;
    int injTA, injTB;            // sparse injection time indices (injTB < 0: single term)
    float injCA, injCB;
    int recTA, recTB;            // sparse recording time indices (recTB < 0: single term)
    float recCA, recCB;
    long long accOffA, accOffB;  // accumulation slices (offsets into acc)
    float hAccA, hAccB;
    int fs;                      // free surface at the top interior row
};

}  // namespace aio
