// Device-side definitions shared by the DEM-MPH kernels.
//
// Layout in HBM (all arrays indexed by the particle's position in the current
// cell-sorted order, as the reference's arrays are after
// calculateCellParticle, source/DEM-MPH.cpp:1288-1519):
//   - FP64 vectors as three component planes  v[d * N + i]  (coalesced SoA),
//   - per-particle scalars as flat arrays,
//   - the sorted cell keys packed with their payload as 64-bit words
//     (key << 32 | original slot), padded to the power of two above N,
//   - cell_start[k] = first sorted slot whose key is >= k, k in [0, 3T]:
//     fluid cells are keys [0,T), solid [T,2T), wall [2T,3T),
//   - chunks: the warp work list; each chunk is <= 32 consecutive particles
//     of one (class, cell) key, so the 32 lanes of a warp share one stencil.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dmph.h"

namespace dmph {

constexpr int kTypes = DMPH_TYPE_COUNT;
constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
// list reuse: the widest list skin past MaxRadius, in hundredths of dx (the
// cells are MaxRadius + this wide)
constexpr int kSkinMaxHundredths = 40;

__host__ __device__ inline bool is_fluid(int t) { return DMPH_FLUID_BEGIN <= t && t < DMPH_FLUID_END; }
__host__ __device__ inline bool is_solid(int t) { return DMPH_SOLID_BEGIN <= t && t < DMPH_SOLID_END; }
__host__ __device__ inline bool is_wall(int t) { return DMPH_WALL_BEGIN <= t && t < DMPH_WALL_END; }

// Constants of one scene, passed by value to every kernel (kernel parameters
// live in the constant bank, so reads are broadcast).  Every derived constant
// is computed on the host with the reference's own expression order, so the
// device sees bit-identical values.
struct DevParams {
    int dim;
    int N;       // ParticleCount
    int T;       // TotalCellCount
    int cc[3];   // CellCount
    int P2;      // PowerParticleCount
    int P2log;   // ParticleCountPower
    int surface_tension;
    int wall_dem_coeffs;
    double dx, V;          // ParticleSpacing, ParticleVolume
    double W[3], hW[3];    // DomainWidth and 0.5*DomainWidth
    double dmin[3];        // DomainMin
    double cw[3];          // CellWidth
    double RA, RG, RP, RV; // kernel radii
    double RA2, RG2, RP2, RV2, rc2, dx2;  // squared radii, (MaxRadius+MARGIN)^2, dx*dx
    double Ba, Bg, Bp, Bv; // (1/Sw)/h^dim of each kernel
    double N0a, N0p, R2g, CofK;
    double viscC;          // 8 (2D) or 10 (3D)
    double dt, ddt;        // Dt, DEMDt
    double Reff;           // dx*dx/(dx+dx)
    double g[3];
    double CofA[kTypes];
    double ai[kTypes];     // CofA[t]*CofK*CofK
    double mass[kTypes];   // Density*ParticleVolume
    double density[kTypes], bulk[kTypes], bvisc[kTypes], svisc[kTypes];
    double friction[kTypes];
    double ratio[kTypes][kTypes];
    double Eeff[kTypes][kTypes];      // effective Young modulus of a type pair
    double KtFac[kTypes][kTypes];     // 8 yi yj / ((1+pi)(2-pi)yj + (1+pj)(2-pj)yi)
    double logE[kTypes];              // log(RestitutionCoefficient)
    double cnDen[kTypes];             // sqrt(pi^2 + log(e)^2)
    double ctFac[kTypes];             // -2 log(e) / sqrt(pi^2 + log(e)^2)
    // pair-symmetric contact constants of the rigid-clump mode
    double pairDamp[kTypes][kTypes];  // -2 log(e_ij) / sqrt(pi^2 + log(e_ij)^2), e_ij = (e_i + e_j)/2
    double pairFric[kTypes][kTypes];  // (mu_i + mu_j)/2
};

struct Chunk {
    int i0;   // first sorted slot
    int cnt;  // 1..32 particles
};

// Device-resident bounds of the current cell sort, written by the rebuild
// kernels and read by every kernel that walks chunks or slot ranges, so that
// launch shapes never depend on host-side values (a step can be captured in a
// CUDA graph and replayed).
enum DevBound {
    B_CH_S0 = 0,    // first solid chunk
    B_CH_W0 = 1,    // first wall chunk
    B_CH_END = 2,   // number of chunks
    B_CH_WET = 3,   // end of the wall chunks with fluid in reach (FP32 pass A)
    B_FE = 4,       // fluid slots [0, fe)
    B_SB = 5,       // solid slots [sb, se)
    B_SE = 6,
    B_NEED = 7,     // rebuild decided for this step
    B_REBUILDS = 8, // rebuilds since creation
    B_LIST_OVF = 9, // a Verlet list of the last rebuild overflowed (FP32 list mode): stencil passes run
    B_LIST_SPLIT = 10, // the FP32 lists hold no wall-wall pairs (built with the walls at rest)
    B_NONFINITE = 11,  // a drift met a non-finite position or velocity (sticky; no rebuild runs while set)
    // list reuse (FP32 lists kept across rebuild triggers): B_NEED = 1 for a
    // full rebuild (sort and lists), 2 for a trigger that keeps the lists
    B_SKIN = 12,        // skin of the current lists past MaxRadius, hundredths of dx (10 = MARGIN)
    B_SKIN_NEXT = 13,   // skin of the lists the next build makes
    B_GAP = 14,         // steps since the last rebuild trigger
    B_LIST_BUILDS = 15, // full rebuilds (cell sort and lists) since creation, the first excluded
    B_COUNT = 16
};

enum ChunkRange { CR_ALL = 0, CR_FLUID_SOLID = 1, CR_SOLID = 2, CR_WALL = 3, CR_WET = 4 };

__device__ __forceinline__ void chunk_range(const int *dB, int kind, int &b, int &e)
{
    switch (kind) {
    case CR_FLUID_SOLID: b = 0; e = dB[B_CH_W0]; break;
    case CR_SOLID: b = dB[B_CH_S0]; e = dB[B_CH_W0]; break;
    case CR_WALL: b = dB[B_CH_W0]; e = dB[B_CH_END]; break;
    case CR_WET: b = 0; e = dB[B_CH_WET]; break;
    default: b = 0; e = dB[B_CH_END]; break;
    }
}

// Grid of a persistent kernel: as many blocks as can be resident at once on
// the device (queried once per kernel through the occupancy API).
inline int persistent_grid(const void *kernel, int block_threads)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block_threads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return sms * per_sm;
}

// elementwise slot loop over [dB[kb], dB[ke]) (kb < 0: from 0)
#define FOR_EACH_SLOT(dB, kb, ke, i)                                                                   \
    const int sb_ = (kb) < 0 ? 0 : dB[kb], se_ = dB[ke];                                              \
    for (int i = sb_ + blockIdx.x * blockDim.x + threadIdx.x; i < se_; i += gridDim.x * blockDim.x)

// persistent warp loop over the chunks of a range: every warp of the grid
// takes chunks b + w, b + w + W, ...
#define FOR_EACH_CHUNK(dB, kind, WARPS_PER_BLOCK, cidx)                                        \
    int cb_, ce_;                                                                            \
    chunk_range(dB, kind, cb_, ce_);                                                         \
    for (int cidx = cb_ + blockIdx.x * (WARPS_PER_BLOCK) + (int)(threadIdx.x >> 5); cidx < ce_; \
         cidx += gridDim.x * (WARPS_PER_BLOCK))

// 64-bit sort word: key in the high half, payload (slot) in the low half
__host__ __device__ inline uint32_t word_key(unsigned long long w) { return (uint32_t)(w >> 32); }
__host__ __device__ inline uint32_t word_slot(unsigned long long w) { return (uint32_t)(w & 0xffffffffull); }

__host__ __device__ inline int wrapi(int a, int c) { return ((a) % c + c) % c; }

__host__ __device__ inline int cell_id(const DevParams &P, int ix, int iy, int iz)
{
    if (P.dim == 2) return wrapi(ix, P.cc[0]) * P.cc[1] + wrapi(iy, P.cc[1]);
    return wrapi(ix, P.cc[0]) * P.cc[1] * P.cc[2] + wrapi(iy, P.cc[1]) * P.cc[2] + wrapi(iz, P.cc[2]);
}

// The periodic 3x3(x3) stencil of a cell in the reference's visiting order
// (calculateNeighbor, source/DEM-MPH.cpp:1553-1575 and the loops after it):
// per axis the wrapped neighbours c-1, c, c+1 rotated to start at
// jmin = max(0, 2r - (c+r) % C), which lists them in ascending wrapped index;
// x outer, z inner.  Returns the number of cells (27 in 3D, 9 in 2D).
// `key_cell` is the sorted key reduced modulo T.
__host__ __device__ inline int stencil_cell(const DevParams &P, int key_cell, int s)
{
    const int c1 = P.cc[1], c2 = P.cc[2];
    const int ic[3] = {key_cell / (c1 * c2), (key_cell / c2) % c1, key_cell % c2};
    const int nz = (P.dim == 2) ? 1 : 3;
    const int sidx[3] = {s / (3 * nz), (s / nz) % 3, s % nz};
    int out[3];
    for (int d = 0; d < 3; d++) {
        const int r = (P.dim == 2 && d == 2) ? 0 : 1;
        const int n = 2 * r + 1;
        const int b = (2 * r) - (ic[d] + r) % P.cc[d];
        const int jmin = b > 0 ? b : 0;
        const int j = (jmin + sidx[d]) % n;
        out[d] = wrapi(ic[d] - r + j, P.cc[d]);
    }
    return cell_id(P, out[0], out[1], out[2]);
}

__host__ __device__ inline int stencil_size(const DevParams &P) { return P.dim == 2 ? 9 : 27; }

}  // namespace dmph
