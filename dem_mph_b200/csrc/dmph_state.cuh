// Device pointers of one solver context (see dmph_device.cuh for the layout).
#pragma once

#include "dmph_device.cuh"

namespace dmph {

struct DevState {
    // FP32 Verlet lists (list mode): entry k of slot i at
    // nbl[((k / 8) * N + i) * 8 + k % 8] = j | the offset (dx, dy, dz) of j's
    // rebuild-time cell from i's, each + 1 in two bits at bits 24, 26, 28 |
    // j's class (kEntrySolid, kEntryWall); ascending j; nbn[i] = count, -1
    // for slots without a list (dry walls).  A wall entry of lists built with
    // the walls at rest is a wall that stays put until the next rebuild.  Lists built with the walls at rest (dB[B_LIST_SPLIT] = 1) leave
    // the wall-wall pairs out of the walls' lists: their pass-A sums cannot
    // change before the next rebuild and are kept in vsp_st (FP64 strain sum)
    // and st4 (surface-tension density sum, gravity-centre sum)
    unsigned *nbl;
    int *nbn;
    int nbl_cap;
    double *vsp_st;
    float4 *st4;
    int *st_valid;  // 1: the slot's vsp_st and st4 hold (cleared whenever walls change slots)
    // FP64 particle state, component planes v[d*N + i], current sorted order
    double *pos, *vel, *frc, *xref;
    int *type, *pidx;
    // per-particle fields of the fluid passes
    double *vsp, *divp, *pres;      // VolStrainP, DivergenceP, PressureP
    double *densA, *pA, *gc;        // DensityA, PressureA, GravityCenter (3 planes)
    // DEM per-particle constants (persist across steps, never permuted)
    double *kn, *cn, *kt, *ct;
    double *alpha, *dragC;
    int *nc, *snc;                  // NeighborCount, SolidNeighborCount at rebuild
    // cell structure
    unsigned long long *skey;       // sorted (key << 32 | slot), P2 entries
    int *cell_start;                // 3T + 1 entries
    Chunk *chunks;
    // FP32 split-precision state (DMPH_PRECISION_FP32_SPLIT): positions relative
    // to the origin of the particle's rebuild-time cell, the cell coordinates
    // and type packed in .w (pack_cell), so every pair is formed in the frame
    // of one cell with FP32 magnitudes of a few particle spacings; v4.w holds
    // the pressure of the last pass A (0 for solids and for walls without
    // fluid in reach), read by pass B together with the velocity
    float4 *p4, *v4, *f4, *xref4, *gc4;
    // list reuse: positions (FP32 frame) when the current lists were built
    float4 *xrefL4;
    float *pres32, *vsp32, *div32, *densA32, *pA32;
    float *alpha32, *dragC32;
    // rigid clumps (DMPH_FLAG_RIGID_CLUMPS): body of each slot (-1: none) and
    // the density of each body; null when the mode is off
    int *bid;
    const double *body_rho;
    double *frc_dem;  // FP64 planes: DEM contact force of the current substep (clump mode)
};

// per-particle density: a debris body's own density when the particle belongs
// to one, else the density of its type
__device__ __forceinline__ double particle_density(const DevState &S, const DevParams &P, int i, int t)
{
    if (S.bid) {
        const int b = S.bid[i];
        if (b >= 0) return S.body_rho[b];
    }
    return P.density[t];
}

// Rigid debris bodies, FP64 (no counterpart in the reference).  Members are
// stored in body order (CSR over bodies) by their input row; slot_of_row maps
// a row to its current sorted slot and is refreshed at every rebuild.
struct DevBodies {
    int B;
    const int *ptr;         // B+1
    const int *member_row;  // members, by body
    int *slot_of_row;       // N
    const double *r0;       // 3 per member: offset from the centre of mass, body frame
    double *X, *V, *L;      // 3 per body: centre of mass, velocity, angular momentum (world)
    double *q;              // 4 per body: orientation (w, x, y, z), body -> world
    const double *M;        // mass
    const double *Iinv0;    // 9 per body: inverse inertia tensor, body frame
    double *Fsum, *Tsum;    // 3 per body: last substep's total force and torque (diagnostics)
};

// Blocked list layout: the entries of a particle come in blocks of 8 (one
// 32-byte sector); block b of slot i is at ((b * N) + i) * 8.  The build fills
// each particle's sectors one entry after the other, and a warp of consecutive
// slots reads entry k of its 32 particles from 32 sectors that also hold the
// particles' next entries.
constexpr unsigned kEntrySlot = 0xFFFFFFu;        // j
constexpr unsigned kEntrySolid = 1u << 30;         // j is debris
constexpr unsigned kEntryWall = 1u << 31;          // j is a wall
// cell offsets in -1..1 -> entry bits 24-29
__host__ __device__ __forceinline__ unsigned entry_offsets(int dx, int dy, int dz)
{
    return ((unsigned)(dx + 1) << 24) | ((unsigned)(dy + 1) << 26) | ((unsigned)(dz + 1) << 28);
}
// offset along axis a as a float: the two bits v = offset + 1 are placed in
// the mantissa of 2^23 (2^23 + v exactly), and 2^23 + 1 is subtracted
__host__ __device__ __forceinline__ float entry_offset(unsigned e, int a)
{
    union {
        unsigned u;
        float f;
    } c;
    c.u = 0x4B000000u | ((e >> (24 + 2 * a)) & 3u);
    return c.f - 8388609.0f;
}

__host__ __device__ __forceinline__ long long list_index(int k, int i, long long ld)
{
    return (((long long)(k >> 3)) * ld + i) * 8 + (k & 7);
}


#ifdef __CUDACC__
// rigid-body helpers shared by the body kernels and the surrogate
__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ void quat_to_R(const double *q, double R[3][3])
{
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    R[0][0] = 1.0 - 2.0 * (y * y + z * z);
    R[0][1] = 2.0 * (x * y - w * z);
    R[0][2] = 2.0 * (x * z + w * y);
    R[1][0] = 2.0 * (x * y + w * z);
    R[1][1] = 1.0 - 2.0 * (x * x + z * z);
    R[1][2] = 2.0 * (y * z - w * x);
    R[2][0] = 2.0 * (x * z - w * y);
    R[2][1] = 2.0 * (y * z + w * x);
    R[2][2] = 1.0 - 2.0 * (x * x + y * y);
}

// w = R I0^-1 R^T L
__device__ __forceinline__ void omega_of(const double R[3][3], const double *Ii, const double *L, double *w)
{
    double a[3], b[3];
    for (int r = 0; r < 3; r++) a[r] = R[0][r] * L[0] + R[1][r] * L[1] + R[2][r] * L[2];  // R^T L
    for (int r = 0; r < 3; r++) b[r] = Ii[3 * r] * a[0] + Ii[3 * r + 1] * a[1] + Ii[3 * r + 2] * a[2];
    for (int r = 0; r < 3; r++) w[r] = R[r][0] * b[0] + R[r][1] * b[1] + R[r][2] * b[2];
}

#endif

// .w of the FP32 position: type (3 bits) | cx (10) | cy (10) | cz (9)
__host__ __device__ inline unsigned pack_cell(int t, int cx, int cy, int cz)
{
    return (unsigned)t | ((unsigned)cx << 3) | ((unsigned)cy << 13) | ((unsigned)cz << 23);
}
__host__ __device__ inline int unpack_type(unsigned w) { return (int)(w & 7u); }
__host__ __device__ inline int unpack_cx(unsigned w) { return (int)((w >> 3) & 1023u); }
__host__ __device__ inline int unpack_cy(unsigned w) { return (int)((w >> 13) & 1023u); }
__host__ __device__ inline int unpack_cz(unsigned w) { return (int)((w >> 23) & 511u); }

// FP32 copies of the scene constants used by the split-precision kernels
struct DevParams32 {
    float cw[3];
    float dx, V, dt, ddt, dx2;
    float RP2, RV2, RA2, RG2;
    float iRP, iRV, iRA, iRG;            // 1/h
    float Bp, Bv, Ba, Bg;                // (1/Sw)/h^dim
    float dwp, dwv, dwg;                 // -2 B / h of the quadratic kernels
    float N0p, N0a, R2g_inv_RG;          // RG / R2g
    float viscC, Reff, Vdx;              // V/dx
    float g[3];
    float mass[kTypes], density[kTypes], bulk[kTypes], bvisc[kTypes], svisc[kTypes], friction[kTypes];
    float CofA[kTypes], ai[kTypes];
    float ratio[kTypes][kTypes];
    float Eeff[kTypes][kTypes], KtFac[kTypes][kTypes];
    float logE[kTypes], cnDen[kTypes], ctFac[kTypes];
    float drag_pref;                     // 0.5 dx^3
    float dwpV;                          // -2 Bp / RP * V
    double N0p32;                        // lattice sum evaluated with the FP32 kernel arithmetic
    float muij[kTypes][kTypes];          // C * harmonic-mean viscosity * 2 Bv / RV * V
};

// Moving-wall constants (calculateWall, source/DEM-MPH.cpp:2846-2900)
struct WallMotion {
    double R[kTypes][3][3];
    double C[kTypes][3];
    double Vel[kTypes][3];
    double Om[kTypes][3];
    int moving;  // 1 when 0.2 <= Time <= 0.4 for this step
};

// One scene of an ensemble as the ensemble kernels see it (a device array of
// these is the scene table)
constexpr int kMaxEnsemble = 256;
constexpr int kPassVariants = 5;
constexpr int kListVariants = 4;
struct EnsScene {
    DevParams P;
    DevParams32 Q;
    DevState S;
    int *dB;
    unsigned long long *maxshift;  // the scene's max-shift accumulator (drift -> decision)
    DevBodies Bd;                  // its rigid bodies (B = 0: none)
    int demSteps;                  // DEM substeps per step of the scene
};

#ifdef __CUDACC__
// Block-wide exclusive prefix of a per-scene count over the scene table:
// pre[k] = sum of count(j) for j < k, pre[ns] the total (in shared memory,
// kMaxEnsemble + 1 entries); every thread of the block must call it.
template <class Count>
__device__ __forceinline__ int ens_count_prefix(int ns, int *pre, Count count)
{
    for (int k = threadIdx.x; k < ns; k += blockDim.x) pre[k + 1] = count(k);
    __syncthreads();
    if (threadIdx.x == 0) {
        pre[0] = 0;
        for (int k = 0; k < ns; ++k) pre[k + 1] += pre[k];
    }
    __syncthreads();
    return pre[ns];
}
// the scene k with pre[k] <= g < pre[k + 1] (pre ascending)
__device__ __forceinline__ int ens_scene_at(const int *pre, int ns, int g)
{
    int lo = 0, hi = ns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
#endif

}  // namespace dmph
