// FP64 timestep kernels (the parity build).
//
// Compiled with -fmad=false and IEEE division/sqrt: every expression keeps
// the reference's evaluation order (source/DEM-MPH.cpp), so that results
// agree with the reference bit for bit except where CUDA's pow() differs
// from the host libm by an ulp (drag coefficient only).
//
// Per step:  k_drift (convection, walls, periodic wrap, force reset and the
// rebuild trigger fused), then after an optional rebuild k_pass_a (densities,
// divergence, pressure), k_pass_b (all fluid forces, drag, buoyancy, gravity,
// fluid velocity update), and per DEM substep k_dem_force + k_dem_integrate.
#include <math_constants.h>

#include "dmph_state.cuh"
#include "dmph_traverse.cuh"

namespace dmph {

__device__ __forceinline__ double pmod(double a, double w) { return ((a) - (w)*floor((a) / (w))); }

// Mod(x_j - x_i + W/2, W) - W/2 of every pair loop (:76 and e.g. :2145).
// When 0 <= t <= 0.75 W, floor(t/W) is 0 and Mod returns t exactly, so the
// division is skipped; any other t takes the reference formula.
__device__ __forceinline__ double rel1(double xj, double xi, double W, double hW)
{
    const double t = xj - xi + hW;
    const double m = (t >= 0.0 && t <= 0.75 * W) ? t : pmod(t, W);
    return m - hW;
}

// smoothing kernels :272-342; B = (1/Sw)/h^dim
__device__ __forceinline__ double k_wa(double r, double B, double h) { return B * (r / h) * (1.0 - (r / h)) * (1.0 - (r / h)); }
__device__ __forceinline__ double k_dwa(double r, double B, double h)
{
    return B * (1.0 - (r / h)) * (1.0 - 3.0 * (r / h)) * (1.0 / h);
}
__device__ __forceinline__ double k_w(double r, double B, double h) { return B * ((1.0 - r / h) * (1.0 - r / h)); }
__device__ __forceinline__ double k_dw(double r, double B, double h) { return B * (-2.0 / h * (1.0 - r / h)); }

struct TileA {
    double x[kWarp], y[kWarp], z[kWarp], vx[kWarp], vy[kWarp], vz[kWarp];
    int t[kWarp];
};
struct TileB {
    double x[kWarp], y[kWarp], z[kWarp], vx[kWarp], vy[kWarp], vz[kWarp], p[kWarp];
    double pa[kWarp], gx[kWarp], gy[kWarp], gz[kWarp];
    int t[kWarp];
};

constexpr int kWarpsPerBlock = 4;

// ------------------------------------------------------------------ drift
// calculateConvection :1860, calculateWall :2846, calculatePeriodicBoundary
// :3153, resetForce :1894 and the displacement reduction of
// neighborCalculation :1264-1286, fused; max |dx|^2 is reduced into *maxshift
// as the bit pattern of a non-negative double.
__global__ void k_drift(DevParams P, DevState S, WallMotion Wm, unsigned long long *maxshift)
{
    const int N = P.N;
    double m2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int t = S.type[i];
        double x[3], v[3];
        for (int d = 0; d < 3; d++) {
            x[d] = S.pos[d * N + i];
            v[d] = S.vel[d * N + i];
        }
        if (is_fluid(t))
            for (int d = 0; d < 3; d++) x[d] += v[d] * P.dt;
        if (is_wall(t)) {
            if (Wm.moving) {
                double r[3] = {x[0] - Wm.C[t][0], x[1] - Wm.C[t][1], x[2] - Wm.C[t][2]};
                const double(*R)[3] = Wm.R[t];
                const double *w = Wm.Om[t];
                r[0] = R[0][0] * r[0] + R[0][1] * r[1] + R[0][2] * r[2];
                r[1] = R[1][0] * r[0] + R[1][1] * r[1] + R[1][2] * r[2];
                r[2] = R[2][0] * r[0] + R[2][1] * r[1] + R[2][2] * r[2];
                v[0] = w[1] * r[2] - w[2] * r[1] + Wm.Vel[t][0];
                v[1] = w[2] * r[0] - w[0] * r[2] + Wm.Vel[t][1];
                v[2] = w[0] * r[1] - w[1] * r[0] + Wm.Vel[t][2];
                x[0] = r[0] + Wm.C[t][0] + Wm.Vel[t][0] * P.dt;
                x[1] = r[1] + Wm.C[t][1] + Wm.Vel[t][1] * P.dt;
                x[2] = r[2] + Wm.C[t][2] + Wm.Vel[t][2] * P.dt;
            } else {
                v[0] = 0.0;
                v[1] = 0.0;
                v[2] = 0.0;
            }
        }
        double d3[3];
        for (int d = 0; d < 3; d++) {
            x[d] = pmod(x[d] - P.dmin[d], P.W[d]) + P.dmin[d];
            S.pos[d * N + i] = x[d];
            S.vel[d * N + i] = v[d];
            S.frc[d * N + i] = 0.0;
            d3[d] = pmod(x[d] - S.xref[d * N + i] + 0.5 * P.W[d], P.W[d]) - 0.5 * P.W[d];
        }
        const double s = d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2];
        m2 = s > m2 ? s : m2;
        // a non-finite position or velocity makes the maximum +inf, which the
        // rebuild decision reports instead of rebuilding
        if (!isfinite(x[0] + x[1] + x[2] + v[0] + v[1] + v[2])) m2 = CUDART_INF;
    }
    // warp then block max; one atomic per block
    unsigned long long b = __double_as_longlong(m2);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_down_sync(kFull, b, o);
        b = ob > b ? ob : b;
    }
    __shared__ unsigned long long red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long mx = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) mx = red[w] > mx ? red[w] : mx;
        atomicMax(maxshift, mx);
    }
}

// ------------------------------------------------------------------ pass A
// calculateDensityA :1956, calculateGravityCenter :1987, calculateDensityP
// :2129, calculateDivergenceP :2158, calculatePhysicalCoefficients :1918 and
// the pressures of calculatePressureP :2203-2208 and calculatePressureA
// :2026-2031, for every particle.
// LIST: walk each particle's Verlet list (the reference's own neighbour list,
// same order) instead of the stencil; gate: this stencil launch stands in
// only after a list overflow
template <bool LIST>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_pass_a(DevParams P, DevState S, const int *dB, int range,
                                                                   int init_only, int gate)
{
    if (LIST ? dB[B_LIST_OVF] != 0 : (gate && dB[B_LIST_OVF] == 0)) return;
    __shared__ TileA tiles[kWarpsPerBlock];
    TileA &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    auto body = [&](const int i, const bool active, const int key_cell, const int ii) {
        const int ti = S.type[ii];
        const double xi = S.pos[ii], yi = S.pos[N + ii], zi = S.pos[2 * N + ii];
        const double vxi = S.vel[ii], vyi = S.vel[N + ii], vzi = S.vel[2 * N + ii];
        double vsp = 0.0, div = 0.0, dA = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
        const bool st = P.surface_tension;
        traverse_pairs<LIST>(
            P, S, key_cell, lane, active, i, 7u,
            [&](int j, int slot) {
                tl.x[slot] = S.pos[j];
                tl.y[slot] = S.pos[N + j];
                tl.z[slot] = S.pos[2 * N + j];
                tl.vx[slot] = S.vel[j];
                tl.vy[slot] = S.vel[N + j];
                tl.vz[slot] = S.vel[2 * N + j];
                tl.t[slot] = S.type[j];
            },
            [&](int j, int s) {
                if (j == i) return;
                const double q0 = rel1(tl.x[s], xi, P.W[0], P.hW[0]);
                const double q1 = rel1(tl.y[s], yi, P.W[1], P.hW[1]);
                const double q2 = rel1(tl.z[s], zi, P.W[2], P.hW[2]);
                const double r2 = (q0 * q0 + q1 * q1 + q2 * q2);
                const int tj = tl.t[s];
                if (st && !(is_solid(ti) && is_wall(tj))) {
                    const double ratio = P.ratio[ti][tj];
                    if (r2 <= P.RA2) dA += ratio * k_wa(sqrt(r2), P.Ba, P.RA);
                    if (r2 <= P.RG2) {
                        const double w = ratio * k_w(sqrt(r2), P.Bg, P.RG);
                        g0 += q0 * w / P.R2g * P.RG;
                        g1 += q1 * w / P.R2g * P.RG;
                        g2 += q2 * w / P.R2g * P.RG;
                    }
                }
                if (r2 <= P.RP2) {
                    const double r = sqrt(r2);
                    vsp += k_w(r, P.Bp, P.RP);
                    const bool skip = (is_solid(ti) && is_wall(tj)) || (is_solid(tj) && is_wall(ti)) ||
                                      (is_solid(tj) && is_solid(ti));
                    if (!skip) {
                        const double dw = k_dw(r, P.Bp, P.RP);
                        const double e0 = q0 / r, e1 = q1 / r, e2 = q2 / r;
                        const double u0 = tl.vx[s] - vxi, u1 = tl.vy[s] - vyi, u2 = tl.vz[s] - vzi;
                        div -= u0 * e0 * dw;
                        div -= u1 * e1 * dw;
                        div -= u2 * e2 * dw;
                    }
                }
            });
        if (!active) return;
        const double volstrain = (vsp - P.N0p);
        S.vsp[i] = volstrain;
        if (st) {
            S.densA[i] = dA;
            S.gc[i] = g0;
            S.gc[N + i] = g1;
            S.gc[2 * N + i] = g2;
        }
        if (init_only) return;  // initialisation evaluates only the densities (:423-425)
        S.divp[i] = div;
        double kappa = P.bulk[ti];
        if (volstrain < 0.0) kappa = 0.0;
        if (!is_solid(ti)) S.pres[i] = -P.bvisc[ti] * div + kappa * volstrain;
        if (st) {
            double pa = P.CofA[ti] * (dA - P.N0a) / P.dx;
            if (P.N0a <= dA) pa = 0.0;
            S.pA[i] = pa;
        }
    };
    if (LIST) {
        // one thread per slot: nothing in the list walk is warp-synchronous
        const int end = range == CR_ALL ? N : dB[B_SE];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) body(i, true, 0, i);
    } else {
        FOR_EACH_CHUNK(dB, range, kWarpsPerBlock, cidx)
        {
            const Chunk ch = S.chunks[cidx];
            const int i = ch.i0 + lane;
            const bool active = lane < ch.cnt;
            body(i, active, (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T), active ? i : ch.i0);
        }
    }
}

// ------------------------------------------------------------------ pass B
// For fluid and solid particles: calculateDragForce :2740 (twice, :490 and
// :512), calculatePressureP :2210-2245, calculatePressureA :2033-2070,
// calculateDiffuseInterface :2074-2126, calculateViscosityV :2248-2292,
// calculateBuoyancyForce :2699-2737, calculateGravity :2811 and
// (calculateAcceleration :2832 follows in k_fluid_accel).  Each reference kernel's per-particle sum is
// kept in its own accumulator and added to Force in the reference's call
// order, so the sums are bit-identical.  Wall particles are not visited:
// their forces are reset at the next step without ever being read.
template <bool LIST>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_pass_b(DevParams P, DevState S, const int *dB, int range,
                                                                   int gate)
{
    if (LIST ? dB[B_LIST_OVF] != 0 : (gate && dB[B_LIST_OVF] == 0)) return;
    __shared__ TileB tiles[kWarpsPerBlock];
    TileB &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    auto body = [&](const int i, const bool active, const int key_cell, const int ii) {
        const int ti = S.type[ii];
        const bool sol = is_solid(ti);
        const double xi = S.pos[ii], yi = S.pos[N + ii], zi = S.pos[2 * N + ii];
        const double vxi = S.vel[ii], vyi = S.vel[N + ii], vzi = S.vel[2 * N + ii];
        const double Pi = S.pres[ii];
        const bool st = P.surface_tension;
        double pai = 0.0, gci0 = 0.0, gci1 = 0.0, gci2 = 0.0;
        if (st) {
            pai = S.pA[ii];
            gci0 = S.gc[ii];
            gci1 = S.gc[N + ii];
            gci2 = S.gc[2 * N + ii];
        }
        const double mui = P.svisc[ti];
        const double rhoi = particle_density(S, P, ii, ti);
        double alpha = 0.0;
        if (sol) {
            const int nci = S.nc[ii];
            alpha = nci > 0 ? (double)(S.snc[ii]) / (nci) : 0.0;
        }
        const double ai = P.ai[ti];
        double fP[3] = {0.0, 0.0, 0.0}, fA[3] = {0.0, 0.0, 0.0}, fI[3] = {0.0, 0.0, 0.0};
        double fV[3] = {0.0, 0.0, 0.0}, fD[3] = {0.0, 0.0, 0.0}, fB[3] = {0.0, 0.0, 0.0};
        double dragc = 0.0;
        bool have_drag = false;
        traverse_pairs<LIST>(
            P, S, key_cell, lane, active, i, 7u,
            [&](int j, int slot) {
                tl.x[slot] = S.pos[j];
                tl.y[slot] = S.pos[N + j];
                tl.z[slot] = S.pos[2 * N + j];
                tl.vx[slot] = S.vel[j];
                tl.vy[slot] = S.vel[N + j];
                tl.vz[slot] = S.vel[2 * N + j];
                tl.p[slot] = S.pres[j];
                tl.t[slot] = S.type[j];
                if (st) {
                    tl.pa[slot] = S.pA[j];
                    tl.gx[slot] = S.gc[j];
                    tl.gy[slot] = S.gc[N + j];
                    tl.gz[slot] = S.gc[2 * N + j];
                }
            },
            [&](int j, int s) {
                if (j == i) return;
                const double q[3] = {rel1(tl.x[s], xi, P.W[0], P.hW[0]), rel1(tl.y[s], yi, P.W[1], P.hW[1]),
                                     rel1(tl.z[s], zi, P.W[2], P.hW[2])};
                const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                const int tj = tl.t[s];
                const double u[3] = {tl.vx[s] - vxi, tl.vy[s] - vyi, tl.vz[s] - vzi};
                // pressure (solid i skipped entirely; fluid i skips no pair)
                if (!sol && r2 < P.RP2) {
                    const double r = sqrt(r2);
                    const double dw = k_dw(r, P.Bp, P.RP);
                    const double pij = Pi + tl.p[s];
                    for (int d = 0; d < 3; d++) fP[d] += pij * (dw * q[d] / r) * P.V;
                }
                const bool sw = (sol && is_wall(tj)) || (is_solid(tj) && is_wall(ti));
                if (st && !sw) {
                    const double rij_ = P.ratio[ti][tj], rji_ = P.ratio[tj][ti];
                    if (r2 < P.RA2) {
                        const double r = sqrt(r2);
                        const double dwij = rij_ * k_dwa(r, P.Ba, P.RA);
                        const double dwji = rji_ * k_dwa(r, P.Ba, P.RA);
                        const double paj = tl.pa[s];
                        for (int d = 0; d < 3; d++) fA[d] += (pai * dwij + paj * dwji) * (q[d] / r) * P.V;
                    }
                    if (r2 < P.RG2) {
                        const double r = sqrt(r2);
                        const double wij = rij_ * k_w(r, P.Bg, P.RG);
                        const double wji = rji_ * k_w(r, P.Bg, P.RG);
                        const double gj[3] = {tl.gx[s], tl.gy[s], tl.gz[s]};
                        const double gi[3] = {gci0, gci1, gci2};
                        const double aj = ai;  // the reference uses particle i's CofA here (:2088)
                        for (int d = 0; d < 3; d++)
                            fI[d] -= (aj * gj[d] * wji - ai * gi[d] * wij) / P.R2g * P.RG * (P.V / P.dx);
                        const double dwij = rij_ * k_dw(r, P.Bg, P.RG);
                        const double dwji = rji_ * k_dw(r, P.Bg, P.RG);
                        double gr = 0.0;
                        for (int d = 0; d < 3; d++) gr += (aj * gj[d] * dwji - ai * gi[d] * dwij) * q[d];
                        for (int d = 0; d < 3; d++) fI[d] -= (gr) * (q[d] / r) / P.R2g * P.RG * (P.V / P.dx);
                    }
                }
                // viscosity (solid i skips wall j)
                if (!(sol && is_wall(tj)) && r2 < P.RV2) {
                    const double r = sqrt(r2);
                    const double dwij = -k_dw(r, P.Bv, P.RV);
                    const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                    const double muj = P.svisc[tj];
                    const double muij = 2.0 * (mui * muj) / (mui + muj);
                    const double dot = (u[0] * e[0] + u[1] * e[1] + u[2] * e[2]);
                    for (int d = 0; d < 3; d++) fV[d] += P.viscC * muij * dot * e[d] * dwij / r * P.V;
                }
                // drag and buoyancy on solids from fluid neighbours
                if (sol && r2 < P.RP2 && is_fluid(tj)) {
                    const double Vs = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                    const double Re = alpha * rhoi * Vs * P.dx / (P.svisc[tj]);
                    double cd;
                    if (alpha < 0.8)
                        cd = (4.0 / 3.0) * (150.0 * (1.0 - alpha) / (alpha * Re) + 1.75);
                    else if (Re <= 1000.0 && alpha >= 0.8)
                        cd = 24.0 * (1.0 + 0.15 * pow(Re, 0.687)) / (alpha * Re) * pow(alpha, -2.65);
                    else
                        cd = 0.44;
                    dragc = cd;
                    have_drag = true;
                    for (int d = 0; d < 3; d++) fD[d] += 0.5 * cd * rhoi * P.dx * P.dx * P.dx * u[d] * Vs;
                    const double w = k_w(sqrt(r2), P.Bp, P.RP);
                    const double rhoj = P.density[tj];
                    for (int d = 0; d < 3; d++) fB[d] += rhoj * P.V * P.g[d] * w;
                }
            });
        if (!active) return;
        double F[3] = {0.0, 0.0, 0.0};
        const double m = sol ? rhoi * P.V : P.mass[ti];
        if (sol) {
            for (int d = 0; d < 3; d++) F[d] += fD[d];
            if (st)
                for (int d = 0; d < 3; d++) F[d] += fA[d];
            if (st)
                for (int d = 0; d < 3; d++) F[d] += fI[d];
            for (int d = 0; d < 3; d++) F[d] += fV[d];
            for (int d = 0; d < 3; d++) F[d] += fD[d];
            for (int d = 0; d < 3; d++) F[d] -= fB[d];
            for (int d = 0; d < 3; d++) F[d] += m * P.g[d];
            S.alpha[i] = alpha;
            if (have_drag) S.dragC[i] = dragc;
        } else {
            for (int d = 0; d < 3; d++) F[d] += fP[d];
            if (st)
                for (int d = 0; d < 3; d++) F[d] += fA[d];
            if (st)
                for (int d = 0; d < 3; d++) F[d] += fI[d];
            for (int d = 0; d < 3; d++) F[d] += fV[d];
            for (int d = 0; d < 3; d++) F[d] += m * P.g[d];
        }
        for (int d = 0; d < 3; d++) S.frc[d * N + i] = F[d];
    };
    if (LIST) {
        // one thread per slot: nothing in the list walk is warp-synchronous
        const int end = dB[B_SE];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) body(i, true, 0, i);
    } else {
        FOR_EACH_CHUNK(dB, range, kWarpsPerBlock, cidx)
        {
            const Chunk ch = S.chunks[cidx];
            const int i = ch.i0 + lane;
            const bool active = lane < ch.cnt;
            body(i, active, (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T), active ? i : ch.i0);
        }
    }
}

// ------------------------------------------------------------------ DEM
// One substep of the DEM loop :536-550 for solid particles (and, with
// DMPH_FLAG_WALL_DEM_COEFFS, the output-only constants of wall particles):
// calculateNormalDirectionCoefficient :2298 and
// calculateTangentialDirectionCoefficient :2346 take the constants of the
// LAST neighbour within dx (the highest sorted index, since candidates come in
// ascending order) and keep the old values when there is none;
// calculateNormalDirectionForce :2560 and calculateTangentialDirectionForce
// :2614 add their sums to Force in that order.  calculateInertialTensor and
// calculateTorque only feed arrays nothing reads and are not run.
// MIXED: FP32 split mode, where solids and walls keep FP64 master positions in
// S.pos/S.vel but fluid particles live in the FP32 arrays p4/v4.
// LIST (FP64 build): each lane walks its particle's Verlet list, which is the
// reference's own NeighborInd (the neighbours within MaxRadius+MARGIN at the
// last rebuild, fluid then solid then wall cells in its visiting order), as
// the reference's DEM functions do; the stencil walk visits the same
// candidates in the same order, so both give the same bits.  gate: this
// stencil launch stands in only after a list overflow.

// the contact of one pair within dx (calculateNormalDirectionForce
// :2560-2612 and calculateTangentialDirectionForce :2614-2696, with the
// reference's stray Dt on the normal damping and its component-wise v_n)
__device__ __forceinline__ void dem_pair(const DevParams &P, double kn, double cn, double kt, double ct, double mu_f,
                                         const double q[3], double r2, double vxj, double vyj, double vzj,
                                         double vxi, double vyi, double vzi, double fN[3], double fT[3])
{
    const double r = sqrt(r2);
    const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
    const double u[3] = {vxj - vxi, vyj - vyi, vzj - vzi};
    double vn[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < 3; d++) vn[d] += u[d] * e[d];
    for (int d = 0; d < 3; d++) fN[d] += -kn * (P.dx - r) * e[d] - (cn * vn[d] * e[d] * P.dt);
    double vn2[3], vt[3], dtv[3] = {0.0, 0.0, 0.0}, sN[3], sT[3];
    for (int d = 0; d < 3; d++) vn2[d] = u[d] * e[d];
    for (int d = 0; d < 3; d++) vt[d] = u[d] - vn2[d] * e[d];
    for (int d = 0; d < 3; d++) dtv[d] += vt[d] * P.ddt;
    for (int d = 0; d < 3; d++) sN[d] = -kn * (P.dx - r) * e[d] - (cn * vn2[d] * e[d] * P.dt);
    const double aFn = mu_f * sqrt(sN[0] * sN[0] + sN[1] * sN[1] + sN[2] * sN[2]);
    for (int d = 0; d < 3; d++) sT[d] = -kt * dtv[d] - (ct * vt[d]);
    const double aFt = sqrt(sT[0] * sT[0] + sT[1] * sT[1] + sT[2] * sT[2]);
    if (aFn > aFt) {
        for (int d = 0; d < 3; d++) fT[d] += -kt * dtv[d] - (ct * vt[d]);
    } else {
        const double avt = sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
        if (avt != 0)
            for (int d = 0; d < 3; d++) fT[d] += aFn * vt[d] / avt;
    }
}

template <bool MIXED, bool LIST>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_dem_force(DevParams P, DevState S, const int *dB, int range,
                                                                      int forces, int gate)
{
    if (LIST ? dB[B_LIST_OVF] != 0 : (gate && dB[B_LIST_OVF] == 0)) return;
    __shared__ TileA tiles[kWarpsPerBlock];
    TileA &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    FOR_EACH_CHUNK(dB, range, kWarpsPerBlock, cidx)
    {
        const Chunk ch = S.chunks[cidx];
        const int i = ch.i0 + lane;
        const bool active = lane < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        const int ii = active ? i : ch.i0;
        const int ti = S.type[ii];
        const double xi = S.pos[ii], yi = S.pos[N + ii], zi = S.pos[2 * N + ii];
        const double vxi = S.vel[ii], vyi = S.vel[N + ii], vzi = S.vel[2 * N + ii];
        const int nlist = (LIST && active) ? S.nbn[i] : 0;
        auto stage = [&](int j, int slot) {
            const int t = S.type[j];
            if (MIXED && is_fluid(t)) {
                const float4 p = S.p4[j];
                const float4 v = S.v4[j];
                const unsigned w = __float_as_uint(p.w);
                tl.x[slot] = P.dmin[0] + unpack_cx(w) * P.cw[0] + (double)p.x;
                tl.y[slot] = P.dmin[1] + unpack_cy(w) * P.cw[1] + (double)p.y;
                tl.z[slot] = P.dmin[2] + unpack_cz(w) * P.cw[2] + (double)p.z;
                tl.vx[slot] = v.x;
                tl.vy[slot] = v.y;
                tl.vz[slot] = v.z;
            } else {
                tl.x[slot] = S.pos[j];
                tl.y[slot] = S.pos[N + j];
                tl.z[slot] = S.pos[2 * N + j];
                tl.vx[slot] = S.vel[j];
                tl.vy[slot] = S.vel[N + j];
                tl.vz[slot] = S.vel[2 * N + j];
            }
            tl.t[slot] = t;
        };
        // 1) last neighbour within dx
        int tlast = -1;
        double r2last = 0.0;
        if (LIST) {
            for (int k = 0; k < nlist; ++k) {
                const int j = (int)(__ldg(S.nbl + list_index(k, i, N)) & kEntrySlot);
                if (j == i) continue;
                const double q0 = rel1(S.pos[j], xi, P.W[0], P.hW[0]);
                const double q1 = rel1(S.pos[N + j], yi, P.W[1], P.hW[1]);
                const double q2 = rel1(S.pos[2 * N + j], zi, P.W[2], P.hW[2]);
                const double r2 = (q0 * q0 + q1 * q1 + q2 * q2);
                if (r2 <= P.dx2) {
                    tlast = S.type[j];
                    r2last = r2;
                }
            }
        } else {
            traverse_stencil(P, S.cell_start, key_cell, lane, active, 7u, stage, [&](int j, int s) {
                if (j == i) return;
                const double q0 = rel1(tl.x[s], xi, P.W[0], P.hW[0]);
                const double q1 = rel1(tl.y[s], yi, P.W[1], P.hW[1]);
                const double q2 = rel1(tl.z[s], zi, P.W[2], P.hW[2]);
                const double r2 = (q0 * q0 + q1 * q1 + q2 * q2);
                if (r2 <= P.dx2) {
                    tlast = tl.t[s];
                    r2last = r2;
                }
            });
        }
        double kn, cn, kt, ct;
        if (active) {
            if (tlast >= 0) {
                const double r = sqrt(r2last);
                const double ov = fmax(0.0, P.dx - r);
                kn = (4.0 / 3.0) * P.Eeff[ti][tlast] * sqrt(P.Reff * ov);
                const double mi = P.mass[ti], mj = P.mass[tlast];
                const double mij = mi * mj / (mi + mj);
                cn = -2.0 * sqrt(mij * kn) * P.logE[ti] / P.cnDen[ti];
                kt = P.KtFac[ti][tlast] * sqrt(P.Reff * sqrt(ov));
                ct = P.ctFac[ti] * sqrt(mij * kt);
                S.kn[i] = kn;
                S.cn[i] = cn;
                S.kt[i] = kt;
                S.ct[i] = ct;
            } else {
                kn = S.kn[i];
                cn = S.cn[i];
                kt = S.kt[i];
                ct = S.ct[i];
            }
        }
        if (!forces) continue;  // warp-uniform
        // 2) normal and tangential forces from non-fluid neighbours within dx
        double fN[3] = {0.0, 0.0, 0.0}, fT[3] = {0.0, 0.0, 0.0};
        const double mu_f = P.friction[ti];
        if (LIST) {
            for (int k = 0; k < nlist; ++k) {
                const int j = (int)(__ldg(S.nbl + list_index(k, i, N)) & kEntrySlot);
                if (j == i || is_fluid(S.type[j])) continue;
                const double q[3] = {rel1(S.pos[j], xi, P.W[0], P.hW[0]), rel1(S.pos[N + j], yi, P.W[1], P.hW[1]),
                                     rel1(S.pos[2 * N + j], zi, P.W[2], P.hW[2])};
                const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                if (r2 <= P.dx2)
                    dem_pair(P, kn, cn, kt, ct, mu_f, q, r2, S.vel[j], S.vel[N + j], S.vel[2 * N + j], vxi, vyi, vzi,
                             fN, fT);
            }
        } else {
            traverse_stencil(P, S.cell_start, key_cell, lane, active, 6u, stage, [&](int j, int s) {
                if (j == i) return;
                const double q[3] = {rel1(tl.x[s], xi, P.W[0], P.hW[0]), rel1(tl.y[s], yi, P.W[1], P.hW[1]),
                                     rel1(tl.z[s], zi, P.W[2], P.hW[2])};
                const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                if (r2 <= P.dx2)
                    dem_pair(P, kn, cn, kt, ct, mu_f, q, r2, tl.vx[s], tl.vy[s], tl.vz[s], vxi, vyi, vzi, fN, fT);
            });
        }
        if (!active) continue;
        for (int d = 0; d < 3; d++) {
            double F = S.frc[d * N + i];
            F += fN[d];
            F += fT[d];
            S.frc[d * N + i] = F;
        }
    }
}

// calculateAcceleration :2832-2843 over the fluid slots [b, e).  A kernel of
// its own: pass B reads the velocities of neighbouring particles, so they may
// only change once every force of the step is known.
__global__ void k_fluid_accel(DevParams P, DevState S, const int *dB)
{
    const int N = P.N;
    FOR_EACH_SLOT(dB, -1, B_FE, i)
    {
        const double m = P.mass[S.type[i]];
        for (int d = 0; d < 3; d++) S.vel[d * N + i] += S.frc[d * N + i] / m * P.dt;
    }
}

// calculateDEMconvection :1872-1891 over the solid slots [b, e)
__global__ void k_dem_integrate(DevParams P, DevState S, const int *dB)
{
    const int N = P.N;
    FOR_EACH_SLOT(dB, B_SB, B_SE, i)
    {
        const double m = P.mass[S.type[i]];
        for (int d = 0; d < 3; d++) {
            double v = S.vel[d * N + i];
            v += S.frc[d * N + i] / m * P.ddt;
            S.vel[d * N + i] = v;
            S.pos[d * N + i] += v * P.ddt;
        }
    }
}

// ------------------------------------------------------------------ rebuild
// NeighborCount / SolidNeighborCount of calculateNeighbor :1546-1678 (counts
// of particles within MaxRadius+MARGIN at rebuild time, self included; the
// rebuild-time positions are kept in xref).
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_counts(DevParams P, DevState S, const int *dB, int range,
                                                                   int gate)
{
    // gate: the FP32 lists count the debris (k_counts_list), this walk stands
    // in after a list overflow
    if (gate && dB[B_LIST_OVF] == 0) return;
    __shared__ TileA tiles[kWarpsPerBlock];
    TileA &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    FOR_EACH_CHUNK(dB, range, kWarpsPerBlock, cidx)
    {
        const Chunk ch = S.chunks[cidx];
        const int i = ch.i0 + lane;
        const bool active = lane < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        const int ii = active ? i : ch.i0;
        const double xi = S.xref[ii], yi = S.xref[N + ii], zi = S.xref[2 * N + ii];
        int cnt = 0, scnt = 0;
        traverse_stencil(
            P, S.cell_start, key_cell, lane, active, 7u,
            [&](int j, int slot) {
                tl.x[slot] = S.xref[j];
                tl.y[slot] = S.xref[N + j];
                tl.z[slot] = S.xref[2 * N + j];
                tl.t[slot] = S.type[j];
            },
            [&](int j, int s) {
                const double q0 = rel1(tl.x[s], xi, P.W[0], P.hW[0]);
                const double q1 = rel1(tl.y[s], yi, P.W[1], P.hW[1]);
                const double q2 = rel1(tl.z[s], zi, P.W[2], P.hW[2]);
                const double r2 = q0 * q0 + q1 * q1 + q2 * q2;
                if (r2 <= P.rc2) {
                    cnt++;
                    if (is_solid(tl.t[s])) scnt++;
                }
            });
        if (!active) continue;
        S.nc[i] = cnt;
        S.snc[i] = scnt;
    }
}

// FP32 list mode: NeighborCount and SolidNeighborCount of the debris slots
// from their Verlet lists, which hold every particle within rc of them (and
// a thin shell past it); the reference's FP64 distance test on the
// rebuild-time positions decides, as in k_counts, and i itself counts as
// in the reference's list.  One warp per debris particle.
// need_gate: run only on a step whose B_NEED is that value (list reuse: a
// trigger that keeps the lists); 0: always (inside a rebuild)
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_counts_list(DevParams P, DevState S, const int *dB,
                                                                      int need_gate)
{
    if (dB[B_LIST_OVF]) return;
    if (need_gate && dB[B_NEED] != need_gate) return;
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    const long long ld = N;
    const int sb = dB[B_SB], se = dB[B_SE];
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int i = sb + blockIdx.x * (blockDim.x >> 5) + (int)(threadIdx.x >> 5); i < se; i += nwarps) {
        const int n = S.nbn[i];
        const double xi = S.xref[i], yi = S.xref[N + i], zi = S.xref[2 * N + i];
        int cnt = 0, scnt = 0;
        for (int k = lane; k < n; k += kWarp) {
            const int j = (int)(__ldg(S.nbl + list_index(k, i, ld)) & kEntrySlot);
            const double q0 = rel1(S.xref[j], xi, P.W[0], P.hW[0]);
            const double q1 = rel1(S.xref[N + j], yi, P.W[1], P.hW[1]);
            const double q2 = rel1(S.xref[2 * N + j], zi, P.W[2], P.hW[2]);
            const double r2 = q0 * q0 + q1 * q1 + q2 * q2;
            if (r2 <= P.rc2) {
                cnt++;
                if (is_solid(S.type[j])) scnt++;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(kFull, cnt, o);
            scnt += __shfl_xor_sync(kFull, scnt, o);
        }
        if (lane == 0) {
            S.nc[i] = cnt + 1;  // i itself
            S.snc[i] = scnt + 1;
        }
    }
}

// Fill pass of the CSR neighbour list (calculateNeighbor :1725-1840); ptr
// holds the exclusive scan of NeighborCount.
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_neighbor_fill(DevParams P, DevState S, const int *dB, int range, const long long *ptr,
                                                                          int *ind)
{
    __shared__ TileA tiles[kWarpsPerBlock];
    TileA &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    FOR_EACH_CHUNK(dB, range, kWarpsPerBlock, cidx)
    {
        const Chunk ch = S.chunks[cidx];
        const int i = ch.i0 + lane;
        const bool active = lane < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        const int ii = active ? i : ch.i0;
        const double xi = S.xref[ii], yi = S.xref[N + ii], zi = S.xref[2 * N + ii];
        long long w = active ? ptr[i] : 0;
        const long long wend = active ? ptr[i + 1] : 0;
        traverse_stencil(
            P, S.cell_start, key_cell, lane, active, 7u,
            [&](int j, int slot) {
                tl.x[slot] = S.xref[j];
                tl.y[slot] = S.xref[N + j];
                tl.z[slot] = S.xref[2 * N + j];
            },
            [&](int j, int s) {
                const double q0 = rel1(tl.x[s], xi, P.W[0], P.hW[0]);
                const double q1 = rel1(tl.y[s], yi, P.W[1], P.hW[1]);
                const double q2 = rel1(tl.z[s], zi, P.W[2], P.hW[2]);
                const double r2 = q0 * q0 + q1 * q1 + q2 * q2;
                if (r2 <= P.rc2 && w < wend) ind[w++] = j;
            });
    }
}

// launch helpers (host side of this translation unit)
void launch_drift(const DevParams &P, const DevState &S, const WallMotion &Wm, unsigned long long *maxshift,
                  int sms, cudaStream_t st)
{
    const int threads = 256;
    int blocks = (P.N + threads - 1) / threads;
    const int cap = sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_drift<<<blocks, threads, 0, st>>>(P, S, Wm, maxshift);
}

constexpr int kBlock = kWarpsPerBlock * kWarp;
constexpr int kElemGrid = 148 * 4;

// Verlet lists of the FP64 build: exactly the reference's NeighborInd
// (calculateNeighbor :1521-1851): every j, i itself included, with
// |x_j - x_i|^2 <= (MaxRadius + MARGIN)^2 at the rebuild-time positions, in
// ascending slot order; blocked layout as in the FP32 build, entry = j
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp) k_build_list64(DevParams P, DevState S, int *dB)
{
    __shared__ TileA tiles[kWarpsPerBlock];
    TileA &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    const int cap = S.nbl_cap;
    FOR_EACH_CHUNK(dB, CR_ALL, kWarpsPerBlock, cidx)
    {
        const Chunk ch = S.chunks[cidx];
        const int i = ch.i0 + lane;
        const bool active = lane < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        const int ii = active ? i : ch.i0;
        const double xi = S.xref[ii], yi = S.xref[N + ii], zi = S.xref[2 * N + ii];
        int cnt = 0;
        traverse_stencil(
            P, S.cell_start, key_cell, lane, active, 7u,
            [&](int j, int slot) {
                tl.x[slot] = S.xref[j];
                tl.y[slot] = S.xref[N + j];
                tl.z[slot] = S.xref[2 * N + j];
            },
            [&](int j, int s) {
                const double q0 = rel1(tl.x[s], xi, P.W[0], P.hW[0]);
                const double q1 = rel1(tl.y[s], yi, P.W[1], P.hW[1]);
                const double q2 = rel1(tl.z[s], zi, P.W[2], P.hW[2]);
                const double r2 = q0 * q0 + q1 * q1 + q2 * q2;
                if (r2 <= P.rc2) {
                    if (cnt < cap) S.nbl[list_index(cnt, i, N)] = (unsigned)j;
                    ++cnt;
                }
            });
        if (!active) continue;
        if (cnt > cap) atomicExch(dB + B_LIST_OVF, 1);
        S.nbn[i] = cnt < cap ? cnt : cap;
    }
}

void launch_build_list64(const DevParams &P, const DevState &S, int *dB, cudaStream_t st)
{
    cudaMemsetAsync(dB + B_LIST_OVF, 0, sizeof(int), st);
    static const int g = persistent_grid((const void *)k_build_list64, kBlock);
    k_build_list64<<<g, kBlock, 0, st>>>(P, S, dB);
}

void launch_pass_a(const DevParams &P, const DevState &S, const int *dB, int range, int init_only, cudaStream_t st,
                   int list, int gate)
{
    if (list) {
        static const int g = persistent_grid((const void *)k_pass_a<true>, kBlock);
        k_pass_a<true><<<g, kBlock, 0, st>>>(P, S, dB, range, init_only, 0);
    } else {
        static const int g = persistent_grid((const void *)k_pass_a<false>, kBlock);
        k_pass_a<false><<<g, kBlock, 0, st>>>(P, S, dB, range, init_only, gate);
    }
}
// Virial stress and pressure of the output cadence
// (calculateVirialStressAtParticle, source/DEM-MPH.cpp:2904-3149): the
// reference runs four passes over the neighbour list (pressure P, attractive
// pressure A, viscosity V, diffuse interface G) and adds each pass's
// per-particle stress matrix in turn.  The four matrices are accumulated here
// in one traversal, pair by pair in list order, and added in the same order,
// so the result is the reference's to the last bit.  Reads the FP64 planes:
// pos, vel, pres, pA, gc (FP32 builds widen into them first).
__global__ void __launch_bounds__(kBlock) k_virial(DevParams P, DevState S, const int *dB, double *vir)
{
    __shared__ TileA tiles[kWarpsPerBlock];
    TileA &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int N = P.N;
    const double C = P.dim == 2 ? 8.0 : 10.0;
    FOR_EACH_CHUNK(dB, CR_ALL, kWarpsPerBlock, cidx)
    {
        const Chunk ch = S.chunks[cidx];
        const int i = ch.i0 + lane;
        const bool active = lane < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        const int ii = active ? i : ch.i0;
        const int ti = S.type[ii];
        const double xi = S.pos[ii], yi = S.pos[N + ii], zi = S.pos[2 * N + ii];
        const double vxi = S.vel[ii], vyi = S.vel[N + ii], vzi = S.vel[2 * N + ii];
        const double Pi = S.pres[ii], PAi = S.pA[ii];
        const double gci[3] = {S.gc[ii], S.gc[N + ii], S.gc[2 * N + ii]};
        const double mui = P.svisc[ti];
        const double a = P.CofA[ti] * (P.CofK) * (P.CofK);
        double sP[3][3] = {{0.0}}, sA[3][3] = {{0.0}}, sV[3][3] = {{0.0}}, sG[3][3] = {{0.0}};
        traverse_stencil(
            P, S.cell_start, key_cell, lane, active, 7u,
            [&](int j, int slot) {
                tl.x[slot] = S.pos[j];
                tl.y[slot] = S.pos[N + j];
                tl.z[slot] = S.pos[2 * N + j];
                tl.vx[slot] = S.vel[j];
                tl.vy[slot] = S.vel[N + j];
                tl.vz[slot] = S.vel[2 * N + j];
                tl.t[slot] = S.type[j];
            },
            [&](int j, int s) {
                if (j == i) return;
                const double q[3] = {rel1(tl.x[s], xi, P.W[0], P.hW[0]), rel1(tl.y[s], yi, P.W[1], P.hW[1]),
                                     rel1(tl.z[s], zi, P.W[2], P.hW[2])};
                const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                const int tj = tl.t[s];
                if (P.RP * P.RP - r2 > 0) {
                    const double r = sqrt(r2);
                    const double dw = k_dw(r, P.Bp, P.RP);
                    const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                    double f[3];
                    for (int d = 0; d < 3; d++) f[d] = (Pi)*g[d] * P.V;
                    for (int d = 0; d < 3; d++)
                        for (int e = 0; e < 3; e++) sP[d][e] += 1.0 * f[d] * q[e] / P.V;
                }
                if (P.RA * P.RA - r2 > 0) {
                    const double ratio = P.ratio[ti][tj];
                    const double r = sqrt(r2);
                    const double dw = ratio * k_dwa(r, P.Ba, P.RA);
                    const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                    double f[3];
                    for (int d = 0; d < 3; d++) f[d] = (PAi)*g[d] * P.V;
                    for (int d = 0; d < 3; d++)
                        for (int e = 0; e < 3; e++) sA[d][e] += 1.0 * f[d] * q[e] / P.V;
                }
                if (P.RV * P.RV - r2 > 0) {
                    const double r = sqrt(r2);
                    const double dw = -k_dw(r, P.Bv, P.RV);
                    const double e_[3] = {q[0] / r, q[1] / r, q[2] / r};
                    const double u[3] = {tl.vx[s] - vxi, tl.vy[s] - vyi, tl.vz[s] - vzi};
                    const double muj = P.svisc[tj];
                    const double muij = 2.0 * (mui * muj) / (mui + muj);
                    double f[3];
                    for (int d = 0; d < 3; d++)
                        f[d] = C * muij * (u[0] * e_[0] + u[1] * e_[1] + u[2] * e_[2]) * e_[d] * dw / r * P.V;
                    for (int d = 0; d < 3; d++)
                        for (int e = 0; e < 3; e++) sV[d][e] += 0.5 * f[d] * q[e] / P.V;
                }
                if (P.RG * P.RG - r2 > 0) {
                    const double ratio = P.ratio[ti][tj];
                    const double r = sqrt(r2);
                    const double w = ratio * k_w(r, P.Bg, P.RG);
                    double f[3];
                    for (int d = 0; d < 3; d++) f[d] = -a * (-gci[d]) * w / P.R2g * P.RG * (P.V / P.dx);
                    for (int d = 0; d < 3; d++)
                        for (int e = 0; e < 3; e++) sG[d][e] += 1.0 * f[d] * q[e] / P.V;
                    const double dw = ratio * k_dw(r, P.Bg, P.RG);
                    const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                    double gr = 0.0;
                    for (int d = 0; d < 3; d++) gr += (-gci[d]) * q[d];
                    for (int d = 0; d < 3; d++) f[d] = -a * (gr)*g[d] / P.R2g * P.RG * (P.V / P.dx);
                    for (int d = 0; d < 3; d++)
                        for (int e = 0; e < 3; e++) sG[d][e] += 1.0 * f[d] * q[e] / P.V;
                }
            });
        if (!active) continue;
        double vs[3][3];
        for (int d = 0; d < 3; d++)
            for (int e = 0; e < 3; e++) vs[d][e] = (((0.0 + sP[d][e]) + sA[d][e]) + sV[d][e]) + sG[d][e];
        vir[i] = P.dim == 2 ? -1.0 / 2.0 * (vs[0][0] + vs[1][1]) : -1.0 / 3.0 * (vs[0][0] + vs[1][1] + vs[2][2]);
    }
}

void launch_virial(const DevParams &P, const DevState &S, const int *dB, double *vir, cudaStream_t st)
{
    static const int g = persistent_grid((const void *)k_virial, kBlock);
    k_virial<<<g, kBlock, 0, st>>>(P, S, dB, vir);
}

void launch_pass_b(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st, int list, int gate)
{
    if (list) {
        static const int g = persistent_grid((const void *)k_pass_b<true>, kBlock);
        k_pass_b<true><<<g, kBlock, 0, st>>>(P, S, dB, CR_FLUID_SOLID, 0);
    } else {
        static const int g = persistent_grid((const void *)k_pass_b<false>, kBlock);
        k_pass_b<false><<<g, kBlock, 0, st>>>(P, S, dB, CR_FLUID_SOLID, gate);
    }
}
void launch_dem_force(const DevParams &P, const DevState &S, const int *dB, int range, int forces, cudaStream_t st,
                      bool mixed, bool list)
{
    if (mixed) {
        static const int g = persistent_grid((const void *)k_dem_force<true, false>, kBlock);
        k_dem_force<true, false><<<g, kBlock, 0, st>>>(P, S, dB, range, forces, 0);
        return;
    }
    if (list) {
        static const int gl = persistent_grid((const void *)k_dem_force<false, true>, kBlock);
        k_dem_force<false, true><<<gl, kBlock, 0, st>>>(P, S, dB, range, forces, 0);
    }
    static const int g = persistent_grid((const void *)k_dem_force<false, false>, kBlock);
    k_dem_force<false, false><<<g, kBlock, 0, st>>>(P, S, dB, range, forces, list ? 1 : 0);
}
void launch_fluid_accel(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st)
{
    k_fluid_accel<<<kElemGrid, 256, 0, st>>>(P, S, dB);
}
void launch_dem_integrate(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st)
{
    k_dem_integrate<<<kElemGrid / 4, 256, 0, st>>>(P, S, dB);
}
void launch_counts(const DevParams &P, const DevState &S, const int *dB, int range, cudaStream_t st)
{
    static const int g = persistent_grid((const void *)k_counts, kBlock);
    k_counts<<<g, kBlock, 0, st>>>(P, S, dB, range, 0);
}

void launch_counts_list(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st)
{
    static const int gl = persistent_grid((const void *)k_counts_list, kBlock);
    k_counts_list<<<gl, kBlock, 0, st>>>(P, S, dB, 0);
    static const int g = persistent_grid((const void *)k_counts, kBlock);
    k_counts<<<g, kBlock, 0, st>>>(P, S, dB, CR_SOLID, 1);
}
void launch_counts_list_kept(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st)
{
    static const int gl = persistent_grid((const void *)k_counts_list, kBlock);
    k_counts_list<<<gl, kBlock, 0, st>>>(P, S, dB, 2);
}
void launch_neighbor_fill(const DevParams &P, const DevState &S, const int *dB, const long long *ptr, int *ind,
                          cudaStream_t st)
{
    static const int g = persistent_grid((const void *)k_neighbor_fill, kBlock);
    k_neighbor_fill<<<g, kBlock, 0, st>>>(P, S, dB, CR_ALL, ptr, ind);
}

}  // namespace dmph
