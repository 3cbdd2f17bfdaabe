// Rigid debris clumps (DMPH_FLAG_RIGID_CLUMPS).  No counterpart in the
// reference: there, debris particles move individually (calculateDEMconvection,
// source/DEM-MPH.cpp:1872-1891) and the torque/inertia code
// (:2402-2557) feeds nothing.  Here each debris body is rigid:
//
//   1. k_clump_dem: for every body particle, the spring-dashpot contact force
//      from particles of OTHER bodies, free debris and walls within dx.  The
//      pair constants follow the reference's Hertz-type formulas (effective
//      modulus, overlap, restitution damping; :2318-2338, :2374-2396) but are
//      evaluated per pair with pair-symmetric restitution and friction, the
//      normal damping is the projection c_n (u.e) e, and the tangential force
//      opposes sliding and is capped by Coulomb friction.  The force acts at
//      the contact midpoint, so the offset torque 0.5 q x F is kept too; pair
//      forces are antisymmetric and total linear and angular momentum of
//      colliding bodies are conserved.
//   2. k_body_step: one block per body reduces, in FP64 (warp shuffles, then
//      across the block's warps in a fixed order), the total force
//      F = sum(fluid + contact) and torque
//      T = sum(R r0 x f + contact offset torques) over its members (gathered
//      through slot_of_row, so the reduction order is the body's fixed member
//      order, independent of the cell sort), then advances the body in FP64:
//      V += F/M dt, X += V dt, L += T dt, q <- exp(w dt / 2) q with
//      w = R I0^-1 R^T L, and places every member at X + R r0 with velocity
//      V + w x (R r0).
#include "dmph_internal.h"
#include "dmph_traverse.cuh"

namespace dmph {

__global__ void k_slot_of_row(int N, const int *__restrict__ pidx, int *__restrict__ slot_of_row)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) slot_of_row[pidx[i]] = i;
}

// Contact of debris particle i (position xi, velocity vi, type ti, body bi,
// mass mi) with candidate j: skipped when j is i, of the same body, or not
// within dx; otherwise the pair force and the offset torque are added to F, T.
__device__ __forceinline__ void clump_pair(const DevParams &P, const DevState &S, int i, const double *xi,
                                           const double *vi, int ti, int bi, double mi, int j, double *F, double *T)
{
    const int N = P.N;
    if (j == i) return;
    const int bj = S.bid[j];
    if (bi >= 0 && bj == bi) return;
    double q[3];
    for (int k = 0; k < 3; k++) {
        q[k] = S.pos[k * N + j] - xi[k];
        q[k] -= P.W[k] * rint(q[k] / P.W[k]);
    }
    const double r2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    if (r2 > P.dx2 || r2 <= 0.0) return;
    const int tj = S.type[j];
    const double r = sqrt(r2);
    const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
    const double ov = P.dx - r;
    const double u[3] = {S.vel[j] - vi[0], S.vel[N + j] - vi[1], S.vel[2 * N + j] - vi[2]};
    const double un = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];
    const double mj = (bj >= 0 ? S.body_rho[bj] : P.density[tj]) * P.V;
    const double mij = mi * mj / (mi + mj);
    const double kn = (4.0 / 3.0) * P.Eeff[ti][tj] * sqrt(P.Reff * ov);
    const double cn = sqrt(mij * kn) * P.pairDamp[ti][tj];
    const double kt = P.KtFac[ti][tj] * sqrt(P.Reff * sqrt(ov));
    const double ct = sqrt(mij * kt) * P.pairDamp[ti][tj];
    double f[3], ut[3];
    const double fnm = fmin(-kn * ov + cn * un, 0.0);  // no adhesion
    for (int k = 0; k < 3; k++) {
        f[k] = fnm * e[k];
        ut[k] = u[k] - un * e[k];
    }
    const double ctot = ct + kt * P.ddt;
    const double aut = sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
    const double cap = P.pairFric[ti][tj] * fabs(fnm);
    const double ft = ctot * aut > cap && aut > 0.0 ? cap / aut : ctot;
    for (int k = 0; k < 3; k++) f[k] += ft * ut[k];
    for (int k = 0; k < 3; k++) F[k] += f[k];
    // offset of the contact midpoint from the particle centre: 0.5 q
    T[0] += 0.5 * (q[1] * f[2] - q[2] * f[1]);
    T[1] += 0.5 * (q[2] * f[0] - q[0] * f[2]);
    T[2] += 0.5 * (q[0] * f[1] - q[1] * f[0]);
}

__device__ __forceinline__ void clump_store(const DevParams &P, const DevState &S, int i, int lane, double *F,
                                            double *T)
{
    const int N = P.N;
    for (int k = 0; k < 3; k++) {
        F[k] = warp_sum(F[k]);
        T[k] = warp_sum(T[k]);
    }
    if (lane == 0)
        for (int k = 0; k < 3; k++) {
            S.frc_dem[k * N + i] = F[k];
            S.frc_dem[(3 + k) * N + i] = T[k];
        }
}

// One warp per debris particle i (slots [sb, se) walked by a persistent
// grid); the lanes stride over the candidates of the neighbour cells that
// can hold a contact partner: contacts need |x_j - x_i| <= dx, so only the
// neighbour cells within 1.6 dx of i's rebuild-time position (about 8 of the
// 27) are visited, for the solid and wall classes.  FP64 on the master
// planes; per-lane partial sums are combined with warp shuffles.  One warp
// per debris particle i (lane = its lane).
__device__ __forceinline__ void clump_dem_stencil_particle(const DevParams &P, const DevState &S, int i, int lane)
{
    const int N = P.N;
    const double xi[3] = {S.pos[i], S.pos[N + i], S.pos[2 * N + i]};
    const double vi[3] = {S.vel[i], S.vel[N + i], S.vel[2 * N + i]};
    const int ti = S.type[i];
    const int bi = S.bid[i];
    const double mi = particle_density(S, P, i, ti) * P.V;
    // rebuild-time cell and the neighbour cells within reach
    const int key_cell = (int)(word_key(S.skey[i]) % (unsigned)P.T);
    int c[3];
    if (P.dim == 2) {
        c[0] = key_cell / P.cc[1];
        c[1] = key_cell % P.cc[1];
        c[2] = 0;
    } else {
        c[0] = key_cell / (P.cc[1] * P.cc[2]);
        c[1] = (key_cell / P.cc[2]) % P.cc[1];
        c[2] = key_cell % P.cc[2];
    }
    // contact partners are within dx now; positions drift at most 0.05 dx
    // from their rebuild-time values between rebuild checks, and up to
    // about 0.25 dx inside one surrogate block: 1.6 dx covers both
    const double reach = 1.6 * P.dx;
    int lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        const double loc = S.xref[k * N + i] - (P.dmin[k] + c[k] * P.cw[k]);
        const bool flat = (k == 2 && P.dim == 2);
        lo[k] = flat ? 0 : (loc < reach ? -1 : 0);
        hi[k] = flat ? 0 : (P.cw[k] - loc < reach ? 1 : 0);
    }
    double F[3] = {0.0, 0.0, 0.0}, T[3] = {0.0, 0.0, 0.0};
    // the (cell, class) ranges to visit, fetched by 16 lanes at once:
    // lane r < 16 holds range r = (cell index r / 2 of the <= 8 cells,
    // class 1 + r % 2)
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    const int nranges = 2 * nx * ny * nz;
    int rb = 0, re = 0;
    if (lane < nranges) {
        const int c_ = lane >> 1, cls = 1 + (lane & 1);
        const int oz = lo[2] + c_ % nz, oy = lo[1] + (c_ / nz) % ny, ox = lo[0] + c_ / (nz * ny);
        const int off = cls * P.T + cell_id(P, c[0] + ox, c[1] + oy, c[2] + oz);
        rb = __ldg(S.cell_start + off);
        re = __ldg(S.cell_start + off + 1);
    }
    for (int r = 0; r < nranges; ++r) {
        const int jb = __shfl_sync(kFull, rb, r), je = __shfl_sync(kFull, re, r);
        for (int j = jb + lane; j < je; j += kWarp) clump_pair(P, S, i, xi, vi, ti, bi, mi, j, F, T);
    }
    clump_store(P, S, i, lane, F, T);
}

// gate: the FP32 Verlet lists are in use, and this walk stands in only after
// a list overflow
__global__ void __launch_bounds__(8 * kWarp) k_clump_dem(DevParams P, DevState S, const int *dB, int gate)
{
    if (gate && dB[B_LIST_OVF] == 0) return;
    const int lane = threadIdx.x & 31;
    const int sb = dB[B_SB], se = dB[B_SE];
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int i = sb + blockIdx.x * (blockDim.x >> 5) + (int)(threadIdx.x >> 5); i < se; i += nwarps)
        clump_dem_stencil_particle(P, S, i, lane);
}

// FP32 list mode: one warp per debris particle over its Verlet list (radius
// MaxRadius + MARGIN, far beyond the contact distance dx plus any drift
// before the next rebuild), whose entries carry the class of j, so the fluid
// entries are passed over without a gather.
__device__ __forceinline__ void clump_dem_list_particle(const DevParams &P, const DevState &S, int i, int lane)
{
    const int N = P.N;
    const long long ld = N;
    const int cnt = S.nbn[i];
    const double xi[3] = {S.pos[i], S.pos[N + i], S.pos[2 * N + i]};
    const double vi[3] = {S.vel[i], S.vel[N + i], S.vel[2 * N + i]};
    const int ti = S.type[i];
    const int bi = S.bid[i];
    const double mi = particle_density(S, P, i, ti) * P.V;
    double F[3] = {0.0, 0.0, 0.0}, T[3] = {0.0, 0.0, 0.0};
    // four entries per lane loaded before any is used (lists hold at
    // most 192 entries in 3D: at most two rounds)
    for (int k0 = 0; k0 < cnt; k0 += 4 * kWarp) {
        unsigned e[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + lane + u * kWarp;
            e[u] = k < cnt ? __ldg(S.nbl + list_index(k, i, ld)) : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (e[u] & (kEntrySolid | kEntryWall))
                clump_pair(P, S, i, xi, vi, ti, bi, mi, (int)(e[u] & kEntrySlot), F, T);
    }
    clump_store(P, S, i, lane, F, T);
}

__global__ void __launch_bounds__(8 * kWarp) k_clump_dem_list(DevParams P, DevState S, const int *dB)
{
    if (dB[B_LIST_OVF]) return;
    const int lane = threadIdx.x & 31;
    const int sb = dB[B_SB], se = dB[B_SE];
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int i = sb + blockIdx.x * (blockDim.x >> 5) + (int)(threadIdx.x >> 5); i < se; i += nwarps)
        clump_dem_list_particle(P, S, i, lane);
}

// One block per body: its threads take the members, the per-thread sums are
// reduced by warp shuffles and then across the block's warps in warp order
constexpr int kBodyThreads = 256;

template <bool F32>
__device__ __forceinline__ void body_step_block(const DevParams &P, const DevState &S, const DevBodies &Bd, int b)
{
    constexpr int NW = kBodyThreads / kWarp;
    __shared__ double red[NW][6];
    __shared__ double tot[6];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int N = P.N;
    const int m0 = Bd.ptr[b], m1 = Bd.ptr[b + 1];
    double q[4] = {Bd.q[4 * b], Bd.q[4 * b + 1], Bd.q[4 * b + 2], Bd.q[4 * b + 3]};
    double R[3][3];
    quat_to_R(q, R);
    double F[3] = {0.0, 0.0, 0.0}, T[3] = {0.0, 0.0, 0.0};
    for (int m = m0 + (int)threadIdx.x; m < m1; m += kBodyThreads) {
        const int i = Bd.slot_of_row[Bd.member_row[m]];
        double f[3];
        if (F32) {
            const float4 ff = S.f4[i];
            f[0] = ff.x;
            f[1] = ff.y;
            f[2] = ff.z;
        } else {
            for (int k = 0; k < 3; k++) f[k] = S.frc[k * N + i];
        }
        for (int k = 0; k < 3; k++) f[k] += S.frc_dem[k * N + i];
        const double *r0 = Bd.r0 + 3 * m;
        double r[3];
        for (int k = 0; k < 3; k++) r[k] = R[k][0] * r0[0] + R[k][1] * r0[1] + R[k][2] * r0[2];
        for (int k = 0; k < 3; k++) F[k] += f[k];
        T[0] += r[1] * f[2] - r[2] * f[1] + S.frc_dem[3 * N + i];
        T[1] += r[2] * f[0] - r[0] * f[2] + S.frc_dem[4 * N + i];
        T[2] += r[0] * f[1] - r[1] * f[0] + S.frc_dem[5 * N + i];
    }
    for (int k = 0; k < 3; k++) {
        F[k] = warp_sum(F[k]);
        T[k] = warp_sum(T[k]);
    }
    if (lane == 0)
        for (int k = 0; k < 3; k++) {
            red[wid][k] = F[k];
            red[wid][3 + k] = T[k];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0.0;
        for (int w = 0; w < NW; ++w) a += red[w][threadIdx.x];
        tot[threadIdx.x] = a;
    }
    __syncthreads();
    for (int k = 0; k < 3; k++) {
        F[k] = tot[k];
        T[k] = tot[3 + k];
    }
    // integrate (every thread holds the same values)
    const double dt = P.ddt, M = Bd.M[b];
    double X[3], V[3], L[3];
    for (int k = 0; k < 3; k++) {
        V[k] = Bd.V[3 * b + k] + F[k] / M * dt;
        X[k] = Bd.X[3 * b + k] + V[k] * dt;
        L[k] = Bd.L[3 * b + k] + T[k] * dt;
    }
    const double *Ii = Bd.Iinv0 + 9 * b;
    double w[3];
    omega_of(R, Ii, L, w);
    const double wn = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (wn > 0.0) {
        const double h = 0.5 * wn * dt;
        const double c = cos(h), sn = sin(h) / wn;
        const double d[4] = {c, w[0] * sn, w[1] * sn, w[2] * sn};
        const double nq[4] = {d[0] * q[0] - d[1] * q[1] - d[2] * q[2] - d[3] * q[3],
                              d[0] * q[1] + d[1] * q[0] + d[2] * q[3] - d[3] * q[2],
                              d[0] * q[2] - d[1] * q[3] + d[2] * q[0] + d[3] * q[1],
                              d[0] * q[3] + d[1] * q[2] - d[2] * q[1] + d[3] * q[0]};
        const double inv = 1.0 / sqrt(nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3]);
        for (int k = 0; k < 4; k++) q[k] = nq[k] * inv;
    }
    quat_to_R(q, R);
    omega_of(R, Ii, L, w);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; k++) {
            Bd.X[3 * b + k] = X[k];
            Bd.V[3 * b + k] = V[k];
            Bd.L[3 * b + k] = L[k];
            Bd.Fsum[3 * b + k] = F[k];
            Bd.Tsum[3 * b + k] = T[k];
        }
        for (int k = 0; k < 4; k++) Bd.q[4 * b + k] = q[k];
    }
    // place the members
    for (int m = m0 + (int)threadIdx.x; m < m1; m += kBodyThreads) {
        const int i = Bd.slot_of_row[Bd.member_row[m]];
        const double *r0 = Bd.r0 + 3 * m;
        double r[3], x[3], v[3];
        for (int k = 0; k < 3; k++) r[k] = R[k][0] * r0[0] + R[k][1] * r0[1] + R[k][2] * r0[2];
        for (int k = 0; k < 3; k++) x[k] = X[k] + r[k];
        v[0] = V[0] + w[1] * r[2] - w[2] * r[1];
        v[1] = V[1] + w[2] * r[0] - w[0] * r[2];
        v[2] = V[2] + w[0] * r[1] - w[1] * r[0];
        if (F32) {
            float4 p = S.p4[i];
            const unsigned pw = __float_as_uint(p.w);
            const int c[3] = {unpack_cx(pw), unpack_cy(pw), unpack_cz(pw)};
            float rr[3];
            for (int k = 0; k < 3; k++) {
                double a = x[k] - (P.dmin[k] + c[k] * P.cw[k]);
                a -= P.W[k] * rint(a / P.W[k]);
                rr[k] = (float)a;
            }
            S.p4[i] = make_float4(rr[0], rr[1], rr[2], p.w);
            S.v4[i] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
        } else {
            for (int k = 0; k < 3; k++) {
                const double t = x[k] - P.dmin[k];
                S.pos[k * N + i] = (t - P.W[k] * floor(t / P.W[k])) + P.dmin[k];
                S.vel[k * N + i] = v[k];
            }
        }
    }
}

template <bool F32>
__global__ void __launch_bounds__(kBodyThreads) k_body_step(DevParams P, DevState S, DevBodies Bd)
{
    body_step_block<F32>(P, S, Bd, blockIdx.x);
}

// ---- ensemble: the contacts and body updates of every scene in one launch
// each (substep `sub`; scenes with fewer DEM substeps take no part in the
// later ones)

// one warp per debris particle of every scene whose lists are usable
// (LIST) or overflowed (stencil walk)
template <bool LIST>
__global__ void __launch_bounds__(8 * kWarp) k_ens_clump_dem(const EnsScene *__restrict__ tab, int ns, int sub)
{
    __shared__ int pre[kMaxEnsemble + 1];
    const int total = ens_count_prefix(ns, pre, [&](int k) {
        const EnsScene &e = tab[k];
        const bool ovf = e.dB[B_LIST_OVF] != 0;
        return (sub < e.demSteps && e.Bd.B > 0 && ovf != LIST) ? e.dB[B_SE] - e.dB[B_SB] : 0;
    });
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int g = blockIdx.x * (blockDim.x >> 5) + (int)(threadIdx.x >> 5); g < total; g += nwarps) {
        const int k = ens_scene_at(pre, ns, g);
        const EnsScene &e = tab[k];
        const int i = e.dB[B_SB] + g - pre[k];
        if (LIST) clump_dem_list_particle(e.P, e.S, i, lane);
        else clump_dem_stencil_particle(e.P, e.S, i, lane);
    }
}

// one block per body of every scene; bpre[k] = bodies of the scenes before k
__global__ void __launch_bounds__(kBodyThreads) k_ens_body_step(const EnsScene *__restrict__ tab, int ns,
                                                                 const int *__restrict__ bpre, int sub)
{
    const int g = blockIdx.x;
    int lo = 0, hi = ns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bpre[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    const EnsScene &e = tab[lo];
    if (sub >= e.demSteps) return;  // block-uniform
    body_step_block<false>(e.P, e.S, e.Bd, g - bpre[lo]);
}

void launch_ens_clump_dem(const EnsScene *tab, int ns, int sub, cudaStream_t st)
{
    static const int gl = persistent_grid((const void *)k_ens_clump_dem<true>, 8 * kWarp);
    k_ens_clump_dem<true><<<gl, 8 * kWarp, 0, st>>>(tab, ns, sub);
    static const int g = persistent_grid((const void *)k_ens_clump_dem<false>, 8 * kWarp);
    k_ens_clump_dem<false><<<g, 8 * kWarp, 0, st>>>(tab, ns, sub);
}

void launch_ens_body_step(const EnsScene *tab, int ns, const int *bpre, int total_bodies, int sub, cudaStream_t st)
{
    if (total_bodies > 0) k_ens_body_step<<<total_bodies, kBodyThreads, 0, st>>>(tab, ns, bpre, sub);
}

void launch_slot_of_row(const DevParams &P, const int *pidx, int *slot_of_row, cudaStream_t st)
{
    k_slot_of_row<<<(P.N + 255) / 256, 256, 0, st>>>(P.N, pidx, slot_of_row);
}

// Both precisions run the clump contacts and the body update in FP64 on the
// FP64 state of solids and walls (in the FP32 split mode these planes are the
// solids' and walls' master copies, refreshed into the FP32 arrays after the
// substeps), so the template's FP32 branches are not instantiated.
void launch_clump_dem(const DevParams &P, const DevState &S, const int *dB, bool lists, cudaStream_t st)
{
    if (lists) {
        static const int gl = persistent_grid((const void *)k_clump_dem_list, 8 * kWarp);
        k_clump_dem_list<<<gl, 8 * kWarp, 0, st>>>(P, S, dB);
    }
    static const int g = persistent_grid((const void *)k_clump_dem, 8 * kWarp);
    k_clump_dem<<<g, 8 * kWarp, 0, st>>>(P, S, dB, lists ? 1 : 0);
}

void launch_body_step(const DevParams &P, const DevState &S, const DevBodies &Bd, bool f32, cudaStream_t st)
{
    (void)f32;
    if (Bd.B <= 0) return;
    k_body_step<false><<<Bd.B, kBodyThreads, 0, st>>>(P, S, Bd);
}

}  // namespace dmph
