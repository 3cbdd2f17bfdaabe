// FP32 split-precision timestep kernels (DMPH_PRECISION_FP32_SPLIT).
//
// Same step structure, pair sets and per-particle semantics as the FP64
// kernels in dmph_f64.cu (which restate the reference, source/DEM-MPH.cpp),
// but the pair arithmetic runs in FP32 on positions stored relative to the
// origin of each particle's rebuild-time cell: a neighbour j is shifted into
// the frame of i's cell by the minimum-image cell offset times the cell width,
// so every difference is formed between numbers of a few particle spacings.
// The per-pair arithmetic (pair_a32, pair_b32) is shared by two walks:
//   * Verlet lists (default): built at each rebuild by k_build_list32, walked
//     by one thread per particle (k_pass_a32_list, k_pass_b32_list);
//   * the warp-cooperative stencil (k_pass_a32, k_pass_b32, 1/2/4 lanes per
//     particle), used after a list overflow, in DMPH_PAIRS_STENCIL mode and by
//     the stencil ensemble kernels.
// Pass A uses correctly rounded square roots (its strain sum cancels against
// N0p); pass B uses the approximate reciprocal square root.  Sums that cancel
// are carried in FP64.  Accuracy is checked against the FP64 oracle: forces
// within 1e-5 of each particle's force scale at equal pressures.
#include <math_constants.h>

#include "dmph_state.cuh"
#include "dmph_traverse.cuh"

#include <type_traits>

namespace dmph {



struct Tile32 {
    float4 p[kWarp];  // position in the frame of the warp's cell; .w = type as float bits
    float4 v[kWarp];  // velocity; .w = pressure (pass B)
};
struct TileST {
    float4 g[kWarp];  // gravity centre; .w = attractive pressure
};


__device__ __forceinline__ int min_image_cell(int d, int c)
{
    return d > 1 ? d - c : (d < -1 ? d + c : d);
}

// stage particle j into the tile in the frame of cell (ci)
__device__ __forceinline__ void stage32(const DevParams &P, const DevParams32 &Q, const DevState &S, Tile32 &tl,
                                        int j, int slot, int cix, int ciy, int ciz, bool with_pressure)
{
    const float4 pj = S.p4[j];
    const unsigned w = __float_as_uint(pj.w);
    const int dx = min_image_cell(unpack_cx(w) - cix, P.cc[0]);
    const int dy = min_image_cell(unpack_cy(w) - ciy, P.cc[1]);
    const int dz = min_image_cell(unpack_cz(w) - ciz, P.cc[2]);
    tl.p[slot] = make_float4(fmaf((float)dx, Q.cw[0], pj.x), fmaf((float)dy, Q.cw[1], pj.y),
                             fmaf((float)dz, Q.cw[2], pj.z), __int_as_float(unpack_type(w)));
    float4 vj = S.v4[j];
    if (with_pressure) vj.w = S.pres32[j];
    tl.v[slot] = vj;
}

__device__ __forceinline__ void chunk_cell(const DevParams &P, int key_cell, int &cx, int &cy, int &cz)
{
    cx = key_cell / (P.cc[1] * P.cc[2]);
    cy = (key_cell / P.cc[2]) % P.cc[1];
    cz = key_cell % P.cc[2];
}

// ---------------------------------------------------------------- drift
// drift of slot i (fluid moves, walls move or stop, everything's force is
// reset); returns |x - x_ref|^2 in the FP32 frame, +inf for a non-finite
// position or velocity
__device__ __forceinline__ float drift32_slot(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                              const WallMotion &Wm, int i)
{
    const int N = P.N;
    float4 p = S.p4[i];
    float4 v = S.v4[i];
    const unsigned w = __float_as_uint(p.w);
    const int t = unpack_type(w);
    if (is_fluid(t)) {
        p.x = fmaf(v.x, Q.dt, p.x);
        p.y = fmaf(v.y, Q.dt, p.y);
        p.z = fmaf(v.z, Q.dt, p.z);
    } else if (is_wall(t)) {
        if (Wm.moving) {
            const double o[3] = {P.dmin[0] + unpack_cx(w) * P.cw[0], P.dmin[1] + unpack_cy(w) * P.cw[1],
                                 P.dmin[2] + unpack_cz(w) * P.cw[2]};
            double x[3] = {o[0] + p.x, o[1] + p.y, o[2] + p.z}, vv[3];
            double r[3] = {x[0] - Wm.C[t][0], x[1] - Wm.C[t][1], x[2] - Wm.C[t][2]};
            const double(*R)[3] = Wm.R[t];
            const double *om = Wm.Om[t];
            r[0] = R[0][0] * r[0] + R[0][1] * r[1] + R[0][2] * r[2];
            r[1] = R[1][0] * r[0] + R[1][1] * r[1] + R[1][2] * r[2];
            r[2] = R[2][0] * r[0] + R[2][1] * r[1] + R[2][2] * r[2];
            vv[0] = om[1] * r[2] - om[2] * r[1] + Wm.Vel[t][0];
            vv[1] = om[2] * r[0] - om[0] * r[2] + Wm.Vel[t][1];
            vv[2] = om[0] * r[1] - om[1] * r[0] + Wm.Vel[t][2];
            for (int d = 0; d < 3; d++) x[d] = r[d] + Wm.C[t][d] + Wm.Vel[t][d] * P.dt;
            p.x = (float)(x[0] - o[0]);
            p.y = (float)(x[1] - o[1]);
            p.z = (float)(x[2] - o[2]);
            v = make_float4((float)vv[0], (float)vv[1], (float)vv[2], 0.f);
            for (int d = 0; d < 3; d++) {
                const double t0 = x[d] - P.dmin[d];
                S.pos[d * N + i] = (t0 - P.W[d] * floor(t0 / P.W[d])) + P.dmin[d];
                S.vel[d * N + i] = vv[d];
            }
        } else {
            v = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int d = 0; d < 3; d++) S.vel[d * N + i] = 0.0;
        }
    }
    S.p4[i] = p;
    S.v4[i] = v;
    S.f4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 r = S.xref4[i];
    const float dx = p.x - r.x, dy = p.y - r.y, dz = p.z - r.z;
    // a non-finite position or velocity makes the maximum +inf, which the
    // rebuild decision reports instead of rebuilding
    if (!isfinite(p.x + p.y + p.z + v.x + v.y + v.z)) return CUDART_INF_F;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// block maximum of m2, as double bits so the decision compares like the FP64
// path, into *maxshift (one atomic per block); all threads of the block call it
__device__ __forceinline__ void block_max_shift(float m2, unsigned long long *maxshift)
{
    unsigned long long b = __double_as_longlong((double)m2);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_down_sync(kFull, b, o);
        b = ob > b ? ob : b;
    }
    __shared__ unsigned long long red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long mx = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) mx = red[k] > mx ? red[k] : mx;
        atomicMax(maxshift, mx);
    }
    __syncthreads();
}

// REUSE (list reuse): also the largest displacement since the lists were
// built, into *maxshiftL
template <bool REUSE>
__global__ void k_drift32(DevParams P, DevParams32 Q, DevState S, WallMotion Wm, unsigned long long *maxshift,
                          unsigned long long *maxshiftL)
{
    float m2 = 0.f, mL = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.N; i += gridDim.x * blockDim.x) {
        m2 = fmaxf(m2, drift32_slot(P, Q, S, Wm, i));
        if (REUSE) {
            const float4 p = S.p4[i], r = S.xrefL4[i];
            const float dx = p.x - r.x, dy = p.y - r.y, dz = p.z - r.z;
            mL = fmaxf(mL, fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        }
    }
    block_max_shift(m2, maxshift);
    if (REUSE) block_max_shift(mL, maxshiftL);
}

// list reuse: a trigger that keeps the lists makes the current positions the
// trigger positions, as a full rebuild does (k_permute32 writes xref and
// xref4): the FP32 frame positions, and the FP64 ones (the fluid's from the
// FP32 state as k_export32 forms them, the debris' FP64 masters)
__global__ void k_kept_trigger32(DevParams P, DevState S, const int *dB, int n)
{
    if (dB[B_NEED] != 2) return;
    const int N = P.N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = S.p4[i];
        S.xref4[i] = p;
        const unsigned w = __float_as_uint(p.w);
        if (is_fluid(unpack_type(w))) {
            const int c[3] = {unpack_cx(w), unpack_cy(w), unpack_cz(w)};
            const float pr[3] = {p.x, p.y, p.z};
            for (int d = 0; d < 3; d++) {
                const double a = P.dmin[d] + c[d] * P.cw[d] + (double)pr[d];
                const double t = a - P.dmin[d];
                S.xref[d * N + i] = (t - P.W[d] * floor(t / P.W[d])) + P.dmin[d];
            }
        } else {
            for (int d = 0; d < 3; d++) S.xref[d * N + i] = S.pos[d * N + i];
        }
    }
}

// The drift of every scene of an ensemble in one launch (scenes whose walls
// are at rest: no wall motion), each scene's maximum into its own
// accumulator.
__global__ void k_ens_drift32(const EnsScene *__restrict__ tab, int ns)
{
    WallMotion rest;
    rest.moving = 0;
    for (int k = 0; k < ns; ++k) {
        const EnsScene &e = tab[k];
        float m2 = 0.f;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < e.P.N; i += gridDim.x * blockDim.x)
            m2 = fmaxf(m2, drift32_slot(e.P, e.Q, e.S, rest, i));
        block_max_shift(m2, e.maxshift);
    }
}

// ---------------------------------------------------- pass A pair math
// Shared by the stencil kernels and the Verlet-list kernels, so both paths
// evaluate identical arithmetic.
struct IA {  // particle i of pass A
    float4 pi, vi;
    int ti;
    bool si, wi;
};
// VolStrainP = sum(w) - N0p cancels to ~1e-3 of the sum, so that sum is
// carried in FP64 (one add per pair); the divergence terms go into a short
// FP32 partial (dq: the pairs of one block of 8 list entries, or one pair in
// the stencil walk) that is added to the FP64 sum at the end of the block
// (flush_a); the pair terms stay FP32
struct AccA {
    double vsp, div;
    float dA, g0, g1, g2;
    float dq;
};

__device__ __forceinline__ void flush_a(AccA &A)
{
    A.div += (double)A.dq;
    A.dq = 0.f;
}

// one pair (pj in the frame of i's cell, .w = type bits), within the cut-off
template <bool ST>
__device__ __forceinline__ void pair_a32(const DevParams32 &Q, const IA &I, const float4 pj, const float4 vj, AccA &A)
{
    const float q0 = pj.x - I.pi.x, q1 = pj.y - I.pi.y, q2 = pj.z - I.pi.z;
    const float r2 = fmaf(q0, q0, fmaf(q1, q1, q2 * q2));
    const int tj = __float_as_int(pj.w);
    // correctly rounded sqrt for the weights: the approximate reciprocal
    // square root has a bias that would add up over ~100 neighbours in the
    // strain sum; the divergence (zero at rest) takes the approximate 1/r
    const float r = sqrtf(r2);
    const float ir = rsqrtf(r2);
    if (!ST || r2 <= Q.RP2) {
        const float a = fmaf(-r, Q.iRP, 1.f);  // 1 - r/h
        A.vsp += (double)(Q.Bp * a * a);
        const bool sj = is_solid(tj);
        if (!((I.si && is_wall(tj)) || (sj && I.wi) || (sj && I.si))) {
            const float uq = fmaf(vj.x - I.vi.x, q0, fmaf(vj.y - I.vi.y, q1, (vj.z - I.vi.z) * q2));
            A.dq -= uq * ir * Q.dwp * a;  // -(u.e) dw
        }
    }
    if (ST && !(I.si && is_wall(tj))) {
        const float ratio = Q.ratio[I.ti][tj];
        if (r2 <= Q.RA2) {
            const float x = r * Q.iRA;
            A.dA = fmaf(ratio * Q.Ba * x * (1.f - x), (1.f - x), A.dA);
        }
        if (r2 <= Q.RG2) {
            const float a = fmaf(-r, Q.iRG, 1.f);
            const float w = ratio * Q.Bg * a * a * Q.R2g_inv_RG;
            A.g0 = fmaf(q0, w, A.g0);
            A.g1 = fmaf(q1, w, A.g1);
            A.g2 = fmaf(q2, w, A.g2);
        }
    }
}

template <bool ST>
__device__ __forceinline__ void finish_a32(const DevParams &P, const DevParams32 &Q, const DevState &S, int i,
                                           const IA &I, const AccA &A)
{
    const double volstrain = A.vsp - Q.N0p32;
    S.vsp32[i] = (float)volstrain;
    S.div32[i] = (float)A.div;
    const double kappa = volstrain < 0.0 ? 0.0 : P.bulk[I.ti];
    if (!I.si) {
        // the pressure also goes to v4.w, where pass B gathers it together with
        // the velocity (solids keep 0 there, as their PressureP stays 0)
        const float pres = (float)(-P.bvisc[I.ti] * A.div + kappa * volstrain);
        S.pres32[i] = pres;
        reinterpret_cast<float *>(S.v4 + i)[3] = pres;
    }
    if (ST) {
        S.densA32[i] = A.dA;
        float pa = Q.CofA[I.ti] * (A.dA - Q.N0a) / Q.dx;
        if (Q.N0a <= A.dA) pa = 0.f;
        S.pA32[i] = pa;
        S.gc4[i] = make_float4(A.g0, A.g1, A.g2, 0.f);
    }
}

// ---------------------------------------------------------------- pass A
// Densities, divergence and pressures (the FP32 counterpart of k_pass_a in
// dmph_f64.cu).  Each staged batch of 32 candidates is first reduced to a
// per-lane bitmask of the candidates within the cut-off (a branch-free,
// fully unrolled distance test), then each lane walks its own set bits, so
// the kernel-weight arithmetic runs only for pairs that contribute.
template <bool ST, int L>
__device__ __forceinline__ void pass_a32_body(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                               Tile32 &tl, int lane, int cidx)
{
    {
        const Chunk ch = S.chunks[cidx];
        // L lanes per particle: lane = part * G + p holds particle p and tests
        // candidates [part * G, part * G + G) of every staged batch
        constexpr int G = kWarp / L;
        const int part = lane / G;
        const int i = ch.i0 + (lane % G);
        const bool active = (lane % G) < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        int cix, ciy, ciz;
        chunk_cell(P, key_cell, cix, ciy, ciz);
        const int ii = active ? i : ch.i0;
        const float4 pi = S.p4[ii];
        const float4 vi = S.v4[ii];
        const int ti = unpack_type(__float_as_uint(pi.w));
        const IA I{pi, vi, ti, is_solid(ti), is_wall(ti)};
        const float cut2 = ST ? fmaxf(Q.RP2, fmaxf(Q.RA2, Q.RG2)) : Q.RP2;
        AccA A{0.0, 0.0, 0.f, 0.f, 0.f, 0.f, 0.f};
        traverse_stencil_batched(
            P, S.cell_start, key_cell, lane, 7u,
            [&](int j, int slot) { stage32(P, Q, S, tl, j, slot, cix, ciy, ciz, false); },
            [&](int base, int nb) {
                if (!active) return;
                unsigned m = 0;
    #pragma unroll
                for (int s0 = 0; s0 < G; ++s0) {
                    const int s = part * G + s0;
                    const float4 pj = tl.p[s];
                    const float q0 = pj.x - pi.x, q1 = pj.y - pi.y, q2 = pj.z - pi.z;
                    const float r2 = fmaf(q0, q0, fmaf(q1, q1, q2 * q2));
                    m |= (s < nb && r2 <= cut2) ? (1u << s) : 0u;
                }
                const int self = i - base;
                if (self >= 0 && self < kWarp) m &= ~(1u << self);
                while (m) {
                    const int s = __ffs(m) - 1;
                    m &= m - 1;
                    pair_a32<ST>(Q, I, tl.p[s], tl.v[s], A);
                    flush_a(A);
                }
            });
        // combine the L partial sums of each particle
        for (int o = G; o < kWarp; o <<= 1) {
            A.vsp += __shfl_xor_sync(kFull, A.vsp, o);
            A.div += __shfl_xor_sync(kFull, A.div, o);
            if (ST) {
                A.dA += __shfl_xor_sync(kFull, A.dA, o);
                A.g0 += __shfl_xor_sync(kFull, A.g0, o);
                A.g1 += __shfl_xor_sync(kFull, A.g1, o);
                A.g2 += __shfl_xor_sync(kFull, A.g2, o);
            }
        }
        if (!active || part != 0) return;
        finish_a32<ST>(P, Q, S, i, I, A);
    }
}

// ---------------------------------------------------- pass B pair math
struct IB {  // particle i of pass B
    float4 pi, vi, gi;  // gi: gravity centre, .w = attractive pressure (surface tension)
    int ti;
    bool sol;
    float Pi, rhoi, alpha;
};
// The pressure and viscous pair terms both point along the pair direction
// and nearly cancel over the neighbourhood: they are summed as one FP32
// coefficient per pair into a short FP32 partial (fq: the pairs of one block
// of 8 list entries, or one pair in the stencil walk), which is added to the
// FP64 sum f at the end of the block (flush_b).
struct AccB {
    double3 f;  // pressure + viscous terms (fluid), viscous terms (debris)
    float3 fq;  // pending FP32 partial of f
    float3 fD, fB, fS;
    float dragc;
    int drag_j;  // candidate that wrote dragc: the last one in the reference's order wins
};

__device__ __forceinline__ AccB acc_b_zero()
{
    AccB B;
    B.f = make_double3(0.0, 0.0, 0.0);
    B.fq = make_float3(0.f, 0.f, 0.f);
    B.fD = B.fq;
    B.fB = B.fq;
    B.fS = B.fq;
    B.dragc = 0.f;
    B.drag_j = -1;
    return B;
}

__device__ __forceinline__ void flush_b(AccB &B)
{
    B.f.x += (double)B.fq.x;
    B.f.y += (double)B.fq.y;
    B.f.z += (double)B.fq.z;
    B.fq = make_float3(0.f, 0.f, 0.f);
}

template <bool ST>
__device__ __forceinline__ IB make_ib(const DevParams &P, const DevState &S, int ii, float4 pi, float4 vi, int ti)
{
    IB I;
    I.pi = pi;
    I.vi = vi;
    I.ti = ti;
    I.sol = is_solid(ti);
    I.Pi = S.pres32[ii];
    I.rhoi = (float)particle_density(S, P, ii, ti);
    I.gi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ST) {
        I.gi = S.gc4[ii];
        I.gi.w = S.pA32[ii];
    }
    I.alpha = 0.f;
    if (I.sol) {
        const int nci = S.nc[ii];
        I.alpha = nci > 0 ? (float)S.snc[ii] / (float)nci : 0.f;
    }
    return I;
}

// one pair (pj in the frame of i's cell, .w = type bits; vj.w = pressure of
// j; gj = gravity centre of j, .w its attractive pressure), j its slot.
// CLS: 0 = i is fluid, 1 = i is debris, 2 = either (read from I.sol).
template <bool ST, int CLS = 2>
__device__ __forceinline__ void pair_b32(const DevParams32 &Q, const IB &I, const float4 pj, const float4 vj,
                                         const float4 gj, int j, AccB &B)
{
    const float q0 = pj.x - I.pi.x, q1 = pj.y - I.pi.y, q2 = pj.z - I.pi.z;
    const float r2 = fmaf(q0, q0, fmaf(q1, q1, q2 * q2));
    const int tj = __float_as_int(pj.w);
    const int ti = I.ti;
    const bool sol = CLS == 2 ? I.sol : CLS == 1;
    const float u0 = vj.x - I.vi.x, u1 = vj.y - I.vi.y, u2 = vj.z - I.vi.z;
    const float ir = rsqrtf(r2);
    const float r = r2 * ir;
    if (!sol) {
        float c = 0.f;
        if (r2 < Q.RP2) {
            const float a = fmaf(-r, Q.iRP, 1.f);
            c = (I.Pi + vj.w) * Q.dwpV * a * ir;  // (Pi+Pj) dw/r V
        }
        if (r2 < Q.RV2) {
            const float a = fmaf(-r, Q.iRV, 1.f);
            const float uq = fmaf(u0, q0, fmaf(u1, q1, u2 * q2));
            // C mu (u.e) e (-dw)/r V with e = q/r
            c += Q.muij[ti][tj] * uq * a * (ir * ir * ir);
        }
        B.fq.x = fmaf(c, q0, B.fq.x);
        B.fq.y = fmaf(c, q1, B.fq.y);
        B.fq.z = fmaf(c, q2, B.fq.z);
    } else {
        if (!is_wall(tj) && r2 < Q.RV2) {
            const float a = fmaf(-r, Q.iRV, 1.f);
            const float uq = fmaf(u0, q0, fmaf(u1, q1, u2 * q2));
            const float c = Q.muij[ti][tj] * uq * a * (ir * ir * ir);
            B.fq.x = fmaf(c, q0, B.fq.x);
            B.fq.y = fmaf(c, q1, B.fq.y);
            B.fq.z = fmaf(c, q2, B.fq.z);
        }
        if (r2 < Q.RP2 && is_fluid(tj)) {
            const float alpha = I.alpha, rhoi = I.rhoi;
            const float Vs = sqrtf(fmaf(u0, u0, fmaf(u1, u1, u2 * u2)));
            const float Re = alpha * rhoi * Vs * Q.dx / Q.svisc[tj];
            float cd;
            if (alpha < 0.8f)
                cd = (4.f / 3.f) * (150.f * (1.f - alpha) / (alpha * Re) + 1.75f);
            else if (Re <= 1000.f)
                cd = 24.f * (1.f + 0.15f * powf(Re, 0.687f)) / (alpha * Re) * powf(alpha, -2.65f);
            else
                cd = 0.44f;
            B.dragc = cd;
            B.drag_j = j;
            // at zero relative velocity the reference's expression is inf * 0
            // (Re = 0 makes cd infinite, :2785-2791); cd * Vs stays finite as
            // Vs -> 0, so the drag force's limit there is 0, which this build
            // uses (the FP64 parity build keeps the reference's NaN)
            if (Vs > 0.f) {
                const float c = cd * rhoi * Q.drag_pref * Vs;
                B.fD.x = fmaf(c, u0, B.fD.x);
                B.fD.y = fmaf(c, u1, B.fD.y);
                B.fD.z = fmaf(c, u2, B.fD.z);
            }
            const float a = fmaf(-r, Q.iRP, 1.f);
            const float wb = Q.density[tj] * Q.V * Q.Bp * a * a;
            B.fB.x = fmaf(wb, Q.g[0], B.fB.x);
            B.fB.y = fmaf(wb, Q.g[1], B.fB.y);
            B.fB.z = fmaf(wb, Q.g[2], B.fB.z);
        }
    }
    if (ST && !((sol && is_wall(tj)) || (is_solid(tj) && is_wall(ti)))) {
        const float4 gi = I.gi;
        const float rij_ = Q.ratio[ti][tj], rji_ = Q.ratio[tj][ti];
        if (r2 < Q.RA2) {
            const float x = r * Q.iRA;
            const float dwa = Q.Ba * (1.f - x) * (1.f - 3.f * x) * Q.iRA;
            const float c = (gi.w * rij_ + gj.w * rji_) * dwa * ir * Q.V;
            B.fS.x = fmaf(c, q0, B.fS.x);
            B.fS.y = fmaf(c, q1, B.fS.y);
            B.fS.z = fmaf(c, q2, B.fS.z);
        }
        if (r2 < Q.RG2) {
            const float a = fmaf(-r, Q.iRG, 1.f);
            const float w2 = Q.Bg * a * a, dw2 = Q.dwg * a;
            const float ai = Q.ai[ti];
            const float k = Q.R2g_inv_RG * Q.Vdx;
            B.fS.x -= (ai * gj.x * rji_ * w2 - ai * gi.x * rij_ * w2) * k;
            B.fS.y -= (ai * gj.y * rji_ * w2 - ai * gi.y * rij_ * w2) * k;
            B.fS.z -= (ai * gj.z * rji_ * w2 - ai * gi.z * rij_ * w2) * k;
            const float gr = (ai * gj.x * rji_ * dw2 - ai * gi.x * rij_ * dw2) * q0 +
                             (ai * gj.y * rji_ * dw2 - ai * gi.y * rij_ * dw2) * q1 +
                             (ai * gj.z * rji_ * dw2 - ai * gi.z * rij_ * dw2) * q2;
            const float c = gr * ir * k;
            B.fS.x -= c * q0;
            B.fS.y -= c * q1;
            B.fS.z -= c * q2;
        }
    }
}

template <int CLS = 2>
__device__ __forceinline__ void finish_b32(const DevParams &P, const DevParams32 &Q, const DevState &S, int i,
                                           const IB &I, const AccB &B)
{
    const bool sol = CLS == 2 ? I.sol : CLS == 1;
    const float m = sol ? I.rhoi * Q.V : Q.mass[I.ti];
    float4 F;
    if (sol) {
        F.x = (float)(2.0 * B.fD.x + B.fS.x + B.f.x - B.fB.x + (double)m * P.g[0]);
        F.y = (float)(2.0 * B.fD.y + B.fS.y + B.f.y - B.fB.y + (double)m * P.g[1]);
        F.z = (float)(2.0 * B.fD.z + B.fS.z + B.f.z - B.fB.z + (double)m * P.g[2]);
        S.alpha32[i] = I.alpha;
        if (B.drag_j >= 0) S.dragC32[i] = B.dragc;
    } else {
        F.x = (float)(B.f.x + B.fS.x + (double)m * P.g[0]);
        F.y = (float)(B.f.y + B.fS.y + (double)m * P.g[1]);
        F.z = (float)(B.f.z + B.fS.z + (double)m * P.g[2]);
    }
    F.w = 0.f;
    S.f4[i] = F;
}

// ---------------------------------------------------------------- pass B
// All fluid forces (the FP32 counterpart of k_pass_b), same two-phase batch
// scheme.  Chunks hold one particle class, so the fluid/solid split below is
// uniform across the warp.
template <bool ST, int L>
__device__ __forceinline__ void pass_b32_body(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                               Tile32 &tl, TileST &ts, int lane, int cidx)
{
    {
        const Chunk ch = S.chunks[cidx];
        constexpr int G = kWarp / L;  // L lanes per particle, as in pass A
        const int part = lane / G;
        const int i = ch.i0 + (lane % G);
        const bool active = (lane % G) < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        int cix, ciy, ciz;
        chunk_cell(P, key_cell, cix, ciy, ciz);
        const int ii = active ? i : ch.i0;
        const float4 pi = S.p4[ii];
        const float4 vi = S.v4[ii];
        const int ti = unpack_type(__float_as_uint(pi.w));
        const IB I = make_ib<ST>(P, S, ii, pi, vi, ti);
        const float cut2 = ST ? fmaxf(fmaxf(Q.RP2, Q.RV2), fmaxf(Q.RA2, Q.RG2)) : fmaxf(Q.RP2, Q.RV2);
        AccB B = acc_b_zero();
        traverse_stencil_batched(
            P, S.cell_start, key_cell, lane, 7u,
            [&](int j, int slot) {
                stage32(P, Q, S, tl, j, slot, cix, ciy, ciz, true);
                if (ST) {
                    float4 g = S.gc4[j];
                    g.w = S.pA32[j];
                    ts.g[slot] = g;
                }
            },
            [&](int base, int nb) {
                if (!active) return;
                unsigned m = 0;
    #pragma unroll
                for (int s0 = 0; s0 < G; ++s0) {
                    const int s = part * G + s0;
                    const float4 pj = tl.p[s];
                    const float q0 = pj.x - pi.x, q1 = pj.y - pi.y, q2 = pj.z - pi.z;
                    const float r2 = fmaf(q0, q0, fmaf(q1, q1, q2 * q2));
                    m |= (s < nb && r2 < cut2) ? (1u << s) : 0u;
                }
                const int self = i - base;
                if (self >= 0 && self < kWarp) m &= ~(1u << self);
                while (m) {
                    const int s = __ffs(m) - 1;
                    m &= m - 1;
                    pair_b32<ST>(Q, I, tl.p[s], tl.v[s], ST ? ts.g[s] : make_float4(0.f, 0.f, 0.f, 0.f), base + s, B);
                    flush_b(B);
                }
            });
        for (int o = G; o < kWarp; o <<= 1) {
            B.f.x += __shfl_xor_sync(kFull, B.f.x, o);
            B.f.y += __shfl_xor_sync(kFull, B.f.y, o);
            B.f.z += __shfl_xor_sync(kFull, B.f.z, o);
            B.fD.x += __shfl_xor_sync(kFull, B.fD.x, o);
            B.fD.y += __shfl_xor_sync(kFull, B.fD.y, o);
            B.fD.z += __shfl_xor_sync(kFull, B.fD.z, o);
            B.fB.x += __shfl_xor_sync(kFull, B.fB.x, o);
            B.fB.y += __shfl_xor_sync(kFull, B.fB.y, o);
            B.fB.z += __shfl_xor_sync(kFull, B.fB.z, o);
            if (ST) {
                B.fS.x += __shfl_xor_sync(kFull, B.fS.x, o);
                B.fS.y += __shfl_xor_sync(kFull, B.fS.y, o);
                B.fS.z += __shfl_xor_sync(kFull, B.fS.z, o);
            }
            const int oj = __shfl_xor_sync(kFull, B.drag_j, o);
            const float oc = __shfl_xor_sync(kFull, B.dragc, o);
            if (oj > B.drag_j) {
                B.drag_j = oj;
                B.dragc = oc;
            }
        }
        if (!active || part != 0) return;
        finish_b32(P, Q, S, i, I, B);
    }
}

// ------------------------------------------------------- Verlet lists
// List mode of the FP32 build: at every rebuild each particle of pass A's
// range (fluid, debris, walls with fluid in reach) records the particles
// within the reference's list radius MaxRadius + MARGIN at the rebuild-time
// positions (calculateNeighbor, source/DEM-MPH.cpp:1521-1851, uses the same
// radius), in ascending slot order; the rebuild trigger bounds every later
// displacement by MARGIN/2, so every pair a kernel accepts until the next
// rebuild is in the list.  The passes then run one thread per particle over
// its list instead of over the ~800 candidates of the 27-cell stencil.
// Candidates are staged in pairs (2k, 2k+1) so that one packed FP32x2 FMA
// (__ffma2_rn, sm_100) advances the distance tests of both: the same
// round-to-nearest FMAs as scalar fmaf, half the issued instructions.
struct TileL {
    float4 xy[kWarp / 2];  // (x_2k, x_2k+1, y_2k, y_2k+1) in the frame of the warp's cell
    float4 zw[kWarp / 2];  // (z_2k, z_2k+1, |p_2k|^2, |p_2k+1|^2)
    unsigned e[kWarp];     // list entry of the candidate
    int t[kWarp];          // type of the candidate
};
__device__ __forceinline__ void tile_put(TileL &tl, int s, float x, float y, float z, float w)
{
    float *a = reinterpret_cast<float *>(&tl.xy[s >> 1]);
    float *b = reinterpret_cast<float *>(&tl.zw[s >> 1]);
    a[s & 1] = x;
    a[2 + (s & 1)] = y;
    b[s & 1] = z;
    b[2 + (s & 1)] = w;
}
__device__ __forceinline__ float4 tile_get(const TileL &tl, int s)
{
    const float *a = reinterpret_cast<const float *>(&tl.xy[s >> 1]);
    const float *b = reinterpret_cast<const float *>(&tl.zw[s >> 1]);
    return make_float4(a[s & 1], a[2 + (s & 1)], b[s & 1], b[2 + (s & 1)]);
}

// split: the walls are at rest until the next rebuild (set by the host when no
// wall motion is active).  Wall-wall pairs are then summed here, once, with
// pass A's arithmetic (pair_a32 on the same FP32 positions), and only the
// pairs of a wall with fluid or debris go to its list; pass A reads the
// velocity of every wall entry of such lists as zero instead of gathering it.
// One chunk with L lanes per particle: lane = part * G + p holds particle p
// (G = 32 / L) and tests candidates [part * G, part * G + G) of every staged
// batch, so chunks of at most 16 (8) particles take half (a quarter) of the
// distance tests per lane.  A particle's entries stay in ascending order:
// each part writes after the entries of the lower parts of the same batch.
template <bool ST, int L>
__device__ __forceinline__ void build_list32_chunk(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                                   int *dB, float rc2, int split, TileL &tl, int lane, int cidx)
{
    constexpr int G = kWarp / L;
    const int part = lane / G, pl = lane % G;
    const int cap = S.nbl_cap;
    const long long ld = P.N;
    const float cut2 = ST ? fmaxf(Q.RP2, fmaxf(Q.RA2, Q.RG2)) : Q.RP2;  // pass A's
    const Chunk ch = S.chunks[cidx];
    const int i = ch.i0 + pl;
    const bool active = pl < ch.cnt;
    const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
    int cix, ciy, ciz;
    chunk_cell(P, key_cell, cix, ciy, ciz);
    const float4 pi = S.p4[active ? i : ch.i0];
    const int ti = unpack_type(__float_as_uint(pi.w));
    // walls at rest: their wall-wall sums were made at an earlier rebuild and
    // still hold (same slots, same positions) when st_valid says so for the
    // whole chunk; the walk then skips the wall candidates altogether
    const bool keep_sums = split && is_wall(ti) && __all_sync(kFull, !active || S.st_valid[i] != 0);
    const bool wall_i = split && is_wall(ti) && !keep_sums;
    const IA I{pi, make_float4(0.f, 0.f, 0.f, 0.f), ti, is_solid(ti), is_wall(ti)};
    AccA A{0.0, 0.0, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float a0 = -2.f * pi.x, a1 = -2.f * pi.y, a2 = -2.f * pi.z;
    const float thr = rc2 * (1.f + 1e-4f) - fmaf(pi.x, pi.x, fmaf(pi.y, pi.y, pi.z * pi.z));
    int cnt = 0;
    traverse_stencil_batched(
        P, S.cell_start, key_cell, lane, keep_sums ? 3u : 7u,
        [&](int j, int slot) {
            const float4 pj = S.p4[j];
            const unsigned w = __float_as_uint(pj.w);
            const int tj = unpack_type(w);
            const int dx = min_image_cell(unpack_cx(w) - cix, P.cc[0]);
            const int dy = min_image_cell(unpack_cy(w) - ciy, P.cc[1]);
            const int dz = min_image_cell(unpack_cz(w) - ciz, P.cc[2]);
            const float x = fmaf((float)dx, Q.cw[0], pj.x), y = fmaf((float)dy, Q.cw[1], pj.y),
                        z = fmaf((float)dz, Q.cw[2], pj.z);
            tile_put(tl, slot, x, y, z, fmaf(x, x, fmaf(y, y, z * z)));
            tl.t[slot] = tj;
            tl.e[slot] = (unsigned)j | entry_offsets(dx, dy, dz) | (is_solid(tj) ? kEntrySolid : 0u) |
                         (is_wall(tj) ? kEntryWall : 0u);
        },
        [&](int base, int nb) {
            // called by every lane: the count exchange below needs them all.
            // Slots past the batch get a huge norm, so the tests need no
            // bounds check.
            if (lane >= nb) tile_put(tl, lane, 0.f, 0.f, 0.f, 1.0e30f);
            __syncwarp();
            unsigned m = 0;  // bit s0: candidate part * G + s0
            if (active) {
                // |pj - pi|^2 = |pj|^2 - 2 pi.pj + |pi|^2, three FMAs per
                // candidate; its rounding (a few 1e-6 of rc^2 at these
                // magnitudes) is covered by testing against rc^2 (1 + 1e-4),
                // so the list holds every pair within rc and a 5e-5 rc shell
                const float2 A0 = make_float2(a0, a0), A1 = make_float2(a1, a1), A2 = make_float2(a2, a2);
#pragma unroll
                for (int s0 = 0; s0 < G; s0 += 2) {
                    const int k = (part * G + s0) >> 1;
                    const float4 xy = tl.xy[k], zw = tl.zw[k];
                    // fmaf(a0, x, fmaf(a1, y, fmaf(a2, z, w))) of both candidates
                    float2 d = __ffma2_rn(A2, make_float2(zw.x, zw.y), make_float2(zw.z, zw.w));
                    d = __ffma2_rn(A1, make_float2(xy.z, xy.w), d);
                    d = __ffma2_rn(A0, make_float2(xy.x, xy.y), d);
                    m |= (d.x <= thr) ? (1u << s0) : 0u;
                    m |= (d.y <= thr) ? (2u << s0) : 0u;
                }
                const int self = i - base - part * G;
                if (self >= 0 && self < G) m &= ~(1u << self);
                // a batch holds candidates of one class: static walls are
                // summed here (each part its own) and not listed
                if (wall_i && (tl.e[0] & kEntryWall)) {
                    unsigned w = m;
                    while (w) {
                        const int s0 = __ffs(w) - 1;
                        w &= w - 1;
                        const float4 pp = tile_get(tl, part * G + s0);
                        const float4 pj = make_float4(pp.x, pp.y, pp.z, __int_as_float(tl.t[part * G + s0]));
                        const float q0 = pj.x - pi.x, q1 = pj.y - pi.y, q2 = pj.z - pi.z;
                        if (fmaf(q0, q0, fmaf(q1, q1, q2 * q2)) <= cut2)
                            pair_a32<ST>(Q, I, pj, make_float4(0.f, 0.f, 0.f, 0.f), A);
                    }
                    m = 0;
                }
            }
            const int c = __popc(m);
            int before = 0, total = c;
            if (L > 1) {
                total = 0;
#pragma unroll
                for (int q = 0; q < L; ++q) {
                    const int cq = __shfl_sync(kFull, c, q * G + pl);
                    before += q < part ? cq : 0;
                    total += cq;
                }
            }
            if (m) {
                // entry k of slot i sits at block k / 8 (stride 8 N words), word k % 8
                int k = cnt + before;
                unsigned *blk = S.nbl + list_index(k & ~7, i, ld);
                const unsigned *te = tl.e + part * G;
                if (k + c <= cap) {  // the usual case: no capacity test per entry
                    while (m) {      // ascending candidate order
                        const int s0 = __ffs(m) - 1;
                        m &= m - 1;
                        blk[k & 7] = te[s0];
                        ++k;
                        if ((k & 7) == 0) blk += 8 * ld;
                    }
                } else {
                    while (m) {
                        const int s0 = __ffs(m) - 1;
                        m &= m - 1;
                        if (k < cap) blk[k & 7] = te[s0];
                        ++k;
                        if ((k & 7) == 0) blk += 8 * ld;
                    }
                }
            }
            cnt += total;
        });
    if (L > 1 && wall_i) {
        // the parts' static sums, combined
        for (int o = G; o < kWarp; o <<= 1) {
            A.vsp += __shfl_xor_sync(kFull, A.vsp, o);
            if (ST) {
                A.dA += __shfl_xor_sync(kFull, A.dA, o);
                A.g0 += __shfl_xor_sync(kFull, A.g0, o);
                A.g1 += __shfl_xor_sync(kFull, A.g1, o);
                A.g2 += __shfl_xor_sync(kFull, A.g2, o);
            }
        }
    }
    if (!active || part != 0) return;
    if (cnt > cap) atomicExch(dB + B_LIST_OVF, 1);
    S.nbn[i] = cnt < cap ? cnt : cap;
    if (wall_i) {
        S.vsp_st[i] = A.vsp;
        S.st4[i] = make_float4(A.dA, A.g0, A.g1, A.g2);
        S.st_valid[i] = 1;
    }
}

// WPB warps per block, MINB resident blocks per SM requested from the
// register allocator (the launch variants of dmph_autotune_list_build)
// skin_from_dB (list reuse): the list radius is MaxRadius plus the skin
// dB[B_SKIN_NEXT] (hundredths of dx, MARGIN at least), recorded in dB[B_SKIN]
template <bool ST, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * kWarp, MINB) k_build_list32(DevParams P, DevParams32 Q, DevState S, int *dB,
                                                                   float rc2, int split, int skin_from_dB)
{
    __shared__ TileL tiles[WPB];
    TileL &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    if (skin_from_dB) {
        const int h = dB[B_SKIN_NEXT] > 10 ? dB[B_SKIN_NEXT] : 10;
        const float rl = (float)(sqrt(P.rc2) - 0.1 * P.dx + 0.01 * h * P.dx);
        rc2 = rl * rl;
        if (blockIdx.x == 0 && threadIdx.x == 0) dB[B_SKIN] = h;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) dB[B_LIST_SPLIT] = split;
    FOR_EACH_CHUNK(dB, CR_WET, WPB, cidx)
    {
        const int n = S.chunks[cidx].cnt;
        if (n <= 8) build_list32_chunk<ST, 4>(P, Q, S, dB, rc2, split, tl, lane, cidx);
        else if (n <= 16) build_list32_chunk<ST, 2>(P, Q, S, dB, rc2, split, tl, lane, cidx);
        else build_list32_chunk<ST, 1>(P, Q, S, dB, rc2, split, tl, lane, cidx);
    }
}

// Lists built with the walls at rest become invalid once a wall moves: the
// step enqueues this guard in a moving-wall window, and the stencil passes
// stand in until a rebuild makes complete lists.
__global__ void k_list_wall_guard(int *dB)
{
    if (dB[B_LIST_SPLIT]) dB[B_LIST_OVF] = 1;
}

// entries k0 .. k0 + BATCH - 1 of slot i (BATCH divides 8, so they sit in one
// block and load as one vector); entries past the count read as slot 0
template <int BATCH, bool TAIL = true>
__device__ __forceinline__ void load_entries(const DevState &S, int k0, int cnt, int i, long long ld, unsigned *e)
{
    const unsigned *src = S.nbl + list_index(k0, i, ld);
    if (BATCH == 4) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(src));
        e[0] = v.x;
        e[1] = v.y;
        e[2] = v.z;
        e[3] = v.w;
    } else if (BATCH == 2) {
        const uint2 v = __ldg(reinterpret_cast<const uint2 *>(src));
        e[0] = v.x;
        e[1] = v.y;
    } else {
        e[0] = __ldg(src);
    }
    if (TAIL) {
#pragma unroll
        for (int u = 0; u < BATCH; ++u)
            if (k0 + u >= cnt) e[u] = 0u;
    }
}

// j's position in the frame of i's cell, type bits in .w
__device__ __forceinline__ float4 list_pos(const DevParams32 &Q, const DevState &S, unsigned e, int &j)
{
    j = (int)(e & kEntrySlot);
    const float4 pj = __ldg(S.p4 + j);  // positions are read-only in the passes
    return make_float4(fmaf(entry_offset(e, 0), Q.cw[0], pj.x), fmaf(entry_offset(e, 1), Q.cw[1], pj.y),
                       fmaf(entry_offset(e, 2), Q.cw[2], pj.z), __int_as_float(unpack_type(__float_as_uint(pj.w))));
}

// BATCH list entries at a time: their index loads, then their gathers, are
// independent, so the latencies overlap; pairs are still taken in list order
// split: the lists of the last rebuild hold no wall-wall pairs; a wall's sums
// start from the ones the build made of them
template <bool ST, int BATCH>
__device__ __forceinline__ void pass_a32_list_slot(const DevParams &P, const DevParams32 &Q, const DevState &S, int i,
                                                   int split)
{
    const int cnt = S.nbn[i];
    if (cnt < 0) return;
    const long long ld = P.N;
    const float cut2 = ST ? fmaxf(Q.RP2, fmaxf(Q.RA2, Q.RG2)) : Q.RP2;
    const float4 pi = S.p4[i];
    const int ti = unpack_type(__float_as_uint(pi.w));
    const IA I{pi, S.v4[i], ti, is_solid(ti), is_wall(ti)};
    AccA A{0.0, 0.0, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (split && I.wi) {
        A.vsp = S.vsp_st[i];
        if (ST) {
            const float4 t = S.st4[i];
            A.dA = t.x;
            A.g0 = t.y;
            A.g1 = t.z;
            A.g2 = t.w;
        }
    }
    for (int k0 = 0; k0 < cnt; k0 += BATCH) {
        unsigned e[BATCH];
        load_entries<BATCH>(S, k0, cnt, i, ld, e);
        float4 pj[BATCH], vj[BATCH];
        int j[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            pj[u] = list_pos(Q, S, e[u], j[u]);
            // pass A writes only the .w (pressure) of v4, which it does not
            // read; a wall at rest has zero velocity, which is not gathered
            vj[u] = (split && (e[u] & kEntryWall)) ? make_float4(0.f, 0.f, 0.f, 0.f) : __ldg(S.v4 + j[u]);
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const float q0 = pj[u].x - pi.x, q1 = pj[u].y - pi.y, q2 = pj[u].z - pi.z;
            if (k0 + u < cnt && fmaf(q0, q0, fmaf(q1, q1, q2 * q2)) <= cut2) pair_a32<ST>(Q, I, pj[u], vj[u], A);
        }
        // one FP64 add per block of 8 entries, whatever BATCH is
        if (((k0 + BATCH) & 7) == 0) flush_a(A);
    }
    flush_a(A);
    finish_a32<ST>(P, Q, S, i, I, A);
}

template <bool ST, int BATCH, int MINB>
__global__ void __launch_bounds__(256, MINB) k_pass_a32_list(DevParams P, DevParams32 Q, DevState S, const int *dB)
{
    if (dB[B_LIST_OVF]) return;
    const int split = dB[B_LIST_SPLIT];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.N; i += gridDim.x * blockDim.x)
        pass_a32_list_slot<ST, BATCH>(P, Q, S, i, split);
}

// CLS: 0 = slot i holds fluid, 1 = debris, 2 = either.  The single-scene
// step runs the fluid slots [0, fe) here and the debris slots [sb, se) in
// k_pass_b32_list_debris, so the fluid kernel carries none of the drag and
// buoyancy state.
template <bool ST, int BATCH, int CLS = 2>
__device__ __forceinline__ void pass_b32_list_slot(const DevParams &P, const DevParams32 &Q, const DevState &S, int i)
{
    const int cnt = S.nbn[i];
    if (cnt < 0) return;
    const long long ld = P.N;
    const float cut2 = ST ? fmaxf(fmaxf(Q.RP2, Q.RV2), fmaxf(Q.RA2, Q.RG2)) : fmaxf(Q.RP2, Q.RV2);
    const float4 pi = S.p4[i];
    const int ti = unpack_type(__float_as_uint(pi.w));
    const IB I = make_ib<ST>(P, S, i, pi, S.v4[i], ti);
    AccB B = acc_b_zero();
    // full batches without per-entry count tests, then the partial one
    auto batch = [&](int k0, auto tail) {
        constexpr bool TAIL = decltype(tail)::value;
        unsigned e[BATCH];
        load_entries<BATCH, TAIL>(S, k0, cnt, i, ld, e);
        float4 pj[BATCH], vj[BATCH];
        int j[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            pj[u] = list_pos(Q, S, e[u], j[u]);
            vj[u] = __ldg(S.v4 + j[u]);  // .w = pressure, written by pass A (read-only here)
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const float q0 = pj[u].x - pi.x, q1 = pj[u].y - pi.y, q2 = pj[u].z - pi.z;
            if ((!TAIL || k0 + u < cnt) && fmaf(q0, q0, fmaf(q1, q1, q2 * q2)) < cut2) {
                float4 gj = make_float4(0.f, 0.f, 0.f, 0.f);
                if (ST) {
                    gj = S.gc4[j[u]];
                    gj.w = S.pA32[j[u]];
                }
                pair_b32<ST, CLS>(Q, I, pj[u], vj[u], gj, j[u], B);
            }
        }
    };
    const int full = cnt & ~(BATCH - 1);
    int k0 = 0;
    for (; k0 < full; k0 += BATCH) {
        batch(k0, std::false_type{});
        // one FP64 add per block of 8 entries, whatever BATCH is, so every
        // launch variant gives the same bits
        if (((k0 + BATCH) & 7) == 0) flush_b(B);
    }
    if (k0 < cnt) batch(k0, std::true_type{});
    flush_b(B);
    finish_b32<CLS>(P, Q, S, i, I, B);
}

template <bool ST, int BATCH, int MINB, int CLS>
__global__ void __launch_bounds__(256, MINB) k_pass_b32_list(DevParams P, DevParams32 Q, DevState S, const int *dB)
{
    if (dB[B_LIST_OVF]) return;
    FOR_EACH_SLOT(dB, CLS == 1 ? B_SB : -1, CLS == 0 ? B_FE : B_SE, i)
    pass_b32_list_slot<ST, BATCH, CLS>(P, Q, S, i);
}

// Debris slots [sb, se): few particles, each with a long list, so one warp
// per particle with the lanes over its entries (lane l takes entries l,
// l + 32, ...); every pair goes to the FP64 sums on its own and the lanes'
// sums are combined by shuffles; the drag coefficient of the last candidate
// in list order (the largest j) wins, as in the reference.
template <bool ST>
__device__ __forceinline__ void pass_b32_debris_warp(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                                     int i, int lane)
{
    const int cnt = S.nbn[i];
    if (cnt < 0) return;
    const long long ld = P.N;
    const float cut2 = ST ? fmaxf(fmaxf(Q.RP2, Q.RV2), fmaxf(Q.RA2, Q.RG2)) : fmaxf(Q.RP2, Q.RV2);
    const float4 pi = S.p4[i];
    const int ti = unpack_type(__float_as_uint(pi.w));
    const IB I = make_ib<ST>(P, S, i, pi, S.v4[i], ti);
    AccB B = acc_b_zero();
    for (int k = lane; k < cnt; k += kWarp) {
        const unsigned e = __ldg(S.nbl + list_index(k, i, ld));
        int j;
        const float4 pj = list_pos(Q, S, e, j);
        const float4 vj = __ldg(S.v4 + j);
        const float q0 = pj.x - pi.x, q1 = pj.y - pi.y, q2 = pj.z - pi.z;
        if (fmaf(q0, q0, fmaf(q1, q1, q2 * q2)) < cut2) {
            float4 gj = make_float4(0.f, 0.f, 0.f, 0.f);
            if (ST) {
                gj = S.gc4[j];
                gj.w = S.pA32[j];
            }
            pair_b32<ST, 1>(Q, I, pj, vj, gj, j, B);
            flush_b(B);
        }
    }
    for (int o = 1; o < kWarp; o <<= 1) {
        B.f.x += __shfl_xor_sync(kFull, B.f.x, o);
        B.f.y += __shfl_xor_sync(kFull, B.f.y, o);
        B.f.z += __shfl_xor_sync(kFull, B.f.z, o);
        B.fD.x += __shfl_xor_sync(kFull, B.fD.x, o);
        B.fD.y += __shfl_xor_sync(kFull, B.fD.y, o);
        B.fD.z += __shfl_xor_sync(kFull, B.fD.z, o);
        B.fB.x += __shfl_xor_sync(kFull, B.fB.x, o);
        B.fB.y += __shfl_xor_sync(kFull, B.fB.y, o);
        B.fB.z += __shfl_xor_sync(kFull, B.fB.z, o);
        if (ST) {
            B.fS.x += __shfl_xor_sync(kFull, B.fS.x, o);
            B.fS.y += __shfl_xor_sync(kFull, B.fS.y, o);
            B.fS.z += __shfl_xor_sync(kFull, B.fS.z, o);
        }
        const int oj = __shfl_xor_sync(kFull, B.drag_j, o);
        const float oc = __shfl_xor_sync(kFull, B.dragc, o);
        if (oj > B.drag_j) {
            B.drag_j = oj;
            B.dragc = oc;
        }
    }
    if (lane == 0) finish_b32<1>(P, Q, S, i, I, B);
}

template <bool ST>
__global__ void __launch_bounds__(256) k_pass_b32_list_debris(DevParams P, DevParams32 Q, DevState S, const int *dB)
{
    if (dB[B_LIST_OVF]) return;
    const int lane = threadIdx.x & 31;
    const int sb = dB[B_SB], se = dB[B_SE];
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int i = sb + blockIdx.x * (blockDim.x >> 5) + (int)(threadIdx.x >> 5); i < se; i += nwarps)
        pass_b32_debris_warp<ST>(P, Q, S, i, lane);
}

// chunk bodies dispatched on the chunk's size: 4 lanes per particle for up to
// 8 particles, 2 for up to 16, 1 otherwise, so that small chunks (cells at
// free surfaces, walls and debris) keep the warp busy
template <bool ST>
__device__ __forceinline__ void pass_a32_chunk(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                               Tile32 &tl, int lane, int cidx)
{
    const int cnt = S.chunks[cidx].cnt;
    if (cnt <= 8) pass_a32_body<ST, 4>(P, Q, S, tl, lane, cidx);
    else if (cnt <= 16) pass_a32_body<ST, 2>(P, Q, S, tl, lane, cidx);
    else pass_a32_body<ST, 1>(P, Q, S, tl, lane, cidx);
}

template <bool ST>
__device__ __forceinline__ void pass_b32_chunk(const DevParams &P, const DevParams32 &Q, const DevState &S,
                                               Tile32 &tl, TileST &ts, int lane, int cidx)
{
    const int cnt = S.chunks[cidx].cnt;
    if (cnt <= 8) pass_b32_body<ST, 4>(P, Q, S, tl, ts, lane, cidx);
    else if (cnt <= 16) pass_b32_body<ST, 2>(P, Q, S, tl, ts, lane, cidx);
    else pass_b32_body<ST, 1>(P, Q, S, tl, ts, lane, cidx);
}

// ------------------------------------------------- pass kernels (one scene)
// Persistent grids; WPB warps per block (one shared tile per warp) and MINB
// resident blocks per SM requested from the register allocator are the
// autotuned launch parameters (dmph_autotune).
template <bool ST, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * kWarp, MINB) k_pass_a32(DevParams P, DevParams32 Q, DevState S, const int *dB,
                                                                int range, int gate)
{
    // gate: list mode, where this stencil pass stands in only after a list overflow
    if (gate && dB[B_LIST_OVF] == 0) return;
    __shared__ Tile32 tiles[WPB];
    const int lane = threadIdx.x & 31;
    FOR_EACH_CHUNK(dB, range, WPB, cidx) pass_a32_chunk<ST>(P, Q, S, tiles[threadIdx.x >> 5], lane, cidx);
}

template <bool ST, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * kWarp, MINB) k_pass_b32(DevParams P, DevParams32 Q, DevState S, const int *dB,
                                                                int range, int gate)
{
    if (gate && dB[B_LIST_OVF] == 0) return;
    __shared__ Tile32 tiles[WPB];
    __shared__ TileST tst[ST ? WPB : 1];
    const int lane = threadIdx.x & 31;
    FOR_EACH_CHUNK(dB, range, WPB, cidx)
    pass_b32_chunk<ST>(P, Q, S, tiles[threadIdx.x >> 5], tst[ST ? (threadIdx.x >> 5) : 0], lane, cidx);
}

// ------------------------------------------------- pass kernels (ensemble)
// One persistent launch over the chunks of every scene of an ensemble: the
// scenes' chunk ranges are concatenated (prefix sums built per block from
// each scene's device bounds), each warp maps its global chunk index to a
// scene by binary search and runs the same per-chunk body with that scene's
// parameters and state, read from the scene table in global memory.
__device__ __forceinline__ int ens_prefix(const EnsScene *__restrict__ tab, int ns, int range, int *pre, int *beg,
                                          int gate)
{
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
        int b, e;
        chunk_range(tab[k].dB, range, b, e);
        // gate: list mode, where the stencil walks only scenes whose lists overflowed
        const bool skip = gate && tab[k].S.nbn != nullptr && tab[k].dB[B_LIST_OVF] == 0;
        beg[k] = b;
        pre[k + 1] = skip ? 0 : e - b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        pre[0] = 0;
        for (int k = 0; k < ns; ++k) pre[k + 1] += pre[k];
    }
    __syncthreads();
    return pre[ns];
}

__device__ __forceinline__ int ens_scene_of(const int *pre, int ns, int g)
{
    int lo = 0, hi = ns - 1;  // largest k with pre[k] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int WPB, int MINB>
__global__ void __launch_bounds__(WPB * kWarp, MINB) k_ens_pass_a32(const EnsScene *__restrict__ tab, int ns, int range,
                                                                    int gate)
{
    __shared__ Tile32 tiles[WPB];
    __shared__ int pre[kMaxEnsemble + 1], beg[kMaxEnsemble];
    const int total = ens_prefix(tab, ns, range, pre, beg, gate);
    const int lane = threadIdx.x & 31;
    for (int g = blockIdx.x * WPB + (int)(threadIdx.x >> 5); g < total; g += gridDim.x * WPB) {
        const int k = ens_scene_of(pre, ns, g);
        const EnsScene &e = tab[k];
        const int cidx = beg[k] + g - pre[k];
        if (e.P.surface_tension) pass_a32_chunk<true>(e.P, e.Q, e.S, tiles[threadIdx.x >> 5], lane, cidx);
        else pass_a32_chunk<false>(e.P, e.Q, e.S, tiles[threadIdx.x >> 5], lane, cidx);
    }
}

template <int WPB, int MINB>
__global__ void __launch_bounds__(WPB * kWarp, MINB) k_ens_pass_b32(const EnsScene *__restrict__ tab, int ns, int gate)
{
    __shared__ Tile32 tiles[WPB];
    __shared__ TileST tst[WPB];
    __shared__ int pre[kMaxEnsemble + 1], beg[kMaxEnsemble];
    const int total = ens_prefix(tab, ns, CR_FLUID_SOLID, pre, beg, gate);
    const int lane = threadIdx.x & 31;
    for (int g = blockIdx.x * WPB + (int)(threadIdx.x >> 5); g < total; g += gridDim.x * WPB) {
        const int k = ens_scene_of(pre, ns, g);
        const EnsScene &e = tab[k];
        const int cidx = beg[k] + g - pre[k];
        const int w = threadIdx.x >> 5;
        if (e.P.surface_tension) pass_b32_chunk<true>(e.P, e.Q, e.S, tiles[w], tst[w], lane, cidx);
        else pass_b32_chunk<false>(e.P, e.Q, e.S, tiles[w], tst[w], lane, cidx);
    }
}

// List-mode ensemble passes: one thread per slot over the concatenated slot
// ranges of the scenes (kind 0: all slots, pass A; 1: fluid slots, pass B;
// 2: debris slots, pass B); a scene whose lists overflowed at its last
// rebuild is left to the stencil ensemble kernels, which then run for that
// scene only.
__device__ __forceinline__ int ens_slot_prefix(const EnsScene *__restrict__ tab, int ns, int kind, int *pre)
{
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
        const EnsScene &e = tab[k];
        const bool ok = e.S.nbn != nullptr && e.dB[B_LIST_OVF] == 0;
        const int n = kind == 0 ? e.P.N : (kind == 1 ? e.dB[B_FE] : e.dB[B_SE] - e.dB[B_SB]);
        pre[k + 1] = ok ? n : 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        pre[0] = 0;
        for (int k = 0; k < ns; ++k) pre[k + 1] += pre[k];
    }
    __syncthreads();
    return pre[ns];
}

template <bool PASS_B>
__global__ void __launch_bounds__(256) k_ens_pass_list(const EnsScene *__restrict__ tab, int ns)
{
    __shared__ int pre[kMaxEnsemble + 1];
    const int total = ens_slot_prefix(tab, ns, PASS_B ? 1 : 0, pre);
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const int k = ens_scene_of(pre, ns, g);
        const EnsScene &e = tab[k];
        const int i = g - pre[k];
        if (PASS_B) {  // fluid slots; the debris slots go to k_ens_pass_b_debris
            if (e.P.surface_tension) pass_b32_list_slot<true, 2, 0>(e.P, e.Q, e.S, i);
            else pass_b32_list_slot<false, 2, 0>(e.P, e.Q, e.S, i);
        } else {
            const int split = e.dB[B_LIST_SPLIT];
            if (e.P.surface_tension) pass_a32_list_slot<true, 2>(e.P, e.Q, e.S, i, split);
            else pass_a32_list_slot<false, 2>(e.P, e.Q, e.S, i, split);
        }
    }
}

// pass B of the debris slots of all scenes: one warp per particle, as in the
// single-scene step
__global__ void __launch_bounds__(256) k_ens_pass_b_debris(const EnsScene *__restrict__ tab, int ns)
{
    __shared__ int pre[kMaxEnsemble + 1];
    const int total = ens_slot_prefix(tab, ns, 2, pre);
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int g = blockIdx.x * (blockDim.x >> 5) + (int)(threadIdx.x >> 5); g < total; g += nwarps) {
        const int k = ens_scene_of(pre, ns, g);
        const EnsScene &e = tab[k];
        const int i = e.dB[B_SB] + g - pre[k];
        if (e.P.surface_tension) pass_b32_debris_warp<true>(e.P, e.Q, e.S, i, lane);
        else pass_b32_debris_warp<false>(e.P, e.Q, e.S, i, lane);
    }
}

__global__ void k_ens_fluid_accel32(const EnsScene *__restrict__ tab, int ns)
{
    for (int k = 0; k < ns; ++k) {
        const EnsScene &e = tab[k];
        const int fe = e.dB[B_FE];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < fe; i += gridDim.x * blockDim.x) {
            const float4 f = e.S.f4[i];
            float4 v = e.S.v4[i];
            const float c = e.Q.dt / e.Q.mass[unpack_type(__float_as_uint(e.S.p4[i].w))];
            v.x = fmaf(f.x, c, v.x);
            v.y = fmaf(f.y, c, v.y);
            v.z = fmaf(f.z, c, v.z);
            e.S.v4[i] = v;
        }
    }
}

__global__ void k_fluid_accel32(DevParams32 Q, DevState S, const int *dB)
{
    FOR_EACH_SLOT(dB, -1, B_FE, i)
    {
        const float4 f = S.f4[i];
        float4 v = S.v4[i];
        const float k = Q.dt / Q.mass[unpack_type(__float_as_uint(S.p4[i].w))];
        v.x = fmaf(f.x, k, v.x);
        v.y = fmaf(f.y, k, v.y);
        v.z = fmaf(f.z, k, v.z);
        S.v4[i] = v;
    }
}

// ------------------------------------------------------- layout conversion
// FP32 split state -> FP64 absolute positions (wrapped into the periodic
// domain like calculatePeriodicBoundary :3153) and velocities, into the FP64
// planes; used by the rebuild (cell keys) and by the state getters.
__global__ void k_export32(DevParams P, DevState S, double *pos, double *vel, int fluid_only)
{
    const int N = P.N;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 p = S.p4[i];
    const float4 v = S.v4[i];
    const unsigned w = __float_as_uint(p.w);
    // solids and walls keep their FP64 master state in the planes
    if (fluid_only && !is_fluid(unpack_type(w))) return;
    const int c[3] = {unpack_cx(w), unpack_cy(w), unpack_cz(w)};
    const float pr[3] = {p.x, p.y, p.z};
    const float vr[3] = {v.x, v.y, v.z};
    for (int d = 0; d < 3; d++) {
        const double a = P.dmin[d] + c[d] * P.cw[d] + (double)pr[d];
        const double t = a - P.dmin[d];
        pos[d * N + i] = (t - P.W[d] * floor(t / P.W[d])) + P.dmin[d];
        if (vel) vel[d * N + i] = (double)vr[d];
    }
}

// permutation of the FP32 state at a rebuild: the new slot's cell comes from
// its sorted key, its position is re-expressed relative to that cell
// slots [0, n) (n < N: the walls keep their slots, see enqueue_rebuild)
__global__ void k_permute32(DevParams P, int n, const unsigned long long *__restrict__ words,
                            const double *__restrict__ xabs,
                            const float4 *__restrict__ v_in, const int *__restrict__ type_in,
                            const int *__restrict__ pidx_in, float4 *__restrict__ p_out, float4 *__restrict__ v_out,
                            int *__restrict__ type_out, int *__restrict__ pidx_out, double *__restrict__ xref,
                            float4 *__restrict__ xref4, const int *__restrict__ bid_in, int *__restrict__ bid_out,
                            const double *__restrict__ vabs, double *__restrict__ pos_out, double *__restrict__ vel_out,
                            float4 *__restrict__ xrefL4)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.N;
    if (i >= n) return;
    const unsigned long long wd = words[i];
    const int src = (int)word_slot(wd);
    const int kc = (int)(word_key(wd) % (unsigned)P.T);
    int c[3];
    c[0] = kc / (P.cc[1] * P.cc[2]);
    c[1] = (kc / P.cc[2]) % P.cc[1];
    c[2] = kc % P.cc[2];
    const int t = type_in[src];
    float r[3];
    for (int d = 0; d < 3; d++) {
        const double x = xabs[d * N + src];
        xref[d * N + i] = x;
        pos_out[d * N + i] = x;
        vel_out[d * N + i] = vabs[d * N + src];
        r[d] = (float)(x - (P.dmin[d] + c[d] * P.cw[d]));
    }
    const float4 p = make_float4(r[0], r[1], r[2], __uint_as_float(pack_cell(t, c[0], c[1], c[2])));
    p_out[i] = p;
    xref4[i] = p;
    if (xrefL4) xrefL4[i] = p;
    v_out[i] = v_in[src];
    type_out[i] = t;
    pidx_out[i] = pidx_in[src];
    if (bid_in) bid_out[i] = bid_in[src];
}

// FP64 planes -> FP32 split state in the current cells (dmph_set_state, create)
__global__ void k_import32(DevParams P, DevState S, const double *pos, const double *vel)
{
    const int N = P.N;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float4 p = S.p4[i];
    const unsigned w = __float_as_uint(p.w);
    const int c[3] = {unpack_cx(w), unpack_cy(w), unpack_cz(w)};
    float r[3];
    for (int d = 0; d < 3; d++) {
        double a = pos[d * N + i] - (P.dmin[d] + c[d] * P.cw[d]);
        // nearest periodic image of the cell origin
        a -= P.W[d] * rint(a / P.W[d]);
        r[d] = (float)a;
    }
    S.p4[i] = make_float4(r[0], r[1], r[2], p.w);
    if (vel) S.v4[i] = make_float4((float)vel[i], (float)vel[N + i], (float)vel[2 * N + i], 0.f);
}

// FP32 mode: the DEM and the rigid bodies run in FP64 on the solids' FP64
// master state (the planes S.pos/S.vel), so contacts see exact lattice
// spacings.  Before the substeps, the solids' FP32 fluid forces seed the FP64
// force planes; after them, the FP32 positions and velocities of the solids
// are refreshed from the masters.
__device__ __forceinline__ void solid_force_to64_slot(const DevParams &P, const DevState &S, int i)
{
    const float4 f = S.f4[i];
    S.frc[i] = f.x;
    S.frc[P.N + i] = f.y;
    S.frc[2 * P.N + i] = f.z;
}
__device__ __forceinline__ void sync_solid32_slot(const DevParams &P, const DevState &S, int i)
{
    const int N = P.N;
    const float4 p = S.p4[i];
    const unsigned w = __float_as_uint(p.w);
    const int c[3] = {unpack_cx(w), unpack_cy(w), unpack_cz(w)};
    float r[3];
    for (int d = 0; d < 3; d++) {
        double a = S.pos[d * N + i] - (P.dmin[d] + c[d] * P.cw[d]);
        a -= P.W[d] * rint(a / P.W[d]);
        r[d] = (float)a;
    }
    S.p4[i] = make_float4(r[0], r[1], r[2], p.w);
    S.v4[i] = make_float4((float)S.vel[i], (float)S.vel[N + i], (float)S.vel[2 * N + i], 0.f);
}
__global__ void k_solid_force_to64(DevParams P, DevState S, const int *dB)
{
    FOR_EACH_SLOT(dB, B_SB, B_SE, i) solid_force_to64_slot(P, S, i);
}
__global__ void k_sync_solids32(DevParams P, DevState S, const int *dB)
{
    FOR_EACH_SLOT(dB, B_SB, B_SE, i) sync_solid32_slot(P, S, i);
}
// the same over every scene of an ensemble, one launch each
__global__ void k_ens_solid_force_to64(const EnsScene *__restrict__ tab, int ns)
{
    for (int k = 0; k < ns; ++k) {
        const EnsScene &e = tab[k];
        FOR_EACH_SLOT(e.dB, B_SB, B_SE, i) solid_force_to64_slot(e.P, e.S, i);
    }
}
__global__ void k_ens_sync_solids32(const EnsScene *__restrict__ tab, int ns)
{
    for (int k = 0; k < ns; ++k) {
        const EnsScene &e = tab[k];
        FOR_EACH_SLOT(e.dB, B_SB, B_SE, i) sync_solid32_slot(e.P, e.S, i);
    }
}
void launch_solid_force_to64(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st)
{
    k_solid_force_to64<<<148, 256, 0, st>>>(P, S, dB);
}
void launch_sync_solids32(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st)
{
    k_sync_solids32<<<148, 256, 0, st>>>(P, S, dB);
}
void launch_ens_drift32(const EnsScene *tab, int ns, int sms, cudaStream_t st)
{
    k_ens_drift32<<<sms * 8, 256, 0, st>>>(tab, ns);
}
void launch_ens_solid_force_to64(const EnsScene *tab, int ns, cudaStream_t st)
{
    k_ens_solid_force_to64<<<148, 256, 0, st>>>(tab, ns);
}
void launch_ens_sync_solids32(const EnsScene *tab, int ns, cudaStream_t st)
{
    k_ens_sync_solids32<<<148, 256, 0, st>>>(tab, ns);
}

// The lattice sum N0p (initializeWeight :1078-1119) evaluated with exactly
// the FP32 arithmetic of pass A.  VolStrainP = sum(w) - N0p cancels; any
// rounding bias of the FP32 kernel evaluation (constants 1/h and B are
// rounded once) then appears identically in both terms and drops out.
__global__ void k_lattice32(DevParams P, DevParams32 Q, double *out)
{
    const int range = (int)(P.RP / P.dx + 3.0);
    const int zr = P.dim == 2 ? 0 : range;
    double sum = 0.0;
    for (int ix = -range; ix <= range; ++ix)
        for (int iy = -range; iy <= range; ++iy)
            for (int iz = -zr; iz <= zr; ++iz) {
                if (ix == 0 && iy == 0 && iz == 0) continue;
                const float q0 = (float)(P.dx * ix), q1 = (float)(P.dx * iy), q2 = (float)(P.dx * iz);
                const float r2 = fmaf(q0, q0, fmaf(q1, q1, q2 * q2));
                if (r2 <= Q.RP2) {
                    const float r = sqrtf(r2);
                    const float a = fmaf(-r, Q.iRP, 1.f);
                    sum += (double)(Q.Bp * a * a);
                }
            }
    *out = sum;
}

double lattice_n0p32(const DevParams &P, const DevParams32 &Q, cudaStream_t st)
{
    double *d = nullptr, h = P.N0p;
    if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return h;
    k_lattice32<<<1, 1, 0, st>>>(P, Q, d);
    if (cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        h = P.N0p;
    cudaFree(d);
    return h;
}

// widen an FP32 field to FP64 (getters)
__global__ void k_widen_f(const float *in, double *out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}
__global__ void k_widen_f4(const float4 *in, double *out, int count, int stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 v = in[i];
    out[i] = v.x;
    out[stride + i] = v.y;
    out[2 * stride + i] = v.z;
}

// ---------------------------------------------------------------- host side
DevParams32 make_params32(const DevParams &P)
{
    DevParams32 Q;
    for (int d = 0; d < 3; d++) {
        Q.cw[d] = (float)P.cw[d];
        Q.g[d] = (float)P.g[d];
    }
    Q.dx = (float)P.dx;
    Q.V = (float)P.V;
    Q.dt = (float)P.dt;
    Q.ddt = (float)P.ddt;
    Q.dx2 = (float)P.dx2;
    Q.RP2 = (float)P.RP2;
    Q.RV2 = (float)P.RV2;
    Q.RA2 = (float)P.RA2;
    Q.RG2 = (float)P.RG2;
    Q.iRP = (float)(1.0 / P.RP);
    Q.iRV = (float)(1.0 / P.RV);
    Q.iRA = (float)(1.0 / P.RA);
    Q.iRG = (float)(1.0 / P.RG);
    Q.Bp = (float)P.Bp;
    Q.Bv = (float)P.Bv;
    Q.Ba = (float)P.Ba;
    Q.Bg = (float)P.Bg;
    Q.dwp = (float)(-2.0 * P.Bp / P.RP);
    Q.dwv = (float)(-2.0 * P.Bv / P.RV);
    Q.dwg = (float)(-2.0 * P.Bg / P.RG);
    Q.N0p = (float)P.N0p;
    Q.N0a = (float)P.N0a;
    Q.R2g_inv_RG = (float)(P.RG / P.R2g);
    Q.viscC = (float)P.viscC;
    Q.Reff = (float)P.Reff;
    Q.Vdx = (float)(P.V / P.dx);
    Q.drag_pref = (float)(0.5 * P.dx * P.dx * P.dx);
    Q.dwpV = (float)(-2.0 * P.Bp / P.RP * P.V);
    for (int t = 0; t < kTypes; t++) {
        Q.mass[t] = (float)P.mass[t];
        Q.density[t] = (float)P.density[t];
        Q.bulk[t] = (float)P.bulk[t];
        Q.bvisc[t] = (float)P.bvisc[t];
        Q.svisc[t] = (float)P.svisc[t];
        Q.friction[t] = (float)P.friction[t];
        Q.CofA[t] = (float)P.CofA[t];
        Q.ai[t] = (float)P.ai[t];
        Q.logE[t] = (float)P.logE[t];
        Q.cnDen[t] = (float)P.cnDen[t];
        Q.ctFac[t] = (float)P.ctFac[t];
        for (int u = 0; u < kTypes; u++) {
            Q.ratio[t][u] = (float)P.ratio[t][u];
            Q.Eeff[t][u] = (float)P.Eeff[t][u];
            Q.KtFac[t][u] = (float)P.KtFac[t][u];
            // C mu_ij (-dw/da) V / h-free part of the viscous pair term: C * harmonic-mean mu * 2B/h * V
            const double mu = (P.svisc[t] + P.svisc[u]) > 0.0 ? 2.0 * (P.svisc[t] * P.svisc[u]) / (P.svisc[t] + P.svisc[u]) : 0.0;
            Q.muij[t][u] = (float)(P.viscC * mu * (2.0 * P.Bv / P.RV) * P.V);
        }
    }
    return Q;
}

void launch_drift32(const DevParams &P, const DevParams32 &Q, const DevState &S, const WallMotion &Wm,
                    unsigned long long *maxshift, int sms, cudaStream_t st, unsigned long long *maxshiftL)
{
    int blocks = (P.N + 255) / 256;
    if (blocks > sms * 8) blocks = sms * 8;
    if (maxshiftL)
        k_drift32<true><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(P, Q, S, Wm, maxshift, maxshiftL);
    else
        k_drift32<false><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(P, Q, S, Wm, maxshift, nullptr);
}
void launch_kept_trigger32(const DevParams &P, const DevState &S, const int *dB, int n, cudaStream_t st)
{
    k_kept_trigger32<<<148 * 4, 256, 0, st>>>(P, S, dB, n);
}
// launch-parameter variants the autotuner chooses from: warps per block x
// requested resident blocks per SM
#define DMPH_PASS_VARIANTS(X) X(0, 8, 1) X(1, 4, 1) X(2, 16, 1) X(3, 8, 4) X(4, 4, 8)

template <class K>
static int grid_for(K kernel, int threads)
{
    return persistent_grid((const void *)kernel, threads);
}

void launch_pass_a32(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int range,
                     int variant, cudaStream_t st, int gate)
{
#define DMPH_LAUNCH_A(ID, WPB, MINB)                                                              \
    case ID:                                                                                      \
        if (P.surface_tension) {                                                                  \
            static const int g = grid_for(k_pass_a32<true, WPB, MINB>, WPB * kWarp);              \
            k_pass_a32<true, WPB, MINB><<<g, WPB * kWarp, 0, st>>>(P, Q, S, dB, range, gate);           \
        } else {                                                                                  \
            static const int g = grid_for(k_pass_a32<false, WPB, MINB>, WPB * kWarp);             \
            k_pass_a32<false, WPB, MINB><<<g, WPB * kWarp, 0, st>>>(P, Q, S, dB, range, gate);          \
        }                                                                                         \
        break;
    switch (variant) {
        DMPH_PASS_VARIANTS(DMPH_LAUNCH_A)
    default: break;
    }
#undef DMPH_LAUNCH_A
}

void launch_pass_b32(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int variant,
                     cudaStream_t st, int gate)
{
#define DMPH_LAUNCH_B(ID, WPB, MINB)                                                              \
    case ID:                                                                                      \
        if (P.surface_tension) {                                                                  \
            static const int g = grid_for(k_pass_b32<true, WPB, MINB>, WPB * kWarp);              \
            k_pass_b32<true, WPB, MINB><<<g, WPB * kWarp, 0, st>>>(P, Q, S, dB, CR_FLUID_SOLID, gate);  \
        } else {                                                                                  \
            static const int g = grid_for(k_pass_b32<false, WPB, MINB>, WPB * kWarp);             \
            k_pass_b32<false, WPB, MINB><<<g, WPB * kWarp, 0, st>>>(P, Q, S, dB, CR_FLUID_SOLID, gate); \
        }                                                                                         \
        break;
    switch (variant) {
        DMPH_PASS_VARIANTS(DMPH_LAUNCH_B)
    default: break;
    }
#undef DMPH_LAUNCH_B
}

// launch variants of the list build: warps per block x requested resident
// blocks per SM (8 x 3 at 80 registers; 8 x 4 and 4 x 8 at 64)
#define DMPH_BUILD_VARIANTS(X) X(0, 8, 3) X(1, 8, 4) X(2, 4, 8)

void launch_build_list32(const DevParams &P, const DevParams32 &Q, const DevState &S, int *dB, int split,
                         cudaStream_t st, int variant, int skin_from_dB)
{
    cudaMemsetAsync(dB + B_LIST_OVF, 0, sizeof(int), st);
    cudaMemsetAsync(S.nbn, 0xFF, sizeof(int) * (size_t)P.N, st);
#define DMPH_LAUNCH_BUILD(ID, WPB, MINB)                                                              \
    case ID:                                                                                          \
        if (P.surface_tension) {                                                                      \
            static const int g = grid_for(k_build_list32<true, WPB, MINB>, WPB * kWarp);              \
            k_build_list32<true, WPB, MINB><<<g, WPB * kWarp, 0, st>>>(P, Q, S, dB, (float)P.rc2, split,      \
                                                                       skin_from_dB);                 \
        } else {                                                                                      \
            static const int g = grid_for(k_build_list32<false, WPB, MINB>, WPB * kWarp);             \
            k_build_list32<false, WPB, MINB><<<g, WPB * kWarp, 0, st>>>(P, Q, S, dB, (float)P.rc2, split,     \
                                                                        skin_from_dB);                \
        }                                                                                             \
        break;
    switch (variant) {
        DMPH_BUILD_VARIANTS(DMPH_LAUNCH_BUILD)
    default: break;
    }
#undef DMPH_LAUNCH_BUILD
}

void launch_list_wall_guard(int *dB, cudaStream_t st)
{
    k_list_wall_guard<<<1, 1, 0, st>>>(dB);
}

// list-pass variants the autotuner chooses from: entries per batch x
// resident blocks of 256 threads requested per SM
#define DMPH_LIST_VARIANTS(X) X(0, 1, 4) X(1, 2, 3) X(2, 4, 2) X(3, 2, 4)

void launch_pass_a32_list(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int variant,
                          cudaStream_t st)
{
#define DMPH_LAUNCH_LA(ID, BATCH, MINB)                                                   \
    case ID:                                                                              \
        if (P.surface_tension) {                                                          \
            static const int g = grid_for(k_pass_a32_list<true, BATCH, MINB>, 256);       \
            k_pass_a32_list<true, BATCH, MINB><<<g, 256, 0, st>>>(P, Q, S, dB);           \
        } else {                                                                          \
            static const int g = grid_for(k_pass_a32_list<false, BATCH, MINB>, 256);      \
            k_pass_a32_list<false, BATCH, MINB><<<g, 256, 0, st>>>(P, Q, S, dB);          \
        }                                                                                 \
        break;
    switch (variant) {
        DMPH_LIST_VARIANTS(DMPH_LAUNCH_LA)
    default: break;
    }
#undef DMPH_LAUNCH_LA
}

void launch_pass_b32_list(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int variant,
                          cudaStream_t st)
{
    // fluid slots with the tuned variant
#define DMPH_LAUNCH_LB(ID, BATCH, MINB)                                                   \
    case ID:                                                                              \
        if (P.surface_tension) {                                                          \
            static const int g = grid_for(k_pass_b32_list<true, BATCH, MINB, 0>, 256);    \
            k_pass_b32_list<true, BATCH, MINB, 0><<<g, 256, 0, st>>>(P, Q, S, dB);        \
        } else {                                                                          \
            static const int g = grid_for(k_pass_b32_list<false, BATCH, MINB, 0>, 256);   \
            k_pass_b32_list<false, BATCH, MINB, 0><<<g, 256, 0, st>>>(P, Q, S, dB);       \
        }                                                                                 \
        break;
    switch (variant) {
        DMPH_LIST_VARIANTS(DMPH_LAUNCH_LB)
    default: break;
    }
#undef DMPH_LAUNCH_LB
    // debris slots: one warp per particle
    if (P.surface_tension) {
        static const int g = grid_for(k_pass_b32_list_debris<true>, 256);
        k_pass_b32_list_debris<true><<<g, 256, 0, st>>>(P, Q, S, dB);
    } else {
        static const int g = grid_for(k_pass_b32_list_debris<false>, 256);
        k_pass_b32_list_debris<false><<<g, 256, 0, st>>>(P, Q, S, dB);
    }
}

void launch_ens_pass_a32(const EnsScene *tab, int ns, int variant, cudaStream_t st, int gate)
{
#define DMPH_LAUNCH_EA(ID, WPB, MINB)                                                     \
    case ID: {                                                                            \
        static const int g = grid_for(k_ens_pass_a32<WPB, MINB>, WPB * kWarp);            \
        k_ens_pass_a32<WPB, MINB><<<g, WPB * kWarp, 0, st>>>(tab, ns, CR_WET, gate);            \
        break;                                                                            \
    }
    switch (variant) {
        DMPH_PASS_VARIANTS(DMPH_LAUNCH_EA)
    default: break;
    }
#undef DMPH_LAUNCH_EA
}

void launch_ens_pass_b32(const EnsScene *tab, int ns, int variant, cudaStream_t st, int gate)
{
#define DMPH_LAUNCH_EB(ID, WPB, MINB)                                                     \
    case ID: {                                                                            \
        static const int g = grid_for(k_ens_pass_b32<WPB, MINB>, WPB * kWarp);            \
        k_ens_pass_b32<WPB, MINB><<<g, WPB * kWarp, 0, st>>>(tab, ns, gate);                    \
        break;                                                                            \
    }
    switch (variant) {
        DMPH_PASS_VARIANTS(DMPH_LAUNCH_EB)
    default: break;
    }
#undef DMPH_LAUNCH_EB
}

void launch_ens_pass_list(const EnsScene *tab, int ns, bool pass_b, cudaStream_t st)
{
    if (pass_b) {
        static const int g = grid_for(k_ens_pass_list<true>, 256);
        k_ens_pass_list<true><<<g, 256, 0, st>>>(tab, ns);
        static const int gd = grid_for(k_ens_pass_b_debris, 256);
        k_ens_pass_b_debris<<<gd, 256, 0, st>>>(tab, ns);
    } else {
        static const int g = grid_for(k_ens_pass_list<false>, 256);
        k_ens_pass_list<false><<<g, 256, 0, st>>>(tab, ns);
    }
}

void launch_ens_fluid_accel32(const EnsScene *tab, int ns, cudaStream_t st)
{
    k_ens_fluid_accel32<<<148 * 4, 256, 0, st>>>(tab, ns);
}

void launch_fluid_accel32(const DevParams32 &Q, const DevState &S, const int *dB, cudaStream_t st)
{
    k_fluid_accel32<<<148 * 4, 256, 0, st>>>(Q, S, dB);
}
void launch_export32(const DevParams &P, const DevState &S, double *pos, double *vel, cudaStream_t st)
{
    k_export32<<<(P.N + 255) / 256, 256, 0, st>>>(P, S, pos, vel, 1);
}
void launch_import32(const DevParams &P, const DevState &S, const double *pos, const double *vel, cudaStream_t st)
{
    k_import32<<<(P.N + 255) / 256, 256, 0, st>>>(P, S, pos, vel);
}
void launch_permute32(const DevParams &P, int n, const unsigned long long *words, const double *xabs,
                      const float4 *v_in, const int *type_in, const int *pidx_in, float4 *p_out, float4 *v_out,
                      int *type_out, int *pidx_out, double *xref, float4 *xref4, const int *bid_in, int *bid_out,
                      const double *vabs, double *pos_out, double *vel_out, cudaStream_t st, float4 *xrefL4)
{
    k_permute32<<<(n + 255) / 256, 256, 0, st>>>(P, n, words, xabs, v_in, type_in, pidx_in, p_out, v_out, type_out,
                                                 pidx_out, xref, xref4, bid_in, bid_out, vabs, pos_out, vel_out,
                                                 xrefL4);
}
void launch_widen_f(const float *in, double *out, int n, cudaStream_t st)
{
    if (n > 0) k_widen_f<<<(n + 255) / 256, 256, 0, st>>>(in, out, n);
}
void launch_widen_f4(const float4 *in, double *out, int count, int stride, cudaStream_t st)
{
    if (count > 0) k_widen_f4<<<(count + 255) / 256, 256, 0, st>>>(in, out, count, stride);
}

}  // namespace dmph
