// Learned surrogate of K solver steps (no counterpart in the reference).
//
// A surrogate call advances the FP32 split state by K steps at once:
//   1. pass A and pass B at the current state (pressures, forces),
//   2. k_features32: 48 cell-list aggregated features per fluid and debris
//      particle, in one stencil traversal,
//   3. the MLP on the tensor cores (dmph_mlp.cu) predicts, per particle, the
//      K-step velocity increment and the residual of the position increment
//      beyond what the velocity history implies:
//          dv = (y[0:3] a_s + r a0) K dt
//          dx = K dt v0 + (K - 1)/2 dt dv + y[3:6] * (K dt)^2 a_s
//      (exact for a constant acceleration with y[3:6] = 0); a0 is the
//      acceleration of the block start, r = 1 when the network learns the
//      residual on it (default) and 0 when it learns the whole increment,
//   4. k_apply32 moves the fluid particles; debris advance by the solver's
//      own DEM or rigid-body substeps for the K steps with the fluid force of
//      the block start held; walls stay put,
//   5. the usual device-side rebuild decision.
// Training data come from the solver itself: at the start of a K-step block
// the features and (x, v) of every fluid/debris particle are recorded, the
// plain solver runs K steps, and the increments (matched by original id
// across rebuilds) become the targets of a sampled subset, appended to a
// ring-buffer pool.  Every `check_interval` surrogate calls one block runs on
// the plain solver instead, as the judge: the network's prediction of that
// block's velocity increments is compared with what the solver did (relative
// L2, fast particles weighted up), and above `tolerance` the driver falls back
// to the plain solver for `fallback_blocks` blocks, during which it keeps
// collecting samples and training.
#include <math_constants.h>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "dmph_ctx.h"
#include "dmph_mlp.h"
#include "dmph_traverse.cuh"

namespace dmph {

// surge-front histograms over the domain's x extent: 65,536 bins (0.05 mm
// on a 3.3 m domain), finer than the front moves in one block
constexpr int kFrontBins = 1 << 16;
constexpr int kFrontThreads = 1024;

struct FeatScales {
    float inv_vs, inv_as, inv_Ps, inv_W0, inv_dx;
    float vs, as;
    float K, dt;    // substeps, FP32 time step
    float residual; // 1: the network predicts dv - K dt a0 (a0 = acceleration at the block start)
    float ts;       // unit of the velocity-increment outputs (an acceleration): |g| / 16
};

struct Surrogate {
    dmph_surrogate_params prm{};
    MlpParamsDev M;
    int adam_t = 0;
    int n_rows = 0;  // fluid + debris slots
    int n_fluid = 0;
    FeatScales fs{};
    // per-slot buffers (capacity N)
    __nv_bfloat16 *X = nullptr;  // features [N][64]
    float *Y = nullptr;          // outputs [N][16]
    __nv_bfloat16 *H[2] = {nullptr, nullptr};
    float4 *v0 = nullptr;   // start-of-block velocity
    float4 *a0 = nullptr;   // start-of-block acceleration (pass B force / mass)
    double *x0 = nullptr;   // start-of-block absolute position (3 per row)
    int *orig = nullptr;    // start-of-block original id
    int *inv = nullptr;     // original id -> current slot
    // sample pool
    __nv_bfloat16 *poolX = nullptr;
    float *poolT = nullptr;
    long long pool_cap = 0, pool_count = 0;
    unsigned long long *d_cursor = nullptr;
    // training batch
    int B = 0;
    __nv_bfloat16 *Xb = nullptr, *XTb = nullptr, *Hb[3] = {}, *HTb[3] = {}, *dZ[2] = {}, *dZT[2] = {};
    __nv_bfloat16 *dY = nullptr, *dYT = nullptr;
    float *Yb = nullptr, *Tb = nullptr;
    float *d_loss = nullptr;
    int *d_err = nullptr;
    int *d_bad = nullptr;
    double *d_acc = nullptr;  // judge sums
    float *feat32 = nullptr;  // optional FP32 copy of the features (tests)
    std::vector<void *> allocs;
    dmph_surrogate_stats st{};
    int fallback_left = 0;
    int since_check = 0;
    // surge-front judge: histograms of fluid x (predicted, solver), the two
    // fronts, the front at the first call, the accumulated deviation estimate
    unsigned *d_hist = nullptr;
    float *d_histv = nullptr;  // predicted minus solver x-velocity, summed per bin of the solver's positions
    double *d_front = nullptr;
    double front_start = 0.0;
    bool front_start_set = false;
    double front_est = 0.0;
    unsigned long long block_seed = 0;
    // the tail of a surrogate call as one graph: apply the prediction, the
    // debris substeps, the rebuild decision with the rebuild as an IF node
    // (recorded at the first call of each dmph_surrogate_advance)
    cudaGraph_t tail_graph = nullptr;
    cudaGraphExec_t tail_exec = nullptr;
    int *h_bad = nullptr;  // pinned
};

namespace {

constexpr int kFeatWarps = 8;

__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

struct TileF {
    float4 p[kWarp];  // position in the frame of the warp's cell; .w = type
    float4 v[kWarp];  // velocity; .w = pressure
    float4 a[kWarp];  // acceleration of the last force evaluation
};

__device__ __forceinline__ float particle_mass32(const DevParams &P, const DevState &S, int j, int t)
{
    return (float)(particle_density(S, P, j, t) * P.V);
}

// ------------------------------------------------------------ features
// one neighbour j of i (pj in the frame of i's cell, .w = type; vj.w =
// pressure; aj its acceleration) into the feature sums f
__device__ __forceinline__ void feature_pair(const DevParams32 &Q, const float4 pi, const float4 vi, const float *ai,
                                             float Pi, const float4 pj, const float4 vj, const float4 aj, float divi,
                                             float divj, float *f)
{
    const int tj = __float_as_int(pj.w);
    const float q[3] = {pj.x - pi.x, pj.y - pi.y, pj.z - pi.z};
    const float r = sqrtf(fmaf(q[0], q[0], fmaf(q[1], q[1], q[2] * q[2])));
    const float ir = r > 0.f ? 1.f / r : 0.f;
    const float e[3] = {q[0] * ir, q[1] * ir, q[2] * ir};
    const float a = fmaf(-r, Q.iRP, 1.f);
    const float w = a * a;
    const float u[3] = {vj.x - vi.x, vj.y - vi.y, vj.z - vi.z};
    const int cls = is_fluid(tj) ? 0 : (is_solid(tj) ? 1 : 2);
    f[11 + cls] += w;
    for (int d = 0; d < 3; ++d) f[14 + 3 * cls + d] += w * q[d];
    for (int d = 0; d < 3; ++d) f[23 + d] += w * u[d];
    f[26] += w * (aj.x - ai[0]);
    f[27] += w * (aj.y - ai[1]);
    f[28] += w * (aj.z - ai[2]);
    f[29] += w * e[0] * e[0];
    f[30] += w * e[1] * e[1];
    f[31] += w * e[2] * e[2];
    f[32] += w * e[0] * e[1];
    f[33] += w * e[0] * e[2];
    f[34] += w * e[1] * e[2];
    const float ue = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];
    f[35] += w * ue;
    f[36] += w * (e[1] * u[2] - e[2] * u[1]);
    f[37] += w * (e[2] * u[0] - e[0] * u[2]);
    f[38] += w * (e[0] * u[1] - e[1] * u[0]);
    const float dp = vj.w - Pi;
    f[39] += w * dp;
    for (int d = 0; d < 3; ++d) f[40 + d] += w * dp * e[d];
    f[43] += 1.f;
    if (cls == 2)
        for (int d = 0; d < 3; ++d) f[44 + d] += w * u[d];
    f[47] += w * r * Q.iRP;
    // the spread of the velocity divergence around i: the pressure changes at
    // the rate K div, so its gradient is what changes i's pressure force over
    // the coming steps (information two neighbours away)
    const float dd = divj - divi;
    f[48] += w * dd;
    for (int d = 0; d < 3; ++d) f[49 + d] += w * dd * e[d];
}

// own state, normalisation and the BF16 row of slot i
__device__ __forceinline__ void feature_finish(const DevParams32 &Q, const DevState &S, const FeatScales &F, int i,
                                               int ti, const float4 vi, const float *ai, float Pi, float *f,
                                               __nv_bfloat16 *__restrict__ X, float *__restrict__ X32)
{
    f[0] = vi.x * F.inv_vs;
    f[1] = vi.y * F.inv_vs;
    f[2] = vi.z * F.inv_vs;
    f[3] = ai[0] * F.inv_as;
    f[4] = ai[1] * F.inv_as;
    f[5] = ai[2] * F.inv_as;
    f[6] = Pi * F.inv_Ps;
    f[7] = S.vsp32[i] / Q.N0p;
    f[8] = S.div32[i] * Q.dx * F.inv_vs;
    f[9] = is_fluid(ti) ? 1.f : 0.f;
    f[10] = is_solid(ti) ? 1.f : 0.f;
    for (int k = 11; k < 14; ++k) f[k] *= F.inv_W0;
    for (int k = 14; k < 23; ++k) f[k] *= F.inv_W0 * F.inv_dx;
    for (int k = 23; k < 26; ++k) f[k] *= F.inv_W0 * F.inv_vs;
    for (int k = 26; k < 29; ++k) f[k] *= F.inv_W0 * F.inv_as;
    for (int k = 29; k < 35; ++k) f[k] *= F.inv_W0;
    for (int k = 35; k < 39; ++k) f[k] *= F.inv_W0 * F.inv_vs;
    for (int k = 39; k < 43; ++k) f[k] *= F.inv_W0 * F.inv_Ps;
    f[43] *= 0.01f;
    for (int k = 44; k < 47; ++k) f[k] *= F.inv_W0 * F.inv_vs;
    f[47] *= F.inv_W0;
    for (int k = 48; k < 52; ++k) f[k] *= F.inv_W0 * Q.dx * F.inv_vs;
    __align__(16) __nv_bfloat16 h[kMlpIn];
    for (int k = 0; k < kMlpIn; ++k) h[k] = __float2bfloat16_rn(k < kMlpFeatures ? f[k] : 0.f);
    uint4 *dst = reinterpret_cast<uint4 *>(X + (long long)i * kMlpIn);
    for (int k = 0; k < kMlpIn / 8; ++k) dst[k] = reinterpret_cast<const uint4 *>(h)[k];
    if (X32)
        for (int k = 0; k < kMlpFeatures; ++k) X32[(long long)i * kMlpFeatures + k] = f[k];
}

// the 27-cell walk (stencil mode, and after a list overflow: gate)
__global__ void __launch_bounds__(kFeatWarps * kWarp) k_features32(DevParams P, DevParams32 Q, DevState S,
                                                                   const int *dB, FeatScales F,
                                                                   __nv_bfloat16 *__restrict__ X,
                                                                   float *__restrict__ X32, int gate)
{
    if (gate && dB[B_LIST_OVF] == 0) return;
    __shared__ TileF tiles[kFeatWarps];
    TileF &tl = tiles[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    FOR_EACH_CHUNK(dB, CR_FLUID_SOLID, kFeatWarps, cidx)
    {
        const Chunk ch = S.chunks[cidx];
        const int i = ch.i0 + lane;
        const bool active = lane < ch.cnt;
        const int key_cell = (int)(word_key(S.skey[ch.i0]) % (unsigned)P.T);
        const int cix = key_cell / (P.cc[1] * P.cc[2]);
        const int ciy = (key_cell / P.cc[2]) % P.cc[1];
        const int ciz = key_cell % P.cc[2];
        const int ii = active ? i : ch.i0;
        const float4 pi = S.p4[ii];
        const float4 vi = S.v4[ii];
        const int ti = unpack_type(__float_as_uint(pi.w));
        const float mi = particle_mass32(P, S, ii, ti);
        const float4 fi = S.f4[ii];
        const float ai[3] = {fi.x / mi, fi.y / mi, fi.z / mi};
        const float Pi = S.pres32[ii];
        const float divi = S.div32[ii];
        float f[kMlpFeatures];
#pragma unroll
        for (int k = 0; k < kMlpFeatures; ++k) f[k] = 0.f;
        traverse_stencil_batched(
            P, S.cell_start, key_cell, lane, 7u,
            [&](int j, int slot) {
                const float4 pj = S.p4[j];
                const unsigned w = __float_as_uint(pj.w);
                int dx = unpack_cx(w) - cix, dy = unpack_cy(w) - ciy, dz = unpack_cz(w) - ciz;
                dx = dx > 1 ? dx - P.cc[0] : (dx < -1 ? dx + P.cc[0] : dx);
                dy = dy > 1 ? dy - P.cc[1] : (dy < -1 ? dy + P.cc[1] : dy);
                dz = dz > 1 ? dz - P.cc[2] : (dz < -1 ? dz + P.cc[2] : dz);
                const int tj = unpack_type(w);
                tl.p[slot] = make_float4(fmaf((float)dx, Q.cw[0], pj.x), fmaf((float)dy, Q.cw[1], pj.y),
                                         fmaf((float)dz, Q.cw[2], pj.z), __int_as_float(tj));
                float4 vj = S.v4[j];
                vj.w = S.pres32[j];
                tl.v[slot] = vj;
                const float4 fj = S.f4[j];
                const float mj = particle_mass32(P, S, j, tj);
                tl.a[slot] = make_float4(fj.x / mj, fj.y / mj, fj.z / mj, S.div32[j]);
            },
            [&](int base, int nb) {
                if (!active) return;
                unsigned m = 0;
#pragma unroll
                for (int s = 0; s < kWarp; ++s) {
                    const float4 pj = tl.p[s];
                    const float q0 = pj.x - pi.x, q1 = pj.y - pi.y, q2 = pj.z - pi.z;
                    const float r2 = fmaf(q0, q0, fmaf(q1, q1, q2 * q2));
                    m |= (s < nb && r2 < Q.RP2) ? (1u << s) : 0u;
                }
                const int self = i - base;
                if (self >= 0 && self < kWarp) m &= ~(1u << self);
                while (m) {
                    const int s = __ffs(m) - 1;
                    m &= m - 1;
                    feature_pair(Q, pi, vi, ai, Pi, tl.p[s], tl.v[s], tl.a[s], divi, tl.a[s].w, f);
                }
            });
        if (!active) continue;
        feature_finish(Q, S, F, i, ti, vi, ai, Pi, f, X, X32);
    }
}

// Verlet-list mode: one thread per fluid or debris slot over its list (the
// particles within the list radius at the last rebuild, ascending slot; their
// cell offsets in the entries), the pairs within RadiusP taken in list order
__global__ void __launch_bounds__(256) k_features32_list(DevParams P, DevParams32 Q, DevState S, const int *dB,
                                                          FeatScales F, __nv_bfloat16 *__restrict__ X,
                                                          float *__restrict__ X32)
{
    if (dB[B_LIST_OVF]) return;
    const int se = dB[B_SE];
    const long long ld = P.N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < se; i += gridDim.x * blockDim.x) {
        const float4 pi = S.p4[i];
        const int ti = unpack_type(__float_as_uint(pi.w));
        if (is_wall(ti)) continue;  // the slots [0, se) are fluid then debris
        const float4 vi = S.v4[i];
        const float mi = particle_mass32(P, S, i, ti);
        const float4 fi = S.f4[i];
        const float ai[3] = {fi.x / mi, fi.y / mi, fi.z / mi};
        const float Pi = S.pres32[i];
        const float divi = S.div32[i];
        float f[kMlpFeatures];
#pragma unroll
        for (int k = 0; k < kMlpFeatures; ++k) f[k] = 0.f;
        const int cnt = S.nbn[i];
        for (int k = 0; k < cnt; ++k) {
            const unsigned e = __ldg(S.nbl + list_index(k, i, ld));
            const int j = (int)(e & kEntrySlot);
            const float4 pj = __ldg(S.p4 + j);
            const int tj = unpack_type(__float_as_uint(pj.w));
            const float4 pjr = make_float4(fmaf(entry_offset(e, 0), Q.cw[0], pj.x),
                                           fmaf(entry_offset(e, 1), Q.cw[1], pj.y),
                                           fmaf(entry_offset(e, 2), Q.cw[2], pj.z), __int_as_float(tj));
            const float q0 = pjr.x - pi.x, q1 = pjr.y - pi.y, q2 = pjr.z - pi.z;
            if (!(fmaf(q0, q0, fmaf(q1, q1, q2 * q2)) < Q.RP2)) continue;
            float4 vj = __ldg(S.v4 + j);
            vj.w = __ldg(S.pres32 + j);
            const float4 fj = __ldg(S.f4 + j);
            const float mj = particle_mass32(P, S, j, tj);
            feature_pair(Q, pi, vi, ai, Pi, pjr, vj, make_float4(fj.x / mj, fj.y / mj, fj.z / mj, 0.f), divi,
                         __ldg(S.div32 + j), f);
        }
        feature_finish(Q, S, F, i, ti, vi, ai, Pi, f, X, X32);
    }
}

__device__ __forceinline__ void abs_pos(const DevParams &P, const float4 p, double *x)
{
    const unsigned w = __float_as_uint(p.w);
    x[0] = P.dmin[0] + unpack_cx(w) * P.cw[0] + (double)p.x;
    x[1] = P.dmin[1] + unpack_cy(w) * P.cw[1] + (double)p.y;
    x[2] = P.dmin[2] + unpack_cz(w) * P.cw[2] + (double)p.z;
}

// start-of-block record of the fluid/debris slots
__global__ void k_record_start(DevParams P, DevState S, const int *dB, float4 *v0, float4 *a0, double *x0, int *orig)
{
    FOR_EACH_SLOT(dB, -1, B_SE, i)
    {
        const float4 p = S.p4[i];
        double x[3];
        abs_pos(P, p, x);
        for (int d = 0; d < 3; ++d) x0[3 * (long long)i + d] = x[d];
        v0[i] = S.v4[i];
        const float4 f = S.f4[i];
        const float m = particle_mass32(P, S, i, unpack_type(__float_as_uint(p.w)));
        a0[i] = make_float4(f.x / m, f.y / m, f.z / m, 0.f);
        orig[i] = S.pidx[i];
    }
}

__global__ void k_inverse_perm(DevParams P, DevState S, int *inv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.N; i += gridDim.x * blockDim.x) inv[S.pidx[i]] = i;
}

__device__ __forceinline__ double min_image(const DevParams &P, double d, int k)
{
    return d - P.W[k] * rint(d / P.W[k]);
}

// normalised targets of one recorded row (start slot s)
__device__ __forceinline__ void row_targets(const DevParams &P, const DevState &S, const FeatScales &F,
                                            const float4 *v0, const float4 *a0, const double *x0, const int *orig,
                                            const int *inv, int s, float *t, double *dv, double *dx)
{
    const float4 as0 = a0[s];
    const double base[3] = {F.residual * as0.x / F.ts, F.residual * as0.y / F.ts, F.residual * as0.z / F.ts};
    const int j = inv[orig[s]];
    double x1[3];
    abs_pos(P, S.p4[j], x1);
    const float4 v1 = S.v4[j];
    const float4 vs = v0[s];
    dv[0] = (double)v1.x - vs.x;
    dv[1] = (double)v1.y - vs.y;
    dv[2] = (double)v1.z - vs.z;
    const double v0d[3] = {vs.x, vs.y, vs.z};
    const double Kdt = (double)F.K * F.dt;
    for (int d = 0; d < 3; ++d) {
        dx[d] = min_image(P, x1[d] - x0[3 * (long long)s + d], d);
        // clipped at +-2 g: the few particles that strike a wall within the
        // block would otherwise dominate the squared loss
        t[d] = (float)fmin(32.0, fmax(-32.0, dv[d] / (Kdt * F.ts) - base[d]));
        // the displacement follows from the velocity increment (below); its
        // remainder is not learned, so that the loss is the increment's alone
        (void)v0d;
        t[3 + d] = 0.f;
    }
}

// importance of a row: fast particles (the surge front, splashes) are rare
// but decide the front position, so they are kept and judged with a weight
// growing with the squared speed at the block start
__device__ __forceinline__ float row_weight(const FeatScales &F, float4 v)
{
    return 1.f + 20.f * (v.x * v.x + v.y * v.y + v.z * v.z) * F.inv_vs * F.inv_vs;
}

// append a sampled subset of the recorded rows to the pool (ring buffer)
__global__ void k_record_end(DevParams P, DevState S, const int *dB, FeatScales F, const float4 *v0,
                             const float4 *a0, const double *x0, const int *orig, const int *inv,
                             const __nv_bfloat16 *X, __nv_bfloat16 *poolX, float *poolT, unsigned long long *cursor,
                             long long cap, unsigned keep_threshold, unsigned long long seed)
{
    // fluid rows: debris move with the DEM and rigid-body substeps in surrogate blocks
    FOR_EACH_SLOT(dB, -1, B_FE, s)
    {
        const float u = (float)(mix64(seed ^ (unsigned long long)s) >> 40) * (1.f / 16777216.f);
        if (u * 4294967296.f > (float)keep_threshold) continue;  // every fluid row alike
        float t[6];
        double dv[3], dx[3];
        row_targets(P, S, F, v0, a0, x0, orig, inv, s, t, dv, dx);
        bool finite = true;
        for (int k = 0; k < 6; ++k) finite = finite && isfinite(t[k]);
        if (!finite) continue;
        const long long r = (long long)(atomicAdd(cursor, 1ull) % (unsigned long long)cap);
        const uint4 *src = reinterpret_cast<const uint4 *>(X + (long long)s * kMlpIn);
        uint4 *dst = reinterpret_cast<uint4 *>(poolX + r * kMlpIn);
        for (int k = 0; k < kMlpIn / 8; ++k) dst[k] = src[k];
        for (int k = 0; k < kMlpOut; ++k) poolT[r * kMlpOut + k] = k < 6 ? t[k] : 0.f;
    }
}

// judge: prediction of the block (outputs Y of the start features) against
// what the solver did; speed-weighted sums of squares over fluid rows
// bin of an x position among kFrontBins over the domain's x extent (clamped)
__device__ __forceinline__ int front_bin(const DevParams &P, double x)
{
    const int b = (int)floor((x - P.dmin[0]) / P.W[0] * kFrontBins);
    return b < 0 ? 0 : (b >= kFrontBins ? kFrontBins - 1 : b);
}

// hist (kFrontBins each): x of the fluid as the network predicted the block
// (from its start, block-start slots) and as the solver ended it; histv: the
// predicted minus the solver's x-velocity at the block's end, by the bin of
// the solver's position
__global__ void k_judge(DevParams P, DevState S, const int *dB, FeatScales F, const float4 *v0, const float4 *a0,
                        const double *x0, const int *orig, const int *inv, const float *Y, double *acc,
                        unsigned *hist, float *histv)
{
    double e[4] = {0.0, 0.0, 0.0, 0.0};  // |dx err|^2, |dx|^2, |dv err|^2, |dv|^2
    FOR_EACH_SLOT(dB, -1, B_FE, s)
    {
        float t[6];
        double dv[3], dx[3];
        row_targets(P, S, F, v0, a0, x0, orig, inv, s, t, dv, dx);
        const double Kdt = (double)F.K * F.dt;
        const float4 vs = v0[s], as0 = a0[s];
        const double v0d[3] = {vs.x, vs.y, vs.z};
        const double ad[3] = {as0.x, as0.y, as0.z};
        const double wgt = row_weight(F, vs);
        for (int d = 0; d < 3; ++d) {
            const double pdv = ((double)Y[(long long)s * kMlpOut + d] * F.ts + F.residual * ad[d]) * Kdt;
            const double pdx = Kdt * v0d[d] + 0.5 * (F.K - 1.0) * F.dt * pdv;
            e[0] += wgt * (pdx - dx[d]) * (pdx - dx[d]);
            e[1] += wgt * dx[d] * dx[d];
            e[2] += wgt * (pdv - dv[d]) * (pdv - dv[d]);
            e[3] += wgt * dv[d] * dv[d];
            if (d == 0 && hist) {
                const int bs = front_bin(P, x0[3 * (long long)s] + dx[0]);
                atomicAdd(hist + front_bin(P, x0[3 * (long long)s] + pdx), 1u);
                atomicAdd(hist + kFrontBins + bs, 1u);
                atomicAdd(histv + bs, (float)(pdv - dv[0]));
            }
        }
    }
    for (int k = 0; k < 4; ++k) {
        double v = e[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(acc + k, v);
    }
}

// x of the current fluid positions into hist
__global__ void k_front_now(DevParams P, DevState S, const int *dB, unsigned *hist)
{
    FOR_EACH_SLOT(dB, -1, B_FE, s)
    {
        double x[3];
        abs_pos(P, S.p4[s], x);
        atomicAdd(hist + front_bin(P, x[0]), 1u);
    }
}

// the surge front of histogram blockIdx.x: the upper edge of the bin below
// which 99% of the counted fluid lies (each thread sums a run of bins, one
// thread walks the run sums from the top, then the run that holds the
// quantile bin by bin).  With histv (the second histogram only): front[2] =
// the mean of histv over the front's 1% (bins from the quantile bin up)
__global__ void __launch_bounds__(kFrontThreads) k_front_quantiles(const DevParams P, const unsigned *hist,
                                                                  double *front, const float *histv)
{
    constexpr int kRun = kFrontBins / kFrontThreads;
    __shared__ unsigned long long run[kFrontThreads];
    __shared__ double runv[kFrontThreads];
    const unsigned *c = hist + (long long)blockIdx.x * kFrontBins;
    const bool vel = histv && blockIdx.x == 1;
    unsigned long long sum = 0;
    double sv = 0.0;
    for (int b = 0; b < kRun; ++b) {
        sum += c[threadIdx.x * kRun + b];
        if (vel) sv += histv[threadIdx.x * kRun + b];
    }
    run[threadIdx.x] = sum;
    runv[threadIdx.x] = sv;
    __syncthreads();
    if (threadIdx.x != 0) return;
    unsigned long long total = 0;
    for (int r = 0; r < kFrontThreads; ++r) total += run[r];
    const unsigned long long beyond = total / 100;  // the 1% furthest downstream
    unsigned long long acc = 0;
    int r = kFrontThreads - 1;
    double accv = 0.0;
    for (; r > 0 && acc + run[r] <= beyond; --r) {
        acc += run[r];
        accv += runv[r];
    }
    int b = (r + 1) * kRun - 1;
    for (; b > r * kRun; --b) {
        acc += c[b];
        if (vel) accv += histv[b];
        if (acc > beyond) break;
    }
    if (b == r * kRun) {  // the run's lowest bin holds the quantile
        acc += c[b];
        if (vel) accv += histv[b];
    }
    front[blockIdx.x] = P.dmin[0] + (double)(b + 1) * P.W[0] / kFrontBins;
    if (vel) front[2] = acc > 0 ? accv / (double)acc : 0.0;
}

// every prediction of the rows that will be applied is finite
__global__ void k_check_finite(const int *dB, const float *Y, int solids_too, int *bad)
{
    FOR_EACH_SLOT(dB, -1, solids_too ? B_SE : B_FE, i)
    {
        for (int k = 0; k < kMlpTargets; ++k)
            if (!isfinite(Y[(long long)i * kMlpOut + k])) atomicExch(bad, 1);
    }
}

// apply the prediction to the fluid slots (and to individual debris
// particles when they are not rigid bodies)
__global__ void k_apply32(DevParams P, DevState S, const int *dB, FeatScales F, const float *Y, int solids_too,
                          int *bad)
{
    const int N = P.N;
    const int end_key = solids_too ? B_SE : B_FE;
    FOR_EACH_SLOT(dB, -1, end_key, i)
    {
        const float *y = Y + (long long)i * kMlpOut;
        const float Kdt = F.K * F.dt;
        float4 p = S.p4[i];
        float4 v = S.v4[i];
        float ab[3] = {0.f, 0.f, 0.f};
        if (F.residual != 0.f) {
            const float4 f = S.f4[i];
            const float m = particle_mass32(P, S, i, unpack_type(__float_as_uint(p.w)));
            ab[0] = f.x / m;
            ab[1] = f.y / m;
            ab[2] = f.z / m;
        }
        const float dvx = (y[0] * F.ts + ab[0]) * Kdt, dvy = (y[1] * F.ts + ab[1]) * Kdt,
                    dvz = (y[2] * F.ts + ab[2]) * Kdt;
        // K steps of x += v dt with v growing by dv / K a step
        const float h = 0.5f * (F.K - 1.f) * F.dt;
        const float dxx = Kdt * v.x + h * dvx;
        const float dxy = Kdt * v.y + h * dvy;
        const float dxz = Kdt * v.z + h * dvz;
        if (!(isfinite(dxx) && isfinite(dxy) && isfinite(dxz) && isfinite(dvx) && isfinite(dvy) && isfinite(dvz))) {
            atomicExch(bad, 1);
            continue;
        }
        const int t = unpack_type(__float_as_uint(p.w));
        if (is_fluid(t)) {
            p.x += dxx;
            p.y += dxy;
            p.z += dxz;
            v.x += dvx;
            v.y += dvy;
            v.z += dvz;
            S.p4[i] = p;
            S.v4[i] = v;
        } else {
            // debris without rigid bodies: FP64 master state, then the FP32 copy
            const double dxd[3] = {dxx, dxy, dxz}, dvd[3] = {dvx, dvy, dvz};
            for (int d = 0; d < 3; ++d) {
                const double a = S.pos[d * N + i] + dxd[d] - P.dmin[d];
                S.pos[d * N + i] = (a - P.W[d] * floor(a / P.W[d])) + P.dmin[d];
                S.vel[d * N + i] += dvd[d];
            }
        }
    }
}

// largest displacement since the last rebuild (FP32 frame), for the decision
__global__ void k_maxshift32(DevParams P, DevState S, unsigned long long *maxshift)
{
    float m2 = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.N; i += gridDim.x * blockDim.x) {
        const float4 p = S.p4[i], r = S.xref4[i];
        const float dx = p.x - r.x, dy = p.y - r.y, dz = p.z - r.z;
        m2 = fmaxf(m2, fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        if (!isfinite(p.x + p.y + p.z)) m2 = CUDART_INF_F;  // reported by the decision, no rebuild
    }
    unsigned long long b = __double_as_longlong((double)m2);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_down_sync(kFull, b, o);
        b = ob > b ? ob : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(maxshift, b);
}

// minibatch of pool rows: row-major and transposed features, targets
__global__ void k_gather_batch(const __nv_bfloat16 *poolX, const float *poolT, long long count, int B,
                               unsigned long long seed, __nv_bfloat16 *Xb, __nv_bfloat16 *XTb, float *Tb)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
        const long long r = (long long)(mix64(seed ^ (unsigned long long)i * 0x9E3779B97F4A7C15ull) %
                                        (unsigned long long)count);
        const __nv_bfloat16 *src = poolX + r * kMlpIn;
        for (int k = 0; k < kMlpIn; ++k) {
            const __nv_bfloat16 h = src[k];
            Xb[(long long)i * kMlpIn + k] = h;
            XTb[(long long)k * B + i] = h;
        }
        for (int k = 0; k < kMlpOut; ++k) Tb[(long long)i * kMlpOut + k] = poolT[r * kMlpOut + k];
    }
}

template <class T>
int salloc(dmph_ctx *ctx, Surrogate *s, T **p, size_t count)
{
    if (cudaMalloc((void **)p, count * sizeof(T) + 16) != cudaSuccess) {
        ctx->err = "surrogate: device allocation failed";
        return DMPH_ENOMEM;
    }
    cudaMemset(*p, 0, count * sizeof(T) + 16);
    s->allocs.push_back(*p);
    return DMPH_OK;
}

#define SA(ptr, n)                                \
    do {                                          \
        const int rc_ = salloc(ctx, s, &(ptr), (n)); \
        if (rc_) return rc_;                      \
    } while (0)

// ---------------------------------------------------------- MLP driver
GemmArgs gemm(const __nv_bfloat16 *A, long long lda, const __nv_bfloat16 *B, long long ldb, long long M, int N,
              long long K, int epi, int *err)
{
    GemmArgs g;
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.M = M;
    g.N = N;
    g.K = K;
    g.epi = epi;
    g.err = err;
    return g;
}

// forward over rows [0, n) of X (row-major [n][64]) into Y [n][16]: the
// fused kernel (dmph_mlp.cu, k_mlp_fwd)
int mlp_forward(dmph_ctx *ctx, Surrogate *s, const __nv_bfloat16 *X, long long n, float *Y, cudaStream_t st)
{
    const int rc = launch_mlp_forward(s->M, X, n, Y, s->d_err, ctx->sms, st);
    if (rc) {
        ctx->err = "surrogate: the fused MLP's tensor map could not be made (" + std::to_string(rc) + ")";
        return DMPH_ECUDA;
    }
    return DMPH_OK;
}

// the same through one GEMM per layer (the training path's forward kernels;
// dmph_mlp_forward_layers compares the two)
void mlp_forward_layers(Surrogate *s, const __nv_bfloat16 *X, long long n, float *Y, cudaStream_t st)
{
    const MlpParamsDev &M = s->M;
    const __nv_bfloat16 *in = X;
    long long ld = kMlpIn;
    for (int l = 0; l < 3; ++l) {
        GemmArgs g = gemm(in, ld, M.wb[l], M.in[l], n, kMlpHidden, M.in[l], EPI_RELU, s->d_err);
        g.bias = M.w + M.boff[l];
        g.outB = s->H[l & 1];
        g.ldo = kMlpHidden;
        launch_gemm(g, 1, st);
        in = s->H[l & 1];
        ld = kMlpHidden;
    }
    GemmArgs g = gemm(in, ld, M.wb[3], kMlpHidden, n, kMlpOut, kMlpHidden, EPI_OUT, s->d_err);
    g.bias = M.w + M.boff[3];
    g.outF = Y;
    g.ldo = kMlpOut;
    launch_gemm(g, 1, st);
}

// loss and gradient of the batch in Xb/XTb/Tb (B rows) into M.grad
void mlp_backprop(Surrogate *s, cudaStream_t st)
{
    const MlpParamsDev &M = s->M;
    const long long B = s->B;
    const int ks = (int)(B / 1024);
    cudaMemsetAsync(s->d_loss, 0, sizeof(float), st);
    const __nv_bfloat16 *in = s->Xb;
    long long ld = kMlpIn;
    for (int l = 0; l < 3; ++l) {
        GemmArgs g = gemm(in, ld, M.wb[l], M.in[l], B, kMlpHidden, M.in[l], EPI_RELU, s->d_err);
        g.bias = M.w + M.boff[l];
        g.outB = s->Hb[l];
        g.ldo = kMlpHidden;
        g.outT = s->HTb[l];
        g.ldT = B;
        launch_gemm(g, 1, st);
        in = s->Hb[l];
        ld = kMlpHidden;
    }
    {
        GemmArgs g = gemm(s->Hb[2], kMlpHidden, M.wb[3], kMlpHidden, B, kMlpOut, kMlpHidden, EPI_OUT, s->d_err);
        g.bias = M.w + M.boff[3];
        g.outF = s->Yb;
        g.ldo = kMlpOut;
        g.target = s->Tb;
        g.ldt = kMlpOut;
        g.n_valid = kMlpTargets;
        g.grad_scale = 2.f / (float)(B * kMlpTargets);
        g.loss = s->d_loss;
        g.outB = s->dY;
        g.outT = s->dYT;
        g.ldT = B;
        launch_gemm(g, 1, st);
    }
    // layer 4: dW4^T = H3^T dY, db4, dZ3 = (dY W4) * [H3 > 0]
    {
        GemmArgs g = gemm(s->HTb[2], B, s->dYT, B, kMlpHidden, kMlpOut, B, EPI_WGRAD, s->d_err);
        g.outF = M.grad + M.woff[3];
        g.ldo = kMlpHidden;
        g.transpose_out = 1;
        launch_gemm(g, ks, st);
        launch_row_sums(s->dYT, B, kMlpOut, (int)B, M.grad + M.boff[3], st);
        GemmArgs h = gemm(s->dY, kMlpOut, M.wt[3], kMlpOut, B, kMlpHidden, kMlpOut, EPI_BWD_RELU, s->d_err);
        h.mask = s->Hb[2];
        h.ldm = kMlpHidden;
        h.outB = s->dZ[0];
        h.ldo = kMlpHidden;
        h.outT = s->dZT[0];
        h.ldT = B;
        launch_gemm(h, 1, st);
    }
    // hidden layers 3, 2, 1
    int cur = 0;
    for (int l = 2; l >= 0; --l) {
        const __nv_bfloat16 *act_T = l > 0 ? s->HTb[l - 1] : s->XTb;
        const int nin = M.in[l];
        GemmArgs g = gemm(s->dZT[cur], B, act_T, B, kMlpHidden, nin, B, EPI_WGRAD, s->d_err);
        g.outF = M.grad + M.woff[l];
        g.ldo = nin;
        launch_gemm(g, ks, st);
        launch_row_sums(s->dZT[cur], B, kMlpHidden, (int)B, M.grad + M.boff[l], st);
        if (l == 0) break;
        GemmArgs h = gemm(s->dZ[cur], kMlpHidden, M.wt[l], kMlpHidden, B, kMlpHidden, kMlpHidden, EPI_BWD_RELU,
                          s->d_err);
        h.mask = s->Hb[l - 1];
        h.ldm = kMlpHidden;
        h.outB = s->dZ[cur ^ 1];
        h.ldo = kMlpHidden;
        h.outT = s->dZT[cur ^ 1];
        h.ldT = B;
        launch_gemm(h, 1, st);
        cur ^= 1;
    }
}

void feat_scales(dmph_ctx *ctx, Surrogate *s)
{
    const dmph_params &p = ctx->p;
    const double rho = p.density[1] > 0 ? p.density[1] : 1000.0;
    const double c0 = p.bulk_modulus[1] > 0 ? std::sqrt(p.bulk_modulus[1] / rho) : 10.0;
    const double vs = c0 / 10.0;
    const double g = std::sqrt(p.gravity[0] * p.gravity[0] + p.gravity[1] * p.gravity[1] + p.gravity[2] * p.gravity[2]);
    const double as = g > 0 ? g : 1.0;
    const double W0 = ctx->Q.N0p32 / ctx->Q.Bp;
    FeatScales &F = s->fs;
    F.vs = (float)vs;
    F.as = (float)as;
    F.ts = (float)(as / 16.0);
    F.inv_vs = (float)(1.0 / vs);
    F.inv_as = (float)(1.0 / as);
    F.inv_Ps = (float)(1.0 / (rho * vs * vs));
    F.inv_W0 = (float)(1.0 / W0);
    F.inv_dx = (float)(1.0 / ctx->P.dx);
    F.K = (float)s->prm.substeps;
    F.residual = s->prm.residual ? 1.f : 0.f;
    F.dt = (float)ctx->P.dt;
}

int grid_slots(const dmph_ctx *ctx) { return ctx->sms * 4; }

// pass A, pass B and the features at the current state
void enqueue_features(dmph_ctx *ctx, Surrogate *s, float *x32, cudaStream_t st)
{
    enqueue_pair_passes32(ctx, st);
    if (ctx->use_list) {
        static const int gl = persistent_grid((const void *)k_features32_list, 256);
        k_features32_list<<<gl, 256, 0, st>>>(ctx->P, ctx->Q, ctx->S, ctx->dB, s->fs, s->X, x32);
    }
    static const int g = persistent_grid((const void *)k_features32, kFeatWarps * kWarp);
    k_features32<<<g, kFeatWarps * kWarp, 0, st>>>(ctx->P, ctx->Q, ctx->S, ctx->dB, s->fs, s->X, x32,
                                                   ctx->use_list ? 1 : 0);
}

int check_err(dmph_ctx *ctx, Surrogate *s)
{
    int e = 0;
    CK(cudaMemcpyAsync(&e, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (e) {
        ctx->err = "surrogate: a tensor-core wait ran out";
        return DMPH_ETIMEOUT;
    }
    return DMPH_OK;
}

// one block of K plain steps that records samples (and, with judge, scores
// the network's prediction of the same block)
int plain_block(dmph_ctx *ctx, Surrogate *s, bool judge, double *ex, double *ev, double *fronts = nullptr)
{
    cudaStream_t st = ctx->st;
    enqueue_features(ctx, s, nullptr, st);
    const int gs = grid_slots(ctx);
    k_record_start<<<gs, 256, 0, st>>>(ctx->P, ctx->S, ctx->dB, s->v0, s->a0, s->x0, s->orig);
    if (judge) {
        const int rc = mlp_forward(ctx, s, s->X, s->n_rows, s->Y, st);
        if (rc) return rc;
    }
    CK(cudaGetLastError());
    for (int k = 0; k < s->prm.substeps; ++k) {
        const int rc = step_once(ctx);
        if (rc) return rc;
    }
    k_inverse_perm<<<gs, 256, 0, st>>>(ctx->P, ctx->S, s->inv);
    if (judge) {
        CK(cudaMemsetAsync(s->d_acc, 0, 4 * sizeof(double), st));
        CK(cudaMemsetAsync(s->d_hist, 0, 2 * kFrontBins * sizeof(unsigned), st));
        CK(cudaMemsetAsync(s->d_histv, 0, kFrontBins * sizeof(float), st));
        k_judge<<<gs, 256, 0, st>>>(ctx->P, ctx->S, ctx->dB, s->fs, s->v0, s->a0, s->x0, s->orig, s->inv, s->Y,
                                    s->d_acc, s->d_hist, s->d_histv);
        k_front_quantiles<<<2, kFrontThreads, 0, st>>>(ctx->P, s->d_hist, s->d_front, s->d_histv);
    }
    // keep about pool/16 rows of every block
    const double keep = std::min(1.0, (double)s->pool_cap / 16.0 / std::max(1, s->n_fluid));
    const unsigned thr = (unsigned)std::min(4294967295.0, keep * 4294967296.0);
    k_record_end<<<gs, 256, 0, st>>>(ctx->P, ctx->S, ctx->dB, s->fs, s->v0, s->a0, s->x0, s->orig, s->inv, s->X,
                                     s->poolX,
                                     s->poolT, s->d_cursor, s->pool_cap, thr, s->block_seed++ * 0x632BE59BD9B4E019ull);
    CK(cudaGetLastError());
    unsigned long long cur = 0;
    double acc[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(&cur, s->d_cursor, sizeof(cur), cudaMemcpyDeviceToHost, st));
    double fr[3] = {0.0, 0.0, 0.0};
    if (judge) {
        CK(cudaMemcpyAsync(acc, s->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(fr, s->d_front, sizeof(fr), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    s->pool_count = std::min<long long>((long long)cur, s->pool_cap);
    s->st.samples = (int64_t)cur;
    s->st.plain_blocks++;
    if (judge) {
        *ex = std::sqrt(acc[0] / std::max(acc[1], 1e-300));
        *ev = std::sqrt(acc[2] / std::max(acc[3], 1e-300));
        if (fronts) {
            fronts[0] = fr[0];  // front of the network's prediction of the block
            fronts[1] = fr[1];  // the solver's
            fronts[2] = fr[2];  // mean x-velocity error of the front's fluid
        }
    }
    return check_err(ctx, s);
}

int train(dmph_ctx *ctx, Surrogate *s, int iters, float *loss_out)
{
    if (s->pool_count < s->B / 4) {
        ctx->err = "surrogate: too few samples to train (collect first)";
        return DMPH_EINVAL;
    }
    cudaStream_t st = ctx->st;
    float loss = 0.f;
    for (int it = 0; it < iters; ++it) {
        k_gather_batch<<<ctx->sms * 4, 256, 0, st>>>(s->poolX, s->poolT, s->pool_count, s->B,
                                                     0xA5A5ull + (unsigned long long)s->st.train_iters * 0x9E37ull,
                                                     s->Xb, s->XTb, s->Tb);
        mlp_backprop(s, st);
        s->adam_t++;
        launch_adam(s->M, s->prm.learning_rate, s->adam_t, st);
        launch_weights_to_bf16(s->M, st);
        CK(cudaGetLastError());
        s->st.train_iters++;
    }
    CK(cudaMemcpyAsync(&loss, s->d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    const int rc = check_err(ctx, s);
    if (rc) return rc;
    loss /= (float)((double)s->B * kMlpTargets);  // mean squared error of the last batch
    s->st.last_loss = loss;
    if (loss_out) *loss_out = loss;
    return DMPH_OK;
}

void drop_tail(Surrogate *s)
{
    if (s->tail_exec) cudaGraphExecDestroy(s->tail_exec);
    if (s->tail_graph) cudaGraphDestroy(s->tail_graph);
    s->tail_exec = nullptr;
    s->tail_graph = nullptr;
}

// the part of a surrogate call after the prediction was found finite: apply
// it to the fluid, advance the debris by the solver's own DEM or rigid-body
// substeps with the fluid force of the block start held, clear the forces as
// a drift would, and take the reference's rebuild decision on the device
void enqueue_tail_ops(dmph_ctx *ctx, Surrogate *s, unsigned long long cond, cudaStream_t st)
{
    const int gs = grid_slots(ctx);
    k_apply32<<<gs, 256, 0, st>>>(ctx->P, ctx->S, ctx->dB, s->fs, s->Y, 0, s->d_bad);
    if (s->n_rows > s->n_fluid) enqueue_dem_block(ctx, s->prm.substeps, st);
    cudaMemsetAsync(ctx->S.f4, 0, sizeof(float4) * (size_t)ctx->P.N, st);
    cudaMemsetAsync(ctx->maxshift, 0, sizeof(unsigned long long), st);
    k_maxshift32<<<gs, 256, 0, st>>>(ctx->P, ctx->S, ctx->maxshift);
    launch_decide(ctx->P, ctx->maxshift, ctx->dB, cond, st);
}

int capture_tail(dmph_ctx *ctx, Surrogate *s)
{
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    CK(cudaStreamBeginCaptureToGraph(ctx->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_tail_ops(ctx, s, (unsigned long long)cond, ctx->st);
    int rc = capture_rebuild_if(ctx, cond, ctx->st);
    cudaGraph_t g2 = g;
    const cudaError_t ce = cudaStreamEndCapture(ctx->st, &g2);
    if (rc || ce != cudaSuccess) {
        cudaGraphDestroy(g);
        if (!rc) ctx->err = std::string("surrogate tail capture: ") + cudaGetErrorString(ce);
        return rc ? rc : DMPH_ECUDA;
    }
    CK(cudaGraphInstantiate(&s->tail_exec, g, 0));
    s->tail_graph = g;
    return DMPH_OK;
}

// one surrogate call: K steps of simulated time.  One host synchronisation:
// whether every prediction is finite (a non-finite one leaves the state
// untouched and sends the driver back to the plain solver); the rest runs as
// the recorded tail graph, whose rebuild decision is taken on the device.
int surrogate_block(dmph_ctx *ctx, Surrogate *s)
{
    cudaStream_t st = ctx->st;
    enqueue_features(ctx, s, nullptr, st);
    {
        const int rc = mlp_forward(ctx, s, s->X, s->n_fluid, s->Y, st);
        if (rc) return rc;
    }
    CK(cudaMemsetAsync(s->d_bad, 0, sizeof(int), st));
    const int gs = grid_slots(ctx);
    k_check_finite<<<gs, 256, 0, st>>>(ctx->dB, s->Y, 0, s->d_bad);
    CK(cudaMemcpyAsync(s->h_bad, s->d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (*s->h_bad) {
        ctx->err = "surrogate: non-finite prediction";
        return DMPH_ENAN;
    }
    if (ctx->prof) {
        // phase timing synchronises inside the DEM phase: no recorded graph
        enqueue_tail_ops(ctx, s, 0, st);
        CK(cudaMemcpyAsync(s->h_bad, ctx->dB + B_NEED, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (*s->h_bad) {
            enqueue_rebuild(ctx, false, st);
            ctx->launches += rebuild_launches(ctx, false);
            ctx->host_rebuilds++;
        }
    } else {
        if (!s->tail_exec) {
            const int rc = capture_tail(ctx, s);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(s->tail_exec, st));
    }
    // pair passes (list mode: 5, stencil: 2), features (list mode: 2), 4
    // GEMMs, check, apply, maxshift, decide; the rebuilds the graph runs are
    // counted by the device's rebuild counter
    ctx->launches += (ctx->use_list ? 15 : 11) + (s->n_rows > s->n_fluid ? dem_block_launches(ctx, s->prm.substeps) : 0);
    for (int k = 0; k < s->prm.substeps; ++k) advance_host_clock(ctx);
    s->st.calls++;
    return DMPH_OK;
}

// the walls never move when every wall type has zero velocity and spin and
// an identity rotation (then the moving-wall window changes nothing)
bool walls_static(const dmph_ctx *ctx)
{
    const WallMotion &W = ctx->Wm;
    for (int t = DMPH_WALL_BEGIN; t < DMPH_WALL_END; ++t)
        for (int a = 0; a < 3; ++a) {
            if (W.Vel[t][a] != 0.0 || W.Om[t][a] != 0.0) return false;
            for (int b = 0; b < 3; ++b)
                if (W.R[t][a][b] != (a == b ? 1.0 : 0.0)) return false;
        }
    return true;
}

bool surrogate_allowed(const dmph_ctx *ctx, const Surrogate *s)
{
    // the first step (wall centres move while Time <= 0) and blocks that reach
    // into the window of moving walls run plain
    const double t1 = ctx->time + s->prm.substeps * ctx->P.dt;
    if (!(0.0 < ctx->time)) return false;
    return walls_static(ctx) || !(t1 >= 0.2 && 0.4 >= ctx->time);
}

}  // namespace

void surrogate_release(dmph_ctx *ctx)
{
    Surrogate *s = ctx->sg;
    if (!s) return;
    drop_tail(s);
    if (s->h_bad) cudaFreeHost(s->h_bad);
    for (void *p : s->allocs) cudaFree(p);
    delete s;
    ctx->sg = nullptr;
}

}  // namespace dmph

// ================================================================ C ABI
extern "C" int dmph_surrogate_params_default(dmph_surrogate_params *p)
{
    if (!p) return DMPH_EINVAL;
    p->substeps = 8;
    p->check_interval = 50;
    p->tolerance = 0.02;
    p->fallback_blocks = 50;
    p->train_iters_per_block = 4;
    p->batch = 65536;
    p->pool_rows = 1 << 22;
    p->learning_rate = 1e-3f;
    p->seed = 1234;
    p->residual = 1;
    p->front_tolerance = 0.0;
    return DMPH_OK;
}

extern "C" int dmph_surrogate_enable(dmph_ctx *ctx, const dmph_surrogate_params *prm)
{
    using namespace dmph;
    if (!ctx || !prm) return DMPH_EINVAL;
    if (!ctx->fp32) {
        ctx->err = "the surrogate runs on the FP32 split build";
        return DMPH_EINVAL;
    }
    if (ctx->list_reuse) {
        ctx->err = "the surrogate does not run with list reuse (DMPH_FLAG_LIST_REUSE)";
        return DMPH_EINVAL;
    }
    if (prm->substeps < 1 || prm->check_interval < 1 || prm->batch < 8192 || prm->batch % 8192 ||
        prm->pool_rows < prm->batch || !(prm->tolerance > 0 || prm->front_tolerance > 0) ||
        !(prm->front_tolerance >= 0) || prm->fallback_blocks < 1) {
        ctx->err = "surrogate parameters out of range (batch a multiple of 8192, pool >= batch)";
        return DMPH_ERANGE;
    }
    surrogate_release(ctx);
    Surrogate *s = new Surrogate();
    ctx->sg = s;
    s->prm = *prm;
    const long long N = ctx->P.N;
    int b[B_COUNT];
    int rc = read_bounds(ctx, b);
    if (rc) return rc;
    s->n_rows = b[B_SE];
    s->n_fluid = b[B_FE];
    // parameters
    MlpParamsDev &M = s->M;
    const int ins[4] = {kMlpIn, kMlpHidden, kMlpHidden, kMlpHidden};
    const int outs[4] = {kMlpHidden, kMlpHidden, kMlpHidden, kMlpOut};
    int off = 0;
    for (int l = 0; l < 4; ++l) {
        M.in[l] = ins[l];
        M.out[l] = outs[l];
        M.woff[l] = off;
        off += ins[l] * outs[l];
        M.boff[l] = off;
        off += outs[l];
    }
    M.count = off;
    SA(M.w, off);
    SA(M.m, off);
    SA(M.v, off);
    SA(M.grad, off);
    for (int l = 0; l < 4; ++l) {
        SA(M.wb[l], (size_t)ins[l] * outs[l]);
        SA(M.wt[l], (size_t)ins[l] * outs[l]);
    }
    // He-uniform initial weights (mt19937_64 from the seed), output layer x0.1, zero biases
    std::vector<float> w(off, 0.f);
    std::mt19937_64 rng(prm->seed);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    for (int l = 0; l < 4; ++l) {
        const float a = std::sqrt(6.f / (float)(l == 0 ? kMlpFeatures : ins[l])) * (l == 3 ? 0.1f : 1.f);
        for (int o = 0; o < outs[l]; ++o)
            for (int k = 0; k < ins[l]; ++k)
                w[M.woff[l] + o * ins[l] + k] = (l == 0 && k >= kMlpFeatures) ? 0.f : a * U(rng);
    }
    CK(cudaMemcpy(M.w, w.data(), sizeof(float) * off, cudaMemcpyHostToDevice));
    launch_weights_to_bf16(M, ctx->st);
    // buffers
    SA(s->X, (size_t)N * kMlpIn);
    SA(s->Y, (size_t)N * kMlpOut);
    SA(s->H[0], (size_t)N * kMlpHidden);
    SA(s->H[1], (size_t)N * kMlpHidden);
    SA(s->v0, (size_t)N);
    SA(s->a0, (size_t)N);
    SA(s->x0, (size_t)N * 3);
    SA(s->orig, (size_t)N);
    SA(s->inv, (size_t)N);
    s->pool_cap = prm->pool_rows;
    SA(s->poolX, (size_t)s->pool_cap * kMlpIn);
    SA(s->poolT, (size_t)s->pool_cap * kMlpOut);
    SA(s->d_cursor, 1);
    s->B = prm->batch;
    const size_t B = (size_t)s->B;
    SA(s->Xb, B * kMlpIn);
    SA(s->XTb, B * kMlpIn);
    for (int l = 0; l < 3; ++l) {
        SA(s->Hb[l], B * kMlpHidden);
        SA(s->HTb[l], B * kMlpHidden);
    }
    for (int l = 0; l < 2; ++l) {
        SA(s->dZ[l], B * kMlpHidden);
        SA(s->dZT[l], B * kMlpHidden);
    }
    SA(s->dY, B * kMlpOut);
    SA(s->dYT, B * kMlpOut);
    SA(s->Yb, B * kMlpOut);
    SA(s->Tb, B * kMlpOut);
    SA(s->d_loss, 1);
    SA(s->d_err, 1);
    SA(s->d_bad, 1);
    SA(s->d_acc, 4);
    SA(s->d_hist, 2 * kFrontBins);
    SA(s->d_histv, kFrontBins);
    SA(s->d_front, 4);
    CK(cudaMallocHost(&s->h_bad, sizeof(int)));
    feat_scales(ctx, s);
    CK(cudaStreamSynchronize(ctx->st));
    drop_graph(ctx);
    return DMPH_OK;
}

static dmph::Surrogate *need_sg(dmph_ctx *ctx)
{
    if (!ctx) return nullptr;
    if (!ctx->sg) ctx->err = "surrogate not enabled (dmph_surrogate_enable)";
    return ctx->sg;
}

extern "C" int dmph_surrogate_collect(dmph_ctx *ctx, int nblocks)
{
    dmph::Surrogate *s = need_sg(ctx);
    if (!s) return DMPH_EINVAL;
    for (int k = 0; k < nblocks; ++k) {
        const int rc = dmph::plain_block(ctx, s, false, nullptr, nullptr);
        if (rc) return rc;
    }
    return DMPH_OK;
}

// the training pool's rows (features as recorded, BF16 widened to FP32;
// targets), oldest first once the ring has wrapped
extern "C" int dmph_surrogate_get_samples(dmph_ctx *ctx, float *X, float *T, int capacity, int *rows)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s || capacity < 0 || (capacity > 0 && (!X || !T))) return DMPH_EINVAL;
    unsigned long long cur = 0;
    CK(cudaMemcpyAsync(&cur, s->d_cursor, sizeof(cur), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    const long long count = std::min<long long>((long long)cur, s->pool_cap);
    const long long n = std::min<long long>(count, capacity);
    // the ring's oldest row is at cur % cap once it has wrapped
    const long long start = (long long)cur > s->pool_cap ? (long long)(cur % (unsigned long long)s->pool_cap) : 0;
    std::vector<__nv_bfloat16> xb((size_t)n * kMlpIn);
    for (long long done = 0; done < n;) {
        const long long r0 = (start + done) % s->pool_cap;
        const long long len = std::min(n - done, s->pool_cap - r0);
        CK(cudaMemcpyAsync(xb.data() + done * kMlpIn, s->poolX + r0 * kMlpIn, sizeof(__nv_bfloat16) * len * kMlpIn,
                           cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(T + done * kMlpOut, s->poolT + r0 * kMlpOut, sizeof(float) * len * kMlpOut,
                           cudaMemcpyDeviceToHost, ctx->st));
        done += len;
    }
    CK(cudaStreamSynchronize(ctx->st));
    for (size_t i = 0; i < xb.size(); ++i) X[i] = __bfloat162float(xb[i]);
    if (rows) *rows = (int)n;
    return DMPH_OK;
}

// append rows to the training pool's ring (features rounded to BF16), as if
// recorded: samples from other scenes for a training corpus
extern "C" int dmph_surrogate_add_samples(dmph_ctx *ctx, const float *X, const float *T, int n)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s || n < 0 || (n > 0 && (!X || !T))) return DMPH_EINVAL;
    if (n == 0) return DMPH_OK;
    unsigned long long cur = 0;
    CK(cudaMemcpyAsync(&cur, s->d_cursor, sizeof(cur), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::vector<__nv_bfloat16> xb((size_t)n * kMlpIn);
    for (size_t i = 0; i < xb.size(); ++i) xb[i] = __float2bfloat16_rn(X[i]);
    // rows beyond the capacity only overwrite earlier ones: keep the last cap
    const long long skip = n > s->pool_cap ? n - s->pool_cap : 0;
    for (long long done = skip; done < n;) {
        const long long r0 = (long long)((cur + (unsigned long long)done) % (unsigned long long)s->pool_cap);
        const long long len = std::min(n - done, s->pool_cap - r0);
        CK(cudaMemcpyAsync(s->poolX + r0 * kMlpIn, xb.data() + done * kMlpIn, sizeof(__nv_bfloat16) * len * kMlpIn,
                           cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(s->poolT + r0 * kMlpOut, T + done * kMlpOut, sizeof(float) * len * kMlpOut,
                           cudaMemcpyHostToDevice, ctx->st));
        done += len;
    }
    cur += (unsigned long long)n;
    CK(cudaMemcpyAsync(s->d_cursor, &cur, sizeof(cur), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    s->pool_count = std::min<long long>((long long)cur, s->pool_cap);
    s->st.samples = (int64_t)cur;
    return DMPH_OK;
}

extern "C" int dmph_surrogate_train(dmph_ctx *ctx, int iters, float *loss)
{
    dmph::Surrogate *s = need_sg(ctx);
    if (!s) return DMPH_EINVAL;
    return dmph::train(ctx, s, iters, loss);
}

extern "C" int dmph_surrogate_advance(dmph_ctx *ctx, int nblocks)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s) return DMPH_EINVAL;
    drop_tail(s);  // recorded again with the context's current settings
    drop_graph(ctx);
    if (s->prm.front_tolerance > 0 && !s->front_start_set) {
        // the front the travel is measured from: at the first call
        CK(cudaMemsetAsync(s->d_hist, 0, kFrontBins * sizeof(unsigned), ctx->st));
        k_front_now<<<grid_slots(ctx), 256, 0, ctx->st>>>(ctx->P, ctx->S, ctx->dB, s->d_hist);
        k_front_quantiles<<<1, kFrontThreads, 0, ctx->st>>>(ctx->P, s->d_hist, s->d_front, nullptr);
        CK(cudaMemcpyAsync(&s->front_start, s->d_front, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        s->front_start_set = true;
    }
    for (int k = 0; k < nblocks; ++k) {
        int rc = DMPH_OK;
        if (s->fallback_left > 0 || !surrogate_allowed(ctx, s)) {
            // plain block: keep collecting and training while the surrogate is out
            rc = plain_block(ctx, s, false, nullptr, nullptr);
            if (!rc && s->fallback_left > 0) {
                s->fallback_left--;
                if (s->prm.train_iters_per_block > 0 && s->pool_count >= s->B / 4)
                    rc = train(ctx, s, s->prm.train_iters_per_block, nullptr);
            }
        } else if (s->since_check >= s->prm.check_interval) {
            double ex = 0, ev = 0, fr[3] = {0.0, 0.0, 0.0};
            const int calls = s->since_check;
            rc = plain_block(ctx, s, true, &ex, &ev, fr);
            s->since_check = 0;
            s->st.judged++;
            s->st.last_error = ex;
            s->st.last_error_v = ev;
            // the velocity increments carry the dynamics; the displacements are
            // mostly the known drift K dt v0 and would hide their error
            bool fall = s->prm.tolerance > 0 && !(ev <= s->prm.tolerance);
            if (s->prm.front_tolerance > 0) {
                // the deviation a call makes in the front: its position error
                // within the block, and the error of the front fluid's
                // velocity, which persists and moves the front over the calls
                // that follow; those since the last judged block each taken
                // to have made it, added up
                const double kdt = (double)s->prm.substeps * ctx->P.dt;
                const double d = std::fabs(fr[0] - fr[1]) + std::fabs(fr[2]) * kdt * std::max(1, calls) * 0.5;
                s->front_est += d * std::max(1, calls);
                const double travel = std::max(fr[1] - s->front_start, 10.0 * ctx->P.dx);
                s->st.last_front_dev = d;
                s->st.front_estimate = s->front_est / travel;
                if (!(s->st.front_estimate <= s->prm.front_tolerance)) fall = true;
            }
            if (!rc && fall) {
                s->st.fallbacks++;
                s->fallback_left = s->prm.fallback_blocks;
                s->front_est = 0.0;
            }
        } else {
            rc = surrogate_block(ctx, s);
            if (rc == DMPH_ENAN) {
                // nothing was applied: fall back and continue with the plain solver
                s->st.fallbacks++;
                s->fallback_left = s->prm.fallback_blocks;
                ctx->err.clear();
                rc = DMPH_OK;
            }
            s->since_check++;
        }
        if (rc) return rc;
    }
    return check_err(ctx, s);  // a tensor-core wait that ran out, in any call
}

extern "C" int dmph_surrogate_get_stats(dmph_ctx *ctx, dmph_surrogate_stats *out)
{
    dmph::Surrogate *s = need_sg(ctx);
    if (!s || !out) return DMPH_EINVAL;
    *out = s->st;
    out->pool_rows = s->pool_count;
    out->in_fallback = s->fallback_left > 0 ? 1 : 0;
    return DMPH_OK;
}

extern "C" int dmph_surrogate_get_weights(dmph_ctx *ctx, float *w, int count)
{
    dmph::Surrogate *s = need_sg(ctx);
    if (!s) return DMPH_EINVAL;
    if (!w) return s->M.count;
    if (count != s->M.count) return DMPH_ERANGE;
    CK(cudaMemcpy(w, s->M.w, sizeof(float) * count, cudaMemcpyDeviceToHost));
    return DMPH_OK;
}

extern "C" int dmph_surrogate_set_weights(dmph_ctx *ctx, const float *w, int count)
{
    dmph::Surrogate *s = need_sg(ctx);
    if (!s || !w) return DMPH_EINVAL;
    if (count != s->M.count) return DMPH_ERANGE;
    CK(cudaMemcpy(s->M.w, w, sizeof(float) * count, cudaMemcpyHostToDevice));
    dmph::launch_weights_to_bf16(s->M, ctx->st);
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

// MLP on host rows (n x 64 features, FP32) -> n x 16 outputs
// layers: through one GEMM per layer instead of the fused kernel
static int mlp_forward_host(dmph_ctx *ctx, const float *X, int n, float *Y, bool layers)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s || !X || !Y || n <= 0) return DMPH_EINVAL;
    if (n > ctx->P.N) return DMPH_ERANGE;
    std::vector<__nv_bfloat16> xb((size_t)n * kMlpIn);
    for (size_t i = 0; i < xb.size(); ++i) xb[i] = __float2bfloat16_rn(X[i]);
    CK(cudaMemcpyAsync(s->X, xb.data(), xb.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, ctx->st));
    if (layers) {
        mlp_forward_layers(s, s->X, n, s->Y, ctx->st);
    } else {
        const int rc = mlp_forward(ctx, s, s->X, n, s->Y, ctx->st);
        if (rc) return rc;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(Y, s->Y, sizeof(float) * (size_t)n * kMlpOut, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return check_err(ctx, s);
}

extern "C" int dmph_mlp_forward(dmph_ctx *ctx, const float *X, int n, float *Y)
{
    return mlp_forward_host(ctx, X, n, Y, false);
}

extern "C" int dmph_mlp_forward_layers(dmph_ctx *ctx, const float *X, int n, float *Y)
{
    return mlp_forward_host(ctx, X, n, Y, true);
}

// device time of the forward pass over the first n rows of the features the
// surrogate holds (the last call's or judge's), averaged over reps runs
extern "C" int dmph_mlp_forward_timed(dmph_ctx *ctx, int n, int reps, int layers, float *ms)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s || !ms || n <= 0 || reps <= 0) return DMPH_EINVAL;
    if (n > ctx->P.N) return DMPH_ERANGE;
    auto run = [&]() -> int {
        if (layers) {
            mlp_forward_layers(s, s->X, n, s->Y, ctx->st);
            return DMPH_OK;
        }
        return mlp_forward(ctx, s, s->X, n, s->Y, ctx->st);
    };
    int rc = run();  // warm-up
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev0, ctx->st));
    for (int r = 0; r < reps && !rc; ++r) rc = run();
    CK(cudaEventRecord(ctx->ev1, ctx->st));
    CK(cudaEventSynchronize(ctx->ev1));
    if (rc) return rc;
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    *ms = t / (float)reps;
    return check_err(ctx, s);
}

// loss and parameter gradient of one batch of host rows (n = the batch size)
extern "C" int dmph_mlp_gradient(dmph_ctx *ctx, const float *X, const float *T, int n, float *grad, float *loss)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s || !X || !T || !grad) return DMPH_EINVAL;
    if (n != s->B) {
        ctx->err = "dmph_mlp_gradient: n must equal the training batch";
        return DMPH_ERANGE;
    }
    std::vector<__nv_bfloat16> xb((size_t)n * kMlpIn), xt((size_t)n * kMlpIn);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < kMlpIn; ++k) {
            const __nv_bfloat16 h = __float2bfloat16_rn(X[(size_t)i * kMlpIn + k]);
            xb[(size_t)i * kMlpIn + k] = h;
            xt[(size_t)k * n + i] = h;
        }
    CK(cudaMemcpyAsync(s->Xb, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(s->XTb, xt.data(), xt.size() * 2, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(s->Tb, T, sizeof(float) * (size_t)n * kMlpOut, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemsetAsync(s->M.grad, 0, sizeof(float) * s->M.count, ctx->st));
    mlp_backprop(s, ctx->st);
    CK(cudaGetLastError());
    float l = 0.f;
    CK(cudaMemcpyAsync(grad, s->M.grad, sizeof(float) * s->M.count, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&l, s->d_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemsetAsync(s->M.grad, 0, sizeof(float) * s->M.count, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (loss) *loss = l / (float)((double)n * kMlpTargets);
    return check_err(ctx, s);
}

// features of the current state (pass A, pass B, features) for the fluid and
// debris slots [0, rows), FP32, rows x 48; returns rows through *rows
extern "C" int dmph_surrogate_features(dmph_ctx *ctx, float *F, int *rows)
{
    using namespace dmph;
    Surrogate *s = need_sg(ctx);
    if (!s || !F) return DMPH_EINVAL;
    if (!s->feat32) SA(s->feat32, (size_t)ctx->P.N * kMlpFeatures);
    enqueue_features(ctx, s, s->feat32, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(F, s->feat32, sizeof(float) * (size_t)s->n_rows * kMlpFeatures, cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (rows) *rows = s->n_rows;
    return DMPH_OK;
}
