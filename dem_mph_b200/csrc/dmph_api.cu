// The C ABI of libdmph.so (include/dmph.h): solver contexts and the step
// driver that stands in for the reference main loop
// (source/DEM-MPH.cpp:438-581).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dmph_ctx.h"

using namespace dmph;

namespace {
thread_local std::string g_create_err;
// set by failing calls that take no context and must not allocate
// (dmph_cell_sort_noalloc); cleared by dmph_create
thread_local const char *g_noctx_literal = nullptr;
}


// state: the allocation is part of the context's state (a checkpoint holds
// it); false for output buffers allocated on first request
template <class T>
static int dalloc(dmph_ctx *ctx, T **ptr, size_t count, bool state = true)
{
    void *p = nullptr;
    const size_t bytes = count ? count * sizeof(T) : 16;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return DMPH_ENOMEM;
    }
    ctx->allocs.push_back({p, bytes, state});
    *ptr = (T *)p;
    return cudaMemsetAsync(p, 0, count ? count * sizeof(T) : 16, ctx->st) == cudaSuccess ? DMPH_OK : DMPH_ECUDA;
}


static void release(dmph_ctx *ctx)
{
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    surrogate_release(ctx);
    drop_graph(ctx);
    if (ctx->st2) cudaStreamDestroy(ctx->st2);
    ctx->st2 = nullptr;
    for (const auto &a : ctx->allocs) cudaFree(a.p);
    ctx->allocs.clear();
    if (ctx->h_maxshift) cudaFreeHost(ctx->h_maxshift);
    if (ctx->h_small) cudaFreeHost(ctx->h_small);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->pe0) cudaEventDestroy(ctx->pe0);
    if (ctx->pe1) cudaEventDestroy(ctx->pe1);
    if (ctx->pl0) cudaEventDestroy(ctx->pl0);
    if (ctx->pl1) cudaEventDestroy(ctx->pl1);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    ctx->h_maxshift = nullptr;
    ctx->h_small = nullptr;
    ctx->ev0 = ctx->ev1 = nullptr;
    ctx->st = nullptr;
}

// number of kernels launch_bitonic issues for n = 2^nlog words
static long long bitonic_launches(int n, int nlog) { return bitonic_launch_count(n, nlog); }

// calculateCellParticle :1288 + the parts of calculateNeighbor the step needs.
// Every launch has a static shape and every range lives in ctx->dB, so the
// sequence can be recorded into a CUDA graph; permuted arrays are written to
// the second buffers and copied back, so device pointers never change.
void dmph::enqueue_rebuild(dmph_ctx *ctx, bool first, cudaStream_t st)
{
    const DevParams &P = ctx->P;
    const size_t N = (size_t)P.N;
    DevState &S = ctx->S;
    if (ctx->fp32 && !first) launch_export32(P, S, S.pos, nullptr, st);
    // the counting sort orders a cell's particles its own way; the reference's
    // per-particle DEM constants take the last neighbour in the network's
    // order (:2305-2341), so scenes with debris outside rigid bodies keep
    // the network
    const bool csort = ctx->csort && (ctx->n_solid == 0 || ctx->Bd.B > 0);
    // walls at rest stay in their cells, and the stable counting sort keeps
    // their relative order, so after the first sort every wall keeps its slot
    // (walls sort after fluid and debris, whose counts never change): the
    // permutation and the copies then cover only the fluid and debris slots
    const size_t np = (ctx->fp32 && csort && ctx->walls_rest && !first) ? (size_t)(ctx->n_fluid + ctx->n_solid) : N;
    if (csort) {
        launch_counting_sort(P, (int)np, S.pos, S.type, ctx->ckeys, ctx->ccounts, ctx->words2, ctx->words,
                             S.cell_start, ctx->bsums, ctx->total, st);
    } else {
        launch_keys(P, S.pos, S.type, ctx->words, st);
        launch_bitonic(ctx->words, P.P2, P.P2log, st);
        launch_cell_start(P, ctx->words, S.cell_start, st);
    }
    if (ctx->fp32) {
        // the walls' wall-wall sums are kept only while every wall keeps its slot
        if (np == N && S.st_valid) cudaMemsetAsync(S.st_valid, 0, N * sizeof(int), st);
        launch_permute32(P, (int)np, ctx->words, S.pos, S.v4, S.type, S.pidx, ctx->p4b, ctx->v4b, ctx->type2,
                         ctx->pidx2, S.xref, S.xref4, S.bid, ctx->bid2, S.vel, ctx->pos2, ctx->vel2, st,
                         ctx->list_reuse ? S.xrefL4 : nullptr);
        cudaMemcpyAsync(S.p4, ctx->p4b, np * sizeof(float4), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(S.v4, ctx->v4b, np * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    } else {
        launch_permute(P, ctx->words, S.pos, S.vel, S.type, S.pidx, ctx->pos2, ctx->vel2, ctx->type2, ctx->pidx2,
                       S.xref, S.bid, ctx->bid2, st);
    }
    for (int d = 0; d < 3; d++) {
        cudaMemcpyAsync(S.pos + d * N, ctx->pos2 + d * N, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(S.vel + d * N, ctx->vel2 + d * N, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
    cudaMemcpyAsync(S.type, ctx->type2, np * sizeof(int), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(S.pidx, ctx->pidx2, np * sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (S.bid) {
        cudaMemcpyAsync(S.bid, ctx->bid2, np * sizeof(int), cudaMemcpyDeviceToDevice, st);
        launch_slot_of_row(P, S.pidx, ctx->Bd.slot_of_row, st);
    }
    S.skey = ctx->words;
    launch_chunks(P, ctx->words, S.cell_start, ctx->flag, ctx->offs, ctx->bsums, ctx->total, S.chunks, st);
    launch_bounds(P, S.cell_start, ctx->offs, ctx->total, ctx->dB, st);
    if (ctx->fp32)
        launch_wet_partition(P, ctx->words, S.cell_start, S.chunks, ctx->chunks2, ctx->dB, ctx->flag, ctx->offs,
                             ctx->bsums, ctx->total, st);
    if (ctx->use_list) {
        // the list build alone is also timed as phase 6 (inside phase 1)
        if (ctx->prof) cudaEventRecord(ctx->pl0, st);
        if (ctx->fp32)
            launch_build_list32(P, ctx->Q, S, ctx->dB, ctx->Wm.moving ? 0 : 1, st, ctx->var_build,
                                ctx->list_reuse ? 1 : 0);
        else launch_build_list64(P, S, ctx->dB, st);
        if (ctx->prof) {
            cudaEventRecord(ctx->pl1, st);
            cudaEventSynchronize(ctx->pl1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->pl0, ctx->pl1);
            ctx->phase_ms[6] += ms;
            ctx->phase_n[6] += 1;
        }
    }
    if (ctx->fp32 && ctx->use_list && !ctx->all_counts) launch_counts_list(P, S, ctx->dB, st);
    else launch_counts(P, S, ctx->dB, ctx->all_counts ? CR_ALL : CR_SOLID, st);
}

long long dmph::rebuild_launches(const dmph_ctx *ctx, bool first)
{
    const DevParams &P = ctx->P;
    const long long sort =
        ctx->csort && (ctx->n_solid == 0 || ctx->Bd.B > 0) ? 6 : 1 + bitonic_launches(P.P2, P.P2log) + 1;
    return sort + 1 + (ctx->fp32 && !first ? 1 : 0) + 5 + 1 +
           (ctx->fp32 ? 6 : 0) + (ctx->fp32 && ctx->use_list && !ctx->all_counts ? 2 : 1) + (ctx->S.bid ? 1 : 0) +
           (ctx->use_list ? 1 : 0);
}

// phase timing (dmph_set_profiling): events around one phase, synchronised
static void phase_begin(dmph_ctx *ctx)
{
    if (ctx->prof) cudaEventRecord(ctx->pe0, ctx->st);
}
static void phase_end(dmph_ctx *ctx, int ph)
{
    if (!ctx->prof) return;
    cudaEventRecord(ctx->pe1, ctx->st);
    cudaEventSynchronize(ctx->pe1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->pe0, ctx->pe1);
    ctx->phase_ms[ph] += ms;
    ctx->phase_n[ph] += 1;
}

// drift + rebuild decision (first part of a step)
bool dmph::reuse_active(const dmph_ctx *ctx)
{
    // (the neighbour counts of every particle, DMPH_FLAG_ALL_NEIGHBOR_COUNTS,
    // are made by the full rebuild only)
    return ctx->list_reuse && ctx->fp32 && ctx->use_list && ctx->walls_rest && ctx->csort && !ctx->Wm.moving &&
           !ctx->all_counts && (ctx->n_solid == 0 || ctx->Bd.B > 0);
}

// Head of a step: drift and the rebuild decision (B_NEED: 0 none, 1 full
// rebuild, 2 with list reuse a trigger that keeps the lists, whose trigger
// positions and debris counts the two gated kernels after the decision
// refresh)
void dmph::enqueue_head(dmph_ctx *ctx, unsigned long long graph_cond, cudaStream_t st)
{
    const DevParams &P = ctx->P;
    const bool reuse = reuse_active(ctx);
    cudaMemsetAsync(ctx->maxshift, 0, sizeof(unsigned long long), st);
    if (reuse) cudaMemsetAsync(ctx->maxshiftL, 0, sizeof(unsigned long long), st);
    if (ctx->fp32)
        launch_drift32(P, ctx->Q, ctx->S, ctx->Wm, ctx->maxshift, ctx->sms, st, reuse ? ctx->maxshiftL : nullptr);
    else
        launch_drift(P, ctx->S, ctx->Wm, ctx->maxshift, ctx->sms, st);
    launch_decide(P, ctx->maxshift, ctx->dB, graph_cond, st, reuse ? ctx->maxshiftL : nullptr);
    if (reuse) {
        launch_kept_trigger32(P, ctx->S, ctx->dB, ctx->n_fluid + ctx->n_solid, st);
        launch_counts_list_kept(P, ctx->S, ctx->dB, st);
    }
}

// kernels enqueue_head launches
static long long head_launches(const dmph_ctx *ctx) { return reuse_active(ctx) ? 4 : 2; }

// the pair passes (first part of a step's tail)
void dmph::enqueue_passes(dmph_ctx *ctx, cudaStream_t st)
{
    const DevParams &P = ctx->P;
    DevState &S = ctx->S;
    const int *dB = ctx->dB;
    if (ctx->fp32) {
        const DevParams32 &Q = ctx->Q;
        phase_begin(ctx);
        if (ctx->use_list && ctx->Wm.moving) launch_list_wall_guard(ctx->dB, st);
        if (ctx->use_list) launch_pass_a32_list(P, Q, S, dB, ctx->var_la, st);
        launch_pass_a32(P, Q, S, dB, CR_WET, ctx->var_a, st, ctx->use_list ? 1 : 0);
        phase_end(ctx, 2);
        phase_begin(ctx);
        if (ctx->use_list) launch_pass_b32_list(P, Q, S, dB, ctx->var_lb, st);
        launch_pass_b32(P, Q, S, dB, ctx->var_b, st, ctx->use_list ? 1 : 0);
        launch_fluid_accel32(Q, S, dB, st);
        phase_end(ctx, 3);
    } else {
        const int lst = ctx->use_list ? 1 : 0;
        phase_begin(ctx);
        if (lst) launch_pass_a(P, S, dB, CR_ALL, 0, st, 1, 0);
        launch_pass_a(P, S, dB, CR_ALL, 0, st, 0, lst);
        phase_end(ctx, 2);
        phase_begin(ctx);
        if (lst) launch_pass_b(P, S, dB, st, 1, 0);
        launch_pass_b(P, S, dB, st, 0, lst);
        launch_fluid_accel(P, S, dB, st);
        phase_end(ctx, 3);
    }
}

// pass A and pass B of the FP32 build without the fluid update (surrogate
// evaluations): over the Verlet lists in list mode, with the stencil kernels
// standing in after a list overflow
void dmph::enqueue_pair_passes32(dmph_ctx *ctx, cudaStream_t st)
{
    const DevParams &P = ctx->P;
    const DevParams32 &Q = ctx->Q;
    if (ctx->use_list && ctx->Wm.moving) launch_list_wall_guard(ctx->dB, st);
    if (ctx->use_list) launch_pass_a32_list(P, Q, ctx->S, ctx->dB, ctx->var_la, st);
    launch_pass_a32(P, Q, ctx->S, ctx->dB, CR_WET, ctx->var_a, st, ctx->use_list ? 1 : 0);
    if (ctx->use_list) launch_pass_b32_list(P, Q, ctx->S, ctx->dB, ctx->var_lb, st);
    launch_pass_b32(P, Q, ctx->S, ctx->dB, ctx->var_b, st, ctx->use_list ? 1 : 0);
}

// the DEM substeps or rigid bodies (second part of a step's tail)
void dmph::enqueue_dem(dmph_ctx *ctx, cudaStream_t st)
{
    const DevParams &P = ctx->P;
    DevState &S = ctx->S;
    const int *dB = ctx->dB;
    phase_begin(ctx);
    if (ctx->fp32) {
        // DEM and rigid bodies in FP64 on the solids' and walls' master state
        launch_solid_force_to64(P, S, dB, st);
        for (int k = 0; k < ctx->demSteps; ++k) {
            if (ctx->Bd.B > 0) {
                launch_clump_dem(P, S, dB, ctx->use_list, st);
                launch_body_step(P, S, ctx->Bd, true, st);
                continue;
            }
            launch_dem_force(P, S, dB, CR_SOLID, 1, st, true);
            if (P.wall_dem_coeffs) launch_dem_force(P, S, dB, CR_WALL, 0, st, true);
            launch_dem_integrate(P, S, dB, st);
        }
        launch_sync_solids32(P, S, dB, st);
    } else {
        for (int k = 0; k < ctx->demSteps; ++k) {
            if (ctx->Bd.B > 0) {
                launch_clump_dem(P, S, dB, false, st);
                launch_body_step(P, S, ctx->Bd, false, st);
                continue;
            }
            launch_dem_force(P, S, dB, CR_SOLID, 1, st, false, ctx->use_list);
            if (P.wall_dem_coeffs) launch_dem_force(P, S, dB, CR_WALL, 0, st, false, ctx->use_list);
            launch_dem_integrate(P, S, dB, st);
        }
    }
    phase_end(ctx, ctx->Bd.B > 0 ? 5 : 4);
}

// The DEM substeps of `steps` steps with the fluid force held (the surrogate's
// block).  With rigid bodies in the FP32 build the fluid force goes to the
// FP64 planes once and the FP32 copies of the debris are refreshed once, at
// the end (the contact forces have planes of their own and the substeps read
// the FP64 masters); otherwise the steps' DEM phases one after the other.
void dmph::enqueue_dem_block(dmph_ctx *ctx, int steps, cudaStream_t st)
{
    if (!(ctx->fp32 && ctx->Bd.B > 0)) {
        for (int k = 0; k < steps; ++k) enqueue_dem(ctx, st);
        return;
    }
    const DevParams &P = ctx->P;
    DevState &S = ctx->S;
    phase_begin(ctx);
    launch_solid_force_to64(P, S, ctx->dB, st);
    for (int k = 0; k < steps * ctx->demSteps; ++k) {
        launch_clump_dem(P, S, ctx->dB, ctx->use_list, st);
        launch_body_step(P, S, ctx->Bd, true, st);
    }
    launch_sync_solids32(P, S, ctx->dB, st);
    phase_end(ctx, 5);
}

long long dmph::dem_block_launches(const dmph_ctx *ctx, int steps)
{
    if (!(ctx->fp32 && ctx->Bd.B > 0)) return steps * dem_launches(ctx);
    return 2 + (long long)steps * ctx->demSteps * (ctx->use_list ? 3 : 2);
}

// the force passes and the DEM substeps (second part of a step)
static void enqueue_tail(dmph_ctx *ctx, cudaStream_t st)
{
    enqueue_passes(ctx, st);
    enqueue_dem(ctx, st);
}

long long dmph::dem_launches(const dmph_ctx *ctx)
{
    // clump contacts (FP32 list mode: list walk and gated cell walk) and the
    // body update, or the reference's DEM force(s) and integration
    // (FP64 list mode: each DEM force launch is a list walk and a gated cell walk)
    const long long nforce = (!ctx->fp32 && ctx->use_list) ? 2 : 1;
    const long long dem = ctx->Bd.B > 0 ? (ctx->fp32 && ctx->use_list ? 3 : 2)
                                        : nforce * (1 + (ctx->P.wall_dem_coeffs ? 1 : 0)) + 1;
    return ctx->demSteps * dem + (ctx->fp32 ? 2 : 0);
}

long long dmph::tail_launches(const dmph_ctx *ctx, bool graph)
{
    // list mode: pass A list, pass B list (FP32: fluid and debris kernels,
    // and the list guard in a moving-wall window, which graphs never cover)
    return 3 + dem_launches(ctx) +
           (ctx->use_list ? (ctx->fp32 ? 3 + (!graph && ctx->Wm.moving ? 1 : 0) : 2) : 0);
}

void dmph::advance_host_clock(dmph_ctx *ctx)
{
    // WallCenter moves only while `0.0 < Time < 0.2` holds, i.e. Time <= 0 (:2892)
    if (!(0.0 < ctx->time))
        for (int t = DMPH_WALL_BEGIN; t < DMPH_WALL_END; ++t)
            for (int d = 0; d < 3; d++) ctx->Wm.C[t][d] += ctx->Wm.Vel[t][d] * ctx->P.dt;
    ctx->time += ctx->P.dt;
    ctx->steps++;
}

// One step recorded as a CUDA graph: head, an IF node whose body is the
// rebuild (its condition set on the device by the decision kernel), tail.
// Valid while the head's parameters do not change: no moving-wall window and
// Time > 0 (the wall centres move only while Time <= 0).
// Record, on a capturing stream, the head of a step followed by an IF node
// whose body is the rebuild; the decision kernel of the head sets the
// condition on the device.
static int capture_head_and_rebuild(dmph_ctx *ctx, cudaGraph_t g, cudaStream_t st)
{
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    enqueue_head(ctx, (unsigned long long)cond, st);
    return capture_rebuild_if(ctx, cond, st);
}

// On a capturing stream: an IF node after the stream's current work whose
// body is the scene's rebuild, run when a decision kernel sets `cond`
int dmph::capture_rebuild_if(dmph_ctx *ctx, cudaGraphConditionalHandle cond, cudaStream_t st)
{
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t cg = nullptr;
    CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(ctx->st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_rebuild(ctx, false, ctx->st2);
    CK(cudaStreamEndCapture(ctx->st2, &body));
    return DMPH_OK;
}

// One step recorded as a CUDA graph: head, an IF node whose body is the
// rebuild (its condition set on the device by the decision kernel), tail.
// Valid while the head's parameters do not change: no moving-wall window and
// Time > 0 (the wall centres move only while Time <= 0).
static int build_graph(dmph_ctx *ctx)
{
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    CK(cudaStreamBeginCaptureToGraph(ctx->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = capture_head_and_rebuild(ctx, g, ctx->st);
    if (rc) {
        cudaStreamEndCapture(ctx->st, &g);
        cudaGraphDestroy(g);
        return rc;
    }
    enqueue_tail(ctx, ctx->st);
    CK(cudaStreamEndCapture(ctx->st, &g));
    CK(cudaGraphInstantiate(&ctx->gexec, g, 0));
    ctx->graph = g;
    return DMPH_OK;
}

void dmph::drop_graph(dmph_ctx *ctx)
{
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    ctx->gexec = nullptr;
    ctx->graph = nullptr;
}

// calculateWall moves the walls while 0.2 <= Time <= 0.4 (:2857)
static bool in_wall_window(const dmph_ctx *ctx)
{
    return ctx->time >= 0.2 && 0.4 >= ctx->time && !(ctx->fp32 && ctx->walls_rest);
}

static bool graph_usable(const dmph_ctx *ctx)
{
    return ctx->use_graph && !ctx->prof && 0.0 < ctx->time && !in_wall_window(ctx);
}

int dmph::step_once(dmph_ctx *ctx)
{
    ctx->Wm.moving = in_wall_window(ctx) ? 1 : 0;
    if (graph_usable(ctx)) {
        if (!ctx->gexec) {
            const int rc = build_graph(ctx);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(ctx->gexec, ctx->st));
        ctx->graph_steps++;
        advance_host_clock(ctx);
        return DMPH_OK;
    }
    phase_begin(ctx);
    enqueue_head(ctx, 0, ctx->st);
    phase_end(ctx, 0);
    CK(cudaMemcpyAsync(ctx->h_small, ctx->dB + B_NEED, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->launches += head_launches(ctx);
    if (ctx->h_small[0] == 1) {
        phase_begin(ctx);
        enqueue_rebuild(ctx, false, ctx->st);
        phase_end(ctx, 1);
        ctx->launches += rebuild_launches(ctx, false);
        ctx->host_rebuilds++;
    }
    enqueue_tail(ctx, ctx->st);
    ctx->launches += tail_launches(ctx);
    CK(cudaGetLastError());
    advance_host_clock(ctx);
    return DMPH_OK;
}

// host copy of the device bounds (synchronises the stream)
int dmph::read_bounds(dmph_ctx *ctx, int *b)
{
    CK(cudaMemcpyAsync(ctx->h_small, ctx->dB, B_COUNT * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int k = 0; k < B_COUNT; k++) b[k] = ctx->h_small[k];
    return DMPH_OK;
}

extern "C" int dmph_create(const dmph_params *p, int n, const int *type, const double *x3, const double *v3,
                           dmph_ctx **out)
{
    g_create_err.clear();
    g_noctx_literal = nullptr;
    if (!out) return DMPH_EINVAL;
    *out = nullptr;
    if (!p || !type || !x3 || !v3) {
        g_create_err = "null argument";
        return DMPH_EINVAL;
    }
    if (p->precision != DMPH_PRECISION_FP64 && p->precision != DMPH_PRECISION_FP32_SPLIT) {
        g_create_err = "unknown precision";
        return DMPH_EINVAL;
    }
    for (int i = 0; i < n; i++)
        if (type[i] < 0 || type[i] >= DMPH_TYPE_COUNT) {
            g_create_err = "particle type outside 0..5 at row " + std::to_string(i);
            return DMPH_EINVAL;
        }
    dmph_ctx *ctx = new dmph_ctx();
    ctx->p = *p;
    int rc = derive_params(*p, n, ctx->P, ctx->Wm, ctx->err);
    if (rc) {
        g_create_err = ctx->err;
        delete ctx;
        return rc;
    }
    for (int i = 0; i < n; i++) {
        ctx->n_solid += (type[i] >= DMPH_SOLID_BEGIN && type[i] < DMPH_SOLID_END) ? 1 : 0;
        ctx->n_fluid += type[i] < DMPH_SOLID_BEGIN ? 1 : 0;
    }
    ctx->walls_rest = true;
    for (int t = DMPH_WALL_BEGIN; t < DMPH_WALL_END; ++t)
        for (int d = 0; d < 3; ++d)
            if (p->wall_velocity[t][d] != 0.0 || p->wall_omega[t][d] != 0.0) ctx->walls_rest = false;
    for (long long k = 0; k < 3ll * n; k++)
        if (!std::isfinite(x3[k]) || !std::isfinite(v3[k])) {
            g_create_err = "non-finite position or velocity at row " + std::to_string(k / 3);
            delete ctx;
            return DMPH_ENAN;
        }
    ctx->all_counts = (p->flags & DMPH_FLAG_ALL_NEIGHBOR_COUNTS) != 0;
    ctx->fp32 = p->precision == DMPH_PRECISION_FP32_SPLIT;
    if (ctx->fp32) {
        const int *cc = ctx->P.cc;
        const bool fits = cc[0] <= 1024 && cc[1] <= 1024 && cc[2] <= 512;
        const bool wide = cc[0] >= 3 && cc[1] >= 3 && (p->dim == 2 ? cc[2] == 1 : cc[2] >= 3);
        if (!fits || !wide) {
            g_create_err = "FP32 split precision needs 3..1024 cells along x and y and 3..512 along z (1 in 2D)";
            delete ctx;
            return DMPH_EINVAL;
        }
        ctx->Q = make_params32(ctx->P);
    }
    ctx->demSteps = p->dt / p->dem_dt;  // (int)(Dt/DEMDt), :434
    ctx->time = p->time;
    auto fail = [&](int code) {
        g_create_err = ctx->err;
        release(ctx);
        delete ctx;
        return code;
    };
#define CKC(call)                                                                                \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                       \
            return fail(DMPH_ECUDA);                                                             \
        }                                                                                        \
    } while (0)
    int dev = 0;
    CKC(cudaGetDevice(&dev));
    ctx->device = dev;
    CKC(cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, dev));
    CKC(cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking));
    CKC(cudaStreamCreateWithFlags(&ctx->st2, cudaStreamNonBlocking));
    CKC(cudaEventCreate(&ctx->ev0));
    CKC(cudaEventCreate(&ctx->ev1));
    CKC(cudaEventCreate(&ctx->pe0));
    CKC(cudaEventCreate(&ctx->pe1));
    CKC(cudaEventCreate(&ctx->pl0));
    CKC(cudaEventCreate(&ctx->pl1));
    CKC(cudaMallocHost(&ctx->h_maxshift, sizeof(unsigned long long)));
    CKC(cudaMallocHost(&ctx->h_small, 2 * B_COUNT * sizeof(int)));
    const DevParams &P = ctx->P;
    const size_t N = (size_t)n, N3 = 3 * N;
    DevState &S = ctx->S;
#define AL(ptr, cnt)                                  \
    do {                                              \
        int r_ = dalloc(ctx, &(ptr), (size_t)(cnt));  \
        if (r_) return fail(r_);                      \
    } while (0)
    AL(S.pos, N3);
    AL(S.vel, N3);
    AL(S.frc, N3);
    AL(S.xref, N3);
    AL(S.type, N);
    AL(S.pidx, N);
    AL(S.vsp, N);
    AL(S.divp, N);
    AL(S.pres, N);
    AL(S.densA, N);
    AL(S.pA, N);
    AL(S.gc, N3);
    AL(S.kn, N);
    AL(S.cn, N);
    AL(S.kt, N);
    AL(S.ct, N);
    AL(S.alpha, N);
    AL(S.dragC, N);
    AL(S.nc, N);
    AL(S.snc, N);
    AL(S.cell_start, (size_t)3 * P.T + 1);
    AL(S.chunks, N + 64);
    AL(ctx->chunks2, N + 64);
    AL(ctx->pos2, N3);
    AL(ctx->vel2, N3);
    AL(ctx->type2, N);
    AL(ctx->pidx2, N);
    AL(ctx->words, (size_t)P.P2);
    if (ctx->fp32 && 3LL * P.T + 1 <= kCountingSortMaxKeys) {
        ctx->csort = true;
        AL(ctx->ckeys, N);
        AL(ctx->ccounts, 3 * (size_t)P.T + 1);
        AL(ctx->words2, N);
    }
    if (ctx->fp32) {
        AL(S.p4, N);
        AL(S.v4, N);
        AL(S.f4, N);
        AL(S.xref4, N);
        AL(S.gc4, N);
        AL(ctx->p4b, N);
        AL(ctx->v4b, N);
        AL(S.pres32, N);
        AL(S.vsp32, N);
        AL(S.div32, N);
        AL(S.densA32, N);
        AL(S.pA32, N);
        AL(S.alpha32, N);
        AL(S.dragC32, N);
    }
    {
        // Verlet lists: the lattice holds 122 (3D) / 28 (2D) particles within
        // MaxRadius + MARGIN = 3.1 dx; the capacity leaves room for compression
        S.nbl_cap = P.dim == 2 ? 64 : 192;
        AL(S.nbl, (size_t)S.nbl_cap * N);
        AL(S.nbn, N);
        if (ctx->fp32) {
            AL(S.vsp_st, N);
            AL(S.st4, N);
            AL(S.st_valid, N);
        }
        ctx->use_list = true;
    }
    AL(ctx->flag, N);
    AL(ctx->offs, N);
    AL(ctx->bsums, 4096);
    AL(ctx->total, 4);
    AL(ctx->maxshift, 1);
    AL(ctx->dB, B_COUNT);
    if (ctx->fp32 && (p->flags & DMPH_FLAG_LIST_REUSE)) {
        ctx->list_reuse = true;
        AL(S.xrefL4, N);
        AL(ctx->maxshiftL, 1);
    }
    {
        // the lists of the first build have the MARGIN skin
        const int skin[2] = {10, 10};
        CKC(cudaMemcpyAsync(ctx->dB + B_SKIN, skin, sizeof(skin), cudaMemcpyHostToDevice, ctx->st));
        CKC(cudaStreamSynchronize(ctx->st));
    }
    // upload: interleaved x,y,z rows -> component planes
    {
        std::vector<double> planes(N3);
        for (size_t i = 0; i < N; i++)
            for (int d = 0; d < 3; d++) planes[d * N + i] = x3[3 * i + d];
        CKC(cudaMemcpyAsync(S.pos, planes.data(), N3 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        CKC(cudaStreamSynchronize(ctx->st));
        for (size_t i = 0; i < N; i++)
            for (int d = 0; d < 3; d++) planes[d * N + i] = v3[3 * i + d];
        CKC(cudaMemcpyAsync(S.vel, planes.data(), N3 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        CKC(cudaMemcpyAsync(S.type, type, N * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
        std::vector<int> iota(N);
        for (size_t i = 0; i < N; i++) iota[i] = (int)i;
        CKC(cudaMemcpyAsync(S.pidx, iota.data(), N * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
        CKC(cudaStreamSynchronize(ctx->st));
    }
    if (ctx->fp32) {
        // velocities of the FP32 state (positions are set by the first rebuild)
        std::vector<float4> v4(N);
        for (size_t i = 0; i < N; i++)
            v4[i] = make_float4((float)v3[3 * i], (float)v3[3 * i + 1], (float)v3[3 * i + 2], 0.f);
        CKC(cudaMemcpyAsync(S.v4, v4.data(), N * sizeof(float4), cudaMemcpyHostToDevice, ctx->st));
        CKC(cudaStreamSynchronize(ctx->st));
    }
    // initial sort, neighbour counts and densities (:419-425)
    if (ctx->fp32) ctx->Q.N0p32 = lattice_n0p32(P, ctx->Q, ctx->st);
    enqueue_rebuild(ctx, true, ctx->st);
    if (ctx->fp32)
        launch_pass_a32(P, ctx->Q, ctx->S, ctx->dB, CR_ALL, ctx->var_a, ctx->st);
    else
        launch_pass_a(P, S, ctx->dB, CR_ALL, 1, ctx->st);
    CKC(cudaGetLastError());
    CKC(cudaStreamSynchronize(ctx->st));
#undef AL
#undef CKC
    ctx->launches = 0;
    *out = ctx;
    return DMPH_OK;
}

int dmph::check_finite(dmph_ctx *ctx)
{
    if (!ctx->nonfinite) {
        CK(cudaMemcpyAsync(ctx->h_small, ctx->dB + B_NONFINITE, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        ctx->nonfinite = ctx->h_small[0] != 0;
    }
    if (!ctx->nonfinite) return DMPH_OK;
    ctx->err = "non-finite position or velocity met by a step (no neighbour rebuild runs until dmph_set_state "
               "replaces the state)";
    return DMPH_ENAN;
}

// the steps of dmph_step / dmph_step_timed, with the non-finite check every
// kFiniteCheckEvery steps and at the end
static int run_steps(dmph_ctx *ctx, int nsteps)
{
    if (ctx->nonfinite) return check_finite(ctx);
    for (int s = 0; s < nsteps; s++) {
        const int rc = step_once(ctx);
        if (rc) return rc;
        if ((s + 1) % kFiniteCheckEvery == 0 && s + 1 < nsteps) {
            const int rf = check_finite(ctx);
            if (rf) return rf;
        }
    }
    return DMPH_OK;
}

extern "C" int dmph_step(dmph_ctx *ctx, int nsteps)
{
    if (!ctx || nsteps < 0) return DMPH_EINVAL;
    const int rc = run_steps(ctx, nsteps);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return check_finite(ctx);
}

extern "C" int dmph_step_timed(dmph_ctx *ctx, int nsteps, float *device_ms)
{
    if (!ctx || nsteps < 0) return DMPH_EINVAL;
    CK(cudaEventRecord(ctx->ev0, ctx->st));
    const int rc = run_steps(ctx, nsteps);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->st));
    CK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (device_ms) *device_ms = ms;
    return check_finite(ctx);
}

// device planes -> caller's x,y,z buffer through a staging buffer (pos2 or
// vel2, free between steps); the copy is enqueued, the caller synchronises
static int d2h_planes_async(dmph_ctx *ctx, const double *dev, double *stage, double *x3)
{
    const size_t N = (size_t)ctx->P.N;
    launch_planes_to_xyz(dev, stage, (int)N, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(x3, stage, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    return DMPH_OK;
}

static int d2h_planes(dmph_ctx *ctx, const double *dev, double *x3)
{
    const int rc = d2h_planes_async(ctx, dev, ctx->pos2, x3);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

extern "C" int dmph_get_state(dmph_ctx *ctx, int *type, double *x3, double *v3, int *orig_id)
{
    if (!ctx) return DMPH_EINVAL;
    const size_t N = (size_t)ctx->P.N;
    if (ctx->fp32 && (x3 || v3)) launch_export32(ctx->P, ctx->S, ctx->S.pos, ctx->S.vel, ctx->st);
    if (x3) {
        int rc = d2h_planes_async(ctx, ctx->S.pos, ctx->pos2, x3);
        if (rc) return rc;
    }
    if (v3) {
        int rc = d2h_planes_async(ctx, ctx->S.vel, ctx->vel2, v3);
        if (rc) return rc;
    }
    if (type) CK(cudaMemcpyAsync(type, ctx->S.type, N * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    if (orig_id) CK(cudaMemcpyAsync(orig_id, ctx->S.pidx, N * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

extern "C" int dmph_set_state(dmph_ctx *ctx, const double *x3, const double *v3)
{
    if (!ctx) return DMPH_EINVAL;
    const size_t N = (size_t)ctx->P.N;
    if (x3) {
        CK(cudaMemcpyAsync(ctx->pos2, x3, 3 * N * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        launch_xyz_to_planes(ctx->pos2, ctx->S.pos, (int)N, ctx->st);
    }
    if (v3) {
        CK(cudaMemcpyAsync(ctx->vel2, v3, 3 * N * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        launch_xyz_to_planes(ctx->vel2, ctx->S.vel, (int)N, ctx->st);
    }
    if (ctx->fp32) {
        if (!x3) launch_export32(ctx->P, ctx->S, ctx->S.pos, nullptr, ctx->st);
        launch_import32(ctx->P, ctx->S, ctx->S.pos, v3 ? ctx->S.vel : nullptr, ctx->st);
    }
    // a new state: the next drift checks it afresh
    CK(cudaMemsetAsync(ctx->dB + B_NONFINITE, 0, sizeof(int), ctx->st));
    ctx->nonfinite = false;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

// ---- split steps and row-level state (domain decomposition over ranks)

// B_NEED of a step whose rebuild the caller decided (dmph_step_finish)
__global__ void k_set_need(int *dB, int need)
{
    dB[B_NEED] = need;
    dB[B_REBUILDS] += need;
    dB[B_LIST_BUILDS] += need;
    if (need) dB[B_SKIN_NEXT] = 10;  // lists with the MARGIN skin (no list reuse in split steps)
}

extern "C" int dmph_step_begin(dmph_ctx *ctx, double *max_shift2)
{
    if (!ctx) return DMPH_EINVAL;
    if (ctx->in_split_step) {
        ctx->err = "dmph_step_begin: the previous step was not finished";
        return DMPH_EINVAL;
    }
    drop_graph(ctx);  // split steps run as individual launches
    ctx->Wm.moving = in_wall_window(ctx) ? 1 : 0;
    const DevParams &P = ctx->P;
    CK(cudaMemsetAsync(ctx->maxshift, 0, sizeof(unsigned long long), ctx->st));
    if (ctx->fp32)
        launch_drift32(P, ctx->Q, ctx->S, ctx->Wm, ctx->maxshift, ctx->sms, ctx->st);
    else
        launch_drift(P, ctx->S, ctx->Wm, ctx->maxshift, ctx->sms, ctx->st);
    CK(cudaMemcpyAsync(ctx->h_maxshift, ctx->maxshift, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->launches += 1;
    double m2;
    std::memcpy(&m2, ctx->h_maxshift, sizeof(double));
    ctx->split_m2 = m2;
    ctx->in_split_step = true;
    if (max_shift2) *max_shift2 = m2;
    return DMPH_OK;
}

extern "C" int dmph_step_finish(dmph_ctx *ctx, int rebuild)
{
    if (!ctx) return DMPH_EINVAL;
    // a context that has not stepped yet may finish the step whose drift ran
    // before it was created (its creation made the rebuild of that step)
    const bool fresh = ctx->steps == 0 && !ctx->in_split_step;
    if (!ctx->in_split_step && !fresh) {
        ctx->err = "dmph_step_finish: no step begun";
        return DMPH_EINVAL;
    }
    if (fresh) {
        if (rebuild) {
            ctx->err = "dmph_step_finish: a new context's first step has had its rebuild";
            return DMPH_EINVAL;
        }
        drop_graph(ctx);
        ctx->Wm.moving = in_wall_window(ctx) ? 1 : 0;
        ctx->split_m2 = 0.0;
    }
    ctx->in_split_step = false;
    if (!std::isfinite(ctx->split_m2)) {
        // positions become cell indices in the rebuild: never from non-finite ones
        ctx->nonfinite = true;
        CK(cudaMemsetAsync(ctx->dB + B_NONFINITE, 0xFF, sizeof(int), ctx->st));
        return check_finite(ctx);
    }
    k_set_need<<<1, 1, 0, ctx->st>>>(ctx->dB, rebuild ? 1 : 0);
    ctx->launches += 1;
    if (rebuild) {
        enqueue_rebuild(ctx, false, ctx->st);
        ctx->launches += rebuild_launches(ctx, false);
        ctx->host_rebuilds++;
    }
    enqueue_tail(ctx, ctx->st);
    ctx->launches += tail_launches(ctx);
    CK(cudaGetLastError());
    advance_host_clock(ctx);
    CK(cudaStreamSynchronize(ctx->st));
    return check_finite(ctx);
}

__global__ void k_rows_io(DevParams P, double *pos, double *vel, const int *__restrict__ slot_of_row,
                          const int *__restrict__ rows, int count, double *x3, double *v3, int set)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int r = rows[k];
    if (r < 0 || r >= P.N) return;  // rejected on the host
    const int i = slot_of_row[r];
    for (int d = 0; d < 3; d++) {
        if (set) {
            if (x3) pos[d * P.N + i] = x3[3 * k + d];
            if (v3) vel[d * P.N + i] = v3[3 * k + d];
        } else {
            if (x3) x3[3 * k + d] = pos[d * P.N + i];
            if (v3) v3[3 * k + d] = vel[d * P.N + i];
        }
    }
}

// positions / velocities of input rows through the FP64 planes (exported
// from and imported into the FP32 state in the split build)
static int rows_io(dmph_ctx *ctx, int count, const int *rows, double *x3, double *v3, bool set)
{
    if (!ctx || count < 0 || (count > 0 && !rows)) return DMPH_EINVAL;
    const int N = ctx->P.N;
    if (count > N) return ctx->err = "more rows than particles", DMPH_ERANGE;
    for (int k = 0; k < count; k++)
        if (rows[k] < 0 || rows[k] >= N) return ctx->err = "row outside the grid", DMPH_ERANGE;
    if (count == 0) return DMPH_OK;
    const DevState &S = ctx->S;
    // scratch free between steps: flag (rows), offs (slot of each row),
    // pos2 / vel2 (the values)
    CK(cudaMemcpyAsync(ctx->flag, rows, sizeof(int) * count, cudaMemcpyHostToDevice, ctx->st));
    launch_slot_of_row(ctx->P, S.pidx, ctx->offs, ctx->st);
    if (ctx->fp32) launch_export32(ctx->P, S, S.pos, S.vel, ctx->st);
    if (set) {
        if (x3) CK(cudaMemcpyAsync(ctx->pos2, x3, sizeof(double) * 3 * count, cudaMemcpyHostToDevice, ctx->st));
        if (v3) CK(cudaMemcpyAsync(ctx->vel2, v3, sizeof(double) * 3 * count, cudaMemcpyHostToDevice, ctx->st));
    }
    k_rows_io<<<(count + 255) / 256, 256, 0, ctx->st>>>(ctx->P, S.pos, S.vel, ctx->offs, ctx->flag, count,
                                                         x3 ? ctx->pos2 : nullptr, v3 ? ctx->vel2 : nullptr,
                                                         set ? 1 : 0);
    if (set && ctx->fp32) launch_import32(ctx->P, S, S.pos, S.vel, ctx->st);
    if (!set) {
        if (x3) CK(cudaMemcpyAsync(x3, ctx->pos2, sizeof(double) * 3 * count, cudaMemcpyDeviceToHost, ctx->st));
        if (v3) CK(cudaMemcpyAsync(v3, ctx->vel2, sizeof(double) * 3 * count, cudaMemcpyDeviceToHost, ctx->st));
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

extern "C" int dmph_get_rows(dmph_ctx *ctx, int count, const int *rows, double *x3, double *v3)
{
    return rows_io(ctx, count, rows, x3, v3, false);
}

extern "C" int dmph_set_rows(dmph_ctx *ctx, int count, const int *rows, const double *x3, const double *v3)
{
    return rows_io(ctx, count, rows, const_cast<double *>(x3), const_cast<double *>(v3), true);
}

extern "C" int dmph_get_field(dmph_ctx *ctx, int field_id, void *out)
{
    if (!ctx || !out) return DMPH_EINVAL;
    const size_t N = (size_t)ctx->P.N;
    const DevState &S = ctx->S;
    const double *src = nullptr;
    if (ctx->fp32) {
        // widen the FP32 field into its FP64 twin, then copy as in FP64 mode
        const int n = (int)N;
        switch (field_id) {
        case DMPH_FIELD_FORCE: {  // fluid slots only: the solids' FP64 forces include their contacts
            int b[B_COUNT];
            const int rc = read_bounds(ctx, b);
            if (rc) return rc;
            launch_widen_f4(S.f4, S.frc, b[B_FE], n, ctx->st);
            break;
        }
        case DMPH_FIELD_GRAVITY_CENTER: launch_widen_f4(S.gc4, S.gc, n, n, ctx->st); break;
        case DMPH_FIELD_VOL_STRAIN_P: launch_widen_f(S.vsp32, S.vsp, n, ctx->st); break;
        case DMPH_FIELD_DIVERGENCE_P: launch_widen_f(S.div32, S.divp, n, ctx->st); break;
        case DMPH_FIELD_PRESSURE_P: launch_widen_f(S.pres32, S.pres, n, ctx->st); break;
        case DMPH_FIELD_DENSITY_A: launch_widen_f(S.densA32, S.densA, n, ctx->st); break;
        case DMPH_FIELD_PRESSURE_A: launch_widen_f(S.pA32, S.pA, n, ctx->st); break;
        case DMPH_FIELD_ALPHA: launch_widen_f(S.alpha32, S.alpha, n, ctx->st); break;
        case DMPH_FIELD_DRAG_C: launch_widen_f(S.dragC32, S.dragC, n, ctx->st); break;
        default: break;
        }
        CK(cudaGetLastError());
    }
    if (field_id == DMPH_FIELD_VIRIAL_PRESSURE) {
        if (!ctx->vir) {
            const int rc = dalloc(ctx, &ctx->vir, N, false);
            if (rc) return rc;
        }
        if (ctx->fp32) {
            // the FP64 planes of the state the virial reads
            const int n = (int)N;
            launch_export32(ctx->P, S, S.pos, S.vel, ctx->st);
            launch_widen_f(S.pres32, S.pres, n, ctx->st);
            launch_widen_f(S.pA32, S.pA, n, ctx->st);
            launch_widen_f4(S.gc4, S.gc, n, n, ctx->st);
        }
        launch_virial(ctx->P, S, ctx->dB, ctx->vir, ctx->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, ctx->vir, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        return DMPH_OK;
    }
    switch (field_id) {
    case DMPH_FIELD_FORCE: return d2h_planes(ctx, S.frc, (double *)out);
    case DMPH_FIELD_GRAVITY_CENTER: return d2h_planes(ctx, S.gc, (double *)out);
    case DMPH_FIELD_VOL_STRAIN_P: src = S.vsp; break;
    case DMPH_FIELD_DIVERGENCE_P: src = S.divp; break;
    case DMPH_FIELD_PRESSURE_P: src = S.pres; break;
    case DMPH_FIELD_DENSITY_A: src = S.densA; break;
    case DMPH_FIELD_PRESSURE_A: src = S.pA; break;
    case DMPH_FIELD_NORMAL_SPRING: src = S.kn; break;
    case DMPH_FIELD_NORMAL_DAMPING: src = S.cn; break;
    case DMPH_FIELD_TANGENTIAL_SPRING: src = S.kt; break;
    case DMPH_FIELD_TANGENTIAL_DAMPING: src = S.ct; break;
    case DMPH_FIELD_ALPHA: src = S.alpha; break;
    case DMPH_FIELD_DRAG_C: src = S.dragC; break;
    case DMPH_FIELD_NEIGHBOR_COUNT:
        CK(cudaMemcpyAsync(out, S.nc, N * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        return DMPH_OK;
    case DMPH_FIELD_SOLID_NEIGHBOR_COUNT:
        CK(cudaMemcpyAsync(out, S.snc, N * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        return DMPH_OK;
    case DMPH_FIELD_CELL_INDEX: {
        std::vector<unsigned long long> w(N);
        CK(cudaMemcpyAsync(w.data(), ctx->words, N * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        int *o = (int *)out;
        for (size_t i = 0; i < N; i++) o[i] = (int)word_key(w[i]);
        return DMPH_OK;
    }
    case DMPH_FIELD_MASS: {
        std::vector<int> t(N);
        CK(cudaMemcpyAsync(t.data(), S.type, N * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        double *o = (double *)out;
        for (size_t i = 0; i < N; i++) o[i] = ctx->P.mass[t[i]];
        return DMPH_OK;
    }
    default: ctx->err = "unknown field id"; return DMPH_EINVAL;
    }
    CK(cudaMemcpyAsync(out, src, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

extern "C" int dmph_get_params(dmph_ctx *ctx, dmph_params *out)
{
    if (!ctx || !out) return DMPH_EINVAL;
    *out = ctx->p;
    out->time = ctx->time;
    return DMPH_OK;
}

extern "C" int dmph_get_rebuild_stats(dmph_ctx *ctx, int64_t *triggers, int64_t *list_builds)
{
    if (!ctx) return DMPH_EINVAL;
    int b[B_COUNT];
    const int rc = read_bounds(ctx, b);
    if (rc) return rc;
    if (triggers) *triggers = b[B_REBUILDS];
    if (list_builds) *list_builds = b[B_LIST_BUILDS];
    return DMPH_OK;
}

extern "C" int dmph_get_info(dmph_ctx *ctx, dmph_info *info)
{
    if (!ctx || !info) return DMPH_EINVAL;
    std::memset(info, 0, sizeof(*info));
    const DevParams &P = ctx->P;
    info->n = P.N;
    int b[B_COUNT];
    const int rc = read_bounds(ctx, b);
    if (rc) return rc;
    info->n_fluid = b[B_FE];
    info->n_solid = b[B_SE] - b[B_SB];
    info->n_wall = P.N - b[B_SE];
    for (int d = 0; d < 3; d++) {
        info->cell_count[d] = P.cc[d];
        info->cell_width[d] = P.cw[d];
    }
    info->total_cell_count = P.T;
    info->power_count = P.P2;
    info->dem_substeps = ctx->demSteps;
    info->steps = ctx->steps;
    info->rebuilds = b[B_REBUILDS];
    info->time = ctx->time;
    info->n0a = P.N0a;
    info->n0p = P.N0p;
    info->r2g = P.R2g;
    info->max_radius = std::sqrt(P.rc2) - 0.1 * P.dx;
    info->num_bodies = ctx->Bd.B;
    info->surface_tension = P.surface_tension;
    {
        const long long graph_rebuilds = b[B_LIST_BUILDS] - ctx->host_rebuilds;
        info->kernel_launches = ctx->launches + ctx->graph_steps * (head_launches(ctx) + tail_launches(ctx, true)) +
                                graph_rebuilds * rebuild_launches(ctx, false);
    }
    return DMPH_OK;
}

// global sums over the fluid and debris slots [0, se): each thread adds its
// grid-stride slots, each block reduces in a fixed order and the blocks'
// partial sums are added in block order, so a state always gives the same bits
constexpr int kSumBlocks = 296, kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_global_sums(DevParams P, DevState S, const int *__restrict__ dB,
                                                            double *__restrict__ part)
{
    const int N = P.N;
    const int se = dB[B_SE];
    double a[DMPH_SUM_COUNT] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < se; i += gridDim.x * blockDim.x) {
        const int t = S.type[i];
        const double m = is_solid(t) ? particle_density(S, P, i, t) * P.V : P.mass[t];
        const double v0 = S.vel[i], v1 = S.vel[N + i], v2 = S.vel[2 * N + i];
        a[DMPH_SUM_MASS] += m;
        a[DMPH_SUM_MOMENTUM_X] += m * v0;
        a[DMPH_SUM_MOMENTUM_Y] += m * v1;
        a[DMPH_SUM_MOMENTUM_Z] += m * v2;
        a[DMPH_SUM_KINETIC] += 0.5 * m * (v0 * v0 + v1 * v1 + v2 * v2);
        a[DMPH_SUM_POTENTIAL] -= m * (P.g[0] * S.pos[i] + P.g[1] * S.pos[N + i] + P.g[2] * S.pos[2 * N + i]);
    }
    __shared__ double red[kSumThreads / 32][DMPH_SUM_COUNT];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < DMPH_SUM_COUNT; ++k) {
        a[k] = warp_sum(a[k]);
        if (lane == 0) red[w][k] = a[k];
    }
    __syncthreads();
    if (threadIdx.x < DMPH_SUM_COUNT) {
        double x = 0.0;
        for (int q = 0; q < kSumThreads / 32; ++q) x += red[q][threadIdx.x];
        part[blockIdx.x * DMPH_SUM_COUNT + threadIdx.x] = x;
    }
}

__global__ void k_global_sums_final(const double *__restrict__ part, double *__restrict__ out)
{
    const int k = threadIdx.x;
    if (k >= DMPH_SUM_COUNT) return;
    double x = 0.0;
    for (int b = 0; b < kSumBlocks; ++b) x += part[b * DMPH_SUM_COUNT + k];
    out[k] = x;
}

extern "C" int dmph_get_global_sums(dmph_ctx *ctx, double sums[DMPH_SUM_COUNT])
{
    if (!ctx || !sums) return DMPH_EINVAL;
    if (!ctx->sums) {  // partial sums and the result, allocated on first use
        const int rc = dalloc(ctx, &ctx->sums, (size_t)(kSumBlocks + 1) * DMPH_SUM_COUNT, false);
        if (rc) return rc;
    }
    if (ctx->fp32) launch_export32(ctx->P, ctx->S, ctx->S.pos, ctx->S.vel, ctx->st);
    k_global_sums<<<kSumBlocks, kSumThreads, 0, ctx->st>>>(ctx->P, ctx->S, ctx->dB, ctx->sums);
    double *out = ctx->sums + (size_t)kSumBlocks * DMPH_SUM_COUNT;
    k_global_sums_final<<<1, 32, 0, ctx->st>>>(ctx->sums, out);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(sums, out, DMPH_SUM_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

// sums of the list lengths over all slots and over the fluid and debris slots
__global__ void k_list_stats(const int *__restrict__ nbn, int n, const int *__restrict__ dB,
                             unsigned long long *__restrict__ out)
{
    const int se = dB[B_SE];
    unsigned long long a = 0, b = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = nbn[i];
        if (c > 0) {
            a += (unsigned long long)c;
            if (i < se) b += (unsigned long long)c;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, a);
        atomicAdd(out + 1, b);
    }
}

extern "C" int dmph_get_list_stats(dmph_ctx *ctx, int64_t *entries_pass_a, int64_t *entries_pass_b,
                                   int32_t *overflowed)
{
    if (!ctx) return DMPH_EINVAL;
    unsigned long long h[2] = {0, 0};
    int ovf = 0;
    if (ctx->use_list) {
        if (!ctx->stats) {  // two counters, allocated on first use
            const int rc = dalloc(ctx, &ctx->stats, 2, false);
            if (rc) return rc;
        }
        CK(cudaMemsetAsync(ctx->stats, 0, 2 * sizeof(unsigned long long), ctx->st));
        k_list_stats<<<ctx->sms * 4, 256, 0, ctx->st>>>(ctx->S.nbn, ctx->P.N, ctx->dB, ctx->stats);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h, ctx->stats, sizeof(h), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(&ovf, ctx->dB + B_LIST_OVF, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    if (entries_pass_a) *entries_pass_a = (int64_t)h[0];
    if (entries_pass_b) *entries_pass_b = (int64_t)h[1];
    if (overflowed) *overflowed = ovf ? 1 : 0;
    return DMPH_OK;
}

extern "C" int dmph_get_neighbor_list(dmph_ctx *ctx, int64_t *ptr, int32_t *ind, int64_t capacity)
{
    if (!ctx || !ptr) return DMPH_EINVAL;
    const DevParams &P = ctx->P;
    const size_t N = (size_t)P.N;
    // counts of every particle at the last rebuild
    launch_counts(P, ctx->S, ctx->dB, CR_ALL, ctx->st);
    CK(cudaGetLastError());
    std::vector<int> nc(N);
    CK(cudaMemcpyAsync(nc.data(), ctx->S.nc, N * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ptr[0] = 0;
    for (size_t i = 0; i < N; i++) ptr[i + 1] = ptr[i] + nc[i];
    int rc = DMPH_OK;
    if (ind) {
        if (capacity < ptr[N]) {
            ctx->err = "neighbour list capacity too small";
            rc = DMPH_ERANGE;
        } else {
            long long *dptr = nullptr;
            int *dind = nullptr;
            CK(cudaMalloc(&dptr, (N + 1) * sizeof(long long)));
            if (cudaMalloc(&dind, (size_t)(ptr[N] > 0 ? ptr[N] : 1) * sizeof(int)) != cudaSuccess) {
                cudaFree(dptr);
                ctx->err = "cudaMalloc of the neighbour list failed";
                return DMPH_ENOMEM;
            }
            cudaMemcpyAsync(dptr, ptr, (N + 1) * sizeof(long long), cudaMemcpyHostToDevice, ctx->st);
            launch_neighbor_fill(P, ctx->S, ctx->dB, dptr, dind, ctx->st);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ind, dind, (size_t)ptr[N] * sizeof(int), cudaMemcpyDeviceToHost, ctx->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
            cudaFree(dptr);
            cudaFree(dind);
            if (e != cudaSuccess) {
                ctx->err = std::string("neighbour list: ") + cudaGetErrorString(e);
                return DMPH_ECUDA;
            }
        }
    }
    // restore the step's own counts (solids only unless all were requested)
    if (!ctx->all_counts) {
        // the hot path reads counts of solids only; the full recount above
        // computed the same values for them, so nothing to restore
    }
    return rc;
}

// 3x3 inverse (FP64, host)
static bool inverse3(const double a[9], double o[9])
{
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (!(std::fabs(det) > 0.0)) return false;
    const double id = 1.0 / det;
    o[0] = c00 * id;
    o[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    o[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    o[3] = c01 * id;
    o[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    o[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    o[6] = c02 * id;
    o[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    o[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

extern "C" int dmph_set_bodies(dmph_ctx *ctx, int nbodies, const int *body_of_row, const double *body_density)
{
    if (!ctx || nbodies <= 0 || !body_of_row || !body_density) return DMPH_EINVAL;
    if (ctx->Bd.B > 0 || ctx->steps > 0) {
        ctx->err = "dmph_set_bodies must be called once, before the first step";
        return DMPH_EINVAL;
    }
    const DevParams &P = ctx->P;
    const int N = P.N;
    std::vector<int> type(N), pidx(N);
    std::vector<double> x(3 * (size_t)N), v(3 * (size_t)N);
    int rc = dmph_get_state(ctx, type.data(), x.data(), v.data(), pidx.data());
    if (rc) return rc;
    // rows -> current data
    std::vector<int> slot_of_row(N);
    for (int i = 0; i < N; i++) slot_of_row[pidx[i]] = i;
    std::vector<std::vector<int>> members(nbodies);
    for (int r = 0; r < N; r++) {
        const int b = body_of_row[r];
        const int t = type[slot_of_row[r]];
        if (b < -1 || b >= nbodies) return ctx->err = "body index out of range", DMPH_EINVAL;
        if (b >= 0 && !is_solid(t)) return ctx->err = "a body member is not a solid particle", DMPH_EINVAL;
        if (b < 0 && is_solid(t)) return ctx->err = "every solid particle must belong to a body", DMPH_EINVAL;
        if (b >= 0) members[b].push_back(r);
    }
    for (int b = 0; b < nbodies; b++) {
        if (members[b].empty()) return ctx->err = "empty body", DMPH_EINVAL;
        if (!(body_density[b] > 0.0)) return ctx->err = "body density must be positive", DMPH_EINVAL;
    }
    std::vector<int> ptr(nbodies + 1, 0), mrow;
    std::vector<double> r0, X(3 * nbodies), V(3 * nbodies), L(3 * nbodies), q(4 * nbodies), M(nbodies),
        Iinv(9 * nbodies);
    for (int b = 0; b < nbodies; b++) {
        const double m = body_density[b] * P.V;
        const auto &mb = members[b];
        // unwrap the members around the first one (periodic domain)
        const double *x0 = &x[3 * (size_t)slot_of_row[mb[0]]];
        double c[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
        std::vector<double> xu(3 * mb.size());
        for (size_t k = 0; k < mb.size(); k++) {
            const int i = slot_of_row[mb[k]];
            for (int d = 0; d < 3; d++) {
                double dd = x[3 * (size_t)i + d] - x0[d];
                dd -= P.W[d] * std::nearbyint(dd / P.W[d]);
                xu[3 * k + d] = x0[d] + dd;
                c[d] += xu[3 * k + d];
                vc[d] += v[3 * (size_t)i + d];
            }
        }
        for (int d = 0; d < 3; d++) {
            c[d] /= (double)mb.size();
            vc[d] /= (double)mb.size();
        }
        const double a = 0.4 * m * (0.5 * P.dx) * (0.5 * P.dx);  // solid-sphere inertia of each particle
        double I[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Lb[3] = {0, 0, 0};
        for (size_t k = 0; k < mb.size(); k++) {
            const int i = slot_of_row[mb[k]];
            const double r[3] = {xu[3 * k] - c[0], xu[3 * k + 1] - c[1], xu[3 * k + 2] - c[2]};
            const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            for (int p = 0; p < 3; p++)
                for (int qq = 0; qq < 3; qq++) I[3 * p + qq] += m * ((p == qq ? rr : 0.0) - r[p] * r[qq]);
            for (int p = 0; p < 3; p++) I[4 * p] += a;
            const double u[3] = {v[3 * (size_t)i] - vc[0], v[3 * (size_t)i + 1] - vc[1], v[3 * (size_t)i + 2] - vc[2]};
            Lb[0] += m * (r[1] * u[2] - r[2] * u[1]);
            Lb[1] += m * (r[2] * u[0] - r[0] * u[2]);
            Lb[2] += m * (r[0] * u[1] - r[1] * u[0]);
            mrow.push_back(mb[k]);
            for (int d = 0; d < 3; d++) r0.push_back(r[d]);
        }
        ptr[b + 1] = (int)mrow.size();
        if (!inverse3(I, &Iinv[9 * b])) return ctx->err = "singular body inertia", DMPH_EINVAL;
        for (int d = 0; d < 3; d++) {
            X[3 * b + d] = c[d];
            V[3 * b + d] = vc[d];
            L[3 * b + d] = Lb[d];
        }
        q[4 * b] = 1.0;
        q[4 * b + 1] = q[4 * b + 2] = q[4 * b + 3] = 0.0;
        M[b] = m * (double)mb.size();
    }
    // device arrays
    const size_t nm = mrow.size();
    DevBodies &Bd = ctx->Bd;
    int *dptr = nullptr, *dmrow = nullptr, *dsor = nullptr, *dbid = nullptr, *dbid2 = nullptr;
    double *dr0 = nullptr, *dX = nullptr, *dV = nullptr, *dL = nullptr, *dq = nullptr, *dM = nullptr, *dI = nullptr,
           *dF = nullptr, *dT = nullptr, *drho = nullptr, *dfd = nullptr;
#define AB(ptr_, cnt_)                                      \
    do {                                                    \
        int r_ = dalloc(ctx, &(ptr_), (size_t)(cnt_));      \
        if (r_) return r_;                                  \
    } while (0)
    AB(dptr, nbodies + 1);
    AB(dmrow, nm);
    AB(dsor, N);
    AB(dbid, N);
    AB(dbid2, N);
    AB(dr0, 3 * nm);
    AB(dX, 3 * nbodies);
    AB(dV, 3 * nbodies);
    AB(dL, 3 * nbodies);
    AB(dq, 4 * nbodies);
    AB(dM, nbodies);
    AB(dI, 9 * nbodies);
    AB(dF, 3 * nbodies);
    AB(dT, 3 * nbodies);
    AB(drho, nbodies);
    AB(dfd, 6 * (size_t)N);
#undef AB
    std::vector<int> bid(N);
    for (int i = 0; i < N; i++) bid[i] = body_of_row[pidx[i]];
    CK(cudaMemcpyAsync(dptr, ptr.data(), (nbodies + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dmrow, mrow.data(), nm * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dsor, slot_of_row.data(), N * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dbid, bid.data(), N * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dr0, r0.data(), 3 * nm * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dX, X.data(), 3 * nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dV, V.data(), 3 * nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dL, L.data(), 3 * nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dq, q.data(), 4 * nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dM, M.data(), nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dI, Iinv.data(), 9 * nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(drho, body_density, nbodies * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    Bd.B = nbodies;
    Bd.ptr = dptr;
    Bd.member_row = dmrow;
    Bd.slot_of_row = dsor;
    Bd.r0 = dr0;
    Bd.X = dX;
    Bd.V = dV;
    Bd.L = dL;
    Bd.q = dq;
    Bd.M = dM;
    Bd.Iinv0 = dI;
    Bd.Fsum = dF;
    Bd.Tsum = dT;
    ctx->S.bid = dbid;
    ctx->bid2 = dbid2;
    ctx->S.body_rho = drho;
    ctx->S.frc_dem = dfd;
    ctx->body_of_row.assign(body_of_row, body_of_row + N);
    ctx->body_density.assign(body_density, body_density + nbodies);
    return DMPH_OK;
}

extern "C" int dmph_get_bodies(dmph_ctx *ctx, double *X, double *V, double *q, double *L, double *mass, double *F,
                               double *T)
{
    if (!ctx) return DMPH_EINVAL;
    const DevBodies &Bd = ctx->Bd;
    const size_t B = (size_t)Bd.B;
    if (B == 0) return DMPH_OK;
    if (X) CK(cudaMemcpyAsync(X, Bd.X, 3 * B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (V) CK(cudaMemcpyAsync(V, Bd.V, 3 * B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (q) CK(cudaMemcpyAsync(q, Bd.q, 4 * B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (L) CK(cudaMemcpyAsync(L, Bd.L, 3 * B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (mass) CK(cudaMemcpyAsync(mass, Bd.M, B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (F) CK(cudaMemcpyAsync(F, Bd.Fsum, 3 * B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (T) CK(cudaMemcpyAsync(T, Bd.Tsum, 3 * B * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return DMPH_OK;
}

extern "C" int dmph_set_pair_mode(dmph_ctx *ctx, int mode)
{
    if (!ctx) return DMPH_EINVAL;
    if (mode != DMPH_PAIRS_STENCIL && mode != DMPH_PAIRS_VERLET_LIST) return DMPH_EINVAL;
    const bool want = mode == DMPH_PAIRS_VERLET_LIST;
    if (want && !ctx->use_list) {
        // lists of the current cell sort
        if (ctx->fp32)
            launch_build_list32(ctx->P, ctx->Q, ctx->S, ctx->dB, ctx->Wm.moving ? 0 : 1, ctx->st, ctx->var_build);
        else launch_build_list64(ctx->P, ctx->S, ctx->dB, ctx->st);
        if (ctx->list_reuse) {
            // lists of the MARGIN skin, made away from a rebuild: the next
            // trigger remakes them
            const int ten = 10;
            CK(cudaMemcpyAsync(ctx->dB + B_SKIN, &ten, sizeof(int), cudaMemcpyHostToDevice, ctx->st));
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->st));
    }
    ctx->use_list = want;
    drop_graph(ctx);
    return DMPH_OK;
}

extern "C" int dmph_set_graph(dmph_ctx *ctx, int enable)
{
    if (!ctx) return DMPH_EINVAL;
    ctx->use_graph = enable != 0;
    return DMPH_OK;
}

extern "C" int dmph_set_profiling(dmph_ctx *ctx, int enable)
{
    if (!ctx) return DMPH_EINVAL;
    ctx->prof = enable != 0;
    for (int k = 0; k < DMPH_PHASE_COUNT; k++) {
        ctx->phase_ms[k] = 0.0;
        ctx->phase_n[k] = 0;
    }
    return DMPH_OK;
}

extern "C" int dmph_get_phase_times(dmph_ctx *ctx, double *ms, int64_t *launches, int n)
{
    if (!ctx || n < 0) return DMPH_EINVAL;
    for (int k = 0; k < n && k < DMPH_PHASE_COUNT; k++) {
        if (ms) ms[k] = ctx->phase_ms[k];
        if (launches) launches[k] = ctx->phase_n[k];
    }
    return DMPH_OK;
}

extern "C" int dmph_destroy(dmph_ctx *ctx)
{
    if (!ctx) return DMPH_OK;  // like free(NULL)
    release(ctx);
    delete ctx;
    return DMPH_OK;
}

namespace dmph {
void set_noctx_message(const char *literal) { g_noctx_literal = literal; }
void set_noctx_error(const std::string &msg)
{
    g_noctx_literal = nullptr;
    g_create_err = msg;
}
}  // namespace dmph

extern "C" const char *dmph_last_error(dmph_ctx *ctx)
{
    if (!ctx) return g_noctx_literal ? g_noctx_literal : g_create_err.c_str();
    return ctx->err.c_str();
}

extern "C" const char *dmph_version(void)
{
    static const std::string v = std::string("libdmph ") + std::to_string(DMPH_ABI_VERSION) +
                                 " sm_100a nvcc " + std::to_string(__CUDACC_VER_MAJOR__) + "." +
                                 std::to_string(__CUDACC_VER_MINOR__);
    return v.c_str();
}

// ------------------------------------------------------------- autotuner
// Times every launch variant of a pair pass on the live state (the passes are
// pure functions of the state they read, so repeating them changes nothing)
// and keeps the fastest.
template <class Launch>
static int time_variants(dmph_ctx *ctx, cudaStream_t st, Launch &&launch, float *ms_out, int *best,
                         int nvar = kPassVariants)
{
    float best_ms = 1e30f;
    *best = 0;
    for (int v = 0; v < nvar; ++v) {
        launch(v);  // warm-up: first launch of a variant also sizes its grid
        CK(cudaEventRecord(ctx->ev0, st));
        for (int r = 0; r < 3; ++r) launch(v);
        CK(cudaEventRecord(ctx->ev1, st));
        CK(cudaEventSynchronize(ctx->ev1));
        CK(cudaGetLastError());
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        ms /= 3.f;
        if (ms_out) ms_out[v] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            *best = v;
        }
    }
    return DMPH_OK;
}

extern "C" int dmph_autotune(dmph_ctx *ctx, int *variant_a, int *variant_b, float *ms_a, float *ms_b)
{
    if (!ctx) return DMPH_EINVAL;
    if (!ctx->fp32) {
        ctx->err = "dmph_autotune: the FP64 parity build has one launch shape";
        return DMPH_EINVAL;
    }
    const DevParams &P = ctx->P;
    const DevParams32 &Q = ctx->Q;
    if (ctx->use_list) {
        // list mode: the variants of the list passes (the lists of the last
        // rebuild are valid for the current state)
        int rc = time_variants(ctx, ctx->st, [&](int v) { launch_pass_a32_list(P, Q, ctx->S, ctx->dB, v, ctx->st); },
                               ms_a, &ctx->var_la, kListVariants);
        if (rc) return rc;
        launch_pass_a32_list(P, Q, ctx->S, ctx->dB, ctx->var_la, ctx->st);
        rc = time_variants(ctx, ctx->st, [&](int v) { launch_pass_b32_list(P, Q, ctx->S, ctx->dB, v, ctx->st); },
                           ms_b, &ctx->var_lb, kListVariants);
        if (rc) return rc;
        launch_pass_b32_list(P, Q, ctx->S, ctx->dB, ctx->var_lb, ctx->st);
        CK(cudaStreamSynchronize(ctx->st));
        drop_graph(ctx);
        if (variant_a) *variant_a = ctx->var_la;
        if (variant_b) *variant_b = ctx->var_lb;
        return DMPH_OK;
    }
    int rc = time_variants(ctx, ctx->st, [&](int v) { launch_pass_a32(P, Q, ctx->S, ctx->dB, CR_WET, v, ctx->st); },
                           ms_a, &ctx->var_a);
    if (rc) return rc;
    // pass A of the chosen variant last, so the pressures pass B reads are its own
    launch_pass_a32(P, Q, ctx->S, ctx->dB, CR_WET, ctx->var_a, ctx->st);
    rc = time_variants(ctx, ctx->st, [&](int v) { launch_pass_b32(P, Q, ctx->S, ctx->dB, v, ctx->st); }, ms_b,
                       &ctx->var_b);
    if (rc) return rc;
    launch_pass_b32(P, Q, ctx->S, ctx->dB, ctx->var_b, ctx->st);
    CK(cudaStreamSynchronize(ctx->st));
    drop_graph(ctx);
    if (variant_a) *variant_a = ctx->var_a;
    if (variant_b) *variant_b = ctx->var_b;
    return DMPH_OK;
}

extern "C" int dmph_autotune_list_build(dmph_ctx *ctx, int steps_per_variant, int *variant, float *ms)
{
    if (!ctx || steps_per_variant <= 0) return DMPH_EINVAL;
    if (!ctx->fp32 || !ctx->use_list) {
        ctx->err = "dmph_autotune_list_build: FP32 split build in Verlet-list mode only";
        return DMPH_EINVAL;
    }
    // every variant builds the same lists, so the steps it times are the
    // steps the caller would have run anyway
    const bool graph = ctx->use_graph;
    drop_graph(ctx);
    ctx->use_graph = false;
    const bool prof = ctx->prof;
    int best = ctx->var_build;
    float best_ms = 1e30f;
    int rc = DMPH_OK;
    for (int v = 0; v < kBuildVariants && !rc; ++v) {
        ctx->var_build = v;
        dmph_set_profiling(ctx, 1);
        rc = dmph_step(ctx, steps_per_variant);
        const long long n = ctx->phase_n[6];
        const float t = n > 0 ? (float)(ctx->phase_ms[6] / (double)n) : -1.f;
        if (ms) ms[v] = t;
        if (!rc && n > 0 && t < best_ms) {
            best_ms = t;
            best = v;
        }
    }
    dmph_set_profiling(ctx, prof ? 1 : 0);
    ctx->var_build = best;
    ctx->use_graph = graph;
    if (variant) *variant = best;
    return rc;
}

extern "C" int dmph_set_variants(dmph_ctx *ctx, int variant_a, int variant_b)
{
    if (!ctx) return DMPH_EINVAL;
    const int nv = ctx->use_list ? kListVariants : kPassVariants;
    if (variant_a < 0 || variant_a >= nv || variant_b < 0 || variant_b >= nv) {
        ctx->err = "launch variant out of range";
        return DMPH_ERANGE;
    }
    if (ctx->use_list) {
        ctx->var_la = variant_a;
        ctx->var_lb = variant_b;
    } else {
        ctx->var_a = variant_a;
        ctx->var_b = variant_b;
    }
    drop_graph(ctx);
    return DMPH_OK;
}

// ------------------------------------------------------------- ensemble
struct dmph_ensemble {
    std::vector<dmph_ctx *> scenes;
    EnsScene *tab = nullptr;  // device scene table
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> fork;  // one per scene: scene joined the ensemble stream
    cudaEvent_t join = nullptr;
    int var_a = 0, var_b = 0;
    bool use_graph = true;
    bool use_list = false;  // pair passes over the members' Verlet lists
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long long launches = 0, steps = 0, graph_steps = 0;
    std::string err;
    dmph_ctx *ctx0 = nullptr;  // for error strings of the helpers
    // fused: every scene's drift and rebuild decision run as one launch each,
    // and the DEM / rigid-body tails of all scenes as one launch per kernel
    // (list mode, walls at rest, debris as rigid bodies or none)
    bool fused = false;
    int max_dem = 0;                        // most DEM substeps of any scene
    int total_bodies = 0;
    int *bpre = nullptr;                    // device: prefix of the scenes' body counts
    unsigned long long *handles = nullptr;  // device: the IF-node conditions of the recorded step
    // per-phase timing of the ensemble passes (dmph_ensemble_set_profiling)
    bool prof = false;
    cudaEvent_t pe0 = nullptr, pe1 = nullptr;
    double phase_ms[DMPH_PHASE_COUNT] = {0};
    long long phase_n[DMPH_PHASE_COUNT] = {0};
};

#define EK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            e->err = std::string(#call) + ": " + cudaGetErrorString(e_);                  \
            return DMPH_ECUDA;                                                            \
        }                                                                                 \
    } while (0)

static void ens_drop_graph(dmph_ensemble *e)
{
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->gexec = nullptr;
    e->graph = nullptr;
}

static void ens_release(dmph_ensemble *e)
{
    if (e->st) cudaStreamSynchronize(e->st);
    ens_drop_graph(e);
    if (e->tab) cudaFree(e->tab);
    if (e->bpre) cudaFree(e->bpre);
    if (e->handles) cudaFree(e->handles);
    e->bpre = nullptr;
    e->handles = nullptr;
    for (cudaEvent_t v : e->fork) cudaEventDestroy(v);
    if (e->join) cudaEventDestroy(e->join);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->pe0) cudaEventDestroy(e->pe0);
    if (e->pe1) cudaEventDestroy(e->pe1);
    if (e->st) cudaStreamDestroy(e->st);
    e->tab = nullptr;
    e->fork.clear();
    e->join = e->ev0 = e->ev1 = e->pe0 = e->pe1 = nullptr;
    e->st = nullptr;
}

extern "C" int dmph_ensemble_create(dmph_ctx *const *scenes, int nscenes, dmph_ensemble **out)
{
    if (!out) return DMPH_EINVAL;
    *out = nullptr;
    if (!scenes || nscenes <= 0 || nscenes > kMaxEnsemble) return DMPH_ERANGE;
    int dev = -1;
    for (int k = 0; k < nscenes; ++k) {
        dmph_ctx *c = scenes[k];
        if (!c || !c->fp32) return DMPH_EINVAL;  // the ensemble kernels are the FP32 split passes
        if (c->list_reuse) {
            c->err = "list reuse (DMPH_FLAG_LIST_REUSE) is not supported in an ensemble";
            return DMPH_EINVAL;
        }
        for (int j = 0; j < k; ++j)
            if (scenes[j] == c) return DMPH_EINVAL;
        if (dev < 0) dev = c->device;
        if (c->device != dev) return DMPH_EINVAL;
    }
    cudaSetDevice(dev);
    dmph_ensemble *e = new dmph_ensemble();
    e->scenes.assign(scenes, scenes + nscenes);
    e->ctx0 = scenes[0];
    std::vector<EnsScene> h(nscenes);
    for (int k = 0; k < nscenes; ++k) {
        dmph_ctx *c = scenes[k];
        h[k].P = c->P;
        h[k].Q = c->Q;
        h[k].S = c->S;
        h[k].dB = c->dB;
        h[k].maxshift = c->maxshift;
        h[k].Bd = c->Bd;
        h[k].demSteps = c->demSteps;
    }
    cudaError_t ce = cudaMalloc((void **)&e->tab, sizeof(EnsScene) * nscenes);
    if (ce == cudaSuccess) ce = cudaMemcpy(e->tab, h.data(), sizeof(EnsScene) * nscenes, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e->ev0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e->ev1);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e->pe0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e->pe1);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->join, cudaEventDisableTiming);
    e->fork.assign(nscenes, nullptr);
    for (int k = 0; ce == cudaSuccess && k < nscenes; ++k)
        ce = cudaEventCreateWithFlags(&e->fork[k], cudaEventDisableTiming);
    if (ce != cudaSuccess) {
        ens_release(e);
        delete e;
        return DMPH_ECUDA;
    }
    // list mode when every member is in list mode
    e->use_list = true;
    for (dmph_ctx *c : e->scenes) e->use_list = e->use_list && c->use_list;
    if (!e->use_list)
        for (dmph_ctx *c : e->scenes) c->use_list = false;
    for (dmph_ctx *c : e->scenes) drop_graph(c);
    // fused heads and tails
    e->fused = e->use_list;
    std::vector<int> bpre(nscenes + 1, 0);
    for (int k = 0; k < nscenes; ++k) {
        dmph_ctx *c = e->scenes[k];
        e->fused = e->fused && c->walls_rest && (c->Bd.B > 0 || c->n_solid == 0);
        e->max_dem = std::max(e->max_dem, c->demSteps);
        bpre[k + 1] = bpre[k] + c->Bd.B;
    }
    e->total_bodies = bpre[nscenes];
    if (e->fused) {
        ce = cudaMalloc((void **)&e->bpre, sizeof(int) * (nscenes + 1));
        if (ce == cudaSuccess)
            ce = cudaMemcpy(e->bpre, bpre.data(), sizeof(int) * (nscenes + 1), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMalloc((void **)&e->handles, sizeof(unsigned long long) * nscenes);
        // the drift accumulates into cleared accumulators; the decision clears them after
        for (int k = 0; ce == cudaSuccess && k < nscenes; ++k)
            ce = cudaMemset(e->scenes[k]->maxshift, 0, sizeof(unsigned long long));
        if (ce != cudaSuccess) {
            ens_release(e);
            delete e;
            return DMPH_ECUDA;
        }
    }
    *out = e;
    return DMPH_OK;
}

// the pair passes of all scenes: one persistent launch each
// profiling (never inside a graph): events around a phase on the ensemble
// stream, accumulated into phase k
static void ens_phase_begin(dmph_ensemble *e)
{
    if (e->prof) cudaEventRecord(e->pe0, e->st);
}
static void ens_phase_end(dmph_ensemble *e, int k)
{
    if (!e->prof) return;
    cudaEventRecord(e->pe1, e->st);
    cudaEventSynchronize(e->pe1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e->pe0, e->pe1);
    e->phase_ms[k] += ms;
    e->phase_n[k] += 1;
}

static void ens_enqueue_passes(dmph_ensemble *e)
{
    const int ns = (int)e->scenes.size();
    if (e->use_list) {
        ens_phase_begin(e);
        launch_ens_pass_list(e->tab, ns, false, e->st);
        launch_ens_pass_a32(e->tab, ns, e->var_a, e->st, 1);
        ens_phase_end(e, 2);
        ens_phase_begin(e);
        launch_ens_pass_list(e->tab, ns, true, e->st);
        launch_ens_pass_b32(e->tab, ns, e->var_b, e->st, 1);
        ens_phase_end(e, 3);
    } else {
        ens_phase_begin(e);
        launch_ens_pass_a32(e->tab, ns, e->var_a, e->st);
        ens_phase_end(e, 2);
        ens_phase_begin(e);
        launch_ens_pass_b32(e->tab, ns, e->var_b, e->st);
        ens_phase_end(e, 3);
    }
    launch_ens_fluid_accel32(e->tab, ns, e->st);
}

// kernels of one fused ensemble step outside the scenes' rebuilds
static long long ens_fused_launches(const dmph_ensemble *e)
{
    return 2 + (e->use_list ? 6 : 3) + 2 + 3LL * e->max_dem;
}

// One fused ensemble step: one drift launch and one decision launch for all
// scenes, each scene's rebuild when its decision asks for one (an IF node per
// scene when conds is given, set by the decision kernel; else read on the
// host), the ensemble passes, then the DEM tails of all scenes as one launch
// per kernel and substep.
static int ens_enqueue_fused(dmph_ensemble *e, const std::vector<cudaGraphConditionalHandle> *conds)
{
    const int ns = (int)e->scenes.size();
    for (dmph_ctx *c : e->scenes) c->Wm.moving = 0;  // walls at rest in every scene
    launch_ens_drift32(e->tab, ns, e->ctx0->sms, e->st);
    launch_ens_decide(e->tab, ns, conds ? e->handles : nullptr, e->st);
    EK(cudaEventRecord(e->join, e->st));
    for (int k = 0; k < ns; ++k) {
        dmph_ctx *c = e->scenes[k];
        EK(cudaStreamWaitEvent(c->st, e->join, 0));
        if (conds) {
            const int rc = capture_rebuild_if(c, (*conds)[k], c->st);
            if (rc) {
                e->err = c->err;
                return rc;
            }
        } else {
            EK(cudaMemcpyAsync(c->h_small, c->dB + B_NEED, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        }
    }
    if (!conds) {
        for (dmph_ctx *c : e->scenes) {
            EK(cudaStreamSynchronize(c->st));
            if (c->h_small[0]) {
                enqueue_rebuild(c, false, c->st);
                c->launches += rebuild_launches(c, false);
                c->host_rebuilds++;
            }
        }
    }
    for (int k = 0; k < ns; ++k) {
        EK(cudaEventRecord(e->fork[k], e->scenes[k]->st));
        EK(cudaStreamWaitEvent(e->st, e->fork[k], 0));
    }
    ens_enqueue_passes(e);
    launch_ens_solid_force_to64(e->tab, ns, e->st);
    for (int sub = 0; sub < e->max_dem; ++sub) {
        launch_ens_clump_dem(e->tab, ns, sub, e->st);
        launch_ens_body_step(e->tab, ns, e->bpre, e->total_bodies, sub, e->st);
    }
    launch_ens_sync_solids32(e->tab, ns, e->st);
    EK(cudaGetLastError());
    return DMPH_OK;
}

// Enqueue one ensemble step.  graph_mode: the heads carry conditional rebuild
// nodes (capture); otherwise the rebuild decisions are read on the host.
static int ens_enqueue_step(dmph_ensemble *e, cudaGraph_t g)
{
    const int ns = (int)e->scenes.size();
    // heads (and rebuilds) of every scene on its own stream
    EK(cudaEventRecord(e->join, e->st));
    for (int k = 0; k < ns; ++k) {
        dmph_ctx *c = e->scenes[k];
        c->Wm.moving = in_wall_window(c) ? 1 : 0;
        EK(cudaStreamWaitEvent(c->st, e->join, 0));
        if (g) {
            const int rc = capture_head_and_rebuild(c, g, c->st);
            if (rc) {
                e->err = c->err;
                return rc;
            }
        } else {
            enqueue_head(c, 0, c->st);
            EK(cudaMemcpyAsync(c->h_small, c->dB + B_NEED, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        }
    }
    if (!g) {
        for (int k = 0; k < ns; ++k) {
            dmph_ctx *c = e->scenes[k];
            EK(cudaStreamSynchronize(c->st));
            c->launches += 2;
            if (c->h_small[0]) {
                enqueue_rebuild(c, false, c->st);
                c->launches += rebuild_launches(c, false);
                c->host_rebuilds++;
            }
            if (e->use_list && c->Wm.moving) {
                launch_list_wall_guard(c->dB, c->st);
                c->launches++;
            }
        }
    }
    for (int k = 0; k < ns; ++k) {
        EK(cudaEventRecord(e->fork[k], e->scenes[k]->st));
        EK(cudaStreamWaitEvent(e->st, e->fork[k], 0));
    }
    ens_enqueue_passes(e);
    EK(cudaGetLastError());
    EK(cudaEventRecord(e->join, e->st));
    // DEM / rigid bodies per scene, then join
    for (int k = 0; k < ns; ++k) {
        dmph_ctx *c = e->scenes[k];
        EK(cudaStreamWaitEvent(c->st, e->join, 0));
        enqueue_dem(c, c->st);
        EK(cudaEventRecord(e->fork[k], c->st));
        EK(cudaStreamWaitEvent(e->st, e->fork[k], 0));
    }
    EK(cudaGetLastError());
    return DMPH_OK;
}

static long long ens_step_launches(const dmph_ensemble *e)
{
    if (e->fused) return ens_fused_launches(e);
    long long n = 3 + (e->use_list ? 3 : 0);  // list passes: A, B fluid, B debris
    for (const dmph_ctx *c : e->scenes) n += 2 + dem_launches(c);
    return n;
}

static bool ens_graph_usable(const dmph_ensemble *e)
{
    if (!e->use_graph || e->prof) return false;
    for (const dmph_ctx *c : e->scenes)
        if (c->prof || !(0.0 < c->time) || in_wall_window(c)) return false;
    return true;
}

static int ens_build_graph(dmph_ensemble *e)
{
    cudaGraph_t g = nullptr;
    EK(cudaGraphCreate(&g, 0));
    std::vector<cudaGraphConditionalHandle> conds;
    if (e->fused) {
        // one condition per scene, set by the ensemble decision kernel
        const int ns = (int)e->scenes.size();
        conds.resize(ns);
        std::vector<unsigned long long> h(ns);
        for (int k = 0; k < ns; ++k) {
            EK(cudaGraphConditionalHandleCreate(&conds[k], g, 0, cudaGraphCondAssignDefault));
            h[k] = (unsigned long long)conds[k];
        }
        EK(cudaMemcpy(e->handles, h.data(), sizeof(unsigned long long) * ns, cudaMemcpyHostToDevice));
    }
    EK(cudaStreamBeginCaptureToGraph(e->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const int rc = e->fused ? ens_enqueue_fused(e, &conds) : ens_enqueue_step(e, g);
    cudaGraph_t g2 = g;
    const cudaError_t ce = cudaStreamEndCapture(e->st, &g2);
    if (rc || ce != cudaSuccess) {
        cudaGraphDestroy(g);
        if (!rc) e->err = std::string("ensemble capture: ") + cudaGetErrorString(ce);
        return rc ? rc : DMPH_ECUDA;
    }
    EK(cudaGraphInstantiate(&e->gexec, g, 0));
    e->graph = g;
    return DMPH_OK;
}

static int ens_step_once(dmph_ensemble *e)
{
    if (ens_graph_usable(e)) {
        if (!e->gexec) {
            const int rc = ens_build_graph(e);
            if (rc) return rc;
        }
        EK(cudaGraphLaunch(e->gexec, e->st));
        e->graph_steps++;
    } else if (e->fused) {
        const int rc = ens_enqueue_fused(e, nullptr);
        if (rc) return rc;
        e->launches += ens_fused_launches(e);
    } else {
        const int rc = ens_enqueue_step(e, nullptr);
        if (rc) return rc;
        e->launches += 3 + (e->use_list ? 2 : 0);
        for (dmph_ctx *c : e->scenes) c->launches += dem_launches(c);
    }
    for (dmph_ctx *c : e->scenes) {
        advance_host_clock(c);
    }
    e->steps++;
    return DMPH_OK;
}

// DMPH_ENAN when a scene's drift met a non-finite position or velocity
static int ens_check_finite(dmph_ensemble *e)
{
    for (size_t k = 0; k < e->scenes.size(); ++k) {
        dmph_ctx *c = e->scenes[k];
        if (check_finite(c) == DMPH_ENAN) {
            e->err = "scene " + std::to_string(k) + ": " + c->err;
            return DMPH_ENAN;
        }
    }
    return DMPH_OK;
}

extern "C" int dmph_ensemble_step(dmph_ensemble *e, int nsteps)
{
    if (!e || nsteps < 0) return DMPH_EINVAL;
    for (int s = 0; s < nsteps; ++s) {
        const int rc = ens_step_once(e);
        if (rc) return rc;
    }
    EK(cudaStreamSynchronize(e->st));
    return ens_check_finite(e);
}

extern "C" int dmph_ensemble_step_timed(dmph_ensemble *e, int nsteps, float *device_ms)
{
    if (!e || nsteps < 0) return DMPH_EINVAL;
    EK(cudaEventRecord(e->ev0, e->st));
    for (int s = 0; s < nsteps; ++s) {
        const int rc = ens_step_once(e);
        if (rc) return rc;
    }
    EK(cudaEventRecord(e->ev1, e->st));
    EK(cudaEventSynchronize(e->ev1));
    float ms = 0.f;
    EK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    if (device_ms) *device_ms = ms;
    return ens_check_finite(e);
}

extern "C" int dmph_ensemble_autotune(dmph_ensemble *e, int *variant_a, int *variant_b, float *ms_a, float *ms_b)
{
    if (!e) return DMPH_EINVAL;
    const int ns = (int)e->scenes.size();
    dmph_ctx *ctx = e->ctx0;
    for (dmph_ctx *c : e->scenes) cudaStreamSynchronize(c->st);
    int rc = time_variants(ctx, e->st, [&](int v) { launch_ens_pass_a32(e->tab, ns, v, e->st); }, ms_a, &e->var_a);
    if (rc) {
        e->err = ctx->err;
        return rc;
    }
    launch_ens_pass_a32(e->tab, ns, e->var_a, e->st);
    rc = time_variants(ctx, e->st, [&](int v) { launch_ens_pass_b32(e->tab, ns, v, e->st); }, ms_b, &e->var_b);
    if (rc) {
        e->err = ctx->err;
        return rc;
    }
    launch_ens_pass_b32(e->tab, ns, e->var_b, e->st);
    EK(cudaStreamSynchronize(e->st));
    ens_drop_graph(e);
    if (variant_a) *variant_a = e->var_a;
    if (variant_b) *variant_b = e->var_b;
    return DMPH_OK;
}

extern "C" int dmph_ensemble_set_graph(dmph_ensemble *e, int enable)
{
    if (!e) return DMPH_EINVAL;
    e->use_graph = enable != 0;
    return DMPH_OK;
}

extern "C" int dmph_ensemble_info(dmph_ensemble *e, int64_t *kernel_launches, int64_t *steps)
{
    if (!e) return DMPH_EINVAL;
    if (kernel_launches) {
        // graph steps: every scene's head, the ensemble passes and every tail
        // (rebuilds inside graphs are counted by the scenes' own counters)
        *kernel_launches = e->launches + e->graph_steps * ens_step_launches(e);
    }
    if (steps) *steps = e->steps;
    return DMPH_OK;
}

extern "C" const char *dmph_ensemble_last_error(dmph_ensemble *e)
{
    return e ? e->err.c_str() : "null ensemble";
}

extern "C" int dmph_ensemble_set_profiling(dmph_ensemble *e, int enable)
{
    if (!e) return DMPH_EINVAL;
    e->prof = enable != 0;
    for (int k = 0; k < DMPH_PHASE_COUNT; k++) {
        e->phase_ms[k] = 0.0;
        e->phase_n[k] = 0;
    }
    return DMPH_OK;
}

extern "C" int dmph_ensemble_get_phase_times(dmph_ensemble *e, double *ms, int64_t *launches, int n)
{
    if (!e || n < 0) return DMPH_EINVAL;
    for (int k = 0; k < n && k < DMPH_PHASE_COUNT; k++) {
        if (ms) ms[k] = e->phase_ms[k];
        if (launches) launches[k] = e->phase_n[k];
    }
    return DMPH_OK;
}

extern "C" int dmph_ensemble_destroy(dmph_ensemble *e)
{
    if (!e) return DMPH_OK;
    ens_release(e);
    delete e;
    return DMPH_OK;
}

