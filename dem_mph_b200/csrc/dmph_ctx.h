// The solver context behind the C ABI and the step helpers shared by the
// step driver (dmph_api.cu) and the surrogate driver (dmph_surrogate.cu).
#pragma once

#include <string>
#include <vector>

#include "dmph.h"
#include "dmph_internal.h"

namespace dmph {
struct Surrogate;
}

// private header of the library: the context is written with the library's own types
using namespace dmph;

struct dmph_ctx {
    dmph_params p;
    DevParams P;
    DevParams32 Q;
    bool fp32 = false;
    // every wall type has zero velocity and zero angular velocity: in the FP32
    // build the 0.2-0.4 s wall window then moves nothing (the FP32 positions
    // keep their bits), so it is stepped like any other time
    bool walls_rest = false;
    WallMotion Wm;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int sms = 148;
    int device = 0;
    DevState S{};
    // second buffers of the permuted arrays
    double *pos2 = nullptr, *vel2 = nullptr;
    int *type2 = nullptr, *pidx2 = nullptr;
    float4 *p4b = nullptr, *v4b = nullptr;  // second buffers of the FP32 state
    int *bid2 = nullptr;                     // second buffer of the body ids
    DevBodies Bd{};                          // rigid clumps (B = 0: off)
    unsigned long long *words = nullptr;
    // FP32 counting sort (csort): per-particle keys, per-key counts and the
    // scattered words before each key's range is ordered
    bool csort = false;
    int n_solid = 0;  // debris particles (types 2-3) of the scene
    int n_fluid = 0;  // fluid particles (types 0-1)
    int *ckeys = nullptr, *ccounts = nullptr;
    unsigned long long *words2 = nullptr;
    int *flag = nullptr, *offs = nullptr, *bsums = nullptr, *total = nullptr;
    unsigned long long *maxshift = nullptr;
    // list reuse (DMPH_FLAG_LIST_REUSE): largest displacement since the
    // lists were built, and whether the flag was given
    unsigned long long *maxshiftL = nullptr;
    bool list_reuse = false;
    unsigned long long *stats = nullptr;      // dmph_get_list_stats counters
    double *sums = nullptr;                   // dmph_get_global_sums partials and result
    unsigned long long *h_maxshift = nullptr;  // pinned
    int *h_small = nullptr;                    // pinned scratch for small read-backs
    int *dB = nullptr;         // device bounds (DevBound)
    cudaStream_t st2 = nullptr;      // capture stream of the rebuild body
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long long graph_steps = 0, host_rebuilds = 0;
    int var_a = 0, var_b = 0;  // launch variants of the FP32 pair passes (dmph_autotune)
    bool use_list = false;     // FP32 pair passes over Verlet lists built at each rebuild
    int var_la = 1, var_lb = 1;  // launch variants of the list passes
    int var_build = 0;           // launch variant of the FP32 list build (dmph_autotune_list_build)
    double *vir = nullptr;        // virial pressure (allocated on the first request)
    Chunk *chunks2 = nullptr;  // partition scratch
    int demSteps = 0;
    double time = 0.0;
    long long steps = 0, rebuilds = 0;
    long long launches = 0;  // kernels launched by dmph_step
    bool all_counts = false;
    bool prof = false;
    bool nonfinite = false;  // a step met a non-finite position or velocity (until dmph_set_state)
    bool in_split_step = false;  // dmph_step_begin ran, dmph_step_finish not yet
    double split_m2 = 0.0;       // the max shift dmph_step_begin reported
    cudaEvent_t pe0 = nullptr, pe1 = nullptr, pl0 = nullptr, pl1 = nullptr;
    double phase_ms[DMPH_PHASE_COUNT] = {0};
    long long phase_n[DMPH_PHASE_COUNT] = {0};
    std::string err;
    // every device allocation of the context, in allocation order; `state`
    // ones (all but the lazily allocated output buffers) make a checkpoint
    struct DevAlloc {
        void *p;
        size_t bytes;
        bool state;
    };
    std::vector<DevAlloc> allocs;
    // dmph_set_bodies' arguments (a checkpoint re-creates the same bodies)
    std::vector<int> body_of_row;
    std::vector<double> body_density;
    dmph::Surrogate *sg = nullptr;  // surrogate state (dmph_surrogate_enable)
};


#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                             \
            return DMPH_ECUDA;                                                                         \
        }                                                                                              \
    } while (0)

namespace dmph {

// step pieces (dmph_api.cu)
void enqueue_rebuild(dmph_ctx *ctx, bool first, cudaStream_t st);
long long rebuild_launches(const dmph_ctx *ctx, bool first);
void enqueue_head(dmph_ctx *ctx, unsigned long long graph_cond, cudaStream_t st);
void enqueue_passes(dmph_ctx *ctx, cudaStream_t st);
void enqueue_pair_passes32(dmph_ctx *ctx, cudaStream_t st);
void enqueue_dem(dmph_ctx *ctx, cudaStream_t st);
// the DEM substeps of `steps` steps with the fluid force held (surrogate block)
void enqueue_dem_block(dmph_ctx *ctx, int steps, cudaStream_t st);
long long dem_block_launches(const dmph_ctx *ctx, int steps);
long long dem_launches(const dmph_ctx *ctx);
long long tail_launches(const dmph_ctx *ctx, bool graph = false);
void advance_host_clock(dmph_ctx *ctx);
int step_once(dmph_ctx *ctx);
int read_bounds(dmph_ctx *ctx, int *b);
// on a capturing stream: an IF node whose body is the rebuild, run when a
// decision kernel sets cond
int capture_rebuild_if(dmph_ctx *ctx, cudaGraphConditionalHandle cond, cudaStream_t st);
// DMPH_ENAN once a drift has met a non-finite position or velocity
// (B_NONFINITE; synchronises the stream), else DMPH_OK
int check_finite(dmph_ctx *ctx);
constexpr int kFiniteCheckEvery = 256;  // steps between two checks inside one dmph_step call
void drop_graph(dmph_ctx *ctx);
// list reuse in effect for the next steps: the flag, the FP32 build with
// lists, walls at rest, the counting sort, no debris outside rigid bodies,
// no neighbour counts kept for every particle
bool reuse_active(const dmph_ctx *ctx);

// surrogate (dmph_surrogate.cu)
void surrogate_release(dmph_ctx *ctx);

}  // namespace dmph
