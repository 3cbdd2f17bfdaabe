// Checkpoint files for an exact resume (dmph_checkpoint_write / _open).
//
// The reference restarts from a .prof file (source/DEM-MPH.cpp:433, :690,
// :853-877), which holds positions, velocities and types only; the restarted
// run rebuilds its neighbour lists at the restart positions, re-derives the
// DEM constants and wall centres, and so follows another trajectory.  A
// checkpoint here holds the context's whole device state (every allocation
// made by dmph_create and dmph_set_bodies, in allocation order: the sorted
// particle arrays, the positions of the last rebuild, the cell sort, the
// neighbour lists, the DEM constants, the body states and the device bounds)
// and its host clock, so a context opened from it steps to the same bits as
// the one that wrote it.
//
// Layout (native byte order and structure layouts of this library):
//   "DMPHCKPT", u32 version, u32 sizeof(dmph_params), u32 sizeof(HostBlock), u32 0
//   i32 n, i32 nbodies, i32 nalloc, i32 user_bytes
//   dmph_params (the creation parameters), HostBlock, user bytes
//   i32 type[n], f64 x[3n], f64 v[3n]         by input row
//   i32 body_of_row[n], f64 density[nbodies]   when nbodies > 0
//   u64 bytes[nalloc], then the allocations' bytes
//   "DMPHEND."
// Opening creates a context from the parameters, rows and bodies (which
// allocates the same arrays in the same order), checks the allocation table
// against it and overwrites every array and the clock.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dmph_ctx.h"

namespace {

constexpr char kMagic[8] = {'D', 'M', 'P', 'H', 'C', 'K', 'P', 'T'};
constexpr char kTrailer[8] = {'D', 'M', 'P', 'H', 'E', 'N', 'D', '.'};
constexpr uint32_t kVersion = 1;
constexpr size_t kStage = 64u << 20;  // pinned staging buffer of the copies

// the host side of the context that stepping changes
struct HostBlock {
    double time;
    long long steps, rebuilds, graph_steps, host_rebuilds, launches;
    int nonfinite, use_list, var_a, var_b, var_la, var_lb, var_build, use_graph;
    WallMotion Wm;
};

struct Header {
    char magic[8];
    uint32_t version, params_bytes, host_bytes, reserved;
    int32_t n, nbodies, nalloc, user_bytes;
};

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) std::fclose(f);
    }
};

struct Pinned {
    void *p = nullptr;
    ~Pinned()
    {
        if (p) cudaFreeHost(p);
    }
};

size_t state_allocs(const dmph_ctx *ctx, std::vector<uint64_t> *bytes)
{
    size_t k = 0;
    for (const auto &a : ctx->allocs)
        if (a.state) {
            if (bytes) bytes->push_back(a.bytes);
            ++k;
        }
    return k;
}

bool put(FILE *f, const void *p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }
bool get(FILE *f, void *p, size_t bytes) { return bytes == 0 || std::fread(p, 1, bytes, f) == bytes; }

}  // namespace

extern "C" int dmph_checkpoint_write(dmph_ctx *ctx, const char *path, const void *user, int user_bytes)
{
    if (!ctx) return DMPH_EINVAL;
    if (!path || user_bytes < 0 || user_bytes > DMPH_CHECKPOINT_USER_MAX || (user_bytes > 0 && !user)) {
        ctx->err = "dmph_checkpoint_write: bad argument";
        return DMPH_EINVAL;
    }
    if (ctx->in_split_step) {
        ctx->err = "dmph_checkpoint_write between dmph_step_begin and dmph_step_finish";
        return DMPH_EINVAL;
    }
    if (ctx->nonfinite) {
        ctx->err = "dmph_checkpoint_write: the state is non-finite";
        return DMPH_ENAN;
    }
    const int n = ctx->P.N;
    std::vector<int> type(n), pidx(n), trow(n);
    std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n), xrow(3 * (size_t)n), vrow(3 * (size_t)n);
    // first: in the FP32 build this refreshes the FP64 copies of the state,
    // which then go into the file as the context continues with them
    int rc = dmph_get_state(ctx, type.data(), x.data(), v.data(), pidx.data());
    if (rc) return rc;
    for (int i = 0; i < n; i++) {
        const int r = pidx[i];
        trow[r] = type[i];
        for (int d = 0; d < 3; d++) {
            xrow[3 * (size_t)r + d] = x[3 * (size_t)i + d];
            vrow[3 * (size_t)r + d] = v[3 * (size_t)i + d];
        }
    }
    const int nb = ctx->Bd.B;
    std::vector<uint64_t> bytes;
    const size_t nalloc = state_allocs(ctx, &bytes);
    Header h;
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.params_bytes = sizeof(dmph_params);
    h.host_bytes = sizeof(HostBlock);
    h.reserved = 0;
    h.n = n;
    h.nbodies = nb;
    h.nalloc = (int32_t)nalloc;
    h.user_bytes = user_bytes;
    HostBlock hb;
    std::memset(&hb, 0, sizeof(hb));
    hb.time = ctx->time;
    hb.steps = ctx->steps;
    hb.rebuilds = ctx->rebuilds;
    hb.graph_steps = ctx->graph_steps;
    hb.host_rebuilds = ctx->host_rebuilds;
    hb.launches = ctx->launches;
    hb.nonfinite = ctx->nonfinite ? 1 : 0;
    hb.use_list = ctx->use_list ? 1 : 0;
    hb.var_a = ctx->var_a;
    hb.var_b = ctx->var_b;
    hb.var_la = ctx->var_la;
    hb.var_lb = ctx->var_lb;
    hb.var_build = ctx->var_build;
    hb.use_graph = ctx->use_graph ? 1 : 0;
    hb.Wm = ctx->Wm;
    File fh;
    fh.f = std::fopen(path, "wb");
    if (!fh.f) {
        ctx->err = std::string("cannot open ") + path + " for writing";
        return DMPH_EIO;
    }
    bool ok = put(fh.f, &h, sizeof(h)) && put(fh.f, &ctx->p, sizeof(dmph_params)) && put(fh.f, &hb, sizeof(hb)) &&
              put(fh.f, user, (size_t)user_bytes) && put(fh.f, trow.data(), sizeof(int) * (size_t)n) &&
              put(fh.f, xrow.data(), sizeof(double) * 3 * (size_t)n) &&
              put(fh.f, vrow.data(), sizeof(double) * 3 * (size_t)n);
    if (ok && nb > 0)
        ok = put(fh.f, ctx->body_of_row.data(), sizeof(int) * (size_t)n) &&
             put(fh.f, ctx->body_density.data(), sizeof(double) * (size_t)nb);
    ok = ok && put(fh.f, bytes.data(), sizeof(uint64_t) * nalloc);
    Pinned stage;
    CK(cudaMallocHost(&stage.p, kStage));
    for (const auto &a : ctx->allocs) {
        if (!ok) break;
        if (!a.state) continue;
        for (size_t off = 0; ok && off < a.bytes; off += kStage) {
            const size_t len = a.bytes - off < kStage ? a.bytes - off : kStage;
            CK(cudaMemcpyAsync(stage.p, (const char *)a.p + off, len, cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
            ok = put(fh.f, stage.p, len);
        }
    }
    ok = ok && put(fh.f, kTrailer, 8);
    const int closed = std::fclose(fh.f);
    fh.f = nullptr;
    if (!ok || closed != 0) {
        ctx->err = std::string("cannot write ") + path;
        return DMPH_EIO;
    }
    return DMPH_OK;
}

extern "C" int dmph_checkpoint_open(const char *path, dmph_ctx **out, void *user, int user_capacity, int *user_bytes)
{
    if (!out || !path || user_capacity < 0) return set_noctx_error("dmph_checkpoint_open: bad argument"), DMPH_EINVAL;
    *out = nullptr;
    if (user_bytes) *user_bytes = 0;
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) return set_noctx_error(std::string("cannot open ") + path), DMPH_EIO;
    const std::string bad = std::string(path) + " is not a checkpoint of this library";
    Header h;
    if (!get(fh.f, &h, sizeof(h)) || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion ||
        h.params_bytes != sizeof(dmph_params) || h.host_bytes != sizeof(HostBlock) || h.n <= 0 || h.nbodies < 0 ||
        h.nalloc <= 0 || h.user_bytes < 0 || h.user_bytes > DMPH_CHECKPOINT_USER_MAX)
        return set_noctx_error(bad), DMPH_EIO;
    if (h.user_bytes > user_capacity || (h.user_bytes > 0 && !user))
        return set_noctx_error("dmph_checkpoint_open: the file holds " + std::to_string(h.user_bytes) +
                               " user bytes, more than the buffer given"),
               DMPH_EINVAL;
    const int n = h.n, nb = h.nbodies;
    dmph_params p;
    HostBlock hb;
    std::vector<int> type(n), body_of_row(nb > 0 ? n : 0);
    std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n), dens(nb);
    std::vector<char> ubuf(h.user_bytes);
    bool ok = get(fh.f, &p, sizeof(p)) && get(fh.f, &hb, sizeof(hb)) && get(fh.f, ubuf.data(), ubuf.size()) &&
              get(fh.f, type.data(), sizeof(int) * (size_t)n) && get(fh.f, x.data(), sizeof(double) * 3 * (size_t)n) &&
              get(fh.f, v.data(), sizeof(double) * 3 * (size_t)n);
    if (ok && nb > 0)
        ok = get(fh.f, body_of_row.data(), sizeof(int) * (size_t)n) &&
             get(fh.f, dens.data(), sizeof(double) * (size_t)nb);
    std::vector<uint64_t> bytes(h.nalloc);
    ok = ok && get(fh.f, bytes.data(), sizeof(uint64_t) * bytes.size());
    if (!ok) return set_noctx_error(bad + " (truncated)"), DMPH_EIO;
    // a context shaped like the one that wrote the file
    dmph_ctx *ctx = nullptr;
    int rc = dmph_create(&p, n, type.data(), x.data(), v.data(), &ctx);
    if (rc) return rc;
    auto fail = [&](int code, const std::string &msg) {
        dmph_destroy(ctx);
        set_noctx_error(msg);
        return code;
    };
    if (nb > 0) {
        rc = dmph_set_bodies(ctx, nb, body_of_row.data(), dens.data());
        if (rc) return fail(rc, std::string("dmph_checkpoint_open: ") + dmph_last_error(ctx));
    }
    std::vector<uint64_t> mine;
    if (state_allocs(ctx, &mine) != bytes.size() || mine != bytes)
        return fail(DMPH_EIO, bad + " (its device arrays differ from this build's)");
    Pinned stage;
    if (cudaMallocHost(&stage.p, kStage) != cudaSuccess) return fail(DMPH_ECUDA, "cudaMallocHost failed");
    for (const auto &a : ctx->allocs) {
        if (!a.state) continue;
        for (size_t off = 0; off < a.bytes; off += kStage) {
            const size_t len = a.bytes - off < kStage ? a.bytes - off : kStage;
            if (!get(fh.f, stage.p, len)) return fail(DMPH_EIO, bad + " (truncated)");
            if (cudaMemcpyAsync((char *)a.p + off, stage.p, len, cudaMemcpyHostToDevice, ctx->st) != cudaSuccess ||
                cudaStreamSynchronize(ctx->st) != cudaSuccess)
                return fail(DMPH_ECUDA, "dmph_checkpoint_open: copy to the device failed");
        }
    }
    char tail[8];
    if (!get(fh.f, tail, 8) || std::memcmp(tail, kTrailer, 8) != 0 || std::fgetc(fh.f) != EOF)
        return fail(DMPH_EIO, bad + " (bad end)");
    ctx->time = hb.time;
    ctx->steps = hb.steps;
    ctx->rebuilds = hb.rebuilds;
    ctx->graph_steps = hb.graph_steps;
    ctx->host_rebuilds = hb.host_rebuilds;
    ctx->launches = hb.launches;
    ctx->nonfinite = hb.nonfinite != 0;
    ctx->use_list = hb.use_list != 0;
    ctx->var_a = hb.var_a;
    ctx->var_b = hb.var_b;
    ctx->var_la = hb.var_la;
    ctx->var_lb = hb.var_lb;
    ctx->var_build = hb.var_build;
    ctx->use_graph = hb.use_graph != 0;
    ctx->Wm = hb.Wm;
    drop_graph(ctx);
    if (h.user_bytes > 0) std::memcpy(user, ubuf.data(), ubuf.size());
    if (user_bytes) *user_bytes = h.user_bytes;
    *out = ctx;
    return DMPH_OK;
}
