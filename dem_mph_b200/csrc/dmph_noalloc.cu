// Allocation-free cell sort: dmph_cell_sort_noalloc (see include/dmph.h).
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA stream is
// being captured into a graph, solvers embedded in a host framework that owns
// every device allocation through its own pool, and real-time loops that must
// not touch the driver's allocator once running.  This entry point gives them
// the neighbour-rebuild sort (cell keys + the reference's bitonic network, the
// same kernels the solver context runs) with its scratch space in a
// file-scope device array instead of a cudaMalloc'd buffer.  The caller passes
// device buffers for the inputs and outputs.
//
// The scratch array holds the 64-bit sort words (key << 32 | slot) of the
// power-of-two padded array, so the particle count is limited to
// kNoAllocMaxWords - 1.  It is part of the library image: every GPU that loads
// libdmph.so keeps these 4 MiB until the process exits.
//
// The array's device address belongs to the CUDA context that loaded the
// module.  It is looked up with cudaGetSymbolAddress and cached together with
// the context's process-unique id (cuCtxGetId, reached through
// cudaGetDriverEntryPointByVersion so that the library needs no link against
// libcuda).  A call under another context (after cudaDeviceReset, or a
// primary context released and made again) finds a different id and looks the
// address up again, so a stale address is never used.
#include <cuda.h>

#include <mutex>

#include "dmph_internal.h"

namespace {

constexpr int kNoAllocMaxWords = 1 << 19;  // 4 MiB of sort words
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_sort_scratch[kNoAllocMaxWords];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// host-side cache of the scratch array's device address: per device slot, the
// id of the context it was looked up in and the address
struct ScratchSlot {
    std::mutex mu;
    unsigned long long ctx_id = 0;  // 0: nothing cached
    unsigned long long *addr = nullptr;
};
ScratchSlot g_slots[kMaxDevices];

std::once_flag g_entry_once;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

void resolve_entry_points()
{
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_id = (CtxGetIdFn)f;
}

// id of the calling thread's current context, 0 when there is none yet
unsigned long long current_ctx_id()
{
    if (!g_ctx_get_current || !g_ctx_get_id) return 0;
    CUcontext c = nullptr;
    if (g_ctx_get_current(&c) != CUDA_SUCCESS || !c) return 0;
    unsigned long long id = 0;
    if (g_ctx_get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// device address of g_sort_scratch in the current context, or nullptr (the
// reason is left in *why)
unsigned long long *scratch_address(int dev, const char **why)
{
    std::call_once(g_entry_once, resolve_entry_points);
    if (!g_ctx_get_current || !g_ctx_get_id) {
        *why = "dmph_cell_sort_noalloc: the driver does not provide cuCtxGetCurrent/cuCtxGetId";
        return nullptr;
    }
    ScratchSlot &s = g_slots[dev];
    std::lock_guard<std::mutex> lock(s.mu);
    const unsigned long long id = current_ctx_id();
    if (id != 0 && id == s.ctx_id && s.addr) return s.addr;
    // set-up in this context (the lookup also makes the primary context
    // current when the thread has none yet, so the id is read afterwards)
    void *a = nullptr;
    if (cudaGetSymbolAddress(&a, g_sort_scratch) != cudaSuccess || !a) {
        *why = "dmph_cell_sort_noalloc: cudaGetSymbolAddress of the scratch array failed";
        return nullptr;
    }
    const unsigned long long id2 = current_ctx_id();
    if (id2 == 0) {
        *why = "dmph_cell_sort_noalloc: no current CUDA context after the scratch lookup";
        return nullptr;
    }
    s.ctx_id = id2;
    s.addr = (unsigned long long *)a;
    return s.addr;
}

__global__ void k_unpack_sorted(const unsigned long long *__restrict__ words, int n, int *__restrict__ key,
                                int *__restrict__ perm)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long w = words[i];
    key[i] = (int)dmph::word_key(w);
    perm[i] = (int)dmph::word_slot(w);
}

int fail(int code, const char *literal)
{
    dmph::set_noctx_message(literal);
    return code;
}

}  // namespace

extern "C" int dmph_cell_sort_noalloc(const dmph_params *p, int n, const double *pos_planes, const int *type,
                                      int32_t *sorted_key, int32_t *perm, void *stream)
{
    if (!p || !pos_planes || !type || !sorted_key || !perm)
        return fail(DMPH_EINVAL, "dmph_cell_sort_noalloc: null argument");
    if (n <= 0) return fail(DMPH_EINVAL, "dmph_cell_sort_noalloc: particle count must be positive");
    if (n >= kNoAllocMaxWords)
        return fail(DMPH_ERANGE, "dmph_cell_sort_noalloc: particle count above DMPH_NOALLOC_MAX_WORDS - 1");
    dmph::DevParams P;
    dmph::WallMotion Wm;
    const char *msg = "";
    const int rc = dmph::derive_params(*p, n, P, Wm, &msg);
    if (rc) return fail(rc, msg);
    if (P.P2 > kNoAllocMaxWords)
        return fail(DMPH_ERANGE, "dmph_cell_sort_noalloc: padded particle count above DMPH_NOALLOC_MAX_WORDS");

    // an error left pending on this thread by earlier work is not this call's:
    // leave it for its owner to read and run nothing
    if (cudaPeekAtLastError() != cudaSuccess)
        return fail(DMPH_ECUDA, "dmph_cell_sort_noalloc: a CUDA error from earlier work is pending on this thread");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(DMPH_ECUDA, "dmph_cell_sort_noalloc: cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices) return fail(DMPH_ERANGE, "dmph_cell_sort_noalloc: device index above 63");
    const char *why = "";
    unsigned long long *words = scratch_address(dev, &why);
    if (!words) {
        (void)cudaGetLastError();  // the failed lookup's own error
        return fail(DMPH_ECUDA, why);
    }

    cudaStream_t st = (cudaStream_t)stream;
    // every one of the P2 words is rewritten by the key kernel (the padding
    // included), so nothing of the previous call's contents needs clearing
    dmph::launch_keys(P, pos_planes, type, words, st);
    dmph::launch_bitonic(words, P.P2, P.P2log, st);
    k_unpack_sorted<<<(n + 255) / 256, 256, 0, st>>>(words, n, sorted_key, perm);
    if (cudaGetLastError() != cudaSuccess)
        return fail(DMPH_ECUDA, "dmph_cell_sort_noalloc: a kernel launch failed");
    return DMPH_OK;
}
