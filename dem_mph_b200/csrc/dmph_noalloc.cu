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
#include <atomic>
#include <string>

#include "dmph_internal.h"

namespace {

constexpr int kNoAllocMaxWords = 1 << 19;  // 4 MiB of sort words
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_sort_scratch[kNoAllocMaxWords];

// host-side cache of the scratch array's device address, one per device
std::atomic<unsigned long long *> g_scratch_addr[kMaxDevices];

// error sink for the parameter derivation, reserved when the library loads so
// that validating a call never allocates
struct ReservedString {
    std::string s;
    ReservedString() { s.reserve(512); }
};
ReservedString g_noalloc_err;

__global__ void k_unpack_sorted(const unsigned long long *__restrict__ words, int n, int *__restrict__ key,
                                int *__restrict__ perm)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long w = words[i];
    key[i] = (int)dmph::word_key(w);
    perm[i] = (int)dmph::word_slot(w);
}

}  // namespace

extern "C" int dmph_cell_sort_noalloc(const dmph_params *p, int n, const double *pos_planes, const int *type,
                                      int32_t *sorted_key, int32_t *perm, void *stream)
{
    if (!p || !pos_planes || !type || !sorted_key || !perm || n <= 0) return DMPH_EINVAL;
    if (n >= kNoAllocMaxWords) return DMPH_ERANGE;
    dmph::DevParams P;
    dmph::WallMotion Wm;
    const int rc = dmph::derive_params(*p, n, P, Wm, g_noalloc_err.s);
    if (rc) return rc;
    if (P.P2 > kNoAllocMaxWords) return DMPH_ERANGE;

    // set-up, once per device, with that device current: the host-side name of
    // g_sort_scratch is not a device address, so ask the runtime for it
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DMPH_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return DMPH_ERANGE;
    unsigned long long *words = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!words) {
        void *addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_sort_scratch) != cudaSuccess || !addr) return DMPH_ECUDA;
        words = (unsigned long long *)addr;
        g_scratch_addr[dev].store(words, std::memory_order_release);
    }

    cudaStream_t st = (cudaStream_t)stream;
    // every one of the P2 words is rewritten by the key kernel (the padding
    // included), so nothing of the previous call's contents needs clearing
    dmph::launch_keys(P, pos_planes, type, words, st);
    dmph::launch_bitonic(words, P.P2, P.P2log, st);
    k_unpack_sorted<<<(n + 255) / 256, 256, 0, st>>>(words, n, sorted_key, perm);
    return cudaGetLastError() == cudaSuccess ? DMPH_OK : DMPH_ECUDA;
}
