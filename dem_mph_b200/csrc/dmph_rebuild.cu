// Neighbour rebuild: cell keys, the bitonic sort, cell ranges, permutation and
// the warp work list (calculateCellParticle, source/DEM-MPH.cpp:1288-1519).
//
// The reference sorts (key, slot) pairs with a bitonic network over the
// power-of-two padded array (:1317-1338).  The network swaps equal keys inside
// descending sub-blocks, so the order of particles within a cell depends on
// the network itself; the DEM contact constants take the last neighbour within
// dx (:2305-2341), which depends on that order.  The same network is therefore
// run here, exactly: stages whose compare distance is below the tile size are
// done in shared memory (one launch per outer stage), the wider ones as
// global passes.  Keys and slots travel as one 64-bit word; only the key half
// is compared, as in the reference.
#include "dmph_state.cuh"

namespace dmph {

constexpr int kSortTileLog = 12;  // 4096 words = 32 KiB of shared memory per block
constexpr int kSortTile = 1 << kSortTileLog;
constexpr int kSortThreads = 1024;
constexpr int kSortFuse = 4;  // global sub-passes done per launch

// cell key + class offset of particle i (:1295-1313)
__device__ __forceinline__ int particle_key(const DevParams &P, const double *__restrict__ pos,
                                            const int *__restrict__ type, int i)
{
    const int N = P.N;
    const int ix = ((int)floor((pos[i] - P.dmin[0]) / P.cw[0])) % P.cc[0];
    const int iy = ((int)floor((pos[N + i] - P.dmin[1]) / P.cw[1])) % P.cc[1];
    const int iz = ((int)floor((pos[2 * N + i] - P.dmin[2]) / P.cw[2])) % P.cc[2];
    int k = cell_id(P, ix, iy, iz);
    const int t = type[i];
    if (is_solid(t))
        k += P.T;
    else if (is_wall(t))
        k += 2 * P.T;
    return k;
}

// cell key and identity payload; pad with 3T
__global__ void k_keys(DevParams P, const double *__restrict__ pos, const int *__restrict__ type,
                       unsigned long long *__restrict__ words)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.P2) return;
    const int N = P.N;
    unsigned long long w;
    if (i < N)
        w = ((unsigned long long)(uint32_t)particle_key(P, pos, type, i) << 32) | (uint32_t)i;
    else
        w = ((unsigned long long)(uint32_t)(3 * P.T) << 32) | (uint32_t)N;
    words[i] = w;
}

template <class T>
int launch_exclusive_scan(const T *in, T *out, int n, T *block_sums, T *total, cudaStream_t st);

// ------------------------------------------------ FP32: counting sort
// The FP32 build sorts the cell keys with a counting sort instead of the
// reference's bitonic network: the particles of a (class, cell) key keep
// their previous relative order (a stable sort), so every particle's cell
// and neighbour set are the reference's while the order inside a cell is
// this build's own.  Keys are counted, the counts scanned into cell_start,
// the particles scattered with an atomic cursor per key, and each key's
// range finally ordered by previous slot, so the result does not depend on
// the order of the atomics.
__global__ void k_count_keys(DevParams P, const double *__restrict__ pos, const int *__restrict__ type,
                             int *__restrict__ keys, int *__restrict__ counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.N) return;
    const int k = particle_key(P, pos, type, i);
    keys[i] = k;
    atomicAdd(counts + k, 1);
}

// slots [0, n) (n < N: the walls keep their slots and their words)
__global__ void k_scatter_keys(DevParams P, int n, const int *__restrict__ keys, const int *__restrict__ start,
                               int *__restrict__ cursor, unsigned long long *__restrict__ tmp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = keys[i];
    tmp[start[k] + atomicAdd(cursor + k, 1)] = ((unsigned long long)(uint32_t)k << 32) | (uint32_t)i;
}

// one warp per 32 keys; each key's range is ordered by rank (the number of
// smaller words in the range), for any range length
// keys [0, nseg)
__global__ void k_sort_cells(DevParams P, int nseg, const unsigned long long *__restrict__ tmp,
                             const int *__restrict__ start, unsigned long long *__restrict__ words)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int k0 = gw * 32; k0 < nseg; k0 += nw * 32) {
        const int kl = k0 + lane;
        const int b_l = kl < nseg ? start[kl] : 0;
        const int n_l = kl < nseg ? start[kl + 1] - b_l : 0;
        if (n_l == 1) words[b_l] = tmp[b_l];
        unsigned todo = __ballot_sync(kFull, n_l >= 2);
        while (todo) {
            const int t = __ffs(todo) - 1;
            todo &= todo - 1;
            const int b = __shfl_sync(kFull, b_l, t), n = __shfl_sync(kFull, n_l, t);
            for (int e0 = 0; e0 < n; e0 += kWarp) {
                const int e = e0 + lane;
                const unsigned long long w = e < n ? tmp[b + e] : 0ull;
                int rank = 0;
                for (int f0 = 0; f0 < n; f0 += kWarp) {
                    const unsigned long long wf = f0 + lane < n ? tmp[b + f0 + lane] : 0ull;
                    const int lim = n - f0 < kWarp ? n - f0 : kWarp;
                    for (int u = 0; u < lim; ++u) rank += __shfl_sync(kFull, wf, u) < w ? 1 : 0;
                }
                if (e < n) words[b + rank] = w;
            }
        }
    }
}

int launch_counting_sort(const DevParams &P, int n_move, const double *pos, const int *type, int *keys, int *counts,
                         unsigned long long *tmp, unsigned long long *words, int *cell_start, int *block_sums,
                         int *total, cudaStream_t st)
{
    // n_move < N: the walls, which sort last, keep their slots (see
    // enqueue_rebuild), so only the slots [0, n_move) are scattered and only
    // the fluid and debris keys ordered; the walls still count for cell_start
    const int nk = 3 * P.T + 1;
    const int g = (P.N + 255) / 256;
    cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nk, st);
    k_count_keys<<<g, 256, 0, st>>>(P, pos, type, keys, counts);
    const int rc = launch_exclusive_scan<int>(counts, cell_start, nk, block_sums, total, st);
    if (rc) return rc;
    cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nk, st);
    k_scatter_keys<<<(n_move + 255) / 256, 256, 0, st>>>(P, n_move, keys, cell_start, counts, tmp);
    k_sort_cells<<<148 * 8, 256, 0, st>>>(P, n_move < P.N ? 2 * P.T : 3 * P.T, tmp, cell_start, words);
    return 0;
}

__device__ __forceinline__ void cmp_exchange(unsigned long long &a, unsigned long long &b, bool up)
{
    // swap when (key_a > key_b) == up  (:1326)
    if ((word_key(a) > word_key(b)) == up) {
        const unsigned long long t = a;
        a = b;
        b = t;
    }
}

// Stages (stage, dist) with dist < tile, from `stage_lo` (starting at
// dist_start) to `stage_hi`, inside one tile in shared memory.
__global__ void __launch_bounds__(kSortThreads) k_bitonic_local(unsigned long long *words, int tile, int stage_lo,
                                                                 int stage_hi, int dist_start)
{
    __shared__ unsigned long long sm[kSortTile];
    const int base = blockIdx.x * tile;
    for (int k = threadIdx.x; k < tile; k += blockDim.x) sm[k] = words[base + k];
    __syncthreads();
    for (int stage = stage_lo; stage <= stage_hi; ++stage) {
        int dist = (stage == stage_lo) ? dist_start : (1 << stage);
        if (dist > tile / 2) dist = tile / 2;
        for (; dist >= 1; dist >>= 1) {
            for (int t = threadIdx.x; t < tile / 2; t += blockDim.x) {
                const int lo = (t / dist) * 2 * dist + (t % dist);  // local index with bit `dist` clear
                const int g = base + lo;
                const bool up = ((g >> stage) & 2) == 0;
                cmp_exchange(sm[lo], sm[lo + dist], up);
            }
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < tile; k += blockDim.x) words[base + k] = sm[k];
}

// R consecutive sub-passes of one stage, distances dist, dist/2, ...,
// dist >> (R-1), all at least the tile: those sub-passes compare the words
// base + m * h (h = dist >> (R-1), m < 2^R) only among themselves, so each
// thread loads such a group, applies the R sub-passes in order in registers
// and stores it back.  Consecutive threads own consecutive bases, so every
// load and store is coalesced.  All words of a group lie in one aligned
// block of 2 * dist <= 2^(stage+1) words and share the direction bit.
template <int R>
__global__ void k_bitonic_global(unsigned long long *words, int n, int stage, int dist)
{
    const int h = dist >> (R - 1);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (n >> R)) return;
    const int base = (t / h) * 2 * dist + (t % h);
    const bool up = ((base >> stage) & 2) == 0;
    unsigned long long v[1 << R];
#pragma unroll
    for (int m = 0; m < (1 << R); ++m) v[m] = words[base + m * h];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int d = 1 << (R - 1 - r);
#pragma unroll
        for (int m = 0; m < (1 << R); ++m)
            if ((m & d) == 0) cmp_exchange(v[m], v[m + d], up);
    }
#pragma unroll
    for (int m = 0; m < (1 << R); ++m) words[base + m * h] = v[m];
}

// cell_start[c] = number of sorted keys below c, c in [0, 3T]  (the begin/end
// arrays of :1340-1438 are cell_start[k] and cell_start[k+1])
__global__ void k_cell_start(DevParams P, const unsigned long long *__restrict__ words, int *__restrict__ start)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > 3 * P.T) return;
    int lo = 0, hi = P.N;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((int)word_key(words[mid]) < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    start[c] = lo;
}

// gather ParticleIndex, Property, Position, Velocity (:1455-1518) into the
// other buffer and snapshot NeighborCalculatedPosition (:1842-1850)
__global__ void k_permute(DevParams P, const unsigned long long *__restrict__ words, const double *__restrict__ pos_in,
                          const double *__restrict__ vel_in, const int *__restrict__ type_in,
                          const int *__restrict__ pidx_in, double *__restrict__ pos_out, double *__restrict__ vel_out,
                          int *__restrict__ type_out, int *__restrict__ pidx_out, double *__restrict__ xref,
                          const int *__restrict__ bid_in, int *__restrict__ bid_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.N;
    if (i >= N) return;
    const int src = (int)word_slot(words[i]);
    for (int d = 0; d < 3; d++) {
        const double x = pos_in[d * N + src];
        pos_out[d * N + i] = x;
        xref[d * N + i] = x;
        vel_out[d * N + i] = vel_in[d * N + src];
    }
    type_out[i] = type_in[src];
    pidx_out[i] = pidx_in[src];
    if (bid_in) bid_out[i] = bid_in[src];
}

// chunk heads: a slot starts a chunk when it starts its key's range or is a
// multiple of 32 into it
__global__ void k_chunk_flags(DevParams P, const unsigned long long *__restrict__ words, const int *__restrict__ start,
                              int *__restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.N) return;
    const int k = (int)word_key(words[i]);
    flag[i] = ((i - start[k]) % kWarp) == 0 ? 1 : 0;
}

__global__ void k_chunk_write(DevParams P, const unsigned long long *__restrict__ words, const int *__restrict__ start,
                              const int *__restrict__ flag, const int *__restrict__ offs, Chunk *__restrict__ chunks)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.N || !flag[i]) return;
    const int k = (int)word_key(words[i]);
    const int end = start[k + 1];
    Chunk c;
    c.i0 = i;
    c.cnt = min(kWarp, end - i);
    chunks[offs[i]] = c;
}

// ------------------------------------------------------------ prefix sums
// Exclusive scan of n int32 values (n <= kScanBlock * kScanBlock * 4) in
// three launches; out[n] receives the total.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int *sh, int &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    const int warp_prefix = w > 0 ? sh[w - 1] : 0;
    total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_local(const T *__restrict__ in, T *__restrict__ out, int n,
                                                             T *__restrict__ block_sums)
{
    __shared__ int sh[32];
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : T(0);
        s += v[k];
    }
    int total;
    const int ex = block_exclusive_scan((int)s, sh, total);
    T run = (T)ex;
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = (T)total;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(T *__restrict__ sums, int nb, T *__restrict__ total_out)
{
    // one block: exclusive scan of the block sums in place (nb <= kScanBlock)
    __shared__ int sh[32];
    const int base = threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < nb) ? sums[base + k] : T(0);
        s += v[k];
    }
    int total;
    const int ex = block_exclusive_scan((int)s, sh, total);
    T run = (T)ex;
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < nb) sums[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) *total_out = (T)total;
}

template <class T>
__global__ void k_scan_add(T *__restrict__ out, int n, const T *__restrict__ sums)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] += sums[i / kScanBlock];
}

// --------------------------------------------------------------- host side
void launch_keys(const DevParams &P, const double *pos, const int *type, unsigned long long *words, cudaStream_t st)
{
    k_keys<<<(P.P2 + 255) / 256, 256, 0, st>>>(P, pos, type, words);
}

int bitonic_launch_count(int n, int nlog)
{
    const int tlog = n < kSortTile ? nlog : kSortTileLog;
    int c = tlog > 0 ? 1 : 0;
    for (int stage = tlog; stage < nlog; ++stage) c += (stage - tlog + kSortFuse) / kSortFuse + 1;
    return c;
}

void launch_bitonic(unsigned long long *words, int n, int nlog, cudaStream_t st)
{
    const int tile = n < kSortTile ? n : kSortTile;
    const int tlog = n < kSortTile ? nlog : kSortTileLog;
    const int threads = tile / 2 > kSortThreads ? kSortThreads : (tile / 2 > 0 ? tile / 2 : 1);
    const int blocks = n / tile;
    // all stages whose distance fits the tile: stages 0 .. tlog-1
    if (tlog > 0) k_bitonic_local<<<blocks, threads, 0, st>>>(words, tile, 0, tlog - 1, 1);
    for (int stage = tlog; stage < nlog; ++stage) {
        // the distances 2^stage .. tile, up to kSortFuse of them per launch
        int dist = 1 << stage;
        int left = stage - tlog + 1;
        while (left > 0) {
            const int r = left < kSortFuse ? left : kSortFuse;
            const int groups = n >> r;
            const int g = (groups + 255) / 256;
            switch (r) {
            case 1: k_bitonic_global<1><<<g, 256, 0, st>>>(words, n, stage, dist); break;
            case 2: k_bitonic_global<2><<<g, 256, 0, st>>>(words, n, stage, dist); break;
            case 3: k_bitonic_global<3><<<g, 256, 0, st>>>(words, n, stage, dist); break;
            default: k_bitonic_global<4><<<g, 256, 0, st>>>(words, n, stage, dist); break;
            }
            dist >>= r;
            left -= r;
        }
        k_bitonic_local<<<blocks, threads, 0, st>>>(words, tile, stage, stage, tile / 2);
    }
}

void launch_cell_start(const DevParams &P, const unsigned long long *words, int *start, cudaStream_t st)
{
    const int n = 3 * P.T + 1;
    k_cell_start<<<(n + 255) / 256, 256, 0, st>>>(P, words, start);
}

void launch_permute(const DevParams &P, const unsigned long long *words, const double *pos_in, const double *vel_in,
                    const int *type_in, const int *pidx_in, double *pos_out, double *vel_out, int *type_out,
                    int *pidx_out, double *xref, const int *bid_in, int *bid_out, cudaStream_t st)
{
    k_permute<<<(P.N + 255) / 256, 256, 0, st>>>(P, words, pos_in, vel_in, type_in, pidx_in, pos_out, vel_out,
                                                 type_out, pidx_out, xref, bid_in, bid_out);
}

template <class T>
int launch_exclusive_scan(const T *in, T *out, int n, T *block_sums, T *total, cudaStream_t st)
{
    const int nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb > kScanBlock) return DMPH_ERANGE;
    k_scan_local<T><<<nb, kScanThreads, 0, st>>>(in, out, n, block_sums);
    k_scan_sums<T><<<1, kScanThreads, 0, st>>>(block_sums, nb, total);
    k_scan_add<T><<<(n + 255) / 256, 256, 0, st>>>(out, n, block_sums);
    return 0;
}
template int launch_exclusive_scan<int>(const int *, int *, int, int *, int *, cudaStream_t);

void launch_chunks(const DevParams &P, const unsigned long long *words, const int *start, int *flag, int *offs,
                   int *block_sums, int *total, Chunk *chunks, cudaStream_t st)
{
    k_chunk_flags<<<(P.N + 255) / 256, 256, 0, st>>>(P, words, start, flag);
    launch_exclusive_scan<int>(flag, offs, P.N, block_sums, total, st);
    k_chunk_write<<<(P.N + 255) / 256, 256, 0, st>>>(P, words, start, flag, offs, chunks);
}

// Device-side bounds after the chunk build: slot ranges of the classes from
// cell_start, chunk ranges from the chunk-head scan (offs[i] = chunks before
// slot i).  One thread.
__global__ void k_bounds(DevParams P, const int *__restrict__ start, const int *__restrict__ offs,
                         const int *__restrict__ total, int *__restrict__ dB)
{
    const int N = P.N;
    const int sb = start[P.T], wb = start[2 * P.T], nch = *total;
    dB[B_FE] = sb;
    dB[B_SB] = sb;
    dB[B_SE] = wb;
    dB[B_CH_S0] = sb < N ? offs[sb] : nch;
    dB[B_CH_W0] = wb < N ? offs[wb] : nch;
    dB[B_CH_END] = nch;
    dB[B_CH_WET] = nch;
}

// Wall chunks whose 27-cell stencil holds no fluid particle ("dry" walls):
// their pressure is read only by fluid neighbours, and no fluid particle can
// come within reach before the next rebuild (the stencil covers every pair
// within MaxRadius+MARGIN at the rebuild, and the trigger keeps every pair
// that is within RadiusP now inside that radius), so the FP32 build skips
// them in pass A.  flag[k] = 1 for wet wall chunk ch_w0 + k, 0 beyond the
// wall chunks (the scan runs over n slots).
__global__ void k_wet_flags(DevParams P, const unsigned long long *__restrict__ words,
                            const int *__restrict__ start, const Chunk *__restrict__ chunks, const int *__restrict__ dB,
                            int n, int *__restrict__ flag)
{
    const int cb = dB[B_CH_W0], ce = dB[B_CH_END];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int wet = 0;
        if (cb + k < ce) {
            const int kc = (int)(word_key(words[chunks[cb + k].i0]) % (unsigned)P.T);
            const int ns = stencil_size(P);
            for (int s = 0; s < ns && !wet; s++) {
                const int cell = stencil_cell(P, kc, s);
                wet = start[cell + 1] > start[cell];  // fluid keys are [0, T)
            }
        }
        flag[k] = wet;
    }
}

// stable partition of the wall chunks: wet first, then dry (into tmp)
__global__ void k_partition_chunks(const Chunk *__restrict__ in, Chunk *__restrict__ tmp, const int *__restrict__ dB,
                                   const int *__restrict__ flag, const int *__restrict__ offs,
                                   const int *__restrict__ total)
{
    const int cb = dB[B_CH_W0], n = dB[B_CH_END] - cb, nwet = *total;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int dst = flag[k] ? offs[k] : nwet + (k - offs[k]);
        tmp[cb + dst] = in[cb + k];
    }
}
__global__ void k_copy_chunks(const Chunk *__restrict__ tmp, Chunk *__restrict__ out, int *__restrict__ dB,
                              const int *__restrict__ total)
{
    const int cb = dB[B_CH_W0], n = dB[B_CH_END] - cb;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[cb + k] = tmp[cb + k];
    if (blockIdx.x == 0 && threadIdx.x == 0) dB[B_CH_WET] = cb + *total;
}

// rebuild decision of neighborCalculation (:1276-1285) from the reduced max
// displacement: max |dx|^2 > (0.5 MARGIN)^2
// rebuild decision of :1264-1286 (max shift since the last rebuild above half
// the margin).  A maximum of +inf (the drift met a non-finite position or
// velocity) sets the sticky B_NONFINITE flag, and no rebuild runs while it is
// set: positions become cell indices only in the rebuild, so every index the
// other kernels use stays the last finite rebuild's.
// The reference's trigger (:1264-1286) on the largest displacement since the
// last rebuild.  Without list reuse (maxshiftL null) every trigger is a full
// rebuild (returns 1).  With it, a trigger keeps the lists (returns 2: the
// trigger positions and neighbour counts are refreshed, no sort) while every
// particle has moved less than S/2 - MARGIN/2 since the lists were built
// (S: their skin past MaxRadius): until the next trigger, which comes before
// any particle moves MARGIN/2 further, every pair within MaxRadius + MARGIN
// then stays within MaxRadius + S of the list-time positions.  A full rebuild
// picks the skin of its lists from the steps since the previous trigger:
// 0.4 dx when triggers come at most four steps apart (the longer lists then
// cost less than the full rebuilds they save), MARGIN otherwise and after a
// list overflow.
__device__ __forceinline__ int decide(const unsigned long long *maxshift, double threshold, int *dB,
                                     const unsigned long long *maxshiftL = nullptr, double dx = 0.0)
{
    const unsigned long long bits = *maxshift;
    if (bits >= 0x7FF0000000000000ull || dB[B_NONFINITE]) {
        dB[B_NONFINITE] = 1;
        dB[B_NEED] = 0;
        return 0;
    }
    const double m2 = __longlong_as_double((long long)bits);
    if (!(m2 > threshold)) {
        dB[B_NEED] = 0;
        dB[B_GAP] += 1;
        return 0;
    }
    int need = 1;
    const int gap = dB[B_GAP] + 1;
    dB[B_GAP] = 0;
    if (maxshiftL) {
        const double mL = __longlong_as_double((long long)*maxshiftL);
        const int h = dB[B_SKIN] > 10 ? dB[B_SKIN] : 10;
        // the FP32 displacements carry a few 1e-7 dx of rounding: 1e-3 dx of slack
        const double lim = (0.005 * h - 0.05 - 0.001) * dx;
        if (!dB[B_LIST_OVF] && lim > 0.0 && mL < lim * lim) need = 2;
        if (need == 1) dB[B_SKIN_NEXT] = dB[B_LIST_OVF] ? 10 : gap <= 4 ? kSkinMaxHundredths : 10;
    }
    dB[B_NEED] = need;
    dB[B_REBUILDS] += 1;
    if (need == 1) dB[B_LIST_BUILDS] += 1;
    return need;
}
__global__ void k_decide(const unsigned long long *maxshift, double threshold, int *dB,
                         const unsigned long long *maxshiftL, double dx)
{
    decide(maxshift, threshold, dB, maxshiftL, dx);
}
// same, inside a CUDA graph: also sets the condition of the graph's rebuild
// node (the full rebuild)
__global__ void k_decide_graph(const unsigned long long *maxshift, double threshold, int *dB,
                               cudaGraphConditionalHandle cond, const unsigned long long *maxshiftL, double dx)
{
    const int need = decide(maxshift, threshold, dB, maxshiftL, dx);
    cudaGraphSetConditional(cond, need == 1 ? 1u : 0u);
}

// The decisions of every scene of an ensemble (thread k: scene k), with the
// threshold of launch_decide; in a graph each scene's IF node gets its
// condition (handles[k]).  The accumulator is cleared for the next drift.
__global__ void k_ens_decide(const EnsScene *__restrict__ tab, int ns, const unsigned long long *handles)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    const EnsScene &e = tab[k];
    const double margin = (0.1 * e.P.dx);
    const double thr = 0.5 * margin * 0.5 * margin;  // :1278
    const int need = decide(e.maxshift, thr, e.dB);
    if (handles) cudaGraphSetConditional((cudaGraphConditionalHandle)handles[k], need ? 1u : 0u);
    *e.maxshift = 0ull;
}
void launch_ens_decide(const EnsScene *tab, int ns, const unsigned long long *handles, cudaStream_t st)
{
    k_ens_decide<<<(ns + 63) / 64, 64, 0, st>>>(tab, ns, handles);
}

void launch_decide(const DevParams &P, const unsigned long long *maxshift, int *dB, unsigned long long graph_cond,
                   cudaStream_t st, const unsigned long long *maxshiftL)
{
    const double margin = (0.1 * P.dx);
    const double thr = 0.5 * margin * 0.5 * margin;  // :1278
    if (graph_cond)
        k_decide_graph<<<1, 1, 0, st>>>(maxshift, thr, dB, (cudaGraphConditionalHandle)graph_cond, maxshiftL, P.dx);
    else
        k_decide<<<1, 1, 0, st>>>(maxshift, thr, dB, maxshiftL, P.dx);
}

void launch_bounds(const DevParams &P, const int *start, const int *offs, const int *total, int *dB, cudaStream_t st)
{
    k_bounds<<<1, 1, 0, st>>>(P, start, offs, total, dB);
}

void launch_wet_partition(const DevParams &P, const unsigned long long *words, const int *start, Chunk *chunks,
                          Chunk *tmp, int *dB, int *flag, int *offs, int *block_sums, int *total, cudaStream_t st)
{
    const int n = P.N;  // upper bound of the number of wall chunks
    k_wet_flags<<<148 * 4, 256, 0, st>>>(P, words, start, chunks, dB, n, flag);
    launch_exclusive_scan<int>(flag, offs, n, block_sums, total, st);
    k_partition_chunks<<<148 * 4, 256, 0, st>>>(chunks, tmp, dB, flag, offs, total);
    k_copy_chunks<<<148 * 4, 256, 0, st>>>(tmp, chunks, dB, total);
}

// int64 neighbour pointers for the CSR diagnostic: small enough to scan on
// the host side of the caller; provided here as a widening copy.
__global__ void k_widen(const int *in, long long *out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}
void launch_widen(const int *in, long long *out, int n, cudaStream_t st)
{
    if (n > 0) k_widen<<<(n + 255) / 256, 256, 0, st>>>(in, out, n);
}

// ---------------------------------------------------- host-layout transfers
// The C ABI takes positions and velocities as x,y,z per particle; the device
// keeps component planes.  These two kernels transpose on the device so that a
// host transfer is one contiguous copy straight from or into the caller's
// buffer.
__global__ void k_xyz_to_planes(const double *__restrict__ xyz, double *__restrict__ planes, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        planes[i] = xyz[3 * (size_t)i];
        planes[(size_t)n + i] = xyz[3 * (size_t)i + 1];
        planes[2 * (size_t)n + i] = xyz[3 * (size_t)i + 2];
    }
}

__global__ void k_planes_to_xyz(const double *__restrict__ planes, double *__restrict__ xyz, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        xyz[3 * (size_t)i] = planes[i];
        xyz[3 * (size_t)i + 1] = planes[(size_t)n + i];
        xyz[3 * (size_t)i + 2] = planes[2 * (size_t)n + i];
    }
}

void launch_xyz_to_planes(const double *xyz, double *planes, int n, cudaStream_t st)
{
    if (n > 0) k_xyz_to_planes<<<(n + 255) / 256, 256, 0, st>>>(xyz, planes, n);
}

void launch_planes_to_xyz(const double *planes, double *xyz, int n, cudaStream_t st)
{
    if (n > 0) k_planes_to_xyz<<<(n + 255) / 256, 256, 0, st>>>(planes, xyz, n);
}

}  // namespace dmph
