// Warp-cooperative cell-stencil traversal.
//
// One warp owns one chunk: up to 32 consecutive sorted particles of one
// (class, cell) key, lane l holding particle i0 + l.  All lanes therefore share
// one periodic 3x3x3 stencil.  The warp walks the candidate particles j of the
// stencil class by class (fluid, solid, wall) and, inside a class, cell by
// cell in ascending cell id; consecutive cell ids are contiguous in the sorted
// order, so each run of consecutive stencil cells is ONE contiguous slice of
// the particle arrays.  Each slice is staged 32 particles at a time into the
// warp's shared-memory tile with coalesced loads and then read by every lane
// as a broadcast.  Candidates are visited in ascending sorted index, which is
// exactly the order of the reference's neighbour list (calculateNeighbor,
// source/DEM-MPH.cpp:1521-1851): fluid cells, then solid, then wall, each
// over the stencil in ascending cell id.  The reference keeps a Verlet list of
// radius MaxRadius+MARGIN; every pair a kernel accepts (distance <= RadiusP,
// RadiusV, RadiusA or dx at the current positions) is in that list because the
// rebuild trigger (:1264-1286) bounds every displacement by MARGIN/2, so
// traversing the rebuild-time cells and testing the current distance visits
// the same pairs in the same order without materialising the list.
#pragma once

#include "dmph_state.cuh"

namespace dmph {

// Stage(j, slot) loads particle j into the warp's tile slot (called by the
// lane that owns the slot); Visit(j, slot) consumes one candidate for the
// lane's own particle (called only on active lanes).  class_mask selects the
// candidate classes (bit 0 fluid, 1 solid, 2 wall).
template <class Stage, class Visit>
__device__ __forceinline__ void traverse_stencil(const DevParams &P, const int *__restrict__ cell_start, int key_cell,
                                                 int lane, bool active, unsigned class_mask, Stage &&stage,
                                                 Visit &&visit)
{
    const int n = stencil_size(P);
    const int my_id = lane < n ? stencil_cell(P, key_cell, lane) : 0;
    const int prev = __shfl_up_sync(kFull, my_id, 1);
    const bool run_start = lane < n && (lane == 0 || my_id != prev + 1);
    const unsigned starts = __ballot_sync(kFull, run_start);
    for (int cls = 0; cls < 3; cls++) {
        if (!((class_mask >> cls) & 1u)) continue;
        const int off = cls * P.T;
        unsigned m = starts;
        while (m) {
            const int s = __ffs(m) - 1;
            m &= m - 1;
            const int e = m ? (__ffs(m) - 1) : n;
            const int lo = __shfl_sync(kFull, my_id, s);
            const int hi = __shfl_sync(kFull, my_id, e - 1);
            const int jb = __ldg(cell_start + off + lo);
            const int je = __ldg(cell_start + off + hi + 1);
            for (int base = jb; base < je; base += kWarp) {
                const int j = base + lane;
                if (j < je) stage(j, lane);
                __syncwarp();
                const int nb = min(kWarp, je - base);
                if (active)
                    for (int s2 = 0; s2 < nb; ++s2) visit(base + s2, s2);
                __syncwarp();
            }
        }
    }
}

}  // namespace dmph

namespace dmph {

// Same walk as traverse_stencil, but hands each staged batch of up to 32
// candidates to Batch(base, nb), called by every lane of the warp (active or
// not) between the staging barriers, so the caller can first build a per-lane
// bitmask of the candidates in range and then loop over the set bits.
template <class Stage, class Batch>
__device__ __forceinline__ void traverse_stencil_batched(const DevParams &P, const int *__restrict__ cell_start,
                                                         int key_cell, int lane, unsigned class_mask, Stage &&stage,
                                                         Batch &&batch)
{
    const int n = stencil_size(P);
    const int my_id = lane < n ? stencil_cell(P, key_cell, lane) : 0;
    const int prev = __shfl_up_sync(kFull, my_id, 1);
    const bool run_start = lane < n && (lane == 0 || my_id != prev + 1);
    const unsigned starts = __ballot_sync(kFull, run_start);
    for (int cls = 0; cls < 3; cls++) {
        if (!((class_mask >> cls) & 1u)) continue;
        const int off = cls * P.T;
        unsigned m = starts;
        while (m) {
            const int s = __ffs(m) - 1;
            m &= m - 1;
            const int e = m ? (__ffs(m) - 1) : n;
            const int lo = __shfl_sync(kFull, my_id, s);
            const int hi = __shfl_sync(kFull, my_id, e - 1);
            const int jb = __ldg(cell_start + off + lo);
            const int je = __ldg(cell_start + off + hi + 1);
            for (int base = jb; base < je; base += kWarp) {
                const int j = base + lane;
                if (j < je) stage(j, lane);
                __syncwarp();
                batch(base, min(kWarp, je - base));
                __syncwarp();
            }
        }
    }
}

}  // namespace dmph

namespace dmph {

// Per-lane walk of a particle's Verlet list (list mode): entry k of slot i is
// visited in list order (ascending j, the order of the reference's neighbour
// list), each lane staging its own candidate into its own tile slot, so the
// same Stage/Visit callbacks serve both walks.  LIST = false walks the stencil.
template <bool LIST, class Stage, class Visit>
__device__ __forceinline__ void traverse_pairs(const DevParams &P, const DevState &S, int key_cell, int lane,
                                               bool active, int i, unsigned class_mask, Stage &&stage, Visit &&visit)
{
    if (!LIST) {
        traverse_stencil(P, S.cell_start, key_cell, lane, active, class_mask, stage, visit);
        return;
    }
    if (!active) return;
    const int cnt = S.nbn[i];
    const long long ld = P.N;
    for (int k = 0; k < cnt; ++k) {
        const int j = (int)(__ldg(S.nbl + list_index(k, i, ld)) & 0xFFFFFFu);
        stage(j, lane);
        visit(j, lane);
    }
}

}  // namespace dmph
