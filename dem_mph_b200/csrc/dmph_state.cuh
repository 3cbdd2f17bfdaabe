// Device pointers of one solver context (see dmph_device.cuh for the layout).
#pragma once

#include "dmph_device.cuh"

namespace dmph {

struct DevState {
    // FP64 particle state, component planes v[d*N + i], current sorted order
    double *pos, *vel, *frc, *xref;
    int *type, *pidx;
    // per-particle fields of the fluid passes
    double *vsp, *divp, *pres;      // VolStrainP, DivergenceP, PressureP
    double *densA, *pA, *gc;        // DensityA, PressureA, GravityCenter (3 planes)
    // DEM per-particle constants (persist across steps, never permuted)
    double *kn, *cn, *kt, *ct;
    double *alpha, *dragC;
    int *nc, *snc;                  // NeighborCount, SolidNeighborCount at rebuild
    // cell structure
    unsigned long long *skey;       // sorted (key << 32 | slot), P2 entries
    int *cell_start;                // 3T + 1 entries
    Chunk *chunks;
};

// Moving-wall constants (calculateWall, source/DEM-MPH.cpp:2846-2900)
struct WallMotion {
    double R[kTypes][3][3];
    double C[kTypes][3];
    double Vel[kTypes][3];
    double Om[kTypes][3];
    int moving;  // 1 when 0.2 <= Time <= 0.4 for this step
};

}  // namespace dmph
