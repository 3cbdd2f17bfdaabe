// Host-side derivation of the scene constants (DevParams) from dmph_params.
//
// Restates initializeWeight (source/DEM-MPH.cpp:1007-1125), the scalar part
// of initializeFluid (:1128-1163), initializeWall (:1166-1205) and
// initializeDomain (:1207-1262) with the reference's expression order; this
// file is compiled with -ffp-contract=off so the doubles come out identical.
// It also folds the per-type-pair DEM factors that the reference recomputes
// inside every pair loop (:2318-2338, :2374-2396) into small tables; each
// table entry is the same expression evaluated once.
#include <cmath>
#include <cstring>
#include <string>

#include "dmph_internal.h"

namespace dmph {

static double kernel_norm(double S, double h, int dim) { return dim == 2 ? 1.0 / S * 1.0 / (h * h) : 1.0 / S * 1.0 / (h * h * h); }
static double w_a(double r, double B, double h) { return B * (r / h) * (1.0 - (r / h)) * (1.0 - (r / h)); }
static double w_2(double r, double B, double h) { return B * ((1.0 - r / h) * (1.0 - r / h)); }

int derive_params(const dmph_params &p, int n, DevParams &P, WallMotion &Wm, const char **msg)
{
    std::memset(&P, 0, sizeof(P));
    std::memset(&Wm, 0, sizeof(Wm));
    if (p.dim != 2 && p.dim != 3) return *msg = "dim must be 2 or 3", DMPH_EINVAL;
    if (n <= 0) return *msg = "particle count must be positive", DMPH_EINVAL;
    // the chunk scan handles up to 4096 blocks of 4096 slots
    if (n > (1 << 24)) return *msg = "particle count above 2^24", DMPH_ERANGE;
    if (!(p.particle_spacing > 0.0)) return *msg = "ParticleSpacing must be positive", DMPH_EINVAL;
    if (!(p.dt > 0.0) || !(p.dem_dt > 0.0)) return *msg = "Dt and DEMDt must be positive", DMPH_EINVAL;
    if (!(p.radius_ratio_a > 0.0) || !(p.radius_ratio_p > 0.0) || !(p.radius_ratio_v > 0.0))
        return *msg = "RadiusRatioA/P/V must be positive", DMPH_EINVAL;
    for (int d = 0; d < 3; d++)
        if (!(p.domain_max[d] > p.domain_min[d])) return *msg = "empty domain extent", DMPH_EINVAL;

    const double dx = p.particle_spacing;
    P.dim = p.dim;
    P.N = n;
    P.dx = dx;
    P.V = p.dim == 2 ? dx * dx : dx * dx * dx;
    P.dt = p.dt;
    P.ddt = p.dem_dt;
    // initializeWeight
    P.RA = p.radius_ratio_a * dx;
    P.RG = p.radius_ratio_a * dx;  // RadiusRatioG = RadiusRatioA (:1009)
    P.RP = p.radius_ratio_p * dx;
    P.RV = p.radius_ratio_v * dx;
    double Swa, Swg, Swp, Swv;
    if (p.dim == 2) {
        Swa = 1.0 / 2.0 * 2.0 / 15.0 * M_PI / dx / dx;
        Swg = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / dx / dx;
        Swp = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / dx / dx;
        Swv = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / dx / dx;
        P.R2g = 1.0 / 2.0 * 1.0 / 30.0 * M_PI * P.RG * P.RG / dx / dx / Swg;
    } else {
        Swa = 1.0 / 3.0 * 1.0 / 5.0 * M_PI / dx / dx / dx;
        Swg = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / dx / dx / dx;
        Swp = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / dx / dx / dx;
        Swv = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / dx / dx / dx;
        P.R2g = 1.0 / 3.0 * 4.0 / 105.0 * M_PI * P.RG * P.RG / dx / dx / dx / Swg;
    }
    P.Ba = kernel_norm(Swa, P.RA, p.dim);
    P.Bg = kernel_norm(Swg, P.RG, p.dim);
    P.Bp = kernel_norm(Swp, P.RP, p.dim);
    P.Bv = kernel_norm(Swv, P.RV, p.dim);
    // lattice sums N0a, N0p (:1031-1120): x outer, z inner
    for (int which = 0; which < 2; which++) {
        const double R = which == 0 ? P.RA : P.RP;
        const int range = (int)(R / dx + 3.0);
        const int zr = p.dim == 2 ? 0 : range;
        double sum = 0.0;
        for (int ix = -range; ix <= range; ++ix)
            for (int iy = -range; iy <= range; ++iy)
                for (int iz = -zr; iz <= zr; ++iz) {
                    if (ix == 0 && iy == 0 && iz == 0) continue;
                    const double x = dx * ((double)ix);
                    const double y = dx * ((double)iy);
                    const double z = dx * ((double)iz);
                    const double r2 = p.dim == 2 ? x * x + y * y : x * x + y * y + z * z;
                    if (r2 <= R * R) {
                        const double r = std::sqrt(r2);
                        sum += which == 0 ? w_a(r, P.Ba, R) : w_2(r, P.Bp, R);
                    }
                }
        (which == 0 ? P.N0a : P.N0p) = sum;
    }
    // initializeFluid constants
    double integN, integX;
    if (p.dim == 2) {
        P.CofK = 0.350778153;
        integN = 0.024679383;
        integX = 0.226126699;
    } else {
        P.CofK = 0.326976006;
        integN = 0.021425779;
        integX = 0.233977488;
    }
    for (int t = 0; t < kTypes; t++) {
        P.CofA[t] = p.surface_tension[t] / ((P.RG / dx) * (integN + P.CofK * P.CofK * integX));
        P.ai[t] = P.CofA[t] * (P.CofK) * (P.CofK);
        P.mass[t] = p.density[t] * P.V;
        P.density[t] = p.density[t];
        P.bulk[t] = p.bulk_modulus[t];
        P.bvisc[t] = p.bulk_viscosity[t];
        P.svisc[t] = p.shear_viscosity[t];
        P.friction[t] = p.viscous_friction_coefficient[t];
        for (int u = 0; u < kTypes; u++) P.ratio[t][u] = p.interaction_ratio[t][u];
    }
    // DEM per-type factors (:2318-2338, :2374-2396)
    for (int ti = 0; ti < kTypes; ti++) {
        const double le = std::log(p.restitution_coefficient[ti]);
        P.logE[ti] = le;
        P.cnDen[ti] = std::sqrt(M_PI * M_PI + le * le);
        P.ctFac[ti] = -2 * le / std::sqrt(M_PI * M_PI + le * le);
        for (int tj = 0; tj < kTypes; tj++) {
            const double yi = p.young_modulus[ti], yj = p.young_modulus[tj];
            const double pi_ = p.poisson_ratio[ti], pj = p.poisson_ratio[tj];
            P.Eeff[ti][tj] = (yi * yj) / ((1 - pi_ * pi_) * yj + (1 - pj * pj) * yi);
            P.KtFac[ti][tj] = 8.0 * yi * yj / (((1 + pi_) * (2 - pi_) * yj) + ((1 + pj) * (2 - pj) * yi));
            const double eij = 0.5 * (p.restitution_coefficient[ti] + p.restitution_coefficient[tj]);
            const double lij = eij > 0.0 ? std::log(eij) : 0.0;
            P.pairDamp[ti][tj] = eij > 0.0 ? -2.0 * lij / std::sqrt(M_PI * M_PI + lij * lij) : 0.0;
            P.pairFric[ti][tj] = 0.5 * (p.viscous_friction_coefficient[ti] + p.viscous_friction_coefficient[tj]);
        }
    }
    P.Reff = dx * dx / (dx + dx);
    P.viscC = p.dim == 2 ? 8.0 : 10.0;
    for (int d = 0; d < 3; d++) P.g[d] = p.gravity[d];
    P.surface_tension = 0;
    {
        bool any = false;
        for (int t = 0; t < kTypes; t++)
            for (int u = 0; u < kTypes; u++) any = any || p.interaction_ratio[t][u] != 0.0;
        if (p.flags & DMPH_FLAG_SURFACE_TENSION_ON) any = true;
        if (p.flags & DMPH_FLAG_SURFACE_TENSION_OFF) any = false;
        P.surface_tension = any ? 1 : 0;
    }
    P.wall_dem_coeffs = (p.flags & DMPH_FLAG_WALL_DEM_COEFFS) ? 1 : 0;

    // initializeDomain
    double maxR = 0.0;
    maxR = (P.RA > maxR) ? P.RA : maxR;
    maxR = (P.RG > maxR) ? P.RG : maxR;
    maxR = (P.RP > maxR) ? P.RP : maxR;
    maxR = (P.RV > maxR) ? P.RV : maxR;
    const double margin = (0.1 * dx);
    double cc[3];
    for (int d = 0; d < 3; d++) {
        P.W[d] = p.domain_max[d] - p.domain_min[d];
        P.hW[d] = 0.5 * P.W[d];
        P.dmin[d] = p.domain_min[d];
    }
    // list reuse (FP32 build): cells of MaxRadius + the widest list skin
    // (instead of + MARGIN): the 3-cell stencil then holds every pair within
    // the widest list radius at a rebuild, and every pair within
    // MaxRadius + MARGIN of particles up to (skin - MARGIN) / 2 from the
    // positions of the last sort (the neighbour counts between rebuilds)
    const bool reuse = (p.flags & DMPH_FLAG_LIST_REUSE) && p.precision == DMPH_PRECISION_FP32_SPLIT;
    const double cell_r = reuse ? maxR + 0.01 * kSkinMaxHundredths * dx : maxR + margin;
    cc[0] = std::floor((p.domain_max[0] - p.domain_min[0]) / cell_r);
    cc[1] = std::floor((p.domain_max[1] - p.domain_min[1]) / cell_r);
    cc[2] = p.dim == 2 ? 1 : std::floor((p.domain_max[2] - p.domain_min[2]) / cell_r);
    for (int d = 0; d < 3; d++)
        if (!(cc[d] >= 1.0) || cc[d] > 1.0e7) return *msg = "domain narrower than one neighbour cell", DMPH_EINVAL;
    const double tot = cc[0] * cc[1] * cc[2];
    if (3.0 * tot + 1.0 > 2.0e9) return *msg = "too many cells", DMPH_ERANGE;
    for (int d = 0; d < 3; d++) P.cc[d] = (int)cc[d];
    P.T = (int)tot;
    for (int d = 0; d < 3; d++) P.cw[d] = P.W[d] / P.cc[d];
    // the reference asserts a 3-cell stencil per axis (:1540-1543)
    for (int d = 0; d < (p.dim == 2 ? 2 : 3); d++)
        if ((int)std::ceil(cell_r / P.cw[d]) > 1) return *msg = "cell width below the neighbour radius", DMPH_EINVAL;
    P.rc2 = (maxR + margin) * (maxR + margin);
    P.RA2 = P.RA * P.RA;
    P.RG2 = P.RG * P.RG;
    P.RP2 = P.RP * P.RP;
    P.RV2 = P.RV * P.RV;
    P.dx2 = dx * dx;
    int lg = 0;
    while ((n >> lg) != 0) ++lg;
    P.P2log = lg;
    P.P2 = 1 << lg;

    // initializeWall: theta is |omega|^2, kept as in the reference
    for (int t = DMPH_WALL_BEGIN; t < DMPH_WALL_END; t++) {
        const double *w = p.wall_omega[t];
        double nrm[3] = {0.0, 0.0, 0.0}, q[4];
        const double theta = std::fabs(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (theta != 0.0)
            for (int d = 0; d < 3; d++) nrm[d] = w[d] / theta;
        q[0] = nrm[0] * std::sin(theta * p.dt / 2.0);
        q[1] = nrm[1] * std::sin(theta * p.dt / 2.0);
        q[2] = nrm[2] * std::sin(theta * p.dt / 2.0);
        q[3] = std::cos(theta * p.dt / 2.0);
        double(*R)[3] = Wm.R[t];
        R[0][0] = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[0][1] = 2.0 * (q[0] * q[1] - q[2] * q[3]);
        R[0][2] = 2.0 * (q[0] * q[2] + q[1] * q[3]);
        R[1][0] = 2.0 * (q[0] * q[1] + q[2] * q[3]);
        R[1][1] = -q[0] * q[0] + q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[1][2] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
        R[2][0] = 2.0 * (q[0] * q[2] - q[1] * q[3]);
        R[2][1] = 2.0 * (q[1] * q[2] + q[0] * q[3]);
        R[2][2] = -q[0] * q[0] - q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        for (int d = 0; d < 3; d++) {
            Wm.C[t][d] = p.wall_center[t][d];
            Wm.Vel[t][d] = p.wall_velocity[t][d];
            Wm.Om[t][d] = p.wall_omega[t][d];
        }
    }
    return DMPH_OK;
}

int derive_params(const dmph_params &p, int n, DevParams &P, WallMotion &Wm, std::string &err)
{
    const char *msg = "";
    const int rc = derive_params(p, n, P, Wm, &msg);
    if (rc) err = msg;
    return rc;
}

}  // namespace dmph
