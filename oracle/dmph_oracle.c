/*
 * dmph_oracle.c — CPU restatement of the reference DEM-MPH explicit step.
 *
 * TEST INFRASTRUCTURE ONLY (see dmph_oracle.h).  Parity is pinned against the
 * reference built from its own source (oracle/_ref) and the golden fixtures.
 *
 * Every arithmetic expression below keeps the reference's evaluation order
 * (C evaluates * and / left to right and g++ -O3 without -ffast-math keeps
 * that order), so that this restatement reproduces the reference bit for bit;
 * each function cites the reference lines it restates.  All citations are
 * source/DEM-MPH.cpp of Ryo1011gd/DEM_MPH.
 */
#include "dmph_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NT DMPH_TYPE_COUNT

static int is_fluid(int t) { return DMPH_FLUID_BEGIN <= t && t < DMPH_FLUID_END; }
static int is_solid(int t) { return DMPH_SOLID_BEGIN <= t && t < DMPH_SOLID_END; }
static int is_wall(int t) { return DMPH_WALL_BEGIN <= t && t < DMPH_WALL_END; }

struct dmph_oracle {
    dmph_params p;
    int dim, N, P2, P2log;
    double dx, V, W[3];
    double RA, RG, RP, RV, maxR, margin;
    double Swa, Swg, Swp, Swv, N0a, N0p, R2g, CofK, CofA[NT];
    double Ba, Bg, Bp, Bv; /* (1/Sw)/h^d of each kernel */
    double wallR[NT][3][3], wallC[NT][3];
    int cc[3], T;
    double cw[3];
    int demSteps;
    double time;
    long steps, rebuilds;
    /* particle arrays in the current sorted order */
    int *pidx, *prop;
    double *x, *v, *F, *xref;
    double *mass, *kappa, *lambda, *mu;
    double *densA, *gc, *pA, *vsp, *div, *P;
    double *kn, *cn, *kt, *ct, *alpha, *dragC;
    double *fsc; /* per particle: sum of |pair force| terms of the step (test scale, not a reference array) */
    double *vir; /* VirialPressureAtParticle, computed when requested */
    int *nc, *fnc, *snc;
    long *nptr;
    int *nind;
    long nindCount;
    int *key, *payload;
    int *cfb, *cfe, *csb, *cse, *cwb, *cwe;
    int fb, fe, sb, se, wb, we;
    /* rigid bodies (0 = off) */
    int B;
    int *bid;          /* body of each slot, permuted with the sort */
    double *brho;      /* density of each body */
    int *bptr, *bmrow; /* members (input rows) by body */
    double *br0, *bX, *bV, *bL, *bq, *bM, *bIi;
    double *fdem;      /* 6 per particle: contact force and offset torque */
};

/* Mod macro, :76 */
static inline double pmod(double a, double w) { return ((a) - (w)*floor((a) / (w))); }

/* periodic minimum-image displacement x_j - x_i, the xij of every pair loop */
static inline void rel(const dmph_oracle *o, const double *xi, const double *xj, double *q)
{
    for (int d = 0; d < 3; d++) q[d] = pmod(xj[d] - xi[d] + 0.5 * o->W[d], o->W[d]) - 0.5 * o->W[d];
}
static inline double sq3(const double *q) { return (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]); }
static inline double nrm3(double a, double b, double c) { return sqrt(a * a + b * b + c * c); }

/* smoothing kernels, :272-342 ; B = (1/Sw)/h^dim */
static inline double k_wa(double r, double B, double h) { return B * (r / h) * (1.0 - (r / h)) * (1.0 - (r / h)); }
static inline double k_dwa(double r, double B, double h)
{
    return B * (1.0 - (r / h)) * (1.0 - 3.0 * (r / h)) * (1.0 / h);
}
static inline double k_w(double r, double B, double h) { return B * ((1.0 - r / h) * (1.0 - r / h)); }
static inline double k_dw(double r, double B, double h) { return B * (-2.0 / h * (1.0 - r / h)); }

static void *xcalloc(size_t n, size_t s)
{
    void *p = calloc(n ? n : 1, s);
    if (!p) {
        fprintf(stderr, "dmph_oracle: out of memory\n");
        exit(1);
    }
    return p;
}

/* initializeWeight, :1007-1125 */
static void init_weight(dmph_oracle *o)
{
    const double dx = o->dx;
    o->RA = o->p.radius_ratio_a * dx;
    o->RG = o->p.radius_ratio_a * dx; /* RadiusRatioG = RadiusRatioA, :1009 */
    o->RP = o->p.radius_ratio_p * dx;
    o->RV = o->p.radius_ratio_v * dx;
    if (o->dim == 2) {
        o->Swa = 1.0 / 2.0 * 2.0 / 15.0 * M_PI / dx / dx;
        o->Swg = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / dx / dx;
        o->Swp = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / dx / dx;
        o->Swv = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / dx / dx;
        o->R2g = 1.0 / 2.0 * 1.0 / 30.0 * M_PI * o->RG * o->RG / dx / dx / o->Swg;
    } else {
        o->Swa = 1.0 / 3.0 * 1.0 / 5.0 * M_PI / dx / dx / dx;
        o->Swg = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / dx / dx / dx;
        o->Swp = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / dx / dx / dx;
        o->Swv = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / dx / dx / dx;
        o->R2g = 1.0 / 3.0 * 4.0 / 105.0 * M_PI * o->RG * o->RG / dx / dx / dx / o->Swg;
    }
#define HD(h) (o->dim == 2 ? ((h) * (h)) : ((h) * (h) * (h)))
    o->Ba = 1.0 / o->Swa * 1.0 / HD(o->RA);
    o->Bg = 1.0 / o->Swg * 1.0 / HD(o->RG);
    o->Bp = 1.0 / o->Swp * 1.0 / HD(o->RP);
    o->Bv = 1.0 / o->Swv * 1.0 / HD(o->RV);
#undef HD
    /* lattice sums N0a, N0p over a perfect grid, :1031-1120 */
    for (int which = 0; which < 2; which++) {
        const double R = which == 0 ? o->RA : o->RP;
        const int range = (int)(R / dx + 3.0);
        const int zr = o->dim == 2 ? 0 : range;
        double sum = 0.0;
        for (int ix = -range; ix <= range; ++ix)
            for (int iy = -range; iy <= range; ++iy)
                for (int iz = -zr; iz <= zr; ++iz) {
                    if (ix == 0 && iy == 0 && iz == 0) continue;
                    const double x = dx * ((double)ix);
                    const double y = dx * ((double)iy);
                    const double z = dx * ((double)iz);
                    const double r2 = o->dim == 2 ? x * x + y * y : x * x + y * y + z * z;
                    if (r2 <= R * R) {
                        const double r = sqrt(r2);
                        sum += which == 0 ? k_wa(r, o->Ba, R) : k_w(r, o->Bp, R);
                    }
                }
        if (which == 0)
            o->N0a = sum;
        else
            o->N0p = sum;
    }
}

/* initializeFluid, :1128-1163 (the per-particle part is redone every step) */
static void init_fluid(dmph_oracle *o)
{
    double integN, integX;
    if (o->dim == 2) {
        o->CofK = 0.350778153;
        integN = 0.024679383;
        integX = 0.226126699;
    } else {
        o->CofK = 0.326976006;
        integN = 0.021425779;
        integX = 0.233977488;
    }
    for (int t = 0; t < NT; t++)
        o->CofA[t] = o->p.surface_tension[t] / ((o->RG / o->dx) * (integN + o->CofK * o->CofK * integX));
    for (int i = 0; i < o->N; i++) {
        const int t = o->prop[i];
        o->mass[i] = o->p.density[t] * o->V;
        o->kappa[i] = o->p.bulk_modulus[t];
        o->lambda[i] = o->p.bulk_viscosity[t];
        o->mu[i] = o->p.shear_viscosity[t];
    }
}

/* initializeWall, :1166-1205.  theta is |omega|^2 in the reference (abs of the
 * squared norm), kept as is. */
static void init_wall(dmph_oracle *o)
{
    for (int t = DMPH_WALL_BEGIN; t < DMPH_WALL_END; t++) {
        const double *w = o->p.wall_omega[t];
        double n[3] = {0.0, 0.0, 0.0}, q[4];
        const double theta = fabs(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (theta != 0.0)
            for (int d = 0; d < 3; d++) n[d] = w[d] / theta;
        const double dt = o->p.dt;
        q[0] = n[0] * sin(theta * dt / 2.0);
        q[1] = n[1] * sin(theta * dt / 2.0);
        q[2] = n[2] * sin(theta * dt / 2.0);
        q[3] = cos(theta * dt / 2.0);
        double(*R)[3] = o->wallR[t];
        R[0][0] = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[0][1] = 2.0 * (q[0] * q[1] - q[2] * q[3]);
        R[0][2] = 2.0 * (q[0] * q[2] + q[1] * q[3]);
        R[1][0] = 2.0 * (q[0] * q[1] + q[2] * q[3]);
        R[1][1] = -q[0] * q[0] + q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[1][2] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
        R[2][0] = 2.0 * (q[0] * q[2] - q[1] * q[3]);
        R[2][1] = 2.0 * (q[1] * q[2] + q[0] * q[3]);
        R[2][2] = -q[0] * q[0] - q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        for (int d = 0; d < 3; d++) o->wallC[t][d] = o->p.wall_center[t][d];
    }
}

/* initializeDomain, :1207-1262 */
static void init_domain(dmph_oracle *o)
{
    double m = 0.0;
    m = (o->RA > m) ? o->RA : m;
    m = (o->RG > m) ? o->RG : m;
    m = (o->RP > m) ? o->RP : m;
    m = (o->RV > m) ? o->RV : m;
    o->maxR = m;
    double ccount[3];
    for (int d = 0; d < 3; d++) o->W[d] = o->p.domain_max[d] - o->p.domain_min[d];
    ccount[0] = floor((o->p.domain_max[0] - o->p.domain_min[0]) / (o->maxR + o->margin));
    ccount[1] = floor((o->p.domain_max[1] - o->p.domain_min[1]) / (o->maxR + o->margin));
    ccount[2] = o->dim == 2 ? 1 : floor((o->p.domain_max[2] - o->p.domain_min[2]) / (o->maxR + o->margin));
    for (int d = 0; d < 3; d++) o->cc[d] = (int)ccount[d];
    o->T = ccount[0] * ccount[1] * ccount[2];
    for (int d = 0; d < 3; d++) o->cw[d] = o->W[d] / o->cc[d];
}

static inline int wrapi(int a, int c) { return ((a) % c + c) % c; }
static inline int cell_id(const dmph_oracle *o, int ix, int iy, int iz)
{
    if (o->dim == 2) return wrapi(ix, o->cc[0]) * o->cc[1] + wrapi(iy, o->cc[1]);
    return wrapi(ix, o->cc[0]) * o->cc[1] * o->cc[2] + wrapi(iy, o->cc[1]) * o->cc[2] + wrapi(iz, o->cc[2]);
}

/* calculateCellParticle, :1288-1519: key = cell id + class offset, bitonic
 * network over the power-of-two padded array (ties are swapped inside
 * descending sub-blocks, so the network must be reproduced exactly), cell
 * ranges, permutation of ParticleIndex, Property, Position and Velocity. */
static void cell_sort(dmph_oracle *o)
{
    const int N = o->N, P2 = o->P2, T = o->T;
    int *key = o->key, *pay = o->payload;
#pragma omp parallel for
    for (int i = 0; i < P2; i++) {
        if (i < N) {
            const double *x = o->x + 3 * (size_t)i;
            const int ix = ((int)floor((x[0] - o->p.domain_min[0]) / o->cw[0])) % o->cc[0];
            const int iy = ((int)floor((x[1] - o->p.domain_min[1]) / o->cw[1])) % o->cc[1];
            const int iz = ((int)floor((x[2] - o->p.domain_min[2]) / o->cw[2])) % o->cc[2];
            int k = cell_id(o, ix, iy, iz);
            if (is_solid(o->prop[i]))
                k += T;
            else if (is_wall(o->prop[i]))
                k += 2 * T;
            key[i] = k;
            pay[i] = i;
        } else {
            key[i] = 3 * T;
            pay[i] = N;
        }
    }
    for (int stage = 0; stage < o->P2log; ++stage)
        for (int sub = 0; sub <= stage; ++sub) {
            const int dist = 1 << (stage - sub);
#pragma omp parallel for
            for (int i = 0; i < P2; ++i) {
                const int up = ((i >> stage) & 2) == 0;
                if ((i & dist) == 0 && ((key[i] > key[i | dist]) == up)) {
                    const int tk = key[i], tp = pay[i];
                    key[i] = key[i | dist];
                    pay[i] = pay[i | dist];
                    key[i | dist] = tk;
                    pay[i | dist] = tp;
                }
            }
        }
    /* cell ranges: begin = #keys below, end = #keys up to (the reference's
     * boundary detection + count scan gives exactly these, :1340-1438) */
    {
        int *lb = xcalloc((size_t)3 * T + 1, sizeof(int));
        int k = 0;
        for (int c = 0; c <= 3 * T; c++) {
            while (k < N && key[k] < c) k++;
            lb[c] = k;
        }
        for (int c = 0; c < T; c++) {
            o->cfb[c] = lb[c];
            o->cfe[c] = lb[c + 1];
            o->csb[c] = lb[T + c];
            o->cse[c] = lb[T + c + 1];
            o->cwb[c] = lb[2 * T + c];
            o->cwe[c] = lb[2 * T + c + 1];
        }
        free(lb);
    }
    o->fb = o->cfb[0];
    o->fe = o->cfe[T - 1];
    o->sb = o->csb[0];
    o->se = o->cse[T - 1];
    o->wb = o->cwb[0];
    o->we = o->cwe[T - 1];
    /* permute the four arrays the reference permutes (:1455-1518) */
    int *ti = xcalloc((size_t)N, sizeof(int));
    double *td = xcalloc((size_t)3 * N, sizeof(double));
    for (int i = 0; i < N; i++) ti[i] = o->pidx[pay[i]];
    memcpy(o->pidx, ti, sizeof(int) * N);
    for (int i = 0; i < N; i++) ti[i] = o->prop[pay[i]];
    memcpy(o->prop, ti, sizeof(int) * N);
    if (o->bid) {
        for (int i = 0; i < N; i++) ti[i] = o->bid[pay[i]];
        memcpy(o->bid, ti, sizeof(int) * N);
    }
    for (int i = 0; i < N; i++)
        for (int d = 0; d < 3; d++) td[3 * i + d] = o->x[3 * (size_t)pay[i] + d];
    memcpy(o->x, td, sizeof(double) * 3 * N);
    for (int i = 0; i < N; i++)
        for (int d = 0; d < 3; d++) td[3 * i + d] = o->v[3 * (size_t)pay[i] + d];
    memcpy(o->v, td, sizeof(double) * 3 * N);
    free(ti);
    free(td);
}

/* The stencil cells of particle i in the reference's visiting order
 * (:1553-1575 and the triple loop that follows): along each axis the three
 * wrapped neighbour indices in ascending order (the jXmin rotation produces
 * exactly that, duplicates included when an axis has fewer than 3 cells);
 * x outer, z inner. */
static int stencil(const dmph_oracle *o, int i, int *cells)
{
    const int k = o->key[i];
    const int c1 = o->cc[1], c2 = o->cc[2];
    const int ic[3] = {(k / (c1 * c2)) % o->T, (k / c2) % c1, k % c2};
    int ax[3][3], na[3];
    for (int d = 0; d < 3; d++) {
        const int r = (o->dim == 2 && d == 2) ? 0 : 1;
        na[d] = 2 * r + 1;
        int tmp[3];
        for (int j = 0; j < na[d]; j++) tmp[j] = wrapi(ic[d] - r + j, o->cc[d]);
        /* rotate so the sequence starts at jmin = max(0, 2r - (ic+r)%C) */
        const int b = (2 * r) - (ic[d] + r) % o->cc[d];
        const int jmin = b > 0 ? b : 0;
        for (int j = 0; j < na[d]; j++) ax[d][j] = tmp[(jmin + j) % na[d]];
    }
    int n = 0;
    for (int a = 0; a < na[0]; a++)
        for (int b = 0; b < na[1]; b++)
            for (int c = 0; c < na[2]; c++) cells[n++] = cell_id(o, ax[0][a], ax[1][b], ax[2][c]);
    return n;
}

/* calculateNeighbor, :1521-1851 */
static void build_neighbors(dmph_oracle *o)
{
    const int N = o->N;
    const double rc2 = (o->maxR + o->margin) * (o->maxR + o->margin);
    const int *begs[3] = {o->cfb, o->csb, o->cwb}, *ends[3] = {o->cfe, o->cse, o->cwe};
#pragma omp parallel for
    for (int i = 0; i < N; i++) {
        int cells[27];
        const int nc = stencil(o, i, cells);
        int cnt[3] = {0, 0, 0};
        for (int cls = 0; cls < 3; cls++)
            for (int s = 0; s < nc; s++)
                for (int j = begs[cls][cells[s]]; j < ends[cls][cells[s]]; j++) {
                    double q[3];
                    rel(o, o->x + 3 * (size_t)i, o->x + 3 * (size_t)j, q);
                    if (sq3(q) <= rc2) cnt[cls]++;
                }
        o->nc[i] = cnt[0] + cnt[1] + cnt[2];
        o->fnc[i] = cnt[0];
        o->snc[i] = cnt[1];
    }
    o->nptr[0] = 0;
    for (int i = 0; i < N; i++) o->nptr[i + 1] = o->nptr[i] + o->nc[i];
    o->nindCount = o->nptr[N];
    free(o->nind);
    o->nind = xcalloc((size_t)o->nindCount, sizeof(int));
#pragma omp parallel for
    for (int i = 0; i < N; i++) {
        int cells[27];
        const int nc = stencil(o, i, cells);
        long w = o->nptr[i];
        for (int cls = 0; cls < 3; cls++)
            for (int s = 0; s < nc; s++)
                for (int j = begs[cls][cells[s]]; j < ends[cls][cells[s]]; j++) {
                    double q[3];
                    rel(o, o->x + 3 * (size_t)i, o->x + 3 * (size_t)j, q);
                    if (sq3(q) <= rc2) o->nind[w++] = j;
                }
    }
    memcpy(o->xref, o->x, sizeof(double) * 3 * N);
}

#define FOR_NEIGHBORS(o, i, j)                                                                                \
    for (long jn_ = (o)->nptr[i], je_ = (o)->nptr[(i) + 1], j = 0; jn_ < je_ && ((j = (o)->nind[jn_]), 1); \
         jn_++)

/* calculateDensityA :1956-1984 */
static void density_a(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double sum = 0.0;
        FOR_NEIGHBORS(o, i, j)
        {
            if (is_solid(o->prop[i]) && is_wall(o->prop[j])) continue;
            if (i == j) continue;
            const double ratio = o->p.interaction_ratio[o->prop[i]][o->prop[j]];
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (o->RA * o->RA - r2 >= 0) sum += ratio * k_wa(sqrt(r2), o->Ba, o->RA);
        }
        o->densA[i] = sum;
    }
}

/* calculateGravityCenter :1987-2019 */
static void gravity_center(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double s[3] = {0.0, 0.0, 0.0};
        FOR_NEIGHBORS(o, i, j)
        {
            if (is_solid(o->prop[i]) && is_wall(o->prop[j])) continue;
            if (i == j) continue;
            const double ratio = o->p.interaction_ratio[o->prop[i]][o->prop[j]];
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (o->RG * o->RG - r2 >= 0) {
                const double w = ratio * k_w(sqrt(r2), o->Bg, o->RG);
                for (int d = 0; d < 3; d++) s[d] += q[d] * w / o->R2g * o->RG;
            }
        }
        for (int d = 0; d < 3; d++) o->gc[3 * i + d] = s[d];
    }
}

/* calculateDensityP :2129-2156 */
static void density_p(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double sum = 0.0;
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (o->RP * o->RP - r2 >= 0) sum += k_w(sqrt(r2), o->Bp, o->RP);
        }
        o->vsp[i] = (sum - o->N0p);
    }
}

/* calculateDivergenceP :2158-2198 (solid-wall, wall-solid and solid-solid
 * pairs skipped; fluid-solid pairs kept) */
static void divergence_p(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double sum = 0.0;
        const int ti = o->prop[i];
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            const int tj = o->prop[j];
            if (is_solid(ti) && is_wall(tj)) continue;
            if (is_solid(tj) && is_wall(ti)) continue;
            if (is_solid(tj) && is_solid(ti)) continue;
            if (o->RP * o->RP - r2 >= 0) {
                const double r = sqrt(r2);
                const double dw = k_dw(r, o->Bp, o->RP);
                const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                double u[3];
                for (int d = 0; d < 3; d++) u[d] = o->v[3 * j + d] - o->v[3 * i + d];
                for (int d = 0; d < 3; d++) sum -= u[d] * e[d] * dw;
            }
        }
        o->div[i] = sum;
    }
}

/* calculatePhysicalCoefficients :1918-1949 */
static void physical_coefficients(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        const int t = o->prop[i];
        o->mass[i] = o->p.density[t] * o->V;
        if (o->bid && o->bid[i] >= 0) o->mass[i] = o->brho[o->bid[i]] * o->V;
        o->kappa[i] = o->p.bulk_modulus[t];
        if (o->vsp[i] < 0.0) o->kappa[i] = 0.0;
        o->lambda[i] = o->p.bulk_viscosity[t];
        o->mu[i] = o->p.shear_viscosity[t];
    }
}

/* calculateDragForce :2740-2807 (solid range; DragC of the last fluid
 * neighbour is the per-particle output; the solid's own density is used) */
static void drag_force(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = o->sb; i < o->se; ++i) {
        double f[3] = {0.0, 0.0, 0.0};
        if (o->nc[i] > 0)
            o->alpha[i] = (double)(o->snc[i]) / (o->nc[i]);
        else
            o->alpha[i] = 0.0;
        const double rho = (o->bid && o->bid[i] >= 0) ? o->brho[o->bid[i]] : o->p.density[o->prop[i]];
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
            if (o->RP * o->RP - r2 > 0 && is_fluid(o->prop[j])) {
                double u[3];
                for (int d = 0; d < 3; d++) u[d] = o->v[3 * j + d] - o->v[3 * i + d];
                const double Vs = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                const double a = o->alpha[i];
                const double Re = a * rho * Vs * o->dx / (o->mu[j]);
                double cd;
                if (a < 0.8)
                    cd = (4.0 / 3.0) * (150.0 * (1.0 - a) / (a * Re) + 1.75);
                else if (Re <= 1000.0 && a >= 0.8)
                    cd = 24.0 * (1.0 + 0.15 * pow(Re, 0.687)) / (a * Re) * pow(a, -2.65);
                else
                    cd = 0.44;
                o->dragC[i] = cd;
                for (int d = 0; d < 3; d++) f[d] += 0.5 * cd * rho * o->dx * o->dx * o->dx * u[d] * Vs;
                o->fsc[i] += fabs(0.5 * cd * rho * o->dx * o->dx * o->dx * Vs * Vs);
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += f[d];
    }
}

/* calculatePressureP :2200-2246 (solids neither get a pressure nor a
 * pressure force; their PressureP is never written and stays 0) */
static void pressure_force(dmph_oracle *o, const double *P, double *F, double *fsc);

static void pressure_p(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        if (is_solid(o->prop[i])) continue;
        o->P[i] = -o->lambda[i] * o->div[i] + o->kappa[i] * o->vsp[i];
    }
    pressure_force(o, o->P, o->F, o->fsc);
}

/* the pressure-gradient force of calculatePressureP :2213-2246 for a given
 * pressure field, added to F (and its term magnitudes to fsc when non-NULL) */
static void pressure_force(dmph_oracle *o, const double *P, double *F, double *fsc)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        const int ti = o->prop[i];
        if (is_solid(ti)) continue;
        double f[3] = {0.0, 0.0, 0.0};
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            const int tj = o->prop[j];
            if (is_solid(ti) && is_wall(tj)) continue;
            if (is_solid(tj) && is_wall(ti)) continue;
            if (is_solid(tj) && is_solid(ti)) continue;
            if (o->RP * o->RP - r2 > 0) {
                const double r = sqrt(r2);
                const double dw = k_dw(r, o->Bp, o->RP);
                const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                for (int d = 0; d < 3; d++) f[d] += (P[i] + P[j]) * g[d] * o->V;
                if (fsc) fsc[i] += fabs((P[i] + P[j]) * dw * o->V);
            }
        }
        for (int d = 0; d < 3; d++) F[3 * i + d] += f[d];
    }
}

/* calculatePressureA :2022-2071 */
static void pressure_a(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        o->pA[i] = o->CofA[o->prop[i]] * (o->densA[i] - o->N0a) / o->dx;
        if (o->N0a <= o->densA[i]) o->pA[i] = 0.0;
    }
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double f[3] = {0.0, 0.0, 0.0};
        const int ti = o->prop[i];
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            const int tj = o->prop[j];
            const double rij_ = o->p.interaction_ratio[ti][tj];
            const double rji_ = o->p.interaction_ratio[tj][ti];
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (is_solid(ti) && is_wall(tj)) continue;
            if (is_solid(tj) && is_wall(ti)) continue;
            if (o->RA * o->RA - r2 > 0) {
                const double r = sqrt(r2);
                const double dwij = rij_ * k_dwa(r, o->Ba, o->RA);
                const double dwji = rji_ * k_dwa(r, o->Ba, o->RA);
                const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                for (int d = 0; d < 3; d++) f[d] += (o->pA[i] * dwij + o->pA[j] * dwji) * e[d] * o->V;
                o->fsc[i] += fabs((o->pA[i] * dwij + o->pA[j] * dwji) * o->V);
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += f[d];
    }
}

/* calculateDiffuseInterface :2074-2127 (aj uses particle i's CofA, as in the
 * reference :2088) */
static void diffuse_interface(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        const int ti = o->prop[i];
        const double ai = o->CofA[ti] * (o->CofK) * (o->CofK);
        double f[3] = {0.0, 0.0, 0.0};
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            const double aj = o->CofA[ti] * (o->CofK) * (o->CofK);
            const int tj = o->prop[j];
            const double rij_ = o->p.interaction_ratio[ti][tj];
            const double rji_ = o->p.interaction_ratio[tj][ti];
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (is_solid(ti) && is_wall(tj)) continue;
            if (is_solid(tj) && is_wall(ti)) continue;
            if (o->RG * o->RG - r2 > 0) {
                const double r = sqrt(r2);
                const double wij = rij_ * k_w(r, o->Bg, o->RG);
                const double wji = rji_ * k_w(r, o->Bg, o->RG);
                const double *gi = o->gc + 3 * i, *gj = o->gc + 3 * j;
                for (int d = 0; d < 3; d++)
                    f[d] -= (aj * gj[d] * wji - ai * gi[d] * wij) / o->R2g * o->RG * (o->V / o->dx);
                const double dwij = rij_ * k_dw(r, o->Bg, o->RG);
                const double dwji = rji_ * k_dw(r, o->Bg, o->RG);
                const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                double gr = 0.0;
                for (int d = 0; d < 3; d++) gr += (aj * gj[d] * dwji - ai * gi[d] * dwij) * q[d];
                for (int d = 0; d < 3; d++) f[d] -= (gr)*e[d] / o->R2g * o->RG * (o->V / o->dx);
                o->fsc[i] += (fabs(gr) + nrm3(aj * gj[0] * wji - ai * gi[0] * wij, aj * gj[1] * wji - ai * gi[1] * wij,
                                              aj * gj[2] * wji - ai * gi[2] * wij)) /
                             o->R2g * o->RG * (o->V / o->dx);
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += f[d];
    }
}

/* calculateViscosityV :2248-2293 (factor 8 in 2D, 10 in 3D) */
static void viscosity_v(dmph_oracle *o)
{
    const double C = o->dim == 2 ? 8.0 : 10.0;
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double f[3] = {0.0, 0.0, 0.0};
        const int ti = o->prop[i];
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (is_solid(ti) && is_wall(o->prop[j])) continue;
            if (o->RV * o->RV - r2 > 0) {
                const double r = sqrt(r2);
                const double dwij = -k_dw(r, o->Bv, o->RV);
                const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                double u[3];
                for (int d = 0; d < 3; d++) u[d] = o->v[3 * j + d] - o->v[3 * i + d];
                const double muij = 2.0 * (o->mu[i] * o->mu[j]) / (o->mu[i] + o->mu[j]);
                for (int d = 0; d < 3; d++)
                    f[d] += C * muij * (u[0] * e[0] + u[1] * e[1] + u[2] * e[2]) * e[d] * dwij / r * o->V;
                o->fsc[i] += fabs(C * muij * nrm3(u[0], u[1], u[2]) * dwij / r * o->V);
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += f[d];
    }
}

/* calculateBuoyancyForce :2699-2738 */
static void buoyancy_force(dmph_oracle *o)
{
#pragma omp parallel for
    for (int i = o->sb; i < o->se; ++i) {
        double f[3] = {0.0, 0.0, 0.0};
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
            if (o->RP * o->RP - r2 > 0 && is_fluid(o->prop[j])) {
                const double w = k_w(sqrt(r2), o->Bp, o->RP);
                for (int d = 0; d < 3; d++) f[d] += o->p.density[o->prop[j]] * o->V * o->p.gravity[d] * w;
                o->fsc[i] += fabs(o->p.density[o->prop[j]] * o->V * w) *
                             nrm3(o->p.gravity[0], o->p.gravity[1], o->p.gravity[2]);
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] -= f[d];
    }
}

/* calculateGravity :2811-2829, calculateAcceleration :2832-2843 */
static void gravity_and_acceleration(dmph_oracle *o)
{
    for (int i = o->fb; i < o->fe; ++i)
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += o->mass[i] * o->p.gravity[d];
    for (int i = o->sb; i < o->se; ++i)
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += o->mass[i] * o->p.gravity[d];
    for (int i = o->fb; i < o->fe; ++i)
        for (int d = 0; d < 3; d++) o->v[3 * i + d] += o->F[3 * i + d] / o->mass[i] * o->p.dt;
}

/* calculateNormalDirectionCoefficient :2298-2343 and
 * calculateTangentialDirectionCoefficient :2346-2399: per particle, the
 * constants of the LAST neighbour (any type) within dx; left untouched when
 * none is in range (values persist across steps and are not permuted by the
 * sort).  The tangential function's uninitialised vij only feeds unused
 * temporaries and is omitted. */
static void dem_coefficients(dmph_oracle *o)
{
    const double dx = o->dx;
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        const int ti = o->prop[i];
        if (is_fluid(ti)) continue;
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
            if (r2 <= dx * dx) {
                const int tj = o->prop[j];
                const double r = sqrt(r2);
                const double yi = o->p.young_modulus[ti], yj = o->p.young_modulus[tj];
                const double pi_ = o->p.poisson_ratio[ti], pj = o->p.poisson_ratio[tj];
                const double Eeff = (yi * yj) / ((1 - pi_ * pi_) * yj + (1 - pj * pj) * yi);
                const double Reff = dx * dx / (dx + dx);
                const double ov = fmax(0.0, dx - r);
                o->kn[i] = (4.0 / 3.0) * Eeff * sqrt(Reff * ov);
                const double le = log(o->p.restitution_coefficient[ti]);
                const double mij = o->mass[i] * o->mass[j] / (o->mass[i] + o->mass[j]);
                o->cn[i] = -2.0 * sqrt(mij * o->kn[i]) * le / sqrt(M_PI * M_PI + le * le);
            }
        }
    }
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        const int ti = o->prop[i];
        if (is_fluid(ti)) continue;
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
            if (r2 <= dx * dx) {
                const int tj = o->prop[j];
                const double r = sqrt(r2);
                const double yi = o->p.young_modulus[ti], yj = o->p.young_modulus[tj];
                const double pi_ = o->p.poisson_ratio[ti], pj = o->p.poisson_ratio[tj];
                const double Reff = dx * dx / (dx + dx);
                const double ov = fmax(0.0, dx - r);
                const double ks = 8.0 * yi * yj / (((1 + pi_) * (2 - pi_) * yj) + ((1 + pj) * (2 - pj) * yi)) *
                                  sqrt(Reff * sqrt(ov));
                o->kt[i] = ks;
                const double le = log(o->p.restitution_coefficient[ti]);
                const double damp = -2 * le / sqrt(M_PI * M_PI + le * le);
                const double mij = (o->mass[i] * o->mass[j]) / (o->mass[i] + o->mass[j]);
                o->ct[i] = damp * sqrt(mij * ks);
            }
        }
    }
}

/* calculateNormalDirectionForce :2560-2611 and
 * calculateTangentialDirectionForce :2614-2696 (component-wise v_n, stray Dt
 * factor on the normal damping, Coulomb cap; forces accumulate on top of the
 * fluid forces and of earlier substeps) */
static void dem_forces(dmph_oracle *o)
{
    const double dx = o->dx, dt = o->p.dt, ddt = o->p.dem_dt;
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double f[3] = {0.0, 0.0, 0.0};
        const int ti = o->prop[i];
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
            if (is_fluid(ti)) continue;
            if (is_fluid(o->prop[j])) continue;
            if (r2 <= dx * dx) {
                const double r = sqrt(r2);
                const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                double u[3] = {0.0, 0.0, 0.0}, vn[3] = {0.0, 0.0, 0.0};
                for (int d = 0; d < 3; d++) u[d] = o->v[3 * j + d] - o->v[3 * i + d];
                for (int d = 0; d < 3; d++) vn[d] += u[d] * e[d];
                for (int d = 0; d < 3; d++)
                    f[d] += -o->kn[i] * (dx - r) * e[d] - (o->cn[i] * vn[d] * e[d] * dt);
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += f[d];
    }
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double f[3] = {0.0, 0.0, 0.0};
        const int ti = o->prop[i];
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3], u[3], vn[3];
            rel(o, o->x + 3 * i, o->x + 3 * j, q);
            const double r2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
            for (int d = 0; d < 3; d++) u[d] = o->v[3 * j + d] - o->v[3 * i + d];
            if (is_fluid(ti)) continue;
            if (is_fluid(o->prop[j])) continue;
            if (r2 <= dx * dx) {
                const double r = sqrt(r2);
                const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
                for (int d = 0; d < 3; d++) vn[d] = u[d] * e[d];
                const double vt[3] = {u[0] - vn[0] * e[0], u[1] - vn[1] * e[1], u[2] - vn[2] * e[2]};
                double dtv[3] = {0.0, 0.0, 0.0}, sN[3], sT[3];
                for (int d = 0; d < 3; d++) dtv[d] += vt[d] * ddt;
                for (int d = 0; d < 3; d++) sN[d] = -o->kn[i] * (dx - r) * e[d] - (o->cn[i] * vn[d] * e[d] * dt);
                const double aFn =
                    o->p.viscous_friction_coefficient[ti] * sqrt(sN[0] * sN[0] + sN[1] * sN[1] + sN[2] * sN[2]);
                for (int d = 0; d < 3; d++) sT[d] = -o->kt[i] * dtv[d] - (o->ct[i] * vt[d]);
                const double aFt = sqrt(sT[0] * sT[0] + sT[1] * sT[1] + sT[2] * sT[2]);
                if (aFn > aFt) {
                    for (int d = 0; d < 3; d++) f[d] += -o->kt[i] * dtv[d] - (o->ct[i] * vt[d]);
                } else {
                    const double avt = sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
                    if (avt != 0)
                        for (int d = 0; d < 3; d++) f[d] += aFn * vt[d] / avt;
                }
            }
        }
        for (int d = 0; d < 3; d++) o->F[3 * i + d] += f[d];
    }
}

/* calculateDEMconvection :1872-1891 */
static void dem_convection(dmph_oracle *o)
{
    const double ddt = o->p.dem_dt;
    for (int i = o->sb; i < o->se; ++i)
        for (int d = 0; d < 3; d++) o->v[3 * i + d] += o->F[3 * i + d] / o->mass[i] * ddt;
    for (int i = o->sb; i < o->se; ++i)
        for (int d = 0; d < 3; d++) o->x[3 * i + d] += o->v[3 * i + d] * ddt;
}

/* calculateWall :2846-2900, with its in-place rotation (r[0] is updated
 * before r[1] and r[2] use it) and its `0.0 < Time < 0.2` test, which C reads
 * as (0.0 < Time) < 0.2 and is therefore true only while Time <= 0. */
static void wall_motion(dmph_oracle *o)
{
    for (int i = o->wb; i < o->we; ++i)
        for (int d = 0; d < 3; d++) o->F[3 * i + d] = 0.0;
    const double t = o->time, dt = o->p.dt;
    for (int i = o->wb; i < o->we; ++i) {
        double *x = o->x + 3 * i, *v = o->v + 3 * i;
        if (t >= 0.2 && 0.4 >= t) {
            const int k = o->prop[i];
            double r[3] = {x[0] - o->wallC[k][0], x[1] - o->wallC[k][1], x[2] - o->wallC[k][2]};
            const double(*R)[3] = o->wallR[k];
            const double *w = o->p.wall_omega[k], *V = o->p.wall_velocity[k];
            r[0] = R[0][0] * r[0] + R[0][1] * r[1] + R[0][2] * r[2];
            r[1] = R[1][0] * r[0] + R[1][1] * r[1] + R[1][2] * r[2];
            r[2] = R[2][0] * r[0] + R[2][1] * r[1] + R[2][2] * r[2];
            v[0] = w[1] * r[2] - w[2] * r[1] + V[0];
            v[1] = w[2] * r[0] - w[0] * r[2] + V[1];
            v[2] = w[0] * r[1] - w[1] * r[0] + V[2];
            x[0] = r[0] + o->wallC[k][0] + V[0] * dt;
            x[1] = r[1] + o->wallC[k][1] + V[1] * dt;
            x[2] = r[2] + o->wallC[k][2] + V[2] * dt;
        } else {
            v[0] = 0.0;
            v[1] = 0.0;
            v[2] = 0.0;
        }
    }
    if (!(0.0 < t))
        for (int k = DMPH_WALL_BEGIN; k < DMPH_WALL_END; ++k)
            for (int d = 0; d < 3; d++) o->wallC[k][d] += o->p.wall_velocity[k][d] * dt;
}

/* neighborCalculation :1264-1286: the largest squared displacement since the
 * last rebuild, and the trigger on it */
static double max_shift2(dmph_oracle *o)
{
    double m = 0.0;
    for (int i = 0; i < o->N; i++) {
        double d3[3];
        for (int d = 0; d < 3; d++)
            d3[d] = pmod(o->x[3 * i + d] - o->xref[3 * i + d] + 0.5 * o->W[d], o->W[d]) - 0.5 * o->W[d];
        const double s = d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2];
        if (s > m) m = s;
    }
    return m;
}
static int need_rebuild(dmph_oracle *o) { return max_shift2(o) > 0.5 * o->margin * 0.5 * o->margin; }

/* ---- rigid debris bodies (no reference counterpart; the library's
 * DMPH_FLAG_RIGID_CLUMPS mode restated in FP64).  Contact force per pair of
 * particles of different bodies (or a body and a wall) within dx: Hertz-type
 * normal spring with the pair's effective modulus, projected normal damping,
 * tangential viscous force capped by Coulomb friction, acting at the contact
 * midpoint; then per body: total force and torque, semi-implicit Euler for the
 * centre of mass and angular momentum, exact quaternion rotation by w dt. */
static void clump_dem(dmph_oracle *o)
{
    const double dx = o->dx, Reff = dx * dx / (dx + dx);
#pragma omp parallel for
    for (int i = o->sb; i < o->se; ++i) {
        const int ti = o->prop[i], bi = o->bid[i];
        const double mi = o->mass[i];
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        FOR_NEIGHBORS(o, i, j)
        {
            const int tj = o->prop[j];
            if (j == i || is_fluid(tj) || (bi >= 0 && o->bid[j] == bi)) continue;
            double q[3];
            for (int d = 0; d < 3; d++) {
                q[d] = o->x[3 * j + d] - o->x[3 * i + d];
                q[d] -= o->W[d] * nearbyint(q[d] / o->W[d]);
            }
            const double r2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
            if (r2 > dx * dx || r2 <= 0.0) continue;
            const double r = sqrt(r2), ov = dx - r;
            const double e[3] = {q[0] / r, q[1] / r, q[2] / r};
            const double u[3] = {o->v[3 * j] - o->v[3 * i], o->v[3 * j + 1] - o->v[3 * i + 1],
                                 o->v[3 * j + 2] - o->v[3 * i + 2]};
            const double un = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];
            const double mj = (o->bid[j] >= 0 ? o->brho[o->bid[j]] : o->p.density[tj]) * o->V;
            const double mij = mi * mj / (mi + mj);
            const double yi = o->p.young_modulus[ti], yj = o->p.young_modulus[tj];
            const double pi_ = o->p.poisson_ratio[ti], pj = o->p.poisson_ratio[tj];
            const double Eeff = (yi * yj) / ((1 - pi_ * pi_) * yj + (1 - pj * pj) * yi);
            const double ktf = 8.0 * yi * yj / (((1 + pi_) * (2 - pi_) * yj) + ((1 + pj) * (2 - pj) * yi));
            const double eij = 0.5 * (o->p.restitution_coefficient[ti] + o->p.restitution_coefficient[tj]);
            const double lij = eij > 0.0 ? log(eij) : 0.0;
            const double damp = eij > 0.0 ? -2.0 * lij / sqrt(M_PI * M_PI + lij * lij) : 0.0;
            const double fric =
                0.5 * (o->p.viscous_friction_coefficient[ti] + o->p.viscous_friction_coefficient[tj]);
            const double kn = (4.0 / 3.0) * Eeff * sqrt(Reff * ov);
            const double cn = sqrt(mij * kn) * damp;
            const double kt = ktf * sqrt(Reff * sqrt(ov));
            const double ct = sqrt(mij * kt) * damp;
            double f[3], ut[3];
            const double fnm = fmin(-kn * ov + cn * un, 0.0);
            for (int d = 0; d < 3; d++) {
                f[d] = fnm * e[d];
                ut[d] = u[d] - un * e[d];
            }
            const double ctot = ct + kt * o->p.dem_dt;
            const double aut = sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
            const double cap = fric * fabs(fnm);
            const double ft = ctot * aut > cap && aut > 0.0 ? cap / aut : ctot;
            for (int d = 0; d < 3; d++) f[d] += ft * ut[d];
            for (int d = 0; d < 3; d++) F[d] += f[d];
            T[0] += 0.5 * (q[1] * f[2] - q[2] * f[1]);
            T[1] += 0.5 * (q[2] * f[0] - q[0] * f[2]);
            T[2] += 0.5 * (q[0] * f[1] - q[1] * f[0]);
        }
        for (int d = 0; d < 3; d++) {
            o->fdem[6 * (size_t)i + d] = F[d];
            o->fdem[6 * (size_t)i + 3 + d] = T[d];
        }
    }
}

static void quat_R(const double *q, double R[3][3])
{
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    R[0][0] = 1.0 - 2.0 * (y * y + z * z);
    R[0][1] = 2.0 * (x * y - w * z);
    R[0][2] = 2.0 * (x * z + w * y);
    R[1][0] = 2.0 * (x * y + w * z);
    R[1][1] = 1.0 - 2.0 * (x * x + z * z);
    R[1][2] = 2.0 * (y * z - w * x);
    R[2][0] = 2.0 * (x * z - w * y);
    R[2][1] = 2.0 * (y * z + w * x);
    R[2][2] = 1.0 - 2.0 * (x * x + y * y);
}

static void body_omega(const double R[3][3], const double *Ii, const double *L, double *w)
{
    double a[3], b[3];
    for (int r = 0; r < 3; r++) a[r] = R[0][r] * L[0] + R[1][r] * L[1] + R[2][r] * L[2];
    for (int r = 0; r < 3; r++) b[r] = Ii[3 * r] * a[0] + Ii[3 * r + 1] * a[1] + Ii[3 * r + 2] * a[2];
    for (int r = 0; r < 3; r++) w[r] = R[r][0] * b[0] + R[r][1] * b[1] + R[r][2] * b[2];
}

static void body_step(dmph_oracle *o)
{
    int *slot = xcalloc((size_t)o->N, sizeof(int));
    for (int i = 0; i < o->N; i++) slot[o->pidx[i]] = i;
    const double dt = o->p.dem_dt;
    for (int b = 0; b < o->B; b++) {
        double *q = o->bq + 4 * b, R[3][3];
        quat_R(q, R);
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        for (int m = o->bptr[b]; m < o->bptr[b + 1]; m++) {
            const int i = slot[o->bmrow[m]];
            const double *r0 = o->br0 + 3 * m;
            double r[3], f[3];
            for (int k = 0; k < 3; k++) r[k] = R[k][0] * r0[0] + R[k][1] * r0[1] + R[k][2] * r0[2];
            for (int k = 0; k < 3; k++) f[k] = o->F[3 * i + k] + o->fdem[6 * (size_t)i + k];
            for (int k = 0; k < 3; k++) F[k] += f[k];
            T[0] += r[1] * f[2] - r[2] * f[1] + o->fdem[6 * (size_t)i + 3];
            T[1] += r[2] * f[0] - r[0] * f[2] + o->fdem[6 * (size_t)i + 4];
            T[2] += r[0] * f[1] - r[1] * f[0] + o->fdem[6 * (size_t)i + 5];
        }
        double *X = o->bX + 3 * b, *V = o->bV + 3 * b, *L = o->bL + 3 * b, w[3];
        for (int k = 0; k < 3; k++) {
            V[k] += F[k] / o->bM[b] * dt;
            X[k] += V[k] * dt;
            L[k] += T[k] * dt;
        }
        const double *Ii = o->bIi + 9 * b;
        body_omega(R, Ii, L, w);
        const double wn = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (wn > 0.0) {
            const double h = 0.5 * wn * dt, c = cos(h), sn = sin(h) / wn;
            const double d[4] = {c, w[0] * sn, w[1] * sn, w[2] * sn};
            const double nq[4] = {d[0] * q[0] - d[1] * q[1] - d[2] * q[2] - d[3] * q[3],
                                  d[0] * q[1] + d[1] * q[0] + d[2] * q[3] - d[3] * q[2],
                                  d[0] * q[2] - d[1] * q[3] + d[2] * q[0] + d[3] * q[1],
                                  d[0] * q[3] + d[1] * q[2] - d[2] * q[1] + d[3] * q[0]};
            const double inv = 1.0 / sqrt(nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3]);
            for (int k = 0; k < 4; k++) q[k] = nq[k] * inv;
        }
        quat_R(q, R);
        body_omega(R, Ii, L, w);
        for (int m = o->bptr[b]; m < o->bptr[b + 1]; m++) {
            const int i = slot[o->bmrow[m]];
            const double *r0 = o->br0 + 3 * m;
            double r[3];
            for (int k = 0; k < 3; k++) r[k] = R[k][0] * r0[0] + R[k][1] * r0[1] + R[k][2] * r0[2];
            for (int k = 0; k < 3; k++) o->x[3 * i + k] = pmod(X[k] + r[k] - o->p.domain_min[k], o->W[k]) + o->p.domain_min[k];
            o->v[3 * i] = V[0] + w[1] * r[2] - w[2] * r[1];
            o->v[3 * i + 1] = V[1] + w[2] * r[0] - w[0] * r[2];
            o->v[3 * i + 2] = V[2] + w[0] * r[1] - w[1] * r[0];
        }
    }
    free(slot);
}

/* one iteration of the main loop, :450-579 */
/* the step before the rebuild decision: drift, walls, wrap, force reset */
static void step_head(dmph_oracle *o)
{
    const int N = o->N;
    for (int i = o->fb; i < o->fe; ++i)
        for (int d = 0; d < 3; d++) o->x[3 * i + d] += o->v[3 * i + d] * o->p.dt; /* calculateConvection :1860 */
    wall_motion(o);
    for (int i = 0; i < N; ++i) /* calculatePeriodicBoundary :3153 */
        for (int d = 0; d < 3; d++)
            o->x[3 * i + d] = pmod(o->x[3 * i + d] - o->p.domain_min[d], o->W[d]) + o->p.domain_min[d];
    memset(o->F, 0, sizeof(double) * 3 * N); /* resetForce :1894 */
    memset(o->fsc, 0, sizeof(double) * N);
}

/* the step after the decision: the rebuild when asked for, then the passes,
 * the fluid update and the DEM substeps */
static void step_tail(dmph_oracle *o, int rebuild)
{
    if (rebuild) {
        cell_sort(o);
        build_neighbors(o);
        o->rebuilds++;
    }
    density_a(o);
    gravity_center(o);
    density_p(o);
    divergence_p(o);
    physical_coefficients(o);
    drag_force(o);
    pressure_p(o);
    pressure_a(o);
    diffuse_interface(o);
    viscosity_v(o);
    drag_force(o);
    buoyancy_force(o);
    gravity_and_acceleration(o);
    for (int s = 0; s < o->demSteps; s++) {
        if (o->B > 0) {
            clump_dem(o);
            body_step(o);
            continue;
        }
        dem_coefficients(o);
        dem_forces(o);
        dem_convection(o);
    }
    o->time += o->p.dt;
    o->steps++;
}

static void step_once(dmph_oracle *o)
{
    step_head(o);
    step_tail(o, need_rebuild(o));
}

int dmph_oracle_step_begin(dmph_oracle *o, double *m2)
{
    if (!o) return DMPH_EINVAL;
    step_head(o);
    if (m2) *m2 = max_shift2(o);
    return 0;
}

int dmph_oracle_step_finish(dmph_oracle *o, int rebuild)
{
    if (!o) return DMPH_EINVAL;
    step_tail(o, rebuild);
    return 0;
}

/* positions and velocities of the given input rows (ParticleIndex), read or
 * written (set != 0) */
int dmph_oracle_rows(dmph_oracle *o, int count, const int *rows, double *x3, double *v3, int set)
{
    if (!o || count < 0 || (count && !rows)) return DMPH_EINVAL;
    int *slot = xcalloc((size_t)o->N, sizeof(int));
    for (int i = 0; i < o->N; i++) slot[o->pidx[i]] = i;
    for (int k = 0; k < count; k++) {
        if (rows[k] < 0 || rows[k] >= o->N) {
            free(slot);
            return DMPH_ERANGE;
        }
        const int i = slot[rows[k]];
        for (int d = 0; d < 3; d++) {
            if (set) {
                if (x3) o->x[3 * (size_t)i + d] = x3[3 * k + d];
                if (v3) o->v[3 * (size_t)i + d] = v3[3 * k + d];
            } else {
                if (x3) x3[3 * k + d] = o->x[3 * (size_t)i + d];
                if (v3) v3[3 * k + d] = o->v[3 * (size_t)i + d];
            }
        }
    }
    free(slot);
    return 0;
}

dmph_oracle *dmph_oracle_create(const dmph_params *p, int n, const int *type, const double *x3, const double *v3)
{
    if (!p || n <= 0 || !type || !x3 || !v3) return NULL;
    if (p->dim != 2 && p->dim != 3) return NULL;
    dmph_oracle *o = xcalloc(1, sizeof(*o));
    o->p = *p;
    o->dim = p->dim;
    o->N = n;
    o->dx = p->particle_spacing;
    o->V = o->dim == 2 ? o->dx * o->dx : o->dx * o->dx * o->dx;
    o->margin = (0.1 * o->dx);
    o->time = p->time;
    o->P2log = 0;
    while ((n >> o->P2log) != 0) ++o->P2log;
    o->P2 = 1 << o->P2log;
    const size_t N = (size_t)n;
    o->pidx = xcalloc(N, sizeof(int));
    o->prop = xcalloc(N, sizeof(int));
    o->x = xcalloc(3 * N, sizeof(double));
    o->v = xcalloc(3 * N, sizeof(double));
    o->F = xcalloc(3 * N, sizeof(double));
    o->xref = xcalloc(3 * N, sizeof(double));
    o->mass = xcalloc(N, sizeof(double));
    o->kappa = xcalloc(N, sizeof(double));
    o->lambda = xcalloc(N, sizeof(double));
    o->mu = xcalloc(N, sizeof(double));
    o->densA = xcalloc(N, sizeof(double));
    o->gc = xcalloc(3 * N, sizeof(double));
    o->pA = xcalloc(N, sizeof(double));
    o->vsp = xcalloc(N, sizeof(double));
    o->div = xcalloc(N, sizeof(double));
    o->P = xcalloc(N, sizeof(double));
    o->kn = xcalloc(N, sizeof(double));
    o->cn = xcalloc(N, sizeof(double));
    o->kt = xcalloc(N, sizeof(double));
    o->ct = xcalloc(N, sizeof(double));
    o->alpha = xcalloc(N, sizeof(double));
    o->dragC = xcalloc(N, sizeof(double));
    o->fsc = xcalloc(N, sizeof(double));
    o->vir = xcalloc(N, sizeof(double));
    o->nc = xcalloc(N, sizeof(int));
    o->fnc = xcalloc(N, sizeof(int));
    o->snc = xcalloc(N, sizeof(int));
    o->nptr = xcalloc(N + 1, sizeof(long));
    o->key = xcalloc((size_t)o->P2, sizeof(int));
    o->payload = xcalloc((size_t)o->P2, sizeof(int));
    for (int i = 0; i < n; i++) {
        o->pidx[i] = i;
        o->prop[i] = type[i];
        for (int d = 0; d < 3; d++) {
            o->x[3 * i + d] = x3[3 * i + d];
            o->v[3 * i + d] = v3[3 * i + d];
        }
    }
    init_weight(o);
    init_fluid(o);
    init_wall(o);
    init_domain(o);
    if (o->T <= 0) {
        dmph_oracle_destroy(o);
        return NULL;
    }
    const size_t T = (size_t)o->T;
    o->cfb = xcalloc(T, sizeof(int));
    o->cfe = xcalloc(T, sizeof(int));
    o->csb = xcalloc(T, sizeof(int));
    o->cse = xcalloc(T, sizeof(int));
    o->cwb = xcalloc(T, sizeof(int));
    o->cwe = xcalloc(T, sizeof(int));
    o->demSteps = p->dt / p->dem_dt;
    cell_sort(o);
    build_neighbors(o);
    density_a(o);
    gravity_center(o);
    density_p(o);
    return o;
}

/* The cell sort of calculateCellParticle (:1288-1338) alone, for checking
 * the library's allocation-free sort: keys and permutation of n particles
 * given as interleaved x3 and type, without the neighbour build. */
int dmph_oracle_cell_sort(const dmph_params *p, int n, const int *type, const double *x3, int *key, int *perm)
{
    if (!p || n <= 0 || !type || !x3 || !key || !perm) return DMPH_EINVAL;
    if (p->dim != 2 && p->dim != 3) return DMPH_EINVAL;
    dmph_oracle *o = xcalloc(1, sizeof(*o));
    o->p = *p;
    o->dim = p->dim;
    o->N = n;
    o->dx = p->particle_spacing;
    o->margin = (0.1 * o->dx);
    while ((n >> o->P2log) != 0) ++o->P2log;
    o->P2 = 1 << o->P2log;
    const size_t N = (size_t)n;
    o->pidx = xcalloc(N, sizeof(int));
    o->prop = xcalloc(N, sizeof(int));
    o->x = xcalloc(3 * N, sizeof(double));
    o->v = xcalloc(3 * N, sizeof(double));
    o->key = xcalloc((size_t)o->P2, sizeof(int));
    o->payload = xcalloc((size_t)o->P2, sizeof(int));
    for (int i = 0; i < n; i++) {
        o->pidx[i] = i;
        o->prop[i] = type[i];
        for (int d = 0; d < 3; d++) o->x[3 * i + d] = x3[3 * i + d];
    }
    init_weight(o);
    init_domain(o);
    if (o->T <= 0) {
        dmph_oracle_destroy(o);
        return DMPH_EINVAL;
    }
    const size_t T = (size_t)o->T;
    o->cfb = xcalloc(T, sizeof(int));
    o->cfe = xcalloc(T, sizeof(int));
    o->csb = xcalloc(T, sizeof(int));
    o->cse = xcalloc(T, sizeof(int));
    o->cwb = xcalloc(T, sizeof(int));
    o->cwe = xcalloc(T, sizeof(int));
    cell_sort(o);
    memcpy(key, o->key, sizeof(int) * N);
    memcpy(perm, o->pidx, sizeof(int) * N);
    dmph_oracle_destroy(o);
    return 0;
}

int dmph_oracle_step(dmph_oracle *o, int nsteps)
{
    if (!o || nsteps < 0) return DMPH_EINVAL;
    for (int s = 0; s < nsteps; s++) step_once(o);
    return 0;
}

typedef struct {
    const char *name;
    size_t off;
    int kind; /* 0 int32 scalar-per-particle, 1 f64 per particle, 2 f64x3, 3 int32[T], 4 int32[P2] */
} field_t;

#define FO(m) offsetof(dmph_oracle, m)
static const field_t FIELDS[] = {
    {"ParticleIndex", FO(pidx), 0},
    {"Property", FO(prop), 0},
    {"Position", FO(x), 2},
    {"Velocity", FO(v), 2},
    {"Force", FO(F), 2},
    {"Mass", FO(mass), 1},
    {"Kappa", FO(kappa), 1},
    {"VolStrainP", FO(vsp), 1},
    {"DivergenceP", FO(div), 1},
    {"PressureP", FO(P), 1},
    {"DensityA", FO(densA), 1},
    {"GravityCenter", FO(gc), 2},
    {"PressureA", FO(pA), 1},
    {"NormalSpringConstant", FO(kn), 1},
    {"NormalViscousDampingConstant", FO(cn), 1},
    {"TangentialSpringConstant", FO(kt), 1},
    {"TangentialViscousDampingConstant", FO(ct), 1},
    {"alpha", FO(alpha), 1},
    {"DragC", FO(dragC), 1},
    {"ForceScale", FO(fsc), 1},
    {"VirialPressure", FO(vir), 1},
    {"NeighborCount", FO(nc), 0},
    {"FluidNeighborCount", FO(fnc), 0},
    {"SolidNeighborCount", FO(snc), 0},
    {"NeighborCalculatedPosition", FO(xref), 2},
    {"CellIndex", FO(key), 4},
    {"CellParticle", FO(payload), 4},
    {"CellFluidParticleBegin", FO(cfb), 3},
    {"CellFluidParticleEnd", FO(cfe), 3},
    {"CellSolidParticleBegin", FO(csb), 3},
    {"CellSolidParticleEnd", FO(cse), 3},
    {"CellWallParticleBegin", FO(cwb), 3},
    {"CellWallParticleEnd", FO(cwe), 3},
};
#undef FO

long dmph_oracle_size(dmph_oracle *o, const char *name)
{
    if (!o || !name) return -1;
    if (!strcmp(name, "NeighborPtr")) return o->N + 1;
    if (!strcmp(name, "NeighborInd")) return o->nindCount;
    for (size_t k = 0; k < sizeof(FIELDS) / sizeof(FIELDS[0]); k++)
        if (!strcmp(FIELDS[k].name, name)) switch (FIELDS[k].kind) {
            case 0:
            case 1: return o->N;
            case 2: return 3L * o->N;
            case 3: return o->T;
            default: return o->P2;
            }
    return -1;
}

/* calculateVirialStressAtParticle :2904-3149 and the virial pressure: four
 * passes over the neighbour lists (pressure P, attractive pressure A,
 * viscosity V, diffuse interface G), each adding its per-particle stress
 * matrix in turn; pressure = -trace / dim (2D: the x and y entries) */
static void virial(dmph_oracle *o)
{
    const double C = o->dim == 2 ? 8.0 : 10.0;
#pragma omp parallel for
    for (int i = 0; i < o->N; i++) {
        double vs[3][3], sP[3][3] = {{0.0}}, sA[3][3] = {{0.0}}, sV[3][3] = {{0.0}}, sG[3][3] = {{0.0}};
        const int ti = o->prop[i];
        const double *xi = o->x + 3 * i, *vi = o->v + 3 * i;
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, xi, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (o->RP * o->RP - r2 > 0) {
                const double r = sqrt(r2);
                const double dw = k_dw(r, o->Bp, o->RP);
                const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                double f[3];
                for (int d = 0; d < 3; d++) f[d] = (o->P[i]) * g[d] * o->V;
                for (int d = 0; d < 3; d++)
                    for (int e = 0; e < 3; e++) sP[d][e] += 1.0 * f[d] * q[e] / o->V;
            }
        }
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, xi, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (o->RA * o->RA - r2 > 0) {
                const double ratio = o->p.interaction_ratio[ti][o->prop[j]];
                const double r = sqrt(r2);
                const double dw = ratio * k_dwa(r, o->Ba, o->RA);
                const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                double f[3];
                for (int d = 0; d < 3; d++) f[d] = (o->pA[i]) * g[d] * o->V;
                for (int d = 0; d < 3; d++)
                    for (int e = 0; e < 3; e++) sA[d][e] += 1.0 * f[d] * q[e] / o->V;
            }
        }
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, xi, o->x + 3 * j, q);
            const double r2 = sq3(q);
            if (o->RV * o->RV - r2 > 0) {
                const double r = sqrt(r2);
                const double dw = -k_dw(r, o->Bv, o->RV);
                const double e_[3] = {q[0] / r, q[1] / r, q[2] / r};
                const double *vj = o->v + 3 * j;
                const double u[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
                const double muij = 2.0 * (o->mu[i] * o->mu[j]) / (o->mu[i] + o->mu[j]);
                double f[3];
                for (int d = 0; d < 3; d++)
                    f[d] = C * muij * (u[0] * e_[0] + u[1] * e_[1] + u[2] * e_[2]) * e_[d] * dw / r * o->V;
                for (int d = 0; d < 3; d++)
                    for (int e = 0; e < 3; e++) sV[d][e] += 0.5 * f[d] * q[e] / o->V;
            }
        }
        FOR_NEIGHBORS(o, i, j)
        {
            if (i == j) continue;
            double q[3];
            rel(o, xi, o->x + 3 * j, q);
            const double r2 = sq3(q);
            const double *gc = o->gc + 3 * i;
            if (o->RG * o->RG - r2 > 0) {
                const double a = o->CofA[ti] * (o->CofK) * (o->CofK);
                const double ratio = o->p.interaction_ratio[ti][o->prop[j]];
                const double r = sqrt(r2);
                const double w = ratio * k_w(r, o->Bg, o->RG);
                double f[3];
                for (int d = 0; d < 3; d++) f[d] = -a * (-gc[d]) * w / o->R2g * o->RG * (o->V / o->dx);
                for (int d = 0; d < 3; d++)
                    for (int e = 0; e < 3; e++) sG[d][e] += 1.0 * f[d] * q[e] / o->V;
            }
            if (o->RG * o->RG - r2 > 0.0) {
                const double a = o->CofA[ti] * (o->CofK) * (o->CofK);
                const double ratio = o->p.interaction_ratio[ti][o->prop[j]];
                const double r = sqrt(r2);
                const double dw = ratio * k_dw(r, o->Bg, o->RG);
                const double g[3] = {dw * q[0] / r, dw * q[1] / r, dw * q[2] / r};
                double gr = 0.0;
                for (int d = 0; d < 3; d++) gr += (-gc[d]) * q[d];
                double f[3];
                for (int d = 0; d < 3; d++) f[d] = -a * (gr)*g[d] / o->R2g * o->RG * (o->V / o->dx);
                for (int d = 0; d < 3; d++)
                    for (int e = 0; e < 3; e++) sG[d][e] += 1.0 * f[d] * q[e] / o->V;
            }
        }
        for (int d = 0; d < 3; d++)
            for (int e = 0; e < 3; e++) vs[d][e] = (((0.0 + sP[d][e]) + sA[d][e]) + sV[d][e]) + sG[d][e];
        o->vir[i] = o->dim == 2 ? -1.0 / 2.0 * (vs[0][0] + vs[1][1]) : -1.0 / 3.0 * (vs[0][0] + vs[1][1] + vs[2][2]);
    }
}

int dmph_oracle_get(dmph_oracle *o, const char *name, void *out)
{
    if (!o || !name || !out) return DMPH_EINVAL;
    if (!strcmp(name, "NeighborPtr")) {
        memcpy(out, o->nptr, sizeof(long) * (o->N + 1));
        return 0;
    }
    if (!strcmp(name, "NeighborInd")) {
        memcpy(out, o->nind, sizeof(int) * o->nindCount);
        return 0;
    }
    if (!strcmp(name, "VirialPressure")) virial(o);
    for (size_t k = 0; k < sizeof(FIELDS) / sizeof(FIELDS[0]); k++)
        if (!strcmp(FIELDS[k].name, name)) {
            const void *src = *(void *const *)((const char *)o + FIELDS[k].off);
            const int kind = FIELDS[k].kind;
            const size_t es = (kind == 1 || kind == 2) ? sizeof(double) : sizeof(int);
            memcpy(out, src, es * (size_t)dmph_oracle_size(o, name));
            return 0;
        }
    return DMPH_EINVAL;
}

double dmph_oracle_scalar(dmph_oracle *o, const char *name)
{
    if (!o || !name) return NAN;
#define S(n, v) \
    if (!strcmp(name, n)) return (double)(v)
    S("Time", o->time);
    S("ParticleCount", o->N);
    S("PowerParticleCount", o->P2);
    S("TotalCellCount", o->T);
    S("CellCount0", o->cc[0]);
    S("CellCount1", o->cc[1]);
    S("CellCount2", o->cc[2]);
    S("CellWidth0", o->cw[0]);
    S("CellWidth1", o->cw[1]);
    S("CellWidth2", o->cw[2]);
    S("N0a", o->N0a);
    S("N0p", o->N0p);
    S("R2g", o->R2g);
    S("Swa", o->Swa);
    S("Swg", o->Swg);
    S("Swp", o->Swp);
    S("Swv", o->Swv);
    S("MaxRadius", o->maxR);
    S("FluidBegin", o->fb);
    S("FluidEnd", o->fe);
    S("SolidBegin", o->sb);
    S("SolidEnd", o->se);
    S("WallBegin", o->wb);
    S("WallEnd", o->we);
    S("NeighborIndCount", o->nindCount);
    S("DemSteps", o->demSteps);
    S("Rebuilds", o->rebuilds);
    S("Steps", o->steps);
    S("CofK", o->CofK);
#undef S
    return NAN;
}

static int inv3(const double *a, double *out)
{
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (!(fabs(det) > 0.0)) return -1;
    const double id = 1.0 / det;
    out[0] = c00 * id;
    out[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    out[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    out[3] = c01 * id;
    out[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    out[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    out[6] = c02 * id;
    out[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    out[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return 0;
}

int dmph_oracle_pressure_force(dmph_oracle *o, const double *P, double *F)
{
    if (!o || !P || !F) return -1;
    memset(F, 0, sizeof(double) * 3 * (size_t)o->N);
    pressure_force(o, P, F, NULL);
    return 0;
}

int dmph_oracle_set_bodies(dmph_oracle *o, int nb, const int *body_of_row, const double *rho)
{
    if (!o || nb <= 0 || !body_of_row || !rho || o->B > 0 || o->steps > 0) return DMPH_EINVAL;
    const int N = o->N;
    int *slot = xcalloc((size_t)N, sizeof(int));
    for (int i = 0; i < N; i++) slot[o->pidx[i]] = i;
    int *cnt = xcalloc((size_t)nb + 1, sizeof(int));
    for (int r = 0; r < N; r++) {
        const int b = body_of_row[r], t = o->prop[slot[r]];
        if (b < -1 || b >= nb || (b >= 0) != is_solid(t)) {
            free(slot);
            free(cnt);
            return DMPH_EINVAL;
        }
        if (b >= 0) cnt[b + 1]++;
    }
    o->B = nb;
    o->bptr = xcalloc((size_t)nb + 1, sizeof(int));
    for (int b = 0; b < nb; b++) o->bptr[b + 1] = o->bptr[b] + cnt[b + 1];
    const int nm = o->bptr[nb];
    o->bmrow = xcalloc((size_t)nm, sizeof(int));
    o->br0 = xcalloc(3 * (size_t)nm, sizeof(double));
    o->bX = xcalloc(3 * (size_t)nb, sizeof(double));
    o->bV = xcalloc(3 * (size_t)nb, sizeof(double));
    o->bL = xcalloc(3 * (size_t)nb, sizeof(double));
    o->bq = xcalloc(4 * (size_t)nb, sizeof(double));
    o->bM = xcalloc((size_t)nb, sizeof(double));
    o->bIi = xcalloc(9 * (size_t)nb, sizeof(double));
    o->brho = xcalloc((size_t)nb, sizeof(double));
    o->bid = xcalloc((size_t)N, sizeof(int));
    o->fdem = xcalloc(6 * (size_t)N, sizeof(double));
    for (int i = 0; i < N; i++) o->bid[i] = body_of_row[o->pidx[i]];
    int *fill = xcalloc((size_t)nb, sizeof(int));
    for (int r = 0; r < N; r++)
        if (body_of_row[r] >= 0) {
            const int b = body_of_row[r];
            o->bmrow[o->bptr[b] + fill[b]++] = r;
        }
    for (int b = 0; b < nb; b++) {
        o->brho[b] = rho[b];
        const double m = rho[b] * o->V;
        const int m0 = o->bptr[b], m1 = o->bptr[b + 1], n = m1 - m0;
        const double *x0 = o->x + 3 * (size_t)slot[o->bmrow[m0]];
        double c[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
        double *xu = xcalloc(3 * (size_t)n, sizeof(double));
        for (int k = 0; k < n; k++) {
            const int i = slot[o->bmrow[m0 + k]];
            for (int d = 0; d < 3; d++) {
                double dd = o->x[3 * (size_t)i + d] - x0[d];
                dd -= o->W[d] * nearbyint(dd / o->W[d]);
                xu[3 * k + d] = x0[d] + dd;
                c[d] += xu[3 * k + d];
                vc[d] += o->v[3 * (size_t)i + d];
            }
        }
        for (int d = 0; d < 3; d++) {
            c[d] /= (double)n;
            vc[d] /= (double)n;
        }
        const double a = 0.4 * m * (0.5 * o->dx) * (0.5 * o->dx);
        double I[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, L[3] = {0, 0, 0};
        for (int k = 0; k < n; k++) {
            const int i = slot[o->bmrow[m0 + k]];
            const double r[3] = {xu[3 * k] - c[0], xu[3 * k + 1] - c[1], xu[3 * k + 2] - c[2]};
            const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) I[3 * p + q] += m * ((p == q ? rr : 0.0) - r[p] * r[q]);
            for (int p = 0; p < 3; p++) I[4 * p] += a;
            const double u[3] = {o->v[3 * (size_t)i] - vc[0], o->v[3 * (size_t)i + 1] - vc[1],
                                 o->v[3 * (size_t)i + 2] - vc[2]};
            L[0] += m * (r[1] * u[2] - r[2] * u[1]);
            L[1] += m * (r[2] * u[0] - r[0] * u[2]);
            L[2] += m * (r[0] * u[1] - r[1] * u[0]);
            for (int d = 0; d < 3; d++) o->br0[3 * (m0 + k) + d] = r[d];
        }
        free(xu);
        if (inv3(I, o->bIi + 9 * b)) {
            free(slot);
            free(cnt);
            free(fill);
            return DMPH_EINVAL;
        }
        for (int d = 0; d < 3; d++) {
            o->bX[3 * b + d] = c[d];
            o->bV[3 * b + d] = vc[d];
            o->bL[3 * b + d] = L[d];
        }
        o->bq[4 * b] = 1.0;
        o->bM[b] = m * (double)n;
    }
    free(slot);
    free(cnt);
    free(fill);
    return 0;
}

int dmph_oracle_get_bodies(dmph_oracle *o, double *X, double *V, double *q, double *L, double *M)
{
    if (!o) return DMPH_EINVAL;
    const size_t B = (size_t)o->B;
    if (X) memcpy(X, o->bX, 3 * B * sizeof(double));
    if (V) memcpy(V, o->bV, 3 * B * sizeof(double));
    if (q) memcpy(q, o->bq, 4 * B * sizeof(double));
    if (L) memcpy(L, o->bL, 3 * B * sizeof(double));
    if (M) memcpy(M, o->bM, B * sizeof(double));
    return 0;
}

void dmph_oracle_destroy(dmph_oracle *o)
{
    if (!o) return;
    free(o->bid);
    free(o->brho);
    free(o->bptr);
    free(o->bmrow);
    free(o->br0);
    free(o->bX);
    free(o->bV);
    free(o->bL);
    free(o->bq);
    free(o->bM);
    free(o->bIi);
    free(o->fdem);
    void **ptrs[] = {(void **)&o->pidx,  (void **)&o->prop,  (void **)&o->x,      (void **)&o->v,
                     (void **)&o->F,     (void **)&o->xref,  (void **)&o->mass,   (void **)&o->kappa,
                     (void **)&o->lambda, (void **)&o->mu,   (void **)&o->densA,  (void **)&o->gc,
                     (void **)&o->pA,    (void **)&o->vsp,   (void **)&o->div,    (void **)&o->P,
                     (void **)&o->kn,    (void **)&o->cn,    (void **)&o->kt,     (void **)&o->ct,
                     (void **)&o->alpha, (void **)&o->dragC, (void **)&o->fsc, (void **)&o->vir,    (void **)&o->nc,
                     (void **)&o->fnc,
                     (void **)&o->snc,   (void **)&o->nptr,  (void **)&o->nind,   (void **)&o->key,
                     (void **)&o->payload, (void **)&o->cfb, (void **)&o->cfe,    (void **)&o->csb,
                     (void **)&o->cse,   (void **)&o->cwb,   (void **)&o->cwe};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); k++) free(*ptrs[k]);
    free(o);
}
