/*
 * dmph_oracle.h — CPU restatement of the reference DEM-MPH explicit step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU library is compared
 * against; it is never linked into libdmph.so, the `dem_mph` executable or
 * anything the timestep path calls.  Only tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py load it.
 *
 * It restates, in plain C with OpenMP, the FP64 algorithm of
 * source/DEM-MPH.cpp (Ryo1011gd/DEM_MPH), including its quirks (see the
 * comments at each function).  It is pinned against the reference itself:
 * oracle/Makefile builds the reference's own source into oracle/_ref/, and
 * tests/test_oracle_pin.py and the committed golden fixtures under
 * tests/golden/ check that this restatement reproduces it bit for bit.
 */
#ifndef DMPH_ORACLE_H
#define DMPH_ORACLE_H

#include "../include/dmph.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dmph_oracle dmph_oracle;

dmph_oracle *dmph_oracle_create(const dmph_params *p, int n, const int *type, const double *x3, const double *v3);
int dmph_oracle_step(dmph_oracle *o, int nsteps);
/* number of elements of a named array (see dmph_oracle_get) or -1 */
long dmph_oracle_size(dmph_oracle *o, const char *name);
/* copy a named array (names as in the reference: "Position", "Force", ...) */
int dmph_oracle_get(dmph_oracle *o, const char *name, void *out);
/* scalar by name ("Time", "N0a", "Rebuilds", ...) */
double dmph_oracle_scalar(dmph_oracle *o, const char *name);
/* rigid debris bodies (the library's DMPH_FLAG_RIGID_CLUMPS mode; no
 * reference counterpart): same model as dmph_set_bodies, restated in FP64 */
/* Pressure-gradient force (calculatePressureP :2213-2246) of a given pressure
 * field on the current positions and neighbour lists, written to F[3N]. */
int dmph_oracle_pressure_force(dmph_oracle *o, const double *P, double *F);
int dmph_oracle_set_bodies(dmph_oracle *o, int nbodies, const int *body_of_row, const double *body_density);
/* X,V,L 3 per body, q 4 per body, M 1 per body (any may be NULL) */
int dmph_oracle_get_bodies(dmph_oracle *o, double *X, double *V, double *q, double *L, double *M);
/* one step split at the rebuild decision: begin runs the drift, walls, wrap
 * and force reset and reports the largest squared displacement since the last
 * rebuild; finish runs the rebuild when asked for, then the rest of the step */
int dmph_oracle_step_begin(dmph_oracle *o, double *max_shift2);
int dmph_oracle_step_finish(dmph_oracle *o, int rebuild);
/* positions / velocities (either may be NULL) of input rows: set = 0 reads
 * them into x3, v3 (3 per row), set = 1 writes them */
int dmph_oracle_rows(dmph_oracle *o, int count, const int *rows, double *x3, double *v3, int set);
/* the cell sort alone (keys and permutation, n of each), no neighbour build */
int dmph_oracle_cell_sort(const dmph_params *p, int n, const int *type, const double *x3, int *key, int *perm);
void dmph_oracle_destroy(dmph_oracle *o);

#ifdef __cplusplus
}
#endif
#endif
