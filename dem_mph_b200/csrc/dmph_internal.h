// Internal declarations shared by the translation units of libdmph.so.
#pragma once

#include <string>

#include "dmph_state.cuh"

namespace dmph {

int derive_params(const dmph_params &p, int n, DevParams &P, WallMotion &Wm, std::string &err);
// same checks; on failure *msg points at a string literal (allocates nothing)
int derive_params(const dmph_params &p, int n, DevParams &P, WallMotion &Wm, const char **msg);
// dmph_api.cu: message that dmph_last_error(NULL) returns on the calling
// thread until the next failing call without a context (a string literal)
void set_noctx_message(const char *literal);
// the same for calls that may allocate (dmph_checkpoint_open)
void set_noctx_error(const std::string &msg);

// dmph_rebuild.cu
void launch_keys(const DevParams &P, const double *pos, const int *type, unsigned long long *words, cudaStream_t st);
void launch_bitonic(unsigned long long *words, int n, int nlog, cudaStream_t st);
int bitonic_launch_count(int n, int nlog);  // kernels launch_bitonic issues
void launch_cell_start(const DevParams &P, const unsigned long long *words, int *start, cudaStream_t st);
// FP32 build: stable counting sort of the cell keys into words[0, N) and
// cell_start (6 kernels); slots from n_move on (walls that keep their slots)
// are left as they are; nonzero when 3T + 1 keys exceed the scan's range
int launch_counting_sort(const DevParams &P, int n_move, const double *pos, const int *type, int *keys, int *counts,
                         unsigned long long *tmp, unsigned long long *words, int *cell_start, int *block_sums,
                         int *total, cudaStream_t st);
constexpr long long kCountingSortMaxKeys = 4096LL * 4096LL;
void launch_permute(const DevParams &P, const unsigned long long *words, const double *pos_in, const double *vel_in,
                    const int *type_in, const int *pidx_in, double *pos_out, double *vel_out, int *type_out,
                    int *pidx_out, double *xref, const int *bid_in, int *bid_out, cudaStream_t st);
template <class T>
int launch_exclusive_scan(const T *in, T *out, int n, T *block_sums, T *total, cudaStream_t st);
void launch_chunks(const DevParams &P, const unsigned long long *words, const int *start, int *flag, int *offs,
                   int *block_sums, int *total, Chunk *chunks, cudaStream_t st);
void launch_widen(const int *in, long long *out, int n, cudaStream_t st);
void launch_bounds(const DevParams &P, const int *start, const int *offs, const int *total, int *dB, cudaStream_t st);
void launch_wet_partition(const DevParams &P, const unsigned long long *words, const int *start, Chunk *chunks,
                          Chunk *tmp, int *dB, int *flag, int *offs, int *block_sums, int *total, cudaStream_t st);
// maxshiftL: largest displacement since the lists were built (list reuse),
// null without list reuse
void launch_decide(const DevParams &P, const unsigned long long *maxshift, int *dB, unsigned long long graph_cond,
                   cudaStream_t st, const unsigned long long *maxshiftL = nullptr);

// dmph_f64.cu
void launch_drift(const DevParams &P, const DevState &S, const WallMotion &Wm, unsigned long long *maxshift, int sms,
                  cudaStream_t st);
void launch_pass_a(const DevParams &P, const DevState &S, const int *dB, int range, int init_only, cudaStream_t st,
                   int list = 0, int gate = 0);
void launch_build_list64(const DevParams &P, const DevState &S, int *dB, cudaStream_t st);
void launch_virial(const DevParams &P, const DevState &S, const int *dB, double *vir, cudaStream_t st);
void launch_pass_b(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st, int list = 0, int gate = 0);
void launch_fluid_accel(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st);
// list (FP64 build): walk the Verlet lists, with the stencil walk gated on a
// list overflow (2 kernels)
void launch_dem_force(const DevParams &P, const DevState &S, const int *dB, int range, int forces, cudaStream_t st,
                      bool mixed = false, bool list = false);
void launch_dem_integrate(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st);
void launch_counts(const DevParams &P, const DevState &S, const int *dB, int range, cudaStream_t st);
// FP32 list mode, debris counts from the lists (with the stencil walk gated
// on a list overflow): 2 kernels
void launch_counts_list(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st);
// list reuse: the same debris counts on a trigger that keeps the lists
// (B_NEED = 2; 1 kernel, a no-op on other steps)
void launch_counts_list_kept(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st);
void launch_neighbor_fill(const DevParams &P, const DevState &S, const int *dB, const long long *ptr, int *ind,
                          cudaStream_t st);

// dmph_f32.cu
DevParams32 make_params32(const DevParams &P);
// maxshiftL (list reuse, else null): also the largest displacement since the
// lists were built (from S.xrefL4)
void launch_drift32(const DevParams &P, const DevParams32 &Q, const DevState &S, const WallMotion &Wm,
                    unsigned long long *maxshift, int sms, cudaStream_t st, unsigned long long *maxshiftL = nullptr);
// list reuse, a trigger that keeps the lists (B_NEED = 2; a no-op on other
// steps): the trigger positions of the first n slots (FP32 and FP64) become
// the current ones
void launch_kept_trigger32(const DevParams &P, const DevState &S, const int *dB, int n, cudaStream_t st);
void launch_pass_a32(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int range, int variant,
                     cudaStream_t st, int gate = 0);
void launch_pass_b32(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int variant,
                     cudaStream_t st, int gate = 0);
// skin_from_dB (list reuse): the list radius is MaxRadius + dB[B_SKIN_NEXT]
// hundredths of dx (recorded in dB[B_SKIN]) instead of MaxRadius + MARGIN
void launch_build_list32(const DevParams &P, const DevParams32 &Q, const DevState &S, int *dB, int split,
                         cudaStream_t st, int variant = 0, int skin_from_dB = 0);
constexpr int kBuildVariants = 3;  // launch variants of the FP32 list build
void launch_list_wall_guard(int *dB, cudaStream_t st);
void launch_pass_a32_list(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int variant,
                          cudaStream_t st);
void launch_pass_b32_list(const DevParams &P, const DevParams32 &Q, const DevState &S, const int *dB, int variant,
                          cudaStream_t st);
void launch_ens_pass_a32(const EnsScene *tab, int ns, int variant, cudaStream_t st, int gate = 0);
void launch_ens_pass_b32(const EnsScene *tab, int ns, int variant, cudaStream_t st, int gate = 0);
void launch_ens_pass_list(const EnsScene *tab, int ns, bool pass_b, cudaStream_t st);
void launch_ens_fluid_accel32(const EnsScene *tab, int ns, cudaStream_t st);
void launch_fluid_accel32(const DevParams32 &Q, const DevState &S, const int *dB, cudaStream_t st);
void launch_export32(const DevParams &P, const DevState &S, double *pos, double *vel, cudaStream_t st);
void launch_import32(const DevParams &P, const DevState &S, const double *pos, const double *vel, cudaStream_t st);
void launch_permute32(const DevParams &P, int n, const unsigned long long *words, const double *xabs,
                      const float4 *v_in, const int *type_in, const int *pidx_in, float4 *p_out, float4 *v_out,
                      int *type_out, int *pidx_out, double *xref, float4 *xref4, const int *bid_in, int *bid_out,
                      const double *vabs, double *pos_out, double *vel_out, cudaStream_t st,
                      float4 *xrefL4 = nullptr);
void launch_solid_force_to64(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st);
void launch_sync_solids32(const DevParams &P, const DevState &S, const int *dB, cudaStream_t st);
double lattice_n0p32(const DevParams &P, const DevParams32 &Q, cudaStream_t st);
void launch_widen_f(const float *in, double *out, int n, cudaStream_t st);
void launch_widen_f4(const float4 *in, double *out, int count, int stride, cudaStream_t st);

// dmph_bodies.cu
void launch_slot_of_row(const DevParams &P, const int *pidx, int *slot_of_row, cudaStream_t st);
void launch_clump_dem(const DevParams &P, const DevState &S, const int *dB, bool lists, cudaStream_t st);
void launch_body_step(const DevParams &P, const DevState &S, const DevBodies &Bd, bool f32, cudaStream_t st);
// ensemble-wide launches (one per step part over every scene of the table)
void launch_ens_clump_dem(const EnsScene *tab, int ns, int sub, cudaStream_t st);  // 2 kernels
void launch_ens_body_step(const EnsScene *tab, int ns, const int *bpre, int total_bodies, int sub, cudaStream_t st);
void launch_ens_drift32(const EnsScene *tab, int ns, int sms, cudaStream_t st);
void launch_ens_decide(const EnsScene *tab, int ns, const unsigned long long *handles, cudaStream_t st);
void launch_ens_solid_force_to64(const EnsScene *tab, int ns, cudaStream_t st);
void launch_ens_sync_solids32(const EnsScene *tab, int ns, cudaStream_t st);

void launch_xyz_to_planes(const double *xyz, double *planes, int n, cudaStream_t st);
void launch_planes_to_xyz(const double *planes, double *xyz, int n, cudaStream_t st);

}  // namespace dmph
