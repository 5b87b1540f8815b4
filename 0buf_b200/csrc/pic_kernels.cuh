// Host-side launchers of the B200 PIC kernels (one translation unit per form).
#pragma once
#include <cuda_runtime.h>
#include "pic_internal.cuh"

namespace pic {

// plain form (pic_plain.cu, FP64, -fmad=false)
void yee_b_half_plain(const Grid &g, double *const F[12], cudaStream_t s);
void yee_b_complete_plain(const Grid &g, double *const F[12], cudaStream_t s);
void yee_e_update_plain(const Grid &g, double *const F[12], cudaStream_t s);
void j_fold(const Grid &g, double *Jx, double *Jy, double *Jz, cudaStream_t s);
void e_ghosts_plain(const Grid &g, double *Ex, double *Ey, double *Ez, int periodic, cudaStream_t s);
void e_ghosts_mixed(const Grid &g, float *Ex, float *Ey, float *Ez, int periodic, cudaStream_t s);
size_t push_smem_plain(const Grid &g);
// lo32: the tile current's int32 remainder word (every tile holds fewer than
// 2^(31 - kFxLo32MinBits) particles), else the 64-bit one
cudaError_t launch_push_plain(const StepParams &p, bool lo32, cudaStream_t s);
// placement of loaded particles (reference getPointCell + Cell::Insert)
cudaError_t place_particles_plain(const Grid &g, int64_t n, const double *x, const double *y, const double *z,
                                  int *cell_out, cudaStream_t s);

// mixed form (pic_mixed.cu, FP32 with FP64 global J)
void yee_b_half_mixed(const Grid &g, float *const E[3], float *const H[3], cudaStream_t s);
// both B half steps of a step in one pass, H = (H + Q(E)) + Q(E) (pic_step: the push forms the first in shared memory)
void yee_b_both_mixed(const Grid &g, float *const E[3], float *const H[3], cudaStream_t s);
void yee_e_update_mixed(const Grid &g, float *const E[3], float *const H[3], double *const J[3], cudaStream_t s);
size_t push_smem_mixed(const Grid &g);
// dynamic + static shared memory of the mixed push kernel ((size_t)-1 if it cannot be queried)
size_t push_smem_total_mixed(const Grid &g);
cudaError_t launch_push_mixed(const StepParams &p, const MixedMaps &maps, cudaStream_t s);
// largest contribution bound of a species' particles from their momenta (float bits, atomicMax into *out)
cudaError_t contribution_bound_mixed(const Grid &g, const SpeciesView &S, int64_t cap, unsigned *out, cudaStream_t s);
// TMA descriptors of the FP32 E/H arrays for the push's field tile
cudaError_t encode_field_maps(const Grid &g, float *const E[3], float *const H[3], MixedMaps *maps);

// form-independent (pic_common.cu, FP64 parts with -fmad=false)
cudaError_t launch_insert(const StepParams &p, cudaStream_t s);
cudaError_t cell_histogram(const StepParams &p, int *counts, cudaStream_t s);
// native 28-byte layout (reference cell number, FP32 offsets and momenta)
cudaError_t place_particles_cells(const Grid &g, int64_t n, const int *ref_cell, const float *ox, const float *oy,
                                  const float *oz, int *cell_out, cudaStream_t s);
cudaError_t scatter_to_bins_f(const Grid &g, int mixed, int64_t n, const int *cell, const float *ox, const float *oy,
                              const float *oz, const float *px, const float *py, const float *pz, SpeciesView sv,
                              int *fill, cudaStream_t s);
cudaError_t gather_from_bins_f(const Grid &g, int mixed, SpeciesView sv, const int64_t *dense_start, int *cell,
                               float *ox, float *oy, float *oz, float *px, float *py, float *pz, cudaStream_t s);
// flat device list -> per-tile counts of valid particles (cell >= 0)
cudaError_t tile_histogram(const Grid &g, int64_t n, const int *cell, int *tile_counts, cudaStream_t s);
// flat FP64 list -> bins of one species (plain or mixed), fill[] = running counts
cudaError_t scatter_to_bins(const Grid &g, int mixed, int64_t n, const int *cell, const double *x, const double *y,
                            const double *z, const double *px, const double *py, const double *pz,
                            SpeciesView sv, int *fill, cudaStream_t s);
// bins of one species -> flat list in slot order (global FP64 positions)
cudaError_t gather_from_bins(const Grid &g, int mixed, SpeciesView sv, const int64_t *dense_start, double *x,
                             double *y, double *z, double *px, double *py, double *pz, int *cell, cudaStream_t s);
// the particles of one packed cell of tile `tile` (at most cap), count in *count
cudaError_t cell_particles(const Grid &g, int mixed, const SpeciesView &sv, int tile, int cell, int64_t cap, double *x,
                           double *y, double *z, double *px, double *py, double *pz, int64_t *slot, unsigned *count,
                           cudaStream_t s);
// outbox leftovers of one species (after a failed insert) -> flat list appended at offset
cudaError_t gather_outbox(const StepParams &p, int species, unsigned n_out, unsigned *counter, int64_t offset,
                          double *x, double *y, double *z, double *px, double *py, double *pz, int *cell,
                          cudaStream_t s);
// seeded generator straight into bins laid out cell-major within each tile
cudaError_t init_species_bins(const Grid &g, int mixed, SpeciesView sv, int species_index, int ppc, double dx,
                              double dy, double dz, double vth, uint64_t seed, cudaStream_t s);
// seeded generator with per-cell counts (count, first slot per dense cell)
cudaError_t init_cells(const Grid &g, int mixed, SpeciesView sv, int species_index, const int *count,
                       const int *first, double dx, double dy, double dz, double vth, uint64_t seed, cudaStream_t s);
// FP64 reductions: out[0] sum E^2, out[1] sum H^2 over nodes 1..N, out[2] sum E^2 all nodes (reference)
cudaError_t field_energy(const Grid &g, int mixed, const void *const E[3], const void *const H[3], double *out3,
                         cudaStream_t s);
cudaError_t kinetic_energy(const StepParams &p, double *out, cudaStream_t s);
// charge-conservation diagnostic (pic_diag.cu, FP64): rho on the cell-centre
// nodes, folded; G = div E - rho on interior nodes with reductions
// red[0] max |G - G0|, red[1] max |rho|, red[2] sum (G - G0)^2, red[3] max |G0|
cudaError_t charge_density(const StepParams &p, double *rho, cudaStream_t s);
// total mechanical momentum sum (m/q_m) p per species into out[3 s + a] (FP64)
cudaError_t momentum(const StepParams &p, double *out, cudaStream_t s);
cudaError_t gauss_residual(const Grid &g, int mixed, const void *const E[3], const double *rho, double *G, double *G0,
                           int set_baseline, double *red, cudaStream_t s);
// pitched device <-> dense reference-layout buffer (FP64 on the dense side)
cudaError_t pitched_to_dense(const Grid &g, const void *src, int is_float, double *dst, cudaStream_t s);
cudaError_t dense_to_pitched(const Grid &g, const double *src, void *dst, int is_float, cudaStream_t s);

}  // namespace pic
