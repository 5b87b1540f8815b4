// State of the differentiable run (pic_forward / pic_backward), shared by the
// plain-form (pic_adjoint.cu) and FP32-form (pic_adjoint_mixed.cu) units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>
#include "pic0buf.h"
#include "pic_internal.cuh"

struct pic_handle;

namespace pic {

struct AdjStatus {
    unsigned flags;                // ST_STENCIL / ST_NAN seen in the run
    unsigned pad;
    unsigned long long ambiguous;  // cell changes with zero or several receiving cells (resolved, counted)
};

// Buffers live until pic_adjoint_free / the next pic_forward / pic_destroy.
// A "particle state" is the whole population in the fixed order of the run:
// per species the packed cells then 6 value arrays (plain: FP64 global
// positions and momenta; mixed: FP32 in-cell offsets and momenta).
struct AdjState {
    int mixed;
    size_t elem;       // bytes per particle value (8 plain, 4 mixed)
    int nsp;
    int64_t n[kMaxSpecies];
    int steps, K, nseg;
    size_t pbytes;     // one particle state
    char *cur;         // the forward's running state
    char *ckp;         // nseg particle checkpoints
    char *ckf;         // nseg x (E, H): 6 field arrays each, in the form's field type
    char *segp;        // K+1 particle states of the segment being reversed
    char *segf;        // K+1 x (E, H) of that segment
    char *lamp;        // per species lambda_x (3) and lambda_p (3), form's element type
    size_t lamp_bytes;
    double *lamf;      // FP64 lambda_E, lambda_H, lambda_J, lambda_Q (12 arrays)
    void *lamF;        // per particle lambda of the 6 interpolated field values (form's element type)
    void *segF;        // optional: K x the 6 interpolated field values per particle of the segment
    char *rf;          // field set of the recompute (form's layout: 12 arrays)
    char *ha;          // B after the half step of the step being reversed (3 arrays)
    double *hist;      // steps x 3: sum over nodes 1..N of E_c^2 after each step
    double *red;       // reduction scratch
    AdjStatus *st;
    std::vector<double> hhist;  // host copy of hist x cell volume
    cudaEvent_t e0, e1;
    float t_fwd, t_bwd;
    unsigned long long ambiguous;
    int have_forward;
};

inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }
size_t adj_state_bytes(const AdjState &A);
void adj_state_view(const AdjState &A, char *base, int *cell[kMaxSpecies], void *v[kMaxSpecies][6]);

// ---- FP32 form (pic_adjoint_mixed.cu): particle kernels of the fixed-order pass
struct MixSp {
    int64_t n;
    double q_m, m;
    int *cell;     // packed cell
    float *v[6];   // in-cell offsets (cell units) and momenta
};
struct MixOut {
    int *cell;
    float *v[6];
};
struct MixParams {
    Grid g;
    int nsp;
    int64_t off[kMaxSpecies + 1];
    MixSp sp[kMaxSpecies];      // state at the start of the step
    MixOut out[kMaxSpecies];    // push: state after the step (may alias sp)
    const float *E[3];
    const float *H[3];          // push: H after the half step
    double *J[3];
    float *Fout[6];             // push, optional: interpolated fields per particle
    AdjStatus *st;
    // adjoint
    float *lam[kMaxSpecies][6]; // lambda_x (cell units), lambda_p
    const double *LJ[3];
    double *LE[3], *LH[3];
    float *LF[6];
    const float *Fin[6];        // the push's interpolated fields of this step, or null
};
cudaError_t launch_flat_push_mixed(const MixParams &P, cudaStream_t s);
cudaError_t launch_adj_particles_mixed(const MixParams &P, cudaStream_t s);
// Ha = H + Q(E) in FP32 (the forward's half step, out of place); E, H, Ha: 3 arrays of N each
cudaError_t launch_h_half_mixed(const Grid &g, const float *E, const float *H, float *Ha, size_t N, cudaStream_t s);
void adj_gather_mixed(const Grid &g, const SpeciesView &S, const int64_t *d0, int *cell, void *const v[6],
                      cudaStream_t s);
// lambda_p (3 FP32 arrays of n) and p0 (3 FP32 arrays) -> 6 FP64 arrays of n
void adj_widen_mixed(const float *lp, const float *const p0[3], int64_t n, double *out6, cudaStream_t s);

}  // namespace pic
