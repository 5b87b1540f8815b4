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

// FP32 form (pic_adjoint_mixed.cu)
void adj_gather_mixed(const Grid &g, const SpeciesView &S, const int64_t *d0, int *cell, void *const v[6],
                      cudaStream_t s);
int adj_forward_mixed(pic_handle *h, AdjState &A);
int adj_backward_mixed(pic_handle *h, AdjState &A, const pic_loss &L);
// lambda_p (3 FP32 arrays of n) and p0 (3 FP32 arrays) -> 6 FP64 arrays of n
void adj_widen_mixed(const float *lp, const float *const p0[3], int64_t n, double *out6, cudaStream_t s);

}  // namespace pic
