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
    int K2;            // sub-checkpoint interval inside a segment (== K: one level)
    size_t pbytes;     // one particle state
    char *cur;         // the forward's running state
    char *ckp;         // nseg particle checkpoints
    char *ckf;         // nseg x (E, H): 6 field arrays each, in the form's field type
    char *segp;        // K2+1 particle states of the (sub-)segment being reversed
    char *segf;        // K2+1 x (E, H) of that (sub-)segment
    char *subp;        // two levels: ceil(K/K2) sub-checkpoint states of the segment being reversed
    char *subf;        // two levels: their (E, H)
    char *lamp;        // per species lambda_x (3) and lambda_p (3), form's element type
    size_t lamp_bytes;
    double *lamf;      // FP64 lambda_E, lambda_H, lambda_J, lambda_Q (12 arrays)
    void *lamF;        // per particle lambda of the 6 interpolated field values (form's element type)
    void *segF;        // optional: K x the 6 interpolated field values per particle of the segment
    char *rf;          // field set of the recompute (form's layout: 12 arrays)
    char *ha;          // B after the half step of the step being reversed (3 arrays)
    double *hist;      // steps x 3: sum over nodes 1..N of E_c^2 after each step
    // frozen branches (plain form): mode 1 records every step's discrete
    // choices into branch (steps x particles codes), mode 2 replays those of
    // branch_src; step_branch / step_bmode are what the next flat push uses
    unsigned long long *branch;
    const unsigned long long *branch_src;
    int branch_mode;
    unsigned long long *step_branch;
    int step_bmode;
    double *red;       // reduction scratch
    AdjStatus *st;
    std::vector<double> hhist;  // host copy of hist x cell volume
    cudaEvent_t e0, e1;
    float t_fwd, t_bwd;
    unsigned long long ambiguous;
    int have_forward;
};

inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// ---- per-block node box for scatters (adjoint of the interpolation).
// Global atomics cost one L2 sector update each; the 256 particles of a block
// sit in a few neighbouring cells (the fixed order is cell-sorted at the
// start), so the block adds its 48 contributions per particle into a shared
// box over the nodes [cell_min, cell_max + 2] per axis and then adds the box
// into global memory with z-contiguous atomics.  Blocks whose box is larger
// than kBoxNodes per component (particles spread out, or on both sides of a
// periodic boundary) add straight into global memory.
constexpr int kBoxNodes = 640;
struct NodeBox {
    int i0, l0, k0, by, bz, nodes;
};
// block-wide box of the cells (i,l,k) of the valid threads; every thread of
// the block must call it (it synchronises); red needs 6 x (warps) ints
__device__ __forceinline__ NodeBox block_node_box(int i, int l, int k, bool valid, int *red, NodeBox *out) {
    const unsigned FULL = 0xffffffffu;
    int v[6] = {valid ? i : 0x7fffffff, valid ? l : 0x7fffffff, valid ? k : 0x7fffffff,
                valid ? i : -1, valid ? l : -1, valid ? k : -1};
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        v[q] = __reduce_min_sync(FULL, v[q]);
        v[3 + q] = __reduce_max_sync(FULL, v[3 + q]);
    }
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 6; q++) red[q * nw + w] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        int r[6];
        for (int q = 0; q < 6; q++) {
            r[q] = red[q * nw];
            for (int u = 1; u < nw; u++) r[q] = q < 3 ? min(r[q], red[q * nw + u]) : max(r[q], red[q * nw + u]);
        }
        NodeBox b;
        b.i0 = r[0]; b.l0 = r[1]; b.k0 = r[2];
        int bx = r[3] - r[0] + 3, by = r[4] - r[1] + 3, bz = r[5] - r[2] + 3;
        b.by = by;
        b.bz = bz;
        bool ok = r[3] >= 0 && bx > 0 && by > 0 && bz > 0 && bx * by * bz <= kBoxNodes;
        b.nodes = ok ? bx * by * bz : 0;  // 0: no box (no valid particle, or too large)
        *out = b;
    }
    __syncthreads();
    return *out;
}
// 2^e as a double from its exponent bits (|e| < 1000)
__device__ __forceinline__ double pow2_d(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }
// box-local index of global node (gi, gl, gk)
__device__ __forceinline__ int box_index(const NodeBox &b, int gi, int gl, int gk) {
    return ((gi - b.i0) * b.by + (gl - b.l0)) * b.bz + (gk - b.k0);
}
// The box holds integer fixed-point sums: FP32 and FP64 shared-memory atomics
// are compare-and-swap loops, 32-bit integer adds are native.  Quantum
// q = 2^(E-22) with 2^E above the block's largest |lambda_F| (a block-wide
// max): every contribution |lambda_F * weight| < 2^22 q, and one node of a
// 256-particle box receives at most 256 of them per component, < 2^30.  The
// FP32 form adds round(v/q) (error q/2, about 2^-23 of the block maximum, the
// FP32 level); the FP64 form also adds the remainder in units of q 2^-22 into
// a second box (error 2^-45 of the block maximum).
__device__ __forceinline__ int box_exponent(float amax_block) {
    // e with 2^(e-1) <= x < 2^e (x > 0 normal); clamped so that q stays normal
    int e = amax_block > 0.f ? (int)((__float_as_uint(amax_block) >> 23) & 0xff) - 126 : -100;
    return max(e, -100);
}
// block-wide max of a non-negative float (every thread calls; synchronises)
__device__ __forceinline__ float block_max_abs(float v, unsigned *red, unsigned *out) {
    unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(v));
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) red[w] = u;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned m = red[0];
        for (int q = 1; q < nw; q++) m = max(m, red[q]);
        *out = m;
    }
    __syncthreads();
    return __uint_as_float(*out);
}
// add the box (6 components of b.nodes sums, hi (+ lo x 2^-22) in units of q)
// into the six global arrays
__device__ __forceinline__ void flush_node_box(const NodeBox &b, const int *hi, const int *lo, double q,
                                               const Grid &g, double *const dst[6]) {
    const int tot = 6 * b.nodes;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        int h = hi[e], l = lo ? lo[e] : 0;
        if (h == 0 && l == 0) continue;
        double v = ((double)h + (double)l * 0x1p-22) * q;
        int c = e / b.nodes, r = e - c * b.nodes;
        int kk = r % b.bz, ll = (r / b.bz) % b.by, ii = r / (b.bz * b.by);
        atomicAdd(&dst[c][g.node(b.i0 + ii, b.l0 + ll, b.k0 + kk)], v);
    }
}
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
