// Differentiable run of the FP32 mixed form.
#include <cuda_runtime.h>
#include "pic0buf.h"
#include "pic_internal.cuh"
#include "pic_handle.cuh"
#include "pic_adjoint.cuh"

namespace pic {

namespace {
__global__ void k_gather_native(SpeciesView S, const int64_t *__restrict__ d0, int *cell, float *ox, float *oy,
                                float *oz, float *px, float *py, float *pz) {
    int t = blockIdx.x;
    int start = S.tile_start[t], n = S.tile_count[t];
    int64_t base = d0[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int slot = start + j;
        int64_t d = base + j;
        cell[d] = S.cell[slot];
        ox[d] = S.ox[slot]; oy[d] = S.oy[slot]; oz[d] = S.oz[slot];
        px[d] = S.fx[slot]; py[d] = S.fy[slot]; pz[d] = S.fz[slot];
    }
}
__global__ void k_widen(const float *__restrict__ lp, const float *__restrict__ a, const float *__restrict__ b,
                        const float *__restrict__ c, int64_t n, double *out) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    out[j] = lp[j];
    out[n + j] = lp[n + j];
    out[2 * n + j] = lp[2 * n + j];
    out[3 * n + j] = a[j];
    out[4 * n + j] = b[j];
    out[5 * n + j] = c[j];
}
}  // namespace

void adj_gather_mixed(const Grid &g, const SpeciesView &S, const int64_t *d0, int *cell, void *const v[6],
                      cudaStream_t s) {
    k_gather_native<<<g.ntiles, 256, 0, s>>>(S, d0, cell, (float *)v[0], (float *)v[1], (float *)v[2],
                                             (float *)v[3], (float *)v[4], (float *)v[5]);
}

void adj_widen_mixed(const float *lp, const float *const p0[3], int64_t n, double *out6, cudaStream_t s) {
    if (n <= 0) return;
    k_widen<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(lp, p0[0], p0[1], p0[2], n, out6);
}

int adj_forward_mixed(pic_handle *h, AdjState &A) {
    (void)A;
    return pic_host::set_err(h, PIC_ERR_NOT_BUILT, "the FP32 differentiable run is not built yet");
}

int adj_backward_mixed(pic_handle *h, AdjState &A, const pic_loss &L) {
    (void)A;
    (void)L;
    return pic_host::set_err(h, PIC_ERR_NOT_BUILT, "the FP32 differentiable run is not built yet");
}

}  // namespace pic
