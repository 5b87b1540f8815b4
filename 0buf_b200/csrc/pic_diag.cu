// Charge-conservation diagnostic of the B200 PIC step, in FP64 on the GPU.
//
// The reference has no charge density.  Its zigzag deposit (CurrentToMesh,
// cell.h:1306-1422, with pqr's linear weights, cell.h:1511-1693) and its E
// update (emeElement, kernels.cu:1091-1102) conserve a discrete Gauss law
// exactly when the charge is assigned as follows (derived from the deposit's
// stencil, pinned by the oracle tests):
//   rho[N]  = sum_p m_p W_x W_y W_z,  W = the linear (cloud-in-cell) weight of
//             the particle on the node at position (N - 1/2) h per axis, i.e.
//             the nodes sit at cell centres; a particle in cell i with in-cell
//             offset f (cell units) has the nodes i + (f >= 1/2) and one up,
//             the upper one with weight f + 1/2 - (f >= 1/2);
//   fold    per axis x, y, z: rho[n] += rho[0], rho[1] += rho[n+1], then the
//             ghosts rho[0] = rho[n], rho[n+1] = rho[1] -- the transverse-line
//             form of the current fold (periodicCurrentElement,
//             kernels.cu:1124-1146);
//   div E   (div E)[N] = sum_a (E_a[N] - E_a[N - e_a]) / h_a on interior nodes.
// Then G = div E - rho on the interior nodes does not change from step to
// step: E changes by -tau J and rho by -tau div J, the curl terms cancel.
// pic_gauss_check reports how far G has moved from a stored baseline.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include "pic0buf.h"
#include "pic_internal.cuh"
#include "pic_kernels.cuh"
#include "pic_handle.cuh"

namespace pic {
namespace {

// One CTA per tile: every species' particles of the tile add their eight
// weights into a shared (tx+2)(ty+2)(tz+2) node box in 64-bit fixed point
// (exact and order-independent: q = 2^(E-62) with 2^E > sum |m| over the
// tile's particles, each node receives at most that much), then the box is
// added into the global rho.
__global__ void k_charge_tile(StepParams P, double *rho) {
    const Grid &g = P.g;
    const int mixed = P.mixed, nsp = P.nsp;
    const SpeciesView *sp = P.sp;
    extern __shared__ unsigned long long sR[];
    __shared__ double sQ, sInvQ;
    const int t = blockIdx.x;
    const int tk = t % g.ntz, tl = (t / g.ntz) % g.nty, ti = t / (g.ntz * g.nty);
    const int i0 = ti * g.tx, l0 = tl * g.ty, k0 = tk * g.tz;
    const int SX = g.tx + 2, SY = g.ty + 2, SZ = g.tz + 2;
    const int nn = SX * SY * SZ;
    if (threadIdx.x == 0) {
        double bound = 0.0;
        for (int s = 0; s < nsp; s++) bound += fabs(sp[s].m) * (double)sp[s].tile_count[t];
        int e2;
        frexp(bound > 0.0 ? bound : 1.0, &e2);
        sQ = ldexp(1.0, e2 - 62);
        sInvQ = ldexp(1.0, 62 - e2);
    }
    for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) sR[idx] = 0ull;
    __syncthreads();
    const double inv_q = sInvQ;
    const double h[3] = {g.hx, g.hy, g.hz};
    for (int s = 0; s < nsp; s++) {
        const SpeciesView &S = sp[s];
        const int start = S.tile_start[t], count = S.tile_count[t];
        const double m = S.m;
        for (int j = threadIdx.x; j < count; j += blockDim.x) {
            const int slot = start + j;
            const int c = S.cell[slot];
            if (c < 0) continue;
            int ci[3];
            g.cell_ijk(c, ci[0], ci[1], ci[2]);
            double f[3];
            if (mixed) {
                f[0] = (double)S.ox[slot];
                f[1] = (double)S.oy[slot];
                f[2] = (double)S.oz[slot];
            } else {
                const double x[3] = {S.x[slot], S.y[slot], S.z[slot]};
                for (int a = 0; a < 3; a++) f[a] = x[a] / h[a] - (double)ci[a];
            }
            int lo[3];
            double w1[3];
            const int org[3] = {i0, l0, k0};
            bool ok = true;
            for (int a = 0; a < 3; a++) {
                const int up = f[a] >= 0.5;
                w1[a] = f[a] + 0.5 - (double)up;
                lo[a] = ci[a] + up - org[a];  // tile-local index of the lower node
                ok = ok && lo[a] >= 0 && lo[a] + 1 < (a == 0 ? SX : a == 1 ? SY : SZ);
            }
            if (!ok) continue;  // a bin entry outside its tile (never expected)
            const int nb = (lo[0] * SY + lo[1]) * SZ + lo[2];
            for (int b = 0; b < 8; b++) {
                const int ax = b >> 2, ay = (b >> 1) & 1, az = b & 1;
                const double w = (ax ? w1[0] : 1.0 - w1[0]) * (ay ? w1[1] : 1.0 - w1[1]) * (az ? w1[2] : 1.0 - w1[2]);
                fx_add(&sR[nb + (ax * SY + ay) * SZ + az], m * w, inv_q);
            }
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
        const long long v = (long long)sR[idx];
        if (v == 0) continue;
        const int c = idx % SZ, b = (idx / SZ) % SY, a = idx / (SZ * SY);
        if (i0 + a < g.NX && l0 + b < g.NY && k0 + c < g.NZ) atomicAdd(&rho[g.node(i0 + a, l0 + b, k0 + c)], (double)v * sQ);
    }
}

// periodic fold of rho along one axis, on every line of that axis
__global__ void k_rho_fold(Grid g, double *rho, int dir) {
    const int A = dir == 0 ? g.NY : g.NX;
    const int B = dir == 2 ? g.NY : g.NZ;
    const int n = dir == 0 ? g.nx : (dir == 1 ? g.ny : g.nz);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= A * B) return;
    const int a = idx / B, b = idx % B;
    size_t base, stride;
    if (dir == 0) { base = (size_t)a * g.pz + b; stride = (size_t)g.NY * g.pz; }
    else if (dir == 1) { base = (size_t)a * g.NY * g.pz + b; stride = g.pz; }
    else { base = ((size_t)a * g.NY + b) * g.pz; stride = 1; }
    double *r = rho + base;
    r[(size_t)n * stride] += r[0];
    r[stride] += r[(size_t)(n + 1) * stride];
    r[0] = r[(size_t)n * stride];
    r[(size_t)(n + 1) * stride] = r[stride];
}

// G = div E - rho on the interior nodes (0 on the ghosts); optional baseline
// copy; reductions into red[0] max |G - G0|, red[1] max |rho|, red[2] sum (G - G0)^2,
// red[3] max |G0| (non-negative doubles compared through their bit patterns)
template <typename T>
__global__ void k_gauss(Grid g, const T *__restrict__ Ex, const T *__restrict__ Ey, const T *__restrict__ Ez,
                        const double *__restrict__ rho, double *G, double *G0, int set_baseline, double *red) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y, i = blockIdx.z;
    double dmax = 0.0, rmax = 0.0, d2 = 0.0, g0max = 0.0;
    if (k < g.NZ) {
        const size_t n = g.node(i, l, k);
        const bool interior = i >= 1 && i <= g.nx && l >= 1 && l <= g.ny && k >= 1 && k <= g.nz;
        double v = 0.0;
        if (interior) {
            const size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
            v = ((double)Ex[n] - (double)Ex[n - sx]) / g.hx + ((double)Ey[n] - (double)Ey[n - sy]) / g.hy +
                ((double)Ez[n] - (double)Ez[n - 1]) / g.hz - rho[n];
            rmax = fabs(rho[n]);
        }
        if (G) G[n] = v;
        if (set_baseline) G0[n] = v;
        const double base = G0[n];
        dmax = fabs(v - base);
        d2 = (v - base) * (v - base);
        g0max = fabs(base);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
        rmax = fmax(rmax, __shfl_down_sync(0xffffffffu, rmax, o));
        d2 += __shfl_down_sync(0xffffffffu, d2, o);
        g0max = fmax(g0max, __shfl_down_sync(0xffffffffu, g0max, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax((unsigned long long *)&red[0], (unsigned long long)__double_as_longlong(dmax));
        atomicMax((unsigned long long *)&red[1], (unsigned long long)__double_as_longlong(rmax));
        atomicAdd(&red[2], d2);
        atomicMax((unsigned long long *)&red[3], (unsigned long long)__double_as_longlong(g0max));
    }
}

// total mechanical momentum per species, sum over particles of (m/q_m) p, in
// FP64: one block per (tile, species), out[3 s + a]
__global__ void k_momentum(StepParams P, double *out) {
    __shared__ double red[3][32];
    const SpeciesView &S = P.sp[blockIdx.y];
    const int t = blockIdx.x;
    const int start = S.tile_start[t], n = S.tile_count[t];
    const double M = S.m / S.q_m;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int slot = start + j;
        if (S.cell[slot] < 0) continue;
        if (P.mixed) {
            acc[0] += M * (double)S.fx[slot]; acc[1] += M * (double)S.fy[slot]; acc[2] += M * (double)S.fz[slot];
        } else {
            acc[0] += M * S.px[slot]; acc[1] += M * S.py[slot]; acc[2] += M * S.pz[slot];
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int a = 0; a < 3; a++) {
        double v = acc[a];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[a][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double tot = 0.0;
        for (int i = 0; i < nw; i++) tot += red[threadIdx.x][i];
        atomicAdd(&out[3 * blockIdx.y + threadIdx.x], tot);
    }
}

}  // namespace

cudaError_t momentum(const StepParams &p, double *out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, 3 * p.nsp * sizeof(double), s);
    if (e != cudaSuccess) return e;
    k_momentum<<<dim3(p.g.ntiles, p.nsp), 256, 0, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t charge_density(const StepParams &p, double *rho, cudaStream_t s) {
    const Grid &g = p.g;
    cudaError_t e = cudaMemsetAsync(rho, 0, g.nodes_pitched() * sizeof(double), s);
    if (e != cudaSuccess) return e;
    const size_t smem = (size_t)(g.tx + 2) * (g.ty + 2) * (g.tz + 2) * sizeof(unsigned long long);
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(k_charge_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_charge_tile<<<g.ntiles, 256, smem, s>>>(p, rho);
    for (int dir = 0; dir < 3; dir++) {
        const int A = dir == 0 ? g.NY : g.NX;
        const int B = dir == 2 ? g.NY : g.NZ;
        k_rho_fold<<<(A * B + 127) / 128, 128, 0, s>>>(g, rho, dir);
    }
    return cudaGetLastError();
}

cudaError_t gauss_residual(const Grid &g, int mixed, const void *const E[3], const double *rho, double *G, double *G0,
                           int set_baseline, double *red, cudaStream_t s) {
    const int bx = g.NZ >= 128 ? 128 : 32;
    const dim3 grid((g.NZ + bx - 1) / bx, g.NY, g.NX);
    if (mixed)
        k_gauss<float><<<grid, bx, 0, s>>>(g, (const float *)E[0], (const float *)E[1], (const float *)E[2], rho, G,
                                           G0, set_baseline, red);
    else
        k_gauss<double><<<grid, bx, 0, s>>>(g, (const double *)E[0], (const double *)E[1], (const double *)E[2], rho,
                                            G, G0, set_baseline, red);
    return cudaGetLastError();
}

}  // namespace pic

// ------------------------------------------------------------------ C ABI --
using namespace pic;
using namespace pic_host;

namespace {
int ensure_diag(pic_handle *h) {
    const size_t bytes = h->g.nodes_pitched() * sizeof(double);
    if (!h->rho) {
        CK(cudaMalloc(&h->rho, bytes), "alloc rho");
        CK(cudaMalloc(&h->gauss, bytes), "alloc residual");
        CK(cudaMalloc(&h->gauss0, bytes), "alloc residual baseline");
        CK(cudaMemsetAsync(h->gauss0, 0, bytes, h->stream), "memset");
        h->gauss_has_base = 0;
    }
    return PIC_OK;
}

int compute_rho(pic_handle *h) {
    int rc = need_particles(h);
    if (rc) return rc;
    if ((rc = ensure_diag(h))) return rc;
    StepParams p = make_params(h);
    CK(charge_density(p, h->rho, h->stream), "charge density");
    return PIC_OK;
}

int run_gauss(pic_handle *h, int set_baseline, double *red4) {
    int rc = compute_rho(h);
    if (rc) return rc;
    const void *E[3] = {h->f[PIC_EX], h->f[PIC_EY], h->f[PIC_EZ]};
    CK(cudaMemsetAsync(h->dred, 0, 4 * sizeof(double), h->stream), "memset");
    CK(gauss_residual(h->g, h->mixed, E, h->rho, h->gauss, h->gauss0, set_baseline, h->dred, h->stream), "gauss");
    if (set_baseline) h->gauss_has_base = 1;
    if (red4) {
        CK(cudaMemcpyAsync(h->hred, h->dred, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H");
        CK(cudaStreamSynchronize(h->stream), "sync");
        for (int i = 0; i < 4; i++) red4[i] = h->hred[i];
    }
    return PIC_OK;
}
}  // namespace

extern "C" {

int pic_charge_density(pic_handle *h, double *rho_host) {
    if (!h) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    if ((rc = compute_rho(h))) return rc;
    if (rho_host) {
        CK(pitched_to_dense(h->g, h->rho, 0, h->dense, h->stream), "field layout");
        CK(cudaMemcpyAsync(rho_host, h->dense, h->g.nodes_ref() * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
           "D2H rho");
    }
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_gauss_residual(pic_handle *h, double *g_host) {
    if (!h) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    if ((rc = run_gauss(h, 0, nullptr))) return rc;
    if (g_host) {
        CK(pitched_to_dense(h->g, h->gauss, 0, h->dense, h->stream), "field layout");
        CK(cudaMemcpyAsync(g_host, h->dense, h->g.nodes_ref() * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
           "D2H residual");
    }
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_momentum(pic_handle *h, double *out) {
    if (!h || !out) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    if ((rc = need_particles(h))) return rc;
    if ((rc = ensure_diag(h))) return rc;
    StepParams p = make_params(h);
    // the rho array is free scratch between diagnostic calls
    CK(momentum(p, h->rho, h->stream), "momentum");
    CK(cudaMemcpyAsync(out, h->rho, 3 * p.nsp * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H momentum");
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_gauss_check(pic_handle *h, int set_baseline, double *out4) {
    if (!h || !out4) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    if (!set_baseline && !(h->rho && h->gauss_has_base))
        return set_err(h, PIC_ERR_ARG, "pic_gauss_check: no baseline yet (call it with set_baseline = 1 first)");
    double red[4];
    if ((rc = run_gauss(h, set_baseline, red))) return rc;
    int64_t nodes = (int64_t)h->g.nx * h->g.ny * h->g.nz;
    out4[0] = red[0];
    out4[1] = red[1];
    out4[2] = sqrt(red[2] / (double)nodes);
    out4[3] = red[3];
    return PIC_OK;
}

}  // extern "C"
