// Mixed form (FP32 with FP64 global current) kernels of the B200 PIC step.
//
// Same physics and stencils as the plain form (citations there and below),
// re-expressed in cell units so positions never lose resolution with the
// size of the box: a particle is (int32 cell, FP32 offset in [0,1) per axis,
// FP32 momentum).  Push, deposit and Yee run in FP32; the deposit
// pre-reduces each tile's current in shared memory in FP32 and adds the tile
// into the global J in FP64.
#include <cuda_runtime.h>
#include <math.h>
#include "pic_internal.cuh"
#include "pic_kernels.cuh"

namespace pic {
namespace {

constexpr float kOneBelow = 0.99999994f;  // largest float < 1

// ------------------------------------------------------------------ Yee --
// H += Q(E) in FP32 (emh1_Element, kernels.cu:1052-1073; used for both the
// half step and the completion, which adds the same Q again, kernels.cu:1024-1049)
__global__ void k_b_half_mixed(Grid g, const float *__restrict__ Ex, const float *__restrict__ Ey,
                               const float *__restrict__ Ez, float *Hx, float *Hy, float *Hz, float cx, float cy,
                               float cz) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y;
    int i = blockIdx.z;
    if (k >= g.NZ) return;
    size_t n = g.node(i, l, k);
    size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
    if (i <= g.nx + 1 && l <= g.ny && k <= g.nz) Hx[n] += 0.5f * (cz * (Ey[n + 1] - Ey[n]) - cy * (Ez[n + sy] - Ez[n]));
    if (i <= g.nx && l <= g.ny + 1 && k <= g.nz) Hy[n] += 0.5f * (cx * (Ez[n + sx] - Ez[n]) - cz * (Ex[n + 1] - Ex[n]));
    if (i <= g.nx && l <= g.ny && k <= g.nz + 1) Hz[n] += 0.5f * (cy * (Ex[n + sy] - Ex[n]) - cx * (Ey[n + sx] - Ey[n]));
}

// emeElement (kernels.cu:1091-1102) in FP32, tau*J formed in FP64
__global__ void k_e_update_mixed(Grid g, float *Ex, float *Ey, float *Ez, const float *__restrict__ Hx,
                                 const float *__restrict__ Hy, const float *__restrict__ Hz,
                                 const double *__restrict__ Jx, const double *__restrict__ Jy,
                                 const double *__restrict__ Jz, float cx, float cy, float cz, double tau) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y;
    int i = blockIdx.z;
    if (k >= g.NZ) return;
    size_t n = g.node(i, l, k);
    size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
    if (i <= g.nx && l >= 1 && l <= g.ny && k >= 1 && k <= g.nz)
        Ex[n] += cy * (Hz[n] - Hz[n - sy]) - cz * (Hy[n] - Hy[n - 1]) - (float)(tau * Jx[n]);
    if (i >= 1 && i <= g.nx && l <= g.ny && k >= 1 && k <= g.nz)
        Ey[n] += cz * (Hx[n] - Hx[n - 1]) - cx * (Hz[n] - Hz[n - sx]) - (float)(tau * Jy[n]);
    if (i >= 1 && i <= g.nx && l >= 1 && l <= g.ny && k <= g.nz)
        Ez[n] += cx * (Hy[n] - Hy[n - sx]) - cy * (Hx[n] - Hx[n - sy]) - (float)(tau * Jz[n]);
}

// ------------------------------------------------------- particle push --
// Interpolate3D (cell.h:1054-1153) in cell units on the FP32 tile
__device__ __forceinline__ float interp_mixed(const float *__restrict__ T, int SY, int SZ, int n0, int i, int l,
                                              int k, float sx, float sy, float sz) {
    int n = n0 + (i * SY + l) * SZ + k;
    int dz = 1, dy = SZ, dx = SY * SZ;
    float sx1 = 1.f - sx, sy1 = 1.f - sy, sz1 = 1.f - sz;
    float t1 = sx * (sy * (sz * T[n] + sz1 * T[n + dz]) + sy1 * (sz * T[n + dy] + sz1 * T[n + dy + dz]));
    float t2 = sx1 * (sy * (sz * T[n + dx] + sz1 * T[n + dx + dz]) + sy1 * (sz * T[n + dx + dy] + sz1 * T[n + dx + dy + dz]));
    return t1 + t2;
}

// pqr (cell.h:1511-1693) in cell units: the segment xs -> xe (offsets relative
// to the particle's cell origin) starting in the cell-centre index iv (2 or 3)
__device__ __forceinline__ void pqr_mixed(float *__restrict__ sJ, int nn, int SY, int SZ, int n0, const int iv[3],
                                          const float xs[3], const float xe[3], float wx, float wy, float wz) {
    float dx = 0.5f * (xs[0] + xe[0]) - ((float)iv[0] - 2.5f);
    float dy = 0.5f * (xs[1] + xe[1]) - ((float)iv[1] - 2.5f);
    float dz = 0.5f * (xs[2] + xe[2]) - ((float)iv[2] - 2.5f);
    float dx1 = 1.f - dx, dy1 = 1.f - dy, dz1 = 1.f - dz;
    float su = xe[0] - xs[0], sv = xe[1] - xs[1], sw = xe[2] - xs[2];
    const float r12 = 1.f / 12.f;
    float s1 = sv * sw * r12, s2 = su * sw * r12, s3 = su * sv * r12;
    su *= wx;
    sv *= wy;
    sw *= wz;
    int n = n0 + (iv[0] * SY + iv[1]) * SZ + iv[2];
    int ez = 1, ey = SZ, ex = SY * SZ;
    float *Jx = sJ, *Jy = sJ + nn, *Jz = sJ + 2 * nn;
    atomicAdd(&Jx[n], su * (dy1 * dz1 + s1));
    atomicAdd(&Jx[n + ez], su * (dy1 * dz - s1));
    atomicAdd(&Jx[n + ey], su * (dy * dz1 - s1));
    atomicAdd(&Jx[n + ey + ez], su * (dy * dz + s1));
    atomicAdd(&Jy[n], sv * (dx1 * dz1 + s2));
    atomicAdd(&Jy[n + ez], sv * (dx1 * dz - s2));
    atomicAdd(&Jy[n + ex], sv * (dx * dz1 - s2));
    atomicAdd(&Jy[n + ex + ez], sv * (dx * dz + s2));
    atomicAdd(&Jz[n], sw * (dx1 * dy1 + s3));
    atomicAdd(&Jz[n + ey], sw * (dx1 * dy - s3));
    atomicAdd(&Jz[n + ex], sw * (dx * dy1 - s3));
    atomicAdd(&Jz[n + ex + ey], sw * (dx * dy + s3));
}

__global__ void __launch_bounds__(kPushThreads) k_push_mixed(StepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sNHoles, sNFront, sNMove;
    __shared__ double sRed[kPushThreads / 32];
    const Grid &g = P.g;
    const int t = blockIdx.x;
    const int tk = t % g.ntz, tl = (t / g.ntz) % g.nty, ti = t / (g.ntz * g.nty);
    const int i0 = ti * g.tx, l0 = tl * g.ty, k0 = tk * g.tz;
    const int SX = g.tx + 2, SY = g.ty + 2, SZ = g.tz + 2;
    const int nn = SX * SY * SZ;
    float *sF = (float *)smem_raw;  // Ex Ey Ez Hx Hy Hz
    float *sJ = sF + 6 * nn;
    int *sHoles = (int *)(sJ + 3 * nn);
    int *sFront = sHoles + kHoleMax;

    const float *const *E = (const float *const *)P.E;
    const float *const *H = (const float *const *)P.H;
    for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
        int c = idx % SZ, b = (idx / SZ) % SY, a = idx / (SZ * SY);
        int gi = i0 + a, gl = l0 + b, gk = k0 + c;
        bool in = gi < g.NX && gl < g.NY && gk < g.NZ;
        size_t n = in ? g.node(gi, gl, gk) : 0;
        sF[idx] = in ? E[0][n] : 0.f;
        sF[nn + idx] = in ? E[1][n] : 0.f;
        sF[2 * nn + idx] = in ? E[2][n] : 0.f;
        sF[3 * nn + idx] = in ? H[0][n] : 0.f;
        sF[4 * nn + idx] = in ? H[1][n] : 0.f;
        sF[5 * nn + idx] = in ? H[2][n] : 0.f;
        sJ[idx] = 0.f;
        sJ[nn + idx] = 0.f;
        sJ[2 * nn + idx] = 0.f;
    }
    __syncthreads();

    const float ctx = (float)(g.tau / g.hx), cty = (float)(g.tau / g.hy), ctz = (float)(g.tau / g.hz);
    unsigned bad = 0;
    double kin = 0.0;
    unsigned long long moved = 0;
    OutMixed *outbox = (OutMixed *)P.outbox;

    for (int s = 0; s < P.nsp; s++) {
        const SpeciesView &S = P.sp[s];
        const int start = S.tile_start[t];
        const int count = S.tile_count[t];
        const float tau1 = (float)(S.q_m * g.tau * 0.5);
        const double M = S.m / S.q_m;
        // per-species deposit weights a*h/tau (see pqr_mixed)
        const float wx = (float)(S.m * g.hx / g.tau), wy = (float)(S.m * g.hy / g.tau), wz = (float)(S.m * g.hz / g.tau);
        if (threadIdx.x == 0) { sNHoles = 0; sNFront = 0; sNMove = 0; }
        __syncthreads();
        for (int j = threadIdx.x; j < count; j += blockDim.x) {
            const int slot = start + j;
            const int cell = S.cell[slot];
            if (cell < 0) continue;
            int k = cell % g.nz, l = (cell / g.nz) % g.ny, i = cell / (g.nz * g.ny);
            if (i - i0 < 0 || i - i0 >= g.tx || l - l0 < 0 || l - l0 >= g.ty || k - k0 < 0 || k - k0 >= g.tz) {
                bad |= ST_BADCELL;  // a bin entry outside its tile: never index the tile with it
                continue;
            }
            // tile-local node of reference tile index (0,0,0): cell_local - 2
            const int n0 = ((i - i0 - 2) * SY + (l - l0 - 2)) * SZ + (k - k0 - 2);
            float xs[3] = {S.ox[slot], S.oy[slot], S.oz[slot]};
            float pu = S.fx[slot], pv = S.fy[slot], pw = S.fz[slot];

            // ---- GetField (cell.h:1257-1290) in cell units: getCellNumber = 2,
            // getCellNumberCenter = 2 + (offset >= 1/2), weights s1 = 1-o, s2 = 1/2-o (+1)
            const int i1x = 2 + (xs[0] >= 0.5f), i1y = 2 + (xs[1] >= 0.5f), i1z = 2 + (xs[2] >= 0.5f);
            const float s1 = 1.f - xs[0], s2 = (i1x == 2 ? 0.5f : 1.5f) - xs[0];
            const float s3 = 1.f - xs[1], s4 = (i1y == 2 ? 0.5f : 1.5f) - xs[1];
            const float s5 = 1.f - xs[2], s6 = (i1z == 2 ? 0.5f : 1.5f) - xs[2];
            float fEx = interp_mixed(sF, SY, SZ, n0, 2, i1y, i1z, s1, s4, s6);
            float fEy = interp_mixed(sF + nn, SY, SZ, n0, i1x, 2, i1z, s2, s3, s6);
            float fEz = interp_mixed(sF + 2 * nn, SY, SZ, n0, i1x, i1y, 2, s2, s4, s5);
            float fHx = interp_mixed(sF + 3 * nn, SY, SZ, n0, i1x, 2, 2, s2, s3, s5);
            float fHy = interp_mixed(sF + 4 * nn, SY, SZ, n0, 2, i1y, 2, s1, s4, s5);
            float fHz = interp_mixed(sF + 5 * nn, SY, SZ, n0, 2, 2, i1z, s1, s3, s6);

            // ---- Particle::Move (particle.h:65-202), FP32
            pu += tau1 * fEx;
            pv += tau1 * fEy;
            pw += tau1 * fEz;
            float ps = tau1 * rsqrtf(pu * pu + pv * pv + pw * pw + 1.f);
            {
                float bx = ps * fHx, by = ps * fHy, bz = ps * fHz;
                float su = pu + pv * bz - pw * by;
                float sv = pv + pw * bx - pu * bz;
                float sw = pw + pu * by - pv * bx;
                float q1 = bx * bx, q2 = by * by, q3 = bz * bz, q4 = bx * by, q5 = by * bz, q6 = bz * bx;
                float rs = 1.f / (q1 + 1.f + q2 + q3);
                float pu1 = ((q1 + 1.f) * su + (q4 + bz) * sv + (q6 - by) * sw) * rs;
                float pv1 = ((q4 - bz) * su + (q2 + 1.f) * sv + (q5 + bx) * sw) * rs;
                float pw1 = ((q6 + by) * su + (q5 - bx) * sv + (q3 + 1.f) * sw) * rs;
                pu = pu1 + fEx * tau1;
                pv = pv1 + fEy * tau1;
                pw = pw1 + fEz * tau1;
            }
            float p2 = pu * pu + pv * pv + pw * pw;
            float ig = rsqrtf(p2 + 1.f);
            if (!(isfinite(pu) && isfinite(pv) && isfinite(pw))) bad |= ST_NAN;
            // gamma - 1 = p^2 / (gamma + 1), accumulated in FP64
            kin += M * (double)(p2 / (1.f / ig + 1.f));
            float xe[3] = {xs[0] + ctx * (ig * pu), xs[1] + cty * (ig * pv), xs[2] + ctz * (ig * pw)};

            // ---- CurrentToMesh (cell.h:1306-1422) in cell units
            {
                // cell-centre index of the end point from the same exact float
                // thresholds as i1 (x + 2.5 rounded in FP32 would put a point one
                // ulp below a centre plane on the far side of it)
                int i1[3] = {i1x, i1y, i1z}, i2[3];
#pragma unroll
                for (int d = 0; d < 3; d++)
                    i2[d] = 2 + (xe[d] >= 0.5f) + (xe[d] >= 1.5f) - (xe[d] < -0.5f);
                if (i2[0] < 2 || i2[0] > 3 || i2[1] < 2 || i2[1] > 3 || i2[2] < 2 || i2[2] > 3) {
                    bad |= ST_STENCIL;
                } else {
                    int m = 4 * abs(i2[0] - i1[0]) + 2 * abs(i2[1] - i1[1]) + abs(i2[2] - i1[2]);
                    if (m == 0) {
                        pqr_mixed(sJ, nn, SY, SZ, n0, i1, xs, xe, wx, wy, wz);
                    } else {
                        // the crossing plane of an axis that changes centre index is the cell centre 1/2
                        float x2[3], sr;
#define RATIO(d) ((x2[d] - xs[d]) / (xe[d] - xs[d]))
#define PROD(d) ((x2[d] - xs[d]) * (xe[d] - xs[d]))
#define SQ(v) ((v) * (v))
#define RBX(d) (xs[d] + (xe[d] - xs[d]) * sr)
                        switch (m) {
                            case 1: x2[2] = 0.5f; sr = RATIO(2); x2[0] = RBX(0); x2[1] = RBX(1); break;
                            case 2: x2[1] = 0.5f; sr = RATIO(1); x2[0] = RBX(0); x2[2] = RBX(2); break;
                            case 3:
                                x2[1] = 0.5f; x2[2] = 0.5f;
                                sr = (PROD(2) + PROD(1)) / (SQ(xe[2] - xs[2]) + SQ(xe[1] - xs[1]));
                                x2[0] = RBX(0);
                                break;
                            case 4: x2[0] = 0.5f; sr = RATIO(0); x2[1] = RBX(1); x2[2] = RBX(2); break;
                            case 5:
                                x2[0] = 0.5f; x2[2] = 0.5f;
                                sr = (PROD(2) + PROD(0)) / (SQ(xe[2] - xs[2]) + SQ(xe[0] - xs[0]));
                                x2[1] = RBX(1);
                                break;
                            case 6:
                                x2[0] = 0.5f; x2[1] = 0.5f;
                                sr = (PROD(1) + PROD(0)) / (SQ(xe[1] - xs[1]) + SQ(xe[0] - xs[0]));
                                x2[2] = RBX(2);
                                break;
                            default: x2[0] = 0.5f; x2[1] = 0.5f; x2[2] = 0.5f; break;
                        }
#undef RATIO
#undef PROD
#undef SQ
#undef RBX
                        pqr_mixed(sJ, nn, SY, SZ, n0, i1, xs, x2, wx, wy, wz);
                        pqr_mixed(sJ, nn, SY, SZ, n0, i2, x2, xe, wx, wy, wz);
                    }
                }
            }
            // ---- new cell (Reflect cell.h:1427-1478 and migration, in cell units)
            int ci[3] = {i, l, k};
            const int nc[3] = {g.nx, g.ny, g.nz};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (xe[d] >= 1.f) {
                    xe[d] -= 1.f;
                    ci[d] = ci[d] + 1 == nc[d] ? 0 : ci[d] + 1;
                } else if (xe[d] < 0.f) {
                    xe[d] += 1.f;
                    ci[d] = ci[d] == 0 ? nc[d] - 1 : ci[d] - 1;
                }
                xe[d] = fminf(fmaxf(xe[d], 0.f), kOneBelow);
            }
            const int newcell = g.cell_of(ci[0], ci[1], ci[2]);
            if (newcell == cell || g.tile_of_cell(ci[0], ci[1], ci[2]) == t) {
                S.cell[slot] = newcell;
                S.ox[slot] = xe[0]; S.oy[slot] = xe[1]; S.oz[slot] = xe[2];
                S.fx[slot] = pu; S.fy[slot] = pv; S.fz[slot] = pw;
            } else {
                unsigned e = atomicAdd(&P.st->out_count, 1u);
                if (e < P.out_cap) {
                    OutMixed o;
                    o.ox = xe[0]; o.oy = xe[1]; o.oz = xe[2]; o.px = pu; o.py = pv; o.pz = pw;
                    o.cell = newcell;
                    o.species = s;
                    outbox[e] = o;
                    moved++;
                } else {
                    bad |= ST_OUTBOX;
                }
                S.cell[slot] = -1;
                int hpos = atomicAdd(&sNHoles, 1);
                if (hpos < kHoleMax) sHoles[hpos] = j;
                else bad |= ST_HOLES;
            }
        }
        __syncthreads();
        const int L = sNHoles;
        if (L > 0 && L <= kHoleMax) {
            const int newcount = count - L;
            for (int r = threadIdx.x; r < L; r += blockDim.x) {
                int h = sHoles[r];
                if (h < newcount) sFront[atomicAdd(&sNFront, 1)] = h;
            }
            __syncthreads();
            for (int r = threadIdx.x; r < L; r += blockDim.x) {
                int src = start + newcount + r;
                if (S.cell[src] >= 0) {
                    int m = atomicAdd(&sNMove, 1);
                    if (m >= sNFront) { bad |= ST_BADCELL; continue; }
                    int dst = start + sFront[m];
                    S.cell[dst] = S.cell[src];
                    S.ox[dst] = S.ox[src]; S.oy[dst] = S.oy[src]; S.oz[dst] = S.oz[src];
                    S.fx[dst] = S.fx[src]; S.fy[dst] = S.fy[src]; S.fz[dst] = S.fz[src];
                }
            }
            if (threadIdx.x == 0) S.tile_count[t] = newcount;
        }
        __syncthreads();
    }

    for (int idx = threadIdx.x; idx < 3 * nn; idx += blockDim.x) {
        float v = sJ[idx];
        if (v != 0.f) {
            int comp = idx / nn, r = idx % nn;
            int c = r % SZ, b = (r / SZ) % SY, a = r / (SZ * SY);
            if (i0 + a < g.NX && l0 + b < g.NY && k0 + c < g.NZ)
                atomicAdd(&P.J[comp][g.node(i0 + a, l0 + b, k0 + c)], (double)v);
        }
    }
    for (int o = 16; o > 0; o >>= 1) kin += __shfl_down_sync(0xffffffffu, kin, o);
    if ((threadIdx.x & 31) == 0) sRed[threadIdx.x >> 5] = kin;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += sRed[w];
        atomicAdd(&P.st->kinetic, tot);
    }
    if (bad) atomicOr(&P.st->flags, bad);
    if (moved) atomicAdd(&P.st->moved, moved);
}

}  // namespace

static inline dim3 node_grid(const Grid &g, int bx) { return dim3((g.NZ + bx - 1) / bx, g.NY, g.NX); }

void yee_b_half_mixed(const Grid &g, float *const E[3], float *const H[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    int bx = g.NZ >= 128 ? 128 : 32;
    k_b_half_mixed<<<node_grid(g, bx), bx, 0, s>>>(g, E[0], E[1], E[2], H[0], H[1], H[2], cx, cy, cz);
}

void yee_e_update_mixed(const Grid &g, float *const E[3], float *const H[3], double *const J[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    int bx = g.NZ >= 128 ? 128 : 32;
    k_e_update_mixed<<<node_grid(g, bx), bx, 0, s>>>(g, E[0], E[1], E[2], H[0], H[1], H[2], J[0], J[1], J[2], cx,
                                                     cy, cz, g.tau);
}

size_t push_smem_mixed(const Grid &g) {
    size_t nn = (size_t)(g.tx + 2) * (g.ty + 2) * (g.tz + 2);
    return 9 * nn * sizeof(float) + 2 * kHoleMax * sizeof(int);
}

cudaError_t launch_push_mixed(const StepParams &p, cudaStream_t s) {
    size_t smem = push_smem_mixed(p.g);
    cudaError_t e = cudaFuncSetAttribute(k_push_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_push_mixed<<<p.g.ntiles, kPushThreads, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace pic
