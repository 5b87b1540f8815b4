// Form-independent kernels of the B200 PIC step: particle placement and
// binning, migration arrivals, per-cell counts, export, FP64 energy
// reductions and layout conversions.  Compiled with -fmad=false (FP64
// geometry must round like the reference).
#include <cuda_runtime.h>
#include <math.h>
#include "pic_internal.cuh"
#include "pic_kernels.cuh"
#include "pic_rng.cuh"

namespace pic {
namespace {

constexpr float kOneBelow = 0.99999994f;

__device__ __forceinline__ void cell_ijk(const Grid &g, int cell, int &i, int &l, int &k) { g.cell_ijk(cell, i, l, k); }

// getPointCell (cell.h:585-598) + Cell::Insert / isPointInCell (cell.h:717,
// 1754-1768) as used by addParticleListToCells (init.cu:558-592).  Only the
// interior cells hold particles here.
__global__ void k_place(Grid g, int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, int *__restrict__ cell) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double xv = x[p], yv = y[p], zv = z[p];
    int ci = (int)((xv - 0.0) / g.hx), cl = (int)((yv - 0.0) / g.hy), ck = (int)((zv - 0.0) / g.hz);
    int c = -1;
    if (ci >= 0 && ci < g.nx && cl >= 0 && cl < g.ny && ck >= 0 && ck < g.nz) {
        double x0 = (double)ci * g.hx, y0 = (double)cl * g.hy, z0 = (double)ck * g.hz;
        if ((x0 <= xv) && (xv < x0 + g.hx) && (y0 <= yv) && (yv < y0 + g.hy) && (z0 <= zv) && (zv < z0 + g.hz))
            c = g.cell_of(ci, cl, ck);
    }
    cell[p] = c;
}

// Tile of a flat list entry (-1 for a rejected entry or past the end).
__device__ __forceinline__ int entry_tile(const Grid &g, int64_t p, int64_t n, const int *__restrict__ cell, int &c) {
    c = p < n ? cell[p] : -1;
    if (c < 0) return -1;
    int i, l, k;
    cell_ijk(g, c, i, l, k);
    return g.tile_of_cell(i, l, k);
}

// Warp-aggregated per-tile counter: the lanes of a warp with the same tile
// (match.any) take one atomic, issued by their first lane, and each gets the
// old count plus its rank in the group.  Lists arrive grouped by tile, so
// per-lane atomics would put 32 lanes on one address; ranks keep the lanes'
// order, so a warp's entries land contiguously and in input order.  All 32
// lanes must call it.
__device__ __forceinline__ int tile_claim(int *ctr, int t) {
    const unsigned peers = __match_any_sync(0xffffffffu, t);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (t >= 0 && lane == leader) base = atomicAdd(&ctr[t], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(peers & ((1u << lane) - 1));
}

__global__ void k_tile_hist(Grid g, int64_t n, const int *__restrict__ cell, int *tile_counts) {
    int c;
    const int t = entry_tile(g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, n, cell, c);
    tile_claim(tile_counts, t);
}

__device__ __forceinline__ float to_offset(double x, int i, double h) {
    double o = (x - (double)i * h) / h;
    float f = (float)o;
    return fminf(fmaxf(f, 0.f), kOneBelow);
}

__global__ void k_scatter(Grid g, int mixed, int64_t n, const int *__restrict__ cell, const double *__restrict__ x,
                          const double *__restrict__ y, const double *__restrict__ z, const double *__restrict__ px,
                          const double *__restrict__ py, const double *__restrict__ pz, SpeciesView S, int *fill) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int c;
    const int t = entry_tile(g, p, n, cell, c);
    const int rank = tile_claim(fill, t);
    if (t < 0) return;
    int i, l, k;
    cell_ijk(g, c, i, l, k);
    int slot = S.tile_start[t] + rank;
    S.cell[slot] = c;
    if (!mixed) {
        S.x[slot] = x[p]; S.y[slot] = y[p]; S.z[slot] = z[p];
        S.px[slot] = px[p]; S.py[slot] = py[p]; S.pz[slot] = pz[p];
    } else {
        S.ox[slot] = to_offset(x[p], i, g.hx);
        S.oy[slot] = to_offset(y[p], l, g.hy);
        S.oz[slot] = to_offset(z[p], k, g.hz);
        S.fx[slot] = (float)px[p]; S.fy[slot] = (float)py[p]; S.fz[slot] = (float)pz[p];
    }
}

// native-layout load: reference cell number -> interior cell (or -1)
__global__ void k_place_cells(Grid g, int64_t n, const int *__restrict__ ref_cell, const float *__restrict__ ox,
                              const float *__restrict__ oy, const float *__restrict__ oz, int *__restrict__ cell) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int r = ref_cell[p];
    int c = -1;
    if (r >= 0 && (size_t)r < g.nodes_ref()) {
        int k = r % g.NZ, l = (r / g.NZ) % g.NY, i = r / (g.NZ * g.NY);
        bool off = ox[p] >= 0.f && ox[p] < 1.f && oy[p] >= 0.f && oy[p] < 1.f && oz[p] >= 0.f && oz[p] < 1.f;
        if (i < g.nx && l < g.ny && k < g.nz && off) c = g.cell_of(i, l, k);
    }
    cell[p] = c;
}

__global__ void k_scatter_f(Grid g, int mixed, int64_t n, const int *__restrict__ cell, const float *__restrict__ ox,
                            const float *__restrict__ oy, const float *__restrict__ oz, const float *__restrict__ px,
                            const float *__restrict__ py, const float *__restrict__ pz, SpeciesView S, int *fill) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int c;
    const int t = entry_tile(g, p, n, cell, c);
    const int rank = tile_claim(fill, t);
    if (t < 0) return;
    int i, l, k;
    cell_ijk(g, c, i, l, k);
    int slot = S.tile_start[t] + rank;
    S.cell[slot] = c;
    if (mixed) {
        S.ox[slot] = ox[p]; S.oy[slot] = oy[p]; S.oz[slot] = oz[p];
        S.fx[slot] = px[p]; S.fy[slot] = py[p]; S.fz[slot] = pz[p];
    } else {
        S.x[slot] = ((double)i + (double)ox[p]) * g.hx;
        S.y[slot] = ((double)l + (double)oy[p]) * g.hy;
        S.z[slot] = ((double)k + (double)oz[p]) * g.hz;
        S.px[slot] = px[p]; S.py[slot] = py[p]; S.pz[slot] = pz[p];
    }
}


__global__ void k_gather_f(Grid g, int mixed, SpeciesView S, const int64_t *__restrict__ dense_start, int *cell,
                           float *ox, float *oy, float *oz, float *px, float *py, float *pz) {
    int t = blockIdx.x;
    int start = S.tile_start[t], n = S.tile_count[t];
    int64_t d0 = dense_start[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int slot = start + j;
        int c = S.cell[slot];
        int64_t d = d0 + j;
        int i = 0, l = 0, k = 0;
        if (c >= 0) cell_ijk(g, c, i, l, k);
        cell[d] = c < 0 ? -1 : (int)(((size_t)i * g.NY + l) * g.NZ + k);
        if (mixed) {
            ox[d] = S.ox[slot]; oy[d] = S.oy[slot]; oz[d] = S.oz[slot];
            px[d] = S.fx[slot]; py[d] = S.fy[slot]; pz[d] = S.fz[slot];
        } else {
            ox[d] = to_offset(S.x[slot], i, g.hx);
            oy[d] = to_offset(S.y[slot], l, g.hy);
            oz[d] = to_offset(S.z[slot], k, g.hz);
            px[d] = (float)S.px[slot]; py[d] = (float)S.py[slot]; pz[d] = (float)S.pz[slot];
        }
    }
}

// Arrivals of the migration (replaces GPU_ArrangeFlights' Insert, kernels.cu:316-370):
// every outbox entry is appended to its destination tile.  Entries that fit
// are marked done (cell = -1); the rest stay for a rebin.
template <class Out, bool MIXED>
__global__ void k_insert(StepParams P) {
    unsigned n = P.st->out_count;
    if (n > P.out_cap) n = P.out_cap;
    Out *ob = (Out *)P.outbox;
    const Grid &g = P.g;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        Out o = ob[e];
        if (o.cell < 0) continue;
        const SpeciesView &S = P.sp[o.species];
        int i, l, k;
        cell_ijk(g, o.cell, i, l, k);
        int t = g.tile_of_cell(i, l, k);
        int cap = S.tile_start[t + 1] - S.tile_start[t];
        int pos = atomicAdd(&S.tile_count[t], 1);
        if (pos < cap) {
            int slot = S.tile_start[t] + pos;
            S.cell[slot] = o.cell;
            if (MIXED) {
                const OutMixed &q = *(const OutMixed *)&o;
                S.ox[slot] = q.ox; S.oy[slot] = q.oy; S.oz[slot] = q.oz;
                S.fx[slot] = q.px; S.fy[slot] = q.py; S.fz[slot] = q.pz;
            } else {
                const OutPlain &q = *(const OutPlain *)&o;
                S.x[slot] = q.x; S.y[slot] = q.y; S.z[slot] = q.z;
                S.px[slot] = q.px; S.py[slot] = q.py; S.pz[slot] = q.pz;
            }
            ob[e].cell = -1;
        } else {
            atomicAdd(&P.st->overflow_count, 1u);
            atomicOr(&P.st->flags, (unsigned)ST_TILE_FULL);
        }
    }
}

// clamp tile counts after an overflowing insert so the bins stay consistent
__global__ void k_clamp_counts(StepParams P) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.g.ntiles) return;
    for (int s = 0; s < P.nsp; s++) {
        int cap = P.sp[s].tile_start[t + 1] - P.sp[s].tile_start[t];
        if (P.sp[s].tile_count[t] > cap) P.sp[s].tile_count[t] = cap;
    }
}

// per interior cell counts over all species (blockIdx.y = species)
__global__ void k_cell_hist(StepParams P, int *counts) {
    const SpeciesView &S = P.sp[blockIdx.y];
    int t = blockIdx.x;
    int start = S.tile_start[t], n = S.tile_count[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int c = S.cell[start + j];
        if (c < 0) continue;
        int i, l, k;
        cell_ijk(P.g, c, i, l, k);
        if (i < P.g.nx && l < P.g.ny && k < P.g.nz) atomicAdd(&counts[P.g.dense_of(i, l, k)], 1);
    }
}

// the particles of one packed cell in one tile's bin, in no particular order
// (the host sorts them by slot): FP64 global positions and momenta and the slot
__global__ void k_cell_particles(Grid g, int mixed, SpeciesView S, int t, int cell, int64_t cap, double *x, double *y,
                                 double *z, double *px, double *py, double *pz, int64_t *slot, unsigned *count) {
    const int start = S.tile_start[t], n = S.tile_count[t];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int q = start + j;
        if (S.cell[q] != cell) continue;
        const unsigned e = atomicAdd(count, 1u);
        if (e >= cap) continue;
        slot[e] = q;
        if (!mixed) {
            x[e] = S.x[q]; y[e] = S.y[q]; z[e] = S.z[q];
            px[e] = S.px[q]; py[e] = S.py[q]; pz[e] = S.pz[q];
        } else {
            int i, l, k;
            cell_ijk(g, cell, i, l, k);
            x[e] = ((double)i + (double)S.ox[q]) * g.hx;
            y[e] = ((double)l + (double)S.oy[q]) * g.hy;
            z[e] = ((double)k + (double)S.oz[q]) * g.hz;
            px[e] = S.fx[q]; py[e] = S.fy[q]; pz[e] = S.fz[q];
        }
    }
}

// bins -> dense list in slot order (skips dead slots by count, which holds
// none after the compaction)
__global__ void k_gather(Grid g, int mixed, SpeciesView S, const int64_t *__restrict__ dense_start, double *x,
                         double *y, double *z, double *px, double *py, double *pz, int *cell) {
    int t = blockIdx.x;
    int start = S.tile_start[t], n = S.tile_count[t];
    int64_t d0 = dense_start[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int slot = start + j;
        int c = S.cell[slot];
        int64_t d = d0 + j;
        cell[d] = c;
        if (!mixed) {
            x[d] = S.x[slot]; y[d] = S.y[slot]; z[d] = S.z[slot];
            px[d] = S.px[slot]; py[d] = S.py[slot]; pz[d] = S.pz[slot];
        } else {
            int i, l, k;
            if (c < 0) { i = l = k = 0; } else cell_ijk(g, c, i, l, k);
            x[d] = ((double)i + (double)S.ox[slot]) * g.hx;
            y[d] = ((double)l + (double)S.oy[slot]) * g.hy;
            z[d] = ((double)k + (double)S.oz[slot]) * g.hz;
            px[d] = S.fx[slot]; py[d] = S.fy[slot]; pz[d] = S.fz[slot];
        }
    }
}

template <class Out, bool MIXED>
__global__ void k_gather_outbox(StepParams P, int species, unsigned n, unsigned *counter, int64_t offset, double *x,
                                double *y, double *z, double *px, double *py, double *pz, int *cell) {
    unsigned e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    Out o = ((Out *)P.outbox)[e];
    if (o.cell < 0 || o.species != species) return;
    int64_t d = offset + atomicAdd(counter, 1u);
    cell[d] = o.cell;
    if (MIXED) {
        const OutMixed &q = *(const OutMixed *)&o;
        int i, l, k;
        cell_ijk(P.g, q.cell, i, l, k);
        x[d] = ((double)i + (double)q.ox) * P.g.hx;
        y[d] = ((double)l + (double)q.oy) * P.g.hy;
        z[d] = ((double)k + (double)q.oz) * P.g.hz;
        px[d] = q.px; py[d] = q.py; pz[d] = q.pz;
    } else {
        const OutPlain &q = *(const OutPlain *)&o;
        x[d] = q.x; y[d] = q.y; z[d] = q.z;
        px[d] = q.px; py[d] = q.py; pz[d] = q.pz;
    }
}

// seeded generator: one thread per (cell, slot); the tile's slots are laid out
// cell-major (cells in (i,l,k) order inside the tile), ppc per cell
__global__ void k_init_bins(Grid g, int mixed, SpeciesView S, int species_index, int ppc, double dx, double dy,
                            double dz, double vth, uint64_t seed) {
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total = (int64_t)g.ncells() * ppc;
    if (q >= total) return;
    // c: dense cell number (i*Ny + l)*Nz + k, the generator's key
    int c = (int)(q / ppc), slot_in_cell = (int)(q % ppc);
    int k = c % g.nz, l = (c / g.nz) % g.ny, i = c / (g.nz * g.ny);
    int t = g.tile_of_cell(i, l, k);
    int li = i % g.tx, ll = l % g.ty, lk = k % g.tz;
    int ti = i / g.tx, tl = l / g.ty, tk = k / g.tz;
    int ex = min(g.tx, g.nx - ti * g.tx), ey = min(g.ty, g.ny - tl * g.ty), ez = min(g.tz, g.nz - tk * g.tz);
    int cell_in_tile = (li * ey + ll) * ez + lk;
    (void)ex;
    int slot = S.tile_start[t] + cell_in_tile * ppc + slot_in_cell;
    double ox = rng_offset(seed, species_index, c, slot_in_cell, 0);
    double oy = rng_offset(seed, species_index, c, slot_in_cell, 1);
    double oz = rng_offset(seed, species_index, c, slot_in_cell, 2);
    double p0 = dx, p1 = dy, p2 = dz;
    if (vth != 0.0) {
        p0 = dx + vth * rng_normal(seed, species_index, c, slot_in_cell, 0);
        p1 = dy + vth * rng_normal(seed, species_index, c, slot_in_cell, 1);
        p2 = dz + vth * rng_normal(seed, species_index, c, slot_in_cell, 2);
    }
    S.cell[slot] = g.cell_of(i, l, k);
    if (!mixed) {
        S.x[slot] = (double)i * g.hx + ox * g.hx;
        S.y[slot] = (double)l * g.hy + oy * g.hy;
        S.z[slot] = (double)k * g.hz + oz * g.hz;
        S.px[slot] = p0; S.py[slot] = p1; S.pz[slot] = p2;
    } else {
        S.ox[slot] = (float)ox; S.oy[slot] = (float)oy; S.oz[slot] = (float)oz;
        S.fx[slot] = (float)p0; S.fy[slot] = (float)p1; S.fz[slot] = (float)p2;
    }
}

// seeded generator with per-cell counts: one thread per dense cell writes its
// cell's particles at slots first[c] .. first[c] + count[c] - 1
__global__ void k_init_cells(Grid g, int mixed, SpeciesView S, int species_index, const int *__restrict__ count,
                             const int *__restrict__ first, double dx, double dy, double dz, double vth, uint64_t seed) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.ncells()) return;
    const int k = c % g.nz, l = (c / g.nz) % g.ny, i = c / (g.nz * g.ny);
    const int n = count[c], s0 = first[c];
    const int cell = g.cell_of(i, l, k);
    for (int q = 0; q < n; q++) {
        const int slot = s0 + q;
        const double ox = rng_offset(seed, species_index, c, q, 0);
        const double oy = rng_offset(seed, species_index, c, q, 1);
        const double oz = rng_offset(seed, species_index, c, q, 2);
        double p0 = dx, p1 = dy, p2 = dz;
        if (vth != 0.0) {
            p0 = dx + vth * rng_normal(seed, species_index, c, q, 0);
            p1 = dy + vth * rng_normal(seed, species_index, c, q, 1);
            p2 = dz + vth * rng_normal(seed, species_index, c, q, 2);
        }
        S.cell[slot] = cell;
        if (!mixed) {
            S.x[slot] = (double)i * g.hx + ox * g.hx;
            S.y[slot] = (double)l * g.hy + oy * g.hy;
            S.z[slot] = (double)k * g.hz + oz * g.hz;
            S.px[slot] = p0; S.py[slot] = p1; S.pz[slot] = p2;
        } else {
            S.ox[slot] = (float)ox; S.oy[slot] = (float)oy; S.oz[slot] = (float)oz;
            S.fx[slot] = (float)p0; S.fy[slot] = (float)p1; S.fz[slot] = (float)p2;
        }
    }
}

__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    return t;
}

template <typename T>
__global__ void k_field_energy(Grid g, const T *__restrict__ Ex, const T *__restrict__ Ey, const T *__restrict__ Ez,
                               const T *__restrict__ Hx, const T *__restrict__ Hy, const T *__restrict__ Hz,
                               double *out) {
    __shared__ double red[32];
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y, i = blockIdx.z;
    double we = 0.0, wb = 0.0, wr = 0.0;
    if (k < g.NZ) {
        size_t n = g.node(i, l, k);
        double ex = (double)Ex[n], ey = (double)Ey[n], ez = (double)Ez[n];
        wr = ex * ex + ey * ey + ez * ez;  // GPU_getCellEnergy, wrap_kernel.cu:14-36 (all nodes)
        if (i >= 1 && i <= g.nx && l >= 1 && l <= g.ny && k >= 1 && k <= g.nz) {
            double hx = (double)Hx[n], hy = (double)Hy[n], hz = (double)Hz[n];
            we = wr;
            wb = hx * hx + hy * hy + hz * hz;
        }
    }
    double a = block_sum(we, red);
    double b = block_sum(wb, red);
    double c = block_sum(wr, red);
    if (threadIdx.x == 0) {
        atomicAdd(&out[0], a);
        atomicAdd(&out[1], b);
        atomicAdd(&out[2], c);
    }
}

__global__ void k_kinetic(StepParams P, double *out) {
    __shared__ double red[32];
    const SpeciesView &S = P.sp[blockIdx.y];
    int t = blockIdx.x;
    int start = S.tile_start[t], n = S.tile_count[t];
    double M = S.m / S.q_m, acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int slot = start + j;
        if (S.cell[slot] < 0) continue;
        double pu, pv, pw;
        if (P.mixed) { pu = S.fx[slot]; pv = S.fy[slot]; pw = S.fz[slot]; }
        else { pu = S.px[slot]; pv = S.py[slot]; pw = S.pz[slot]; }
        double p2 = pu * pu + pv * pv + pw * pw;
        acc += M * (p2 / (sqrt(1.0 + p2) + 1.0));
    }
    double tot = block_sum(acc, red);
    if (threadIdx.x == 0) atomicAdd(out, tot);
}

template <typename T>
__global__ void k_p2d(Grid g, const T *__restrict__ src, double *dst) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y, i = blockIdx.z;
    if (k >= g.NZ) return;
    dst[((size_t)i * g.NY + l) * g.NZ + k] = (double)src[g.node(i, l, k)];
}

template <typename T>
__global__ void k_d2p(Grid g, const double *__restrict__ src, T *dst) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y, i = blockIdx.z;
    if (k >= g.pz) return;
    dst[g.node(i, l, k)] = k < g.NZ ? (T)src[((size_t)i * g.NY + l) * g.NZ + k] : (T)0;
}

inline unsigned blocks_for(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

cudaError_t place_particles_plain(const Grid &g, int64_t n, const double *x, const double *y, const double *z,
                                  int *cell_out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_place<<<blocks_for(n, 256), 256, 0, s>>>(g, n, x, y, z, cell_out);
    return cudaGetLastError();
}

cudaError_t tile_histogram(const Grid &g, int64_t n, const int *cell, int *tile_counts, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_tile_hist<<<blocks_for(n, 256), 256, 0, s>>>(g, n, cell, tile_counts);
    return cudaGetLastError();
}

cudaError_t scatter_to_bins(const Grid &g, int mixed, int64_t n, const int *cell, const double *x, const double *y,
                            const double *z, const double *px, const double *py, const double *pz, SpeciesView sv,
                            int *fill, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(g, mixed, n, cell, x, y, z, px, py, pz, sv, fill);
    return cudaGetLastError();
}

cudaError_t place_particles_cells(const Grid &g, int64_t n, const int *ref_cell, const float *ox, const float *oy,
                                  const float *oz, int *cell_out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_place_cells<<<blocks_for(n, 256), 256, 0, s>>>(g, n, ref_cell, ox, oy, oz, cell_out);
    return cudaGetLastError();
}

cudaError_t scatter_to_bins_f(const Grid &g, int mixed, int64_t n, const int *cell, const float *ox, const float *oy,
                              const float *oz, const float *px, const float *py, const float *pz, SpeciesView sv,
                              int *fill, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_scatter_f<<<blocks_for(n, 256), 256, 0, s>>>(g, mixed, n, cell, ox, oy, oz, px, py, pz, sv, fill);
    return cudaGetLastError();
}


cudaError_t gather_from_bins_f(const Grid &g, int mixed, SpeciesView sv, const int64_t *dense_start, int *cell,
                               float *ox, float *oy, float *oz, float *px, float *py, float *pz, cudaStream_t s) {
    k_gather_f<<<g.ntiles, 256, 0, s>>>(g, mixed, sv, dense_start, cell, ox, oy, oz, px, py, pz);
    return cudaGetLastError();
}

cudaError_t launch_insert(const StepParams &p, cudaStream_t s) {
    int blocks = 148 * 4;
    if (p.mixed) k_insert<OutMixed, true><<<blocks, 256, 0, s>>>(p);
    else k_insert<OutPlain, false><<<blocks, 256, 0, s>>>(p);
    k_clamp_counts<<<blocks_for(p.g.ntiles, 256), 256, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t cell_histogram(const StepParams &p, int *counts, cudaStream_t s) {
    dim3 grid(p.g.ntiles, p.nsp);
    k_cell_hist<<<grid, 256, 0, s>>>(p, counts);
    return cudaGetLastError();
}

cudaError_t gather_from_bins(const Grid &g, int mixed, SpeciesView sv, const int64_t *dense_start, double *x,
                             double *y, double *z, double *px, double *py, double *pz, int *cell, cudaStream_t s) {
    k_gather<<<g.ntiles, 256, 0, s>>>(g, mixed, sv, dense_start, x, y, z, px, py, pz, cell);
    return cudaGetLastError();
}

cudaError_t cell_particles(const Grid &g, int mixed, const SpeciesView &sv, int tile, int cell, int64_t cap, double *x,
                           double *y, double *z, double *px, double *py, double *pz, int64_t *slot, unsigned *count,
                           cudaStream_t s) {
    k_cell_particles<<<64, 256, 0, s>>>(g, mixed, sv, tile, cell, cap, x, y, z, px, py, pz, slot, count);
    return cudaGetLastError();
}

cudaError_t gather_outbox(const StepParams &p, int species, unsigned n_out, unsigned *counter, int64_t offset,
                          double *x, double *y, double *z, double *px, double *py, double *pz, int *cell,
                          cudaStream_t s) {
    if (n_out == 0) return cudaSuccess;
    if (p.mixed)
        k_gather_outbox<OutMixed, true><<<blocks_for(n_out, 256), 256, 0, s>>>(p, species, n_out, counter, offset, x,
                                                                               y, z, px, py, pz, cell);
    else
        k_gather_outbox<OutPlain, false><<<blocks_for(n_out, 256), 256, 0, s>>>(p, species, n_out, counter, offset, x,
                                                                                y, z, px, py, pz, cell);
    return cudaGetLastError();
}

cudaError_t init_species_bins(const Grid &g, int mixed, SpeciesView sv, int species_index, int ppc, double dx,
                              double dy, double dz, double vth, uint64_t seed, cudaStream_t s) {
    int64_t total = (int64_t)g.ncells() * ppc;
    if (total <= 0) return cudaSuccess;
    k_init_bins<<<blocks_for(total, 256), 256, 0, s>>>(g, mixed, sv, species_index, ppc, dx, dy, dz, vth, seed);
    return cudaGetLastError();
}

cudaError_t init_cells(const Grid &g, int mixed, SpeciesView sv, int species_index, const int *count,
                       const int *first, double dx, double dy, double dz, double vth, uint64_t seed, cudaStream_t s) {
    const int n = g.ncells();
    if (n <= 0) return cudaSuccess;
    k_init_cells<<<(n + 127) / 128, 128, 0, s>>>(g, mixed, sv, species_index, count, first, dx, dy, dz, vth, seed);
    return cudaGetLastError();
}

cudaError_t field_energy(const Grid &g, int mixed, const void *const E[3], const void *const H[3], double *out3,
                         cudaStream_t s) {
    int bx = 128;
    dim3 grid((g.NZ + bx - 1) / bx, g.NY, g.NX);
    if (mixed)
        k_field_energy<float><<<grid, bx, 0, s>>>(g, (const float *)E[0], (const float *)E[1], (const float *)E[2],
                                                  (const float *)H[0], (const float *)H[1], (const float *)H[2], out3);
    else
        k_field_energy<double><<<grid, bx, 0, s>>>(g, (const double *)E[0], (const double *)E[1],
                                                   (const double *)E[2], (const double *)H[0], (const double *)H[1],
                                                   (const double *)H[2], out3);
    return cudaGetLastError();
}

cudaError_t kinetic_energy(const StepParams &p, double *out, cudaStream_t s) {
    dim3 grid(p.g.ntiles, p.nsp);
    k_kinetic<<<grid, 256, 0, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t pitched_to_dense(const Grid &g, const void *src, int is_float, double *dst, cudaStream_t s) {
    int bx = 64;
    dim3 grid((g.NZ + bx - 1) / bx, g.NY, g.NX);
    if (is_float) k_p2d<float><<<grid, bx, 0, s>>>(g, (const float *)src, dst);
    else k_p2d<double><<<grid, bx, 0, s>>>(g, (const double *)src, dst);
    return cudaGetLastError();
}

cudaError_t dense_to_pitched(const Grid &g, const double *src, void *dst, int is_float, cudaStream_t s) {
    int bx = 64;
    dim3 grid((g.pz + bx - 1) / bx, g.NY, g.NX);
    if (is_float) k_d2p<float><<<grid, bx, 0, s>>>(g, src, (float *)dst);
    else k_d2p<double><<<grid, bx, 0, s>>>(g, src, (double *)dst);
    return cudaGetLastError();
}

}  // namespace pic
