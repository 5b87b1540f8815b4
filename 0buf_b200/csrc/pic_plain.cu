// Plain form (FP64, reference arithmetic) kernels of the B200 PIC step.
//
// Compiled with -fmad=false: every FP64 expression below is the reference's
// expression in the reference's order (citations per function), evaluated as
// separate IEEE multiplies and adds like the host build of the reference, so
// that fields match the CPU oracle bit for bit and particles match except
// where the order of the current sums differs (shared/global atomics).
#include <cuda_runtime.h>
#include <math.h>
#include "pic_internal.cuh"
#include "pic_kernels.cuh"

namespace pic {
namespace {

// ------------------------------------------------------------------ Yee --
// emh1_Element (kernels.cu:1052-1073) for the three components over the
// MagneticFieldTrace ranges of MagneticStageOne (gpu_plasma.h:524-538):
//   Hx: i<=Nx+1, l<=Ny, k<=Nz   Q = 0.5*(tau/hz*(Ey[+z]-Ey) - tau/hy*(Ez[+y]-Ez))
//   Hy: i<=Nx, l<=Ny+1, k<=Nz   Q = 0.5*(tau/hx*(Ez[+x]-Ez) - tau/hz*(Ex[+z]-Ex))
//   Hz: i<=Nx, l<=Ny, k<=Nz+1   Q = 0.5*(tau/hy*(Ex[+y]-Ex) - tau/hx*(Ey[+x]-Ey))
__global__ void k_b_half_plain(Grid g, const double *__restrict__ Ex, const double *__restrict__ Ey,
                               const double *__restrict__ Ez, double *Hx, double *Hy, double *Hz, double *Qx,
                               double *Qy, double *Qz, double cx, double cy, double cz) {
    chain_enter();
    // one thread per node of an x plane (l, k flattened: no idle z tail)
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * g.NZ) return;
    const int l = q / g.NZ, k = q - l * g.NZ, i = blockIdx.y;
    size_t n = g.node(i, l, k);
    size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
    if (i <= g.nx + 1 && l <= g.ny && k <= g.nz) {
        double e1_n1 = Ey[n + 1], e1_n = Ey[n], e2_n2 = Ez[n + sy], e2_n = Ez[n];
        double t = 0.5 * (cz * (e1_n1 - e1_n) - cy * (e2_n2 - e2_n));
        Qx[n] = t;
        Hx[n] += t;
    }
    if (i <= g.nx && l <= g.ny + 1 && k <= g.nz) {
        double e1_n1 = Ez[n + sx], e1_n = Ez[n], e2_n2 = Ex[n + 1], e2_n = Ex[n];
        double t = 0.5 * (cx * (e1_n1 - e1_n) - cz * (e2_n2 - e2_n));
        Qy[n] = t;
        Hy[n] += t;
    }
    if (i <= g.nx && l <= g.ny && k <= g.nz + 1) {
        double e1_n1 = Ex[n + sy], e1_n = Ex[n], e2_n2 = Ey[n + sx], e2_n = Ey[n];
        double t = 0.5 * (cy * (e1_n1 - e1_n) - cx * (e2_n2 - e2_n));
        Qz[n] = t;
        Hz[n] += t;
    }
}

// emh2_Element (kernels.cu:1024-1049) over the same ranges
__global__ void k_b_complete_plain(Grid g, double *Hx, double *Hy, double *Hz, const double *__restrict__ Qx,
                                   const double *__restrict__ Qy, const double *__restrict__ Qz) {
    chain_enter();
    // one thread per node of an x plane (l, k flattened: no idle z tail)
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * g.NZ) return;
    const int l = q / g.NZ, k = q - l * g.NZ, i = blockIdx.y;
    size_t n = g.node(i, l, k);
    if (i <= g.nx + 1 && l <= g.ny && k <= g.nz) Hx[n] += Qx[n];
    if (i <= g.nx && l <= g.ny + 1 && k <= g.nz) Hy[n] += Qy[n];
    if (i <= g.nx && l <= g.ny && k <= g.nz + 1) Hz[n] += Qz[n];
}

// emeElement (kernels.cu:1091-1102) over GetElectricFieldStartsDirs ranges
// (gpu_plasma.h:286-304) as called by ElectricFieldEvaluate (gpu_plasma.h:455-483):
//   Ex: i in [0,Nx], l in [1,Ny], k in [1,Nz]: += tau/hy*(Hz-Hz[-y]) - tau/hz*(Hy-Hy[-z]) - tau*Jx
//   Ey: i in [1,Nx], l in [0,Ny], k in [1,Nz]: += tau/hz*(Hx-Hx[-z]) - tau/hx*(Hz-Hz[-x]) - tau*Jy
//   Ez: i in [1,Nx], l in [1,Ny], k in [0,Nz]: += tau/hx*(Hy-Hy[-x]) - tau/hy*(Hx-Hx[-y]) - tau*Jz
__global__ void k_e_update_plain(Grid g, double *Ex, double *Ey, double *Ez, const double *__restrict__ Hx,
                                 const double *__restrict__ Hy, const double *__restrict__ Hz,
                                 const double *__restrict__ Jx, const double *__restrict__ Jy,
                                 const double *__restrict__ Jz, double cx, double cy, double cz, double tau) {
    chain_enter();
    // one thread per node of an x plane (l, k flattened: no idle z tail)
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * g.NZ) return;
    const int l = q / g.NZ, k = q - l * g.NZ, i = blockIdx.y;
    size_t n = g.node(i, l, k);
    size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
    if (i <= g.nx && l >= 1 && l <= g.ny && k >= 1 && k <= g.nz)
        Ex[n] += cy * (Hz[n] - Hz[n - sy]) - cz * (Hy[n] - Hy[n - 1]) - tau * Jx[n];
    if (i >= 1 && i <= g.nx && l <= g.ny && k >= 1 && k <= g.nz)
        Ey[n] += cz * (Hx[n] - Hx[n - 1]) - cx * (Hz[n] - Hz[n - sx]) - tau * Jy[n];
    if (i >= 1 && i <= g.nx && l >= 1 && l <= g.ny && k <= g.nz)
        Ez[n] += cx * (Hy[n] - Hy[n - sx]) - cy * (Hx[n] - Hx[n - sy]) - tau * Jz[n];
}


// --------------------------------------------------------- boundaries --
// A "line" is the set of nodes along one axis at fixed other two indices.
struct Line {
    size_t base, stride;
};
__device__ __forceinline__ Line line_of(const Grid &g, int dir, int a, int b) {
    // getGlobalBoundaryCellNumber, cell.h:885-889: dir 0 -> (N, a, b), 1 -> (a, N, b), 2 -> (a, b, N)
    Line L;
    if (dir == 0) { L.base = (size_t)a * g.pz + b; L.stride = (size_t)g.NY * g.pz; }
    else if (dir == 1) { L.base = (size_t)a * g.NY * g.pz + b; L.stride = g.pz; }
    else { L.base = ((size_t)a * g.NY + b) * g.pz; L.stride = 1; }
    return L;
}

// periodicCurrentElement (kernels.cu:1124-1146) on every line of one axis, all
// three components; SetPeriodicCurrents order (gpu_plasma.h:926-993) is per
// component x, y, z, and the components are independent arrays.
__global__ void k_j_fold(Grid g, double *Jx, double *Jy, double *Jz, int dir) {
    chain_enter();
    int A = dir == 0 ? g.NY : g.NX;
    int B = dir == 2 ? g.NY : g.NZ;
    int N = dir == 0 ? g.NX : (dir == 1 ? g.NY : g.NZ);  // Naxis + 2
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= A * B) return;
    int a = idx / B, b = idx % B;
    Line L = line_of(g, dir, a, b);
    double *J3[3] = {Jx, Jy, Jz};
    for (int comp = 0; comp < 3; comp++) {
        double *E = J3[comp] + L.base;
        size_t n1 = L.stride, n_Nm1 = (size_t)(N - 1) * L.stride;
        if (dir != comp) E[n1] += E[n_Nm1];
        if (dir != 1 || comp != 1) E[n_Nm1] = E[n1];
        size_t n_Nm2 = (size_t)(N - 2) * L.stride;
        E[0] += E[n_Nm2];
        E[n_Nm2] = E[0];
    }
}

// PeriodicBoundaries (gpu_plasma.h:802-870) = periodicElement (kernels.cu:1104-1110)
// E[0] = E[N] then E[N+1] = E[1] on each line of [s1,e1] x [s2,e2]
struct GhostPass {
    void *E;
    int dir, s1, e1, s2, e2, N;
};
// The reference runs the passes in two rounds, A then B.  No node is written
// by both rounds, and no A pass reads a node that B writes; the only order
// between them is B reading ghosts that A wrote.  All passes are copies, so B
// reading A's source node instead gives the same bits, and both rounds run
// in one launch: passes p[0 .. nA) are A, p[nA .. n) are B.
struct GhostPasses {
    GhostPass p[6];
    int nA, n;
};
// node (c[0], c[1], c[2]) of array E, moved to the node an A pass copies into
// it when an A pass writes it
__device__ __forceinline__ size_t ghost_source(const Grid &g, const GhostPasses &P, const void *E, int c[3]) {
    for (int a = 0; a < P.nA; a++) {
        const GhostPass &q = P.p[a];
        if (q.E != E) continue;
        const int d = q.dir;
        const int ca = d == 0 ? c[1] : c[0], cb = d == 2 ? c[1] : c[2];  // the line's (a, b), as in line_of
        if (ca < q.s1 || ca > q.e1 || cb < q.s2 || cb > q.e2) continue;
        if (c[d] == 0) c[d] = q.N;
        else if (c[d] == q.N + 1) c[d] = 1;
    }
    return g.node(c[0], c[1], c[2]);
}
template <typename T>
__global__ void k_e_ghosts(Grid g, GhostPasses P) {
    chain_enter();
    if ((int)blockIdx.y >= P.n) return;
    const GhostPass q = P.p[blockIdx.y];
    const int A = q.e1 - q.s1 + 1, B = q.e2 - q.s2 + 1;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= A * B) return;
    const int la = q.s1 + idx / B, lb = q.s2 + idx % B;
    const Line L = line_of(g, q.dir, la, lb);
    T *E = (T *)q.E;
    size_t srcN = L.base + (size_t)q.N * L.stride, src1 = L.base + L.stride;
    if ((int)blockIdx.y >= P.nA) {
        // line coordinates (x along dir) as in line_of
        int cN[3], c1[3];
        const int d = q.dir, o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
        cN[o1] = c1[o1] = la;
        cN[o2] = c1[o2] = lb;
        cN[d] = q.N;
        c1[d] = 1;
        srcN = ghost_source(g, P, q.E, cN);
        src1 = ghost_source(g, P, q.E, c1);
    }
    E[L.base] = E[srcN];
    E[L.base + (size_t)(q.N + 1) * L.stride] = E[src1];
}


// ------------------------------------------------------- particle push --
enum : int { kCE = 5 };  // CellExtent, cell.h:23

// Interpolate3D, cell.h:1054-1153, on the staged field tile.  (bi,bl,bk) is
// the tile-local node of reference tile index (0,0,0) of the particle's cell,
// i.e. cell_local - 2; the reference tile index (i,l,k) must stay in 2..3 so
// that all 8 taps lie in the staged nodes [cell, cell+2].
__device__ __forceinline__ double interp_plain(const double *__restrict__ T, int SY, int SZ, int bi, int bl,
                                               int bk, int i, int l, int k, double sx, double sx1, double sy,
                                               double sy1, double sz, double sz1, unsigned &bad) {
    if (i < 2 || i > 3 || l < 2 || l > 3 || k < 2 || k > 3) { bad |= ST_STENCIL; return 0.0; }
    int n = ((bi + i) * SY + (bl + l)) * SZ + (bk + k);
    int dz = 1, dy = SZ, dx = SY * SZ;
    double t_ilk = T[n], t_ilk1 = T[n + dz], t_il1k = T[n + dy], t_il1k1 = T[n + dy + dz];
    double t_i1lk = T[n + dx], t_i1lk1 = T[n + dx + dz], t_i1l1k = T[n + dx + dy], t_i1l1k1 = T[n + dx + dy + dz];
    double t1 = sx * (sy * (sz * t_ilk + sz1 * t_ilk1) + sy1 * (sz * t_il1k + sz1 * t_il1k1));
    double t2 = sx1 * (sy * (sz * t_i1lk + sz1 * t_i1lk1) + sy1 * (sz * t_i1l1k + sz1 * t_i1l1k1));
    return t2 + t1;
}

// pqr, cell.h:1511-1693, accumulating into the tile J (shared memory).  The
// reference's divisions by 12 and by tau*h*h are multiplications by their
// reciprocals (rc[d] = 1 / (tau * h_e * h_f), precomputed): the products feed
// only the current's magnitude, never an index, and differ from the quotients
// by an ulp.  LO32 selects the int32 remainder word (fx_add_lo32; words at
// sJ + 3 nn as 3 nn ints), else the 64-bit one (fx_add2; 3 nn words).
template <bool LO32>
__device__ __forceinline__ void pqr_plain(unsigned long long *__restrict__ sJ, double inv_q, double lo_scale, int nn,
                                          int SY, int SZ, int bi, int bl, int bk, const int iv[3], const double x[3],
                                          const double x1[3], double a1, double hx, double hy, double hz,
                                          const double rc[3], double x0, double y0, double z0, unsigned &bad) {
    double dx = (0.50 * (x[0] + x1[0]) - hx * ((double)iv[0] - 2.50) - x0);
    double dy = (0.50 * (x[1] + x1[1]) - hy * ((double)iv[1] - 2.50) - y0);
    double dz = (0.50 * (x[2] + x1[2]) - hz * ((double)iv[2] - 2.50) - z0);
    double a = a1;
    double dx1 = hx - dx, dy1 = hy - dy, dz1 = hz - dz;
    double su = x1[0] - x[0], sv = x1[1] - x[1], sw = x1[2] - x[2];
    constexpr double kTwelfth = 1.0 / 12.0;
    double s1 = sv * sw * kTwelfth, s2 = su * sw * kTwelfth, s3 = su * sv * kTwelfth;
    su = su * a * rc[0];
    sv = sv * a * rc[1];
    sw = sw * a * rc[2];
    if (iv[0] < 2 || iv[0] > 3 || iv[1] < 2 || iv[1] > 3 || iv[2] < 2 || iv[2] > 3) { bad |= ST_STENCIL; return; }
    const int n = ((bi + iv[0]) * SY + (bl + iv[1])) * SZ + (bk + iv[2]);
    const int ez = 1, ey = SZ, ex = SY * SZ;
    int *lo32 = (int *)(sJ + 3 * nn);
    // component c, node offset o from n
    auto add = [&](int c, int o, double v) {
        const int w = c * nn + n + o;
        if (LO32) fx_add_lo32(&sJ[w], &lo32[w], v, inv_q, lo_scale);
        else fx_add2(&sJ[w], &sJ[3 * nn + w], v, inv_q);
    };
    add(0, 0, su * (dy1 * dz1 + s1));
    add(0, ez, su * (dy1 * dz - s1));
    add(0, ey, su * (dy * dz1 - s1));
    add(0, ey + ez, su * (dy * dz + s1));
    add(1, 0, sv * (dx1 * dz1 + s2));
    add(1, ez, sv * (dx1 * dz - s2));
    add(1, ex, sv * (dx * dz1 - s2));
    add(1, ex + ez, sv * (dx * dz + s2));
    add(2, 0, sw * (dx1 * dy1 + s3));
    add(2, ey, sw * (dx1 * dy - s3));
    add(2, ex, sw * (dx * dy1 - s3));
    add(2, ex + ey, sw * (dx * dy + s3));
}

// Reflect, cell.h:1427-1478
__device__ __forceinline__ double reflect_plain(double x, double xm) {
    return (x > xm) * (x - xm) + (x < 0.0) * (xm + x) + (x > 0 && x < xm) * x;
}

// per-axis receivers of a departing particle: the cells of {c-1, c, c+1}
// (wrapped, getWrapCellNumber cell.h:806-853) whose isPointInCell (cell.h:717)
// holds -- the receivers of GPU_ArrangeFlights (kernels.cu:316-370)
__device__ __forceinline__ int receivers(double x, int c, int N, double h, int out[3]) {
    int n = 0;
    for (int d = -1; d <= 1; d++) {
        int j = c + d;
        if (j >= N) j -= N;
        else if (j < 0) j += N;
        double x0 = (double)j * h;
        if ((x0 <= x) && (x < x0 + h)) out[n++] = j;
    }
    return n;
}

// 256 threads, two CTAs per SM: 16 warps per SM at up to 126 registers, no
// spills.  While 64-bit shared atomics were compare-and-swap loops, 512-thread
// CTAs at 64 registers (32 warps, ~240 B of spills) hid their round trips
// better (c2 push 208.7 ms against 246.5 at 256 threads); with the split
// 64-bit add (shared_add64) the atomics cost nothing measurable and 256
// threads win: 71.1 ms against 72.7 (384: 75.0, 448: 76.0).
#ifndef PIC_PLAIN_THREADS
#define PIC_PLAIN_THREADS 256
#endif
#ifndef PIC_PLAIN_MIN_BLOCKS
#define PIC_PLAIN_MIN_BLOCKS 2
#endif
constexpr int kPlainThreads = PIC_PLAIN_THREADS;  // threads per CTA of k_push_plain
// per-warp queue of second zigzag segments: drained when it holds 16 or more
// (at most 32 per drain), so it never holds more than 15 + 32 entries
constexpr int kQPlain = 48;
static_assert(kPlainThreads % 32 == 0, "whole warps");
#ifdef PIC_PLAIN_MIN_BLOCKS
#define PIC_PLAIN_BOUNDS __launch_bounds__(kPlainThreads, PIC_PLAIN_MIN_BLOCKS)
#else
#define PIC_PLAIN_BOUNDS __launch_bounds__(kPlainThreads)
#endif
template <bool LO32>
__global__ void PIC_PLAIN_BOUNDS k_push_plain(StepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sNHoles, sNFront, sNMove;
    __shared__ double sRed[kPlainThreads / 32];
    __shared__ double sQ, sInvQ, sLoScale;
    __shared__ int sQn[kPlainThreads / 32];  // entries in each warp's segment queue
    const Grid &g = P.g;
    const int t = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tk = t % g.ntz, tl = (t / g.ntz) % g.nty, ti = t / (g.ntz * g.nty);
    const int i0 = ti * g.tx, l0 = tl * g.ty, k0 = tk * g.tz;
    const int SX = g.tx + 2, SY = g.ty + 2, SZ = g.tz + 2;
    const int nn = SX * SY * SZ;
    double *sF = (double *)smem_raw;  // Ex Ey Ez Hx Hy Hz
    // fixed-point tile J: 3 nn high words, then the remainder words (3 nn
    // 64-bit, or 3 nn int32 in the first half of that space)
    unsigned long long *sJ = (unsigned long long *)(sF + 6 * nn);
    int *sHoles = (int *)(sJ + 6 * nn);
    int *sFront = sHoles + kHoleMax;
    // this warp's segment queue: x2 and xn (6 x kQPlain doubles), and the
    // start cell (tile-local) with the segment's centre-cell bits
    double *qd = (double *)(sHoles + 2 * kHoleMax) + warp * 6 * kQPlain;
    int *qc = (int *)((double *)(sHoles + 2 * kHoleMax) + (kPlainThreads / 32) * 6 * kQPlain) + warp * kQPlain;
    if (threadIdx.x == 0) {
        double bound = 0.0;
        long long ntile = 0;
        for (int s = 0; s < P.nsp; s++) {
            bound += 2.5 * fabs(P.sp[s].m) * (double)P.sp[s].tile_count[t];
            ntile += P.sp[s].tile_count[t];
        }
        int e2;
        frexp(bound, &e2);  // bound < 2^e2
        sQ = ldexp(1.0, e2 - 62);
        sInvQ = ldexp(1.0, 62 - e2);
        sLoScale = LO32 ? ldexp(1.0, fx_lo32_bits(ntile)) : 1099511627776.0;  // 2^L or 2^40
    }

    // stage E^n and H^{n+1/2} of nodes [i0, i0+tx+2) x [l0, ..) x [k0, ..)
    // (GPU_SetFieldsToCells, kernels.cu:32-49, for all cells of the tile at once)
    const double *const *E = (const double *const *)P.E;
    const double *const *H = (const double *const *)P.H;
    for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
        int c = idx % SZ, b = (idx / SZ) % SY, a = idx / (SZ * SY);
        int gi = i0 + a, gl = l0 + b, gk = k0 + c;
        bool in = gi < g.NX && gl < g.NY && gk < g.NZ;
        size_t n = in ? g.node(gi, gl, gk) : 0;
        sF[idx] = in ? E[0][n] : 0.0;
        sF[nn + idx] = in ? E[1][n] : 0.0;
        sF[2 * nn + idx] = in ? E[2][n] : 0.0;
        sF[3 * nn + idx] = in ? H[0][n] : 0.0;
        sF[4 * nn + idx] = in ? H[1][n] : 0.0;
        sF[5 * nn + idx] = in ? H[2][n] : 0.0;
        for (int w = 0; w < 6; w++) sJ[w * nn + idx] = 0ull;
    }
    __syncthreads();

    const double hx = g.hx, hy = g.hy, hz = g.hz, tau = g.tau;
    const double inv_q = sInvQ, lo_scale = sLoScale;
    // reciprocals of the reference's tau*h*h divisors in pqr
    const double rc[3] = {1.0 / (tau * hy * hz), 1.0 / (tau * hx * hz), 1.0 / (tau * hx * hy)};
    unsigned bad = 0;
    double kin = 0.0;
    unsigned long long moved = 0, dropped = 0, dup = 0;
    OutPlain *outbox = (OutPlain *)P.outbox;

    for (int s = 0; s < P.nsp; s++) {
        const SpeciesView &S = P.sp[s];
        const int start = S.tile_start[t];
        const int count = S.tile_count[t];
        const double q_m = S.q_m, mw = S.m, M = S.m / S.q_m;
        if (threadIdx.x == 0) { sNHoles = 0; sNFront = 0; sNMove = 0; }
        __syncthreads();
        int qn = 0;  // entries in this warp's segment queue (warp-uniform)
        if (lane == 0) sQn[warp] = 0;
        __syncwarp();
        // Whole warps iterate together (the queue is drained by whole warps),
        // and past the last particle until the queue is empty.
        for (int jw = threadIdx.x - lane;; jw += blockDim.x) {
            const bool tail = jw >= count;
            if (tail && qn == 0) break;
            const int j = jw + lane;
            const int slot = start + j;
            // cell < 0: past the bin's end, or a dead slot left by an overflowed compaction
            const int cell = (!tail && j < count) ? S.cell[slot] : -1;
            int i = 0, l = 0, k = 0;
            if (cell >= 0) g.cell_ijk(cell, i, l, k);
            const int bi = i - i0 - 2, bl = l - l0 - 2, bk = k - k0 - 2;
            const bool in_tile = bi >= -2 && bi < g.tx - 2 && bl >= -2 && bl < g.ty - 2 && bk >= -2 && bk < g.tz - 2;
            if (cell >= 0 && !in_tile) bad |= ST_BADCELL;  // a bin entry outside its tile: never index the tile with it
            if (cell >= 0 && in_tile) {
                // Cell ctor, cell.h:731-737
                const double x0 = (double)i * hx, y0 = (double)l * hy, z0 = (double)k * hz;
                double x = S.x[slot], y = S.y[slot], z = S.z[slot];
                double pu = S.px[slot], pv = S.py[slot], pw = S.pz[slot];

                // (x - x0) / h per axis: GetField's tap index and CurrentToMesh's
                // start class both truncate it (divided once, the same bits)
                const double ux = (x - x0) / hx, uy = (y - y0) / hy, uz = (z - z0) / hz;

                // ---- Cell::GetField, cell.h:1257-1290 (InverseKernel 1010-1047)
                double fEx, fEy, fEz, fHx, fHy, fHz;
                if (x < 0 || y < 0 || z < 0) {
                    fEx = fEy = fEz = fHx = fHy = fHz = 0.0;
                } else {
                    int ix = (int)(ux + 1.0) + 1;
                    int i1x = (int)((ux + 1.0) + 1.5);
                    double s1 = (int)(x / hx + 1.0) - x / hx;
                    double s2 = (int)(x / hx + 1.5) - 0.5 - x / hx;
                    int iy = (int)(uy + 1.0) + 1;
                    int i1y = (int)((uy + 1.0) + 1.5);
                    double s3 = (int)(y / hy + 1.0) - y / hy;
                    double s4 = (int)(y / hy + 1.5) - 0.5 - y / hy;
                    int iz = (int)(uz + 1.0) + 1;
                    int i1z = (int)((uz + 1.0) + 1.5);
                    double s5 = (int)(z / hz + 1.0) - z / hz;
                    double s6 = (int)(z / hz + 1.5) - 0.5 - z / hz;
                    double s11 = 1. - s1, s21 = 1. - s2, s31 = 1. - s3, s41 = 1. - s4, s51 = 1. - s5, s61 = 1. - s6;
                    fEx = interp_plain(sF, SY, SZ, bi, bl, bk, ix, i1y, i1z, s1, s11, s4, s41, s6, s61, bad);
                    fEy = interp_plain(sF + nn, SY, SZ, bi, bl, bk, i1x, iy, i1z, s2, s21, s3, s31, s6, s61, bad);
                    fEz = interp_plain(sF + 2 * nn, SY, SZ, bi, bl, bk, i1x, i1y, iz, s2, s21, s4, s41, s5, s51, bad);
                    fHx = interp_plain(sF + 3 * nn, SY, SZ, bi, bl, bk, i1x, iy, iz, s2, s21, s3, s31, s5, s51, bad);
                    fHy = interp_plain(sF + 4 * nn, SY, SZ, bi, bl, bk, ix, i1y, iz, s1, s11, s4, s41, s5, s51, bad);
                    fHz = interp_plain(sF + 5 * nn, SY, SZ, bi, bl, bk, ix, iy, i1z, s1, s11, s3, s31, s6, s61, bad);
                }
                // ---- Particle::Move, particle.h:65-202
                double tau1 = q_m * tau * 0.5;
                pu += tau1 * fEx;
                pv += tau1 * fEy;
                pw += tau1 * fEz;
                // pow(v, -0.5) of the reference as 1 / sqrt(v): two correctly rounded
                // operations, within an ulp of the reference's pow and without its
                // logarithm/exponential code (16 ms of a c2 push)
                double ps = tau1 * (1.0 / sqrt((pu * pu + pv * pv + pw * pw) * 1. + 1.0));
                {
                    double bx = ps * fHx, by = ps * fHy, bz = ps * fHz;
                    double su = pu + pv * bz - pw * by;
                    double sv = pv + pw * bx - pu * bz;
                    double sw = pw + pu * by - pv * bx;
                    double q1 = bx * bx, q2 = by * by, q3 = bz * bz, q4 = bx * by, q5 = by * bz, q6 = bz * bx;
                    // the reference's three divisions by sd as one reciprocal
                    // (continuous values only: within an ulp of the quotients)
                    double sd = q1 + 1. + q2 + q3;
                    const double isd = 1.0 / sd;
                    double pu1 = ((q1 + 1.) * su + (q4 + bz) * sv + (q6 - by) * sw) * isd;
                    double pv1 = ((q4 - bz) * su + (q2 + 1.) * sv + (q5 + bx) * sw) * isd;
                    double pw1 = ((q6 + by) * su + (q5 - bx) * sv + (q3 + 1.) * sw) * isd;
                    pu = pu1 + fEx * tau1;
                    pv = pv1 + fEy * tau1;
                    pw = pw1 + fEz * tau1;
                }
                // gamma = sqrt(p^2 + 1), for the new position and the kinetic energy
                const double p2 = pu * pu + pv * pv + pw * pw;
                const double gam = sqrt(p2 + 1.0);
                ps = 1.0 / gam;
                double xn[3] = {x + tau * (ps * pu), y + tau * (ps * pv), z + tau * (ps * pw)};
                if (!(isfinite(pu) && isfinite(pv) && isfinite(pw))) bad |= ST_NAN;
                kin += M * (p2 / (gam + 1.0));  // gamma - 1 without cancellation

                // ---- Cell::CurrentToMesh, cell.h:1306-1422
                {
                    double xo[3] = {x, y, z}, x2[3] = {0.0, 0.0, 0.0}, sr;
                    const double h3[3] = {hx, hy, hz}, o3[3] = {x0, y0, z0}, r3[3] = {ux, uy, uz};
                    int i1[3], i2[3];
#pragma unroll
                    for (int d = 0; d < 3; d++) {  // getCellNumberCenterCurrent, cell.h:577-578
                        double tt = (r3[d] + 1.5);  // (xo - o3) / h3 + 1.5
                        i1[d] = (int)(tt + 1);
                        double t2 = ((xn[d] - o3[d]) / h3[d] + 1.5);
                        i2[d] = (int)(t2 + 1);
                    }
                    int m = 4 * abs(i2[0] - i1[0]) + 2 * abs(i2[1] - i1[1]) + abs(i2[2] - i1[2]);
#define AVG(d) (h3[d] * (((double)i1[d] + (double)i2[d]) * 0.5 - 2.0) + o3[d])
#define RATIO(d) ((x2[d] - xo[d]) / (xn[d] - xo[d]))
#define PROD(d) ((x2[d] - xo[d]) * (xn[d] - xo[d]))
#define RBX(d) (xo[d] + (xn[d] - xo[d]) * sr)
#define SQ(v) ((v) * (v))
                    switch (m) {
                        case 1: x2[2] = AVG(2); sr = RATIO(2); x2[0] = RBX(0); x2[1] = RBX(1); break;
                        case 2: x2[1] = AVG(1); sr = RATIO(1); x2[0] = RBX(0); x2[2] = RBX(2); break;
                        case 3:
                            x2[1] = AVG(1); x2[2] = AVG(2);
                            sr = (PROD(2) + PROD(1)) / (SQ(xn[2] - xo[2]) + SQ(xn[1] - xo[1]));
                            x2[0] = RBX(0);
                            break;
                        case 4: x2[0] = AVG(0); sr = RATIO(0); x2[1] = RBX(1); x2[2] = RBX(2); break;
                        case 5:
                            x2[0] = AVG(0); x2[2] = AVG(2);
                            sr = (PROD(2) + PROD(0)) / (SQ(xn[2] - xo[2]) + SQ(xn[0] - xo[0]));
                            x2[1] = RBX(1);
                            break;
                        case 6:
                            x2[0] = AVG(0); x2[1] = AVG(1);
                            sr = (PROD(1) + PROD(0)) / (SQ(xn[1] - xo[1]) + SQ(xn[0] - xo[0]));
                            x2[2] = RBX(2);
                            break;
                        case 7: x2[0] = AVG(0); x2[1] = AVG(1); x2[2] = AVG(2); break;
                        default: break;
                    }
#undef AVG
#undef RATIO
#undef PROD
#undef RBX
#undef SQ
                    // the first segment here: xo -> xn, or xo -> x2 when the step
                    // crosses a cell-centre plane.  The second, x2 -> xn, goes to
                    // the warp's queue and is deposited with the warp's other
                    // crossings, 16 to 32 at a time, so that a few crossing lanes do
                    // not make the whole warp run the deposit twice.
                    const bool cross = m >= 1 && m <= 7;
                    double sb[3];
#pragma unroll
                    for (int d = 0; d < 3; d++) sb[d] = cross ? x2[d] : xn[d];
                    pqr_plain<LO32>(sJ, inv_q, lo_scale, nn, SY, SZ, bi, bl, bk, i1, xo, sb, mw, hx, hy, hz, rc, x0, y0,
                                    z0, bad);
                    if (cross) {
                        if (i2[0] >= 2 && i2[0] <= 3 && i2[1] >= 2 && i2[1] <= 3 && i2[2] >= 2 && i2[2] <= 3) {
                            const int e = atomicAdd(&sQn[warp], 1);  // < 15 + 32: drained at 16
#pragma unroll
                            for (int d = 0; d < 3; d++) {
                                qd[d * kQPlain + e] = x2[d];
                                qd[(3 + d) * kQPlain + e] = xn[d];
                            }
                            qc[e] = ((((bi + 2) * g.ty + (bl + 2)) * g.tz + (bk + 2)) << 3) | (i2[0] - 2) |
                                    ((i2[1] - 2) << 1) | ((i2[2] - 2) << 2);
                        } else {
                            bad |= ST_STENCIL;  // pqr's own stencil check
                        }
                    }
                }
                x = reflect_plain(xn[0], g.lx);
                y = reflect_plain(xn[1], g.ly);
                z = reflect_plain(xn[2], g.lz);

                // ---- flyDirection (cell.h:694-701) and the receivers of K8
                int dxd = (((x > x0 + hx) && (x < x0 + 2 * hx)) || ((x < hx) && (i == g.nx - 1)))
                              ? 2 : (((x < x0) || ((x > g.lx - hx) && (i == 0))) ? 0 : 1);
                int dyd = (((y > y0 + hy) && (y < y0 + 2 * hy)) || ((y < hy) && (l == g.ny - 1)))
                              ? 2 : (((y < y0) || ((y > g.ly - hy) && (l == 0))) ? 0 : 1);
                int dzd = (((z > z0 + hz) && (z < z0 + 2 * hz)) || ((z < hz) && (k == g.nz - 1)))
                              ? 2 : (((z < z0) || ((z > g.lz - hz) && (k == 0))) ? 0 : 1);
                int newcell = cell;
                bool leave = false;
                int rx[3], ry[3], rz[3], nrx = 1, nry = 1, nrz = 1;
                if (dxd * 9 + dyd * 3 + dzd != 13) {
                    nrx = receivers(x, i, g.nx, hx, rx);
                    nry = receivers(y, l, g.ny, hy, ry);
                    nrz = receivers(z, k, g.nz, hz, rz);
                    int ncopy = nrx * nry * nrz;
                    if (ncopy == 1 && g.tile_of_cell(rx[0], ry[0], rz[0]) == t) {
                        newcell = g.cell_of(rx[0], ry[0], rz[0]);
                    } else {
                        leave = true;
                        if (ncopy == 0) dropped++;
                        if (ncopy > 1) dup++;
                        if (ncopy > 0) {
                            unsigned e = atomicAdd(&P.st->out_count, (unsigned)ncopy);
                            if (e + ncopy > P.out_cap) {
                                bad |= ST_OUTBOX;
                            } else {
                                for (int a = 0; a < nrx; a++)
                                    for (int b = 0; b < nry; b++)
                                        for (int c = 0; c < nrz; c++) {
                                            OutPlain o;
                                            o.x = x; o.y = y; o.z = z; o.px = pu; o.py = pv; o.pz = pw;
                                            o.cell = g.cell_of(rx[a], ry[b], rz[c]);
                                            o.species = s;
                                            outbox[e++] = o;
                                        }
                                moved++;
                            }
                        }
                    }
                }
                if (leave) {
                    S.cell[slot] = -1;
                    int hpos = atomicAdd(&sNHoles, 1);
                    if (hpos < kHoleMax) sHoles[hpos] = j;
                    else bad |= ST_HOLES;
                } else {
                    S.cell[slot] = newcell;
                    S.x[slot] = x; S.y[slot] = y; S.z[slot] = z;
                    S.px[slot] = pu; S.py[slot] = pv; S.pz[slot] = pw;
                }
            }  // particle
            // ---- the warp's queued second segments, one per lane
            __syncwarp();
            qn = sQn[warp];
            if (qn >= (tail ? 1 : 16)) {
                const int d = qn < 32 ? qn : 32;
                if (lane < d) {
                    const int e = qn - d + lane;
                    const int code = qc[e], lc = code >> 3;
                    const int a = lc / (g.ty * g.tz), b = (lc / g.tz) % g.ty, c = lc % g.tz;
                    const int qi = i0 + a, ql = l0 + b, qk = k0 + c;
                    const int iv[3] = {2 + (code & 1), 2 + ((code >> 1) & 1), 2 + ((code >> 2) & 1)};
                    double sa[3], sb[3];
#pragma unroll
                    for (int dd = 0; dd < 3; dd++) {
                        sa[dd] = qd[dd * kQPlain + e];
                        sb[dd] = qd[(3 + dd) * kQPlain + e];
                    }
                    pqr_plain<LO32>(sJ, inv_q, lo_scale, nn, SY, SZ, a - 2, b - 2, c - 2, iv, sa, sb, mw, hx, hy, hz,
                                    rc, (double)qi * hx, (double)ql * hy, (double)qk * hz, bad);
                }
                qn -= d;
                __syncwarp();
                if (lane == 0) sQn[warp] = qn;
            }
            __syncwarp();
        }
        __syncthreads();
        // ---- compaction of the tile bin (replaces GPU_MakeDepartureLists_rm, kernels.cu:219-242)
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
                    S.x[dst] = S.x[src]; S.y[dst] = S.y[src]; S.z[dst] = S.z[src];
                    S.px[dst] = S.px[src]; S.py[dst] = S.py[src]; S.pz[dst] = S.pz[src];
                }
            }
            if (threadIdx.x == 0) S.tile_count[t] = newcount;
        }
        __syncthreads();
    }

    // ---- tile J -> global J (GPU_WriteAllCurrents, kernels.cu:83-112)
    for (int idx = threadIdx.x; idx < 3 * nn; idx += blockDim.x) {
        const long long ih = (long long)sJ[idx];
        const long long il = LO32 ? (long long)((const int *)(sJ + 3 * nn))[idx] : (long long)sJ[3 * nn + idx];
        if (ih != 0 || il != 0) {
            int comp = idx / nn, r = idx % nn;
            int c = r % SZ, b = (r / SZ) % SY, a = r / (SZ * SY);
            if (i0 + a < g.NX && l0 + b < g.NY && k0 + c < g.NZ)
                atomicAdd(&P.J[comp][g.node(i0 + a, l0 + b, k0 + c)],
                          ((double)ih + (double)il / lo_scale) * sQ);  // exact scale: a power of two
        }
    }
    // ---- kinetic energy and counters
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
    if (dropped) atomicAdd(&P.st->dropped, dropped);
    if (dup) atomicAdd(&P.st->duplicated, dup);
}

}  // namespace

// ------------------------------------------------------------ launchers --
constexpr int kPlaneThreads = 256;
static inline dim3 plane_grid(const Grid &g) {
    return dim3((g.NY * g.NZ + kPlaneThreads - 1) / kPlaneThreads, g.NX);
}

void yee_b_half_plain(const Grid &g, double *const F[12], cudaStream_t s) {
    // getMagneticFieldTimeMeshFactors, gpu_plasma.h:512-522
    double cx = g.tau / (g.hx), cy = g.tau / (g.hy), cz = g.tau / g.hz;
    launch_chained(k_b_half_plain, plane_grid(g), dim3(kPlaneThreads), s, g, F[PIC_EX], F[PIC_EY], F[PIC_EZ], F[PIC_HX],
                   F[PIC_HY], F[PIC_HZ], F[PIC_QX], F[PIC_QY], F[PIC_QZ], cx, cy, cz);
}

void yee_b_complete_plain(const Grid &g, double *const F[12], cudaStream_t s) {
    launch_chained(k_b_complete_plain, plane_grid(g), dim3(kPlaneThreads), s, g, F[PIC_HX], F[PIC_HY], F[PIC_HZ],
                   F[PIC_QX], F[PIC_QY], F[PIC_QZ]);
}

void yee_e_update_plain(const Grid &g, double *const F[12], cudaStream_t s) {
    double cx = g.tau / (g.hx), cy = g.tau / (g.hy), cz = g.tau / g.hz;
    launch_chained(k_e_update_plain, plane_grid(g), dim3(kPlaneThreads), s, g, F[PIC_EX], F[PIC_EY], F[PIC_EZ],
                   F[PIC_HX], F[PIC_HY], F[PIC_HZ], F[PIC_JX], F[PIC_JY], F[PIC_JZ], cx, cy, cz, g.tau);
}


void j_fold(const Grid &g, double *Jx, double *Jy, double *Jz, cudaStream_t s) {
    for (int dir = 0; dir < 3; dir++) {
        int A = dir == 0 ? g.NY : g.NX;
        int B = dir == 2 ? g.NY : g.NZ;
        int n = A * B;
        launch_chained(k_j_fold, dim3((n + 127) / 128), dim3(128), s, g, Jx, Jy, Jz, dir);
    }
}

// ElectricFieldComponentEvaluatePeriodic for Ex, Ey, Ez (gpu_plasma.h:432-452,
// arguments gpu_plasma.h:486-505).  Reference mode skips the y pass of Ex and
// Ez; periodic mode performs it.  Round A holds the first pass of each
// component, round B the second; both run in one launch (GhostPasses).
template <typename T>
static void e_ghosts_t(const Grid &g, T *Ex, T *Ey, T *Ez, int periodic, cudaStream_t s) {
    int Nx = g.nx, Ny = g.ny, Nz = g.nz;
    GhostPasses P{};
    int maxn = 0;
    auto add = [&](T *E, int dir, int s1, int e1, int s2, int e2, int N) {
        P.p[P.n++] = GhostPass{(void *)E, dir, s1, e1, s2, e2, N};
        int n = (e1 - s1 + 1) * (e2 - s2 + 1);
        if (n > maxn) maxn = n;
    };
    // round A: the first pass of each component
    if (periodic) add(Ex, 1, 0, Nx, 1, Nz, Ny);
    add(Ey, 0, 0, Ny, 1, Nz, Nx);
    add(Ez, 0, 1, Ny, 0, Nz, Nx);
    P.nA = P.n;
    // round B: the second (Ey's z pass reads the x ghosts of round A)
    add(Ex, 2, 0, Nx, 0, Ny + 1, Nz);
    add(Ey, 2, 0, Nx + 1, 0, Ny, Nz);
    if (periodic) add(Ez, 1, 0, Nx + 1, 0, Nz, Ny);
    launch_chained(k_e_ghosts<T>, dim3((maxn + 127) / 128, P.n), dim3(128), s, g, P);
}
void e_ghosts_plain(const Grid &g, double *Ex, double *Ey, double *Ez, int periodic, cudaStream_t s) {
    e_ghosts_t<double>(g, Ex, Ey, Ez, periodic, s);
}
void e_ghosts_mixed(const Grid &g, float *Ex, float *Ey, float *Ez, int periodic, cudaStream_t s) {
    e_ghosts_t<float>(g, Ex, Ey, Ez, periodic, s);
}

size_t push_smem_plain(const Grid &g) {
    size_t nn = (size_t)(g.tx + 2) * (g.ty + 2) * (g.tz + 2);
    return 6 * nn * sizeof(double) + 6 * nn * sizeof(unsigned long long) + 2 * kHoleMax * sizeof(int) +
           (size_t)(kPlainThreads / 32) * kQPlain * (6 * sizeof(double) + sizeof(int));
}

cudaError_t launch_push_plain(const StepParams &p, bool lo32, cudaStream_t s) {
    size_t smem = push_smem_plain(p.g);
    auto *kern = lo32 ? k_push_plain<true> : k_push_plain<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<p.g.ntiles, kPlainThreads, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace pic
