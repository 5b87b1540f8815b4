// Mixed form (FP32 with FP64 global current) kernels of the B200 PIC step.
//
// Same physics and stencils as the plain form (citations there and below),
// re-expressed in cell units so positions never lose resolution with the
// size of the box: a particle is (int32 cell, FP32 offset in [0,1) per axis,
// FP32 momentum).  Push, deposit and Yee run in FP32; the deposit
// pre-reduces each tile's current in shared memory (64-bit fixed point, see
// fx_add) and adds the tile into the global J in FP64.
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
    // one thread per node of an x plane (l, k flattened: no idle z tail)
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * g.NZ) return;
    const int l = q / g.NZ, k = q - l * g.NZ, i = blockIdx.y;
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
    // one thread per node of an x plane (l, k flattened: no idle z tail)
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * g.NZ) return;
    const int l = q / g.NZ, k = q - l * g.NZ, i = blockIdx.y;
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
// Interpolate3D (cell.h:1054-1153) in cell units on the FP32 tile, stored as
// yz-quads: Q[n] = (T[n], T[n+dz], T[n+dy], T[n+dy+dz]), so the 8 taps are two
// 128-bit shared loads (the same products and sums, in the same order, as
// the 8 scalar taps)
__device__ __forceinline__ float interp_mixed(const float4 *__restrict__ Q, int SY, int SZ, int n0, int i, int l,
                                              int k, float sx, float sy, float sz) {
    const int n = n0 + (i * SY + l) * SZ + k;
    const float4 A = Q[n], B = Q[n + SY * SZ];
    const float sx1 = 1.f - sx, sy1 = 1.f - sy, sz1 = 1.f - sz;
    float t1 = sx * (sy * (sz * A.x + sz1 * A.y) + sy1 * (sz * A.z + sz1 * A.w));
    float t2 = sx1 * (sy * (sz * B.x + sz1 * B.y) + sy1 * (sz * B.z + sz1 * B.w));
    return t1 + t2;
}

// pqr (cell.h:1511-1693) in cell units: the 12 contributions of the segment
// xs -> xe (offsets relative to the particle's cell origin) whose cell-centre
// index is iv (2 or 3 per axis).  Order: Jx (0,0,0) (0,0,1) (0,1,0) (0,1,1),
// Jy (0,0,0) (0,0,1) (1,0,0) (1,0,1), Jz (0,0,0) (0,1,0) (1,0,0) (1,1,0),
// node offsets (x,y,z) relative to the base node iv.
__device__ __forceinline__ void pqr_mixed(const int iv[3], const float xs[3], const float xe[3], float wx, float wy,
                                          float wz, float v[12]) {
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
    v[0] = su * (dy1 * dz1 + s1);
    v[1] = su * (dy1 * dz - s1);
    v[2] = su * (dy * dz1 - s1);
    v[3] = su * (dy * dz + s1);
    v[4] = sv * (dx1 * dz1 + s2);
    v[5] = sv * (dx1 * dz - s2);
    v[6] = sv * (dx * dz1 - s2);
    v[7] = sv * (dx * dz + s2);
    v[8] = sw * (dx1 * dy1 + s3);
    v[9] = sw * (dx1 * dy - s3);
    v[10] = sw * (dx * dy1 - s3);
    v[11] = sw * (dx * dy + s3);
}

// tile-local J index of contribution j of a segment whose base node is nb
__device__ __forceinline__ int contrib_node(int j, int nb, int nn, int SY, int SZ) {
    int comp = j >> 2, r = j & 3;
    int hi = r >> 1, lo = r & 1;
    int dx = comp == 0 ? 0 : hi;
    int dy = comp == 0 ? hi : (comp == 1 ? 0 : lo);
    int dz = comp == 2 ? 0 : lo;
    return comp * nn + nb + (dx * SY + dy) * SZ + dz;
}

// The split point of a segment that crosses cell-centre planes
// (CurrentToMesh, cell.h:1338-1403), branch-free, in cell units.  An axis
// whose centre index changes crosses the cell centre 1/2 and x2 lies on that
// plane; the other coordinates follow the straight path at the parameter
//   s = sum_c (1/2 - xs_c)(xe_c - xs_c) / sum_c (xe_c - xs_c)^2
// over the crossing axes c -- the reference's formula for one crossing axis
// (cases 1, 2, 4: a ratio) and for two (cases 3, 5, 6: the point nearest to
// both planes); with three crossing axes x2 is the centre.  Without a crossing
// x2 = xe: the second segment then has length 0 and adds nothing.
__device__ __forceinline__ void split_point(const int i1[3], const int i2[3], const float xs[3], const float xe[3],
                                            float x2[3]) {
    float num = 0.f, den = 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        float dl = xe[d] - xs[d];
        bool c = i1[d] != i2[d];
        num += c ? (0.5f - xs[d]) * dl : 0.f;
        den += c ? dl * dl : 0.f;
    }
    const bool any = den > 0.f;
    const float sr = any ? __fdividef(num, den) : 1.f;
#pragma unroll
    for (int d = 0; d < 3; d++) x2[d] = (i1[d] != i2[d]) ? 0.5f : xs[d] + (xe[d] - xs[d]) * sr;
}

// 2^e as float by exponent bits (no library call, no branch);
// valid for -126 < e < 128
__device__ __forceinline__ float pow2f(int e) { return __uint_as_float((unsigned)(e + 127) << 23); }
// e with 2^(e-1) <= x < 2^e for a positive normal float (0 for x = 0)
__device__ __forceinline__ int exponent_above(float x) {
    return x > 0.f ? (int)((__float_as_uint(x) >> 23) & 0xff) - 126 : 0;
}

// One particle's loaded state.
struct PartM {
    int cell;
    float x, y, z, px, py, pz;
};

__device__ __forceinline__ PartM load_part(const SpeciesView &S, int slot) {
    PartM p;
    p.cell = S.cell[slot];
    p.x = S.ox[slot]; p.y = S.oy[slot]; p.z = S.oz[slot];
    p.px = S.fx[slot]; p.py = S.fy[slot]; p.pz = S.fz[slot];
    return p;
}

// Deposit of the warp's current, two levels:
//  1. the depositing lanes form one group per distinct cell (match.any); for
//     up to kGroups groups per warp, lanes add the first zigzag segment of
//     their particle into a per-warp int32 scratch of 54 node slots per group
//     -- the nodes that the segments of a particle in one cell can reach (Jx
//     2x3x3, Jy 3x2x3, Jz 3x3x2 around the cell's stencil origin) -- with
//     native 32-bit shared atomics.  The warp's quantum q_w is a power of two
//     above 2^-22 x the largest possible contribution of any of its lanes
//     (1.0834 |current of the full step|, reduced with redux.sync), so the
//     int32 sums of <= 32 contributions cannot overflow.  The <= 54 sums per
//     group then go into the tile's exact 64-bit fixed-point J (fx_add).
//  2. segments that do not fit that pattern -- the second segment of a
//     particle that crosses a cell-centre plane, and both segments of a lane
//     beyond kGroups distinct cells (bins out of cell order) -- are queued
//     per warp and deposited 32 at a time, one per lane, straight into the
//     tile J, so a few such lanes do not stall the other lanes of their warp.
constexpr int kGroups = 4;
constexpr int kSlots = 54;
// 320 threads, two CTAs per SM (96 registers, no spills): 20 warps per SM
// against 16 with 256 threads at 123 registers; the kernel is issue-bound and
// the extra warps cut the c2 push from 30.5 to 29.2 ms (288 and 384 threads
// measured slower)
#ifndef PIC_MIXED_THREADS
#define PIC_MIXED_THREADS 320
#endif
#ifndef PIC_MIXED_MIN_BLOCKS
#define PIC_MIXED_MIN_BLOCKS 2
#endif
#ifndef PIC_MIXED_QUEUE
#define PIC_MIXED_QUEUE 64
#endif
constexpr int kMixedThreads = PIC_MIXED_THREADS;  // threads per CTA of k_push_mixed
constexpr int kQueue = PIC_MIXED_QUEUE;           // queued segments per warp
static_assert(kMixedThreads % 32 == 0, "whole warps");
static_assert(kHoleMax * sizeof(int) <= (kMixedThreads / 32) * kQueue * 2 * sizeof(float4),
              "the compaction's front-hole list lives in the queues' memory");

// w (in units of 2^e_w) -> units of 2^e_tile, sh = e_w - e_tile, round half up
__device__ __forceinline__ long long rescale(int w, int sh) {
    return sh >= 0 ? (long long)w << sh : (sh > -62 ? ((long long)w + (1ll << (-sh - 1))) >> (-sh) : 0ll);
}

#ifdef PIC_MIXED_MIN_BLOCKS
#define PIC_MIXED_BOUNDS __launch_bounds__(kMixedThreads, PIC_MIXED_MIN_BLOCKS)
#else
#define PIC_MIXED_BOUNDS __launch_bounds__(kMixedThreads)
#endif
__global__ void PIC_MIXED_BOUNDS k_push_mixed(StepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sNHoles, sNFront, sNMove;
    __shared__ double sRed[kMixedThreads / 32];
    __shared__ double sQ;
    __shared__ int sTileE;
    __shared__ float sInvQ;
    // two per-warp group buffers: the flush of one iteration's sums runs in the
    // next iteration, after their shared-memory atomics have completed
    __shared__ int sWarpAcc[kMixedThreads / 32][2][kGroups * kSlots];
    __shared__ int sSlotNode[kSlots];
    // queued segments: {stencil origin node, class bits, start x,y,z, end x,y,z}
    __shared__ float4 sQueue[kMixedThreads / 32][kQueue][2];
    const Grid &g = P.g;
    const int t = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    const int tk = t % g.ntz, tl = (t / g.ntz) % g.nty, ti = t / (g.ntz * g.nty);
    const int i0 = ti * g.tx, l0 = tl * g.ty, k0 = tk * g.tz;
    const int SX = g.tx + 2, SY = g.ty + 2, SZ = g.tz + 2;
    const int nn = SX * SY * SZ;
    // FP32 field tile as yz-quads first (16-byte aligned), then the fixed-point tile J
    float4 *sF = (float4 *)smem_raw;  // Ex Ey Ez Hx Hy Hz
    unsigned long long *sJ = (unsigned long long *)(sF + 6 * nn);
    int *sHoles = (int *)(sJ + 3 * nn);
    // the front-hole list of the compaction reuses the (then drained) queues
    int *sFront = (int *)&sQueue[0][0][0];
    int *wacc = &sWarpAcc[warp][0][0];
    if (threadIdx.x == 0) {
        // quantum of the fixed-point tile J (see fx_add): |contribution| < 1.0834 |m| per segment
        double bound = 0.0;
        for (int s = 0; s < P.nsp; s++) bound += 2.5 * fabs(P.sp[s].m) * (double)P.sp[s].tile_count[t];
        int e2;
        frexp(bound, &e2);
        sQ = ldexp(1.0, e2 - 62);
        sTileE = e2 - 62;  // tile quantum 2^(e2-62)
        sInvQ = (float)ldexp(1.0, 62 - e2);
    }
    for (int e = lane; e < 2 * kGroups * kSlots; e += 32) wacc[e] = 0;
    if (threadIdx.x < kSlots) {
        // slot -> tile-local node offset from a cell's stencil origin (local index 0,0,0)
        const int e = threadIdx.x;
        int comp, a, b, c;
        if (e < 18) { comp = 0; a = e / 9; b = (e / 3) % 3; c = e % 3; }
        else if (e < 36) { comp = 1; a = (e - 18) / 6; b = ((e - 18) / 3) % 2; c = (e - 18) % 3; }
        else { comp = 2; a = (e - 36) / 6; b = ((e - 36) / 2) % 3; c = (e - 36) % 2; }
        sSlotNode[e] = comp * nn + ((2 + a) * SY + (2 + b)) * SZ + (2 + c);
    }

    const float *const *E = (const float *const *)P.E;
    const float *const *H = (const float *const *)P.H;
    const float *Fsrc[6] = {E[0], E[1], E[2], H[0], H[1], H[2]};
    for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
        const int c = idx % SZ, b = (idx / SZ) % SY, a = idx / (SZ * SY);
        const int gi = i0 + a, gl = l0 + b, gk = k0 + c;
        // taps outside the staged tile or the field arrays are never read: 0
        const bool in00 = gi < g.NX && gl < g.NY && gk < g.NZ;
        const bool in01 = in00 && c + 1 < SZ && gk + 1 < g.NZ;
        const bool in10 = in00 && b + 1 < SY && gl + 1 < g.NY;
        const bool in11 = in01 && in10;
        const size_t n = in00 ? g.node(gi, gl, gk) : 0;
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const float *F = Fsrc[f];
            sF[f * nn + idx] = make_float4(in00 ? F[n] : 0.f, in01 ? F[n + 1] : 0.f, in10 ? F[n + g.pz] : 0.f,
                                           in11 ? F[n + g.pz + 1] : 0.f);
        }
        sJ[idx] = 0ull;
        sJ[nn + idx] = 0ull;
        sJ[2 * nn + idx] = 0ull;
    }
    __syncthreads();
    const float inv_q = sInvQ;
    const int tile_e = sTileE;
    const int slotA = sSlotNode[lane], slotB = lane < kSlots - 32 ? sSlotNode[32 + lane] : 0;
    float4(*queue)[2] = sQueue[warp];

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
        unsigned unsorted = 0;
        int qn = 0;  // segments in this warp's queue (warp-uniform)
        // deposit the queued segments [from, from + n), one per lane, into the tile J
        auto drain_range = [&](int from, int n) {
            if (lane < n) {
                const float4 a = queue[from + lane][0], b = queue[from + lane][1];
                const int cl = __float_as_int(a.y);
                const int iv[3] = {2 + (cl & 1), 2 + ((cl >> 1) & 1), 2 + ((cl >> 2) & 1)};
                const float qs[3] = {a.z, a.w, b.x}, qe[3] = {b.y, b.z, b.w};
                float v[12];
                pqr_mixed(iv, qs, qe, wx, wy, wz, v);
                const int nb = __float_as_int(a.x) + (iv[0] * SY + iv[1]) * SZ + iv[2];
#pragma unroll
                for (int q = 0; q < 12; q++) fx_addf(&sJ[contrib_node(q, nb, nn, SY, SZ)], v[q], inv_q);
            }
            __syncwarp();
        };
        auto drain = [&](int n) { drain_range(0, n); };
        auto drain_top32 = [&](int n) { drain_range(n - 32, 32); };
        // add the group sums of buffer buf (groups led by the lanes of lead, stencil
        // origins n0v, warp/tile quantum shift shv) into the tile J and clear them;
        // exact: both quanta are powers of two, the tile bound keeps the sum below 2^62
        auto flush_groups = [&](int *buf, unsigned lead, int n0v, int shv) {
            unsigned lm = lead;
            for (int gi = 0; gi < kGroups && lm; gi++) {
                const int ld = __ffs(lm) - 1;
                lm &= lm - 1;
                const int base = __shfl_sync(FULL, n0v, ld);
                int *wg = buf + gi * kSlots;
                int w = wg[lane];
                if (w) {
                    wg[lane] = 0;
                    const long long add = rescale(w, shv);
                    if (add) atomicAdd(&sJ[base + slotA], (unsigned long long)add);
                }
                if (lane < kSlots - 32) {
                    w = wg[32 + lane];
                    if (w) {
                        wg[32 + lane] = 0;
                        const long long add = rescale(w, shv);
                        if (add) atomicAdd(&sJ[base + slotB], (unsigned long long)add);
                    }
                }
            }
        };
        int gbuf = 0;  // buffer of this iteration's sums; the other one holds the pending ones
        unsigned pend_lead = 0;
        int pend_n0 = 0, pend_sh = 0;
        // warp-synchronous loop: every lane of a warp runs the same iterations;
        // the next particle is loaded before the current one is processed
        const int stride = blockDim.x;
        PartM nxt;
        nxt.cell = -1;
        if (warp * 32 + lane < count) nxt = load_part(S, start + warp * 32 + lane);
        for (int base = warp * 32; base < count; base += stride) {
            const int j = base + lane;
            const int slot = start + j;
            PartM cur = nxt;
            if (j + stride < count) nxt = load_part(S, slot + stride);
            bool active = j < count && cur.cell >= 0;
            int i = i0, l = l0, k = k0;
            if (active) {
                g.cell_ijk(cur.cell, i, l, k);
                if (i - i0 < 0 || i - i0 >= g.tx || l - l0 < 0 || l - l0 >= g.ty || k - k0 < 0 || k - k0 >= g.tz) {
                    bad |= ST_BADCELL;  // a bin entry outside its tile: never index the tile with it
                    active = false;
                    i = i0; l = l0; k = k0;
                }
            }
            // tile-local node of reference tile index (0,0,0): cell_local - 2
            const int n0 = ((i - i0 - 2) * SY + (l - l0 - 2)) * SZ + (k - k0 - 2);
            float xs[3] = {cur.x, cur.y, cur.z};
            if (!active) xs[0] = xs[1] = xs[2] = 0.25f;
            float pu = active ? cur.px : 0.f, pv = active ? cur.py : 0.f, pw = active ? cur.pz : 0.f;

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
                float rs = __fdividef(1.f, q1 + 1.f + q2 + q3);
                float pu1 = ((q1 + 1.f) * su + (q4 + bz) * sv + (q6 - by) * sw) * rs;
                float pv1 = ((q4 - bz) * su + (q2 + 1.f) * sv + (q5 + bx) * sw) * rs;
                float pw1 = ((q6 + by) * su + (q5 - bx) * sv + (q3 + 1.f) * sw) * rs;
                pu = pu1 + fEx * tau1;
                pv = pv1 + fEy * tau1;
                pw = pw1 + fEz * tau1;
            }
            float p2 = pu * pu + pv * pv + pw * pw;
            float ig = rsqrtf(p2 + 1.f);
            // a non-finite momentum component makes p^2 non-finite
            const bool finite = isfinite(p2);
            if (active && !finite) bad |= ST_NAN;
            // gamma - 1 = p^2 / (gamma + 1) = p^2 ig / (1 + ig), accumulated in FP64
            if (active) kin += M * (double)__fdividef(p2 * ig, 1.f + ig);
            float xe[3] = {xs[0] + ctx * (ig * pu), xs[1] + cty * (ig * pv), xs[2] + ctz * (ig * pw)};

            // ---- CurrentToMesh (cell.h:1306-1422) in cell units
            // cell-centre index of the end point from the same exact float
            // thresholds as i1 (x + 2.5 rounded in FP32 would put a point one
            // ulp below a centre plane on the far side of it)
            const int i1[3] = {i1x, i1y, i1z};
            int i2[3];
#pragma unroll
            for (int d = 0; d < 3; d++) i2[d] = 2 + (xe[d] >= 0.5f) + (xe[d] >= 1.5f) - (xe[d] < -0.5f);
            bool dep = active && finite;
            if (dep && (i2[0] < 2 || i2[0] > 3 || i2[1] < 2 || i2[1] > 3 || i2[2] < 2 || i2[2] > 3)) {
                bad |= ST_STENCIL;
                dep = false;
            }
            // warp quantum: 2^(ew-22) with 2^(ew-1) <= wmax < 2^ew, wmax the largest
            // contribution bound of the warp's lanes (1.0834 |current of the full
            // step|, redux.sync max).  Contributions then scale to |w| < 2^22, so the
            // FMA magic-number rounding below is exact, and 64 of them sum below 2^28.
            const float lb = dep ? 1.0834f * fmaxf(fabsf(wx * (xe[0] - xs[0])),
                                                   fmaxf(fabsf(wy * (xe[1] - xs[1])), fabsf(wz * (xe[2] - xs[2]))))
                                 : 0.f;
            const float wmax = __uint_as_float(__reduce_max_sync(FULL, __float_as_uint(lb)));
            const int ew = max(exponent_above(wmax), -100);
            const float inv_qw = pow2f(22 - ew);
            const int sh = ew - 22 - tile_e;  // warp quantum / tile quantum = 2^sh
            // one group per distinct cell among the depositing lanes
            const unsigned same = __match_any_sync(FULL, dep ? cur.cell : -1);
            const int leader = __ffs(same) - 1;
            const unsigned leaders = __ballot_sync(FULL, dep && lane == leader);
            const int grp = __popc(leaders & ((1u << leader) - 1));
            const bool fast = dep && grp < kGroups;
            unsorted += dep && !fast;
            // the second zigzag segment exists only where a cell-centre plane is crossed
            const bool cross = dep && (i2[0] != i1x || i2[1] != i1y || i2[2] != i1z);
            float x2[3] = {xe[0], xe[1], xe[2]};
            if (cross) split_point(i1, i2, xs, xe, x2);
            flush_groups(wacc + (gbuf ^ 1) * (kGroups * kSlots), pend_lead, pend_n0, pend_sh);
            if (fast) {
                float v[12];
                pqr_mixed(i1, xs, x2, wx, wy, wz, v);
                int *wb = wacc + gbuf * (kGroups * kSlots) + grp * kSlots;
                const int cx = i1x - 2, cy = i1y - 2, cz = i1z - 2;
                const int bx = cx * 9 + cy * 3 + cz, by = 18 + cx * 6 + cy * 3 + cz, bz = 36 + cx * 6 + cy * 2 + cz;
                const int off[12] = {bx, bx + 1, bx + 3, bx + 4, by, by + 1, by + 6, by + 7, bz, bz + 2, bz + 6, bz + 8};
#pragma unroll
                for (int q = 0; q < 12; q++) {
                    int w = __float_as_int(fmaf(v[q], inv_qw, 12582912.0f)) - 0x4B400000;  // round(v/q_w)
                    if (w) atomicAdd(&wb[off[q]], w);
                }
            }
            // queue the other segments (warp-aggregated positions)
            {
                const bool t1 = dep && !fast, t2 = cross;
                const unsigned b1 = __ballot_sync(FULL, t1), b2 = __ballot_sync(FULL, t2);
                const unsigned lt = (1u << lane) - 1;
                const int ntask = __popc(b1) + __popc(b2);
                if (ntask) {
                    if (qn + ntask > kQueue) {
                        drain(qn);
                        qn = 0;
                    }
                    int pos = qn + __popc(b1 & lt) + __popc(b2 & lt);
                    const float n0f = __int_as_float(n0);
                    if (t1) {
                        queue[pos][0] = make_float4(n0f, __int_as_float((i1x - 2) | ((i1y - 2) << 1) | ((i1z - 2) << 2)),
                                                    xs[0], xs[1]);
                        queue[pos][1] = make_float4(xs[2], x2[0], x2[1], x2[2]);
                        pos += t2;
                    }
                    if (t2) {
                        queue[pos][0] = make_float4(n0f, __int_as_float((i2[0] - 2) | ((i2[1] - 2) << 1) | ((i2[2] - 2) << 2)),
                                                    x2[0], x2[1]);
                        queue[pos][1] = make_float4(x2[2], xe[0], xe[1], xe[2]);
                    }
                    qn += ntask;
                    if (qn >= 32) {
                        __syncwarp();
                        drain_top32(qn);
                        qn -= 32;
                    }
                }
            }
            pend_lead = leaders;
            pend_n0 = n0;
            pend_sh = sh;
            gbuf ^= 1;
            __syncwarp();

            if (!active) continue;
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
            if ((unsigned)(ci[0] - i0) < (unsigned)g.tx && (unsigned)(ci[1] - l0) < (unsigned)g.ty &&
                (unsigned)(ci[2] - k0) < (unsigned)g.tz) {
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
        flush_groups(wacc + (gbuf ^ 1) * (kGroups * kSlots), pend_lead, pend_n0, pend_sh);
        __syncwarp();
        drain(qn);
        if (unsorted) atomicAdd(&P.st->unsorted[s], (unsigned long long)unsorted);
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
                    int mv = atomicAdd(&sNMove, 1);
                    if (mv >= sNFront) { bad |= ST_BADCELL; continue; }
                    int dst = start + sFront[mv];
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
        long long iv = (long long)sJ[idx];
        if (iv != 0) {
            int comp = idx / nn, r = idx % nn;
            int c = r % SZ, b = (r / SZ) % SY, a = r / (SZ * SY);
            if (i0 + a < g.NX && l0 + b < g.NY && k0 + c < g.NZ)
                atomicAdd(&P.J[comp][g.node(i0 + a, l0 + b, k0 + c)], (double)iv * sQ);
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

constexpr int kPlaneThreads = 256;
static inline dim3 plane_grid(const Grid &g) {
    return dim3((g.NY * g.NZ + kPlaneThreads - 1) / kPlaneThreads, g.NX);
}

void yee_b_half_mixed(const Grid &g, float *const E[3], float *const H[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    k_b_half_mixed<<<plane_grid(g), kPlaneThreads, 0, s>>>(g, E[0], E[1], E[2], H[0], H[1], H[2], cx, cy, cz);
}

void yee_e_update_mixed(const Grid &g, float *const E[3], float *const H[3], double *const J[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    k_e_update_mixed<<<plane_grid(g), kPlaneThreads, 0, s>>>(g, E[0], E[1], E[2], H[0], H[1], H[2], J[0], J[1], J[2], cx,
                                                     cy, cz, g.tau);
}

size_t push_smem_mixed(const Grid &g) {
    size_t nn = (size_t)(g.tx + 2) * (g.ty + 2) * (g.tz + 2);
    return 6 * nn * sizeof(float4) + 3 * nn * sizeof(unsigned long long) + kHoleMax * sizeof(int);
}

size_t push_smem_total_mixed(const Grid &g) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k_push_mixed) != cudaSuccess) return (size_t)-1;
    return push_smem_mixed(g) + a.sharedSizeBytes;
}

cudaError_t launch_push_mixed(const StepParams &p, cudaStream_t s) {
    size_t smem = push_smem_mixed(p.g);
    cudaError_t e = cudaFuncSetAttribute(k_push_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_push_mixed<<<p.g.ntiles, kMixedThreads, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace pic
