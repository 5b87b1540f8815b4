// Mixed form (FP32 with FP64 global current) kernels of the B200 PIC step.
//
// Same physics and stencils as the plain form (citations there and below),
// re-expressed in cell units so positions never lose resolution with the
// size of the box: a particle is (int32 cell, FP32 offset in [0,1) per axis,
// FP32 momentum).  Push, deposit and Yee run in FP32; the deposit
// pre-reduces each tile's current in shared memory (64-bit fixed point, see
// fx_add) and adds the tile into the global J in FP64.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <math.h>
#include <algorithm>
#include "pic_internal.cuh"
#include "pic_kernels.cuh"

namespace pic {
namespace {

constexpr float kOneBelow = 0.99999994f;  // largest float < 1

// ------------------------------------------------------------------ Yee --
// The element updates with every product and sum rounded on its own (no FMA
// contraction), so that every kernel forming them -- the B and E kernels and
// the push's staging of the half step -- gets the same bits.
// emh1_Element (kernels.cu:1052-1073): Q = 1/2 (c1 (a1 - b1) - c2 (a2 - b2))
__device__ __forceinline__ float q_half(float c1, float a1, float b1, float c2, float a2, float b2) {
    return __fmul_rn(0.5f, __fsub_rn(__fmul_rn(c1, __fsub_rn(a1, b1)), __fmul_rn(c2, __fsub_rn(a2, b2))));
}
// emeElement (kernels.cu:1091-1102): E + ((c1 (a1 - b1) - c2 (a2 - b2)) - tau J), tau J formed in FP64
__device__ __forceinline__ float e_step(float e, float c1, float a1, float b1, float c2, float a2, float b2, double tj) {
    return __fadd_rn(e, __fsub_rn(__fsub_rn(__fmul_rn(c1, __fsub_rn(a1, b1)), __fmul_rn(c2, __fsub_rn(a2, b2))),
                                  (float)tj));
}

// Four consecutive z nodes per thread, 128-bit loads and stores (rows start
// on 16 bytes: the z pitch is a multiple of 4), one x plane per blockIdx.y;
// the element arithmetic per node is unchanged.
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, const float v[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void un4(float4 a, float v[4]) { v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; }

// H += Q(E) in FP32 (emh1_Element, kernels.cu:1052-1073; used for both the
// half step and the completion, which adds the same Q again, kernels.cu:1024-1049).
// TWICE: both in one pass, H = (H + Q) + Q -- pic_step's completion, whose
// half step the push formed in shared memory only (the same bits as the two
// separate passes of the sub-step calls)
template <bool TWICE>
__global__ void k_b_half_mixed(Grid g, const float *__restrict__ Ex, const float *__restrict__ Ey,
                               const float *__restrict__ Ez, float *Hx, float *Hy, float *Hz, float cx, float cy,
                               float cz) {
    chain_enter();
    const int nq = g.pz / 4;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * nq) return;
    const int l = q / nq, k0 = (q - l * nq) * 4, i = blockIdx.y;
    const size_t n = g.node(i, l, k0);
    const size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
    float ex[5], ey[5], ez[4], hx[4], hy[4], hz[4], ezy[4] = {}, exy[4] = {}, ezx[4] = {}, eyx[4] = {};
    un4(ld4(Ex + n), ex); un4(ld4(Ey + n), ey); un4(ld4(Ez + n), ez);
    un4(ld4(Hx + n), hx); un4(ld4(Hy + n), hy); un4(ld4(Hz + n), hz);
    ex[4] = k0 + 4 < g.NZ ? Ex[n + 4] : 0.f;  // +z neighbour of the last node
    ey[4] = k0 + 4 < g.NZ ? Ey[n + 4] : 0.f;
    if (l + 1 < g.NY) { un4(ld4(Ez + n + sy), ezy); un4(ld4(Ex + n + sy), exy); }
    if (i + 1 < g.NX) { un4(ld4(Ez + n + sx), ezx); un4(ld4(Ey + n + sx), eyx); }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int k = k0 + j;
        if (i <= g.nx + 1 && l <= g.ny && k <= g.nz) {
            const float q = q_half(cz, ey[j + 1], ey[j], cy, ezy[j], ez[j]);
            hx[j] = __fadd_rn(hx[j], q);
            if (TWICE) hx[j] = __fadd_rn(hx[j], q);
        }
        if (i <= g.nx && l <= g.ny + 1 && k <= g.nz) {
            const float q = q_half(cx, ezx[j], ez[j], cz, ex[j + 1], ex[j]);
            hy[j] = __fadd_rn(hy[j], q);
            if (TWICE) hy[j] = __fadd_rn(hy[j], q);
        }
        if (i <= g.nx && l <= g.ny && k <= g.nz + 1) {
            const float q = q_half(cy, exy[j], ex[j], cx, eyx[j], ey[j]);
            hz[j] = __fadd_rn(hz[j], q);
            if (TWICE) hz[j] = __fadd_rn(hz[j], q);
        }
    }
    st4(Hx + n, hx); st4(Hy + n, hy); st4(Hz + n, hz);
}

// emeElement (kernels.cu:1091-1102) in FP32, tau*J formed in FP64
__global__ void k_e_update_mixed(Grid g, float *Ex, float *Ey, float *Ez, const float *__restrict__ Hx,
                                 const float *__restrict__ Hy, const float *__restrict__ Hz,
                                 const double *__restrict__ Jx, const double *__restrict__ Jy,
                                 const double *__restrict__ Jz, float cx, float cy, float cz, double tau) {
    chain_enter();
    const int nq = g.pz / 4;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NY * nq) return;
    const int l = q / nq, k0 = (q - l * nq) * 4, i = blockIdx.y;
    const size_t n = g.node(i, l, k0);
    const size_t sx = (size_t)g.NY * g.pz, sy = g.pz;
    float ex[4], ey[4], ez[4], hx[5], hy[5], hz[4], hzy[4] = {}, hxy[4] = {}, hzx[4] = {}, hyx[4] = {};
    un4(ld4(Ex + n), ex); un4(ld4(Ey + n), ey); un4(ld4(Ez + n), ez);
    // hx[0], hy[0]: the -z neighbour of the first node; hx[1..4]: the four nodes
    un4(ld4(Hx + n), hx + 1); un4(ld4(Hy + n), hy + 1); un4(ld4(Hz + n), hz);
    hx[0] = k0 > 0 ? Hx[n - 1] : 0.f;
    hy[0] = k0 > 0 ? Hy[n - 1] : 0.f;
    if (l >= 1) { un4(ld4(Hz + n - sy), hzy); un4(ld4(Hx + n - sy), hxy); }
    if (i >= 1) { un4(ld4(Hz + n - sx), hzx); un4(ld4(Hy + n - sx), hyx); }
    const double2 jx0 = *reinterpret_cast<const double2 *>(Jx + n), jx1 = *reinterpret_cast<const double2 *>(Jx + n + 2);
    const double2 jy0 = *reinterpret_cast<const double2 *>(Jy + n), jy1 = *reinterpret_cast<const double2 *>(Jy + n + 2);
    const double2 jz0 = *reinterpret_cast<const double2 *>(Jz + n), jz1 = *reinterpret_cast<const double2 *>(Jz + n + 2);
    const double jx[4] = {jx0.x, jx0.y, jx1.x, jx1.y}, jy[4] = {jy0.x, jy0.y, jy1.x, jy1.y},
                 jz[4] = {jz0.x, jz0.y, jz1.x, jz1.y};
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int k = k0 + j;
        if (i <= g.nx && l >= 1 && l <= g.ny && k >= 1 && k <= g.nz)
            ex[j] = e_step(ex[j], cy, hz[j], hzy[j], cz, hy[j + 1], hy[j], tau * jx[j]);
        if (i >= 1 && i <= g.nx && l <= g.ny && k >= 1 && k <= g.nz)
            ey[j] = e_step(ey[j], cz, hx[j + 1], hx[j], cx, hz[j], hzx[j], tau * jy[j]);
        if (i >= 1 && i <= g.nx && l >= 1 && l <= g.ny && k <= g.nz)
            ez[j] = e_step(ez[j], cx, hy[j + 1], hyx[j], cy, hx[j + 1], hxy[j], tau * jz[j]);
    }
    st4(Ex + n, ex); st4(Ey + n, ey); st4(Ez + n, ez);
}

// ------------------------------------------------------- particle push --
// Interpolate3D (cell.h:1054-1153) in cell units on the FP32 tile, stored as
// yz-quads: Q[n] = (T[n], T[n+dz], T[n+dy], T[n+dy+dz]), so the 8 taps are two
// 128-bit shared loads (the same products and sums, in the same order, as
// the 8 scalar taps).  Q points at the stencil's lower node; the upper x node
// is SYZ quads further; sx, sy, sz weight the lower node of each axis.
// The trilinear weights are applied with packed FP32x2 arithmetic
// (fma.rn.f32x2): x first on the (z lower, z upper) pairs of the lower and
// upper y rows, then y on the pair, then z.  w = (s, 1 - s) per axis, s
// weighting the lower node.
__device__ __forceinline__ float interp_quad2(const float4 *__restrict__ Q, int SYZ, float2 wx, float2 wy, float2 wz) {
    const float4 A = Q[0], B = Q[SYZ];
    const float2 ax = make_float2(wx.x, wx.x), bx = make_float2(wx.y, wx.y);
    const float2 r0 = __ffma2_rn(bx, make_float2(B.x, B.y), __fmul2_rn(ax, make_float2(A.x, A.y)));
    const float2 r1 = __ffma2_rn(bx, make_float2(B.z, B.w), __fmul2_rn(ax, make_float2(A.z, A.w)));
    const float2 r = __ffma2_rn(make_float2(wy.y, wy.y), r1, __fmul2_rn(make_float2(wy.x, wy.x), r0));
    return fmaf(wz.y, r.y, wz.x * r.x);
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

// pqr_mixed with the centre planes given as float offsets c_a = iv_a - 2.5
// (each -1/2 or +1/2: no integer-to-float conversions) and packed FP32x2
// arithmetic, each contribution rounded to an
// integer number of quanta: w[q] = round(v[q] / q_s), via the FMA magic
// number 1.5 * 2^23 (exact for |v / q_s| < 2^22).  inv_qs = 1 / q_s.
__device__ __forceinline__ void pqr_quant(const float cc[3], const float xs[3], const float xe[3], float wx, float wy,
                                          float wz, float inv_qs, int w[12]) {
    const float dx = 0.5f * (xs[0] + xe[0]) - cc[0];
    const float dy = 0.5f * (xs[1] + xe[1]) - cc[1];
    const float dz = 0.5f * (xs[2] + xe[2]) - cc[2];
    const float su = xe[0] - xs[0], sv = xe[1] - xs[1], sw = xe[2] - xs[2];
    const float r12 = 1.f / 12.f;
    const float s1 = sv * sw * r12, s2 = su * sw * r12, s3 = su * sv * r12;
    // per component: (lower, upper) weights of the two transverse axes
    const float2 DZ = make_float2(1.f - dz, dz), DY = make_float2(1.f - dy, dy);
    const float2 M = make_float2(12582912.0f, 12582912.0f);
    const float ax = su * wx * inv_qs, ay = sv * wy * inv_qs, az = sw * wz * inv_qs;
    float2 r[6];
    // Jx: su (dy1 dz1 + s1, dy1 dz - s1, dy dz1 - s1, dy dz + s1)
    r[0] = __ffma2_rn(make_float2(ax, ax), __ffma2_rn(make_float2(DY.x, DY.x), DZ, make_float2(s1, -s1)), M);
    r[1] = __ffma2_rn(make_float2(ax, ax), __ffma2_rn(make_float2(DY.y, DY.y), DZ, make_float2(-s1, s1)), M);
    // Jy: sv (dx1 dz1 + s2, dx1 dz - s2, dx dz1 - s2, dx dz + s2)
    r[2] = __ffma2_rn(make_float2(ay, ay), __ffma2_rn(make_float2(1.f - dx, 1.f - dx), DZ, make_float2(s2, -s2)), M);
    r[3] = __ffma2_rn(make_float2(ay, ay), __ffma2_rn(make_float2(dx, dx), DZ, make_float2(-s2, s2)), M);
    // Jz: sw (dx1 dy1 + s3, dx1 dy - s3, dx dy1 - s3, dx dy + s3)
    r[4] = __ffma2_rn(make_float2(az, az), __ffma2_rn(make_float2(1.f - dx, 1.f - dx), DY, make_float2(s3, -s3)), M);
    r[5] = __ffma2_rn(make_float2(az, az), __ffma2_rn(make_float2(dx, dx), DY, make_float2(-s3, s3)), M);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        w[2 * q] = __float_as_int(r[q].x) - 0x4B400000;
        w[2 * q + 1] = __float_as_int(r[q].y) - 0x4B400000;
    }
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
// x2 = xe: the second segment then has length 0 and adds nothing.  c[a]: the
// centre index changes along axis a.
__device__ __forceinline__ void split_point(const bool c[3], const float xs[3], const float xe[3], float x2[3]) {
    float num = 0.f, den = 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const float dl = xe[d] - xs[d];
        num += c[d] ? (0.5f - xs[d]) * dl : 0.f;
        den += c[d] ? dl * dl : 0.f;
    }
    const float sr = den > 0.f ? __fdividef(num, den) : 1.f;
#pragma unroll
    for (int d = 0; d < 3; d++) x2[d] = c[d] ? 0.5f : xs[d] + (xe[d] - xs[d]) * sr;
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

// ------------------------------------------------- tensor-memory staging --
// The CTA's field tile (6 components, tile + 2-node halo, plus one row in y
// and z for the quads) arrives by six 3D TMA loads (cp.async.bulk.tensor,
// no multicast: every tensor map covers this GPU's own field arrays) into a
// raw staging area, completing on one mbarrier.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, unsigned long long *bar, int c0,
                                            int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
// try_wait suspends for a bounded time per call; 2^20 calls bound the wait
// far above any real TMA latency, after which the CTA reports ST_TMA
constexpr int kTmaWaitLimit = 1 << 20;

// Deposit of the tile current, two levels:
//  1. the first zigzag segment of every particle goes, with native int32
//     shared-memory atomics, into a tile-sized int32 current that two warps
//     share (kJCopies per CTA).  Its quantum q_s = 2^e_s is static per
//     species: cmax bounds one contribution (twice the largest of the species
//     in the last push, or from its momenta before its first push; at most
//     the light-speed bound) and q_s >= 2^-22 cmax keeps the FMA
//     magic-number rounding of a contribution exact.  Each warp adds up, per
//     iteration, the bounds of its lanes' contributions (redux.sync): its
//     share of any node's int32 sum never exceeds that running total.  Before
//     the total could pass 2^30 the warp moves the current into the tile's
//     exact 64-bit fixed-point J (atomicExch, so the other warp's concurrent
//     adds are never lost; rescaled exactly: both quanta are powers of two)
//     and starts its total again at zero, so two warps' shares stay below
//     2^31.  At the end of the species the copies are summed per node into
//     the tile J.
//  2. the second segment of a particle that crosses a cell-centre plane
//     (1-4% of particles), and both segments of a particle whose contribution
//     bound exceeds cmax, are queued per warp and deposited 32 at a time, one
//     per lane, straight into the 64-bit tile J, so a few such lanes do not
//     stall the other lanes of their warp.
// No cell grouping: the bins need not be in cell order.
#ifndef PIC_MIXED_THREADS
#define PIC_MIXED_THREADS 256
#endif
#ifndef PIC_MIXED_MIN_BLOCKS
#define PIC_MIXED_MIN_BLOCKS 2
#endif
#ifndef PIC_MIXED_QUEUE
#define PIC_MIXED_QUEUE 64
#endif
constexpr int kMixedThreads = PIC_MIXED_THREADS;  // threads per CTA of k_push_mixed
constexpr int kMixedWarps = kMixedThreads / 32;
constexpr int kJCopies = kMixedWarps / 2;         // int32 tile currents per CTA: one per two warps
constexpr int kQueue = PIC_MIXED_QUEUE;           // queued segments per warp
constexpr unsigned kOutChunk = 16;                // outbox slots a warp takes from the global counter at once
static_assert(kMixedThreads % 32 == 0, "whole warps");
static_assert(kQueue >= 64, "one iteration can queue two segments per lane");

// w (in units of 2^e_w) -> units of 2^e_tile, sh = e_w - e_tile, round half up
__device__ __forceinline__ long long rescale(long long w, int sh) {
    return sh >= 0 ? w << sh : (sh > -62 ? (w + (1ll << (-sh - 1))) >> (-sh) : 0ll);
}

// shared-memory layout of k_push_mixed (dynamic part), byte offsets
struct MixedSmem {
    size_t raw, raw_e, raw_h, quads, jw, tilej, holes, total;
    // byte offset of component f (Ex Ey Ez Hx Hy Hz) in the raw staging area
    __host__ __device__ size_t raw_of(int f) const { return raw + (f < 3 ? f * raw_e : 3 * raw_e + (f - 3) * raw_h); }
};
__host__ __device__ inline size_t round_up_sz(size_t v, size_t a) { return (v + a - 1) / a * a; }
__host__ __device__ inline MixedSmem mixed_smem(int tx, int ty, int tz) {
    MixedSmem m;
    const size_t SX = tx + 2, SY = ty + 2, SZ = tz + 2, nn = SX * SY * SZ;
    // TMA boxes: the tile + halo plus one row in y and two in z for the quads;
    // E has one more x plane for the forward differences of the B half step
    const size_t box_e = (size_t)(tx + 3) * (ty + 3) * (tz + 4), box_h = (size_t)(tx + 2) * (ty + 3) * (tz + 4);
    m.raw_e = round_up_sz(box_e * sizeof(float), 128);
    m.raw_h = round_up_sz(box_h * sizeof(float), 128);
    const size_t raw_bytes = 3 * m.raw_e + 3 * m.raw_h;
    const size_t jw_bytes = (size_t)kJCopies * 3 * nn * sizeof(int);
    // the raw TMA staging area is consumed (into the quads) before the int32
    // currents are cleared, so the two share memory
    m.raw = 0;
    m.jw = 0;
    m.quads = round_up_sz(raw_bytes > jw_bytes ? raw_bytes : jw_bytes, 128);
    m.tilej = m.quads + 6 * nn * sizeof(float4);
    m.holes = m.tilej + 3 * nn * sizeof(unsigned long long);
    m.total = m.holes + 2 * kHoleMax * sizeof(int);  // holes, then the front holes
    return m;
}

#define PIC_MIXED_BOUNDS __launch_bounds__(kMixedThreads, PIC_MIXED_MIN_BLOCKS)
// TX, TY, TZ: the tile's cells per axis when fixed at compile time (shared-
// memory offsets become immediates), 0 to take them from the grid
template <int TX, int TY, int TZ>
__global__ void PIC_MIXED_BOUNDS k_push_mixed(const __grid_constant__ MixedMaps maps, StepParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long sBar;
    // hole-list counters in three sets by species (s mod 3), so that a species
    // needs no barrier before its loop: thread 0 clears the set of species s+1
    // before the end barrier of species s, after the last use of that set
    // (species s-2's compaction, before the end barrier of species s-1)
    __shared__ int sNHoles[3], sNFront[3], sNMove[3];
    __shared__ double sRed[kMixedWarps];
    __shared__ unsigned sLbMax[kMaxSpecies];
    __shared__ double sQ;
    __shared__ int sTileE;
    __shared__ float sInvQ;
    // queued segments: {stencil origin node, class bits, start x,y,z, end x,y,z}
    __shared__ float4 sQueue[kMixedWarps][kQueue][2];
    const Grid &g = P.g;
    const int tx = TX ? TX : g.tx, ty = TY ? TY : g.ty, tz = TZ ? TZ : g.tz;
    const int t = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    const unsigned lt = (1u << lane) - 1;
    const int tk = t % g.ntz, tl = (t / g.ntz) % g.nty, ti = t / (g.ntz * g.nty);
    const int i0 = ti * tx, l0 = tl * ty, k0 = tk * tz;
    const int SX = tx + 2, SY = ty + 2, SZ = tz + 2;
    const int SYZ = SY * SZ;
    const int nn = SX * SYZ;
    const int BY = ty + 3, BZ = tz + 4;
    const MixedSmem L = mixed_smem(tx, ty, tz);
    float4 *sF = (float4 *)(smem_raw + L.quads);  // Ex Ey Ez Hx Hy Hz as yz-quads
    unsigned long long *sJ = (unsigned long long *)(smem_raw + L.tilej);
    int *sJw = (int *)(smem_raw + L.jw);
    int *sHoles = (int *)(smem_raw + L.holes);
    int *sFront = sHoles + kHoleMax;  // the compaction's holes in front of the new count
    int *myJ = sJw + (warp % kJCopies) * 3 * nn;

    // a TMA destination starts on a 128-byte boundary (block-uniform check)
    if (smem_u32(smem_raw + L.raw) & 127u) {
        if (threadIdx.x == 0) atomicOr(&P.st->flags, ST_TMA);
        return;
    }
    if (threadIdx.x == 0) {
        // quantum of the fixed-point tile J (see fx_add): |contribution| < 1.0834 |m| per segment
        double bound = 0.0;
        for (int s = 0; s < P.nsp; s++) bound += 2.5 * fabs(P.sp[s].m) * (double)P.sp[s].tile_count[t];
        int e2;
        frexp(bound, &e2);
        sQ = ldexp(1.0, e2 - 62);
        sTileE = e2 - 62;  // tile quantum 2^(e2-62)
        sInvQ = (float)ldexp(1.0, 62 - e2);
        mbar_init(&sBar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned e_bytes = (unsigned)((size_t)(SX + 1) * BY * BZ * sizeof(float));
        const unsigned h_bytes = (unsigned)((size_t)SX * BY * BZ * sizeof(float));
        mbar_arrive_expect_tx(&sBar, 3 * e_bytes + 3 * h_bytes);
#pragma unroll
        for (int f = 0; f < 6; f++) tma_load_3d(smem_raw + L.raw_of(f), &maps.m[f], &sBar, k0, l0, i0);
    }
    for (int idx = threadIdx.x; idx < 3 * nn; idx += blockDim.x) sJ[idx] = 0ull;
    bool staged = false;
    for (int it = 0; it < kTmaWaitLimit && !(staged = mbar_try_wait(&sBar, 0)); it++) {
    }
    if (!__syncthreads_and(staged)) {
        if (threadIdx.x == 0) atomicOr(&P.st->flags, ST_TMA);
        return;
    }
    if (P.b_half) {
        // the B half step of the staged tile (pic_step leaves the full-step H
        // in memory): H += Q(E) on its ranges, at the nodes the quads read
        float *R[6];
#pragma unroll
        for (int f = 0; f < 6; f++) R[f] = (float *)(smem_raw + L.raw_of(f));
        const float bcx = (float)(g.tau / g.hx), bcy = (float)(g.tau / g.hy), bcz = (float)(g.tau / g.hz);
        const int sbx = BY * BZ;  // x stride of the raw boxes
        for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
            const int a = idx / SYZ, bc = idx - a * SYZ, b = bc / SZ, c = bc - b * SZ;
            const int gi = i0 + a, gl = l0 + b, gk = k0 + c;
            const int o = (a * BY + b) * BZ + c;
            if (gi <= g.nx + 1 && gl <= g.ny && gk <= g.nz)
                R[3][o] = __fadd_rn(R[3][o], q_half(bcz, R[1][o + 1], R[1][o], bcy, R[2][o + BZ], R[2][o]));
            if (gi <= g.nx && gl <= g.ny + 1 && gk <= g.nz)
                R[4][o] = __fadd_rn(R[4][o], q_half(bcx, R[2][o + sbx], R[2][o], bcz, R[0][o + 1], R[0][o]));
            if (gi <= g.nx && gl <= g.ny && gk <= g.nz + 1)
                R[5][o] = __fadd_rn(R[5][o], q_half(bcy, R[0][o + BZ], R[0][o], bcx, R[1][o + sbx], R[1][o]));
        }
        __syncthreads();
    }
    // raw [a][b][c] (c fastest, extents SX (+1 for E), BY, BZ) -> yz-quads
    // Q[n] = (T[n], T[n+dz], T[n+dy], T[n+dy+dz]); out-of-array taps arrive as 0
    for (int idx = threadIdx.x; idx < 6 * nn; idx += blockDim.x) {
        const int f = idx / nn, r = idx - f * nn;
        const int a = r / SYZ, bc = r - a * SYZ, b = bc / SZ, c = bc - b * SZ;
        const float *R = (const float *)(smem_raw + L.raw_of(f)) + (a * BY + b) * BZ + c;
        sF[idx] = make_float4(R[0], R[1], R[BZ], R[BZ + 1]);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kJCopies * 3 * nn; idx += blockDim.x) sJw[idx] = 0;
    if (threadIdx.x < kMaxSpecies) sLbMax[threadIdx.x] = 0u;
    if (threadIdx.x < 3) { sNHoles[threadIdx.x] = 0; sNFront[threadIdx.x] = 0; sNMove[threadIdx.x] = 0; }
    __syncthreads();
    const float inv_q = sInvQ;
    const int tile_e = sTileE;
    float4(*queue)[2] = sQueue[warp];

    const float ctx = (float)(g.tau / g.hx), cty = (float)(g.tau / g.hy), ctz = (float)(g.tau / g.hz);
    // packed cell index strides of x and y
    const int cstr_x = 1 << (g.by + g.bz), cstr_y = 1 << g.bz;
    // the tile's cells per axis inside the grid (the last tile of an axis can be
    // cut short): a step past them leaves the tile, periodically wrapped or not
    const int txe = min(tx, g.nx - i0), tye = min(ty, g.ny - l0), tze = min(tz, g.nz - k0);
    unsigned bad = 0;
    double kin = 0.0;
    unsigned long long moved = 0;
    OutMixed *outbox = (OutMixed *)P.outbox;
    // this warp's current outbox chunk [ob_base, ob_base + kOutChunk), ob_used
    // slots taken (warp-uniform); chunks come from the global counter
    unsigned ob_base = 0, ob_used = kOutChunk;
    bool ob_any = false;

    for (int s = 0; s < P.nsp; s++) {
        const SpeciesView &S = P.sp[s];
        const int sp = s % 3;  // hole-list counters of this species
        const int start = S.tile_start[t];
        const int count = S.tile_count[t];
        const float tau1 = (float)(S.q_m * g.tau * 0.5);
        const double M = S.m / S.q_m;
        // per-species deposit weights a*h/tau (see pqr_mixed)
        const float wx = (float)(S.m * g.hx / g.tau), wy = (float)(S.m * g.hy / g.tau), wz = (float)(S.m * g.hz / g.tau);
        // contribution bound of the int32 path: twice the last push's largest,
        // else the light-speed bound (|v| < c: |dx| < tau/h per axis)
        const float light = 1.0834f * fmaxf(fabsf(wx) * ctx, fmaxf(fabsf(wy) * cty, fabsf(wz) * ctz));
        const float prev = P.lb_prev ? P.lb_prev[s] : 0.f;
        const float cmax = prev > 0.f ? fminf(2.f * prev, light) : light;
        // int32 quantum 2^e_s >= 2^-22 cmax, per species: one quantum for
        // species of very different speeds would round the slow ones coarsely
        const int e_s = max(exponent_above(cmax * 0x1p-22f), -100);
        const float inv_qs = pow2f(-e_s);
        const int sh = e_s - tile_e;  // int32 quantum / tile quantum = 2^sh
        // running bound of this warp's share of any node's int32 sum, in quanta
        unsigned run = 0;
        auto flush_current = [&]() {
            __syncwarp();
            for (int idx = lane; idx < 3 * nn; idx += 32) {
                if (myJ[idx]) {
                    const int w = atomicExch(&myJ[idx], 0);
                    if (w) shared_add64(&sJ[idx], rescale(w, sh));
                }
            }
            __syncwarp();
        };
        int qn = 0;  // segments in this warp's queue (warp-uniform)
        float lbmax = 0.f;
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
                if ((unsigned)(i - i0) >= (unsigned)tx || (unsigned)(l - l0) >= (unsigned)ty ||
                    (unsigned)(k - k0) >= (unsigned)tz) {
                    bad |= ST_BADCELL;  // a bin entry outside its tile: never index the tile with it
                    active = false;
                    i = i0; l = l0; k = k0;
                }
            }
            // tile-local node of the particle's cell and of reference tile index (0,0,0)
            const int lc = ((i - i0) * SY + (l - l0)) * SZ + (k - k0);
            const int n0 = lc - 2 * (SYZ + SZ + 1);
            float xs[3] = {cur.x, cur.y, cur.z};
            if (!active) xs[0] = xs[1] = xs[2] = 0.25f;
            float pu = active ? cur.px : 0.f, pv = active ? cur.py : 0.f, pw = active ? cur.pz : 0.f;

            // ---- GetField (cell.h:1257-1290) in cell units: getCellNumber = 2,
            // getCellNumberCenter = 2 + (offset >= 1/2), weights s1 = 1-o, s2 = 1/2-o (+1)
            const int cx = xs[0] >= 0.5f, cy = xs[1] >= 0.5f, cz = xs[2] >= 0.5f;
            // centre offsets iv - 2.5 of the particle's cell-centre cell (+-1/2)
            const float cc[3] = {cx ? 0.5f : -0.5f, cy ? 0.5f : -0.5f, cz ? 0.5f : -0.5f};
            // (lower-node weight, upper-node weight) per axis: node-centred n, cell-centred c
            const float2 nx = make_float2(1.f - xs[0], xs[0]), ny = make_float2(1.f - xs[1], xs[1]),
                         nz = make_float2(1.f - xs[2], xs[2]);
            // cell-centred lower weight s2 = (1/2 or 3/2) - o = 1 + c - o (getCellNumberCenter)
            const float2 kx = make_float2(1.f + cc[0] - xs[0], xs[0] - cc[0]),
                         ky = make_float2(1.f + cc[1] - xs[1], xs[1] - cc[1]),
                         kz = make_float2(1.f + cc[2] - xs[2], xs[2] - cc[2]);
            const int ox = cx * SYZ, oy = cy * SZ, oz = cz;
            float fEx = interp_quad2(sF + lc + oy + oz, SYZ, nx, ky, kz);
            float fEy = interp_quad2(sF + nn + lc + ox + oz, SYZ, kx, ny, kz);
            float fEz = interp_quad2(sF + 2 * nn + lc + ox + oy, SYZ, kx, ky, nz);
            float fHx = interp_quad2(sF + 3 * nn + lc + ox, SYZ, kx, ny, nz);
            float fHy = interp_quad2(sF + 4 * nn + lc + oy, SYZ, nx, ky, nz);
            float fHz = interp_quad2(sF + 5 * nn + lc + oz, SYZ, nx, ny, kz);

            // ---- Particle::Move (particle.h:65-202), FP32: the half electric
            // kick, the magnetic rotation, the second half kick.  The reference
            // writes the rotation as the matrix (I + b b^T + [b]x) / (1 + b^2)
            // applied to p + p x b; here it is the algebraically identical
            // two-cross-product form p+ = p + (p + p x b) x (2 b / (1 + b^2)),
            // with fewer operations
            pu += tau1 * fEx;
            pv += tau1 * fEy;
            pw += tau1 * fEz;
            float ps = tau1 * rsqrtf(pu * pu + pv * pv + pw * pw + 1.f);
            {
                const float bx = ps * fHx, by = ps * fHy, bz = ps * fHz;
                const float f = __fdividef(2.f, 1.f + bx * bx + by * by + bz * bz);
                const float su = pu + (pv * bz - pw * by);
                const float sv = pv + (pw * bx - pu * bz);
                const float sw = pw + (pu * by - pv * bx);
                pu += f * (sv * bz - sw * by) + fEx * tau1;
                pv += f * (sw * bx - su * bz) + fEy * tau1;
                pw += f * (su * by - sv * bx) + fEz * tau1;
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
            // cell-centre class of the end point from the same exact float
            // thresholds as the start's (x + 2.5 rounded in FP32 would put a
            // point one ulp below a centre plane on the far side of it); the
            // stencil holds -1/2 <= xe < 3/2 per axis (centre index 2 or 3)
            bool ge[3], crs[3], inside = true;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                ge[d] = xe[d] >= 0.5f;
                inside = inside && xe[d] >= -0.5f && xe[d] < 1.5f;
            }
            crs[0] = ge[0] != (bool)cx;
            crs[1] = ge[1] != (bool)cy;
            crs[2] = ge[2] != (bool)cz;
            bool dep = active && finite;
            if (dep && !inside) {
                bad |= ST_STENCIL;
                dep = false;
            }
            // contribution bound of this particle (1.0834 |current of the full step|)
            const float lb = dep ? 1.0834f * fmaxf(fabsf(wx * (xe[0] - xs[0])),
                                                   fmaxf(fabsf(wy * (xe[1] - xs[1])), fabsf(wz * (xe[2] - xs[2]))))
                                 : 0.f;
            lbmax = fmaxf(lbmax, lb);
            const bool fast = dep && lb <= cmax;
            {
                // |round(v/q_s)| <= lb/q_s + 1/2 per contribution, one contribution per node and lane
                const unsigned add = __reduce_add_sync(FULL, fast ? (unsigned)(lb * inv_qs) + 1u : 0u);
                if (run + add > 0x40000000u) {
                    flush_current();
                    run = 0;
                }
                run += add;
            }
            // the second zigzag segment exists only where a cell-centre plane is crossed
            const bool cross = dep && (crs[0] || crs[1] || crs[2]);
            float x2[3] = {xe[0], xe[1], xe[2]};
            if (cross) split_point(crs, xs, xe, x2);
            if (fast) {
                int w[12];
                pqr_quant(cc, xs, x2, wx, wy, wz, inv_qs, w);
                // Jx (0,0,0) (0,0,1) (0,1,0) (0,1,1); Jy (0,0,0) (0,0,1) (1,0,0) (1,0,1);
                // Jz (0,0,0) (0,1,0) (1,0,0) (1,1,0) from the base node iv = i1
                int *J = myJ + lc + ox + oy + oz;
                const int off[12] = {0, 1, SZ, SZ + 1, nn, nn + 1, nn + SYZ, nn + SYZ + 1,
                                     2 * nn, 2 * nn + SZ, 2 * nn + SYZ, 2 * nn + SYZ + SZ};
#pragma unroll
                for (int q = 0; q < 12; q++) atomicAdd(J + off[q], w[q]);
            }
            // queue the other segments (warp-aggregated positions)
            {
                const bool t1 = dep && !fast, t2 = cross;
                const unsigned b1 = __ballot_sync(FULL, t1), b2 = __ballot_sync(FULL, t2);
                const int ntask = __popc(b1) + __popc(b2);
                if (ntask) {
                    if (qn + ntask > kQueue) {
                        drain_range(0, qn);
                        qn = 0;
                    }
                    int pos = qn + __popc(b1 & lt) + __popc(b2 & lt);
                    const float n0f = __int_as_float(n0);
                    if (t1) {
                        queue[pos][0] = make_float4(n0f, __int_as_float(cx | (cy << 1) | (cz << 2)), xs[0], xs[1]);
                        queue[pos][1] = make_float4(xs[2], x2[0], x2[1], x2[2]);
                        pos += t2;
                    }
                    if (t2) {
                        queue[pos][0] = make_float4(n0f, __int_as_float((int)ge[0] | ((int)ge[1] << 1) | ((int)ge[2] << 2)),
                                                    x2[0], x2[1]);
                        queue[pos][1] = make_float4(x2[2], xe[0], xe[1], xe[2]);
                    }
                    qn += ntask;
                    if (qn >= 32) {
                        __syncwarp();
                        drain_range(qn - 32, 32);
                        qn -= 32;
                    }
                }
            }

            // ---- new cell (Reflect cell.h:1427-1478 and migration, in cell units):
            // per axis a step of -1, 0 or +1 cell; a particle that stays in its
            // tile cannot wrap, so its packed cell index moves by the steps
            int dl[3];
            float xw[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const bool up = xe[d] >= 1.f, dn = xe[d] < 0.f;
                dl[d] = (int)up - (int)dn;
                xw[d] = fminf(fmaxf(xe[d] + (up ? -1.f : (dn ? 1.f : 0.f)), 0.f), kOneBelow);
            }
            const bool stay = (unsigned)(i - i0 + dl[0]) < (unsigned)txe && (unsigned)(l - l0 + dl[1]) < (unsigned)tye &&
                              (unsigned)(k - k0 + dl[2]) < (unsigned)tze;
            if (active && stay) {
                S.cell[slot] = cur.cell + dl[0] * cstr_x + dl[1] * cstr_y + dl[2];
                S.ox[slot] = xw[0]; S.oy[slot] = xw[1]; S.oz[slot] = xw[2];
                S.fx[slot] = pu; S.fy[slot] = pv; S.fz[slot] = pw;
            }
            // leavers: outbox slots from the warp's chunk (a new run of chunks
            // from the global counter only when it is used up) and one
            // hole-list reservation per warp
            const bool leave = active && !stay;
            const unsigned lm = __ballot_sync(FULL, leave);
            if (lm) {
                const int nl = __popc(lm), rank = __popc(lm & lt);
                int hbase = 0;
                if (lane == 0) hbase = atomicAdd(&sNHoles[sp], nl);
                hbase = __shfl_sync(FULL, hbase, 0);
                const unsigned room = kOutChunk - ob_used;
                unsigned nb = 0;
                if ((unsigned)nl > room) {
                    const unsigned need = ((unsigned)nl - room + kOutChunk - 1) / kOutChunk;
                    if (lane == 0) nb = atomicAdd(&P.st->out_count, need * kOutChunk);
                    nb = __shfl_sync(FULL, nb, 0);
                }
                // leaver `rank` takes the room left in the chunk, then the new chunks
                const unsigned e = (unsigned)rank < room ? ob_base + ob_used + rank : nb + (rank - room);
                if ((unsigned)nl > room) {
                    const unsigned over = (unsigned)nl - room;
                    ob_base = nb + (over - 1) / kOutChunk * kOutChunk;
                    ob_used = over - (over - 1) / kOutChunk * kOutChunk;
                    ob_any = true;
                } else {
                    ob_used += nl;
                }
                if (leave) {
                    // the new cell, wrapped periodically
                    int ci[3] = {i + dl[0], l + dl[1], k + dl[2]};
                    const int nc[3] = {g.nx, g.ny, g.nz};
#pragma unroll
                    for (int d = 0; d < 3; d++) ci[d] = ci[d] == nc[d] ? 0 : (ci[d] < 0 ? nc[d] - 1 : ci[d]);
                    if (e < P.out_cap) {
                        OutMixed o;
                        o.ox = xw[0]; o.oy = xw[1]; o.oz = xw[2]; o.px = pu; o.py = pv; o.pz = pw;
                        o.cell = g.cell_of(ci[0], ci[1], ci[2]);
                        o.species = s;
                        outbox[e] = o;
                        moved++;
                    } else {
                        bad |= ST_OUTBOX;
                    }
                    S.cell[slot] = -1;
                    const int hpos = hbase + rank;
                    if (hpos < kHoleMax) sHoles[hpos] = j;
                    else bad |= ST_HOLES;
                }
            }
        }
        __syncwarp();
        drain_range(0, qn);
        // the species' largest contribution bound, for the next push's quantum
        lbmax = __uint_as_float(__reduce_max_sync(FULL, __float_as_uint(lbmax)));
        if (lane == 0 && lbmax > 0.f) atomicMax(&sLbMax[s], __float_as_uint(lbmax));
        if (threadIdx.x == 0) {
            const int nx3 = (s + 1) % 3;
            sNHoles[nx3] = 0; sNFront[nx3] = 0; sNMove[nx3] = 0;
        }
        __syncthreads();
        // int32 currents of the species -> exact 64-bit tile J; clear them
        for (int idx = threadIdx.x; idx < 3 * nn; idx += blockDim.x) {
            long long sum = 0;
#pragma unroll
            for (int c = 0; c < kJCopies; c++) {
                sum += sJw[c * 3 * nn + idx];
                sJw[c * 3 * nn + idx] = 0;
            }
            if (sum) sJ[idx] += (unsigned long long)rescale(sum, sh);
        }
        // compaction: the last live particles of the bin move into the holes in
        // front of the new count
        const int nh = sNHoles[sp];
        if (nh > 0 && nh <= kHoleMax) {
            const int newcount = count - nh;
            for (int r = threadIdx.x; r < nh; r += blockDim.x) {
                int h = sHoles[r];
                if (h < newcount) sFront[atomicAdd(&sNFront[sp], 1)] = h;
            }
            __syncthreads();
            for (int r = threadIdx.x; r < nh; r += blockDim.x) {
                int src = start + newcount + r;
                if (S.cell[src] >= 0) {
                    int mv = atomicAdd(&sNMove[sp], 1);
                    if (mv >= sNFront[sp]) { bad |= ST_BADCELL; continue; }
                    int dst = start + sFront[mv];
                    S.cell[dst] = S.cell[src];
                    S.ox[dst] = S.ox[src]; S.oy[dst] = S.oy[src]; S.oz[dst] = S.oz[src];
                    S.fx[dst] = S.fx[src]; S.fy[dst] = S.fy[src]; S.fz[dst] = S.fz[src];
                }
            }
            if (threadIdx.x == 0) S.tile_count[t] = newcount;
        }
        // the next species adds into the cleared int32 currents
        __syncthreads();
    }
    if (threadIdx.x < P.nsp && P.lb_cur && sLbMax[threadIdx.x]) atomicMax(&P.lb_cur[threadIdx.x], sLbMax[threadIdx.x]);
    __syncthreads();

    // the unused slots of this warp's last outbox chunk: empty entries
    if (ob_any && lane < kOutChunk - ob_used && ob_base + ob_used + lane < P.out_cap)
        outbox[ob_base + ob_used + lane].cell = -1;
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

// Contribution bound of a species from its current momenta, for the first
// push after a load: 1.0834 max over particles and axes of |w_a| (tau/h_a)
// |p_a| / gamma (the bound of a full step at the current velocity), as float
// bits into *out (atomicMax)
__global__ void k_contribution_bound(SpeciesView S, int n, float wx, float wy, float wz, float ctx, float cty,
                                     float ctz, unsigned *out) {
    float m = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (S.cell[i] < 0) continue;
        const float pu = S.fx[i], pv = S.fy[i], pw = S.fz[i];
        const float ig = rsqrtf(pu * pu + pv * pv + pw * pw + 1.f);
        const float b = fmaxf(fabsf(wx) * ctx * fabsf(pu), fmaxf(fabsf(wy) * cty * fabsf(pv), fabsf(wz) * ctz * fabsf(pw)));
        m = fmaxf(m, 1.0834f * b * ig);
    }
    m = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m)));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));
}

}  // namespace

cudaError_t contribution_bound_mixed(const Grid &g, const SpeciesView &S, int64_t cap, unsigned *out, cudaStream_t s) {
    if (cap <= 0) return cudaSuccess;
    const float ctx = (float)(g.tau / g.hx), cty = (float)(g.tau / g.hy), ctz = (float)(g.tau / g.hz);
    const float wx = (float)(S.m * g.hx / g.tau), wy = (float)(S.m * g.hy / g.tau), wz = (float)(S.m * g.hz / g.tau);
    const int blocks = (int)std::min<int64_t>((cap + 255) / 256, 148 * 8);
    k_contribution_bound<<<blocks, 256, 0, s>>>(S, (int)cap, wx, wy, wz, ctx, cty, ctz, out);
    return cudaGetLastError();
}

constexpr int kPlaneThreads = 256;
// one thread per four z nodes of an x plane
static inline dim3 plane_grid(const Grid &g) {
    return dim3((g.NY * (g.pz / 4) + kPlaneThreads - 1) / kPlaneThreads, g.NX);
}

void yee_b_half_mixed(const Grid &g, float *const E[3], float *const H[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    launch_chained(k_b_half_mixed<false>, plane_grid(g), dim3(kPlaneThreads), s, g, E[0], E[1], E[2], H[0], H[1], H[2],
                   cx, cy, cz);
}

void yee_b_both_mixed(const Grid &g, float *const E[3], float *const H[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    launch_chained(k_b_half_mixed<true>, plane_grid(g), dim3(kPlaneThreads), s, g, E[0], E[1], E[2], H[0], H[1], H[2],
                   cx, cy, cz);
}

void yee_e_update_mixed(const Grid &g, float *const E[3], float *const H[3], double *const J[3], cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    launch_chained(k_e_update_mixed, plane_grid(g), dim3(kPlaneThreads), s, g, E[0], E[1], E[2], H[0], H[1], H[2], J[0],
                   J[1], J[2], cx, cy, cz, g.tau);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

cudaError_t encode_field_maps(const Grid &g, float *const E[3], float *const H[3], MixedMaps *maps) {
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return cudaErrorNotSupported;
    // {z, y, x}: z rows of pitch pz floats (a multiple of 4: 16-byte strides);
    // box = tile + halo, z rounded up to whole 16-byte units; the tile's first
    // z node k0 is a multiple of tz (a multiple of 4), so every box starts on
    // a 16-byte boundary
    const cuuint64_t dims[3] = {(cuuint64_t)g.NZ, (cuuint64_t)g.NY, (cuuint64_t)g.NX};
    const cuuint64_t strides[2] = {(cuuint64_t)g.pz * sizeof(float), (cuuint64_t)g.pz * g.NY * sizeof(float)};
    // E has one more x plane (the forward differences of the B half step)
    const cuuint32_t box_e[3] = {(cuuint32_t)(g.tz + 4), (cuuint32_t)(g.ty + 3), (cuuint32_t)(g.tx + 3)};
    const cuuint32_t box_h[3] = {(cuuint32_t)(g.tz + 4), (cuuint32_t)(g.ty + 3), (cuuint32_t)(g.tx + 2)};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (g.tz % 4 != 0 || box_e[0] > 256 || box_e[1] > 256 || box_e[2] > 256) return cudaErrorInvalidValue;
    float *const src[6] = {E[0], E[1], E[2], H[0], H[1], H[2]};
    for (int f = 0; f < 6; f++) {
        CUresult r = encode(&maps->m[f], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)src[f], dims, strides,
                            f < 3 ? box_e : box_h, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

size_t push_smem_mixed(const Grid &g) { return mixed_smem(g.tx, g.ty, g.tz).total; }

using PushMixedFn = void (*)(const MixedMaps, StepParams);
// the instantiation for a grid's tile: fixed dimensions for the automatic tiles, else runtime
static PushMixedFn push_mixed_fn(const Grid &g) {
    if (g.tx == 6 && g.ty == 4 && g.tz == 8) return k_push_mixed<6, 4, 8>;
    if (g.tx == 6 && g.ty == 4 && g.tz == 4) return k_push_mixed<6, 4, 4>;
    if (g.tx == 4 && g.ty == 4 && g.tz == 12) return k_push_mixed<4, 4, 12>;
    if (g.tx == 4 && g.ty == 4 && g.tz == 8) return k_push_mixed<4, 4, 8>;
    if (g.tx == 4 && g.ty == 4 && g.tz == 4) return k_push_mixed<4, 4, 4>;
    return k_push_mixed<0, 0, 0>;
}

size_t push_smem_total_mixed(const Grid &g) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, push_mixed_fn(g)) != cudaSuccess) return (size_t)-1;
    return push_smem_mixed(g) + a.sharedSizeBytes;
}

cudaError_t launch_push_mixed(const StepParams &p, const MixedMaps &maps, cudaStream_t s) {
    const PushMixedFn fn = push_mixed_fn(p.g);
    size_t smem = push_smem_mixed(p.g);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<p.g.ntiles, kMixedThreads, smem, s>>>(maps, p);
    return cudaGetLastError();
}

}  // namespace pic
