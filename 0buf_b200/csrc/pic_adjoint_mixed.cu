// Differentiable run of the FP32 mixed form: the fixed-order push and the
// adjoint particle kernels.  Same arithmetic as k_push_mixed (cell units,
// FP32 offsets and momenta, rsqrtf), with the current added straight into the
// FP64 global J; the adjoint runs in FP32 per particle and adds into FP64
// field adjoints.  Field transposes and the host sequence: pic_adjoint.cu.
#include <cuda_runtime.h>
#include <math.h>
#include "pic0buf.h"
#include "pic_internal.cuh"
#include "pic_handle.cuh"
#include "pic_adjoint.cuh"

namespace pic {

namespace {

constexpr int kT = 256;
constexpr float kOneBelow = 0.99999994f;  // largest float < 1

// see spread_index in pic_adjoint.cu: lane quads take 4 consecutive particles,
// the 8 quads of a warp sit 32 particles apart (about 8 different cells)
__device__ __forceinline__ int64_t spread_index(int t) {
    return (int64_t)blockIdx.x * kT + ((t & 31) >> 2) * 32 + (t >> 5) * 4 + (t & 3);
}
__device__ __forceinline__ int species_of(const int64_t *off, int nsp, int64_t idx) {
    int s = 0;
    while (s + 1 < nsp && idx >= off[s + 1]) s++;
    return s;
}

// GetField in cell units (k_push_mixed): the node-staggered tap is 2 with
// weight 1 - o, the centre-staggered tap 2 + (o >= 1/2) with weight
// (1/2 or 3/2) - o; component c is node-staggered along d when
// (E_c and d == c) or (H_c and d != c)
struct MTaps {
    int tc[3];
    float wn[3], wc[3];
};
__device__ __forceinline__ void taps_mixed(const float x[3], MTaps &T) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
        T.tc[d] = 2 + (x[d] >= 0.5f);
        T.wn[d] = 1.f - x[d];
        T.wc[d] = (T.tc[d] == 2 ? 0.5f : 1.5f) - x[d];
    }
}
__device__ __forceinline__ void comp_taps_m(const MTaps &T, int c, int t[3], float w[3]) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
        bool nd = c < 3 ? d == c : d != c - 3;
        t[d] = nd ? 2 : T.tc[d];
        w[d] = nd ? T.wn[d] : T.wc[d];
    }
}
__device__ __forceinline__ size_t tap_node(const Grid &g, int i, int l, int k, const int t[3]) {
    return g.node(i + t[0] - 2, l + t[1] - 2, k + t[2] - 2);
}
// interp_mixed's expression order
__device__ __forceinline__ float interp_gm(const float *__restrict__ A, size_t n, size_t dx, size_t dy,
                                           const float w[3]) {
    const size_t dz = 1;
    float sx = w[0], sy = w[1], sz = w[2];
    float sx1 = 1.f - sx, sy1 = 1.f - sy, sz1 = 1.f - sz;
    float t1 = sx * (sy * (sz * A[n] + sz1 * A[n + dz]) + sy1 * (sz * A[n + dy] + sz1 * A[n + dy + dz]));
    float t2 = sx1 * (sy * (sz * A[n + dx] + sz1 * A[n + dx + dz]) + sy1 * (sz * A[n + dx + dy] + sz1 * A[n + dx + dy + dz]));
    return t1 + t2;
}
__device__ __forceinline__ void gather_fields_m(const Grid &g, const float *const E[3], const float *const H[3],
                                                int i, int l, int k, const float x[3], float F[6]) {
    MTaps T;
    taps_mixed(x, T);
    const size_t dx = (size_t)g.NY * g.pz, dy = g.pz;
#pragma unroll
    for (int c = 0; c < 6; c++) {
        int t[3];
        float w[3];
        comp_taps_m(T, c, t, w);
        F[c] = interp_gm(c < 3 ? E[c] : H[c - 3], tap_node(g, i, l, k, t), dx, dy, w);
    }
}

// Particle::Move in FP32 as in k_push_mixed, with the adjoint's intermediates
struct BorisM {
    float t, u[3], g1, ps, b[3], s[3], rs, up[3], pp[3], ig, ct[3], xe[3];
};
__device__ __forceinline__ void boris_mixed(float tau1, const float ct[3], const float p[3], const float F[6],
                                            const float xs[3], BorisM &B) {
    B.t = tau1;
    float pu = p[0], pv = p[1], pw = p[2];
    pu += tau1 * F[0];
    pv += tau1 * F[1];
    pw += tau1 * F[2];
    B.u[0] = pu; B.u[1] = pv; B.u[2] = pw;
    B.g1 = rsqrtf(pu * pu + pv * pv + pw * pw + 1.f);
    float ps = tau1 * B.g1;
    B.ps = ps;
    float bx = ps * F[3], by = ps * F[4], bz = ps * F[5];
    B.b[0] = bx; B.b[1] = by; B.b[2] = bz;
    float su = pu + pv * bz - pw * by;
    float sv = pv + pw * bx - pu * bz;
    float sw = pw + pu * by - pv * bx;
    B.s[0] = su; B.s[1] = sv; B.s[2] = sw;
    float q1 = bx * bx, q2 = by * by, q3 = bz * bz, q4 = bx * by, q5 = by * bz, q6 = bz * bx;
    float rs = 1.f / (q1 + 1.f + q2 + q3);
    B.rs = rs;
    float pu1 = ((q1 + 1.f) * su + (q4 + bz) * sv + (q6 - by) * sw) * rs;
    float pv1 = ((q4 - bz) * su + (q2 + 1.f) * sv + (q5 + bx) * sw) * rs;
    float pw1 = ((q6 + by) * su + (q5 - bx) * sv + (q3 + 1.f) * sw) * rs;
    B.up[0] = pu1; B.up[1] = pv1; B.up[2] = pw1;
    pu = pu1 + F[0] * tau1;
    pv = pv1 + F[1] * tau1;
    pw = pw1 + F[2] * tau1;
    B.pp[0] = pu; B.pp[1] = pv; B.pp[2] = pw;
    B.ig = rsqrtf(pu * pu + pv * pv + pw * pw + 1.f);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        B.ct[d] = ct[d];
        B.xe[d] = xs[d] + ct[d] * (B.ig * B.pp[d]);
    }
}

// cell-centre crossings and the split point (split_point in pic_mixed.cu)
struct SplitM {
    int m, i1[3], i2[3];
    float x2[3], sr;
};
__device__ __forceinline__ void split_mixed(const float xs[3], const float xe[3], SplitM &S) {
    float num = 0.f, den = 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        S.i1[d] = 2 + (xs[d] >= 0.5f);
        S.i2[d] = 2 + (xe[d] >= 0.5f) + (xe[d] >= 1.5f) - (xe[d] < -0.5f);
        float dl = xe[d] - xs[d];
        bool c = S.i1[d] != S.i2[d];
        num += c ? (0.5f - xs[d]) * dl : 0.f;
        den += c ? dl * dl : 0.f;
    }
    S.m = 4 * (S.i1[0] != S.i2[0]) + 2 * (S.i1[1] != S.i2[1]) + (S.i1[2] != S.i2[2]);
    const bool any = den > 0.f;
    const float sr = any ? __fdividef(num, den) : 1.f;
    S.sr = sr;
#pragma unroll
    for (int d = 0; d < 3; d++) S.x2[d] = (S.i1[d] != S.i2[d]) ? 0.5f : xs[d] + (xe[d] - xs[d]) * sr;
}
__device__ __forceinline__ bool stencil_ok(const int iv[3]) {
    return iv[0] >= 2 && iv[0] <= 3 && iv[1] >= 2 && iv[1] <= 3 && iv[2] >= 2 && iv[2] <= 3;
}

// pqr_mixed (pic_mixed.cu) into the FP64 global J
__device__ __forceinline__ void seg_mixed(double *const J[3], const Grid &g, int ci, int cl, int ck, const int iv[3],
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
    if (su == 0.f && sv == 0.f && sw == 0.f) return;
    size_t n = tap_node(g, ci, cl, ck, iv);
    const size_t ez = 1, ey = g.pz, ex = (size_t)g.NY * g.pz;
    double *Jx = J[0], *Jy = J[1], *Jz = J[2];
    atomicAdd(&Jx[n], (double)(su * (dy1 * dz1 + s1)));
    atomicAdd(&Jx[n + ez], (double)(su * (dy1 * dz - s1)));
    atomicAdd(&Jx[n + ey], (double)(su * (dy * dz1 - s1)));
    atomicAdd(&Jx[n + ey + ez], (double)(su * (dy * dz + s1)));
    atomicAdd(&Jy[n], (double)(sv * (dx1 * dz1 + s2)));
    atomicAdd(&Jy[n + ez], (double)(sv * (dx1 * dz - s2)));
    atomicAdd(&Jy[n + ex], (double)(sv * (dx * dz1 - s2)));
    atomicAdd(&Jy[n + ex + ez], (double)(sv * (dx * dz + s2)));
    atomicAdd(&Jz[n], (double)(sw * (dx1 * dy1 + s3)));
    atomicAdd(&Jz[n + ey], (double)(sw * (dx1 * dy - s3)));
    atomicAdd(&Jz[n + ex], (double)(sw * (dx * dy1 - s3)));
    atomicAdd(&Jz[n + ex + ey], (double)(sw * (dx * dy + s3)));
}

// transpose of seg_mixed (cell units: h = 1, weights wx, wy, wz)
__device__ __forceinline__ void seg_mixed_rev(const double *const L[3], const Grid &g, int ci, int cl, int ck,
                                              const int iv[3], const float xs[3], const float xe[3], float cu,
                                              float cv, float cw, float gs[3], float ge[3]) {
    float dx = 0.5f * (xs[0] + xe[0]) - ((float)iv[0] - 2.5f);
    float dy = 0.5f * (xs[1] + xe[1]) - ((float)iv[1] - 2.5f);
    float dz = 0.5f * (xs[2] + xe[2]) - ((float)iv[2] - 2.5f);
    float dx1 = 1.f - dx, dy1 = 1.f - dy, dz1 = 1.f - dz;
    float Dx = xe[0] - xs[0], Dy = xe[1] - xs[1], Dz = xe[2] - xs[2];
    const float r12 = 1.f / 12.f;
    float s1 = Dy * Dz * r12, s2 = Dx * Dz * r12, s3 = Dx * Dy * r12;
    float Ax = cu * Dx, Ay = cv * Dy, Az = cw * Dz;
    size_t n = tap_node(g, ci, cl, ck, iv);
    const size_t ez = 1, ey = g.pz, ex = (size_t)g.NY * g.pz;
    float Lx0 = (float)L[0][n], Lx1 = (float)L[0][n + ez], Lx2 = (float)L[0][n + ey], Lx3 = (float)L[0][n + ey + ez];
    float Ly0 = (float)L[1][n], Ly1 = (float)L[1][n + ez], Ly2 = (float)L[1][n + ex], Ly3 = (float)L[1][n + ex + ez];
    float Lz0 = (float)L[2][n], Lz1 = (float)L[2][n + ey], Lz2 = (float)L[2][n + ex], Lz3 = (float)L[2][n + ex + ey];
    float Fx = Lx0 * (dy1 * dz1 + s1) + Lx1 * (dy1 * dz - s1) + Lx2 * (dy * dz1 - s1) + Lx3 * (dy * dz + s1);
    float Fy = Ly0 * (dx1 * dz1 + s2) + Ly1 * (dx1 * dz - s2) + Ly2 * (dx * dz1 - s2) + Ly3 * (dx * dz + s2);
    float Fz = Lz0 * (dx1 * dy1 + s3) + Lz1 * (dx1 * dy - s3) + Lz2 * (dx * dy1 - s3) + Lz3 * (dx * dy + s3);
    float Kx = Lx0 - Lx1 - Lx2 + Lx3, Ky = Ly0 - Ly1 - Ly2 + Ly3, Kz = Lz0 - Lz1 - Lz2 + Lz3;
    float gDx = cu * Fx + (Ay * Ky * Dz + Az * Kz * Dy) * r12;
    float gDy = cv * Fy + (Ax * Kx * Dz + Az * Kz * Dx) * r12;
    float gDz = cw * Fz + (Ax * Kx * Dy + Ay * Ky * Dx) * r12;
    float gdx = Ay * (-Ly0 * dz1 - Ly1 * dz + Ly2 * dz1 + Ly3 * dz) + Az * (-Lz0 * dy1 - Lz1 * dy + Lz2 * dy1 + Lz3 * dy);
    float gdy = Ax * (-Lx0 * dz1 - Lx1 * dz + Lx2 * dz1 + Lx3 * dz) + Az * (-Lz0 * dx1 + Lz1 * dx1 - Lz2 * dx + Lz3 * dx);
    float gdz = Ax * (-Lx0 * dy1 + Lx1 * dy1 - Lx2 * dy + Lx3 * dy) + Ay * (-Ly0 * dx1 + Ly1 * dx1 - Ly2 * dx + Ly3 * dx);
    gs[0] += 0.5f * gdx - gDx; ge[0] += 0.5f * gdx + gDx;
    gs[1] += 0.5f * gdy - gDy; ge[1] += 0.5f * gdy + gDy;
    gs[2] += 0.5f * gdz - gDz; ge[2] += 0.5f * gdz + gDz;
}

// transpose of the split point (crossing planes at 1/2; axes as template arguments)
template <int O>
__device__ __forceinline__ float rbx_rev_m(float sr, const float xo[3], const float xn[3], const float g2[3],
                                           float gx[3], float gn[3]) {
    gx[O] += g2[O] * (1.f - sr);
    gn[O] += g2[O] * sr;
    return g2[O] * (xn[O] - xo[O]);
}
template <int A, int O0, int O1>
__device__ __forceinline__ void split_rev1_m(const SplitM &S, const float xo[3], const float xn[3],
                                             const float g2[3], float gx[3], float gn[3]) {
    const float sr = S.sr;
    float lsr = rbx_rev_m<O0>(sr, xo, xn, g2, gx, gn) + rbx_rev_m<O1>(sr, xo, xn, g2, gx, gn);
    float D = xn[A] - xo[A];
    gx[A] += lsr * (0.5f - xn[A]) / (D * D);
    gn[A] -= lsr * sr / D;
}
template <int A, int B, int O>
__device__ __forceinline__ void split_rev2_m(const SplitM &S, const float xo[3], const float xn[3],
                                             const float g2[3], float gx[3], float gn[3]) {
    const float sr = S.sr;
    float lsr = rbx_rev_m<O>(sr, xo, xn, g2, gx, gn);
    float Da = xn[A] - xo[A], Db = xn[B] - xo[B];
    float f = lsr / (Da * Da + Db * Db);
    float ca = 0.5f - xo[A], cb = 0.5f - xo[B];
    gx[A] += f * (-Da - ca + 2.f * sr * Da);
    gn[A] += f * (ca - 2.f * sr * Da);
    gx[B] += f * (-Db - cb + 2.f * sr * Db);
    gn[B] += f * (cb - 2.f * sr * Db);
}
__device__ __forceinline__ void split_rev_m(const SplitM &S, const float xo[3], const float xn[3], const float g2[3],
                                            float gx[3], float gn[3]) {
    switch (S.m) {
        case 1: split_rev1_m<2, 0, 1>(S, xo, xn, g2, gx, gn); break;
        case 2: split_rev1_m<1, 0, 2>(S, xo, xn, g2, gx, gn); break;
        case 4: split_rev1_m<0, 1, 2>(S, xo, xn, g2, gx, gn); break;
        case 3: split_rev2_m<1, 2, 0>(S, xo, xn, g2, gx, gn); break;
        case 5: split_rev2_m<0, 2, 1>(S, xo, xn, g2, gx, gn); break;
        case 6: split_rev2_m<0, 1, 2>(S, xo, xn, g2, gx, gn); break;
        default: break;  // 7: the centre of the cell
    }
}

// ---- fixed-order push of the FP32 form
__global__ void __launch_bounds__(kT) k_flat_push_mixed(MixParams P) {
    int64_t idx = spread_index(threadIdx.x);
    unsigned bad = 0;
    unsigned long long amb = 0;
    if (idx < P.off[P.nsp]) {
        const Grid &g = P.g;
        int s = species_of(P.off, P.nsp, idx);
        const MixSp &S = P.sp[s];
        int64_t j = idx - P.off[s];
        int cell = S.cell[j];
        int i, l, k;
        g.cell_ijk(cell, i, l, k);
        float xs[3] = {S.v[0][j], S.v[1][j], S.v[2][j]};
        float p[3] = {S.v[3][j], S.v[4][j], S.v[5][j]};
        float F[6];
        gather_fields_m(g, P.E, P.H, i, l, k, xs, F);
        if (P.Fout[0]) {
#pragma unroll
            for (int c = 0; c < 6; c++) P.Fout[c][idx] = F[c];
        }
        const float tau1 = (float)(S.q_m * g.tau * 0.5);
        const float ct[3] = {(float)(g.tau / g.hx), (float)(g.tau / g.hy), (float)(g.tau / g.hz)};
        BorisM B;
        boris_mixed(tau1, ct, p, F, xs, B);
        if (!(isfinite(B.pp[0]) && isfinite(B.pp[1]) && isfinite(B.pp[2]))) bad |= ST_NAN;
        float xe[3] = {B.xe[0], B.xe[1], B.xe[2]};
        SplitM SP;
        split_mixed(xs, xe, SP);
        const float wx = (float)(S.m * g.hx / g.tau), wy = (float)(S.m * g.hy / g.tau), wz = (float)(S.m * g.hz / g.tau);
        if (!stencil_ok(SP.i2) || !(isfinite(xe[0]) && isfinite(xe[1]) && isfinite(xe[2]))) {
            bad |= ST_STENCIL;
        } else {
            seg_mixed(P.J, g, i, l, k, SP.i1, xs, SP.x2, wx, wy, wz);
            seg_mixed(P.J, g, i, l, k, SP.i2, SP.x2, xe, wx, wy, wz);
        }
        // new cell (Reflect and migration in cell units, as k_push_mixed)
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
        const MixOut &O = P.out[s];
        O.cell[j] = g.cell_of(ci[0], ci[1], ci[2]);
        O.v[0][j] = xe[0]; O.v[1][j] = xe[1]; O.v[2][j] = xe[2];
        O.v[3][j] = B.pp[0]; O.v[4][j] = B.pp[1]; O.v[5][j] = B.pp[2];
    }
    if (bad) atomicOr(&P.st->flags, bad);
    if (amb) atomicAdd(&P.st->ambiguous, amb);
}

// ---- adjoint, first pass: recompute, deposit and push transposes
template <bool STORED>
__global__ void __launch_bounds__(kT, 2) k_adj_push_mixed(MixParams P) {
    int64_t idx = spread_index(threadIdx.x);
    if (idx >= P.off[P.nsp]) return;
    const Grid &g = P.g;
    int s = species_of(P.off, P.nsp, idx);
    const MixSp &S = P.sp[s];
    int64_t j = idx - P.off[s];
    int i, l, k;
    g.cell_ijk(S.cell[j], i, l, k);
    float xs[3] = {S.v[0][j], S.v[1][j], S.v[2][j]};
    float p[3] = {S.v[3][j], S.v[4][j], S.v[5][j]};
    float F[6];
    if (STORED) {
#pragma unroll
        for (int c = 0; c < 6; c++) F[c] = P.Fin[c][idx];
    } else {
        gather_fields_m(g, P.E, P.H, i, l, k, xs, F);
    }
    const float tau1 = (float)(S.q_m * g.tau * 0.5);
    const float ct[3] = {(float)(g.tau / g.hx), (float)(g.tau / g.hy), (float)(g.tau / g.hz)};
    BorisM B;
    boris_mixed(tau1, ct, p, F, xs, B);
    SplitM SP;
    split_mixed(xs, B.xe, SP);
    float *const *Lm = P.lam[s];
    float lx[3] = {Lm[0][j], Lm[1][j], Lm[2][j]};
    float lp[3] = {Lm[3][j], Lm[4][j], Lm[5][j]};
    float gx[3] = {0.f, 0.f, 0.f}, gn[3] = {lx[0], lx[1], lx[2]};
    const float wx = (float)(S.m * g.hx / g.tau), wy = (float)(S.m * g.hy / g.tau), wz = (float)(S.m * g.hz / g.tau);
    if (stencil_ok(SP.i2)) {
        if (SP.m != 0) {
            float g2[3] = {0.f, 0.f, 0.f};
            seg_mixed_rev(P.LJ, g, i, l, k, SP.i1, xs, SP.x2, wx, wy, wz, gx, g2);
            seg_mixed_rev(P.LJ, g, i, l, k, SP.i2, SP.x2, B.xe, wx, wy, wz, g2, gn);
            split_rev_m(SP, xs, B.xe, g2, gx, gn);
        } else {  // no crossing: x2 = xe, one segment
            seg_mixed_rev(P.LJ, g, i, l, k, SP.i1, xs, B.xe, wx, wy, wz, gx, gn);
        }
    }
    // xe = xs + ct * ig * p'
    float dot = 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        gx[d] += gn[d];
        dot += gn[d] * B.ct[d] * B.pp[d];
    }
    const float ig3 = B.ig * B.ig * B.ig;
    float lP[3];
#pragma unroll
    for (int d = 0; d < 3; d++) lP[d] = lp[d] + B.ig * B.ct[d] * gn[d] - ig3 * dot * B.pp[d];
    float lF[6];
#pragma unroll
    for (int d = 0; d < 3; d++) lF[d] = B.t * lP[d];
    const float *b = B.b, *sv = B.s, *up = B.up, *u = B.u;
    float bl = b[0] * lP[0] + b[1] * lP[1] + b[2] * lP[2];
    float bs = b[0] * sv[0] + b[1] * sv[1] + b[2] * sv[2];
    float lu_ = lP[0] * up[0] + lP[1] * up[1] + lP[2] * up[2];
    const float inv = B.rs;
    float bxl[3] = {b[1] * lP[2] - b[2] * lP[1], b[2] * lP[0] - b[0] * lP[2], b[0] * lP[1] - b[1] * lP[0]};
    float lxs[3] = {lP[1] * sv[2] - lP[2] * sv[1], lP[2] * sv[0] - lP[0] * sv[2], lP[0] * sv[1] - lP[1] * sv[0]};
    float ls[3], lb[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        ls[d] = (lP[d] + b[d] * bl + bxl[d]) * inv;
        lb[d] = (bs * lP[d] + bl * sv[d] + lxs[d] - 2.f * lu_ * b[d]) * inv;
    }
    float lu[3] = {ls[0] + (b[1] * ls[2] - b[2] * ls[1]), ls[1] + (b[2] * ls[0] - b[0] * ls[2]),
                   ls[2] + (b[0] * ls[1] - b[1] * ls[0])};
    lb[0] += ls[1] * u[2] - ls[2] * u[1];
    lb[1] += ls[2] * u[0] - ls[0] * u[2];
    lb[2] += ls[0] * u[1] - ls[1] * u[0];
    float lps = 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        lF[3 + d] = B.ps * lb[d];
        lps += lb[d] * F[3 + d];
    }
    const float cps = -B.t * B.g1 * B.g1 * B.g1 * lps;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        lu[d] += cps * u[d];
        lF[d] += B.t * lu[d];
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        Lm[d][j] = gx[d];
        Lm[3 + d][j] = lu[d];
    }
#pragma unroll
    for (int c = 0; c < 6; c++) P.LF[c][idx] = lF[c];
}

// ---- adjoint, second pass: interpolation transpose
__global__ void __launch_bounds__(kT) k_adj_interp_mixed(MixParams P) {
    __shared__ int sHi[6 * kBoxNodes];
    __shared__ int sRed[6 * (kT / 32)];
    __shared__ unsigned sMax[kT / 32], sMaxOut;
    __shared__ NodeBox sBox;
    const Grid &g = P.g;
    int64_t idx = spread_index(threadIdx.x);
    const bool valid = idx < P.off[P.nsp];
    int s = 0, i = 0, l = 0, k = 0;
    int64_t j = 0;
    float xs[3] = {0.f, 0.f, 0.f};
    if (valid) {
        s = species_of(P.off, P.nsp, idx);
        const MixSp &S = P.sp[s];
        j = idx - P.off[s];
        xs[0] = S.v[0][j]; xs[1] = S.v[1][j]; xs[2] = S.v[2][j];
        g.cell_ijk(S.cell[j], i, l, k);
    }
    float lam6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float amax = 0.f;
    if (valid) {
#pragma unroll
        for (int c = 0; c < 6; c++) {
            lam6[c] = P.LF[c][idx];
            amax = fmaxf(amax, fabsf(lam6[c]));
        }
    }
    const NodeBox box = block_node_box(i, l, k, valid, sRed, &sBox);
    const float bmax = block_max_abs(amax, sMax, &sMaxOut);
    if (bmax == 0.f) return;  // no adjoint reaches the particles of this block
    const int E = box_exponent(bmax);
    const float inv_q = __uint_as_float((unsigned)(22 - E + 127) << 23);
    for (int e = threadIdx.x; e < 6 * box.nodes; e += blockDim.x) sHi[e] = 0;
    __syncthreads();
    if (valid) {
        MTaps T;
        taps_mixed(xs, T);
        const size_t dX = (size_t)g.NY * g.pz, dY = g.pz, dZ = 1;
        float gx[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int c = 0; c < 6; c++) {
            int t[3];
            float w[3];
            const float lam = lam6[c];
            if (lam == 0.f) continue;
            comp_taps_m(T, c, t, w);
            size_t n = tap_node(g, i, l, k, t);
            const float *Arr = c < 3 ? P.E[c] : P.H[c - 3];
            double *LA = c < 3 ? P.LE[c] : P.LH[c - 3];
            const int b0 = box.nodes ? c * box.nodes + box_index(box, i + t[0] - 2, l + t[1] - 2, k + t[2] - 2) : 0;
            const float W0[2] = {w[0], 1.f - w[0]}, W1[2] = {w[1], 1.f - w[1]}, W2[2] = {w[2], 1.f - w[2]};
            float gr[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int bb = 0; bb < 2; bb++)
#pragma unroll
                    for (int cc = 0; cc < 2; cc++) {
                        size_t m = n + a * dX + bb * dY + cc * dZ;
                        float v = Arr[m];
                        float add = lam * (W0[a] * W1[bb] * W2[cc]);
                        if (box.nodes) {
                            int hi = __float2int_rn(add * inv_q);
                            if (hi) atomicAdd(&sHi[b0 + (a * box.by + bb) * box.bz + cc], hi);
                        } else {
                            atomicAdd(&LA[m], (double)add);
                        }
                        gr[0] += (a ? 1.f : -1.f) * W1[bb] * W2[cc] * v;
                        gr[1] += (bb ? 1.f : -1.f) * W0[a] * W2[cc] * v;
                        gr[2] += (cc ? 1.f : -1.f) * W0[a] * W1[bb] * v;
                    }
            gx[0] += lam * gr[0];
            gx[1] += lam * gr[1];
            gx[2] += lam * gr[2];
        }
        float *const *Lm = P.lam[s];
#pragma unroll
        for (int d = 0; d < 3; d++) Lm[d][j] += gx[d];
    }
    if (box.nodes) {
        __syncthreads();
        double *const dst[6] = {P.LE[0], P.LE[1], P.LE[2], P.LH[0], P.LH[1], P.LH[2]};
        flush_node_box(box, sHi, nullptr, pow2_d(E - 22), g, dst);
    }
}

__global__ void k_h_half_m(Grid g, const float *__restrict__ Ex, const float *__restrict__ Ey,
                           const float *__restrict__ Ez, const float *__restrict__ Hx, const float *__restrict__ Hy,
                           const float *__restrict__ Hz, float *Ax, float *Ay, float *Az, float cx, float cy,
                           float cz) {
    int k = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y, i = blockIdx.z;
    if (k >= g.NZ) return;
    size_t n = g.node(i, l, k), sx = (size_t)g.NY * g.pz, sy = g.pz;
    float hx = Hx[n], hy = Hy[n], hz = Hz[n];
    if (i <= g.nx + 1 && l <= g.ny && k <= g.nz) hx += 0.5f * (cz * (Ey[n + 1] - Ey[n]) - cy * (Ez[n + sy] - Ez[n]));
    if (i <= g.nx && l <= g.ny + 1 && k <= g.nz) hy += 0.5f * (cx * (Ez[n + sx] - Ez[n]) - cz * (Ex[n + 1] - Ex[n]));
    if (i <= g.nx && l <= g.ny && k <= g.nz + 1) hz += 0.5f * (cy * (Ex[n + sy] - Ex[n]) - cx * (Ey[n + sx] - Ey[n]));
    Ax[n] = hx;
    Ay[n] = hy;
    Az[n] = hz;
}

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

inline unsigned blocks_of(int64_t n) { return (unsigned)((n + kT - 1) / kT); }

}  // namespace

cudaError_t launch_flat_push_mixed(const MixParams &P, cudaStream_t s) {
    int64_t n = P.off[P.nsp];
    if (n > 0) k_flat_push_mixed<<<blocks_of(n), kT, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_adj_particles_mixed(const MixParams &P, cudaStream_t s) {
    int64_t n = P.off[P.nsp];
    if (n <= 0) return cudaSuccess;
    if (P.Fin[0]) k_adj_push_mixed<true><<<blocks_of(n), kT, 0, s>>>(P);
    else k_adj_push_mixed<false><<<blocks_of(n), kT, 0, s>>>(P);
    k_adj_interp_mixed<<<blocks_of(n), kT, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_h_half_mixed(const Grid &g, const float *E, const float *H, float *Ha, size_t N, cudaStream_t s) {
    float cx = (float)(g.tau / g.hx), cy = (float)(g.tau / g.hy), cz = (float)(g.tau / g.hz);
    dim3 grid((g.NZ + 31) / 32, g.NY, g.NX);
    k_h_half_m<<<grid, 32, 0, s>>>(g, E, E + N, E + 2 * N, H, H + N, H + 2 * N, Ha, Ha + N, Ha + 2 * N, cx, cy, cz);
    return cudaGetLastError();
}

void adj_gather_mixed(const Grid &g, const SpeciesView &S, const int64_t *d0, int *cell, void *const v[6],
                      cudaStream_t s) {
    k_gather_native<<<g.ntiles, 256, 0, s>>>(S, d0, cell, (float *)v[0], (float *)v[1], (float *)v[2],
                                             (float *)v[3], (float *)v[4], (float *)v[5]);
}

void adj_widen_mixed(const float *lp, const float *const p0[3], int64_t n, double *out6, cudaStream_t s) {
    if (n <= 0) return;
    k_widen<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(lp, p0[0], p0[1], p0[2], n, out6);
}

}  // namespace pic
