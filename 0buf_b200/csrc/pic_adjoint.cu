// Differentiable run of the PIC step (pic_forward / pic_backward): a forward
// pass that keeps every particle in a fixed order and checkpoints the state,
// and hand-written reverse-mode (adjoint) kernels.  Plain form: FP64, same
// arithmetic as k_push_plain (compiled with -fmad=false like it); the FP32
// form lives in pic_adjoint_mixed.cu.
//
// Forward map of one step (Plasma::Step, gpu_plasma.h:605-620), per piece:
//   Q = A E, H_a = H + Q                 (emh1, kernels.cu:1052-1073)
//   particles: F = W(x) [E, H_a]; (p', x') = Boris(p, F, x)   (particle.h:65-202)
//   J = sum_p D(x, x')                    (CurrentToMesh/pqr, cell.h:1306-1693)
//   J <- P J                              (periodicCurrentElement, kernels.cu:1124-1146)
//   H' = H_a + Q                          (emh2, kernels.cu:1024-1049)
//   E' = G (E + tau C H' - tau J)         (emeElement + periodicElement, kernels.cu:1091-1110)
// The reverse step applies the transposes in the opposite order.  Particles
// never change order in this pass (their cell index is rewritten in place),
// so a particle's adjoint (lambda_x, lambda_p) follows it from step to step;
// the deposit's transpose is a gather of lambda_J at the particle's 12 nodes
// per segment and the interpolation's transpose a scatter of lambda_F.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <vector>
#include <algorithm>
#include "pic0buf.h"
#include "pic_internal.cuh"
#include "pic_kernels.cuh"
#include "pic_handle.cuh"
#include "pic_adjoint.cuh"

namespace pic {

namespace {

constexpr int kT = 256;

// ================================================================ plain ==
// one species in flat order: packed cell, global FP64 positions, momenta
struct FlatSp {
    int64_t n;
    double q_m, m;
    int *cell;
    double *v[6];  // x y z px py pz
};
// where the push writes the state after the step (may alias the input)
struct FlatOut {
    int *cell;
    double *v[6];
};
struct FlatParams {
    Grid g;
    int nsp;
    int64_t off[kMaxSpecies + 1];
    FlatSp sp[kMaxSpecies];
    FlatOut out[kMaxSpecies];
    double *Fout[6];  // optional: the six interpolated field values per particle (flat index)
    const double *E[3];
    const double *H[3];
    double *J[3];
    AdjStatus *st;
    // discrete choices of this step, one 48-bit code per particle (flat index):
    // bmode 1 records them, 2 replays them (see branch_code)
    unsigned long long *branch;
    int bmode;
};
// adjoint of one species: lambda_x (3) and lambda_p (3), same order
struct LamSp {
    double *v[6];
};
struct AdjParams {
    FlatParams f;  // state at the start of the step; E = E_n, H = H_a (after the B half step)
    LamSp lam[kMaxSpecies];
    const double *LJ[3];  // lambda_J (after the fold's transpose)
    double *LE[3];        // lambda_E_n (scatter target)
    double *LH[3];        // lambda_H_a (scatter target)
    double *LF[6];        // lambda of the six interpolated field values, per particle (flat index)
    const double *Fin[6]; // the forward's interpolated fields of this step, or null (gather again)
};

// Particle handled by thread t of a 256-thread block.  Consecutive particles
// in the fixed order mostly share a cell, so a warp of consecutive particles
// would send its 32 current / adjoint atomics of one tap to the same few
// nodes.  Lane quads take 4 consecutive particles (one 32-byte sector of an
// FP64 array) and the 8 quads of a warp sit 32 particles apart, i.e. in about
// 8 different cells: loads stay sector-coalesced and atomic conflicts drop ~8x.
__device__ __forceinline__ int64_t spread_index(int t) {
    return (int64_t)blockIdx.x * kT + ((t & 31) >> 2) * 32 + (t >> 5) * 4 + (t & 3);
}

__device__ __forceinline__ int species_of(const int64_t *off, int nsp, int64_t idx) {
    int s = 0;
    while (s + 1 < nsp && idx >= off[s + 1]) s++;
    return s;
}

// staggered interpolation of one particle: lower tap (reference tile index)
// and its weight per axis, node- and centre-staggered (InverseKernel,
// cell.h:1010-1047, as evaluated in Cell::GetField, cell.h:1257-1290)
struct Taps {
    int tn[3], tc[3];
    double wn[3], wc[3];
};
// the discrete part of the taps: tap indices and the integer parts of the
// weights (nI = int(x/h + 1), cI = int(x/h + 1.5)); the weights follow from them
struct TapInts {
    int tn[3], tc[3], nI[3], cI[3];
};
__device__ __forceinline__ void tap_ints(const Grid &g, int i, int l, int k, const double x[3], TapInts &I) {
    const double h3[3] = {g.hx, g.hy, g.hz};
    const int c3[3] = {i, l, k};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double x0 = (double)c3[d] * h3[d];
        I.tn[d] = (int)((x[d] - x0) / h3[d] + 1.0) + 1;
        I.tc[d] = (int)(((x[d] - x0) / h3[d] + 1.0) + 1.5);
        I.nI[d] = (int)(x[d] / h3[d] + 1.0);
        I.cI[d] = (int)(x[d] / h3[d] + 1.5);
    }
}
__device__ __forceinline__ void taps_from(const Grid &g, const double x[3], const TapInts &I, Taps &T) {
    const double h3[3] = {g.hx, g.hy, g.hz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        T.tn[d] = I.tn[d];
        T.tc[d] = I.tc[d];
        T.wn[d] = I.nI[d] - x[d] / h3[d];
        T.wc[d] = I.cI[d] - 0.5 - x[d] / h3[d];
    }
}
__device__ __forceinline__ void taps_plain(const Grid &g, int i, int l, int k, const double x[3], Taps &T) {
    TapInts I;
    tap_ints(g, i, l, k, x, I);
    taps_from(g, x, I, T);
}
// component c (0..2 E, 3..5 H) is node-staggered along axis d when
// (E_c and d == c) or (H_c and d != c)
__device__ __forceinline__ bool node_axis(int c, int d) { return c < 3 ? d == c : d != c - 3; }

// the 8 taps of one component: value (interp_plain's expression order) and
// the tap base; false when a tap leaves the 3-node stencil (CFL violation)
__device__ __forceinline__ bool comp_taps(const Taps &T, int c, int t[3], double w[3]) {
    bool ok = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        bool nd = node_axis(c, d);
        t[d] = nd ? T.tn[d] : T.tc[d];
        w[d] = nd ? T.wn[d] : T.wc[d];
        ok = ok && t[d] >= 2 && t[d] <= 3;
    }
    return ok;
}
__device__ __forceinline__ size_t tap_node(const Grid &g, int i, int l, int k, const int t[3]) {
    return g.node(i + t[0] - 2, l + t[1] - 2, k + t[2] - 2);
}
__device__ __forceinline__ double interp_g(const double *__restrict__ A, size_t n, size_t dx, size_t dy,
                                           const double w[3]) {
    const size_t dz = 1;
    double sx = w[0], sx1 = 1. - w[0], sy = w[1], sy1 = 1. - w[1], sz = w[2], sz1 = 1. - w[2];
    double t_ilk = A[n], t_ilk1 = A[n + dz], t_il1k = A[n + dy], t_il1k1 = A[n + dy + dz];
    double t_i1lk = A[n + dx], t_i1lk1 = A[n + dx + dz], t_i1l1k = A[n + dx + dy], t_i1l1k1 = A[n + dx + dy + dz];
    double t1 = sx * (sy * (sz * t_ilk + sz1 * t_ilk1) + sy1 * (sz * t_il1k + sz1 * t_il1k1));
    double t2 = sx1 * (sy * (sz * t_i1lk + sz1 * t_i1lk1) + sy1 * (sz * t_i1l1k + sz1 * t_i1l1k1));
    return t2 + t1;
}

// fields at the particle (all six components); false if a stencil left range
// (negative_is_zero: the reference's GetField gives no field at a negative
// coordinate; positions are wrapped into [0, L) so a run never meets it, and a
// replay of frozen branches, whose wraps are fixed, leaves it out)
__device__ __forceinline__ bool gather_fields_taps(const Grid &g, const double *const E[3],
                                                   const double *const H[3], int i, int l, int k, const double x[3],
                                                   const Taps &T, double F[6], bool negative_is_zero = true) {
    if (negative_is_zero && (x[0] < 0 || x[1] < 0 || x[2] < 0)) {
        for (int c = 0; c < 6; c++) F[c] = 0.0;
        return true;
    }
    const size_t dx = (size_t)g.NY * g.pz, dy = g.pz;
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 6; c++) {
        int t[3];
        double w[3];
        if (!comp_taps(T, c, t, w)) { ok = false; F[c] = 0.0; continue; }
        F[c] = interp_g(c < 3 ? E[c] : H[c - 3], tap_node(g, i, l, k, t), dx, dy, w);
    }
    return ok;
}
__device__ __forceinline__ bool gather_fields(const Grid &g, const double *const E[3], const double *const H[3],
                                              int i, int l, int k, const double x[3], double F[6]) {
    Taps T;
    taps_plain(g, i, l, k, x, T);
    return gather_fields_taps(g, E, H, i, l, k, x, T, F);
}

// Particle::Move, particle.h:65-202, with the intermediates the adjoint needs
struct Boris {
    double t, u[3], g1, ps, b[3], s[3], sd, up[3], pp[3], g2, x1[3];
};
__device__ __forceinline__ void boris_plain(double q_m, double tau, const double p[3], const double F[6],
                                            const double x[3], Boris &B) {
    double tau1 = q_m * tau * 0.5;
    B.t = tau1;
    double pu = p[0], pv = p[1], pw = p[2];
    pu += tau1 * F[0];
    pv += tau1 * F[1];
    pw += tau1 * F[2];
    B.u[0] = pu; B.u[1] = pv; B.u[2] = pw;
    B.g1 = 1.0 / sqrt((pu * pu + pv * pv + pw * pw) * 1. + 1.0);  // pow(v, -0.5), as in k_push_plain
    double ps = tau1 * B.g1;
    B.ps = ps;
    double bx = ps * F[3], by = ps * F[4], bz = ps * F[5];
    B.b[0] = bx; B.b[1] = by; B.b[2] = bz;
    double su = pu + pv * bz - pw * by;
    double sv = pv + pw * bx - pu * bz;
    double sw = pw + pu * by - pv * bx;
    B.s[0] = su; B.s[1] = sv; B.s[2] = sw;
    double q1 = bx * bx, q2 = by * by, q3 = bz * bz, q4 = bx * by, q5 = by * bz, q6 = bz * bx;
    double sd = q1 + 1. + q2 + q3;
    B.sd = sd;
    double pu1 = ((q1 + 1.) * su + (q4 + bz) * sv + (q6 - by) * sw) / sd;
    double pv1 = ((q4 - bz) * su + (q2 + 1.) * sv + (q5 + bx) * sw) / sd;
    double pw1 = ((q6 + by) * su + (q5 - bx) * sv + (q3 + 1.) * sw) / sd;
    B.up[0] = pu1; B.up[1] = pv1; B.up[2] = pw1;
    pu = pu1 + F[0] * tau1;
    pv = pv1 + F[1] * tau1;
    pw = pw1 + F[2] * tau1;
    B.pp[0] = pu; B.pp[1] = pv; B.pp[2] = pw;
    B.g2 = 1.0 / sqrt(((pu * pu + pv * pv + pw * pw) + 1.0));
    B.x1[0] = x[0] + tau * (B.g2 * pu);
    B.x1[1] = x[1] + tau * (B.g2 * pv);
    B.x1[2] = x[2] + tau * (B.g2 * pw);
}

// zigzag split of CurrentToMesh, cell.h:1306-1422 (m = 4|di| + 2|dl| + |dk|)
struct Split {
    int m, i1[3], i2[3];
    double x2[3], sr;
};
// the discrete part: cell-centre indices of both end points
// (getCellNumberCenterCurrent, cell.h:577-578)
__device__ __forceinline__ void split_ints(const Grid &g, const double xo[3], const double xn[3], const double o3[3],
                                           Split &S) {
    const double h3[3] = {g.hx, g.hy, g.hz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double tt = ((xo[d] - o3[d]) / h3[d] + 1.5);
        S.i1[d] = (int)(tt + 1);
        double t2 = ((xn[d] - o3[d]) / h3[d] + 1.5);
        S.i2[d] = (int)(t2 + 1);
    }
}
// the split case and relay point from S.i1, S.i2
__device__ __forceinline__ void split_from(const Grid &g, const double xo[3], const double xn[3], const double o3[3],
                                           Split &S) {
    const double h3[3] = {g.hx, g.hy, g.hz};
    double *x2 = S.x2;
    x2[0] = x2[1] = x2[2] = 0.0;
    S.sr = 0.0;
    double sr = 0.0;
    const int *i1 = S.i1, *i2 = S.i2;
    int m = 4 * abs(i2[0] - i1[0]) + 2 * abs(i2[1] - i1[1]) + abs(i2[2] - i1[2]);
    S.m = m;
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
    S.sr = sr;
}
__device__ __forceinline__ void split_plain(const Grid &g, const double xo[3], const double xn[3], const double o3[3],
                                            Split &S) {
    split_ints(g, xo, xn, o3, S);
    split_from(g, xo, xn, o3, S);
}

// one pqr segment (cell.h:1511-1693) into the global J, FP64 atomics
__device__ __forceinline__ void seg_plain(double *const J[3], const Grid &g, int ci, int cl, int ck, const int iv[3],
                                          const double x[3], const double x1[3], double a1, const double o3[3],
                                          unsigned &bad) {
    const double hx = g.hx, hy = g.hy, hz = g.hz, tau = g.tau;
    double dx = (0.50 * (x[0] + x1[0]) - hx * ((double)iv[0] - 2.50) - o3[0]);
    double dy = (0.50 * (x[1] + x1[1]) - hy * ((double)iv[1] - 2.50) - o3[1]);
    double dz = (0.50 * (x[2] + x1[2]) - hz * ((double)iv[2] - 2.50) - o3[2]);
    double a = a1;
    double dx1 = hx - dx, dy1 = hy - dy, dz1 = hz - dz;
    double su = x1[0] - x[0], sv = x1[1] - x[1], sw = x1[2] - x[2];
    double s1 = sv * sw / 12.0, s2 = su * sw / 12.0, s3 = su * sv / 12.0;
    su = su * a / (tau * hy * hz);
    sv = sv * a / (tau * hx * hz);
    sw = sw * a / (tau * hx * hy);
    if (iv[0] < 2 || iv[0] > 3 || iv[1] < 2 || iv[1] > 3 || iv[2] < 2 || iv[2] > 3) { bad |= ST_STENCIL; return; }
    size_t n = tap_node(g, ci, cl, ck, iv);
    const size_t ez = 1, ey = g.pz, ex = (size_t)g.NY * g.pz;
    double *Jx = J[0], *Jy = J[1], *Jz = J[2];
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

// transpose of seg_plain: lambda_J gathered at the segment's 12 nodes gives
// the gradient with respect to the segment's end points (added to gs, ge)
__device__ __forceinline__ void seg_plain_rev(const double *const L[3], const Grid &g, int ci, int cl, int ck,
                                              const int iv[3], const double xs[3], const double xe[3], double a,
                                              const double o3[3], double gs[3], double ge[3]) {
    if (iv[0] < 2 || iv[0] > 3 || iv[1] < 2 || iv[1] > 3 || iv[2] < 2 || iv[2] > 3) return;
    const double hx = g.hx, hy = g.hy, hz = g.hz, tau = g.tau;
    double dx = 0.5 * (xs[0] + xe[0]) - hx * ((double)iv[0] - 2.5) - o3[0];
    double dy = 0.5 * (xs[1] + xe[1]) - hy * ((double)iv[1] - 2.5) - o3[1];
    double dz = 0.5 * (xs[2] + xe[2]) - hz * ((double)iv[2] - 2.5) - o3[2];
    double dx1 = hx - dx, dy1 = hy - dy, dz1 = hz - dz;
    double Dx = xe[0] - xs[0], Dy = xe[1] - xs[1], Dz = xe[2] - xs[2];
    double s1 = Dy * Dz / 12.0, s2 = Dx * Dz / 12.0, s3 = Dx * Dy / 12.0;
    double cu = a / (tau * hy * hz), cv = a / (tau * hx * hz), cw = a / (tau * hx * hy);
    double Ax = cu * Dx, Ay = cv * Dy, Az = cw * Dz;
    size_t n = tap_node(g, ci, cl, ck, iv);
    const size_t ez = 1, ey = g.pz, ex = (size_t)g.NY * g.pz;
    double Lx0 = L[0][n], Lx1 = L[0][n + ez], Lx2 = L[0][n + ey], Lx3 = L[0][n + ey + ez];
    double Ly0 = L[1][n], Ly1 = L[1][n + ez], Ly2 = L[1][n + ex], Ly3 = L[1][n + ex + ez];
    double Lz0 = L[2][n], Lz1 = L[2][n + ey], Lz2 = L[2][n + ex], Lz3 = L[2][n + ex + ey];
    double Fx = Lx0 * (dy1 * dz1 + s1) + Lx1 * (dy1 * dz - s1) + Lx2 * (dy * dz1 - s1) + Lx3 * (dy * dz + s1);
    double Fy = Ly0 * (dx1 * dz1 + s2) + Ly1 * (dx1 * dz - s2) + Ly2 * (dx * dz1 - s2) + Ly3 * (dx * dz + s2);
    double Fz = Lz0 * (dx1 * dy1 + s3) + Lz1 * (dx1 * dy - s3) + Lz2 * (dx * dy1 - s3) + Lz3 * (dx * dy + s3);
    double Kx = Lx0 - Lx1 - Lx2 + Lx3, Ky = Ly0 - Ly1 - Ly2 + Ly3, Kz = Lz0 - Lz1 - Lz2 + Lz3;
    // d/d(D): direct factor and the D-products in s1, s2, s3
    double gDx = cu * Fx + (Ay * Ky * Dz + Az * Kz * Dy) / 12.0;
    double gDy = cv * Fy + (Ax * Kx * Dz + Az * Kz * Dx) / 12.0;
    double gDz = cw * Fz + (Ax * Kx * Dy + Ay * Ky * Dx) / 12.0;
    // d/d(dx, dy, dz): the bilinear node weights
    double gdx = Ay * (-Ly0 * dz1 - Ly1 * dz + Ly2 * dz1 + Ly3 * dz) + Az * (-Lz0 * dy1 - Lz1 * dy + Lz2 * dy1 + Lz3 * dy);
    double gdy = Ax * (-Lx0 * dz1 - Lx1 * dz + Lx2 * dz1 + Lx3 * dz) + Az * (-Lz0 * dx1 + Lz1 * dx1 - Lz2 * dx + Lz3 * dx);
    double gdz = Ax * (-Lx0 * dy1 + Lx1 * dy1 - Lx2 * dy + Lx3 * dy) + Ay * (-Ly0 * dx1 + Ly1 * dx1 - Ly2 * dx + Ly3 * dx);
    gs[0] += 0.5 * gdx - gDx; ge[0] += 0.5 * gdx + gDx;
    gs[1] += 0.5 * gdy - gDy; ge[1] += 0.5 * gdy + gDy;
    gs[2] += 0.5 * gdz - gDz; ge[2] += 0.5 * gdz + gDz;
}

// transpose of the split point x2(xo, xn): adds g2 . dx2/dxo to gx, . dx2/dxn
// to gn.  Axis indices are template arguments so the 3-vectors stay in registers.
template <int O>
__device__ __forceinline__ double rbx_rev(double sr, const double xo[3], const double xn[3], const double g2[3],
                                          double gx[3], double gn[3]) {
    // x2[O] = xo[O] + (xn[O] - xo[O]) sr
    gx[O] += g2[O] * (1.0 - sr);
    gn[O] += g2[O] * sr;
    return g2[O] * (xn[O] - xo[O]);
}
template <int A, int O0, int O1>  // one plane crossed on axis A: sr = (c - xo)/(xn - xo)
__device__ __forceinline__ void split_rev1(const Split &S, const double xo[3], const double xn[3],
                                           const double g2[3], double gx[3], double gn[3]) {
    const double sr = S.sr;
    double lsr = rbx_rev<O0>(sr, xo, xn, g2, gx, gn) + rbx_rev<O1>(sr, xo, xn, g2, gx, gn);
    double D = xn[A] - xo[A];
    gx[A] += lsr * (S.x2[A] - xn[A]) / (D * D);
    gn[A] -= lsr * sr / D;
}
template <int A, int B, int O>  // two planes: sr = sum_d (c_d - xo_d)(xn_d - xo_d) / sum_d (xn_d - xo_d)^2
__device__ __forceinline__ void split_rev2(const Split &S, const double xo[3], const double xn[3],
                                           const double g2[3], double gx[3], double gn[3]) {
    const double sr = S.sr;
    double lsr = rbx_rev<O>(sr, xo, xn, g2, gx, gn);
    double Da = xn[A] - xo[A], Db = xn[B] - xo[B];
    double f = lsr / (Da * Da + Db * Db);
    double ca = S.x2[A] - xo[A], cb = S.x2[B] - xo[B];
    gx[A] += f * (-Da - ca + 2.0 * sr * Da);
    gn[A] += f * (ca - 2.0 * sr * Da);
    gx[B] += f * (-Db - cb + 2.0 * sr * Db);
    gn[B] += f * (cb - 2.0 * sr * Db);
}
__device__ __forceinline__ void split_rev(const Split &S, const double xo[3], const double xn[3], const double g2[3],
                                          double gx[3], double gn[3]) {
    switch (S.m) {
        case 1: split_rev1<2, 0, 1>(S, xo, xn, g2, gx, gn); break;
        case 2: split_rev1<1, 0, 2>(S, xo, xn, g2, gx, gn); break;
        case 4: split_rev1<0, 1, 2>(S, xo, xn, g2, gx, gn); break;
        case 3: split_rev2<1, 2, 0>(S, xo, xn, g2, gx, gn); break;
        case 5: split_rev2<0, 2, 1>(S, xo, xn, g2, gx, gn); break;
        case 6: split_rev2<0, 1, 2>(S, xo, xn, g2, gx, gn); break;
        default: break;  // 7: the split point is a fixed corner; 0 / >7: no split
    }
}

// Reflect, cell.h:1427-1478
__device__ __forceinline__ double reflect_g(double x, double xm) {
    return (x > xm) * (x - xm) + (x < 0.0) * (xm + x) + (x > 0 && x < xm) * x;
}
// reflect_g as a choice (0 keep, 1 subtract xm, 2 add xm, 3 the x == xm case: 0)
// and its application; apply_wrap(x, xm, wrap_choice(x, xm)) == reflect_g(x, xm)
__device__ __forceinline__ int wrap_choice(double x, double xm) {
    return x > xm ? 1 : (x < 0.0 ? 2 : (x == xm ? 3 : 0));
}
__device__ __forceinline__ double apply_wrap(double x, double xm, int w) {
    return w == 1 ? x - xm : (w == 2 ? xm + x : (w == 3 ? 0.0 : x));
}

// Frozen branches.  Per particle and step, the discrete choices of the flat
// FP64 push, 16 bits per axis d at bit 16 d: tap indices tn-1, tc-1, the
// integer parts nI - c_d and cI - c_d of the interpolation weights (c the
// cell index), the zigzag cell-centre indices i1-1 and i2-1, the periodic
// wrap and the cell move + 1, 2 bits each.  A forward that replays them is a
// smooth function of the initial state near the recorded run, and it is the
// map the adjoint differentiates, so its finite differences check the
// adjoint without the kinks and jumps of the deposit.
constexpr unsigned ST_BRANCH_RANGE = 64u;  // a choice outside its 2-bit field (recording)
__device__ __forceinline__ bool pack2(unsigned long long &code, int v, int shift) {
    code |= (unsigned long long)(v & 3) << shift;
    return v >= 0 && v <= 3;
}
__device__ __forceinline__ int unpack2(unsigned long long code, int shift) { return (int)((code >> shift) & 3ull); }
// receivers of a departing particle along one axis (GPU_ArrangeFlights, kernels.cu:316-370)
// (count of receiving cells along one axis; `first` = the first of them)
__device__ __forceinline__ int receivers_g(double x, int c, int N, double h, int &first) {
    int n = 0;
    first = c;
#pragma unroll
    for (int d = -1; d <= 1; d++) {
        int j = c + d;
        if (j >= N) j -= N;
        else if (j < 0) j += N;
        double x0 = (double)j * h;
        if ((x0 <= x) && (x < x0 + h)) {
            if (n == 0) first = j;
            n++;
        }
    }
    return n;
}

// flyDirection (cell.h:694-701) + receivers: the particle's new cell.  In the
// fixed-order pass a particle has exactly one successor; the reference's
// rare boundary cases with zero or several receiving cells are counted
// (AdjStatus::ambiguous) and resolved to the first receiver / the old cell.
__device__ __forceinline__ int new_cell_plain(const Grid &g, int cell, int i, int l, int k, const double x[3],
                                              unsigned long long &amb) {
    const double hx = g.hx, hy = g.hy, hz = g.hz;
    const double x0 = (double)i * hx, y0 = (double)l * hy, z0 = (double)k * hz;
    double px = x[0], py = x[1], pz = x[2];
    int dxd = (((px > x0 + hx) && (px < x0 + 2 * hx)) || ((px < hx) && (i == g.nx - 1)))
                  ? 2 : (((px < x0) || ((px > g.lx - hx) && (i == 0))) ? 0 : 1);
    int dyd = (((py > y0 + hy) && (py < y0 + 2 * hy)) || ((py < hy) && (l == g.ny - 1)))
                  ? 2 : (((py < y0) || ((py > g.ly - hy) && (l == 0))) ? 0 : 1);
    int dzd = (((pz > z0 + hz) && (pz < z0 + 2 * hz)) || ((pz < hz) && (k == g.nz - 1)))
                  ? 2 : (((pz < z0) || ((pz > g.lz - hz) && (k == 0))) ? 0 : 1);
    if (dxd * 9 + dyd * 3 + dzd == 13) return cell;
    int rx, ry, rz;
    int nrx = receivers_g(px, i, g.nx, hx, rx);
    int nry = receivers_g(py, l, g.ny, hy, ry);
    int nrz = receivers_g(pz, k, g.nz, hz, rz);
    if (nrx * nry * nrz != 1) amb++;
    if (nrx == 0 || nry == 0 || nrz == 0) return cell;
    return g.cell_of(rx, ry, rz);
}

// ---- flat forward step of all particles (push + deposit + cell update).
// Four CTAs per SM (64 registers, some spills): the kernel gathers its field
// taps from global memory and waits on them; 32 warps per SM hide more of
// that than 16 at 96 registers (c3 forward about 9 % faster)
__global__ void __launch_bounds__(kT, 4) k_flat_push_plain(FlatParams P) {
    int64_t idx = spread_index(threadIdx.x);
    unsigned bad = 0;
    unsigned long long amb = 0;
    if (idx < P.off[P.nsp]) {
        const Grid &g = P.g;
        int s = species_of(P.off, P.nsp, idx);
        const FlatSp &S = P.sp[s];
        int64_t j = idx - P.off[s];
        int cell = S.cell[j];
        int i, l, k;
        g.cell_ijk(cell, i, l, k);
        double x[3] = {S.v[0][j], S.v[1][j], S.v[2][j]};
        double p[3] = {S.v[3][j], S.v[4][j], S.v[5][j]};
        const int c3[3] = {i, l, k};
        const unsigned long long rc = P.bmode == 2 ? P.branch[idx] : 0ull;
        unsigned long long code = 0ull;
        bool inrange = true;
        TapInts TI;
        if (P.bmode == 2) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                TI.tn[d] = unpack2(rc, 16 * d) + 1;
                TI.tc[d] = unpack2(rc, 16 * d + 2) + 1;
                TI.nI[d] = unpack2(rc, 16 * d + 4) + c3[d];
                TI.cI[d] = unpack2(rc, 16 * d + 6) + c3[d];
            }
        } else {
            tap_ints(g, i, l, k, x, TI);
        }
        Taps TT;
        taps_from(g, x, TI, TT);
        double F[6];
        if (!gather_fields_taps(g, P.E, P.H, i, l, k, x, TT, F, P.bmode != 2)) bad |= ST_STENCIL;
        if (P.Fout[0]) {
#pragma unroll
            for (int c = 0; c < 6; c++) P.Fout[c][idx] = F[c];
        }
        Boris B;
        boris_plain(S.q_m, g.tau, p, F, x, B);
        if (!(isfinite(B.pp[0]) && isfinite(B.pp[1]) && isfinite(B.pp[2]))) bad |= ST_NAN;
        const double o3[3] = {(double)i * g.hx, (double)l * g.hy, (double)k * g.hz};
        Split SP;
        if (P.bmode == 2) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                SP.i1[d] = unpack2(rc, 16 * d + 8) + 1;
                SP.i2[d] = unpack2(rc, 16 * d + 10) + 1;
            }
        } else {
            split_ints(g, x, B.x1, o3, SP);
        }
        split_from(g, x, B.x1, o3, SP);
        if (SP.m >= 1 && SP.m <= 7) {
            seg_plain(P.J, g, i, l, k, SP.i1, x, SP.x2, S.m, o3, bad);
            seg_plain(P.J, g, i, l, k, SP.i2, SP.x2, B.x1, S.m, o3, bad);
        } else {
            seg_plain(P.J, g, i, l, k, SP.i1, x, B.x1, S.m, o3, bad);
        }
        const double L3[3] = {g.lx, g.ly, g.lz};
        const int n3[3] = {g.nx, g.ny, g.nz};
        int wr[3];
        double xr[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            wr[d] = P.bmode == 2 ? unpack2(rc, 16 * d + 12) : wrap_choice(B.x1[d], L3[d]);
            xr[d] = apply_wrap(B.x1[d], L3[d], wr[d]);
        }
        const FlatOut &O = P.out[s];
        int ncell;
        if (P.bmode == 2) {
            int r[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                r[d] = c3[d] + unpack2(rc, 16 * d + 14) - 1;
                r[d] = r[d] < 0 ? r[d] + n3[d] : (r[d] >= n3[d] ? r[d] - n3[d] : r[d]);
            }
            ncell = g.cell_of(r[0], r[1], r[2]);
        } else {
            ncell = new_cell_plain(g, cell, i, l, k, xr, amb);
        }
        if (P.bmode == 1) {
            int r[3];
            g.cell_ijk(ncell, r[0], r[1], r[2]);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                int mv = r[d] - c3[d];
                mv = mv > 1 ? mv - n3[d] : (mv < -1 ? mv + n3[d] : mv);
                inrange &= pack2(code, TI.tn[d] - 1, 16 * d);
                inrange &= pack2(code, TI.tc[d] - 1, 16 * d + 2);
                inrange &= pack2(code, TI.nI[d] - c3[d], 16 * d + 4);
                inrange &= pack2(code, TI.cI[d] - c3[d], 16 * d + 6);
                inrange &= pack2(code, SP.i1[d] - 1, 16 * d + 8);
                inrange &= pack2(code, SP.i2[d] - 1, 16 * d + 10);
                inrange &= pack2(code, wr[d], 16 * d + 12);
                inrange &= pack2(code, mv + 1, 16 * d + 14);
            }
            P.branch[idx] = code;
            if (!inrange) bad |= ST_BRANCH_RANGE;
        }
        O.cell[j] = ncell;
        O.v[0][j] = xr[0]; O.v[1][j] = xr[1]; O.v[2][j] = xr[2];
        O.v[3][j] = B.pp[0]; O.v[4][j] = B.pp[1]; O.v[5][j] = B.pp[2];
    }
    if (bad) atomicOr(&P.st->flags, bad);
    if (amb) atomicAdd(&P.st->ambiguous, amb);
}

// ---- adjoint of the particle part of one step, first pass: recompute the
// push, transpose the deposit and the push; lambda_F goes to a scratch array
// (two CTAs per SM: the register cap spills a little but doubles the warps
// that hide the latency of the lambda_J gathers; measured faster)
template <bool STORED>
__global__ void __launch_bounds__(kT, 2) k_adj_push_plain(AdjParams A) {
    const FlatParams &P = A.f;
    int64_t idx = spread_index(threadIdx.x);
    if (idx >= P.off[P.nsp]) return;
    const Grid &g = P.g;
    int s = species_of(P.off, P.nsp, idx);
    const FlatSp &S = P.sp[s];
    const LamSp &Lm = A.lam[s];
    int64_t j = idx - P.off[s];
    int i, l, k;
    g.cell_ijk(S.cell[j], i, l, k);
    double x[3] = {S.v[0][j], S.v[1][j], S.v[2][j]};
    double p[3] = {S.v[3][j], S.v[4][j], S.v[5][j]};
    // recompute the forward
    double F[6];
    if (STORED) {
#pragma unroll
        for (int c = 0; c < 6; c++) F[c] = A.Fin[c][idx];
    } else {
        gather_fields(g, P.E, P.H, i, l, k, x, F);
    }
    Boris B;
    boris_plain(S.q_m, g.tau, p, F, x, B);
    const double o3[3] = {(double)i * g.hx, (double)l * g.hy, (double)k * g.hz};
    Split SP;
    split_plain(g, x, B.x1, o3, SP);
    // incoming adjoint of the particle's state after the step (Reflect: identity)
    double lx[3] = {Lm.v[0][j], Lm.v[1][j], Lm.v[2][j]};
    double lp[3] = {Lm.v[3][j], Lm.v[4][j], Lm.v[5][j]};
    double gx[3] = {0.0, 0.0, 0.0}, gn[3] = {lx[0], lx[1], lx[2]};
    // deposit transpose
    if (SP.m >= 1 && SP.m <= 7) {
        double g2[3] = {0.0, 0.0, 0.0};
        seg_plain_rev(A.LJ, g, i, l, k, SP.i1, x, SP.x2, S.m, o3, gx, g2);
        seg_plain_rev(A.LJ, g, i, l, k, SP.i2, SP.x2, B.x1, S.m, o3, g2, gn);
        split_rev(SP, x, B.x1, g2, gx, gn);
    } else {
        seg_plain_rev(A.LJ, g, i, l, k, SP.i1, x, B.x1, S.m, o3, gx, gn);
    }
    // x1 = x + tau g2 p'
    const double tau = g.tau;
    for (int d = 0; d < 3; d++) gx[d] += gn[d];
    double dot = gn[0] * B.pp[0] + gn[1] * B.pp[1] + gn[2] * B.pp[2];
    double g23 = B.g2 * B.g2 * B.g2;
    double lP[3];
    for (int d = 0; d < 3; d++) lP[d] = lp[d] + tau * B.g2 * gn[d] - tau * g23 * dot * B.pp[d];
    // p' = u' + t E
    double lF[6];
    for (int d = 0; d < 3; d++) lF[d] = B.t * lP[d];
    // u' = (s + b (b.s) + s x b) / sd
    const double *b = B.b, *sv = B.s, *up = B.up, *u = B.u;
    double bl = b[0] * lP[0] + b[1] * lP[1] + b[2] * lP[2];
    double bs = b[0] * sv[0] + b[1] * sv[1] + b[2] * sv[2];
    double lu_ = lP[0] * up[0] + lP[1] * up[1] + lP[2] * up[2];
    double inv = 1.0 / B.sd;
    double bxl[3] = {b[1] * lP[2] - b[2] * lP[1], b[2] * lP[0] - b[0] * lP[2], b[0] * lP[1] - b[1] * lP[0]};
    double lxs[3] = {lP[1] * sv[2] - lP[2] * sv[1], lP[2] * sv[0] - lP[0] * sv[2], lP[0] * sv[1] - lP[1] * sv[0]};
    double ls[3], lb[3];
    for (int d = 0; d < 3; d++) {
        ls[d] = (lP[d] + b[d] * bl + bxl[d]) * inv;
        lb[d] = (bs * lP[d] + bl * sv[d] + lxs[d] - 2.0 * lu_ * b[d]) * inv;
    }
    // s = u + u x b
    double lu[3] = {ls[0] + (b[1] * ls[2] - b[2] * ls[1]), ls[1] + (b[2] * ls[0] - b[0] * ls[2]),
                    ls[2] + (b[0] * ls[1] - b[1] * ls[0])};
    lb[0] += ls[1] * u[2] - ls[2] * u[1];
    lb[1] += ls[2] * u[0] - ls[0] * u[2];
    lb[2] += ls[0] * u[1] - ls[1] * u[0];
    // b = ps H, ps = t (1 + u^2)^-1/2
    double lps = 0.0;
    for (int d = 0; d < 3; d++) {
        lF[3 + d] = B.ps * lb[d];
        lps += lb[d] * F[3 + d];
    }
    double cps = -B.t * B.g1 * B.g1 * B.g1 * lps;
    for (int d = 0; d < 3; d++) lu[d] += cps * u[d];
    // u = p + t E
    double lpo[3];
    for (int d = 0; d < 3; d++) {
        lpo[d] = lu[d];
        lF[d] += B.t * lu[d];
    }
    for (int d = 0; d < 3; d++) {
        Lm.v[d][j] = gx[d];
        Lm.v[3 + d][j] = lpo[d];
    }
#pragma unroll
    for (int c = 0; c < 6; c++) A.LF[c][idx] = lF[c];
}

// ---- adjoint of the interpolation (second pass, few registers): scatter
// lambda_F into lambda_E / lambda_H and add F's position gradient to lambda_x.
// Four CTAs per SM (64 registers): it waits on global gathers, and 32 warps
// per SM hide them better than 16 (c3 backward 591 -> 500 ms for 100 steps)
__global__ void __launch_bounds__(kT, 4) k_adj_interp_plain(AdjParams A) {
    __shared__ int sHi[6 * kBoxNodes], sLo[6 * kBoxNodes];
    __shared__ int sRed[6 * (kT / 32)];
    __shared__ unsigned sMax[kT / 32], sMaxOut;
    __shared__ NodeBox sBox;
    const FlatParams &P = A.f;
    const Grid &g = P.g;
    int64_t idx = spread_index(threadIdx.x);
    bool valid = idx < P.off[P.nsp];
    int s = 0, i = 0, l = 0, k = 0;
    int64_t j = 0;
    double x[3] = {0.0, 0.0, 0.0};
    if (valid) {
        s = species_of(P.off, P.nsp, idx);
        const FlatSp &S = P.sp[s];
        j = idx - P.off[s];
        x[0] = S.v[0][j]; x[1] = S.v[1][j]; x[2] = S.v[2][j];
        g.cell_ijk(S.cell[j], i, l, k);
        valid = !(x[0] < 0 || x[1] < 0 || x[2] < 0);  // else the push saw zero fields
    }
    double lam6[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    float amax = 0.f;
    if (valid) {
#pragma unroll
        for (int c = 0; c < 6; c++) {
            lam6[c] = A.LF[c][idx];
            amax = fmaxf(amax, (float)fabs(lam6[c]));
        }
    }
    const NodeBox box = block_node_box(i, l, k, valid, sRed, &sBox);
    const float bmax = block_max_abs(amax, sMax, &sMaxOut);
    if (bmax == 0.f) return;  // no adjoint reaches the particles of this block
    const int E = box_exponent(bmax);
    const double inv_q = pow2_d(22 - E);
    for (int e = threadIdx.x; e < 6 * box.nodes; e += blockDim.x) sHi[e] = sLo[e] = 0;
    __syncthreads();
    if (valid) {
        Taps T;
        taps_plain(g, i, l, k, x, T);
        const size_t dX = (size_t)g.NY * g.pz, dY = g.pz, dZ = 1;
        double gx[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 6; c++) {
            int t[3];
            double w[3];
            const double lam = lam6[c];
            if (!comp_taps(T, c, t, w) || lam == 0.0) continue;
            size_t n = tap_node(g, i, l, k, t);
            const double *Arr = c < 3 ? P.E[c] : P.H[c - 3];
            double *LA = c < 3 ? A.LE[c] : A.LH[c - 3];
            const int b0 = box.nodes ? c * box.nodes + box_index(box, i + t[0] - 2, l + t[1] - 2, k + t[2] - 2) : 0;
            const double W0[2] = {w[0], 1. - w[0]}, W1[2] = {w[1], 1. - w[1]}, W2[2] = {w[2], 1. - w[2]};
            double gr[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int bb = 0; bb < 2; bb++)
#pragma unroll
                    for (int cc = 0; cc < 2; cc++) {
                        size_t m = n + a * dX + bb * dY + cc * dZ;
                        double v = Arr[m];
                        double add = lam * (W0[a] * W1[bb] * W2[cc]);
                        if (box.nodes) {
                            const int e = b0 + (a * box.by + bb) * box.bz + cc;
                            double vq = add * inv_q;
                            int hi = __double2int_rn(vq);
                            int lo = __double2int_rn((vq - (double)hi) * 0x1p22);
                            if (hi) atomicAdd(&sHi[e], hi);
                            if (lo) atomicAdd(&sLo[e], lo);
                        } else {
                            atomicAdd(&LA[m], add);
                        }
                        gr[0] += (a ? 1.0 : -1.0) * W1[bb] * W2[cc] * v;
                        gr[1] += (bb ? 1.0 : -1.0) * W0[a] * W2[cc] * v;
                        gr[2] += (cc ? 1.0 : -1.0) * W0[a] * W1[bb] * v;
                    }
            gx[0] += lam * gr[0] / g.hx;
            gx[1] += lam * gr[1] / g.hy;
            gx[2] += lam * gr[2] / g.hz;
        }
        const LamSp &Lm = A.lam[s];
        for (int d = 0; d < 3; d++) Lm.v[d][j] += gx[d];
    }
    if (box.nodes) {
        __syncthreads();
        double *const dst[6] = {A.LE[0], A.LE[1], A.LE[2], A.LH[0], A.LH[1], A.LH[2]};
        flush_node_box(box, sHi, sLo, pow2_d(E - 22), g, dst);
    }
}

// ------------------------------------------------------------- fields --
// Yee update ranges (MagneticFieldTrace, gpu_plasma.h:524-551; GetElectricFieldStartsDirs, gpu_plasma.h:286-304)
__device__ __forceinline__ bool in_H(const Grid &g, int c, int i, int l, int k) {
    if (i < 0 || l < 0 || k < 0) return false;
    if (c == 0) return i <= g.nx + 1 && l <= g.ny && k <= g.nz;
    if (c == 1) return i <= g.nx && l <= g.ny + 1 && k <= g.nz;
    return i <= g.nx && l <= g.ny && k <= g.nz + 1;
}
__device__ __forceinline__ bool in_E(const Grid &g, int c, int i, int l, int k) {
    if (i < 0 || l < 0 || k < 0 || i > g.nx || l > g.ny || k > g.nz) return false;
    if (c == 0) return l >= 1 && k >= 1;
    if (c == 1) return i >= 1 && k >= 1;
    return i >= 1 && l >= 1;
}

struct FieldAdj {
    Grid g;
    double cx, cy, cz, tau;
    double *LE[3], *LH[3], *LJ[3], *LQ[3];
};

// E update transpose (5) and the start of B completion's transpose (4):
//   lambda_J = -tau lambda_E on the E ranges, lambda_H += C^T lambda_E,
//   lambda_Q = lambda_H (new) on the H ranges
__global__ void k_adj_e_update(FieldAdj A) {
    const Grid &g = A.g;
    int k = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y, i = blockIdx.z;
    if (k >= g.NZ) return;
    size_t m = g.node(i, l, k);
    auto LEv = [&](int c, int di, int dl, int dk) -> double {
        return in_E(g, c, i + di, l + dl, k + dk) ? A.LE[c][g.node(i + di, l + dl, k + dk)] : 0.0;
    };
    double ex0 = LEv(0, 0, 0, 0), ey0 = LEv(1, 0, 0, 0), ez0 = LEv(2, 0, 0, 0);
    A.LJ[0][m] = -A.tau * ex0;
    A.LJ[1][m] = -A.tau * ey0;
    A.LJ[2][m] = -A.tau * ez0;
    double hx = A.LH[0][m] + A.cz * (ey0 - LEv(1, 0, 0, 1)) - A.cy * (ez0 - LEv(2, 0, 1, 0));
    double hy = A.LH[1][m] - A.cz * (ex0 - LEv(0, 0, 0, 1)) + A.cx * (ez0 - LEv(2, 1, 0, 0));
    double hz = A.LH[2][m] + A.cy * (ex0 - LEv(0, 0, 1, 0)) - A.cx * (ey0 - LEv(1, 1, 0, 0));
    A.LH[0][m] = hx;
    A.LH[1][m] = hy;
    A.LH[2][m] = hz;
    A.LQ[0][m] = in_H(g, 0, i, l, k) ? hx : 0.0;
    A.LQ[1][m] = in_H(g, 1, i, l, k) ? hy : 0.0;
    A.LQ[2][m] = in_H(g, 2, i, l, k) ? hz : 0.0;
}

// transpose of the B half step (1): lambda_Q += lambda_H_a on the H ranges,
// lambda_E += A^T lambda_Q (gather form: each E node collects from the Q
// nodes whose difference reads it)
__global__ void k_adj_b_half(FieldAdj A) {
    const Grid &g = A.g;
    int k = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y, i = blockIdx.z;
    if (k >= g.NZ) return;
    size_t m = g.node(i, l, k);
    auto LQt = [&](int c, int di, int dl, int dk) -> double {
        int a = i + di, b = l + dl, cc = k + dk;
        if (!in_H(g, c, a, b, cc)) return 0.0;
        size_t q = g.node(a, b, cc);
        return A.LQ[c][q] + A.LH[c][q];
    };
    double qx = LQt(0, 0, 0, 0), qy = LQt(1, 0, 0, 0), qz = LQt(2, 0, 0, 0);
    // Qx = 0.5 (cz (Ey[+z] - Ey) - cy (Ez[+y] - Ez))
    // Qy = 0.5 (cx (Ez[+x] - Ez) - cz (Ex[+z] - Ex))
    // Qz = 0.5 (cy (Ex[+y] - Ex) - cx (Ey[+x] - Ey))
    double lex = -0.5 * A.cz * (LQt(1, 0, 0, -1) - qy) + 0.5 * A.cy * (LQt(2, 0, -1, 0) - qz);
    double ley = 0.5 * A.cz * (LQt(0, 0, 0, -1) - qx) - 0.5 * A.cx * (LQt(2, -1, 0, 0) - qz);
    double lez = -0.5 * A.cy * (LQt(0, 0, -1, 0) - qx) + 0.5 * A.cx * (LQt(1, -1, 0, 0) - qy);
    A.LE[0][m] += lex;
    A.LE[1][m] += ley;
    A.LE[2][m] += lez;
}

// H_a = H + Q(E) (the forward B half step, out of place, same rounding)
__global__ void k_h_half(Grid g, const double *__restrict__ Ex, const double *__restrict__ Ey,
                         const double *__restrict__ Ez, const double *__restrict__ Hx, const double *__restrict__ Hy,
                         const double *__restrict__ Hz, double *Ax, double *Ay, double *Az, double cx, double cy,
                         double cz) {
    int k = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y, i = blockIdx.z;
    if (k >= g.NZ) return;
    size_t n = g.node(i, l, k), sx = (size_t)g.NY * g.pz, sy = g.pz;
    double hx = Hx[n], hy = Hy[n], hz = Hz[n];
    if (i <= g.nx + 1 && l <= g.ny && k <= g.nz) hx += 0.5 * (cz * (Ey[n + 1] - Ey[n]) - cy * (Ez[n + sy] - Ez[n]));
    if (i <= g.nx && l <= g.ny + 1 && k <= g.nz) hy += 0.5 * (cx * (Ez[n + sx] - Ez[n]) - cz * (Ex[n + 1] - Ex[n]));
    if (i <= g.nx && l <= g.ny && k <= g.nz + 1) hz += 0.5 * (cy * (Ex[n + sy] - Ex[n]) - cx * (Ey[n + sx] - Ey[n]));
    Ax[n] = hx;
    Ay[n] = hy;
    Az[n] = hz;
}

// lines of one axis (getGlobalBoundaryCellNumber, cell.h:885-889)
__device__ __forceinline__ void line_g(const Grid &g, int dir, int a, int b, size_t &base, size_t &stride) {
    if (dir == 0) { base = (size_t)a * g.pz + b; stride = (size_t)g.NY * g.pz; }
    else if (dir == 1) { base = (size_t)a * g.NY * g.pz + b; stride = g.pz; }
    else { base = ((size_t)a * g.NY + b) * g.pz; stride = 1; }
}

// transpose of the J fold along one axis (periodicCurrentElement, kernels.cu:1124-1146)
__global__ void k_adj_j_fold(Grid g, double *Lx, double *Ly, double *Lz, int dir) {
    int A = dir == 0 ? g.NY : g.NX;
    int B = dir == 2 ? g.NY : g.NZ;
    int N = dir == 0 ? g.NX : (dir == 1 ? g.NY : g.NZ);
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= A * B) return;
    size_t base, st;
    line_g(g, dir, idx / B, idx % B, base, st);
    double *L3[3] = {Lx, Ly, Lz};
    for (int comp = 0; comp < 3; comp++) {
        double *L = L3[comp] + base;
        size_t n1 = st, nm1 = (size_t)(N - 1) * st, nm2 = (size_t)(N - 2) * st;
        // forward: J1 += J[N-1] (dir != comp); J[N-1] = J1 (not y/y); J0 += J[N-2]; J[N-2] = J0
        L[0] += L[nm2];
        L[nm2] = 0.0;
        L[nm2] += L[0];
        if (dir != 1 || comp != 1) {
            L[n1] += L[nm1];
            L[nm1] = 0.0;
        }
        if (dir != comp) L[nm1] += L[n1];
    }
}

// transpose of the E ghost copies E[0] = E[N], E[N+1] = E[1] (periodicElement, kernels.cu:1104-1110)
struct GPass {
    double *L;
    int dir, s1, e1, s2, e2, N;
};
struct GPasses {
    GPass p[3];
    int n;
};
__global__ void k_adj_ghosts(Grid g, GPasses P) {
    if ((int)blockIdx.y >= P.n) return;
    GPass q = P.p[blockIdx.y];
    int A = q.e1 - q.s1 + 1, B = q.e2 - q.s2 + 1;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= A * B) return;
    size_t base, st;
    line_g(g, q.dir, q.s1 + idx / B, q.s2 + idx % B, base, st);
    double *L = q.L + base;
    size_t n1 = st, nN = (size_t)q.N * st, nN1 = (size_t)(q.N + 1) * st;
    L[n1] += L[nN1];
    L[nN1] = 0.0;
    L[nN] += L[0];
    L[0] = 0.0;
}

// loss injection: lambda_E_c += 2 w E_c on nodes 1..N; history sums
template <typename T>
__global__ void k_inject(Grid g, const T *__restrict__ E, double *LE, double w2) {
    int k = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y, i = blockIdx.z;
    if (k < 1 || k > g.nz || l < 1 || l > g.ny || i < 1 || i > g.nx) return;
    size_t n = g.node(i, l, k);
    LE[n] += w2 * (double)E[n];
}

template <typename T>
__global__ void k_history(Grid g, const T *__restrict__ Ex, const T *__restrict__ Ey, const T *__restrict__ Ez,
                          double *out3) {
    __shared__ double red[3][kT / 32];
    int k = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y, i = blockIdx.z;
    double a = 0.0, b = 0.0, c = 0.0;
    if (k >= 1 && k <= g.nz && l >= 1 && l <= g.ny && i >= 1 && i <= g.nx) {
        size_t n = g.node(i, l, k);
        double ex = (double)Ex[n], ey = (double)Ey[n], ez = (double)Ez[n];
        a = ex * ex; b = ey * ey; c = ez * ez;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = a; red[1][w] = b; red[2][w] = c; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int q = 0; q < nw; q++) s += red[threadIdx.x][q];
        atomicAdd(&out3[threadIdx.x], s);
    }
}

// bins -> flat order (tile by tile, slot order): packed cell and FP64 values
__global__ void k_flat_gather_plain(SpeciesView S, const int64_t *__restrict__ d0, int *cell, double *x, double *y,
                                    double *z, double *px, double *py, double *pz) {
    int t = blockIdx.x;
    int start = S.tile_start[t], n = S.tile_count[t];
    int64_t base = d0[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int slot = start + j;
        int64_t d = base + j;
        cell[d] = S.cell[slot];
        x[d] = S.x[slot]; y[d] = S.y[slot]; z[d] = S.z[slot];
        px[d] = S.px[slot]; py[d] = S.py[slot]; pz[d] = S.pz[slot];
    }
}

// p += eps * dp for one species, dp interleaved (px, py, pz) in the order of
// pic_get_particles (tiles in order, slots in order)
__global__ void k_perturb_momenta(SpeciesView S, int mixed, const int64_t *__restrict__ d0,
                                  const double *__restrict__ dp, double eps) {
    const int t = blockIdx.x;
    const int start = S.tile_start[t], n = S.tile_count[t];
    const int64_t base = d0[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int slot = start + j;
        const double *q = dp + 3 * (base + j);
        if (mixed) {
            S.fx[slot] = (float)((double)S.fx[slot] + eps * q[0]);
            S.fy[slot] = (float)((double)S.fy[slot] + eps * q[1]);
            S.fz[slot] = (float)((double)S.fz[slot] + eps * q[2]);
        } else {
            S.px[slot] += eps * q[0];
            S.py[slot] += eps * q[1];
            S.pz[slot] += eps * q[2];
        }
    }
}

// d_drift and d_vth partial sums: out[0..2] += lambda_p, out[3] += lambda_p . (p - drift)
__global__ void k_param_grads(int64_t n, const double *__restrict__ lpx, const double *__restrict__ lpy,
                              const double *__restrict__ lpz, const double *__restrict__ px,
                              const double *__restrict__ py, const double *__restrict__ pz, double dx, double dy,
                              double dz, double *out4) {
    __shared__ double red[4][kT / 32];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        a[0] += lpx[j];
        a[1] += lpy[j];
        a[2] += lpz[j];
        a[3] += lpx[j] * (px[j] - dx) + lpy[j] * (py[j] - dy) + lpz[j] * (pz[j] - dz);
    }
    for (int q = 0; q < 4; q++)
        for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_down_sync(0xffffffffu, a[q], o);
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; q++) red[q][w] = a[q];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[threadIdx.x][q];
        atomicAdd(&out4[threadIdx.x], s);
    }
}

// interleave (px, py, pz) of one species into n x 3
__global__ void k_interleave(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                             const double *__restrict__ c, double *out) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    out[3 * j] = a[j];
    out[3 * j + 1] = b[j];
    out[3 * j + 2] = c[j];
}

inline dim3 node_grid(const Grid &g) { return dim3((g.NZ + 31) / 32, g.NY, g.NX); }
inline unsigned blocks_of(int64_t n) { return (unsigned)((n + kT - 1) / kT); }

}  // namespace

// ======================================================== host: buffers ==
// One particle state of the whole population, carved from one allocation:
// per species the packed cells, then 6 value arrays, each 256-byte aligned.
size_t adj_state_bytes(const AdjState &A) {
    size_t b = 0;
    for (int s = 0; s < A.nsp; s++) {
        b += align256((size_t)A.n[s] * sizeof(int));
        b += 6 * align256((size_t)A.n[s] * A.elem);
    }
    return b;
}
void adj_state_view(const AdjState &A, char *base, int *cell[kMaxSpecies], void *v[kMaxSpecies][6]) {
    size_t o = 0;
    for (int s = 0; s < A.nsp; s++) {
        cell[s] = (int *)(base + o);
        o += align256((size_t)A.n[s] * sizeof(int));
        for (int a = 0; a < 6; a++) {
            v[s][a] = base + o;
            o += align256((size_t)A.n[s] * A.elem);
        }
    }
}

}  // namespace pic

using namespace pic;
using namespace pic_host;

namespace {

// ---- plain-form launch helpers
FlatParams flat_params(pic_handle *h, AdjState &A, char *state, void *const F[PIC_FIELD_COUNT],
                       char *out = nullptr) {
    FlatParams P;
    memset(&P, 0, sizeof(P));
    P.g = h->g;
    P.nsp = A.nsp;
    int *cell[kMaxSpecies];
    void *v[kMaxSpecies][6];
    adj_state_view(A, state, cell, v);
    P.off[0] = 0;
    for (int s = 0; s < A.nsp; s++) {
        P.sp[s].n = A.n[s];
        P.sp[s].q_m = h->sp[s].v.q_m;
        P.sp[s].m = h->sp[s].v.m;
        P.sp[s].cell = cell[s];
        for (int a = 0; a < 6; a++) P.sp[s].v[a] = (double *)v[s][a];
        P.off[s + 1] = P.off[s] + A.n[s];
    }
    for (int c = 0; c < 3; c++) {
        P.E[c] = (const double *)F[PIC_EX + c];
        P.H[c] = (const double *)F[PIC_HX + c];
        P.J[c] = (double *)F[PIC_JX + c];
    }
    adj_state_view(A, out ? out : state, cell, v);
    for (int s = 0; s < A.nsp; s++) {
        P.out[s].cell = cell[s];
        for (int a = 0; a < 6; a++) P.out[s].v[a] = (double *)v[s][a];
    }
    P.st = A.st;
    P.branch = A.step_branch;
    P.bmode = A.step_branch ? A.step_bmode : 0;
    return P;
}

int64_t total_particles(const AdjState &A) {
    int64_t t = 0;
    for (int s = 0; s < A.nsp; s++) t += A.n[s];
    return t;
}

// one forward step of the flat state on the field set F (plain): particles
// read from `state`, written to `out` (the same buffer when out is null)
int flat_step_plain(pic_handle *h, AdjState &A, char *state, void *const F[PIC_FIELD_COUNT], char *out = nullptr,
                    double *Fout = nullptr) {
    const Grid &g = h->g;
    cudaStream_t s = h->stream;
    yee_b_half_plain(g, (double *const *)F, s);
    size_t nodes = g.nodes_pitched();
    for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(F[PIC_JX + c], 0, nodes * sizeof(double), s), "zero J");
    FlatParams P = flat_params(h, A, state, F, out);
    int64_t n = total_particles(A);
    for (int c = 0; c < 6; c++) P.Fout[c] = Fout ? Fout + (size_t)c * n : nullptr;
    if (n > 0) k_flat_push_plain<<<blocks_of(n), kT, 0, s>>>(P);
    CK(cudaGetLastError(), "flat push");
    j_fold(g, (double *)F[PIC_JX], (double *)F[PIC_JY], (double *)F[PIC_JZ], s);
    yee_b_complete_plain(g, (double *const *)F, s);
    yee_e_update_plain(g, (double *const *)F, s);
    e_ghosts_plain(g, (double *)F[PIC_EX], (double *)F[PIC_EY], (double *)F[PIC_EZ],
                   h->cfg.ghosts == PIC_GHOSTS_PERIODIC, s);
    CK(cudaGetLastError(), "flat step fields");
    return PIC_OK;
}

// ghost passes of e_ghosts_t (PeriodicBoundaries arguments, gpu_plasma.h:486-505), as two launches
void ghost_passes(const Grid &g, double *const L[3], int periodic, GPasses &A, GPasses &B, int &maxn) {
    A = GPasses{};
    B = GPasses{};
    maxn = 0;
    int Nx = g.nx, Ny = g.ny, Nz = g.nz;
    auto add = [&](GPasses &P, double *E, int dir, int s1, int e1, int s2, int e2, int N) {
        P.p[P.n++] = GPass{E, dir, s1, e1, s2, e2, N};
        int n = (e1 - s1 + 1) * (e2 - s2 + 1);
        if (n > maxn) maxn = n;
    };
    if (periodic) add(A, L[0], 1, 0, Nx, 1, Nz, Ny);
    add(A, L[1], 0, 0, Ny, 1, Nz, Nx);
    add(A, L[2], 0, 1, Ny, 0, Nz, Nx);
    add(B, L[0], 2, 0, Nx, 0, Ny + 1, Nz);
    add(B, L[1], 2, 0, Nx + 1, 0, Ny, Nz);
    if (periodic) add(B, L[2], 1, 0, Nx + 1, 0, Nz, Ny);
}

int check_adj_status(pic_handle *h, AdjState &A, const char *where) {
    AdjStatus st;
    CK(cudaMemcpyAsync(&st, A.st, sizeof(st), cudaMemcpyDeviceToHost, h->stream), "status");
    CK(cudaStreamSynchronize(h->stream), "sync");
    A.ambiguous = st.ambiguous;
    if (st.flags & ST_NAN) return set_err(h, PIC_ERR_NAN, "non-finite momentum in the differentiable run");
    if (st.flags & ST_BRANCH_RANGE)
        return set_err(h, PIC_ERR_STATE, "branch recording: a discrete choice outside its recorded range");
    if (st.flags & ST_STENCIL) {
        char msg[160];
        snprintf(msg, sizeof(msg), "%s: a particle moved more than half a cell in one step", where);
        return set_err(h, PIC_ERR_STENCIL, msg);
    }
    return PIC_OK;
}

int adj_alloc(pic_handle *h, void **p, size_t bytes, const char *what) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 256);
    if (e != cudaSuccess) {
        char msg[200];
        snprintf(msg, sizeof(msg), "differentiable run: cannot allocate %s (%.2f GB); use a larger ckpt_every or "
                 "fewer particles", what, bytes / 1e9);
        cudaGetLastError();
        return set_err(h, PIC_ERR_NOMEM, msg);
    }
    return PIC_OK;
}

}  // namespace

namespace pic_host {

void adj_free(pic_handle *h) {
    if (!h || !h->adj) return;
    AdjState *A = h->adj;
    void *bufs[] = {A->cur, A->ckp, A->ckf, A->segp, A->segf, A->subp, A->subf, A->lamp, A->lamf, A->rf, A->ha,
                    A->hist, A->st, A->red, A->lamF, A->segF, A->branch};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (A->e0) cudaEventDestroy(A->e0);
    if (A->e1) cudaEventDestroy(A->e1);
    delete A;
    h->adj = nullptr;
}

}  // namespace pic_host

// ====================================================== host: forward ==
namespace {

// field arrays of one state in the form's type: E, H (6 arrays)
inline size_t field_bytes(const pic_handle *h) {
    return h->g.nodes_pitched() * (h->mixed ? sizeof(float) : sizeof(double));
}
// recompute field set: E, H in the form's type, then J (and Q) in FP64
void rf_view(pic_handle *h, AdjState &A, void *RF[PIC_FIELD_COUNT]) {
    const size_t fb = field_bytes(h), db = h->g.nodes_pitched() * sizeof(double);
    for (int a = 0; a < PIC_FIELD_COUNT; a++)
        RF[a] = a < 6 ? A.rf + a * fb : A.rf + 6 * fb + (a - 6) * db;
    if (h->mixed) RF[PIC_QX] = RF[PIC_QY] = RF[PIC_QZ] = nullptr;
}

MixParams mix_params(pic_handle *h, AdjState &A, char *state, void *const F[PIC_FIELD_COUNT], char *out) {
    MixParams P;
    memset(&P, 0, sizeof(P));
    P.g = h->g;
    P.nsp = A.nsp;
    int *cell[kMaxSpecies];
    void *v[kMaxSpecies][6];
    adj_state_view(A, state, cell, v);
    P.off[0] = 0;
    for (int s = 0; s < A.nsp; s++) {
        P.sp[s].n = A.n[s];
        P.sp[s].q_m = h->sp[s].v.q_m;
        P.sp[s].m = h->sp[s].v.m;
        P.sp[s].cell = cell[s];
        for (int a = 0; a < 6; a++) P.sp[s].v[a] = (float *)v[s][a];
        P.off[s + 1] = P.off[s] + A.n[s];
    }
    adj_state_view(A, out ? out : state, cell, v);
    for (int s = 0; s < A.nsp; s++) {
        P.out[s].cell = cell[s];
        for (int a = 0; a < 6; a++) P.out[s].v[a] = (float *)v[s][a];
    }
    for (int c = 0; c < 3; c++) {
        P.E[c] = (const float *)F[PIC_EX + c];
        P.H[c] = (const float *)F[PIC_HX + c];
        P.J[c] = (double *)F[PIC_JX + c];
    }
    P.st = A.st;
    return P;
}

// one forward step of the fixed-order state on the field set F: particles
// read from `state`, written to `out` (same buffer when null); Fout, when
// given, receives the interpolated fields of every particle
int flat_step(pic_handle *h, AdjState &A, char *state, void *const F[PIC_FIELD_COUNT], char *out, void *Fout) {
    if (!h->mixed) return flat_step_plain(h, A, state, F, out, (double *)Fout);
    const Grid &g = h->g;
    cudaStream_t s = h->stream;
    float *const *E = (float *const *)&F[PIC_EX];
    float *const *H = (float *const *)&F[PIC_HX];
    yee_b_half_mixed(g, E, H, s);
    const size_t nodes = g.nodes_pitched();
    for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(F[PIC_JX + c], 0, nodes * sizeof(double), s), "zero J");
    MixParams P = mix_params(h, A, state, F, out);
    const int64_t n = total_particles(A);
    for (int c = 0; c < 6; c++) P.Fout[c] = Fout ? (float *)Fout + (size_t)c * n : nullptr;
    CK(launch_flat_push_mixed(P, s), "flat push");
    j_fold(g, (double *)F[PIC_JX], (double *)F[PIC_JY], (double *)F[PIC_JZ], s);
    yee_b_half_mixed(g, E, H, s);  // completion: the same Q again
    yee_e_update_mixed(g, E, H, (double *const *)&F[PIC_JX], s);
    e_ghosts_mixed(g, E[0], E[1], E[2], h->cfg.ghosts == PIC_GHOSTS_PERIODIC, s);
    CK(cudaGetLastError(), "flat step fields");
    return PIC_OK;
}

int forward_run(pic_handle *h, AdjState &A) {
    const Grid &g = h->g;
    cudaStream_t st = h->stream;
    const size_t fbytes = field_bytes(h);
    CK(cudaEventRecord(A.e0, st), "event");
    for (int n = 0; n < A.steps; n++) {
        if (n % A.K == 0) {
            int c = n / A.K;
            CK(cudaMemcpyAsync(A.ckp + (size_t)c * A.pbytes, A.cur, A.pbytes, cudaMemcpyDeviceToDevice, st), "ckpt");
            for (int a = 0; a < 6; a++)
                CK(cudaMemcpyAsync(A.ckf + ((size_t)c * 6 + a) * fbytes, h->f[PIC_EX + a], fbytes,
                                   cudaMemcpyDeviceToDevice, st), "ckpt fields");
        }
        const size_t np_all = (size_t)total_particles(A);
        if (A.branch_mode == 1) {
            A.step_branch = A.branch + (size_t)n * np_all;
            A.step_bmode = 1;
        } else if (A.branch_mode == 2) {
            A.step_branch = const_cast<unsigned long long *>(A.branch_src) + (size_t)n * np_all;
            A.step_bmode = 2;
        }
        int rc = flat_step(h, A, A.cur, h->f, nullptr, nullptr);
        A.step_branch = nullptr;
        A.step_bmode = 0;
        if (rc) return rc;
        if (h->mixed)
            k_history<float><<<node_grid(g), 32, 0, st>>>(g, (const float *)h->f[PIC_EX], (const float *)h->f[PIC_EY],
                                                          (const float *)h->f[PIC_EZ], A.hist + 3 * n);
        else
            k_history<double><<<node_grid(g), 32, 0, st>>>(g, (const double *)h->f[PIC_EX],
                                                           (const double *)h->f[PIC_EY],
                                                           (const double *)h->f[PIC_EZ], A.hist + 3 * n);
        CK(cudaGetLastError(), "history");
    }
    CK(cudaEventRecord(A.e1, st), "event");
    return PIC_OK;
}

// reverse of step n: EHn = E_n, H_n of the step (form's type, 6 arrays),
// Enext = E after the step, Fin = the push's interpolated fields (or null)
int reverse_step(pic_handle *h, AdjState &A, const pic_loss &L, int n, char *state, const char *EHn,
                 const char *Enext, const void *Fin) {
    const Grid &g = h->g;
    cudaStream_t st = h->stream;
    const size_t N = g.nodes_pitched();
    const size_t fb = field_bytes(h);
    double *LE[3], *LH[3], *LJ[3], *LQ[3];
    for (int c = 0; c < 3; c++) {
        LE[c] = A.lamf + (0 + c) * N;
        LH[c] = A.lamf + (3 + c) * N;
        LJ[c] = A.lamf + (6 + c) * N;
        LQ[c] = A.lamf + (9 + c) * N;
    }
    // loss injection at E_{n+1}
    if (n >= A.steps - L.window) {
        double w2 = 2.0 * g.hx * g.hy * g.hz;
        const char *Ec = Enext + (size_t)L.field * fb;
        if (h->mixed) k_inject<float><<<node_grid(g), 32, 0, st>>>(g, (const float *)Ec, LE[L.field], w2);
        else k_inject<double><<<node_grid(g), 32, 0, st>>>(g, (const double *)Ec, LE[L.field], w2);
    }
    // ghost copies (second launch first)
    GPasses GA, GB;
    int maxn;
    ghost_passes(g, LE, h->cfg.ghosts == PIC_GHOSTS_PERIODIC, GA, GB, maxn);
    dim3 gg((maxn + 127) / 128, 3);
    k_adj_ghosts<<<gg, 128, 0, st>>>(g, GB);
    k_adj_ghosts<<<gg, 128, 0, st>>>(g, GA);
    FieldAdj FA;
    FA.g = g;
    FA.cx = g.tau / g.hx;
    FA.cy = g.tau / g.hy;
    FA.cz = g.tau / g.hz;
    FA.tau = g.tau;
    for (int c = 0; c < 3; c++) { FA.LE[c] = LE[c]; FA.LH[c] = LH[c]; FA.LJ[c] = LJ[c]; FA.LQ[c] = LQ[c]; }
    k_adj_e_update<<<node_grid(g), 32, 0, st>>>(FA);
    for (int dir = 2; dir >= 0; dir--) {
        int a = dir == 0 ? g.NY : g.NX, b = dir == 2 ? g.NY : g.NZ;
        k_adj_j_fold<<<(a * b + 127) / 128, 128, 0, st>>>(g, LJ[0], LJ[1], LJ[2], dir);
    }
    const int64_t np = total_particles(A);
    if (!h->mixed) {
        // H_a of step n
        const double *En = (const double *)EHn, *Hn = (const double *)EHn + 3 * N;
        double *Ha = (double *)A.ha;
        k_h_half<<<node_grid(g), 32, 0, st>>>(g, En, En + N, En + 2 * N, Hn, Hn + N, Hn + 2 * N, Ha, Ha + N,
                                              Ha + 2 * N, FA.cx, FA.cy, FA.cz);
        void *F[PIC_FIELD_COUNT] = {};
        for (int c = 0; c < 3; c++) {
            F[PIC_EX + c] = (void *)(En + c * N);
            F[PIC_HX + c] = (void *)(Ha + c * N);
        }
        AdjParams P;
        memset(&P, 0, sizeof(P));
        P.f = flat_params(h, A, state, F);
        size_t o = 0;
        for (int s = 0; s < A.nsp; s++) {
            for (int a = 0; a < 6; a++) P.lam[s].v[a] = (double *)A.lamp + o + (size_t)a * A.n[s];
            o += 6 * (size_t)A.n[s];
        }
        for (int c = 0; c < 3; c++) { P.LJ[c] = LJ[c]; P.LE[c] = LE[c]; P.LH[c] = LH[c]; }
        for (int c = 0; c < 6; c++) {
            P.LF[c] = (double *)A.lamF + (size_t)c * np;
            P.Fin[c] = Fin ? (const double *)Fin + (size_t)c * np : nullptr;
        }
        if (np > 0) {
            if (Fin) k_adj_push_plain<true><<<blocks_of(np), kT, 0, st>>>(P);
            else k_adj_push_plain<false><<<blocks_of(np), kT, 0, st>>>(P);
            k_adj_interp_plain<<<blocks_of(np), kT, 0, st>>>(P);
        }
    } else {
        const float *En = (const float *)EHn, *Hn = (const float *)EHn + 3 * N;
        float *Ha = (float *)A.ha;
        CK(launch_h_half_mixed(g, En, Hn, Ha, N, st), "half step");
        void *F[PIC_FIELD_COUNT] = {};
        for (int c = 0; c < 3; c++) {
            F[PIC_EX + c] = (void *)(En + c * N);
            F[PIC_HX + c] = (void *)(Ha + c * N);
        }
        MixParams P = mix_params(h, A, state, F, nullptr);
        size_t o = 0;
        for (int s = 0; s < A.nsp; s++) {
            for (int a = 0; a < 6; a++) P.lam[s][a] = (float *)A.lamp + o + (size_t)a * A.n[s];
            o += 6 * (size_t)A.n[s];
        }
        for (int c = 0; c < 3; c++) { P.LJ[c] = LJ[c]; P.LE[c] = LE[c]; P.LH[c] = LH[c]; }
        for (int c = 0; c < 6; c++) {
            P.LF[c] = (float *)A.lamF + (size_t)c * np;
            P.Fin[c] = Fin ? (const float *)Fin + (size_t)c * np : nullptr;
        }
        CK(launch_adj_particles_mixed(P, st), "adjoint particles");
    }
    k_adj_b_half<<<node_grid(g), 32, 0, st>>>(FA);
    CK(cudaGetLastError(), "reverse step");
    return PIC_OK;
}

int backward_run(pic_handle *h, AdjState &A, const pic_loss &L) {
    const Grid &g = h->g;
    cudaStream_t st = h->stream;
    const size_t N = g.nodes_pitched();
    const size_t fbytes = field_bytes(h);
    const int64_t np = total_particles(A);
    const size_t Fstep = (size_t)6 * np * A.elem;  // interpolated fields of one step
    CK(cudaMemsetAsync(A.lamp, 0, A.lamp_bytes, st), "zero lambda");
    CK(cudaMemsetAsync(A.lamf, 0, 12 * N * sizeof(double), st), "zero lambda fields");
    void *RF[PIC_FIELD_COUNT];
    rf_view(h, A, RF);
    CK(cudaEventRecord(A.e0, st), "event");
    const size_t ehb = 6 * fbytes;  // E and H of one state (the first arrays of rf)
    for (int seg = A.nseg - 1; seg >= 0; seg--) {
        const int start = seg * A.K, end = std::min(start + A.K, A.steps), len = end - start;
        const int K2 = A.K2, nsub = (len + K2 - 1) / K2;
        if (nsub > 1) {
            // second level: recompute the segment once, keeping the state and E/H at
            // the start of every sub-segment (the running state lives in segp[0])
            CK(cudaMemcpyAsync(A.segp, A.ckp + (size_t)seg * A.pbytes, A.pbytes, cudaMemcpyDeviceToDevice, st),
               "restore");
            CK(cudaMemcpyAsync(A.rf, A.ckf + (size_t)seg * ehb, ehb, cudaMemcpyDeviceToDevice, st), "restore fields");
            for (int j = 0; j < len; j++) {
                if (j % K2 == 0) {
                    const int q = j / K2;
                    CK(cudaMemcpyAsync(A.subp + (size_t)q * A.pbytes, A.segp, A.pbytes, cudaMemcpyDeviceToDevice, st),
                       "sub-checkpoint");
                    CK(cudaMemcpyAsync(A.subf + (size_t)q * ehb, A.rf, ehb, cudaMemcpyDeviceToDevice, st),
                       "sub-checkpoint fields");
                    if (q == nsub - 1) break;  // the last sub-segment starts here
                }
                int rc = flat_step(h, A, A.segp, RF, nullptr, nullptr);
                if (rc) return rc;
            }
        }
        for (int q = nsub - 1; q >= 0; q--) {
            const int s0 = start + q * K2, s1 = std::min(s0 + K2, end), slen = s1 - s0;
            const char *sp = nsub > 1 ? A.subp + (size_t)q * A.pbytes : A.ckp + (size_t)seg * A.pbytes;
            const char *sf = nsub > 1 ? A.subf + (size_t)q * ehb : A.ckf + (size_t)seg * ehb;
            CK(cudaMemcpyAsync(A.segp, sp, A.pbytes, cudaMemcpyDeviceToDevice, st), "restore");
            CK(cudaMemcpyAsync(A.rf, sf, ehb, cudaMemcpyDeviceToDevice, st), "restore fields");
            for (int j = 0; j < slen; j++) {
                CK(cudaMemcpyAsync(A.segf + (size_t)j * ehb, A.rf, ehb, cudaMemcpyDeviceToDevice, st), "keep fields");
                void *Fj = A.segF ? (char *)A.segF + (size_t)j * Fstep : nullptr;
                int rc = flat_step(h, A, A.segp + (size_t)j * A.pbytes, RF, A.segp + (size_t)(j + 1) * A.pbytes, Fj);
                if (rc) return rc;
            }
            CK(cudaMemcpyAsync(A.segf + (size_t)slen * ehb, A.rf, ehb, cudaMemcpyDeviceToDevice, st), "keep fields");
            for (int j = slen - 1; j >= 0; j--) {
                int rc = reverse_step(h, A, L, s0 + j, A.segp + (size_t)j * A.pbytes, A.segf + (size_t)j * ehb,
                                      A.segf + (size_t)(j + 1) * ehb,
                                      A.segF ? (const char *)A.segF + (size_t)j * Fstep : nullptr);
                if (rc) return rc;
            }
        }
    }
    CK(cudaEventRecord(A.e1, st), "event");
    return PIC_OK;
}

}  // namespace

// ============================================================ C ABI ==
extern "C" {

int pic_forward(pic_handle *h, int steps, int ckpt_every) { return pic_forward2(h, steps, ckpt_every, ckpt_every); }

// pic_forward2, or (src != null) a forward that replays the discrete choices
// recorded by src's last forward
static int forward_impl(pic_handle *h, int steps, int ckpt_every, int sub_every, const pic_handle *src) {
    if (!h) return PIC_ERR_ARG;
    if (steps < 1 || ckpt_every < 1) return set_err(h, PIC_ERR_ARG, "pic_forward: steps and ckpt_every must be >= 1");
    if (sub_every < 1 || sub_every > ckpt_every)
        return set_err(h, PIC_ERR_ARG, "pic_forward2: sub_every must be in 1..ckpt_every");
    int rc = set_device(h);
    if (rc) return rc;
    if ((rc = need_particles(h))) return rc;
    adj_free(h);
    AdjState *Ap = new AdjState();
    h->adj = Ap;
    AdjState &A = *Ap;
    A.mixed = h->mixed;
    A.elem = h->mixed ? sizeof(float) : sizeof(double);
    A.nsp = h->cfg.nspecies;
    A.steps = steps;
    A.K = ckpt_every;
    A.K2 = sub_every;
    A.nseg = (steps + ckpt_every - 1) / ckpt_every;
    const Grid &g = h->g;
    std::vector<std::vector<int>> counts(A.nsp);
    for (int s = 0; s < A.nsp; s++) {
        if ((rc = tile_counts(h, s, counts[s]))) return rc;
        int64_t t = 0;
        for (int c : counts[s]) t += c;
        A.n[s] = t;
    }
    A.pbytes = adj_state_bytes(A);
    const size_t fbytes = g.nodes_pitched() * (h->mixed ? sizeof(float) : sizeof(double));
    if (src) {
        const AdjState *S = src->adj;
        bool same = S && S->branch && !h->mixed && S->nsp == A.nsp && S->steps >= steps;
        for (int s = 0; same && s < A.nsp; s++) same = S->n[s] == A.n[s];
        if (!same)
            return set_err(h, PIC_ERR_ARG,
                           "pic_forward_replay: the source needs a recorded FP64 forward of at least as many steps "
                           "and the same particle counts");
        A.branch_mode = 2;
        A.branch_src = S->branch;
    } else if (h->branch_record && !h->mixed) {
        if ((rc = adj_alloc(h, (void **)&A.branch,
                            (size_t)steps * (size_t)total_particles(A) * sizeof(unsigned long long),
                            "the branch record")))
            return rc;
        A.branch_mode = 1;
    }
    CK(cudaEventCreate(&A.e0), "event");
    CK(cudaEventCreate(&A.e1), "event");
    if ((rc = adj_alloc(h, (void **)&A.cur, A.pbytes, "the particle state"))) return rc;
    if ((rc = adj_alloc(h, (void **)&A.ckp, A.pbytes * A.nseg, "the particle checkpoints"))) return rc;
    if ((rc = adj_alloc(h, (void **)&A.ckf, fbytes * 6 * A.nseg, "the field checkpoints"))) return rc;
    if ((rc = adj_alloc(h, (void **)&A.hist, sizeof(double) * 3 * steps, "the history"))) return rc;
    if ((rc = adj_alloc(h, (void **)&A.st, sizeof(AdjStatus), "the status"))) return rc;
    if ((rc = adj_alloc(h, (void **)&A.red, sizeof(double) * 8, "the reduction scratch"))) return rc;
    CK(cudaMemsetAsync(A.hist, 0, sizeof(double) * 3 * steps, h->stream), "zero history");
    CK(cudaMemsetAsync(A.st, 0, sizeof(AdjStatus), h->stream), "zero status");
    // bins -> flat order
    int *cell[kMaxSpecies];
    void *v[kMaxSpecies][6];
    adj_state_view(A, A.cur, cell, v);
    int64_t *d0 = nullptr;
    CK(cudaMalloc(&d0, (g.ntiles + 1) * sizeof(int64_t)), "alloc");
    for (int s = 0; s < A.nsp; s++) {
        std::vector<int64_t> start(g.ntiles + 1);
        int64_t acc = 0;
        for (int t = 0; t < g.ntiles; t++) { start[t] = acc; acc += counts[s][t]; }
        start[g.ntiles] = acc;
        CK(cudaMemcpyAsync(d0, start.data(), (g.ntiles + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream),
           "H2D");
        if (!h->mixed)
            k_flat_gather_plain<<<g.ntiles, 256, 0, h->stream>>>(h->sp[s].v, d0, cell[s], (double *)v[s][0],
                                                                 (double *)v[s][1], (double *)v[s][2],
                                                                 (double *)v[s][3], (double *)v[s][4],
                                                                 (double *)v[s][5]);
        else
            adj_gather_mixed(g, h->sp[s].v, d0, cell[s], v[s], h->stream);
        CK(cudaGetLastError(), "flat gather");
        CK(cudaStreamSynchronize(h->stream), "sync");
    }
    cudaFree(d0);
    rc = forward_run(h, A);
    if (rc) return rc;
    if ((rc = check_adj_status(h, A, "pic_forward"))) return rc;
    CK(cudaEventElapsedTime(&A.t_fwd, A.e0, A.e1), "timing");
    A.hhist.resize(3 * (size_t)steps);
    CK(cudaMemcpy(A.hhist.data(), A.hist, sizeof(double) * 3 * steps, cudaMemcpyDeviceToHost), "history");
    const double w = g.hx * g.hy * g.hz;
    for (double &x : A.hhist) x *= w;
    // the handle continues from the final state: flat order -> bins
    for (int s = 0; s < A.nsp; s++) {
        if (!h->mixed)
            rc = build_bins(h, s, A.n[s], cell[s], (const double *)v[s][0], (const double *)v[s][1],
                            (const double *)v[s][2], (const double *)v[s][3], (const double *)v[s][4],
                            (const double *)v[s][5], nullptr);
        else
            rc = build_bins_f(h, s, A.n[s], cell[s], (const float *)v[s][0], (const float *)v[s][1],
                              (const float *)v[s][2], (const float *)v[s][3], (const float *)v[s][4],
                              (const float *)v[s][5]);
        if (rc) return rc;
    }
    h->kin_valid = 0;
    A.have_forward = 1;
    return PIC_OK;
}

int pic_forward2(pic_handle *h, int steps, int ckpt_every, int sub_every) {
    return forward_impl(h, steps, ckpt_every, sub_every, nullptr);
}

int pic_branch_record(pic_handle *h, int on) {
    if (!h) return PIC_ERR_ARG;
    if (on && h->mixed) return set_err(h, PIC_ERR_ARG, "pic_branch_record: the FP64 plain form only");
    h->branch_record = on ? 1 : 0;
    return PIC_OK;
}

int pic_perturb_momenta(pic_handle *h, int species, int64_t n, const double *dp, double eps) {
    if (!h || species < 0 || species >= h->cfg.nspecies || n < 0 || (n > 0 && !dp))
        return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    if ((rc = need_particles(h))) return rc;
    const Grid &g = h->g;
    std::vector<int> counts;
    if ((rc = tile_counts(h, species, counts))) return rc;
    std::vector<int64_t> d0(g.ntiles + 1);
    int64_t acc = 0;
    for (int t = 0; t < g.ntiles; t++) { d0[t] = acc; acc += counts[t]; }
    d0[g.ntiles] = acc;
    if (acc != n) return set_err(h, PIC_ERR_ARG, "pic_perturb_momenta: n is not the species' particle count");
    if (n == 0) return PIC_OK;
    int64_t *dd = nullptr;
    double *dv = nullptr;
    CK(cudaMalloc(&dd, (g.ntiles + 1) * sizeof(int64_t)), "alloc");
    cudaError_t e = cudaMalloc(&dv, (size_t)n * 3 * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dd, d0.data(), (g.ntiles + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dv, dp, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        k_perturb_momenta<<<g.ntiles, 256, 0, h->stream>>>(h->sp[species].v, h->mixed, dd, dv, eps);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dd);
    if (dv) cudaFree(dv);
    CK(e, "perturb momenta");
    h->kin_valid = 0;
    return PIC_OK;
}

int pic_forward_replay(pic_handle *h, int steps, const pic_handle *recorded) {
    if (!h || !recorded) return PIC_ERR_ARG;
    if (h->mixed) return set_err(h, PIC_ERR_ARG, "pic_forward_replay: the FP64 plain form only");
    return forward_impl(h, steps, steps, steps, recorded);
}

int pic_forward_history(pic_handle *h, double *out) {
    if (!h || !out) return PIC_ERR_ARG;
    if (!h->adj || !h->adj->have_forward) return set_err(h, PIC_ERR_STATE, "no pic_forward run");
    memcpy(out, h->adj->hhist.data(), h->adj->hhist.size() * sizeof(double));
    return PIC_OK;
}

int pic_loss_value(pic_handle *h, const pic_loss *loss, double *value) {
    if (!h || !loss || !value) return PIC_ERR_ARG;
    if (!h->adj || !h->adj->have_forward) return set_err(h, PIC_ERR_STATE, "no pic_forward run");
    const AdjState &A = *h->adj;
    if (loss->field < 0 || loss->field > 2 || loss->window < 1 || loss->window > A.steps)
        return set_err(h, PIC_ERR_ARG, "pic_loss: field must be PIC_EX..PIC_EZ and window in 1..steps");
    double s = 0.0;
    for (int n = A.steps - loss->window; n < A.steps; n++) s += A.hhist[3 * (size_t)n + loss->field];
    *value = s;
    return PIC_OK;
}

int pic_backward(pic_handle *h, const pic_loss *loss, pic_grads *grads) {
    if (!h || !loss || !grads) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    if (!h->adj || !h->adj->have_forward) return set_err(h, PIC_ERR_STATE, "pic_backward needs a pic_forward run");
    AdjState &A = *h->adj;
    if ((rc = pic_loss_value(h, loss, &grads->loss))) return rc;
    if (loss->species < 0 || loss->species >= A.nsp) return set_err(h, PIC_ERR_ARG, "pic_loss: bad species");
    const Grid &g = h->g;
    const size_t N = g.nodes_pitched();
    const size_t fbytes = N * (h->mixed ? sizeof(float) : sizeof(double));
    int64_t np = total_particles(A);
    if (!A.segp) {
        if ((rc = adj_alloc(h, (void **)&A.segp, A.pbytes * (size_t)(A.K2 + 1), "the segment states"))) return rc;
        if ((rc = adj_alloc(h, (void **)&A.segf, fbytes * 6 * (size_t)(A.K2 + 1), "the segment fields"))) return rc;
        if (A.K2 < A.K) {
            const size_t nsub = (size_t)(A.K + A.K2 - 1) / A.K2;
            if ((rc = adj_alloc(h, (void **)&A.subp, A.pbytes * nsub, "the sub-checkpoint states"))) return rc;
            if ((rc = adj_alloc(h, (void **)&A.subf, fbytes * 6 * nsub, "the sub-checkpoint fields"))) return rc;
        }
        A.lamp_bytes = (size_t)np * 6 * A.elem;
        if ((rc = adj_alloc(h, (void **)&A.lamp, A.lamp_bytes, "the particle adjoints"))) return rc;
        if ((rc = adj_alloc(h, (void **)&A.lamf, N * sizeof(double) * 12, "the field adjoints"))) return rc;
        if ((rc = adj_alloc(h, (void **)&A.rf, N * sizeof(double) * PIC_FIELD_COUNT, "the recompute fields")))
            return rc;
        if ((rc = adj_alloc(h, (void **)&A.ha, fbytes * 3, "the half-step B"))) return rc;
        if ((rc = adj_alloc(h, (void **)&A.lamF, (size_t)np * 6 * A.elem, "the interpolation adjoints"))) return rc;
        // optional: the interpolated fields of every step of a segment, so the
        // adjoint does not gather them again (skipped when memory is short)
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        size_t want = (size_t)np * 6 * A.elem * (size_t)A.K2;
        if (want + ((size_t)4 << 30) < free_b && cudaMalloc((void **)&A.segF, want) != cudaSuccess) {
            A.segF = nullptr;
            cudaGetLastError();
        }
    }
    CK(cudaMemsetAsync(A.st, 0, sizeof(AdjStatus), h->stream), "zero status");
    rc = backward_run(h, A, *loss);
    if (rc) return rc;
    if ((rc = check_adj_status(h, A, "pic_backward"))) return rc;
    CK(cudaEventElapsedTime(&A.t_bwd, A.e0, A.e1), "timing");
    // gradients of the species' initial momenta (adjoint after the sweep) and
    // of its drift / spread; initial momenta from checkpoint 0
    const int s = loss->species;
    const int64_t n = A.n[s];
    size_t o = 0;
    for (int q = 0; q < s; q++) o += 6 * (size_t)A.n[q];
    int *cell0[kMaxSpecies];
    void *v0[kMaxSpecies][6];
    adj_state_view(A, A.ckp, cell0, v0);
    double out4[4] = {0.0, 0.0, 0.0, 0.0};
    double *lp = nullptr;  // FP64 copies of lambda_p (and p0) for the mixed form
    if (n > 0) {
        CK(cudaMemsetAsync(A.red, 0, 4 * sizeof(double), h->stream), "zero");
        const double *l3[3], *p3[3];
        if (!h->mixed) {
            for (int a = 0; a < 3; a++) {
                l3[a] = (const double *)A.lamp + o + (size_t)(3 + a) * n;
                p3[a] = (const double *)v0[s][3 + a];
            }
        } else {
            CK(cudaMalloc(&lp, (size_t)n * 6 * sizeof(double)), "alloc");
            adj_widen_mixed((const float *)A.lamp + o + 3 * (size_t)n, (const float *const *)&v0[s][3], n, lp,
                            h->stream);
            for (int a = 0; a < 3; a++) {
                l3[a] = lp + (size_t)a * n;
                p3[a] = lp + (size_t)(3 + a) * n;
            }
        }
        k_param_grads<<<592, kT, 0, h->stream>>>(n, l3[0], l3[1], l3[2], p3[0], p3[1], p3[2], loss->drift[0],
                                                 loss->drift[1], loss->drift[2], A.red);
        CK(cudaMemcpyAsync(out4, A.red, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H");
        if (grads->d_p0 && grads->n >= n) {
            double *tmp = nullptr;
            CK(cudaMalloc(&tmp, (size_t)n * 3 * sizeof(double)), "alloc");
            k_interleave<<<blocks_of(n), kT, 0, h->stream>>>(n, l3[0], l3[1], l3[2], tmp);
            CK(cudaMemcpyAsync(grads->d_p0, tmp, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
               "D2H");
            CK(cudaStreamSynchronize(h->stream), "sync");
            cudaFree(tmp);
        }
        CK(cudaStreamSynchronize(h->stream), "sync");
        if (lp) cudaFree(lp);
    }
    bool fits = grads->n >= n;
    grads->n = n;
    for (int a = 0; a < 3; a++) grads->d_drift[a] = out4[a];
    grads->d_vth = loss->vth > 0 ? out4[3] / loss->vth : 0.0;
    if (grads->d_p0 && !fits) return set_err(h, PIC_ERR_ARG, "pic_grads: d_p0 capacity too small");
    return PIC_OK;
}

int pic_adjoint_timings(pic_handle *h, float *out2) {
    if (!h || !out2) return PIC_ERR_ARG;
    if (!h->adj) return set_err(h, PIC_ERR_STATE, "no differentiable run");
    out2[0] = h->adj->t_fwd;
    out2[1] = h->adj->t_bwd;
    return PIC_OK;
}

int pic_adjoint_free(pic_handle *h) {
    if (!h) return PIC_ERR_ARG;
    if (set_device(h)) return h->status;
    adj_free(h);
    return PIC_OK;
}

}  // extern "C"
