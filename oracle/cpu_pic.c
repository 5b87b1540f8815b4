/* ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the
 * product library.  Tests, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg are the only users.
 *
 * cpu_pic: a compact CPU restatement of the 0buf electromagnetic PIC time
 * step in plain C, FP64, with the reference's expressions in the reference's
 * order so that it is bit-identical to the reference's own functions (the
 * replay driver in oracle/ref_driver.cu; tests check this).  Differences from
 * the reference are layout only:
 *   - one growable particle list per cell instead of a 5000-slot AoS
 *     (gpucell.h:91-288, cell.h:250-282);
 *   - field values are read straight from the global arrays through the same
 *     index map the 5x5x5 cell tiles use (cell.h:1984-2036), instead of
 *     copying the tiles (identical values: the arrays do not change between
 *     staging and the push);
 *   - the 10 shared-memory current buffers of K12 are replayed serially
 *     (buffer = index % 10, then folded 0..9), and K3's atomics serially in
 *     cell order.  The reference GPU sums these in an unspecified order.
 * Citations are to files of the reference project (snytav/0buf).
 *
 * Build: cc -O2 -fPIC -shared -fopenmp -ffp-contract=off (oracle/Makefile).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { F_EX, F_EY, F_EZ, F_HX, F_HY, F_HZ, F_JX, F_JY, F_JZ, F_QX, F_QY, F_QZ, F_NUM };

typedef struct {
    double x, y, z, pu, pv, pw, m, q_m, x1, y1, z1;
    int sort, direction;
} op_particle;

typedef struct {
    op_particle *p;
    int n, cap;
    /* 5x5x5 current tiles of this cell, cell.h:180 Jx, Jy, Jz */
    double *jt;
} op_cell;

typedef struct {
    int Nx, Ny, Nz;
    double Lx, Ly, Lz, tau, hx, hy, hz;
    long ncell;
    size_t nodes;
    op_cell *cells;
    double *f[F_NUM];
    int threads;
    int status; /* sticky error bits: 1 stencil out of tile, 2 too many departures */
} op_sim;

#define CE 5
#define TILE (CE * CE * CE)
#define T3(a, b, c) (((a) * CE + (b)) * CE + (c))

/* ---------------------------------------------------------------- geometry */
/* getGlobalCellNumber, cell.h:785-801: wraps only indices >= N+2 */
static inline long glob(const op_sim *s, int i, int l, int k) {
    if (i >= s->Nx + 2) i -= s->Nx + 2;
    if (l >= s->Ny + 2) l -= s->Ny + 2;
    if (k >= s->Nz + 2) k -= s->Nz + 2;
    return (long)i * (s->Ny + 2) * (s->Nz + 2) + (long)l * (s->Nz + 2) + k;
}
/* getWrapCellNumber, cell.h:806-853 */
static inline long wrapc(const op_sim *s, int i, int l, int k) {
    if (i >= s->Nx) i -= s->Nx; else if (i < 0) i += s->Nx;
    if (l >= s->Ny) l -= s->Ny; else if (l < 0) l += s->Ny;
    if (k >= s->Nz) k -= s->Nz; else if (k < 0) k += s->Nz;
    return (long)i * (s->Ny + 2) * (s->Nz + 2) + (long)l * (s->Nz + 2) + k;
}
static inline void cell_ijk(const op_sim *s, long n, int *i, int *l, int *k) {
    *k = (int)(n % (s->Nz + 2));
    *l = (int)((n / (s->Nz + 2)) % (s->Ny + 2));
    *i = (int)(n / ((long)(s->Ny + 2) * (s->Nz + 2)));
}
/* Cell(...) ctor, cell.h:731-737 */
typedef struct { int i, l, k; double x0, y0, z0; } cgeo;
static inline cgeo geo(const op_sim *s, long n) {
    cgeo g;
    cell_ijk(s, n, &g.i, &g.l, &g.k);
    g.x0 = (double)g.i * s->hx; g.y0 = (double)g.l * s->hy; g.z0 = (double)g.k * s->hz;
    return g;
}

/* tile element [a][b][c] of the cell tiles: readField / getFortranArrayValue,
 * cell.h:1984-2036: global index (i+a-2, l+b-2, k+c-2), 0 outside [0,size] */
static inline double tile_field(const op_sim *s, const double *E, const cgeo *g, int a, int b, int c) {
    long n = glob(s, g->i + a - 2, g->l + b - 2, g->k + c - 2);
    if (n < 0 || n > (long)s->nodes) return 0.0;
    if (n == (long)s->nodes) return 0.0; /* one past the end: never reached for CE=5 */
    return E[n];
}

/* ------------------------------------------------------------- Yee fields */
/* emh1_Element, kernels.cu:1052-1073 over MagneticFieldTrace ranges */
static void magnetic_trace(op_sim *s, double *Q, double *H, const double *E1, const double *E2,
                           int i_end, int l_end, int k_end, double c1, double c2, int dir) {
    /* getMagneticFieldTraceShifts, gpu_plasma.h:722-733 */
    int d1x = (dir == 1), d1y = (dir == 2), d1z = (dir == 0);
    int d2x = (dir == 2), d2y = (dir == 0), d2z = (dir == 1);
#pragma omp parallel for num_threads(s->threads) schedule(static)
    for (int i = 0; i <= i_end; i++)
        for (int l = 0; l <= l_end; l++)
            for (int k = 0; k <= k_end; k++) {
                long n = glob(s, i, l, k);
                long n1 = glob(s, i + d1x, l + d1y, k + d1z);
                long n2 = glob(s, i + d2x, l + d2y, k + d2z);
                double e1_n1 = E1[n1], e1_n = E1[n], e2_n2 = E2[n2], e2_n = E2[n];
                double t = 0.5 * (c1 * (e1_n1 - e1_n) - c2 * (e2_n2 - e2_n));
                Q[n] = t;
                H[n] += Q[n];
            }
}

/* MagneticStageOne, gpu_plasma.h:524-538; factors gpu_plasma.h:512-522 */
static void b_half(op_sim *s) {
    double cx = s->tau / (s->hx), cy = s->tau / (s->hy), cz = s->tau / s->hz;
    magnetic_trace(s, s->f[F_QX], s->f[F_HX], s->f[F_EY], s->f[F_EZ], s->Nx + 1, s->Ny, s->Nz, cz, cy, 0);
    magnetic_trace(s, s->f[F_QY], s->f[F_HY], s->f[F_EZ], s->f[F_EX], s->Nx, s->Ny + 1, s->Nz, cx, cz, 1);
    magnetic_trace(s, s->f[F_QZ], s->f[F_HZ], s->f[F_EX], s->f[F_EY], s->Nx, s->Ny, s->Nz + 1, cy, cx, 2);
}

/* emh2_Element, kernels.cu:1024-1049; MagneticFieldStageTwo, gpu_plasma.h:540-551 */
static void b_complete(op_sim *s) {
    int ie[3] = {s->Nx + 1, s->Nx, s->Nx}, le[3] = {s->Ny, s->Ny + 1, s->Ny}, ke[3] = {s->Nz, s->Nz, s->Nz + 1};
    for (int c = 0; c < 3; c++) {
        double *Q = s->f[F_QX + c], *H = s->f[F_HX + c];
#pragma omp parallel for num_threads(s->threads) schedule(static)
        for (int i = 0; i <= ie[c]; i++)
            for (int l = 0; l <= le[c]; l++)
                for (int k = 0; k <= ke[c]; k++) {
                    long n = glob(s, i, l, k);
                    H[n] += Q[n];
                }
    }
}

/* emeElement, kernels.cu:1091-1102 over GetElectricFieldStartsDirs ranges,
 * gpu_plasma.h:249-320 (i in [start.x, Nx], l in [start.y, Ny], k in [start.z, Nz]) */
static void e_trace(op_sim *s, double *E, const double *H1, const double *H2, const double *J, int dir,
                    double c1, double c2) {
    int sx = (dir != 0), sy = (dir != 1), sz = (dir != 2);
    int d1x = -(dir == 2), d1y = -(dir == 0), d1z = -(dir == 1);
    int d2x = -(dir == 1), d2y = -(dir == 2), d2z = -(dir == 0);
    double tau = s->tau;
#pragma omp parallel for num_threads(s->threads) schedule(static)
    for (int i = sx; i <= s->Nx; i++)
        for (int l = sy; l <= s->Ny; l++)
            for (int k = sz; k <= s->Nz; k++) {
                long n = glob(s, i, l, k);
                long n1 = glob(s, i + d1x, l + d1y, k + d1z);
                long n2 = glob(s, i + d2x, l + d2y, k + d2z);
                E[n] += c1 * (H1[n] - H1[n1]) - c2 * (H2[n] - H2[n2]) - tau * J[n];
            }
}

/* ElectricFieldEvaluate, gpu_plasma.h:455-483 */
static void e_update(op_sim *s) {
    double cx = s->tau / (s->hx), cy = s->tau / (s->hy), cz = s->tau / s->hz;
    e_trace(s, s->f[F_EX], s->f[F_HZ], s->f[F_HY], s->f[F_JX], 0, cy, cz);
    e_trace(s, s->f[F_EY], s->f[F_HX], s->f[F_HZ], s->f[F_JY], 1, cz, cx);
    e_trace(s, s->f[F_EZ], s->f[F_HY], s->f[F_HX], s->f[F_JZ], 2, cx, cy);
}

/* getGlobalBoundaryCellNumber, cell.h:885-889 */
static inline long bnd(const op_sim *s, int i, int k, int dir, int N) {
    int i1 = (dir == 0) * N + (dir == 1) * i + (dir == 2) * i;
    int l1 = (dir == 0) * i + (dir == 1) * N + (dir == 2) * k;
    int k1 = (dir == 0) * k + (dir == 1) * k + (dir == 2) * N;
    return glob(s, i1, l1, k1);
}

/* PeriodicBoundaries, gpu_plasma.h:802-870 with periodicElement, kernels.cu:1104-1122 */
static void periodic(op_sim *s, double *E, int dir, int st1, int en1, int st2, int en2, int N) {
    for (int a = st1; a <= en1; a++)
        for (int b = st2; b <= en2; b++) E[bnd(s, a, b, dir, 0)] = E[bnd(s, a, b, dir, N)];
    for (int a = st1; a <= en1; a++)
        for (int b = st2; b <= en2; b++) E[bnd(s, a, b, dir, N + 1)] = E[bnd(s, a, b, dir, 1)];
}

/* ElectricFieldComponentEvaluatePeriodic x3, gpu_plasma.h:432-452, 486-505:
 * the y pass is skipped for Ex (dir 0) and Ez (dir 2). */
static void e_ghosts(op_sim *s) {
    int Nx = s->Nx, Ny = s->Ny, Nz = s->Nz;
    periodic(s, s->f[F_EX], 2, 0, Nx, 0, Ny + 1, Nz);
    periodic(s, s->f[F_EY], 0, 0, Ny, 1, Nz, Nx);
    periodic(s, s->f[F_EY], 2, 0, Nx + 1, 0, Ny, Nz);
    periodic(s, s->f[F_EZ], 0, 1, Ny, 0, Nz, Nx);
}

/* periodicCurrentElement, kernels.cu:1124-1146 */
static void j_fold_elem(op_sim *s, int i, int k, double *E, int dir, int dirE, int N) {
    long n1 = bnd(s, i, k, dir, 1), n_Nm1 = bnd(s, i, k, dir, N - 1);
    if (dir != dirE) E[n1] += E[n_Nm1];
    if (dir != 1 || dirE != 1) E[n_Nm1] = E[n1];
    long n_Nm2 = bnd(s, i, k, dir, N - 2), n0 = bnd(s, i, k, dir, 0);
    E[n0] += E[n_Nm2];
    E[n_Nm2] = E[n0];
}

/* SetPeriodicCurrents, gpu_plasma.h:926-993 */
static void j_fold(op_sim *s) {
    for (int c = 0; c < 3; c++) {
        double *J = s->f[F_JX + c];
        for (int i = 0; i <= s->Ny + 1; i++)
            for (int k = 0; k <= s->Nz + 1; k++) j_fold_elem(s, i, k, J, 0, c, s->Nx + 2);
        for (int i = 0; i <= s->Nx + 1; i++)
            for (int k = 0; k <= s->Nz + 1; k++) j_fold_elem(s, i, k, J, 1, c, s->Ny + 2);
        for (int i = 0; i <= s->Nx + 1; i++)
            for (int k = 0; k <= s->Ny + 1; k++) j_fold_elem(s, i, k, J, 2, c, s->Nz + 2);
    }
}

/* ------------------------------------------------------------- particles */
/* Interpolate3D, cell.h:1054-1153, reading the tile through tile_field */
static double interp3(const op_sim *s, const double *E, const cgeo *g, int i, int l, int k, double sx,
                      double sx1, double sy, double sy1, double sz, double sz1, int *bad) {
    if (i < 0 || i > CE) return 0.0;
    if (l < 0 || l > CE) return 0.0;
    if (k < 0 || k > CE) return 0.0;
    if (i + 1 >= CE || l + 1 >= CE || k + 1 >= CE) { *bad = 1; return 0.0; }
    double t_ilk = tile_field(s, E, g, i, l, k), t_ilk1 = tile_field(s, E, g, i, l, k + 1);
    double t_il1k = tile_field(s, E, g, i, l + 1, k), t_il1k1 = tile_field(s, E, g, i, l + 1, k + 1);
    double t_i1lk = tile_field(s, E, g, i + 1, l, k), t_i1lk1 = tile_field(s, E, g, i + 1, l, k + 1);
    double t_i1l1k = tile_field(s, E, g, i + 1, l + 1, k), t_i1l1k1 = tile_field(s, E, g, i + 1, l + 1, k + 1);
    double t1 = sx * (sy * (sz * t_ilk + sz1 * t_ilk1) + sy1 * (sz * t_il1k + sz1 * t_il1k1));
    double t2 = sx1 * (sy * (sz * t_i1lk + sz1 * t_i1lk1) + sy1 * (sz * t_i1l1k + sz1 * t_i1l1k1));
    return t2 + t1;
}

/* Particle::Move, particle.h:65-202, with Cell::GetField, cell.h:1010-1290 */
static void move_particle(const op_sim *s, const cgeo *g, op_particle *p, int *bad) {
    double Ex, Ey, Ez, Hx, Hy, Hz;
    double x = p->x, y = p->y, z = p->z;
    if (x < 0 || y < 0 || z < 0) {
        Ex = Ey = Ez = Hx = Hy = Hz = 0.0;
    } else {
        double hx = s->hx, hy = s->hy, hz = s->hz;
        /* InverseKernel, cell.h:1010-1047; getCellNumber(Center) cell.h:552-565 */
        int ix = (int)((x - g->x0) / hx + 1.0) + 1;
        int i1x = (int)(((x - g->x0) / hx + 1.0) + 1.5);
        double s1 = (int)(x / hx + 1.0) - x / hx;             /* cell.h:1193-1196 */
        double s2 = (int)(x / hx + 1.5) - 0.5 - x / hx;       /* cell.h:1201-1204 */
        int iy = (int)((y - g->y0) / hy + 1.0) + 1;
        int i1y = (int)(((y - g->y0) / hy + 1.0) + 1.5);
        double s3 = (int)(y / hy + 1.0) - y / hy;
        double s4 = (int)(y / hy + 1.5) - 0.5 - y / hy;
        int iz = (int)((z - g->z0) / hz + 1.0) + 1;
        int i1z = (int)(((z - g->z0) / hz + 1.0) + 1.5);
        double s5 = (int)(z / hz + 1.0) - z / hz;
        double s6 = (int)(z / hz + 1.5) - 0.5 - z / hz;
        double s11 = 1. - s1, s21 = 1. - s2, s31 = 1. - s3, s41 = 1. - s4, s51 = 1. - s5, s61 = 1. - s6;
        /* GetElectricField cell.h:746-772, GetMagneticField cell.h:1161-1188 */
        Ex = interp3(s, s->f[F_EX], g, ix, i1y, i1z, s1, s11, s4, s41, s6, s61, bad);
        Ey = interp3(s, s->f[F_EY], g, i1x, iy, i1z, s2, s21, s3, s31, s6, s61, bad);
        Ez = interp3(s, s->f[F_EZ], g, i1x, i1y, iz, s2, s21, s4, s41, s5, s51, bad);
        Hx = interp3(s, s->f[F_HX], g, i1x, iy, iz, s2, s21, s3, s31, s5, s51, bad);
        Hy = interp3(s, s->f[F_HY], g, ix, i1y, iz, s1, s11, s4, s41, s5, s51, bad);
        Hz = interp3(s, s->f[F_HZ], g, ix, iy, i1z, s1, s11, s3, s31, s6, s61, bad);
    }
    double tau = s->tau;
    /* ElectricMove, particle.h:65-75 */
    double tau1 = p->q_m * tau * 0.5;
    p->pu += tau1 * Ex;
    p->pv += tau1 * Ey;
    p->pw += tau1 * Ez;
    double ps = tau1 * pow((p->pu * p->pu + p->pv * p->pv + p->pw * p->pw) * 1. + 1.0, -0.5);
    /* MagneticMove, particle.h:77-99 */
    double pu = p->pu, pv = p->pv, pw = p->pw;
    double bx = ps * Hx, by = ps * Hy, bz = ps * Hz;
    double su = pu + pv * bz - pw * by;
    double sv = pv + pw * bx - pu * bz;
    double sw = pw + pu * by - pv * bx;
    double q1 = bx * bx, q2 = by * by, q3 = bz * bz, q4 = bx * by, q5 = by * bz, q6 = bz * bx;
    double sd = q1 + 1. + q2 + q3;
    double pu1 = ((q1 + 1.) * su + (q4 + bz) * sv + (q6 - by) * sw) / sd;
    double pv1 = ((q4 - bz) * su + (q2 + 1.) * sv + (q5 + bx) * sw) / sd;
    double pw1 = ((q6 + by) * su + (q5 - bx) * sv + (q3 + 1.) * sw) / sd;
    /* particle.h:177-196 */
    p->pu = pu1 + Ex * tau1;
    p->pv = pv1 + Ey * tau1;
    p->pw = pw1 + Ez * tau1;
    ps = pow(((p->pu * p->pu + p->pv * p->pv + p->pw * p->pw) + 1.0), -0.5);
    double u = ps * p->pu, v = ps * p->pv, w = ps * p->pw;
    p->x1 = p->x + tau * u;
    p->y1 = p->y + tau * v;
    p->z1 = p->z + tau * w;
}

/* pqr, cell.h:1511-1693: one straight segment x -> x1 starting in the cell of
 * centre index i; adds 3 components x 4 nodes into the cell's J tiles */
static void pqr(const op_sim *s, const cgeo *g, const int i[3], const double x[3], const double x1[3],
                double a1, double *jt, int *bad) {
    double hx = s->hx, hy = s->hy, hz = s->hz, tau = s->tau;
    double dx = (0.50 * (x[0] + x1[0]) - hx * ((double)i[0] - 2.50) - g->x0);
    double dy = (0.50 * (x[1] + x1[1]) - hy * ((double)i[1] - 2.50) - g->y0);
    double dz = (0.50 * (x[2] + x1[2]) - hz * ((double)i[2] - 2.50) - g->z0);
    double a = a1;
    double dx1 = hx - dx, dy1 = hy - dy, dz1 = hz - dz;
    double su = x1[0] - x[0], sv = x1[1] - x[1], sw = x1[2] - x[2];
    double s1 = sv * sw / 12.0, s2 = su * sw / 12.0, s3 = su * sv / 12.0;
    su = su * a / (tau * hy * hz);
    sv = sv * a / (tau * hx * hz);
    sw = sw * a / (tau * hx * hy);
    if (i[0] < 0 || i[1] < 0 || i[2] < 0 || i[0] + 1 >= CE || i[1] + 1 >= CE || i[2] + 1 >= CE) {
        *bad = 1;
        return;
    }
    double *Jx = jt, *Jy = jt + TILE, *Jz = jt + 2 * TILE;
    Jx[T3(i[0], i[1], i[2])] += su * (dy1 * dz1 + s1);
    Jx[T3(i[0], i[1], i[2] + 1)] += su * (dy1 * dz - s1);
    Jx[T3(i[0], i[1] + 1, i[2])] += su * (dy * dz1 - s1);
    Jx[T3(i[0], i[1] + 1, i[2] + 1)] += su * (dy * dz + s1);
    Jy[T3(i[0], i[1], i[2])] += sv * (dx1 * dz1 + s2);
    Jy[T3(i[0], i[1], i[2] + 1)] += sv * (dx1 * dz - s2);
    Jy[T3(i[0] + 1, i[1], i[2])] += sv * (dx * dz1 - s2);
    Jy[T3(i[0] + 1, i[1], i[2] + 1)] += sv * (dx * dz + s2);
    Jz[T3(i[0], i[1], i[2])] += sw * (dx1 * dy1 + s3);
    Jz[T3(i[0], i[1] + 1, i[2])] += sw * (dx1 * dy - s3);
    Jz[T3(i[0] + 1, i[1], i[2])] += sw * (dx * dy1 - s3);
    Jz[T3(i[0] + 1, i[1] + 1, i[2])] += sw * (dx * dy + s3);
}

/* Reflect, cell.h:1427-1478 */
static inline double reflect1(double x, double xm) {
    return (x > xm) * (x - xm) + (x < 0.0) * (xm + x) + (x > 0 && x < xm) * x;
}

/* CurrentToMesh, cell.h:1306-1422 into buffer jt (3 x 125) */
static void current_to_mesh(const op_sim *s, const cgeo *g, op_particle *p, double *jt, int *bad) {
    double hx = s->hx, hy = s->hy, hz = s->hz;
    double x[3] = {p->x, p->y, p->z}, x1[3] = {p->x1, p->y1, p->z1}, x2[3];
    double sr;
    double h[3] = {hx, hy, hz}, o[3] = {g->x0, g->y0, g->z0};
    int i1[3], i2[3];
    for (int d = 0; d < 3; d++) { /* getCellNumberCenterCurrent, cell.h:577-578 */
        double t = ((x[d] - o[d]) / h[d] + 1.5);
        i1[d] = (int)(t + 1);
        double t2 = ((x1[d] - o[d]) / h[d] + 1.5);
        i2[d] = (int)(t2 + 1);
    }
    int m = 4 * abs(i2[0] - i1[0]) + 2 * abs(i2[1] - i1[1]) + abs(i2[2] - i1[2]);
#define AVG(d) (h[d] * (((double)i1[d] + (double)i2[d]) * 0.5 - 2.0) + o[d])
#define RATIO(d) ((x2[d] - x[d]) / (x1[d] - x[d]))
#define PROD(d) ((x2[d] - x[d]) * (x1[d] - x[d]))
#define RBX(d) (x[d] + (x1[d] - x[d]) * sr)
    switch (m) {
        case 1: x2[2] = AVG(2); sr = RATIO(2); x2[0] = RBX(0); x2[1] = RBX(1); break;
        case 2: x2[1] = AVG(1); sr = RATIO(1); x2[0] = RBX(0); x2[2] = RBX(2); break;
        case 3:
            x2[1] = AVG(1); x2[2] = AVG(2);
            sr = (PROD(2) + PROD(1)) / (pow(x1[2] - x[2], 2.0) + pow(x1[1] - x[1], 2.0));
            x2[0] = RBX(0);
            break;
        case 4: x2[0] = AVG(0); sr = RATIO(0); x2[1] = RBX(1); x2[2] = RBX(2); break;
        case 5:
            x2[0] = AVG(0); x2[2] = AVG(2);
            sr = (PROD(2) + PROD(0)) / (pow(x1[2] - x[2], 2.0) + pow(x1[0] - x[0], 2.0));
            x2[1] = RBX(1);
            break;
        case 6:
            x2[0] = AVG(0); x2[1] = AVG(1);
            sr = (PROD(1) + PROD(0)) / (pow(x1[1] - x[1], 2.0) + pow(x1[0] - x[0], 2.0));
            x2[2] = RBX(2);
            break;
        case 7: x2[0] = AVG(0); x2[1] = AVG(1); x2[2] = AVG(2); break;
        default: break;
    }
#undef AVG
#undef RATIO
#undef PROD
#undef RBX
    if (m >= 1 && m <= 7) {
        pqr(s, g, i1, x, x2, p->m, jt, bad);
        pqr(s, g, i2, x2, x1, p->m, jt, bad);
    } else {
        pqr(s, g, i1, x, x1, p->m, jt, bad);
    }
    p->x = p->x1; p->y = p->y1; p->z = p->z1;
    p->x = reflect1(p->x, s->Lx);
    p->y = reflect1(p->y, s->Ly);
    p->z = reflect1(p->z, s->Lz);
}

static void push(op_sim *s) {
    int bad = 0;
#pragma omp parallel for num_threads(s->threads) schedule(dynamic, 16) reduction(| : bad)
    for (long ci = 0; ci < s->ncell; ci++) {
        op_cell *c = &s->cells[ci];
        if (!c->n) continue;
        cgeo g = geo(s, ci);
        for (int j = 0; j < c->n; j++) move_particle(s, &g, &c->p[j], &bad);
    }
    if (bad) s->status |= 1;
}

/* GPU_CurrentsAllCells (kernels.cu:927-991) replayed: buffer index % 10 */
static void deposit(op_sim *s) {
    int bad = 0;
#pragma omp parallel num_threads(s->threads) reduction(| : bad)
    {
        double *buf = (double *)malloc(sizeof(double) * 10 * 3 * TILE);
#pragma omp for schedule(dynamic, 16)
        for (long ci = 0; ci < s->ncell; ci++) {
            op_cell *c = &s->cells[ci];
            memset(c->jt, 0, sizeof(double) * 3 * TILE);
            if (!c->n) continue;
            cgeo g = geo(s, ci);
            memset(buf, 0, sizeof(double) * 10 * 3 * TILE);
            for (int j = 0; j < c->n; j++) current_to_mesh(s, &g, &c->p[j], buf + (j % 10) * 3 * TILE, &bad);
            for (int e = 0; e < 3 * TILE; e++)
                for (int b = 0; b < 10; b++) c->jt[e] += buf[b * 3 * TILE + e];
        }
        free(buf);
    }
    if (bad) s->status |= 1;
}

/* GPU_WriteAllCurrents, kernels.cu:83-112, serial in cell order */
static void write_j(op_sim *s) {
    double *jx = s->f[F_JX], *jy = s->f[F_JY], *jz = s->f[F_JZ];
    for (long ci = 0; ci < s->ncell; ci++) {
        op_cell *c = &s->cells[ci];
        int i, l, k;
        cell_ijk(s, ci, &i, &l, &k);
        for (int i1 = 0; i1 < CE; i1++)
            for (int l1 = 0; l1 < CE; l1++)
                for (int k1 = 0; k1 < CE; k1++) {
                    long n = glob(s, i + i1 - 2, l + l1 - 2, k + k1 - 2); /* getFortranCellNumber */
                    if (n < 0) n = -n;
                    jx[n] += c->jt[T3(i1, l1, k1)];
                    jy[n] += c->jt[TILE + T3(i1, l1, k1)];
                    jz[n] += c->jt[2 * TILE + T3(i1, l1, k1)];
                }
    }
}

static void zero_j(op_sim *s) {
    memset(s->f[F_JX], 0, sizeof(double) * s->nodes);
    memset(s->f[F_JY], 0, sizeof(double) * s->nodes);
    memset(s->f[F_JZ], 0, sizeof(double) * s->nodes);
    for (long ci = 0; ci < s->ncell; ci++) memset(s->cells[ci].jt, 0, sizeof(double) * 3 * TILE);
}

static int cell_append(op_cell *c, const op_particle *p) {
    if (c->n == c->cap) {
        int ncap = c->cap ? 2 * c->cap : 16;
        op_particle *np = (op_particle *)realloc(c->p, sizeof(op_particle) * ncap);
        if (!np) return -1;
        c->p = np;
        c->cap = ncap;
    }
    c->p[c->n++] = *p;
    return 0;
}

/* isPointInCell, cell.h:717 */
static inline int in_cell(const op_sim *s, const cgeo *g, const op_particle *p) {
    return (g->x0 <= p->x) && (p->x < g->x0 + s->hx) && (g->y0 <= p->y) && (p->y < g->y0 + s->hy) &&
           (g->z0 <= p->z) && (p->z < g->z0 + s->hz);
}

/* flyDirection, cell.h:694-701 */
static inline int fly_direction(const op_sim *s, const cgeo *g, const op_particle *p) {
    double hx = s->hx, hy = s->hy, hz = s->hz;
    int dx = (((p->x > g->x0 + hx) && (p->x < g->x0 + 2 * hx)) || ((p->x < hx) && (g->i == s->Nx - 1)))
                 ? 2 : (((p->x < g->x0) || ((p->x > s->Lx - hx) && (g->i == 0))) ? 0 : 1);
    int dy = (((p->y > g->y0 + hy) && (p->y < g->y0 + 2 * hy)) || ((p->y < hy) && (g->l == s->Ny - 1)))
                 ? 2 : (((p->y < g->y0) || ((p->y > s->Ly - hy) && (g->l == 0))) ? 0 : 1);
    int dz = (((p->z > g->z0 + hz) && (p->z < g->z0 + 2 * hz)) || ((p->z < hz) && (g->k == s->Nz - 1)))
                 ? 2 : (((p->z < g->z0) || ((p->z > s->Lz - hz) && (g->k == 0))) ? 0 : 1);
    return dx * 9 + dy * 3 + dz;
}

/* K5 (kernels.cu:146-216), K8 (kernels.cu:316-370), K6 (kernels.cu:219-242) */
static int migrate(op_sim *s) {
    int too_many = 0;
#pragma omp parallel for num_threads(s->threads) schedule(dynamic, 16) reduction(| : too_many)
    for (long ci = 0; ci < s->ncell; ci++) {
        op_cell *c = &s->cells[ci];
        if (!c->n) continue;
        cgeo g = geo(s, ci);
        int departures = 0;
        for (int j = 0; j < c->n; j++) {
            c->p[j].direction = fly_direction(s, &g, &c->p[j]);
            if (!in_cell(s, &g, &c->p[j])) {
                if (departures == 50) { too_many = 1; break; } /* PARTICLES_FLYING_ONE_DIRECTION */
                departures++;
            }
        }
    }
    if (too_many) { s->status |= 2; return -513131313; }
    /* K8: gather arrivals per interior receiving cell, in (ix,iy,iz,j) order */
    long *cnt = (long *)calloc((size_t)s->ncell, sizeof(long));
    op_particle **arr = (op_particle **)calloc((size_t)s->ncell, sizeof(op_particle *));
    int oom = 0;
#pragma omp parallel for num_threads(s->threads) schedule(dynamic, 4) collapse(3) reduction(| : oom)
    for (int nx = 0; nx < s->Nx; nx++)
        for (int ny = 0; ny < s->Ny; ny++)
            for (int nz = 0; nz < s->Nz; nz++) {
                long n = glob(s, nx, ny, nz);
                cgeo g = geo(s, n);
                long cap = 0;
                for (int ix = 0; ix < 3; ix++)
                    for (int iy = 0; iy < 3; iy++)
                        for (int iz = 0; iz < 3; iz++) {
                            op_cell *sc = &s->cells[wrapc(s, nx + ix - 1, ny + iy - 1, nz + iz - 1)];
                            for (int j = 0; j < sc->n; j++) {
                                if (sc->p[j].direction == 13) continue;
                                if (!in_cell(s, &g, &sc->p[j])) continue;
                                if (cnt[n] == cap) {
                                    cap = cap ? 2 * cap : 8;
                                    op_particle *np = (op_particle *)realloc(arr[n], sizeof(op_particle) * cap);
                                    if (!np) { oom = 1; continue; }
                                    arr[n] = np;
                                }
                                arr[n][cnt[n]] = sc->p[j];
                                arr[n][cnt[n]].direction = 13;
                                cnt[n]++;
                            }
                        }
            }
    for (long ci = 0; ci < s->ncell && !oom; ci++)
        for (long j = 0; j < cnt[ci]; j++)
            if (cell_append(&s->cells[ci], &arr[ci][j])) { oom = 1; break; }
    for (long ci = 0; ci < s->ncell; ci++) free(arr[ci]);
    free(arr);
    free(cnt);
    if (oom) return -2;
    /* K6: swap-with-last removal, cell.h:391-432 */
#pragma omp parallel for num_threads(s->threads) schedule(dynamic, 16)
    for (long ci = 0; ci < s->ncell; ci++) {
        op_cell *c = &s->cells[ci];
        for (int num = 0; num < c->n; num++) {
            if (c->p[num].direction != 13) {
                int last = c->n - 1;
                if (num < last) c->p[num] = c->p[last];
                c->n--;
                num--;
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- API */
void *op_create(int nx, int ny, int nz, double lx, double ly, double lz, double tau) {
    if (nx < 1 || ny < 1 || nz < 1) return NULL;
    op_sim *s = (op_sim *)calloc(1, sizeof(op_sim));
    s->Nx = nx; s->Ny = ny; s->Nz = nz;
    s->Lx = lx; s->Ly = ly; s->Lz = lz; s->tau = tau;
    s->hx = lx / ((double)nx); s->hy = ly / ((double)ny); s->hz = lz / ((double)nz);
    s->ncell = (long)(nx + 2) * (ny + 2) * (nz + 2);
    s->nodes = (size_t)s->ncell;
    s->threads = 1;
    s->cells = (op_cell *)calloc((size_t)s->ncell, sizeof(op_cell));
    for (long c = 0; c < s->ncell; c++) s->cells[c].jt = (double *)calloc(3 * TILE, sizeof(double));
    for (int f = 0; f < F_NUM; f++) s->f[f] = (double *)calloc(s->nodes, sizeof(double));
    return s;
}

void op_destroy(void *h) {
    op_sim *s = (op_sim *)h;
    if (!s) return;
    for (long c = 0; c < s->ncell; c++) { free(s->cells[c].p); free(s->cells[c].jt); }
    free(s->cells);
    for (int f = 0; f < F_NUM; f++) free(s->f[f]);
    free(s);
}

void op_set_threads(void *h, int n) { ((op_sim *)h)->threads = n > 0 ? n : 1; }

/* addParticleListToCells, init.cu:558-592: getPointCell (cell.h:585-598), Insert */
long op_add_particles(void *h, int sort, long n, const double *x, const double *y, const double *z,
                      const double *px, const double *py, const double *pz, double m, double q_m) {
    op_sim *s = (op_sim *)h;
    long inserted = 0;
    for (long i = 0; i < n; i++) {
        int ci = (int)((x[i] - 0.0) / s->hx), cl = (int)((y[i] - 0.0) / s->hy), ck = (int)((z[i] - 0.0) / s->hz);
        long cn = glob(s, ci, cl, ck);
        if (cn < 0 || cn >= s->ncell) continue;
        op_particle p;
        p.x = x[i]; p.y = y[i]; p.z = z[i]; p.pu = px[i]; p.pv = py[i]; p.pw = pz[i];
        p.m = m; p.q_m = q_m; p.x1 = p.y1 = p.z1 = 0.0; p.sort = sort; p.direction = 13;
        cgeo g = geo(s, cn);
        if (!in_cell(s, &g, &p)) continue;
        if (cell_append(&s->cells[cn], &p)) return -1;
        inserted++;
    }
    return inserted;
}

int op_set_field(void *h, int which, const double *src) {
    op_sim *s = (op_sim *)h;
    if (which < 0 || which >= F_NUM) return -1;
    memcpy(s->f[which], src, sizeof(double) * s->nodes);
    return 0;
}

int op_get_field(void *h, int which, double *dst) {
    op_sim *s = (op_sim *)h;
    if (which < 0 || which >= F_NUM) return -1;
    memcpy(dst, s->f[which], sizeof(double) * s->nodes);
    return 0;
}

/* Sub-step ids match oracle/ref_driver.cu: 0 b_half 1 stage 2 zero_j 3 push
 * 4 deposit 5 write_j 6 migrate 7 j_fold 8 b_complete 9 e_update 10 e_ghosts */
int op_substep(void *h, int which) {
    op_sim *s = (op_sim *)h;
    switch (which) {
        case 0: b_half(s); return 0;
        case 1: return 0; /* staging is implicit: fields read through the tile map */
        case 2: zero_j(s); return 0;
        case 3: push(s); return (s->status & 1) ? -3 : 0;
        case 4: deposit(s); return (s->status & 1) ? -3 : 0;
        case 5: write_j(s); return 0;
        case 6: return migrate(s);
        case 7: j_fold(s); return 0;
        case 8: b_complete(s); return 0;
        case 9: e_update(s); return 0;
        case 10: e_ghosts(s); return 0;
        default: return -1;
    }
}

int op_step(void *h) {
    for (int i = 0; i <= 10; i++) {
        int rc = op_substep(h, i);
        if (rc) return rc;
    }
    return 0;
}

int op_status(void *h) { return ((op_sim *)h)->status; }

/* GPU_getCellEnergy, wrap_kernel.cu:14-36, serial order over all nodes */
double op_energy(void *h) {
    op_sim *s = (op_sim *)h;
    double ee = 0.0;
    for (size_t n = 0; n < s->nodes; n++) {
        double ex = s->f[F_EX][n], ey = s->f[F_EY][n], ez = s->f[F_EZ][n];
        double t = ex * ex + ey * ey + ez * ez;
        ee += t;
    }
    return ee;
}

/* Extended FP64 diagnostics (no counterpart in the reference):
 * out[0] = 1/2 sum E^2, out[1] = 1/2 sum H^2 over nodes [1..N] of each axis,
 * out[2] = sum over particles (m/q_m) * (gamma - 1), out[3] = total. */
int op_energies(void *h, double *out) {
    op_sim *s = (op_sim *)h;
    double we = 0.0, wb = 0.0, wk = 0.0;
    for (int i = 1; i <= s->Nx; i++)
        for (int l = 1; l <= s->Ny; l++)
            for (int k = 1; k <= s->Nz; k++) {
                long n = glob(s, i, l, k);
                we += s->f[F_EX][n] * s->f[F_EX][n] + s->f[F_EY][n] * s->f[F_EY][n] + s->f[F_EZ][n] * s->f[F_EZ][n];
                wb += s->f[F_HX][n] * s->f[F_HX][n] + s->f[F_HY][n] * s->f[F_HY][n] + s->f[F_HZ][n] * s->f[F_HZ][n];
            }
    for (long ci = 0; ci < s->ncell; ci++) {
        op_cell *c = &s->cells[ci];
        for (int j = 0; j < c->n; j++) {
            op_particle *p = &c->p[j];
            double p2 = p->pu * p->pu + p->pv * p->pv + p->pw * p->pw;
            wk += (p->m / p->q_m) * (p2 / (sqrt(1.0 + p2) + 1.0)); /* gamma - 1 without cancellation */
        }
    }
    out[0] = 0.5 * we;
    out[1] = 0.5 * wb;
    out[2] = wk;
    out[3] = out[0] + out[1] + out[2];
    return 0;
}

long op_num_particles(void *h) {
    op_sim *s = (op_sim *)h;
    long n = 0;
    for (long ci = 0; ci < s->ncell; ci++) n += s->cells[ci].n;
    return n;
}

int op_get_cell_counts(void *h, int *counts) {
    op_sim *s = (op_sim *)h;
    for (long ci = 0; ci < s->ncell; ci++) counts[ci] = s->cells[ci].n;
    return 0;
}

/* Same export layout as ref_get_particles in oracle/ref_driver.cu */
long op_get_particles(void *h, double *out, int *cell, int *sort, int *direction) {
    op_sim *s = (op_sim *)h;
    long j = 0;
    for (long ci = 0; ci < s->ncell; ci++) {
        op_cell *c = &s->cells[ci];
        for (int i = 0; i < c->n; i++, j++) {
            const op_particle *p = &c->p[i];
            double *o = out + 11 * j;
            o[0] = p->x; o[1] = p->y; o[2] = p->z; o[3] = p->pu; o[4] = p->pv; o[5] = p->pw;
            o[6] = p->m; o[7] = p->q_m; o[8] = p->x1; o[9] = p->y1; o[10] = p->z1;
            cell[j] = (int)ci;
            sort[j] = p->sort;
            direction[j] = p->direction;
        }
    }
    return j;
}

/* ------------------------------------------------ seeded initial particles */
/* Restatement of the library's counter-based generator of the benchmark
 * configurations' particles (0buf_b200/csrc/pic_rng.cuh, used by
 * pic_init_species_host and the device generator): per interior cell
 * (i, l, k) in i, l, k order, dense index c = (i*ny + l)*nz + k, ppc particles
 * at uniform in-cell offsets o in [1e-6, 1 - 1e-6] and momenta
 * drift + vth * N(0,1) per axis (Box-Muller).  Keys: SplitMix64's finaliser
 * (Steele, Lea, Flood 2014) chained over (seed, species, cell, slot, stream).
 * tests/test_oracle_generator.py checks it bit for bit against
 * pic_init_species_host.  The reference has no such generator (its loader is
 * the quiet start of maxwell.cu); this one exists so the CPU baselines and the
 * reference arm build their inputs without the product library. */
static inline uint64_t og_mix(uint64_t z) {
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return z;
}
static inline uint64_t og_key(uint64_t seed, int species, int64_t cell, int slot, int stream) {
    uint64_t h = og_mix(seed + 0x9E3779B97F4A7C15ull);
    h = og_mix(h ^ ((uint64_t)(uint32_t)species * 0xD6E8FEB86659FD93ull));
    h = og_mix(h ^ ((uint64_t)cell * 0xA0761D6478BD642Full));
    h = og_mix(h ^ ((uint64_t)(uint32_t)slot * 0xE7037ED1A0B428DBull));
    h = og_mix(h ^ ((uint64_t)(uint32_t)stream * 0x8EBC6AF09C88C6E3ull));
    return h;
}
static inline double og_uniform(uint64_t seed, int species, int64_t cell, int slot, int stream) {
    return (double)(og_key(seed, species, cell, slot, stream) >> 11) * (1.0 / 9007199254740992.0);
}
static inline double og_offset(uint64_t seed, int species, int64_t cell, int slot, int axis) {
    return 1e-6 + og_uniform(seed, species, cell, slot, axis) * (1.0 - 2e-6);
}
static inline double og_normal(uint64_t seed, int species, int64_t cell, int slot, int axis) {
    int pair = axis < 2 ? 0 : 1;
    double u1 = 1.0 - og_uniform(seed, species, cell, slot, 8 + 2 * pair);
    double u2 = og_uniform(seed, species, cell, slot, 9 + 2 * pair);
    double r = sqrt(-2.0 * log(u1));
    double a = 6.283185307179586 * u2;
    return (axis == 1) ? r * sin(a) : r * cos(a);
}
/* one particle: slot s of dense cell c at (i, l, k); out = x y z px py pz */
static void og_particle(double hx, double hy, double hz, int i, int l, int k, int64_t c, int s, int species,
                        double dx, double dy, double dz, double vth, uint64_t seed, double out[6]) {
    double ox = og_offset(seed, species, c, s, 0);
    double oy = og_offset(seed, species, c, s, 1);
    double oz = og_offset(seed, species, c, s, 2);
    out[0] = (double)i * hx + ox * hx;
    out[1] = (double)l * hy + oy * hy;
    out[2] = (double)k * hz + oz * hz;
    if (vth != 0.0) {
        out[3] = dx + vth * og_normal(seed, species, c, s, 0);
        out[4] = dy + vth * og_normal(seed, species, c, s, 1);
        out[5] = dz + vth * og_normal(seed, species, c, s, 2);
    } else {
        out[3] = dx; out[4] = dy; out[5] = dz;
    }
}

/* The generator into flat arrays (cell-major order), threads over cells. */
int op_gen_species(int nx, int ny, int nz, double lx, double ly, double lz, int species, int ppc, double dx,
                   double dy, double dz, double vth, uint64_t seed, int threads, double *x, double *y, double *z,
                   double *px, double *py, double *pz) {
    if (nx < 1 || ny < 1 || nz < 1 || ppc < 0) return -1;
    double hx = lx / ((double)nx), hy = ly / ((double)ny), hz = lz / ((double)nz);
    long ncell = (long)nx * ny * nz;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static)
    for (long c = 0; c < ncell; c++) {
        int i = (int)(c / ((long)ny * nz)), l = (int)((c / nz) % ny), k = (int)(c % nz);
        for (int s = 0; s < ppc; s++) {
            double o[6];
            long q = c * ppc + s;
            og_particle(hx, hy, hz, i, l, k, c, s, species, dx, dy, dz, vth, seed, o);
            x[q] = o[0]; y[q] = o[1]; z[q] = o[2]; px[q] = o[3]; py[q] = o[4]; pz[q] = o[5];
        }
    }
    return 0;
}

/* The generator straight into the simulation's cell lists, threads over
 * cells: the same particles, in the same per-cell order, as op_gen_species
 * followed by op_add_particles (each generated particle lies strictly inside
 * its cell).  Returns the particles inserted. */
long op_init_species(void *h, int sort, int species, int ppc, double dx, double dy, double dz, double vth,
                     uint64_t seed, double m, double q_m) {
    op_sim *s = (op_sim *)h;
    long ncell = (long)s->Nx * s->Ny * s->Nz;
    long inserted = 0;
    int fail = 0;
#pragma omp parallel for num_threads(s->threads) schedule(dynamic, 64) reduction(+ : inserted) reduction(| : fail)
    for (long c = 0; c < ncell; c++) {
        int i = (int)(c / ((long)s->Ny * s->Nz)), l = (int)((c / s->Nz) % s->Ny), k = (int)(c % s->Nz);
        for (int q = 0; q < ppc; q++) {
            double o[6];
            og_particle(s->hx, s->hy, s->hz, i, l, k, c, q, species, dx, dy, dz, vth, seed, o);
            /* getPointCell as op_add_particles */
            int ci = (int)((o[0] - 0.0) / s->hx), cl = (int)((o[1] - 0.0) / s->hy), ck = (int)((o[2] - 0.0) / s->hz);
            long cn = glob(s, ci, cl, ck);
            if (cn != glob(s, i, l, k)) continue; /* never for offsets inside [1e-6, 1 - 1e-6] */
            op_particle p;
            p.x = o[0]; p.y = o[1]; p.z = o[2]; p.pu = o[3]; p.pv = o[4]; p.pw = o[5];
            p.m = m; p.q_m = q_m; p.x1 = p.y1 = p.z1 = 0.0; p.sort = sort; p.direction = 13;
            cgeo g = geo(s, cn);
            if (!in_cell(s, &g, &p)) continue;
            if (cell_append(&s->cells[cn], &p)) { fail = 1; break; }
            inserted++;
        }
    }
    return fail ? -1 : inserted;
}
