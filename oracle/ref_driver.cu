// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Reference replay driver.  It compiles the reference's OWN __host__ __device__
// physics (cell.h, particle.h, tensor.h and the element functions of
// kernels.cu) for the host CPU, straight from the reference source tree, and
// replays every kernel's grid loop of one 0buf time step in the reference
// order (gpu_plasma.h:605-620 Plasma::Step):
//
//   b_half     MagneticStageOne          gpu_plasma.h:524-538, kernels.cu:1052-1089
//   stage      AssignCellsToArraysGPU    gpu_plasma.h:1006-1036, kernels.cu:32-49
//   zero_j     SetCurrentsToZero         gpu_plasma.h:1693-1741, kernels.cu:9-26
//   push       GPU_StepAllCells          kernels.cu:719-756, 886-924
//   deposit    GPU_CurrentsAllCells      kernels.cu:811-858, 927-991
//   write_j    GPU_WriteAllCurrents      kernels.cu:83-112
//   migrate    K5 / K8 / K6              kernels.cu:146-242, 316-370
//   j_fold     SetPeriodicCurrents       gpu_plasma.h:926-993, kernels.cu:1124-1159
//   b_complete MagneticFieldStageTwo     gpu_plasma.h:540-551, kernels.cu:1024-1049
//   e_update   ElectricFieldEvaluate     gpu_plasma.h:249-320, 455-483, kernels.cu:1091-1102
//   e_ghosts   ...EvaluatePeriodic       gpu_plasma.h:432-452, 486-507, 802-870
//
// The atomics of the reference (K3, K12, K20) are replayed in one fixed
// serial order; the reference GPU sums them in an unspecified order.
//
// Built by oracle/build_ref.sh into oracle/_ref/ (git-ignored).  The only shim
// is a pre-included empty `surface` template (CUDA 12 removed the texture /
// surface reference templates that cell.h:60 declares); no reference file is
// modified or copied.
#include "archAPI.h"
#include "gpucell.h"
#include "add.cu"
#include "kernels.cu"
#include "load_data.h"

#include <vector>
#include <cstring>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { F_EX, F_EY, F_EZ, F_HX, F_HY, F_HZ, F_JX, F_JY, F_JZ, F_QX, F_QY, F_QZ, F_NUM };

struct RefSim {
    int Nx, Ny, Nz;
    double Lx, Ly, Lz, tau;
    std::vector<Cell *> cells;          // (Nx+2)(Ny+2)(Nz+2), index = getGlobalCellNumber
    std::vector<double> f[F_NUM];
    int last_error;
    size_t nodes() const { return (size_t)(Nx + 2) * (Ny + 2) * (Nz + 2); }
    Cell *c0() { return cells[0]; }
};

int g_threads = 1;

// MagneticFieldTrace, gpu_plasma.h:735-767 (grid (iend+1,lend+1,kend+1) of emh1)
void magnetic_trace(RefSim &s, double *Q, double *H, double *E1, double *E2,
                    int i_end, int l_end, int k_end, double c1, double c2, int dir) {
    int3 d1, d2;
    // getMagneticFieldTraceShifts, gpu_plasma.h:722-733
    d1.x = (dir == 0) * 0 + (dir == 1) * 1 + (dir == 2) * 0;
    d1.y = (dir == 0) * 0 + (dir == 1) * 0 + (dir == 2) * 1;
    d1.z = (dir == 0) * 1 + (dir == 1) * 0 + (dir == 2) * 0;
    d2.x = (dir == 0) * 0 + (dir == 1) * 0 + (dir == 2) * 1;
    d2.y = (dir == 0) * 1 + (dir == 1) * 0 + (dir == 2) * 0;
    d2.z = (dir == 0) * 0 + (dir == 1) * 1 + (dir == 2) * 0;
    Cell *c0 = s.c0();
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i <= i_end; i++)
        for (int l = 0; l <= l_end; l++)
            for (int k = 0; k <= k_end; k++)
                emh1_Element(c0, make_int3(i, l, k), Q, H, E1, E2, c1, c2, d1, d2);
}

void b_half(RefSim &s) {  // MagneticStageOne, gpu_plasma.h:524-538
    Cell *c = s.c0();
    double3 c1;
    c1.x = s.tau / (c->get_hx());
    c1.y = s.tau / (c->get_hy());
    c1.z = s.tau / c->get_hz();
    double **f = nullptr; (void)f;
    magnetic_trace(s, s.f[F_QX].data(), s.f[F_HX].data(), s.f[F_EY].data(), s.f[F_EZ].data(),
                   s.Nx + 1, s.Ny, s.Nz, c1.z, c1.y, 0);
    magnetic_trace(s, s.f[F_QY].data(), s.f[F_HY].data(), s.f[F_EZ].data(), s.f[F_EX].data(),
                   s.Nx, s.Ny + 1, s.Nz, c1.x, c1.z, 1);
    magnetic_trace(s, s.f[F_QZ].data(), s.f[F_HZ].data(), s.f[F_EX].data(), s.f[F_EY].data(),
                   s.Nx, s.Ny, s.Nz + 1, c1.y, c1.x, 2);
}

void stage_fields(RefSim &s) {  // GPU_SetFieldsToCells over grid (Nx,Ny,Nz)
    Cell *c0 = s.c0();
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s.Nx; i++)
        for (int l = 0; l < s.Ny; l++)
            for (int k = 0; k < s.Nz; k++) {
                Cell *c = s.cells[c0->getGlobalCellNumber(i, l, k)];
                c->readFieldsFromArrays(s.f[F_EX].data(), s.f[F_EY].data(), s.f[F_EZ].data(),
                                        s.f[F_HX].data(), s.f[F_HY].data(), s.f[F_HZ].data());
            }
}

void zero_j(RefSim &s) {  // SetCurrentArraysToZero + GPU_SetAllCurrentsToZero
    std::memset(s.f[F_JX].data(), 0, sizeof(double) * s.nodes());
    std::memset(s.f[F_JY].data(), 0, sizeof(double) * s.nodes());
    std::memset(s.f[F_JZ].data(), 0, sizeof(double) * s.nodes());
    for (Cell *c : s.cells) {
        std::memset(c->Jx, 0, sizeof(CellDouble));
        std::memset(c->Jy, 0, sizeof(CellDouble));
        std::memset(c->Jz, 0, sizeof(CellDouble));
    }
}

void push(RefSim &s) {  // GPU_StepAllCells -> MoveParticlesInCell -> Cell::MoveSingleParticle
    long n = (long)s.cells.size();
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
    for (long ci = 0; ci < n; ci++) {
        Cell *c = s.cells[ci];
        CellTotalField cf;
        cf.Ex = c->Ex; cf.Ey = c->Ey; cf.Ez = c->Ez;
        cf.Hx = c->Hx; cf.Hy = c->Hy; cf.Hz = c->Hz;
        for (int i = 0; i < c->number_of_particles; i++) c->MoveSingleParticle(i, cf);
    }
}

// writeCurrentComponent, kernels.cu:512-528, serialised
void add_component(CellDouble *J, CurrentTensorComponent *t1, CurrentTensorComponent *t2, int pqr2) {
    J->M[t1->i11][t1->i12][t1->i13] += t1->t[0];
    J->M[t1->i21][t1->i22][t1->i23] += t1->t[1];
    J->M[t1->i31][t1->i32][t1->i33] += t1->t[2];
    J->M[t1->i41][t1->i42][t1->i43] += t1->t[3];
    if (pqr2 == 2) {
        J->M[t2->i11][t2->i12][t2->i13] += t2->t[0];
        J->M[t2->i21][t2->i22][t2->i23] += t2->t[1];
        J->M[t2->i31][t2->i32][t2->i33] += t2->t[2];
        J->M[t2->i41][t2->i42][t2->i43] += t2->t[3];
    }
}

void deposit(RefSim &s) {  // GPU_CurrentsAllCells, kernels.cu:927-991
    long n = (long)s.cells.size();
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
    for (long ci = 0; ci < n; ci++) {
        Cell *c = s.cells[ci];
        std::vector<CellDouble> mx(CURRENT_SUM_BUFFER_LENGTH), my(CURRENT_SUM_BUFFER_LENGTH),
            mz(CURRENT_SUM_BUFFER_LENGTH);
        std::memset(mx.data(), 0, sizeof(CellDouble) * CURRENT_SUM_BUFFER_LENGTH);
        std::memset(my.data(), 0, sizeof(CellDouble) * CURRENT_SUM_BUFFER_LENGTH);
        std::memset(mz.data(), 0, sizeof(CellDouble) * CURRENT_SUM_BUFFER_LENGTH);
        int count = c->number_of_particles;
        for (int index = 0; index < count; index++) {
            DoubleCurrentTensor dt;
            int pqr2;
            c->AccumulateCurrentSingleParticle(index, &pqr2, &dt);
            int b = index % CURRENT_SUM_BUFFER_LENGTH;
            add_component(&mx[b], &dt.t1.Jx, &dt.t2.Jx, pqr2);
            add_component(&my[b], &dt.t1.Jy, &dt.t2.Jy, pqr2);
            add_component(&mz[b], &dt.t1.Jz, &dt.t2.Jz, pqr2);
        }
        // addCellDouble, kernels.cu:550-574 (tile += buffer 0, 1, ..., 9)
        double *jx = (double *)c->Jx->M, *jy = (double *)c->Jy->M, *jz = (double *)c->Jz->M;
        for (int e = 0; e < CellExtent * CellExtent * CellExtent; e++)
            for (int b = 0; b < CURRENT_SUM_BUFFER_LENGTH; b++) {
                jx[e] += ((double *)mx[b].M)[e];
                jy[e] += ((double *)my[b].M)[e];
                jz[e] += ((double *)mz[b].M)[e];
            }
    }
}

void write_j(RefSim &s) {  // GPU_WriteAllCurrents, kernels.cu:83-112, serialised in cell order
    double *jx = s.f[F_JX].data(), *jy = s.f[F_JY].data(), *jz = s.f[F_JZ].data();
    for (Cell *c : s.cells)
        for (int i1 = 0; i1 < CellExtent; i1++)
            for (int l1 = 0; l1 < CellExtent; l1++)
                for (int k1 = 0; k1 < CellExtent; k1++) {
                    int n = c->getFortranCellNumber(c->i + i1 - 1, c->l + l1 - 1, c->k + k1 - 1);
                    if (n < 0) n = -n;
                    jx[n] += c->Jx->M[i1][l1][k1];
                    jy[n] += c->Jy->M[i1][l1][k1];
                    jz[n] += c->Jz->M[i1][l1][k1];
                }
}

int migrate(RefSim &s) {
    Cell *c0 = s.c0();
    long ncell = (long)s.cells.size();
    int err = 0;
    // K5 GPU_MakeDepartureLists, kernels.cu:146-216, grid (Nx+2,Ny+2,Nz+2)
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16) reduction(| : err)
    for (long ci = 0; ci < ncell; ci++) {
        Cell *c = s.cells[ci];
        int ix, iy, iz;
        c->departureListLength = 0;
        for (ix = 0; ix < 3; ix++)
            for (iy = 0; iy < 3; iy++)
                for (iz = 0; iz < 3; iz++) c->departure[ix][iy][iz] = 0;
        for (int num = 0; num < c->number_of_particles; num++) {
            Particle p = c->readParticleFromSurfaceDevice(num);
            c->flyDirection(&p, &ix, &iy, &iz);
            c->writeParticleToSurface(num, &p);
            if (!c->isPointInCell(p.GetX())) {
                c->writeParticleToSurface(num, &p);
                if (c->departureListLength == PARTICLES_FLYING_ONE_DIRECTION) {
                    err |= 1;  // TOO_MANY_PARTICLES, kernels.cu:193-203
                    break;
                }
                c->departureListLength++;
                int num1 = c->departure[ix][iy][iz];
                c->departureList[ix][iy][iz][num1] = p;
                c->departure[ix][iy][iz] += 1;
            }
        }
    }
    if (err) return -513131313;  // TOO_MANY_PARTICLES, cell.h:27
    // K8 GPU_ArrangeFlights, kernels.cu:316-370, grid (Nx,Ny,Nz).  Arrivals carry
    // direction 13, so gathering before appending gives the serial result.
    std::vector<std::vector<Particle>> arrivals(ncell);
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 4) collapse(3)
    for (int nx = 0; nx < s.Nx; nx++)
        for (int ny = 0; ny < s.Ny; ny++)
            for (int nz = 0; nz < s.Nz; nz++) {
                int n = c0->getGlobalCellNumber(nx, ny, nz);
                Cell *c = s.cells[n];
                for (int ix = 0; ix < 3; ix++)
                    for (int iy = 0; iy < 3; iy++)
                        for (int iz = 0; iz < 3; iz++) {
                            int sn = c0->getWrapCellNumber(nx + ix - 1, ny + iy - 1, nz + iz - 1);
                            Cell *snd_c = s.cells[sn];
                            for (int j = 0; j < snd_c->number_of_particles; j++) {
                                Particle p1 = snd_c->readParticleFromSurfaceDevice(j);
                                if (p1.direction != 13) {
                                    p1.direction = 13;
                                    if (c->isPointInCell(p1.GetX())) arrivals[n].push_back(p1);
                                }
                            }
                        }
            }
    for (long ci = 0; ci < ncell; ci++)
        for (Particle &p : arrivals[ci]) {
            if (s.cells[ci]->number_of_particles >= MAX_particles_per_cell) return -2;
            s.cells[ci]->Insert(p);
        }
    // K6 GPU_MakeDepartureLists_rm, kernels.cu:219-242, grid (Nx+2,Ny+2,Nz+2)
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
    for (long ci = 0; ci < ncell; ci++) {
        Cell *c = s.cells[ci];
        for (int num = 0; num < c->number_of_particles; num++) {
            Particle p = c->readParticleFromSurfaceDevice(num);
            if (p.direction != 13) {
                c->removeParticleFromSurfaceDevice(num, &p, &(c->number_of_particles));
                num--;
            }
        }
    }
    return 0;
}

void j_fold(RefSim &s) {  // SetPeriodicCurrents, gpu_plasma.h:926-993
    Cell *c0 = s.c0();
    double *J[3] = {s.f[F_JX].data(), s.f[F_JY].data(), s.f[F_JZ].data()};
    for (int comp = 0; comp < 3; comp++) {
        for (int i = 0; i <= s.Ny + 1; i++)  // axis x, grid (Ny+2,1,Nz+2)
            for (int k = 0; k <= s.Nz + 1; k++) periodicCurrentElement(c0, i, k, J[comp], 0, comp, s.Nx + 2);
        for (int i = 0; i <= s.Nx + 1; i++)  // axis y, grid (Nx+2,1,Nz+2)
            for (int k = 0; k <= s.Nz + 1; k++) periodicCurrentElement(c0, i, k, J[comp], 1, comp, s.Ny + 2);
        for (int i = 0; i <= s.Nx + 1; i++)  // axis z, grid (Nx+2,1,Ny+2)
            for (int k = 0; k <= s.Ny + 1; k++) periodicCurrentElement(c0, i, k, J[comp], 2, comp, s.Nz + 2);
    }
}

void b_complete(RefSim &s) {  // MagneticFieldStageTwo, gpu_plasma.h:540-551
    Cell *c0 = s.c0();
    struct { int q, h, ie, le, ke; } tr[3] = {{F_QX, F_HX, s.Nx + 1, s.Ny, s.Nz},
                                              {F_QY, F_HY, s.Nx, s.Ny + 1, s.Nz},
                                              {F_QZ, F_HZ, s.Nx, s.Ny, s.Nz + 1}};
    for (auto &t : tr) {
        double *Q = s.f[t.q].data(), *H = s.f[t.h].data();
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int i = 0; i <= t.ie; i++)
            for (int l = 0; l <= t.le; l++)
                for (int k = 0; k <= t.ke; k++) emh2_Element(c0, i, l, k, Q, H);
    }
}

// ElectricFieldTrace -> emeGPUIterate, gpu_plasma.h:249-320
void e_trace(RefSim &s, double *E, double *H1, double *H2, double *J, int dir, double c1, double c2) {
    Cell *c0 = s.c0();
    int3 start, d1, d2, finish = make_int3(s.Nx, s.Ny, s.Nz);
    // GetElectricFieldStartsDirs, gpu_plasma.h:286-304
    start.x = (dir == 0) * 0 + (dir == 1) * 1 + (dir == 2) * 1;
    start.y = (dir == 0) * 1 + (dir == 1) * 0 + (dir == 2) * 1;
    start.z = (dir == 0) * 1 + (dir == 1) * 1 + (dir == 2) * 0;
    d1.x = (dir == 0) * 0 + (dir == 1) * 0 + (dir == 2) * (-1);
    d1.y = (dir == 0) * (-1) + (dir == 1) * 0 + (dir == 2) * 0;
    d1.z = (dir == 0) * 0 + (dir == 1) * (-1) + (dir == 2) * 0;
    d2.x = (dir == 0) * 0 + (dir == 1) * (-1) + (dir == 2) * 0;
    d2.y = (dir == 0) * 0 + (dir == 1) * 0 + (dir == 2) * (-1);
    d2.z = (dir == 0) * (-1) + (dir == 1) * 0 + (dir == 2) * 0;
    double tau = s.tau;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int nx = 0; nx <= finish.x - start.x; nx++)
        for (int ny = 0; ny <= finish.y - start.y; ny++)
            for (int nz = 0; nz <= finish.z - start.z; nz++) {
                int3 p = make_int3(start.x + nx, start.y + ny, start.z + nz);
                emeElement(c0, p, E, H1, H2, J, c1, c2, tau, d1, d2);
            }
}

void e_update(RefSim &s) {  // ElectricFieldEvaluate, gpu_plasma.h:455-483
    Cell *c = s.c0();
    double3 c1;
    c1.x = s.tau / (c->get_hx());
    c1.y = s.tau / (c->get_hy());
    c1.z = s.tau / c->get_hz();
    e_trace(s, s.f[F_EX].data(), s.f[F_HZ].data(), s.f[F_HY].data(), s.f[F_JX].data(), 0, c1.y, c1.z);
    e_trace(s, s.f[F_EY].data(), s.f[F_HX].data(), s.f[F_HZ].data(), s.f[F_JY].data(), 1, c1.z, c1.x);
    e_trace(s, s.f[F_EZ].data(), s.f[F_HY].data(), s.f[F_HX].data(), s.f[F_JZ].data(), 2, c1.x, c1.y);
}

// PeriodicBoundaries, gpu_plasma.h:802-870: E[0]=E[N] pass, then E[N+1]=E[1] pass
void periodic(RefSim &s, double *E, int dir, int start1, int end1, int start2, int end2, int N) {
    Cell *c0 = s.c0();
    for (int a = 0; a <= end1 - start1; a++)
        for (int b = 0; b <= end2 - start2; b++) periodicElement(c0, a + start1, b + start2, E, dir, 0, N);
    for (int a = 0; a <= end1 - start1; a++)
        for (int b = 0; b <= end2 - start2; b++) periodicElement(c0, a + start1, b + start2, E, dir, N + 1, 1);
}

void e_ghosts(RefSim &s) {  // ElectricFieldComponentEvaluatePeriodic x3, gpu_plasma.h:432-452, 486-505
    int Nx = s.Nx, Ny = s.Ny, Nz = s.Nz;
    double *Ex = s.f[F_EX].data(), *Ey = s.f[F_EY].data(), *Ez = s.f[F_EZ].data();
    // Ex (dir 0): first boundary (y) skipped, second: z
    periodic(s, Ex, 2, 0, Nx, 0, Ny + 1, Nz);
    // Ey (dir 1): x then z
    periodic(s, Ey, 0, 0, Ny, 1, Nz, Nx);
    periodic(s, Ey, 2, 0, Nx + 1, 0, Ny, Nz);
    // Ez (dir 2): x, second boundary (y) skipped
    periodic(s, Ez, 0, 1, Ny, 0, Nz, Nx);
}

double energy(RefSim &s) {  // GPU_getCellEnergy, wrap_kernel.cu:14-36 (serial order)
    double ee = 0.0;
    const double *Ex = s.f[F_EX].data(), *Ey = s.f[F_EY].data(), *Ez = s.f[F_EZ].data();
    for (size_t n = 0; n < s.nodes(); n++) {
        double ex = Ex[n], ey = Ey[n], ez = Ez[n];
        double t = ex * ex + ey * ey + ez * ez;
        ee += t;
    }
    return ee;
}

}  // namespace

// The reference's random-number state lives in two globals of maxwell.cu
// (cag05a: the three streams; cag05b: Brent's stored uniform) with the
// layouts below; ref_rnd_* set and read it so each call starts from a known
// state.
struct cag05a { long e_1[3]; };
struct cag05b { double e_1[2]; };
extern cag05a cag05a_;
extern cag05b cag05b_;
double rnd_uniform(int dbg_print);                      // maxwell.cu:187-192
double rnd_gaussian(double a, double b, int dbg_print);  // maxwell.cu:194-197

extern "C" {

void ref_set_threads(int n) { g_threads = n > 0 ? n : 1; }

void *ref_create(int nx, int ny, int nz, double lx, double ly, double lz, double tau) {
    if (nx < 1 || ny < 1 || nz < 1) return nullptr;
    RefSim *s = new RefSim();
    s->Nx = nx; s->Ny = ny; s->Nz = nz;
    s->Lx = lx; s->Ly = ly; s->Lz = lz; s->tau = tau;
    s->last_error = 0;
    for (int f = 0; f < F_NUM; f++) s->f[f].assign(s->nodes(), 0.0);
    // InitCells, init.cu:375-394 (creation order i, l, k == getGlobalCellNumber order)
    for (int i = 0; i < nx + 2; i++)
        for (int l = 0; l < ny + 2; l++)
            for (int k = 0; k < nz + 2; k++) {
                Cell *c = new Cell(i, l, k, lx, ly, lz, nx, ny, nz, tau);
                c->Init();
                std::memset(c->Jx, 0, sizeof(CellDouble));
                std::memset(c->Jy, 0, sizeof(CellDouble));
                std::memset(c->Jz, 0, sizeof(CellDouble));
                std::memset(c->Ex, 0, sizeof(CellDouble));
                std::memset(c->Ey, 0, sizeof(CellDouble));
                std::memset(c->Ez, 0, sizeof(CellDouble));
                std::memset(c->Hx, 0, sizeof(CellDouble));
                std::memset(c->Hy, 0, sizeof(CellDouble));
                std::memset(c->Hz, 0, sizeof(CellDouble));
                std::memset(c->Rho, 0, sizeof(CellDouble));
                s->cells.push_back(c);
            }
    return s;
}

void ref_destroy(void *h) {
    RefSim *s = (RefSim *)h;
    if (!s) return;
    for (Cell *c : s->cells) {
        delete c->Jx; delete c->Jy; delete c->Jz; delete c->Ex; delete c->Ey; delete c->Ez;
        delete c->Hx; delete c->Hy; delete c->Hz; delete c->Rho;
        delete[] c->doubParticleArray;
        delete c;
    }
    delete s;
}

// addParticleListToCells, init.cu:558-592: getPointCell + Insert, in array order.
// Returns the number of particles actually inserted.
long ref_add_particles(void *h, int sort, long n, const double *x, const double *y, const double *z,
                       const double *px, const double *py, const double *pz, double m, double q_m) {
    RefSim *s = (RefSim *)h;
    Cell *c0 = s->c0();
    long inserted = 0;
    for (long i = 0; i < n; i++) {
        Particle p(x[i], y[i], z[i], px[i], py[i], pz[i], m, q_m);
        p.sort = (particle_sorts)sort;
        p.x1 = p.y1 = p.z1 = 0.0;
        p.direction = 13;
        p.fortran_number = (int)i;
        double3 d;
        d.x = p.x; d.y = p.y; d.z = p.z;
        int cn = c0->getPointCell(d);
        if (cn < 0 || cn >= (int)s->cells.size()) continue;
        Cell *c = s->cells[cn];
        if (c->number_of_particles >= MAX_particles_per_cell) return -1;
        if (c->Insert(p)) inserted++;
    }
    return inserted;
}

int ref_set_field(void *h, int which, const double *src) {
    RefSim *s = (RefSim *)h;
    if (which < 0 || which >= F_NUM) return -1;
    std::memcpy(s->f[which].data(), src, sizeof(double) * s->nodes());
    return 0;
}

int ref_get_field(void *h, int which, double *dst) {
    RefSim *s = (RefSim *)h;
    if (which < 0 || which >= F_NUM) return -1;
    std::memcpy(dst, s->f[which].data(), sizeof(double) * s->nodes());
    return 0;
}

// Sub-steps in Plasma::Step order.  ids: 0 b_half, 1 stage, 2 zero_j, 3 push,
// 4 deposit, 5 write_j, 6 migrate, 7 j_fold, 8 b_complete, 9 e_update, 10 e_ghosts
int ref_substep(void *h, int which) {
    RefSim *s = (RefSim *)h;
    switch (which) {
        case 0: b_half(*s); return 0;
        case 1: stage_fields(*s); return 0;
        case 2: zero_j(*s); return 0;
        case 3: push(*s); return 0;
        case 4: deposit(*s); return 0;
        case 5: write_j(*s); return 0;
        case 6: return migrate(*s);
        case 7: j_fold(*s); return 0;
        case 8: b_complete(*s); return 0;
        case 9: e_update(*s); return 0;
        case 10: e_ghosts(*s); return 0;
        default: return -1;
    }
}

int ref_step(void *h) {
    for (int i = 0; i <= 10; i++) {
        int rc = ref_substep(h, i);
        if (rc) return rc;
    }
    return 0;
}

double ref_energy(void *h) { return energy(*(RefSim *)h); }

long ref_num_particles(void *h) {
    RefSim *s = (RefSim *)h;
    long n = 0;
    for (Cell *c : s->cells) n += c->number_of_particles;
    return n;
}

int ref_get_cell_counts(void *h, int *counts) {
    RefSim *s = (RefSim *)h;
    for (size_t i = 0; i < s->cells.size(); i++) counts[i] = s->cells[i]->number_of_particles;
    return 0;
}

// Particles in cell order then list order.  out holds 11 doubles per particle:
// x y z pu pv pw m q_m x1 y1 z1; ints: cell, sort, direction.
long ref_get_particles(void *h, double *out, int *cell, int *sort, int *direction) {
    RefSim *s = (RefSim *)h;
    long j = 0;
    for (size_t ci = 0; ci < s->cells.size(); ci++) {
        Cell *c = s->cells[ci];
        for (int i = 0; i < c->number_of_particles; i++, j++) {
            Particle p = c->readParticleFromSurfaceDevice(i);
            double *o = out + 11 * j;
            o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = p.pu; o[4] = p.pv; o[5] = p.pw;
            o[6] = p.m; o[7] = p.q_m; o[8] = p.x1; o[9] = p.y1; o[10] = p.z1;
            cell[j] = (int)ci;
            sort[j] = (int)p.sort;
            direction[j] = p.direction;
        }
    }
    return j;
}

// The reference's own reader of its Fortran-record dump (LoadParticleData,
// load_data.cu:308-341): reads mumu000<nt>.dat from the working directory --
// 12 field records, then the ion, electron and beam sorts.  The particles are
// kept here for ref_mumu_particles.
static std::vector<Particle> g_mumu[3];

void ref_rnd_set(long ix, long iy, long iz, double store) {
    cag05a_.e_1[0] = ix;
    cag05a_.e_1[1] = iy;
    cag05a_.e_1[2] = iz;
    cag05b_.e_1[0] = store;
}

void ref_rnd_get(long *ixyz, double *store) {
    for (int a = 0; a < 3; a++) ixyz[a] = cag05a_.e_1[a];
    *store = cag05b_.e_1[0];
}

void ref_rnd_reset() { ref_rnd_set(1, 255, 25555, 1.0); }  // cag05a_ / cag05b_ initial data

// n uniforms, or n Gaussian deviates of the given mean and spread, from the
// current state
void ref_rnd_uniforms(long n, double *out) {
    for (long j = 0; j < n; j++) out[j] = rnd_uniform(0);
}

void ref_rnd_gaussians(long n, double a, double b, double *out) {
    for (long j = 0; j < n; j++) out[j] = rnd_gaussian(a, b, 0);
}

// InitUniformMaxwellianParticles (maxwell.cu:379-536) from the generator's
// initial state.  par: tex0 tey0 tez0 beam_lx beam_ly beam_lz lx ly lz Tb rimp
// rbd.  Outputs planar: ion[a*jmb + j], el[a*2*jmb + j], beam[a*jmb + j] for
// a = x y z px py pz.  The beam arrays are zeroed first (the reference's are
// unset past the beam count and its electron loop reads them there).
// Returns the beam count.
long ref_quiet_init(int beamf, int jmb, const double *par, int meh, double *ion, double *el, double *beam) {
    ref_rnd_reset();
    memset(beam, 0, sizeof(double) * 6 * (size_t)jmb);
    int real = 0;
    InitUniformMaxwellianParticles(beamf, jmb, par[0], par[1], par[2], par[3], par[4], par[5], &real, par[6],
                                   par[7], par[8], meh, par[9], par[10], par[11], ion, ion + jmb, ion + 2 * jmb,
                                   ion + 3 * jmb, ion + 4 * jmb, ion + 5 * jmb, beam, beam + jmb, beam + 2 * jmb,
                                   beam + 3 * jmb, beam + 4 * jmb, beam + 5 * jmb, el, el + 2 * jmb,
                                   el + 4 * jmb, el + 6 * jmb, el + 8 * jmb, el + 10 * jmb);
    return real;
}

int ref_mumu_load(int nt, int nx, int ny, int nz, long *counts3) {
    for (auto &v : g_mumu) v.clear();
    int rc = LoadParticleData(nt, g_mumu[0], g_mumu[1], g_mumu[2], nx, ny, nz);
    for (int s = 0; s < 3; s++) counts3[s] = (long)g_mumu[s].size();
    return rc;
}

// The reference's quiet start, getUniformMaxwellianParticles
// (maxwell.cu:676-757), from the generator's initial state, into the same
// three lists (ions, electrons, beam) for ref_mumu_particles.
int ref_quiet_default(long *counts3) {
    ref_rnd_reset();
    for (auto &v : g_mumu) v.clear();
    int rc = getUniformMaxwellianParticles(g_mumu[0], g_mumu[1], g_mumu[2]);
    for (int s = 0; s < 3; s++) counts3[s] = (long)g_mumu[s].size();
    return rc;
}

// particle j of sort s as x y z pu pv pw m q_m
long ref_mumu_particles(int sort, double *out8) {
    if (sort < 0 || sort > 2) return -1;
    const std::vector<Particle> &v = g_mumu[sort];
    for (size_t j = 0; j < v.size(); j++) {
        const Particle &p = v[j];
        double *o = out8 + 8 * j;
        o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = p.pu; o[4] = p.pv; o[5] = p.pw; o[6] = p.m; o[7] = p.q_m;
    }
    return (long)v.size();
}

}  // extern "C"
