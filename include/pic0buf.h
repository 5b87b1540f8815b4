/*
 * pic0buf.h -- C ABI of the B200 (sm_100a) 3D electromagnetic PIC time step.
 *
 * This header is the drop-in boundary for the 0buf PIC step.  It replaces
 *   - the reference's arch layer archAPI.h:1-127 (see pic0buf_arch.h), and
 *   - the ~20 cudaLaunchKernel sites of the reference step driver
 *     (class Plasma, gpu_plasma.h:97-2355), which become the pic_* calls below.
 *
 * Conventions kept from the reference:
 *   - every call returns an int status; 0 is success (archAPI.cu:53 returns the
 *     CUDA error code, which is what positive values here are); negative values
 *     are PIC errors (PIC_ERR_*).  No call exits the process.
 *   - field arrays cross the boundary in the reference layout: FP64,
 *     (Nx+2)(Ny+2)(Nz+2) nodes, index i*(Ny+2)*(Nz+2) + l*(Nz+2) + k
 *     (Cell::getGlobalCellNumber, cell.h:796-801).
 *   - cell numbers reported to the caller use the same (Nx+2)(Ny+2)(Nz+2)
 *     numbering; particles only live in the interior cells.
 *   - one host thread per handle; each handle owns one CUDA stream and all
 *     calls on a handle are ordered on it.
 *
 * Plain pointers and sizes only; no C++ or torch types.
 */
#ifndef PIC0BUF_H
#define PIC0BUF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIC0BUF_ABI_VERSION 1

/* precision forms */
#define PIC_FP64_PLAIN 0 /* FP64, reference arithmetic (parity form) */
#define PIC_FP32_MIXED 1 /* FP32 push/deposit/Yee, int32 cell + FP32 offsets, FP64 global J */

/* E ghost refresh (gpu_plasma.h:432-452 skips the y pass for Ex and Ez) */
#define PIC_GHOSTS_REFERENCE 0
#define PIC_GHOSTS_PERIODIC 1

#define PIC_MAX_SPECIES 8

/* field ids for pic_get_field / pic_set_field (Plasma members, gpu_plasma.h:705-707) */
enum pic_field_id {
    PIC_EX = 0, PIC_EY, PIC_EZ,
    PIC_HX, PIC_HY, PIC_HZ,
    PIC_JX, PIC_JY, PIC_JZ,
    PIC_QX, PIC_QY, PIC_QZ, /* half-step magnetic increment (emh1_Element, kernels.cu:1052-1073) */
    PIC_FIELD_COUNT
};

/* errors (negative) */
#define PIC_OK 0
#define PIC_ERR_ARG (-1)            /* bad argument or config */
#define PIC_ERR_NOMEM (-2)          /* device or host allocation failed */
#define PIC_ERR_STENCIL (-3)        /* a particle moved more than half a cell (CFL), stencil left the tile */
#define PIC_ERR_OUTBOX (-4)         /* migration outbox overflowed */
#define PIC_ERR_HOLES (-5)          /* more departures from one tile than the compaction list holds */
#define PIC_ERR_NAN (-6)            /* non-finite momentum after the push */
#define PIC_ERR_STATE (-7)          /* call not valid in the current state */
#define PIC_ERR_NOT_BUILT (-8)      /* feature not available in this build */
#define PIC_ERR_NO_DEVICE (-9)      /* no CUDA device */
#define PIC_ERR_TOO_MANY (-513131313) /* TOO_MANY_PARTICLES, cell.h:27 (never raised: no per-cell cap) */

typedef struct pic_species {
    double q_m;  /* charge to mass ratio (Particle::q_m, particle.h:43) */
    double m;    /* signed charge weight of one macro-particle (Particle::m, particle.h:43) */
    int sort;    /* particle_sorts id, particle_types.h:11 (0 ion, 1 plasma electron, 2 beam) */
    int pad_;
} pic_species;

typedef struct pic_config {
    int nx, ny, nz;          /* interior cells per axis (Plasma::Nx.., gpu_plasma.h:691); each >= 3 */
    double lx, ly, lz;       /* box lengths; h = L/N (Cell ctor, cell.h:731-737) */
    double tau;              /* time step (Plasma::tau) */
    int precision;           /* PIC_FP64_PLAIN or PIC_FP32_MIXED */
    int ghosts;              /* PIC_GHOSTS_REFERENCE or PIC_GHOSTS_PERIODIC */
    int nspecies;            /* 1..PIC_MAX_SPECIES */
    int device;              /* CUDA device ordinal */
    pic_species species[PIC_MAX_SPECIES];
    double capacity_slack;   /* particle slots per tile = count * (1 + slack) + pad; 0 -> 0.25 */
    double outbox_fraction;  /* outbox slots = fraction * total capacity + 65536; 0 -> 0.04 */
    int tile[3];             /* cells per tile (x, y, z); 0 -> automatic: 8 x 4 x 8 (FP64 form),
                                6 x 4 x 8 (FP32 form), capped by the grid. tile[2] % 4 == 0 */
    int capacity_pad;        /* extra slots per tile; negative -> 64 */
    int reserved[7];
} pic_config;

typedef struct pic_handle pic_handle;

/* Fill a config with defaults (precision FP64 plain, reference ghosts, device 0). */
void pic_config_init(pic_config *cfg);

int pic_create(const pic_config *cfg, pic_handle **out);
int pic_destroy(pic_handle *h);

/* Loads (replaces) one species from HOST arrays of global positions and
 * momenta (p = gamma*v, c = 1), in the reference's initial placement:
 * getPointCell + Cell::Insert (init.cu:558-592, cell.h:585-598, 1754-1768).
 * Particles that no cell accepts are dropped; *inserted (may be NULL) gets the
 * number kept. */
int pic_load_particles(pic_handle *h, int species, int64_t n, const double *x, const double *y,
                       const double *z, const double *px, const double *py, const double *pz,
                       int64_t *inserted);
/* Same from DEVICE arrays. */
int pic_load_particles_device(pic_handle *h, int species, int64_t n, const double *x, const double *y,
                              const double *z, const double *px, const double *py, const double *pz,
                              int64_t *inserted);

/* Loads (replaces) one species from HOST arrays in the mixed form's native
 * layout, 28 bytes per particle: reference cell number (interior cells only),
 * FP32 in-cell offsets in [0,1) and FP32 momenta.  The plain form forms its
 * FP64 positions as (i + offset) * h.  Entries with a ghost/out-of-range cell
 * or an offset outside [0,1) are dropped.  Its device staging (about 16 bytes
 * per particle of the largest species loaded, plus 0.5 GB of chunks) stays
 * with the handle for the next load and is freed by pic_destroy. */
int pic_load_particles_cells(pic_handle *h, int species, int64_t n, const int32_t *cell, const float *ox,
                             const float *oy, const float *oz, const float *px, const float *py, const float *pz,
                             int64_t *inserted);
/* Exports one species in the same layout (plain form: offsets rounded to FP32). */
int pic_get_particles_cells(pic_handle *h, int species, int64_t cap, int32_t *cell, float *ox, float *oy,
                            float *oz, float *px, float *py, float *pz, int64_t *n);

/* Seeded uniform-in-cell / Maxwellian species generated on the device:
 * ppc particles per interior cell at uniform in-cell offsets, momenta
 * drift + vth * N(0,1) per axis.  Keyed by (seed, species, cell, slot). */
int pic_init_species_device(pic_handle *h, int species, int ppc, double drift_x, double drift_y,
                            double drift_z, double vth, uint64_t seed);
/* Non-uniform density for the stress configuration (no counterpart in the
 * reference, whose loader is uniform): the expected count of cell (i,l,k) is
 *   ppc_mean * f(i,l,k) / mean over cells of f,
 *   f = (1 + cos_amp cos(2 pi (i + 1/2) / Nx))
 *       * (1 + (bump_peak - 1) exp(-d^2 / (2 bump_sigma^2))),
 * d = distance in cells from the cell centre to bump_centre (the box centre
 * when any of its components is negative), rounded up or down at random
 * keyed by (count_seed, cell) -- two species with the same profile and
 * count_seed get the same count in every cell. */
typedef struct pic_profile {
    double ppc_mean;
    double cos_amp;
    double bump_peak;
    double bump_sigma;
    double bump_centre[3];
    uint64_t count_seed;
} pic_profile;
/* Particles per cell of a profile (host, no GPU): counts[dense cell], dense
 * cell = (i*Ny + l)*Nz + k.  Returns the total in *total. */
int pic_profile_counts(int nx, int ny, int nz, const pic_profile *prof, int32_t *counts, int64_t *total);
/* The device generator with per-cell counts from a profile; particles are
 * keyed by (seed, species, cell, slot) like pic_init_species_device. */
int pic_init_species_profile(pic_handle *h, int species, const pic_profile *prof, double drift_x, double drift_y,
                             double drift_z, double vth, uint64_t seed);
/* The same generator on the host (writes n = Nx*Ny*Nz*ppc particles). */
int pic_init_species_host(int nx, int ny, int nz, double lx, double ly, double lz, int species_index, int ppc,
                          double drift_x, double drift_y, double drift_z, double vth, uint64_t seed,
                          double *x, double *y, double *z, double *px, double *py, double *pz);

/* Fields in the reference layout, FP64 host arrays of (Nx+2)(Ny+2)(Nz+2). */
int pic_set_field(pic_handle *h, int field, const double *host);
int pic_get_field(pic_handle *h, int field, double *host);

/* One full time step, Plasma::Step (gpu_plasma.h:605-620) without the MPI sum. */
int pic_step(pic_handle *h, int nt);
/* n steps back to back; if energies != NULL it receives 4 doubles per step
 * (pic_energy after each step). */
int pic_run(pic_handle *h, int nsteps, double *energies);

/* Sub-steps, in Plasma::Step order, so the control points map 1:1:
 *   pic_b_half        MagneticStageOne            gpu_plasma.h:524-538   (cp 50 after)
 *   pic_stage_fields  AssignCellsToArraysGPU      gpu_plasma.h:1006-1036 (no-op: staged in-kernel)
 *   pic_push_deposit  SetCurrentsToZero + Push + WriteCurrentsFromCellsToArrays
 *                                                 gpu_plasma.h:2058-2090
 *   pic_migrate       reorder_particles           gpu_plasma.h:2035-2046 (cp 270 after)
 *   pic_j_fold        SetPeriodicCurrents         gpu_plasma.h:980-993   (cp 275 before, 400 after)
 *   pic_b_complete    MagneticFieldStageTwo       gpu_plasma.h:540-551   (cp 500 after)
 *   pic_e_update      ElectricFieldEvaluate traces gpu_plasma.h:455-483  (cp 550 after)
 *   pic_e_ghosts      ElectricFieldComponentEvaluatePeriodic x3 gpu_plasma.h:486-507 (cp 600 after)
 */
int pic_b_half(pic_handle *h);
int pic_stage_fields(pic_handle *h);
int pic_push_deposit(pic_handle *h);
int pic_migrate(pic_handle *h);
int pic_j_fold(pic_handle *h);
int pic_b_complete(pic_handle *h);
int pic_e_update(pic_handle *h);
int pic_e_ghosts(pic_handle *h);

/* Particle counts per cell over all species, reference numbering,
 * (Nx+2)(Ny+2)(Nz+2) ints (ghost cells 0). */
int pic_get_cell_counts(pic_handle *h, int *counts);
/* One cell's particles of one species: the counterpart of reading a GPUCell
 * back to the host (GPUCell::copyCellFromDevice, gpucell.h:290-427).  cell is
 * the reference cell number ((i*(Ny+2) + l)*(Nz+2) + k) of an interior cell.
 * Particles live in tile bins, so a cell's particles are the slots of its
 * tile's bin that carry its cell index.  Writes up to cap particles in slot
 * order (global FP64 positions and momenta in either form; NULL arrays are
 * skipped) and their slots (indices into the species' bin storage);
 * *n = the cell's particle count (returned also when it exceeds cap, which is
 * PIC_ERR_ARG), *bin_offset = the first slot of the tile's bin. */
int pic_get_cell_particles(pic_handle *h, int species, int cell, int64_t cap, double *x, double *y, double *z,
                           double *px, double *py, double *pz, int64_t *slot, int64_t *n, int64_t *bin_offset);
int64_t pic_num_particles(pic_handle *h, int species); /* species < 0: all; negative on error */
/* Exports one species to host arrays (capacity cap); positions are global
 * FP64 (the mixed form converts cell + offset).  cell gets the reference cell
 * number.  *n receives the count.  Order is the device bin order. */
int pic_get_particles(pic_handle *h, int species, int64_t cap, double *x, double *y, double *z,
                      double *px, double *py, double *pz, int *cell, int64_t *n);

/* FP64 diagnostics: out[0] = 1/2 sum E^2, out[1] = 1/2 sum H^2 over nodes
 * 1..N of every axis, out[2] = kinetic sum (m/q_m)(gamma-1), out[3] = total.
 * The reference has only sum E^2 over all nodes (GPU_getCellEnergy,
 * wrap_kernel.cu:14-36), which pic_energy_reference returns. */
int pic_energy(pic_handle *h, double *out4);
int pic_energy_reference(pic_handle *h, double *out);
/* Charge conservation in FP64 (no counterpart in the reference, which has no
 * charge density).  rho[N] = sum over particles of m times the linear
 * (cloud-in-cell) weights on the nodes at cell centres -- array index N sits
 * at (N - 1/2) h per axis -- folded across the periodic boundaries like the
 * current (periodicCurrentElement, kernels.cu:1124-1146).  With the zigzag
 * deposit (CurrentToMesh, cell.h:1306-1422) and the E update (emeElement,
 * kernels.cu:1091-1102) the Gauss residual
 *   G[N] = sum_a (E_a[N] - E_a[N - e_a]) / h_a - rho[N]   (interior nodes)
 * stays what it was at the start, up to rounding.
 * pic_charge_density: rho in the reference layout (NULL: compute only).
 * pic_gauss_residual: G in the reference layout (0 on ghost nodes).
 * pic_gauss_check: computes G on the device; with set_baseline != 0 stores it
 *   as the baseline G0.  out4 = [max |G - G0|, max |rho|, rms over interior
 *   nodes of (G - G0), max |G0|].  Without a stored baseline and
 *   set_baseline = 0 it returns PIC_ERR_ARG. */
int pic_charge_density(pic_handle *h, double *rho_host);
int pic_gauss_residual(pic_handle *h, double *g_host);
int pic_gauss_check(pic_handle *h, int set_baseline, double *out4);
/* Total mechanical momentum of each species in FP64: out[3 s + a] = sum over
 * its particles of (m / q_m) p_a (p = gamma v, c = 1).  No counterpart in the
 * reference; used to state the FP32 form's momentum error. */
int pic_momentum(pic_handle *h, double *out);

/* Differentiable run (no counterpart in the reference, which has no
 * gradients).  pic_forward advances the state by `steps` time steps with the
 * same physics as pic_step, keeping every particle in a fixed order, stores
 * the particles and E/B every `ckpt_every` steps, and records the history
 * W[n][c] = h_x h_y h_z sum over nodes 1..N of E_c^2 after step n.
 * pic_backward then sweeps the steps in reverse -- per checkpoint segment it
 * recomputes the forward states and runs the adjoint kernels (transpose of
 * the ghost copies, the E update, the J fold and the B half steps; the
 * deposit's transpose as a gather; the push Jacobian with the interpolation's
 * transpose as a scatter) -- and returns the gradient of
 *   L = sum over the last `window` steps n of W[n][field]
 * with respect to the initial momenta of one species, and through
 * p0 = drift + vth * xi to that species' drift and thermal spread.
 * Particle order of the gradient = pic_get_particles order at the call to
 * pic_forward.  The buffers stay allocated until pic_adjoint_free, the next
 * pic_forward or pic_destroy.  Both forms are supported: the plain form
 * differentiates in FP64, the mixed form in FP32 (particles) with FP64 field
 * adjoints. */
typedef struct pic_loss {
    int field;        /* PIC_EX, PIC_EY or PIC_EZ */
    int window;       /* last steps of the forward run that the loss sums, 1..steps */
    int species;      /* species of the momentum gradient */
    int reserved_i;
    double drift[3];  /* that species' drift at initialisation */
    double vth;       /* that species' thermal spread at initialisation (> 0 for d_vth) */
    double reserved[4];
} pic_loss;

typedef struct pic_grads {
    double loss;        /* out: L */
    double d_drift[3];  /* out: dL/d drift */
    double d_vth;       /* out: dL/d vth = sum_i dL/dp_i . (p_i - drift)/vth */
    int64_t n;          /* in: capacity of d_p0 in particles; out: particles of the species */
    double *d_p0;       /* in: host array of 3*n doubles (px, py, pz of each particle) or NULL;
                           particles in the order pic_get_particles gave at the
                           start of the forward -- this handle's bin order, which
                           depends on its tiling (FP64 form 8x4x8 cells, FP32
                           form 6x4x8), so match particles by their state, not
                           by index, across handles; bins keep the load (or
                           generation) order inside a cell, so a stable sort by
                           cell gives an order common to all tilings */
    double reserved[4];
} pic_grads;

int pic_forward(pic_handle *h, int steps, int ckpt_every);
/* pic_forward with two checkpoint levels for runs whose states do not fit:
 * pic_backward recomputes each ckpt_every-step segment once to keep a state
 * every sub_every steps, then each sub-segment again to reverse it.  Device
 * memory: about steps/ckpt_every + ckpt_every/sub_every + sub_every + 1
 * particle states instead of steps/ckpt_every + ckpt_every + 1, for one more
 * forward recomputation.  sub_every = ckpt_every is pic_forward. */
int pic_forward2(pic_handle *h, int steps, int ckpt_every, int sub_every);
/* Exact checks of the adjoint (no counterpart in the reference).  The
 * deposit's zigzag split and the interpolation's tap choice make L only
 * piecewise smooth, so plain finite differences along dense directions are
 * limited by kinks and jumps.  With pic_branch_record(h, 1) the next
 * pic_forward / pic_forward2 of h (FP64 plain form) records every discrete
 * choice of every particle and step (tap indices, the integer parts of the
 * interpolation weights, the cell-centre indices of the zigzag split, the
 * periodic wraps and the cell moves: 8 bytes per particle-step, kept until
 * pic_adjoint_free / the next pic_forward / pic_destroy).
 * pic_forward_replay(h, steps, rec) runs a forward of h (no checkpoints)
 * that replays rec's recorded choices: a smooth function of the initial
 * state near rec's run, equal to it at the same state, and exactly the map
 * pic_backward differentiates.  h must hold the same particle counts per
 * species in the same order (same generator and seed).
 * pic_perturb_momenta adds eps * dp to the momenta of one species; dp holds
 * 3*n doubles (px, py, pz) in pic_get_particles order. */
int pic_branch_record(pic_handle *h, int on);
int pic_forward_replay(pic_handle *h, int steps, const pic_handle *recorded);
int pic_perturb_momenta(pic_handle *h, int species, int64_t n, const double *dp, double eps);
/* out[n*3 + c] = W[n][c] of the last forward run (host array of 3*steps) */
int pic_forward_history(pic_handle *h, double *out);
int pic_loss_value(pic_handle *h, const pic_loss *loss, double *value);
int pic_backward(pic_handle *h, const pic_loss *loss, pic_grads *grads);
/* device time of the last pic_forward and pic_backward, milliseconds */
int pic_adjoint_timings(pic_handle *h, float *out2);
int pic_adjoint_free(pic_handle *h);

/* Field energies without any allocation.  No counterpart in the reference.
 * For callers that cannot let the library call cudaMalloc (their framework
 * owns all device memory, or a timed loop cannot take cudaMalloc's implicit
 * device synchronisation).  Inputs: caller-owned DEVICE arrays of one field
 * component each in the reference layout ((Nx+2)(Ny+2)(Nz+2) FP64).  Output:
 * out3 (DEVICE, 3 doubles) = 1/2 sum E^2 and 1/2 sum H^2 over the nodes 1..N
 * of every axis (as pic_energy), and sum E^2 over all nodes (as
 * pic_energy_reference).  Work is enqueued on `stream` (a cudaStream_t, NULL
 * for the default stream); the result is ready when the stream reaches it.
 * Scratch: a file-scope device array of PIC_NOALLOC_MAX_BLOCKS x 3 doubles
 * (1.5 MB) that every GPU loading the library holds until exit; at most
 * PIC_NOALLOC_MAX_NODES nodes, larger grids return PIC_ERR_ARG.  The first
 * call on a device looks the array's device address up (cudaGetSymbolAddress),
 * so make that first call before any stream capture.  The address is kept for
 * the life of the process: it assumes the device's primary context lives as
 * long, so do not call this after cudaDeviceReset on that device.  All calls
 * share the array: calls that overlap on the GPU (other streams, other
 * threads) race; serialise them.  The result is deterministic (fixed-order
 * sums).  A CUDA error pending from the caller's own earlier work is returned
 * before anything is launched. */
#define PIC_NOALLOC_MAX_BLOCKS 65536
#define PIC_NOALLOC_MAX_NODES (PIC_NOALLOC_MAX_BLOCKS * 256)
int pic_field_energy_noalloc(int nx, int ny, int nz, const double *Ex, const double *Ey, const double *Ez,
                             const double *Hx, const double *Hy, const double *Hz, double *out3, void *stream);

/* The reference's Fortran-record dump ("mumu" file: LoadParticleData,
 * load_data.cu:308-341; readControlPoint, gpu_plasma.h:1088-1125), used as
 * the on-disk checkpoint/resume of a handle.  Records are an int32 byte
 * count, the payload and the count again: 12 field records (Ex Ey Ez Hx Hy
 * Hz Jx Jy Jz Qx Qy Qz, (Nx+2)(Ny+2)(Nz+2) FP64 in the reference layout),
 * then per particle sort a record (count, q/m, m) and six records x y z px
 * py pz (global positions).  A record holds at most 2^31-1 bytes (the
 * reference reader's int), so a species fits when it has at most
 * 268,435,455 particles.  The host functions need no GPU. */
typedef struct pic_mumu {
    int nx, ny, nz;
    int nsort;                                /* particle sorts in the file */
    double *fields[12];                       /* host arrays; NULL: write zeros / skip on read */
    int64_t count[PIC_MAX_SPECIES];
    double q_m[PIC_MAX_SPECIES], m[PIC_MAX_SPECIES];
    double *p[PIC_MAX_SPECIES][6];            /* x y z px py pz, count[s] each; NULL: zeros / skip */
} pic_mumu;
/* "mumu%03d%08d.dat" of control point num and step nt (the reference's name) */
int pic_mumu_name(int num, int nt, char *buf, int cap);
int pic_mumu_write(const char *path, const pic_mumu *d);
/* fills nsort, count, q_m and m of d (d->nx, ny, nz set by the caller) and
 * checks every record marker */
int pic_mumu_read_counts(const char *path, pic_mumu *d);
/* reads into the caller's arrays; nsort and count must be those of the file */
int pic_mumu_read(const char *path, pic_mumu *d);
/* Checkpoint / resume of a handle through the dump: every species in order,
 * E, H, J and (plain form) Q; the mixed form writes Q as zeros and its FP32
 * offsets as FP64 global positions.  pic_dump_read needs the same grid,
 * species count, q/m and charge weights, replaces every species' particles
 * and sets the stored fields.  No counterpart in the reference beyond the
 * format, which it only reads. */
int pic_dump_write(pic_handle *h, const char *path);
int pic_dump_read(pic_handle *h, const char *path);

/* The reference's random numbers (rnd_uniform / rnd_gaussian, maxwell.h:17-19;
 * g05cae / g05dde, maxwell.cu:77-170): a three-stream combined multiplicative
 * uniform generator in Wichmann-Hill form (moduli 30269 30307 30323) and
 * Brent's table-driven Gaussian (CACM algorithm 488).  The reference keeps the
 * state in globals; here it is the caller's.  pic_rnd_init sets the
 * reference's initial state (seeds 1 255 25555, stored uniform 1). */
typedef struct pic_rnd {
    int32_t ix, iy, iz;
    double store;
} pic_rnd;
void pic_rnd_init(pic_rnd *r);
double pic_rnd_uniform(pic_rnd *r);
double pic_rnd_gaussian(pic_rnd *r, double mean, double sd);
/* Brent's interval table, d[i] ~ Phi^-1(1 - 2^-(i+1)) for i = 0..40, as the
 * reference states it (41 doubles) */
int pic_rnd_table(double *out41);

/* The reference's quiet start (getUniformMaxwellianParticles,
 * maxwell.cu:676-757; InitUniformMaxwellianParticles, maxwell.cu:379-536),
 * the initial state of its default run (InitializeCPU, init.cu:111-139):
 * n_ions ions uniform in the box at rest, one beam electron on each ion inside
 * the beam region (drift rimp along x, spread Tb*rimp) and two plasma
 * electrons on every ion (spreads tex0 tey0 tez0, carrying the return
 * current rbd * beam velocity inside the beam's x/y region).  Host only. */
typedef struct pic_quiet {
    int64_t n_ions;                     /* jmb; 1,600,000 in the reference */
    double tex0, tey0, tez0;            /* electron thermal spreads */
    double Tb, rimp, rbd, ni;           /* beam spread / drift / density, plasma density */
    int meh, lp, beamf;                 /* y offset in boxes, particles per cell, return current on */
    double lx, ly, lz;                  /* box */
    double beam_lx, beam_ly, beam_lz;   /* beam region (centred in y and z) */
} pic_quiet;
/* the reference's values (maxwell.cu:680-696, 716-718) */
int pic_quiet_defaults(pic_quiet *q);
/* ion[6] (x y z px py pz) hold n_ions each, el[6] 2*n_ions, beam[6] n_ions;
 * *n_beam receives the beam electrons written (beam entries past it are
 * untouched: the reference hands n_ions beam entries to its cells whatever
 * the count, from unset memory past it, and its electron pair j reads beam j,
 * taken here as zero past the count -- at the reference's values the beam
 * region is the whole box and the count is n_ions).  q_m3 / m3 (may be NULL)
 * receive q/m and the charge weight of ions, electrons, beam (getMassCharge,
 * maxwell.cu:598-612).  With n_ions = 0 only q_m3 and m3 are written. */
int pic_quiet_start(const pic_quiet *q, double *const ion[6], double *const el[6], double *const beam[6],
                    int64_t *n_beam, double *q_m3, double *m3);

/* Status and errors. */
int pic_sync(pic_handle *h);
int pic_last_status(pic_handle *h);
const char *pic_last_error_string(pic_handle *h);
const char *pic_error_string(int status);
/* Per-step counters of the last step: [0] particles moved to another tile,
 * [1] particles no cell accepted (dropped), [2] particles two or more cells
 * accepted (duplicated), [3] kernel launches of the step. */
int pic_step_counters(pic_handle *h, int64_t *out4);
/* Timings of the last pic_step in milliseconds (CUDA events on the handle's
 * stream): [0] B half step, [1] the push/deposit kernel alone, [2] migration
 * arrivals, [3] J fold + B completion + E update + E ghosts, [4] whole step. */
int pic_step_timings(pic_handle *h, float *out5);
/* Internal sizes for the roofline: [0] tiles [1] total particle slots
 * [2] bytes per particle (28 mixed / 52 plain) [3] field nodes. */
int pic_layout_info(pic_handle *h, int64_t *out4);
/* The CUDA stream of the handle, as void* (cudaStream_t). */
void *pic_stream(pic_handle *h);

#ifdef __cplusplus
}
#endif
#endif /* PIC0BUF_H */
