// C ABI of the B200 PIC step (include/pic0buf.h): handle lifecycle, particle
// binning, the step sequence of Plasma::Step (gpu_plasma.h:605-620), field
// I/O in the reference layout, diagnostics.  Every call returns an int
// status and never exits the process (the reference prints and exit()s,
// e.g. gpu_plasma.h:1904-1910, 1953-1958).
#include <cuda_runtime.h>
#include <string.h>
#include <stdio.h>
#include <math.h>
#include <string>
#include <type_traits>
#include <vector>
#include <algorithm>
#include <functional>
#include "pic0buf.h"
#include "pic_internal.cuh"
#include "pic_kernels.cuh"
#include "pic_rng.cuh"
#include "pic_handle.cuh"

using namespace pic;
using namespace pic_host;

namespace pic_host {

int set_err(pic_handle *h, int code, const char *msg) {
    if (h) {
        h->status = code;
        snprintf(h->err, sizeof(h->err), "%s", msg);
    }
    return code;
}

int cuda_err(pic_handle *h, cudaError_t e, const char *where) {
    if (e == cudaSuccess) return PIC_OK;
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return set_err(h, PIC_ERR_NOMEM, buf);
    return set_err(h, (int)e, buf);
}

cudaError_t dev_alloc(pic_handle *h, void **p, size_t bytes) {
    (void)h;
    return cudaMalloc(p, bytes > 0 ? bytes : 16);
}

void dev_free(pic_handle *h, void *p) {
    (void)h;
    if (p) cudaFree(p);
}

void release_load_scratch(pic_handle *h) {
    if (h->load_buf) cudaFree(h->load_buf);
    h->load_buf = nullptr;
    h->load_bytes = 0;
}


size_t elem_particle(int mixed) { return mixed ? 28 : 52; }

StepParams make_params(pic_handle *h) {
    StepParams p;
    memset(&p, 0, sizeof(p));
    p.g = h->g;
    p.nsp = h->cfg.nspecies;
    p.mixed = h->mixed;
    for (int s = 0; s < p.nsp; s++) p.sp[s] = h->sp[s].v;
    for (int c = 0; c < 3; c++) {
        p.E[c] = h->f[PIC_EX + c];
        p.H[c] = h->f[PIC_HX + c];
        p.J[c] = (double *)h->f[PIC_JX + c];
    }
    p.outbox = h->outbox;
    p.out_cap = h->out_cap;
    p.st = h->st;
    if (h->lb_buf) {
        p.lb_prev = h->lb_buf + h->lb_par * kMaxSpecies;
        p.lb_cur = (unsigned *)(h->lb_buf + (h->lb_par ^ 1) * kMaxSpecies);
    }
    return p;
}

void free_species(pic_handle *h, int s) {
    SpeciesView &v = h->sp[s].v;
    void *ptrs[] = {v.x, v.y, v.z, v.px, v.py, v.pz, v.ox, v.oy, v.oz, v.fx, v.fy, v.fz, v.cell, v.tile_start,
                    v.tile_count};
    for (void *p : ptrs) dev_free(h, p);
    double q_m = v.q_m, m = v.m;
    memset(&v, 0, sizeof(v));
    v.q_m = q_m;
    v.m = m;
    h->sp[s].cap_total = 0;
    h->sp[s].loaded = 0;
    h->sp[s].h_start.clear();
    h->tile_cap_valid = 0;
}

// capacity per tile from counts; allocates the species arrays and uploads the
// tile starts.  Slots start on multiples of 32 particles.
int alloc_species(pic_handle *h, int s, const std::vector<int> &counts) {
    const Grid &g = h->g;
    double slack = h->cfg.capacity_slack > 0 ? h->cfg.capacity_slack : 0.25;
    std::vector<int> start(g.ntiles + 1);
    int64_t acc = 0;
    for (int t = 0; t < g.ntiles; t++) {
        start[t] = (int)acc;
        int64_t pad = h->cfg.capacity_pad >= 0 ? h->cfg.capacity_pad : 64;
        int64_t cap = (int64_t)counts[t] + (int64_t)ceil(counts[t] * slack) + pad;
        if (pad > 0) cap = (cap + 31) / 32 * 32;
        // the FP32 push reads and writes particles in 8-byte pairs: every tile starts on an even slot
        if (h->mixed) cap = (cap + 1) / 2 * 2;
        // the plain form's two-word tile J stays exact up to kFxMaxTileSlots
        // particles in a tile over all species
        if (!h->mixed && cap > kFxMaxTileSlots / h->cfg.nspecies)
            return set_err(h, PIC_ERR_ARG, "too many particles in one tile for the FP64 tile current");
        acc += cap;
        if (acc > 0x7fffff00LL) return set_err(h, PIC_ERR_ARG, "species capacity exceeds 2^31 slots");
    }
    start[g.ntiles] = (int)acc;
    free_species(h, s);
    SpeciesView &v = h->sp[s].v;
    size_t n = (size_t)acc;
    CK(dev_alloc_n(h, &v.cell, n), "alloc cell");
    if (!h->mixed) {
        double **arr[6] = {&v.x, &v.y, &v.z, &v.px, &v.py, &v.pz};
        for (auto a : arr) CK(dev_alloc_n(h, a, n), "alloc particles");
    } else {
        float **arr[6] = {&v.ox, &v.oy, &v.oz, &v.fx, &v.fy, &v.fz};
        for (auto a : arr) CK(dev_alloc_n(h, a, n), "alloc particles");
    }
    CK(dev_alloc_n(h, &v.tile_start, (size_t)g.ntiles + 1), "alloc tile_start");
    CK(dev_alloc_n(h, &v.tile_count, (size_t)g.ntiles), "alloc tile_count");
    CK(cudaMemcpyAsync(v.tile_start, start.data(), (g.ntiles + 1) * sizeof(int), cudaMemcpyHostToDevice, h->stream),
       "upload tile_start");
    CK(cudaMemsetAsync(v.cell, 0xff, n * sizeof(int), h->stream), "clear cells");
    h->sp[s].cap_total = acc;
    h->sp[s].h_start = start;
    h->sp[s].loaded = 1;
    h->sp[s].lb_known = 0;
    h->tile_cap_valid = 0;
    return PIC_OK;
}

int ensure_outbox(pic_handle *h) {
    if (h->outbox_pinned) return PIC_OK;  // leftovers of an overflowing insert still live in it
    int64_t total = 0;
    for (int s = 0; s < h->cfg.nspecies; s++) total += h->sp[s].cap_total;
    double frac = h->cfg.outbox_fraction > 0 ? h->cfg.outbox_fraction : 0.04;
    int64_t want = (int64_t)(frac * (double)total) + 65536;
    if (want > 0x7fffffffLL) want = 0x7fffffffLL;
    if (h->outbox && (int64_t)h->out_cap >= want) return PIC_OK;
    if (h->outbox) cudaFree(h->outbox);
    h->outbox = nullptr;
    CK(cudaMalloc(&h->outbox, (size_t)want * h->out_elem), "alloc outbox");
    h->out_cap = (unsigned)want;
    return PIC_OK;
}

// flat device list (cell computed, -1 = rejected) -> bins of species s
using ScatterFn = std::function<cudaError_t(const SpeciesView &, int *)>;

int build_bins_with(pic_handle *h, int s, int64_t n, int *cell, const ScatterFn &scatter, int64_t *inserted) {
    const Grid &g = h->g;
    ScratchGuard guard(h);
    int *tc = nullptr;
    CK(guard.alloc(&tc, (size_t)g.ntiles), "alloc tile counts");
    CK(cudaMemsetAsync(tc, 0, g.ntiles * sizeof(int), h->stream), "memset");
    CK(tile_histogram(g, n, cell, tc, h->stream), "tile histogram");
    std::vector<int> counts(g.ntiles);
    CK(cudaMemcpyAsync(counts.data(), tc, g.ntiles * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "counts");
    CK(cudaStreamSynchronize(h->stream), "sync");
    int rc = alloc_species(h, s, counts);
    if (rc) return rc;
    CK(cudaMemsetAsync(tc, 0, g.ntiles * sizeof(int), h->stream), "memset");
    CK(scatter(h->sp[s].v, tc), "scatter");
    CK(cudaMemcpyAsync(h->sp[s].v.tile_count, tc, g.ntiles * sizeof(int), cudaMemcpyDeviceToDevice, h->stream),
       "tile counts");
    CK(cudaStreamSynchronize(h->stream), "sync");
    int64_t tot = 0;
    for (int c : counts) tot += c;
    if (inserted) *inserted = tot;
    h->kin_valid = 0;
    return ensure_outbox(h);
}

int build_bins(pic_handle *h, int s, int64_t n, int *cell, const double *x, const double *y, const double *z,
               const double *px, const double *py, const double *pz, int64_t *inserted) {
    const Grid &g = h->g;
    int mixed = h->mixed;
    cudaStream_t st = h->stream;
    return build_bins_with(h, s, n, cell, [&](const SpeciesView &v, int *fill) {
        return scatter_to_bins(g, mixed, n, cell, x, y, z, px, py, pz, v, fill, st);
    }, inserted);
}

int build_bins_f(pic_handle *h, int s, int64_t n, int *cell, const float *ox, const float *oy, const float *oz,
                 const float *px, const float *py, const float *pz) {
    const Grid &g = h->g;
    int mixed = h->mixed;
    cudaStream_t st = h->stream;
    return build_bins_with(h, s, n, cell, [&](const SpeciesView &v, int *fill) {
        return scatter_to_bins_f(g, mixed, n, cell, ox, oy, oz, px, py, pz, v, fill, st);
    }, nullptr);
}

int tile_counts(pic_handle *h, int s, std::vector<int> &counts) {
    counts.assign(h->g.ntiles, 0);
    if (!h->sp[s].loaded) return PIC_OK;
    CK(cudaMemcpyAsync(counts.data(), h->sp[s].v.tile_count, h->g.ntiles * sizeof(int), cudaMemcpyDeviceToHost,
                       h->stream), "counts");
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int load_device(pic_handle *h, int s, int64_t n, const double *x, const double *y, const double *z,
                const double *px, const double *py, const double *pz, int64_t *inserted) {
    ScratchGuard guard(h);
    int *cell = nullptr;
    CK(guard.alloc(&cell, (size_t)(n > 0 ? n : 1)), "alloc cell");
    CK(place_particles_plain(h->g, n, x, y, z, cell, h->stream), "place");
    return build_bins(h, s, n, cell, x, y, z, px, py, pz, inserted);
}

// gather the live particles (+ outbox leftovers) of species s and rebuild its bins
int rebin_species(pic_handle *h, int s, unsigned n_out) {
    const Grid &g = h->g;
    SpeciesView &v = h->sp[s].v;
    std::vector<int> counts(g.ntiles);
    CK(cudaMemcpyAsync(counts.data(), v.tile_count, g.ntiles * sizeof(int), cudaMemcpyDeviceToHost, h->stream),
       "counts");
    CK(cudaStreamSynchronize(h->stream), "sync");
    std::vector<int64_t> dstart(g.ntiles + 1);
    int64_t acc = 0;
    for (int t = 0; t < g.ntiles; t++) { dstart[t] = acc; acc += counts[t]; }
    dstart[g.ntiles] = acc;
    int64_t nmax = acc + n_out;
    ScratchGuard guard(h);
    double *buf = nullptr;
    int *cell = nullptr;
    int64_t *ddst = nullptr;
    unsigned *ctr = nullptr;
    CK(guard.alloc(&buf, (size_t)(nmax > 0 ? nmax : 1) * 6), "rebin buffer");
    CK(guard.alloc(&cell, (size_t)(nmax > 0 ? nmax : 1)), "rebin cells");
    CK(guard.alloc(&ddst, (size_t)g.ntiles + 1), "rebin starts");
    CK(guard.alloc(&ctr, 1), "rebin counter");
    CK(cudaMemsetAsync(ctr, 0, sizeof(unsigned), h->stream), "memset");
    CK(cudaMemcpyAsync(ddst, dstart.data(), (g.ntiles + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream),
       "starts");
    size_t N = (size_t)(nmax > 0 ? nmax : 1);
    double *x = buf, *y = buf + N, *z = buf + 2 * N, *px = buf + 3 * N, *py = buf + 4 * N, *pz = buf + 5 * N;
    CK(gather_from_bins(g, h->mixed, v, ddst, x, y, z, px, py, pz, cell, h->stream), "gather");
    StepParams p = make_params(h);
    CK(gather_outbox(p, s, n_out, ctr, acc, x, y, z, px, py, pz, cell, h->stream), "gather outbox");
    unsigned extra = 0;
    CK(cudaMemcpyAsync(&extra, ctr, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream), "counter");
    CK(cudaStreamSynchronize(h->stream), "sync");
    return build_bins(h, s, acc + extra, cell, x, y, z, px, py, pz, nullptr);
}

int check_status(pic_handle *h) {
    CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream), "status");
    CK(cudaStreamSynchronize(h->stream), "sync");
    const DevStatus &st = *h->st_host;
    h->counters[0] = (int64_t)st.moved;
    h->counters[1] = (int64_t)st.dropped;
    h->counters[2] = (int64_t)st.duplicated;
    char msg[200];
    const unsigned fatal = ST_STENCIL | ST_NAN | ST_BADCELL | ST_OUTBOX | ST_TMA;
    if (st.flags & fatal) {
        int code = (st.flags & ST_NAN) ? PIC_ERR_NAN
                   : (st.flags & ST_STENCIL) ? PIC_ERR_STENCIL
                   : (st.flags & (ST_BADCELL | ST_TMA)) ? PIC_ERR_STATE : PIC_ERR_OUTBOX;
        snprintf(msg, sizeof(msg),
                 "%s (status flags 0x%x: 1 stencil, 2 outbox, 4 holes, 8 nan, 16 tile full, 32 bins, 64 field tile load "
                 "timed out)",
                 pic_error_string(code), st.flags);
        return set_err(h, code, msg);
    }
    if (st.flags & ST_TILE_FULL) {
        unsigned n_out = st.out_count < h->out_cap ? st.out_count : h->out_cap;
        // the outbox keeps every species' leftovers until the last species has
        // taken its own: a rebin must not resize (and so clear) it on the way
        h->outbox_pinned = 1;
        for (int s = 0; s < h->cfg.nspecies; s++) {
            int rc = rebin_species(h, s, n_out);
            if (rc) { h->outbox_pinned = 0; return rc; }
        }
        h->outbox_pinned = 0;
        int rc = ensure_outbox(h);
        if (rc) return rc;
        // leftovers are in the bins now
        CK(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), h->stream), "reset status");
        h->kin_valid = 0;
    }
    if (st.flags & ST_HOLES) {
        // dead slots remain inside the bins; a rebin compacts them
        for (int s = 0; s < h->cfg.nspecies; s++) {
            int rc = rebin_species(h, s, 0);
            if (rc) return rc;
        }
        CK(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), h->stream), "reset status");
        h->kin_valid = 0;
    }
    return PIC_OK;
}

int need_particles(pic_handle *h) {
    for (int s = 0; s < h->cfg.nspecies; s++)
        if (!h->sp[s].loaded) {
            // an empty species: bins with zero counts
            std::vector<int> zero(h->g.ntiles, 0);
            int rc = alloc_species(h, s, zero);
            if (rc) return rc;
            CK(cudaMemsetAsync(h->sp[s].v.tile_count, 0, h->g.ntiles * sizeof(int), h->stream), "memset");
            rc = ensure_outbox(h);
            if (rc) return rc;
        }
    return PIC_OK;
}

int do_b_half(pic_handle *h) {
    if (!h->mixed) yee_b_half_plain(h->g, (double *const *)h->f, h->stream);
    else yee_b_half_mixed(h->g, (float *const *)&h->f[PIC_EX], (float *const *)&h->f[PIC_HX], h->stream);
    CK(cudaGetLastError(), "b_half");
    h->launches += 1;
    return PIC_OK;
}

// The plain push's int32 remainder word needs fewer than 2^(31 - kFxLo32MinBits)
// particles in every tile.  A tile never holds more than its bins' capacities
// (an overflow leaves the particle in the outbox and rebins), so the largest
// per-tile sum of capacities over the species decides for the launch.
bool plain_lo32(pic_handle *h) {
    if (!h->tile_cap_valid) {
        int64_t mx = 0;
        for (int t = 0; t < h->g.ntiles; t++) {
            int64_t c = 0;
            for (int s = 0; s < h->cfg.nspecies; s++) {
                const std::vector<int> &st = h->sp[s].h_start;
                if (!st.empty()) c += st[t + 1] - st[t];
            }
            mx = std::max(mx, c);
        }
        h->tile_cap_max = mx;
        h->tile_cap_valid = 1;
    }
    int b = 0;
    while ((1ll << b) <= h->tile_cap_max) b++;
    return 31 - b >= kFxLo32MinBits;
}

int do_push_deposit(pic_handle *h, int b_half_in_push = 0) {
    int rc = need_particles(h);
    if (rc) return rc;
    // the outbox is sized once for all species (the loads leave that to the
    // first push)
    if ((rc = ensure_outbox(h))) return rc;
    size_t nodes = h->g.nodes_pitched();
    for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(h->f[PIC_JX + c], 0, nodes * sizeof(double), h->stream), "zero J");
    CK(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), h->stream), "reset status");
    if (h->mixed) {
        // species loaded since the last push: their contribution bound from their momenta
        float *prev = h->lb_buf + h->lb_par * kMaxSpecies;
        for (int s = 0; s < h->cfg.nspecies; s++) {
            if (h->sp[s].lb_known) continue;
            CK(cudaMemsetAsync(prev + s, 0, sizeof(float), h->stream), "reset bound");
            CK(contribution_bound_mixed(h->g, h->sp[s].v, h->sp[s].cap_total, (unsigned *)(prev + s), h->stream),
               "contribution bound");
            h->launches += 1;
            h->sp[s].lb_known = 1;
        }
        CK(cudaMemsetAsync(h->lb_buf + (h->lb_par ^ 1) * kMaxSpecies, 0, kMaxSpecies * sizeof(float), h->stream),
           "reset bounds");
    }
    StepParams p = make_params(h);
    p.b_half = b_half_in_push;
    cudaEventRecord(h->ev[2], h->stream);
    CK(h->mixed ? launch_push_mixed(p, h->maps, h->stream) : launch_push_plain(p, plain_lo32(h), h->stream),
       "push_deposit");
    cudaEventRecord(h->ev[3], h->stream);
    if (h->mixed) h->lb_par ^= 1;
    h->launches += 1;
    h->kin_valid = 1;
    return PIC_OK;
}

int do_migrate(pic_handle *h) {
    StepParams p = make_params(h);
    CK(launch_insert(p, h->stream), "insert");
    return check_status(h);
}

int do_b_complete(pic_handle *h) {
    if (!h->mixed) yee_b_complete_plain(h->g, (double *const *)h->f, h->stream);
    else yee_b_half_mixed(h->g, (float *const *)&h->f[PIC_EX], (float *const *)&h->f[PIC_HX], h->stream);
    CK(cudaGetLastError(), "b_complete");
    h->launches += 1;
    return PIC_OK;
}

int do_e_update(pic_handle *h) {
    if (!h->mixed) yee_e_update_plain(h->g, (double *const *)h->f, h->stream);
    else
        yee_e_update_mixed(h->g, (float *const *)&h->f[PIC_EX], (float *const *)&h->f[PIC_HX],
                           (double *const *)&h->f[PIC_JX], h->stream);
    CK(cudaGetLastError(), "e_update");
    h->launches += 1;
    return PIC_OK;
}

int do_e_ghosts(pic_handle *h) {
    int per = h->cfg.ghosts == PIC_GHOSTS_PERIODIC;
    if (!h->mixed)
        e_ghosts_plain(h->g, (double *)h->f[PIC_EX], (double *)h->f[PIC_EY], (double *)h->f[PIC_EZ], per, h->stream);
    else
        e_ghosts_mixed(h->g, (float *)h->f[PIC_EX], (float *)h->f[PIC_EY], (float *)h->f[PIC_EZ], per, h->stream);
    CK(cudaGetLastError(), "e_ghosts");
    h->launches += 1;
    return PIC_OK;
}

int do_j_fold(pic_handle *h) {
    j_fold(h->g, (double *)h->f[PIC_JX], (double *)h->f[PIC_JY], (double *)h->f[PIC_JZ], h->stream);
    CK(cudaGetLastError(), "j_fold");
    h->launches += 3;
    return PIC_OK;
}

int set_device(pic_handle *h) {
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    return PIC_OK;
}

}  // namespace pic_host

extern "C" {

void pic_config_init(pic_config *cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof(*cfg));
    cfg->precision = PIC_FP64_PLAIN;
    cfg->ghosts = PIC_GHOSTS_REFERENCE;
    cfg->nspecies = 1;
    cfg->capacity_slack = 0.25;
    cfg->outbox_fraction = 0.04;
    cfg->capacity_pad = -1;
}

int pic_create(const pic_config *cfg, pic_handle **out) {
    if (!cfg || !out) return PIC_ERR_ARG;
    *out = nullptr;
    if (cfg->nx < 3 || cfg->ny < 3 || cfg->nz < 3) return PIC_ERR_ARG;
    if (!(cfg->lx > 0) || !(cfg->ly > 0) || !(cfg->lz > 0) || !(cfg->tau > 0)) return PIC_ERR_ARG;
    if (cfg->nspecies < 1 || cfg->nspecies > PIC_MAX_SPECIES) return PIC_ERR_ARG;
    if (cfg->precision != PIC_FP64_PLAIN && cfg->precision != PIC_FP32_MIXED) return PIC_ERR_ARG;
    for (int s = 0; s < cfg->nspecies; s++)
        if (!(cfg->species[s].q_m != 0.0) || !isfinite(cfg->species[s].q_m) || !isfinite(cfg->species[s].m))
            return PIC_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PIC_ERR_NO_DEVICE;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return PIC_ERR_ARG;
    pic_handle *h = new pic_handle();
    memset(h->f, 0, sizeof(h->f));
    h->cfg = *cfg;
    h->device = cfg->device;
    h->mixed = cfg->precision == PIC_FP32_MIXED;
    h->out_elem = h->mixed ? sizeof(OutMixed) : sizeof(OutPlain);
    h->outbox = nullptr;
    h->out_cap = 0;
    h->status = 0;
    h->err[0] = 0;
    h->kin_valid = 0;
    h->timed = 0;
    memset(h->counters, 0, sizeof(h->counters));
    memset(h->timings, 0, sizeof(h->timings));
    Grid &g = h->g;
    g.nx = cfg->nx; g.ny = cfg->ny; g.nz = cfg->nz;
    g.NX = g.nx + 2; g.NY = g.ny + 2; g.NZ = g.nz + 2;
    g.pz = (g.NZ + 3) / 4 * 4;
    g.lx = cfg->lx; g.ly = cfg->ly; g.lz = cfg->lz; g.tau = cfg->tau;
    g.hx = cfg->lx / ((double)cfg->nx);  // Cell ctor, cell.h:734
    g.hy = cfg->ly / ((double)cfg->ny);
    g.hz = cfg->lz / ((double)cfg->nz);
    // automatic tiles: 6x4x8 in the FP32 form, whose 256-thread CTAs (an
    // int32 tile current per two warps) then fit two per SM in shared memory
    // (c2 push 18.82 ms against 19.01 for 4x4x12; c4 5.07 against 5.21);
    // 8x4x8 in the FP64 form (c2 push 70.5 ms against 71.1 for 4x4x16)
    g.tx = cfg->tile[0] > 0 ? cfg->tile[0] : std::min(h->mixed ? 6 : 8, g.nx);
    g.ty = cfg->tile[1] > 0 ? cfg->tile[1] : std::min(4, g.ny);
    const int tz_auto = 8;
    g.tz = cfg->tile[2] > 0 ? cfg->tile[2] : (g.nz >= tz_auto ? tz_auto : (g.nz + 3) / 4 * 4);
    if (g.tz % 4 != 0 || g.tx < 1 || g.ty < 1 || g.tx > 16 || g.ty > 16 || g.tz > 32) { delete h; return PIC_ERR_ARG; }
    g.ntx = (g.nx + g.tx - 1) / g.tx;
    g.nty = (g.ny + g.ty - 1) / g.ty;
    g.ntz = (g.nz + g.tz - 1) / g.tz;
    g.ntiles = g.ntx * g.nty * g.ntz;
    auto bits = [](int n) { int b = 0; while ((1 << b) < n) b++; return b; };
    g.bz = bits(g.nz);
    g.by = bits(g.ny);
    if (bits(g.nx) + g.by + g.bz > 31) { delete h; return PIC_ERR_ARG; }  // packed int32 cell index
    for (int s = 0; s < cfg->nspecies; s++) {
        memset(&h->sp[s].v, 0, sizeof(SpeciesView));
        h->sp[s].v.q_m = cfg->species[s].q_m;
        h->sp[s].v.m = cfg->species[s].m;
        h->sp[s].loaded = 0;
        h->sp[s].cap_total = 0;
    }
    int rc = set_device(h);
    if (rc) { delete h; return rc; }
    size_t smem = h->mixed ? push_smem_total_mixed(g) : push_smem_plain(g);
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    if (smem > (size_t)optin) { delete h; return PIC_ERR_ARG; }
    auto fail = [&](cudaError_t e) { pic_destroy(h); return e == cudaErrorMemoryAllocation ? PIC_ERR_NOMEM : (int)e; };
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e) { delete h; return (int)e; }
    for (int i = 0; i < 6; i++) cudaEventCreate(&h->ev[i]);
    if ((e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    for (int i = 0; i < 5; i++)
        if ((e = cudaEventCreateWithFlags(&h->lev[i], cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    size_t nodes = g.nodes_pitched();
    for (int fi = 0; fi < PIC_FIELD_COUNT; fi++) {
        size_t es = sizeof(double);
        if (h->mixed) {
            if (fi >= PIC_QX) continue;
            if (fi < PIC_JX) es = sizeof(float);
        }
        if ((e = cudaMalloc(&h->f[fi], nodes * es)) != cudaSuccess) return fail(e);
        // on the handle's stream: the legacy-stream cudaMemset does not order
        // before work on a non-blocking stream
        if ((e = cudaMemsetAsync(h->f[fi], 0, nodes * es, h->stream)) != cudaSuccess) return fail(e);
    }
    if ((e = cudaMalloc(&h->dense, g.nodes_ref() * sizeof(double))) != cudaSuccess) return fail(e);
    if (h->mixed) {
        if ((e = encode_field_maps(g, (float *const *)&h->f[PIC_EX], (float *const *)&h->f[PIC_HX], &h->maps)) !=
            cudaSuccess)
            return fail(e);

        if ((e = cudaMalloc(&h->lb_buf, 2 * kMaxSpecies * sizeof(float))) != cudaSuccess) return fail(e);
        if ((e = cudaMemsetAsync(h->lb_buf, 0, 2 * kMaxSpecies * sizeof(float), h->stream)) != cudaSuccess)
            return fail(e);
    }
    if ((e = cudaMalloc(&h->st, sizeof(DevStatus))) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(h->st, 0, sizeof(DevStatus), h->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaMallocHost(&h->st_host, sizeof(DevStatus))) != cudaSuccess) return fail(e);
    memset(h->st_host, 0, sizeof(DevStatus));
    if ((e = cudaMalloc(&h->dred, 8 * sizeof(double))) != cudaSuccess) return fail(e);
    if ((e = cudaMallocHost(&h->hred, 8 * sizeof(double))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&h->dcounts, (size_t)g.ncells() * sizeof(int))) != cudaSuccess) return fail(e);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return fail(e);
    *out = h;
    return PIC_OK;
}

int pic_destroy(pic_handle *h) {
    if (!h) return PIC_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    adj_free(h);
    for (int s = 0; s < h->cfg.nspecies; s++) free_species(h, s);
    for (int fi = 0; fi < PIC_FIELD_COUNT; fi++)
        if (h->f[fi]) cudaFree(h->f[fi]);
    if (h->dense) cudaFree(h->dense);
    if (h->outbox) cudaFree(h->outbox);
    if (h->st) cudaFree(h->st);
    if (h->st_host) cudaFreeHost(h->st_host);
    if (h->dred) cudaFree(h->dred);
    if (h->hred) cudaFreeHost(h->hred);
    if (h->dcounts) cudaFree(h->dcounts);
    if (h->lb_buf) cudaFree(h->lb_buf);
    release_load_scratch(h);

    double *diag[3] = {h->rho, h->gauss, h->gauss0};
    for (double *d : diag)
        if (d) cudaFree(d);
    for (int i = 0; i < 6; i++)
        if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    for (int i = 0; i < 5; i++)
        if (h->lev[i]) cudaEventDestroy(h->lev[i]);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return PIC_OK;
}

int pic_load_particles(pic_handle *h, int species, int64_t n, const double *x, const double *y, const double *z,
                       const double *px, const double *py, const double *pz, int64_t *inserted) {
    if (!h || species < 0 || species >= h->cfg.nspecies || n < 0) return set_err(h, PIC_ERR_ARG, "bad argument");
    if (n > 0 && (!x || !y || !z || !px || !py || !pz)) return set_err(h, PIC_ERR_ARG, "null array");
    int rc = set_device(h);
    if (rc) return rc;
    size_t N = (size_t)(n > 0 ? n : 1);
    ScratchGuard guard(h);
    double *buf = nullptr;
    CK(guard.alloc(&buf, N * 6), "alloc load buffer");
    const double *src[6] = {x, y, z, px, py, pz};
    for (int a = 0; a < 6; a++)
        if (n > 0) CK(cudaMemcpyAsync(buf + a * N, src[a], (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream), "H2D particles");
    return load_device(h, species, n, buf, buf + N, buf + 2 * N, buf + 3 * N, buf + 4 * N, buf + 5 * N, inserted);
}

int pic_load_particles_device(pic_handle *h, int species, int64_t n, const double *x, const double *y,
                              const double *z, const double *px, const double *py, const double *pz,
                              int64_t *inserted) {
    if (!h || species < 0 || species >= h->cfg.nspecies || n < 0) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    return load_device(h, species, n, x, y, z, px, py, pz, inserted);
}

// Host -> device in chunks on a second stream, overlapped with the device
// work on the handle's stream (two staging buffers per pass):
//   pass 1  cells and offsets: each chunk is validated and placed
//           (place_particles_cells) and counted per tile as soon as it lands;
//   bins    allocated from the tile counts (one host sync);
//   pass 2  momenta: each chunk is scattered into the bins as it lands.
// Every byte crosses the bus once; the copy engine and the kernels overlap.
static constexpr int64_t kLoadChunk = 1 << 24;  // particles per staged chunk

int pic_load_particles_cells(pic_handle *h, int species, int64_t n, const int32_t *cell, const float *ox,
                             const float *oy, const float *oz, const float *px, const float *py, const float *pz,
                             int64_t *inserted) {
    if (!h || species < 0 || species >= h->cfg.nspecies || n < 0) return set_err(h, PIC_ERR_ARG, "bad argument");
    if (n > 0 && (!cell || !ox || !oy || !oz || !px || !py || !pz)) return set_err(h, PIC_ERR_ARG, "null array");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    cudaStream_t st = h->stream, cs = h->copy_stream;
    const size_t N = (size_t)(n > 0 ? n : 1);
    const size_t C = (size_t)std::min<int64_t>(kLoadChunk, n > 0 ? n : 1);
    const int64_t nchunks = (n + kLoadChunk - 1) / kLoadChunk;
    int *icell = nullptr, *tc = nullptr, *stage_cell[2] = {nullptr, nullptr};
    float *off[3] = {nullptr, nullptr, nullptr}, *stage_mom[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    auto release = [&]() {};  // the staging stays in the handle for the next species
    auto ck = [&](cudaError_t e, const char *where) {
        if (e == cudaSuccess) return PIC_OK;
        cudaStreamSynchronize(cs);
        release();
        return cuda_err(h, e, where);
    };
#define LCK(expr, where) do { int r_ = ck((expr), (where)); if (r_) return r_; } while (0)
    // the staging: cells and offsets of all n particles, the tile counts and
    // two chunks of cells and momenta, carved from one buffer that the
    // handle keeps between loads (allocating and freeing ~16 B per particle
    // for every species cost up to ~0.8 s of a c2 load)
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t need = al(N * 4) + al((size_t)g.ntiles * 4) + 3 * al(N * 4) + 2 * (al(C * 4) + 3 * al(C * 4));
    if (h->load_bytes < need) {
        release_load_scratch(h);
        LCK(dev_alloc(h, &h->load_buf, need), "alloc load buffer");
        h->load_bytes = need;
    }
    {
        char *q = (char *)h->load_buf;
        auto take = [&](auto *&p, size_t bytes) {
            p = (std::remove_reference_t<decltype(p)>)q;
            q += al(bytes);
        };
        take(icell, N * 4);
        take(tc, (size_t)g.ntiles * 4);
        for (int a = 0; a < 3; a++) take(off[a], N * 4);
        for (int b = 0; b < 2; b++) {
            take(stage_cell[b], C * 4);
            for (int a = 0; a < 3; a++) take(stage_mom[b][a], C * 4);
        }
    }
    LCK(cudaMemsetAsync(tc, 0, g.ntiles * sizeof(int), st), "memset");
    // the copy stream may use the new memory once its allocation is ordered before it
    cudaEvent_t ready = h->lev[0], landed[2] = {h->lev[1], h->lev[2]}, used[2] = {h->lev[3], h->lev[4]};
    LCK(cudaEventRecord(ready, st), "event");
    LCK(cudaStreamWaitEvent(cs, ready, 0), "event");
    const float *osrc[3] = {ox, oy, oz}, *psrc[3] = {px, py, pz};
    for (int64_t c = 0; c < nchunks; c++) {  // pass 1
        const int b = (int)(c & 1);
        const size_t o = (size_t)c * kLoadChunk, m = (size_t)std::min<int64_t>(kLoadChunk, n - (int64_t)o);
        if (c >= 2) LCK(cudaStreamWaitEvent(cs, used[b], 0), "event");
        LCK(cudaMemcpyAsync(stage_cell[b], cell + o, m * sizeof(int), cudaMemcpyHostToDevice, cs), "H2D cells");
        for (int a = 0; a < 3; a++)
            LCK(cudaMemcpyAsync(off[a] + o, osrc[a] + o, m * sizeof(float), cudaMemcpyHostToDevice, cs), "H2D offsets");
        LCK(cudaEventRecord(landed[b], cs), "event");
        LCK(cudaStreamWaitEvent(st, landed[b], 0), "event");
        LCK(place_particles_cells(g, (int64_t)m, stage_cell[b], off[0] + o, off[1] + o, off[2] + o, icell + o, st),
            "place");
        LCK(tile_histogram(g, (int64_t)m, icell + o, tc, st), "tile histogram");
        LCK(cudaEventRecord(used[b], st), "event");
    }
    std::vector<int> counts(g.ntiles);
    LCK(cudaMemcpyAsync(counts.data(), tc, g.ntiles * sizeof(int), cudaMemcpyDeviceToHost, st), "counts");
    LCK(cudaStreamSynchronize(st), "sync");
    rc = alloc_species(h, species, counts);
    if (rc) { release(); return rc; }
    SpeciesView v = h->sp[species].v;
    LCK(cudaMemsetAsync(tc, 0, g.ntiles * sizeof(int), st), "memset");
    LCK(cudaEventRecord(ready, st), "event");
    LCK(cudaStreamWaitEvent(cs, ready, 0), "event");
    for (int64_t c = 0; c < nchunks; c++) {  // pass 2
        const int b = (int)(c & 1);
        const size_t o = (size_t)c * kLoadChunk, m = (size_t)std::min<int64_t>(kLoadChunk, n - (int64_t)o);
        if (c >= 2) LCK(cudaStreamWaitEvent(cs, used[b], 0), "event");
        for (int a = 0; a < 3; a++)
            LCK(cudaMemcpyAsync(stage_mom[b][a], psrc[a] + o, m * sizeof(float), cudaMemcpyHostToDevice, cs),
                "H2D momenta");
        LCK(cudaEventRecord(landed[b], cs), "event");
        LCK(cudaStreamWaitEvent(st, landed[b], 0), "event");
        LCK(scatter_to_bins_f(g, h->mixed, (int64_t)m, icell + o, off[0] + o, off[1] + o, off[2] + o,
                              stage_mom[b][0], stage_mom[b][1], stage_mom[b][2], v, tc, st), "scatter");
        LCK(cudaEventRecord(used[b], st), "event");
    }
    LCK(cudaMemcpyAsync(v.tile_count, tc, g.ntiles * sizeof(int), cudaMemcpyDeviceToDevice, st), "tile counts");
    release();
    LCK(cudaStreamSynchronize(st), "sync");
#undef LCK
    int64_t tot = 0;
    for (int c : counts) tot += c;
    if (inserted) *inserted = tot;
    h->kin_valid = 0;
    return PIC_OK;
}

int pic_get_particles_cells(pic_handle *h, int species, int64_t cap, int32_t *cell, float *ox, float *oy, float *oz,
                            float *px, float *py, float *pz, int64_t *n) {
    if (!h || species < 0 || species >= h->cfg.nspecies) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    if (!h->sp[species].loaded) { if (n) *n = 0; return PIC_OK; }
    SpeciesView &v = h->sp[species].v;
    std::vector<int> counts(g.ntiles);
    CK(cudaMemcpyAsync(counts.data(), v.tile_count, g.ntiles * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "counts");
    CK(cudaStreamSynchronize(h->stream), "sync");
    std::vector<int64_t> dstart(g.ntiles + 1);
    int64_t acc = 0;
    for (int t = 0; t < g.ntiles; t++) { dstart[t] = acc; acc += counts[t]; }
    dstart[g.ntiles] = acc;
    if (n) *n = acc;
    if (acc > cap) return set_err(h, PIC_ERR_ARG, "capacity too small");
    if (acc == 0) return PIC_OK;
    size_t N = (size_t)acc;
    ScratchGuard guard(h);
    float *buf = nullptr;
    int *dcell = nullptr;
    int64_t *dd = nullptr;
    CK(guard.alloc(&buf, N * 6), "alloc");
    CK(guard.alloc(&dcell, N), "alloc");
    CK(guard.alloc(&dd, (size_t)g.ntiles + 1), "alloc");
    CK(cudaMemcpyAsync(dd, dstart.data(), (g.ntiles + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream), "H2D");
    CK(gather_from_bins_f(g, h->mixed, v, dd, dcell, buf, buf + N, buf + 2 * N, buf + 3 * N, buf + 4 * N, buf + 5 * N,
                          h->stream), "gather");
    float *dst[6] = {ox, oy, oz, px, py, pz};
    for (int a = 0; a < 6; a++)
        if (dst[a]) CK(cudaMemcpyAsync(dst[a], buf + a * N, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "D2H");
    if (cell) CK(cudaMemcpyAsync(cell, dcell, N * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_init_species_device(pic_handle *h, int species, int ppc, double drift_x, double drift_y, double drift_z,
                            double vth, uint64_t seed) {
    if (!h || species < 0 || species >= h->cfg.nspecies || ppc < 0) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    std::vector<int> counts(g.ntiles);
    for (int ti = 0; ti < g.ntx; ti++)
        for (int tl = 0; tl < g.nty; tl++)
            for (int tk = 0; tk < g.ntz; tk++) {
                int ex = std::min(g.tx, g.nx - ti * g.tx), ey = std::min(g.ty, g.ny - tl * g.ty),
                    ez = std::min(g.tz, g.nz - tk * g.tz);
                counts[(ti * g.nty + tl) * g.ntz + tk] = ex * ey * ez * ppc;
            }
    rc = alloc_species(h, species, counts);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->sp[species].v.tile_count, counts.data(), g.ntiles * sizeof(int), cudaMemcpyHostToDevice,
                       h->stream), "tile counts");
    CK(init_species_bins(g, h->mixed, h->sp[species].v, species, ppc, drift_x, drift_y, drift_z, vth, seed,
                         h->stream), "init species");
    CK(cudaStreamSynchronize(h->stream), "sync");
    h->kin_valid = 0;
    return ensure_outbox(h);
}

int pic_profile_counts(int nx, int ny, int nz, const pic_profile *prof, int32_t *counts, int64_t *total) {
    if (nx < 1 || ny < 1 || nz < 1 || !prof || !counts) return PIC_ERR_ARG;
    if (!(prof->ppc_mean >= 0) || !(prof->bump_peak > 0) || (prof->bump_peak != 1.0 && !(prof->bump_sigma > 0)))
        return PIC_ERR_ARG;
    const int64_t nc = (int64_t)nx * ny * nz;
    double c0[3] = {prof->bump_centre[0], prof->bump_centre[1], prof->bump_centre[2]};
    if (c0[0] < 0 || c0[1] < 0 || c0[2] < 0) { c0[0] = 0.5 * nx; c0[1] = 0.5 * ny; c0[2] = 0.5 * nz; }
    const double two_pi = 6.283185307179586;
    auto f_of = [&](int i, int l, int k) {
        double a = 1.0 + prof->cos_amp * cos(two_pi * (i + 0.5) / nx);
        double dxc = i + 0.5 - c0[0], dyc = l + 0.5 - c0[1], dzc = k + 0.5 - c0[2];
        double b = prof->bump_peak == 1.0 ? 1.0
                   : 1.0 + (prof->bump_peak - 1.0) *
                               exp(-(dxc * dxc + dyc * dyc + dzc * dzc) / (2.0 * prof->bump_sigma * prof->bump_sigma));
        return a * b;
    };
    double sum = 0.0;
    for (int i = 0; i < nx; i++)
        for (int l = 0; l < ny; l++)
            for (int k = 0; k < nz; k++) sum += f_of(i, l, k);
    if (!(sum > 0)) return PIC_ERR_ARG;
    const double scale = prof->ppc_mean * (double)nc / sum;
    int64_t acc = 0;
    for (int i = 0; i < nx; i++)
        for (int l = 0; l < ny; l++)
            for (int k = 0; k < nz; k++) {
                const int64_t c = ((int64_t)i * ny + l) * nz + k;
                const double v = scale * f_of(i, l, k);
                const double fl = floor(v);
                const int n = (int)fl + (rng_uniform(prof->count_seed, -1, c, 0, 31) < v - fl ? 1 : 0);
                counts[c] = n;
                acc += n;
            }
    if (total) *total = acc;
    return PIC_OK;
}

int pic_init_species_profile(pic_handle *h, int species, const pic_profile *prof, double drift_x, double drift_y,
                             double drift_z, double vth, uint64_t seed) {
    if (!h || species < 0 || species >= h->cfg.nspecies || !prof) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    const int nc = g.ncells();
    std::vector<int> cnt(nc), first(nc), tcount(g.ntiles, 0);
    int64_t total = 0;
    if (pic_profile_counts(g.nx, g.ny, g.nz, prof, cnt.data(), &total)) return set_err(h, PIC_ERR_ARG, "bad profile");
    for (int i = 0; i < g.nx; i++)
        for (int l = 0; l < g.ny; l++)
            for (int k = 0; k < g.nz; k++) tcount[g.tile_of_cell(i, l, k)] += cnt[g.dense_of(i, l, k)];
    rc = alloc_species(h, species, tcount);
    if (rc) return rc;
    // slots of a tile: its cells in (i, l, k) order, z fastest (the order the bin sort restores)
    const std::vector<int> &start = h->sp[species].h_start;
    std::vector<int> fill(g.ntiles, 0);
    for (int i = 0; i < g.nx; i++)
        for (int l = 0; l < g.ny; l++)
            for (int k = 0; k < g.nz; k++) {
                const int t = g.tile_of_cell(i, l, k), c = g.dense_of(i, l, k);
                first[c] = start[t] + fill[t];
                fill[t] += cnt[c];
            }
    int *d = nullptr;
    CK(cudaMalloc(&d, 2 * (size_t)nc * sizeof(int)), "alloc counts");
    cudaError_t e = cudaMemcpyAsync(d, cnt.data(), (size_t)nc * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d + nc, first.data(), (size_t)nc * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->sp[species].v.tile_count, tcount.data(), g.ntiles * sizeof(int),
                            cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = init_cells(g, h->mixed, h->sp[species].v, species, d, d + nc, drift_x, drift_y, drift_z, vth, seed,
                       h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    CK(e, "init species (profile)");
    h->kin_valid = 0;
    return ensure_outbox(h);
}

int pic_init_species_host(int nx, int ny, int nz, double lx, double ly, double lz, int species_index, int ppc,
                          double drift_x, double drift_y, double drift_z, double vth, uint64_t seed, double *x,
                          double *y, double *z, double *px, double *py, double *pz) {
    if (nx < 1 || ny < 1 || nz < 1 || ppc < 0 || !x || !y || !z || !px || !py || !pz) return PIC_ERR_ARG;
    double hx = lx / ((double)nx), hy = ly / ((double)ny), hz = lz / ((double)nz);
    int64_t q = 0;
    for (int i = 0; i < nx; i++)
        for (int l = 0; l < ny; l++)
            for (int k = 0; k < nz; k++) {
                int64_t c = ((int64_t)i * ny + l) * nz + k;
                for (int s = 0; s < ppc; s++, q++) {
                    double ox = rng_offset(seed, species_index, c, s, 0);
                    double oy = rng_offset(seed, species_index, c, s, 1);
                    double oz = rng_offset(seed, species_index, c, s, 2);
                    x[q] = (double)i * hx + ox * hx;
                    y[q] = (double)l * hy + oy * hy;
                    z[q] = (double)k * hz + oz * hz;
                    if (vth != 0.0) {
                        px[q] = drift_x + vth * rng_normal(seed, species_index, c, s, 0);
                        py[q] = drift_y + vth * rng_normal(seed, species_index, c, s, 1);
                        pz[q] = drift_z + vth * rng_normal(seed, species_index, c, s, 2);
                    } else {
                        px[q] = drift_x; py[q] = drift_y; pz[q] = drift_z;
                    }
                }
            }
    return PIC_OK;
}

int pic_set_field(pic_handle *h, int field, const double *host) {
    if (!h || field < 0 || field >= PIC_FIELD_COUNT || !host) return set_err(h, PIC_ERR_ARG, "bad argument");
    if (!h->f[field]) return set_err(h, PIC_ERR_ARG, "field not stored in this precision form");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    CK(cudaMemcpyAsync(h->dense, host, g.nodes_ref() * sizeof(double), cudaMemcpyHostToDevice, h->stream), "H2D field");
    int is_float = h->mixed && field < PIC_JX;
    CK(dense_to_pitched(g, h->dense, h->f[field], is_float, h->stream), "field layout");
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_get_field(pic_handle *h, int field, double *host) {
    if (!h || field < 0 || field >= PIC_FIELD_COUNT || !host) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    if (!h->f[field]) {
        memset(host, 0, g.nodes_ref() * sizeof(double));
        return set_err(h, PIC_ERR_ARG, "field not stored in this precision form");
    }
    int is_float = h->mixed && field < PIC_JX;
    CK(pitched_to_dense(g, h->f[field], is_float, h->dense, h->stream), "field layout");
    CK(cudaMemcpyAsync(host, h->dense, g.nodes_ref() * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H field");
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_b_half(pic_handle *h) { return h ? (set_device(h) ? h->status : do_b_half(h)) : PIC_ERR_ARG; }
int pic_stage_fields(pic_handle *h) { return h ? PIC_OK : PIC_ERR_ARG; }
int pic_push_deposit(pic_handle *h) { return h ? (set_device(h) ? h->status : do_push_deposit(h)) : PIC_ERR_ARG; }
int pic_migrate(pic_handle *h) { return h ? (set_device(h) ? h->status : do_migrate(h)) : PIC_ERR_ARG; }
int pic_j_fold(pic_handle *h) { return h ? (set_device(h) ? h->status : do_j_fold(h)) : PIC_ERR_ARG; }
int pic_b_complete(pic_handle *h) { return h ? (set_device(h) ? h->status : do_b_complete(h)) : PIC_ERR_ARG; }
int pic_e_update(pic_handle *h) { return h ? (set_device(h) ? h->status : do_e_update(h)) : PIC_ERR_ARG; }
int pic_e_ghosts(pic_handle *h) { return h ? (set_device(h) ? h->status : do_e_ghosts(h)) : PIC_ERR_ARG; }

int pic_step(pic_handle *h, int nt) {
    (void)nt;
    if (!h) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    h->launches = 0;
    cudaEventRecord(h->ev[0], h->stream);
    // the FP32 form forms the B half step inside the push's staged field tile
    if (!h->mixed && (rc = do_b_half(h))) return rc;
    cudaEventRecord(h->ev[1], h->stream);
    if ((rc = do_push_deposit(h, h->mixed))) return rc;  // records ev[2], ev[3] around the kernel
    StepParams p = make_params(h);
    CK(launch_insert(p, h->stream), "insert");
    h->launches += 2;
    cudaEventRecord(h->ev[4], h->stream);
    if ((rc = do_j_fold(h))) return rc;
    if (h->mixed) {
        // H in memory is still the full-step field: both half steps in one pass
        yee_b_both_mixed(h->g, (float *const *)&h->f[PIC_EX], (float *const *)&h->f[PIC_HX], h->stream);
        CK(cudaGetLastError(), "b_complete");
        h->launches += 1;
    } else if ((rc = do_b_complete(h))) {
        return rc;
    }
    if ((rc = do_e_update(h))) return rc;
    if ((rc = do_e_ghosts(h))) return rc;
    cudaEventRecord(h->ev[5], h->stream);
    rc = check_status(h);
    h->counters[3] = h->launches;
    if (!rc) {
        cudaEventElapsedTime(&h->timings[0], h->ev[0], h->ev[1]);
        cudaEventElapsedTime(&h->timings[1], h->ev[2], h->ev[3]);
        cudaEventElapsedTime(&h->timings[2], h->ev[3], h->ev[4]);
        cudaEventElapsedTime(&h->timings[3], h->ev[4], h->ev[5]);
        cudaEventElapsedTime(&h->timings[4], h->ev[0], h->ev[5]);
        h->timed = 1;
    }
    return rc;
}

int pic_run(pic_handle *h, int nsteps, double *energies) {
    if (!h || nsteps < 0) return PIC_ERR_ARG;
    for (int n = 0; n < nsteps; n++) {
        int rc = pic_step(h, n + 1);
        if (rc) return rc;
        if (energies) {
            rc = pic_energy(h, energies + 4 * n);
            if (rc) return rc;
        }
    }
    return PIC_OK;
}

int pic_get_cell_counts(pic_handle *h, int *counts) {
    if (!h || !counts) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    rc = need_particles(h);
    if (rc) return rc;
    const Grid &g = h->g;
    CK(cudaMemsetAsync(h->dcounts, 0, (size_t)g.ncells() * sizeof(int), h->stream), "memset");
    StepParams p = make_params(h);
    CK(cell_histogram(p, h->dcounts, h->stream), "histogram");
    std::vector<int> c(g.ncells());
    CK(cudaMemcpyAsync(c.data(), h->dcounts, c.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    memset(counts, 0, g.nodes_ref() * sizeof(int));
    for (int i = 0; i < g.nx; i++)
        for (int l = 0; l < g.ny; l++)
            for (int k = 0; k < g.nz; k++) counts[((size_t)i * g.NY + l) * g.NZ + k] = c[g.dense_of(i, l, k)];
    return PIC_OK;
}

int pic_get_cell_particles(pic_handle *h, int species, int cell, int64_t cap, double *x, double *y, double *z,
                           double *px, double *py, double *pz, int64_t *slot, int64_t *n, int64_t *bin_offset) {
    if (!h || species < 0 || species >= h->cfg.nspecies || cap < 0) return set_err(h, PIC_ERR_ARG, "bad argument");
    const Grid &g = h->g;
    // reference cell number ((i*(Ny+2) + l)*(Nz+2) + k) of an interior cell
    const int k = cell % g.NZ, l = (cell / g.NZ) % g.NY, i = cell / (g.NZ * g.NY);
    if (cell < 0 || i >= g.nx || l >= g.ny || k >= g.nz) return set_err(h, PIC_ERR_ARG, "not an interior cell");
    int rc = set_device(h);
    if (rc) return rc;
    if (n) *n = 0;
    if (bin_offset) *bin_offset = 0;
    if (!h->sp[species].loaded) return PIC_OK;
    const SpeciesView &v = h->sp[species].v;
    const int t = g.tile_of_cell(i, l, k);
    int count = 0;
    CK(cudaMemcpyAsync(&count, v.tile_count + t, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "tile count");
    CK(cudaStreamSynchronize(h->stream), "sync");
    if (bin_offset) *bin_offset = h->sp[species].h_start[t];
    const size_t N = (size_t)(count > 0 ? count : 1);
    ScratchGuard guard(h);
    double *buf = nullptr;
    int64_t *dslot = nullptr;
    unsigned *dcnt = nullptr;
    CK(guard.alloc(&buf, 6 * N), "alloc");
    CK(guard.alloc(&dslot, N), "alloc");
    CK(guard.alloc(&dcnt, 1), "alloc");
    CK(cudaMemsetAsync(dcnt, 0, sizeof(unsigned), h->stream), "memset");
    CK(cell_particles(g, h->mixed, v, t, g.cell_of(i, l, k), (int64_t)N, buf, buf + N, buf + 2 * N, buf + 3 * N,
                      buf + 4 * N, buf + 5 * N, dslot, dcnt, h->stream), "cell particles");
    unsigned m = 0;
    CK(cudaMemcpyAsync(&m, dcnt, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    std::vector<double> hb(6 * (size_t)m);
    std::vector<int64_t> hs(m);
    for (int a = 0; a < 6; a++)
        if (m) CK(cudaMemcpyAsync(hb.data() + a * (size_t)m, buf + a * N, m * sizeof(double), cudaMemcpyDeviceToHost,
                                  h->stream), "D2H");
    if (m) CK(cudaMemcpyAsync(hs.data(), dslot, m * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    if (n) *n = m;
    if ((int64_t)m > cap) return set_err(h, PIC_ERR_ARG, "capacity too small");
    // slot order
    std::vector<unsigned> ord(m);
    for (unsigned e = 0; e < m; e++) ord[e] = e;
    std::sort(ord.begin(), ord.end(), [&](unsigned a, unsigned b) { return hs[a] < hs[b]; });
    double *dst[6] = {x, y, z, px, py, pz};
    for (unsigned e = 0; e < m; e++) {
        for (int a = 0; a < 6; a++)
            if (dst[a]) dst[a][e] = hb[a * (size_t)m + ord[e]];
        if (slot) slot[e] = hs[ord[e]];
    }
    return PIC_OK;
}

int64_t pic_num_particles(pic_handle *h, int species) {
    if (!h || species >= h->cfg.nspecies) return PIC_ERR_ARG;
    if (set_device(h)) return h->status;
    int64_t tot = 0;
    std::vector<int> c(h->g.ntiles);
    for (int s = 0; s < h->cfg.nspecies; s++) {
        if (species >= 0 && s != species) continue;
        if (!h->sp[s].loaded) continue;
        if (cudaMemcpyAsync(c.data(), h->sp[s].v.tile_count, c.size() * sizeof(int), cudaMemcpyDeviceToHost,
                            h->stream) != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
            return set_err(h, PIC_ERR_STATE, "count copy failed");
        for (int v : c) tot += v;
    }
    return tot;
}

int pic_get_particles(pic_handle *h, int species, int64_t cap, double *x, double *y, double *z, double *px,
                      double *py, double *pz, int *cell, int64_t *n) {
    if (!h || species < 0 || species >= h->cfg.nspecies) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    const Grid &g = h->g;
    if (!h->sp[species].loaded) { if (n) *n = 0; return PIC_OK; }
    SpeciesView &v = h->sp[species].v;
    std::vector<int> counts(g.ntiles);
    CK(cudaMemcpyAsync(counts.data(), v.tile_count, g.ntiles * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "counts");
    CK(cudaStreamSynchronize(h->stream), "sync");
    std::vector<int64_t> dstart(g.ntiles + 1);
    int64_t acc = 0;
    for (int t = 0; t < g.ntiles; t++) { dstart[t] = acc; acc += counts[t]; }
    dstart[g.ntiles] = acc;
    if (n) *n = acc;
    if (acc > cap) return set_err(h, PIC_ERR_ARG, "capacity too small");
    if (acc == 0) return PIC_OK;
    double *buf = nullptr;
    int *dcell = nullptr;
    int64_t *dd = nullptr;
    size_t N = (size_t)acc;
    CK(cudaMalloc(&buf, N * 6 * sizeof(double)), "alloc");
    CK(cudaMalloc(&dcell, N * sizeof(int)), "alloc");
    CK(cudaMalloc(&dd, (g.ntiles + 1) * sizeof(int64_t)), "alloc");
    CK(cudaMemcpyAsync(dd, dstart.data(), (g.ntiles + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream), "H2D");
    CK(gather_from_bins(g, h->mixed, v, dd, buf, buf + N, buf + 2 * N, buf + 3 * N, buf + 4 * N, buf + 5 * N, dcell,
                        h->stream), "gather");
    double *dst[6] = {x, y, z, px, py, pz};
    for (int a = 0; a < 6; a++)
        if (dst[a]) CK(cudaMemcpyAsync(dst[a], buf + a * N, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H");
    std::vector<int> hc(N);
    CK(cudaMemcpyAsync(hc.data(), dcell, N * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    cudaFree(buf);
    cudaFree(dcell);
    cudaFree(dd);
    if (cell) {
        for (size_t j = 0; j < N; j++) {
            int c = hc[j];
            if (c < 0) { cell[j] = -1; continue; }
            int i, l, k;
            g.cell_ijk(c, i, l, k);
            cell[j] = (int)(((size_t)i * g.NY + l) * g.NZ + k);
        }
    }
    return PIC_OK;
}

int pic_energy(pic_handle *h, double *out4) {
    if (!h || !out4) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    rc = need_particles(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->dred, 0, 8 * sizeof(double), h->stream), "memset");
    const void *E[3] = {h->f[PIC_EX], h->f[PIC_EY], h->f[PIC_EZ]};
    const void *H[3] = {h->f[PIC_HX], h->f[PIC_HY], h->f[PIC_HZ]};
    CK(field_energy(h->g, h->mixed, E, H, h->dred, h->stream), "field energy");
    if (!h->kin_valid) {
        StepParams p = make_params(h);
        CK(kinetic_energy(p, h->dred + 3, h->stream), "kinetic");
    } else {
        CK(cudaMemcpyAsync(h->dred + 3, &h->st->kinetic, sizeof(double), cudaMemcpyDeviceToDevice, h->stream), "kin");
    }
    CK(cudaMemcpyAsync(h->hred, h->dred, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    out4[0] = 0.5 * h->hred[0];
    out4[1] = 0.5 * h->hred[1];
    out4[2] = h->hred[3];
    out4[3] = out4[0] + out4[1] + out4[2];
    return PIC_OK;
}

int pic_energy_reference(pic_handle *h, double *out) {
    if (!h || !out) return set_err(h, PIC_ERR_ARG, "bad argument");
    int rc = set_device(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->dred, 0, 8 * sizeof(double), h->stream), "memset");
    const void *E[3] = {h->f[PIC_EX], h->f[PIC_EY], h->f[PIC_EZ]};
    const void *H[3] = {h->f[PIC_HX], h->f[PIC_HY], h->f[PIC_HZ]};
    CK(field_energy(h->g, h->mixed, E, H, h->dred, h->stream), "field energy");
    CK(cudaMemcpyAsync(h->hred, h->dred, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H");
    CK(cudaStreamSynchronize(h->stream), "sync");
    *out = h->hred[2];
    return PIC_OK;
}

int pic_sync(pic_handle *h) {
    if (!h) return PIC_ERR_ARG;
    int rc = set_device(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream), "sync");
    return PIC_OK;
}

int pic_last_status(pic_handle *h) { return h ? h->status : PIC_ERR_ARG; }
const char *pic_last_error_string(pic_handle *h) { return h ? h->err : "null handle"; }

const char *pic_error_string(int status) {
    switch (status) {
        case PIC_OK: return "success";
        case PIC_ERR_ARG: return "bad argument or configuration";
        case PIC_ERR_NOMEM: return "allocation failed";
        case PIC_ERR_STENCIL: return "a particle moved more than half a cell in one step";
        case PIC_ERR_OUTBOX: return "migration outbox overflowed";
        case PIC_ERR_HOLES: return "too many departures from one tile";
        case PIC_ERR_NAN: return "non-finite momentum";
        case PIC_ERR_STATE: return "call not valid in this state";
        case PIC_ERR_NOT_BUILT: return "feature not built";
        case PIC_ERR_NO_DEVICE: return "no CUDA device";
        case PIC_ERR_TOO_MANY: return "too many particles";
        default: return status > 0 ? cudaGetErrorString((cudaError_t)status) : "unknown error";
    }
}

int pic_step_counters(pic_handle *h, int64_t *out4) {
    if (!h || !out4) return PIC_ERR_ARG;
    for (int i = 0; i < 4; i++) out4[i] = h->counters[i];
    return PIC_OK;
}

int pic_step_timings(pic_handle *h, float *out5) {
    if (!h || !out5) return PIC_ERR_ARG;
    for (int i = 0; i < 5; i++) out5[i] = h->timings[i];
    return h->timed ? PIC_OK : PIC_ERR_STATE;
}

int pic_layout_info(pic_handle *h, int64_t *out4) {
    if (!h || !out4) return PIC_ERR_ARG;
    int64_t slots = 0;
    for (int s = 0; s < h->cfg.nspecies; s++) slots += h->sp[s].cap_total;
    out4[0] = h->g.ntiles;
    out4[1] = slots;
    out4[2] = (int64_t)elem_particle(h->mixed);
    out4[3] = (int64_t)h->g.nodes_ref();
    return PIC_OK;
}

void *pic_stream(pic_handle *h) { return h ? (void *)h->stream : nullptr; }

}  // extern "C"
