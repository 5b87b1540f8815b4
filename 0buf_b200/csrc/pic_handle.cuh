// The handle behind the C ABI (pic_handle) and the host helpers shared by the
// translation units that implement the ABI (pic_capi.cu: the step and I/O;
// pic_adjoint.cu: the differentiable run).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>
#include "pic0buf.h"
#include "pic_internal.cuh"

namespace pic {
struct AdjState;  // checkpoints and adjoint buffers of the differentiable run (pic_adjoint.cu)
}

struct pic_handle {
    pic_config cfg;
    pic::Grid g;
    int mixed;
    int device;
    cudaStream_t stream;
    void *f[PIC_FIELD_COUNT];  // plain: 12 double arrays; mixed: E,H float, J double, Q null
    double *dense;             // one reference-layout FP64 array (I/O staging)
    struct Sp {
        pic::SpeciesView v;
        int64_t cap_total;
        int loaded;
        std::vector<int> h_start;
        // FP32 form: the bound of its contributions is known from a push
        // (cleared whenever the bins are rebuilt)
        int lb_known;
    } sp[pic::kMaxSpecies];
    void *outbox;
    unsigned out_cap;
    int outbox_pinned;  // set while a multi-species rebin still reads leftovers from the outbox
    size_t out_elem;
    pic::DevStatus *st;
    pic::DevStatus *st_host;
    double *dred;   // device reduction scratch
    double *hred;   // pinned
    int *dcounts;   // ncells ints
    int status;
    char err[256];
    int64_t counters[4];
    float timings[5];
    cudaEvent_t ev[6];
    int64_t launches;  // kernels launched by the current/last step
    int timed;
    int kin_valid;  // st->kinetic holds the kinetic energy of the current momenta
    pic::AdjState *adj;
    // charge-conservation diagnostic (pic_diag.cu), allocated on first use:
    // rho, the Gauss residual G = div E - rho and its stored baseline
    double *rho, *gauss, *gauss0;
    int gauss_has_base;
    int branch_record;  // the next pic_forward records its discrete choices (pic_branch_record)
    // second stream and events of the chunked host->device load
    // (pic_load_particles_cells): copies run there while the handle's stream
    // places and scatters the previous chunk
    cudaStream_t copy_stream;
    cudaEvent_t lev[5];
    // FP32 form: TMA descriptors of the E/H arrays (encoded once: the field
    // arrays never move) and the per-species contribution bounds of the last
    // two pushes (2 x PIC_MAX_SPECIES floats; lb_par selects the previous half)
    pic::MixedMaps maps;
    float *lb_buf;
    int lb_par;
    // plain form: the largest per-tile sum of bin capacities over the species
    // (valid while tile_cap_valid; cleared whenever a species' bins change)
    int tile_cap_valid;
    int64_t tile_cap_max;
    // staging of pic_load_particles_cells (cells, offsets, chunks), kept from
    // one species' load to the next and released by pic_destroy
    // (release_load_scratch)
    void *load_buf;
    size_t load_bytes;
};

namespace pic_host {

int set_err(pic_handle *h, int code, const char *msg);
int cuda_err(pic_handle *h, cudaError_t e, const char *where);
int set_device(pic_handle *h);
int need_particles(pic_handle *h);
// device memory of the particle bins and of load/rebin staging (cudaMalloc:
// a stream-ordered pool was measured at 1-4 s to grow by the ~19 GB of one
// c2 species' bins, against 0.16 s for the whole load with cudaMalloc)
cudaError_t dev_alloc(pic_handle *h, void **p, size_t bytes);
void dev_free(pic_handle *h, void *p);
template <class T>
cudaError_t dev_alloc_n(pic_handle *h, T **p, size_t n) {
    return dev_alloc(h, (void **)p, n * sizeof(T));
}
// device buffers freed when the guard leaves scope, so that an error return
// (CK) between allocation and release leaks nothing
struct ScratchGuard {
    pic_handle *h;
    std::vector<void *> bufs;
    explicit ScratchGuard(pic_handle *hh) : h(hh) {}
    template <class T>
    cudaError_t alloc(T **p, size_t n) {
        cudaError_t e = dev_alloc(h, (void **)p, n * sizeof(T));
        if (e == cudaSuccess) bufs.push_back((void *)*p);
        return e;
    }
    ~ScratchGuard() {
        for (void *p : bufs) dev_free(h, p);
    }
};
// frees the load staging (pic_load_particles_cells)
void release_load_scratch(pic_handle *h);
// kernel parameters of the current state (species views, fields, outbox, status)
pic::StepParams make_params(pic_handle *h);
// flat device list of one species (packed cell, FP64 global positions and
// momenta; cell < 0 = rejected) -> bins of species s
int build_bins(pic_handle *h, int s, int64_t n, int *cell, const double *x, const double *y, const double *z,
               const double *px, const double *py, const double *pz, int64_t *inserted);
// flat device list in the native layout (packed cell, FP32 offsets and momenta) -> bins of species s
int build_bins_f(pic_handle *h, int s, int64_t n, int *cell, const float *ox, const float *oy, const float *oz,
                 const float *px, const float *py, const float *pz);
// live particles per tile of species s (host copy)
int tile_counts(pic_handle *h, int s, std::vector<int> &counts);
// the differentiable run's buffers (pic_adjoint.cu)
void adj_free(pic_handle *h);

}  // namespace pic_host

#define CK(expr, where)                                                    \
    do {                                                                   \
        cudaError_t e_ = (expr);                                           \
        if (e_ != cudaSuccess) return pic_host::cuda_err(h, e_, where);    \
    } while (0)
