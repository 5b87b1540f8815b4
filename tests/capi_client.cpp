// A C++ client of the C ABI in include/pic0buf.h: the reference's step driver
// (class Plasma, gpu_plasma.h) with its kernel launches replaced by the
// library's calls, as INTEGRATION.md shows it.  The tests build it with g++
// and link it against 0buf_b200/lib/libpic0buf.so.
//
//   capi_client layout          sizes and field offsets of the ABI structs,
//                               one "name size offsets..." line per struct
//   capi_client run IN OUT      reads a case (grid, species, initial E/H)
//                               from IN, runs Plasma::Step(nt) for
//                               nt = 1..steps and writes, per step, the
//                               per-cell counts, the twelve fields and the
//                               reference's electric energy to OUT
//
// File formats (little endian, no padding):
//   IN : int32 nx ny nz nspecies steps; float64 lx ly lz tau;
//        per species: float64 q_m m; int64 n; float64 x[n] y[n] z[n] px[n] py[n] pz[n];
//        float64 Ex Ey Ez Hx Hy Hz, each (nx+2)(ny+2)(nz+2) in the reference layout
//   OUT: per step: int32 counts[(nx+2)(ny+2)(nz+2)]; float64 twelve fields; float64 energy
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pic0buf.h"

class Plasma {
    pic_handle *h = nullptr;
    int nodes = 0;
    FILE *trace = nullptr;

   public:
    int status = 0;
    // gpu_plasma.h:1574-1589, with the species table in place of the reference's
    // ni / n_per_cell / ion_q_m arguments
    Plasma(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz, double tau, const std::vector<pic_species> &sp) {
        pic_config c;
        pic_config_init(&c);
        c.nx = Nx; c.ny = Ny; c.nz = Nz;
        c.lx = Lx; c.ly = Ly; c.lz = Lz;
        c.tau = tau;
        c.precision = PIC_FP64_PLAIN;
        c.nspecies = (int)sp.size();
        for (size_t s = 0; s < sp.size(); s++) c.species[s] = sp[s];
        check(pic_create(&c, &h));
        nodes = (Nx + 2) * (Ny + 2) * (Nz + 2);
    }
    ~Plasma() { pic_destroy(h); }
    // addParticleListToCells, init.cu:558-592: one call per sort
    void addParticleListToCells(int sort, const std::vector<double> &x, const std::vector<double> &y,
                                const std::vector<double> &z, const std::vector<double> &px,
                                const std::vector<double> &py, const std::vector<double> &pz) {
        int64_t kept = 0;
        check(pic_load_particles(h, sort, (int64_t)x.size(), x.data(), y.data(), z.data(), px.data(), py.data(),
                                 pz.data(), &kept));
        if (kept != (int64_t)x.size()) status = status ? status : PIC_ERR_STATE;
    }
    void setField(int which, const std::vector<double> &a) { check(pic_set_field(h, which, a.data())); }
    void ComputeField_FirstHalfStep(int nt) {  // gpu_plasma.h:367-397
        check(pic_b_half(h));
        checkControlPoint(50, nt, 0);
        check(pic_stage_fields(h));
    }
    int PushParticles(int nt) {  // gpu_plasma.h:554-570
        check(pic_push_deposit(h));
        check(pic_migrate(h));
        checkControlPoint(270, nt, 1);
        return 0;
    }
    void ComputeField_SecondHalfStep(int nt) {  // gpu_plasma.h:399-430
        checkControlPoint(275, nt, 0);
        check(pic_j_fold(h));
        checkControlPoint(400, nt, 0);
        check(pic_b_complete(h));
        checkControlPoint(500, nt, 0);
        check(pic_e_update(h));
        checkControlPoint(550, nt, 0);
        check(pic_e_ghosts(h));
        checkControlPoint(600, nt, 0);
    }
    void Step(int nt) {  // gpu_plasma.h:605-620
        ComputeField_FirstHalfStep(nt);
        PushParticles(nt);
        ComputeField_SecondHalfStep(nt);
        Diagnose(nt);
    }
    double getElectricEnergy() {  // gpu_plasma.h:621-657
        double e = 0.0;
        check(pic_energy_reference(h, &e));
        return e;
    }
    // the control points read device state in the reference layout; this
    // client records the state after each step instead (Diagnose)
    void checkControlPoint(int, int, int) {}
    void traceTo(FILE *f) { trace = f; }
    void Diagnose(int) {
        if (!trace || status) return;
        std::vector<int> counts(nodes);
        check(pic_get_cell_counts(h, counts.data()));
        fwrite(counts.data(), sizeof(int), counts.size(), trace);
        std::vector<double> a(nodes);
        for (int f = 0; f < PIC_FIELD_COUNT; f++) {
            check(pic_get_field(h, f, a.data()));
            fwrite(a.data(), sizeof(double), a.size(), trace);
        }
        const double e = getElectricEnergy();
        fwrite(&e, sizeof(double), 1, trace);
    }
    void check(int rc) {
        if (rc && !status) {
            status = rc;
            fprintf(stderr, "pic0buf: %s\n", h ? pic_last_error_string(h) : pic_error_string(rc));
        }
    }
};

#define OFF(T, f) (long)offsetof(T, f)

static int layout() {
    printf("pic_species %zu %ld %ld %ld\n", sizeof(pic_species), OFF(pic_species, q_m), OFF(pic_species, m),
           OFF(pic_species, sort));
    printf("pic_config %zu %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld\n", sizeof(pic_config),
           OFF(pic_config, nx), OFF(pic_config, ny), OFF(pic_config, nz), OFF(pic_config, lx), OFF(pic_config, ly),
           OFF(pic_config, lz), OFF(pic_config, tau), OFF(pic_config, precision), OFF(pic_config, ghosts),
           OFF(pic_config, nspecies), OFF(pic_config, device), OFF(pic_config, species),
           OFF(pic_config, capacity_slack), OFF(pic_config, outbox_fraction), OFF(pic_config, tile),
           OFF(pic_config, capacity_pad));
    printf("pic_loss %zu %ld %ld %ld %ld %ld\n", sizeof(pic_loss), OFF(pic_loss, field), OFF(pic_loss, window),
           OFF(pic_loss, species), OFF(pic_loss, drift), OFF(pic_loss, vth));
    printf("pic_grads %zu %ld %ld %ld %ld %ld\n", sizeof(pic_grads), OFF(pic_grads, loss), OFF(pic_grads, d_drift),
           OFF(pic_grads, d_vth), OFF(pic_grads, n), OFF(pic_grads, d_p0));
    printf("pic_profile %zu\n", sizeof(pic_profile));
    printf("pic_mumu %zu %ld %ld %ld %ld %ld\n", sizeof(pic_mumu), OFF(pic_mumu, fields), OFF(pic_mumu, count),
           OFF(pic_mumu, q_m), OFF(pic_mumu, m), OFF(pic_mumu, p));
    printf("pic_rnd %zu %ld\n", sizeof(pic_rnd), OFF(pic_rnd, store));
    printf("pic_quiet %zu %ld %ld\n", sizeof(pic_quiet), OFF(pic_quiet, meh), OFF(pic_quiet, lx));
    return 0;
}

template <class T>
static bool rd(FILE *f, T *p, size_t n) {
    return fread(p, sizeof(T), n, f) == n;
}

static int run(const char *in, const char *out) {
    FILE *f = fopen(in, "rb");
    if (!f) return 2;
    int32_t hdr[5];
    double geo[4];
    if (!rd(f, hdr, 5) || !rd(f, geo, 4)) return 2;
    const int nx = hdr[0], ny = hdr[1], nz = hdr[2], nsp = hdr[3], steps = hdr[4];
    std::vector<pic_species> sp(nsp);
    std::vector<std::vector<double>> arr(6 * nsp);
    for (int s = 0; s < nsp; s++) {
        double qm[2];
        int64_t n = 0;
        if (!rd(f, qm, 2) || !rd(f, &n, 1)) return 2;
        sp[s].q_m = qm[0];
        sp[s].m = qm[1];
        sp[s].sort = s;
        for (int a = 0; a < 6; a++) {
            arr[6 * s + a].resize((size_t)n);
            if (n && !rd(f, arr[6 * s + a].data(), (size_t)n)) return 2;
        }
    }
    const size_t nodes = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    std::vector<std::vector<double>> fields(6, std::vector<double>(nodes));
    for (int c = 0; c < 6; c++)
        if (!rd(f, fields[c].data(), nodes)) return 2;
    fclose(f);

    FILE *o = fopen(out, "wb");
    if (!o) return 2;
    int rc;
    {
        Plasma pl(nx, ny, nz, geo[0], geo[1], geo[2], geo[3], sp);
        for (int s = 0; s < nsp; s++)
            pl.addParticleListToCells(s, arr[6 * s], arr[6 * s + 1], arr[6 * s + 2], arr[6 * s + 3],
                                      arr[6 * s + 4], arr[6 * s + 5]);
        for (int c = 0; c < 6; c++) pl.setField(PIC_EX + c, fields[c]);
        pl.traceTo(o);
        for (int nt = 1; nt <= steps && !pl.status; nt++) pl.Step(nt);
        rc = pl.status;
    }
    fclose(o);
    return rc ? 1 : 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && !strcmp(argv[1], "layout")) return layout();
    if (argc >= 4 && !strcmp(argv[1], "run")) return run(argv[2], argv[3]);
    fprintf(stderr, "usage: %s layout | run IN OUT\n", argv[0]);
    return 2;
}
