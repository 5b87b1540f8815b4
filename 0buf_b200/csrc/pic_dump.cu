// The reference's Fortran-record dump ("mumu" file), read and written on the
// host, and the on-disk checkpoint/resume of a handle built on it.
//
// Format (LoadParticleData, load_data.cu:308-341; readControlPoint,
// gpu_plasma.h:1088-1125): Fortran unformatted sequential records, each an
// int32 byte count, the payload, and the same int32 byte count
// (readFortranBinaryArray, load_data.cu:35-63).
//   12 field records: Ex Ey Ez Hx Hy Hz Jx Jy Jz Qx Qy Qz, (Nx+2)(Ny+2)(Nz+2)
//      FP64 each, element n = the reference array index n (the reference reads
//      them straight into its arrays);
//   then per particle sort (ion, plasma electron, beam electron): one record
//      of three FP64 (particle count, q/m, charge weight m)
//      (readBinaryParticleArraysOneSort, load_data.cu:140-250), then six
//      records of count FP64: x, y, z (global positions), px, py, pz.
// A record holds at most 2^31 - 1 bytes (the reader's int byte count), so a
// species of more than 268,435,455 particles does not fit the format.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <stdint.h>
#include <math.h>
#include <algorithm>
#include <vector>
#include "pic0buf.h"
#include "pic_internal.cuh"
#include "pic_handle.cuh"

using namespace pic;
using namespace pic_host;

namespace {

constexpr int64_t kMaxRecord = 0x7fffffffLL;

bool write_record(FILE *f, const void *data, int64_t bytes) {
    if (bytes > kMaxRecord || bytes < 0) return false;
    const int32_t t = (int32_t)bytes;
    if (fwrite(&t, sizeof(t), 1, f) != 1) return false;
    if (bytes > 0 && fwrite(data, 1, (size_t)bytes, f) != (size_t)bytes) return false;
    return fwrite(&t, sizeof(t), 1, f) == 1;
}

bool write_zero_record(FILE *f, int64_t bytes) {
    if (bytes > kMaxRecord || bytes < 0) return false;
    const int32_t t = (int32_t)bytes;
    if (fwrite(&t, sizeof(t), 1, f) != 1) return false;
    std::vector<char> z((size_t)(bytes < (1 << 20) ? bytes : (1 << 20)), 0);
    for (int64_t done = 0; done < bytes;) {
        size_t c = (size_t)std::min<int64_t>((int64_t)z.size(), bytes - done);
        if (fwrite(z.data(), 1, c, f) != c) return false;
        done += c;
    }
    return fwrite(&t, sizeof(t), 1, f) == 1;
}

// reads one record of exactly `bytes` bytes into dst (dst null: skip it);
// 1 ok, 0 clean end of file before the record, -1 malformed
int read_record(FILE *f, void *dst, int64_t bytes) {
    int32_t t0 = 0, t1 = 0;
    size_t r = fread(&t0, sizeof(t0), 1, f);
    if (r != 1) return feof(f) ? 0 : -1;
    if ((int64_t)t0 != bytes) return -1;
    if (dst) {
        if (bytes > 0 && fread(dst, 1, (size_t)bytes, f) != (size_t)bytes) return -1;
    } else if (fseek(f, (long)bytes, SEEK_CUR) != 0) {
        return -1;
    }
    if (fread(&t1, sizeof(t1), 1, f) != 1 || t1 != t0) return -1;
    return 1;
}

// the next record's byte count without consuming it; -1 at end of file
int64_t peek_record(FILE *f) {
    int32_t t = 0;
    long pos = ftell(f);
    if (fread(&t, sizeof(t), 1, f) != 1) return -1;
    fseek(f, pos, SEEK_SET);
    return t;
}

int64_t field_bytes_of(int nx, int ny, int nz) { return (int64_t)(nx + 2) * (ny + 2) * (nz + 2) * 8; }

}  // namespace

extern "C" {

int pic_mumu_name(int num, int nt, char *buf, int cap) {
    if (!buf || cap < 1) return PIC_ERR_ARG;
    int n = snprintf(buf, (size_t)cap, "mumu%03d%08d.dat", num, nt);  // readControlPoint, gpu_plasma.h:1103
    return (n < 0 || n >= cap) ? PIC_ERR_ARG : PIC_OK;
}

int pic_mumu_write(const char *path, const pic_mumu *d) {
    if (!path || !d || d->nx < 1 || d->ny < 1 || d->nz < 1 || d->nsort < 0 || d->nsort > PIC_MAX_SPECIES)
        return PIC_ERR_ARG;
    const int64_t fb = field_bytes_of(d->nx, d->ny, d->nz);
    if (fb > kMaxRecord) return PIC_ERR_ARG;
    for (int s = 0; s < d->nsort; s++)
        if (d->count[s] < 0 || d->count[s] * 8 > kMaxRecord) return PIC_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return PIC_ERR_ARG;
    bool ok = true;
    for (int a = 0; a < 12 && ok; a++)
        ok = d->fields[a] ? write_record(f, d->fields[a], fb) : write_zero_record(f, fb);
    for (int s = 0; s < d->nsort && ok; s++) {
        const double head[3] = {(double)d->count[s], d->q_m[s], d->m[s]};
        ok = write_record(f, head, sizeof(head));
        for (int a = 0; a < 6 && ok; a++) {
            const int64_t bytes = d->count[s] * 8;
            ok = d->p[s][a] ? write_record(f, d->p[s][a], bytes) : write_zero_record(f, bytes);
        }
    }
    if (fclose(f) != 0) ok = false;
    return ok ? PIC_OK : PIC_ERR_ARG;
}

int pic_mumu_read_counts(const char *path, pic_mumu *d) {
    if (!path || !d || d->nx < 1 || d->ny < 1 || d->nz < 1) return PIC_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return PIC_ERR_ARG;
    const int64_t fb = field_bytes_of(d->nx, d->ny, d->nz);
    int rc = PIC_OK;
    for (int a = 0; a < 12 && rc == PIC_OK; a++)
        if (read_record(f, nullptr, fb) != 1) rc = PIC_ERR_ARG;
    int ns = 0;
    while (rc == PIC_OK && peek_record(f) >= 0) {
        if (ns == PIC_MAX_SPECIES) { rc = PIC_ERR_ARG; break; }
        double head[3];
        if (read_record(f, head, sizeof(head)) != 1 || !(head[0] >= 0) || head[0] * 8 > (double)kMaxRecord) {
            rc = PIC_ERR_ARG;
            break;
        }
        const int64_t n = (int64_t)head[0];
        for (int a = 0; a < 6 && rc == PIC_OK; a++)
            if (read_record(f, nullptr, n * 8) != 1) rc = PIC_ERR_ARG;
        d->count[ns] = n;
        d->q_m[ns] = head[1];
        d->m[ns] = head[2];
        ns++;
    }
    fclose(f);
    if (rc == PIC_OK) d->nsort = ns;
    return rc;
}

int pic_mumu_read(const char *path, pic_mumu *d) {
    if (!path || !d) return PIC_ERR_ARG;
    pic_mumu c = *d;
    int rc = pic_mumu_read_counts(path, &c);
    if (rc) return rc;
    if (c.nsort != d->nsort) return PIC_ERR_ARG;
    for (int s = 0; s < d->nsort; s++)
        if (c.count[s] != d->count[s]) return PIC_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return PIC_ERR_ARG;
    const int64_t fb = field_bytes_of(d->nx, d->ny, d->nz);
    for (int a = 0; a < 12 && rc == PIC_OK; a++)
        if (read_record(f, d->fields[a], fb) != 1) rc = PIC_ERR_ARG;
    for (int s = 0; s < d->nsort && rc == PIC_OK; s++) {
        double head[3];
        if (read_record(f, head, sizeof(head)) != 1) rc = PIC_ERR_ARG;
        d->q_m[s] = head[1];
        d->m[s] = head[2];
        for (int a = 0; a < 6 && rc == PIC_OK; a++)
            if (read_record(f, d->p[s][a], d->count[s] * 8) != 1) rc = PIC_ERR_ARG;
    }
    fclose(f);
    return rc;
}

int pic_dump_write(pic_handle *h, const char *path) {
    if (!h || !path) return PIC_ERR_ARG;
    const Grid &g = h->g;
    const size_t nodes = g.nodes_ref();
    pic_mumu d;
    memset(&d, 0, sizeof(d));
    d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
    d.nsort = h->cfg.nspecies;
    std::vector<double> fbuf(nodes * 12, 0.0);
    const int ids[12] = {PIC_EX, PIC_EY, PIC_EZ, PIC_HX, PIC_HY, PIC_HZ, PIC_JX, PIC_JY, PIC_JZ, PIC_QX, PIC_QY, PIC_QZ};
    for (int a = 0; a < 12; a++) {
        d.fields[a] = fbuf.data() + (size_t)a * nodes;
        if (!h->f[ids[a]]) continue;  // Q of the mixed form is not stored: zeros
        int rc = pic_get_field(h, ids[a], d.fields[a]);
        if (rc) return rc;
    }
    std::vector<std::vector<double>> pb(d.nsort);
    for (int s = 0; s < d.nsort; s++) {
        int64_t n = pic_num_particles(h, s);
        if (n < 0) return (int)n;
        if (n * 8 > kMaxRecord) return set_err(h, PIC_ERR_ARG, "pic_dump_write: a species exceeds the dump format's record size");
        pb[s].assign((size_t)(n > 0 ? n : 1) * 6, 0.0);
        std::vector<int> cell((size_t)(n > 0 ? n : 1));
        double *q = pb[s].data();
        int64_t got = 0;
        if (n > 0) {
            int rc = pic_get_particles(h, s, n, q, q + n, q + 2 * n, q + 3 * n, q + 4 * n, q + 5 * n, cell.data(), &got);
            if (rc) return rc;
        }
        d.count[s] = got;
        d.q_m[s] = h->cfg.species[s].q_m;
        d.m[s] = h->cfg.species[s].m;
        for (int a = 0; a < 6; a++) d.p[s][a] = q + (size_t)a * n;
    }
    int rc = pic_mumu_write(path, &d);
    return rc ? set_err(h, rc, "pic_dump_write: cannot write the dump") : PIC_OK;
}

int pic_dump_read(pic_handle *h, const char *path) {
    if (!h || !path) return PIC_ERR_ARG;
    const Grid &g = h->g;
    pic_mumu d;
    memset(&d, 0, sizeof(d));
    d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
    if (pic_mumu_read_counts(path, &d)) return set_err(h, PIC_ERR_ARG, "pic_dump_read: not a dump of this grid");
    if (d.nsort != h->cfg.nspecies) return set_err(h, PIC_ERR_ARG, "pic_dump_read: species count differs");
    for (int s = 0; s < d.nsort; s++)
        if (fabs(d.q_m[s] - h->cfg.species[s].q_m) > 1e-12 * fabs(h->cfg.species[s].q_m) ||
            fabs(d.m[s] - h->cfg.species[s].m) > 1e-12 * fabs(h->cfg.species[s].m))
            return set_err(h, PIC_ERR_ARG, "pic_dump_read: a species' q/m or charge weight differs");
    const size_t nodes = g.nodes_ref();
    std::vector<double> fbuf(nodes * 12);
    for (int a = 0; a < 12; a++) d.fields[a] = fbuf.data() + (size_t)a * nodes;
    std::vector<std::vector<double>> pb(d.nsort);
    for (int s = 0; s < d.nsort; s++) {
        pb[s].resize((size_t)(d.count[s] > 0 ? d.count[s] : 1) * 6);
        for (int a = 0; a < 6; a++) d.p[s][a] = pb[s].data() + (size_t)a * d.count[s];
    }
    if (pic_mumu_read(path, &d)) return set_err(h, PIC_ERR_ARG, "pic_dump_read: malformed dump");
    const int ids[12] = {PIC_EX, PIC_EY, PIC_EZ, PIC_HX, PIC_HY, PIC_HZ, PIC_JX, PIC_JY, PIC_JZ, PIC_QX, PIC_QY, PIC_QZ};
    for (int a = 0; a < 12; a++) {
        if (!h->f[ids[a]]) continue;
        int rc = pic_set_field(h, ids[a], d.fields[a]);
        if (rc) return rc;
    }
    for (int s = 0; s < d.nsort; s++) {
        int64_t kept = 0;
        const int64_t n = d.count[s];
        int rc = pic_load_particles(h, s, n, d.p[s][0], d.p[s][1], d.p[s][2], d.p[s][3], d.p[s][4], d.p[s][5], &kept);
        if (rc) return rc;
        if (kept != n) return set_err(h, PIC_ERR_ARG, "pic_dump_read: particles outside the box");
    }
    return PIC_OK;
}

}  // extern "C"
