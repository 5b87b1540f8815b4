// The reference's quiet start (getUniformMaxwellianParticles,
// maxwell.cu:676-757, with InitUniformMaxwellianParticles, maxwell.cu:379-536,
// and getMassCharge, maxwell.cu:598-612), restated on the host.
//
// Random numbers, drawn from one stream in the reference's order:
//   uniform  a three-stream combined multiplicative generator in the form of
//            Wichmann and Hill (Applied Statistics algorithm AS 183, 1982) as
//            the reference evaluates it (g05cae, maxwell.cu:138-170): streams
//            mod 30269, 30307, 30323 with multipliers 171, 172, 170, each step
//            a*(s mod q) - 2*(s div q) with q = 177, 176, 178 (AS 183's
//            Schrage remainders are 2, 35, 63; the reference subtracts 2 on
//            all three, so its second and third streams are not AS 183's),
//            then + modulus if negative; seeds (1, 255, 25555);
//            u = frac(x/30269 + y/30307 + z/30323);
//   Gaussian R. P. Brent's table-driven method (CACM algorithm 488, 1974;
//            g05dde, maxwell.cu:77-135): a stored uniform (initially 1) picks
//            the table interval by doubling, and a rejection loop on fresh
//            uniforms gives the deviate (table: kBrent below).
// Sequence: for each ion j: z, y, x uniform in the box; for each ion in the
// beam region: the beam's vx deviate, then vy, vz (spread Tb*rimp, drift
// rimp in x), momentum p = v/sqrt(1 - v^2); for each ion j: two electrons at
// its position with transverse deviates vy, vz and a longitudinal deviate
// termx, moving against the beam current where the ion lies in the beam.
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "pic0buf.h"

namespace {

// Brent's table: d[i] ~ Phi^-1(1 - 2^-(i+1)), i = 0..40 (Phi the normal
// distribution function), as the reference states them to 15 decimals
// (g05dde, maxwell.cu:83-97).  Ten entries (i = 4, 9, 10, 17, 27, 28, 29, 31,
// 32, 40) lie one unit of the 15th decimal above the quantile rounded to 15
// decimals, so the values are kept as stated rather than computed: a deviate
// combines table entries, and the reference's deviates need the same doubles.
const double kBrent[41] = {
    0.0, 0.674489750196082, 1.150349380376008, 1.534120544352546,
    1.862731867421652, 2.153874694061456, 2.417559016236505, 2.66006746861746,
    2.885634912426757, 3.097269078198785, 3.297193345691964, 3.487104104114431,
    3.668329285121323, 3.841930685501911, 4.008772594168585, 4.169569323349106,
    4.324919040826046, 4.475328424654204, 4.621231001499247, 4.763001034267814,
    4.900964207963193, 5.035405969463927, 5.166578119728753, 5.294704084854598,
    5.419983174916868, 5.54259405780294, 5.662697617459439, 5.780439324478935,
    5.895951216739571, 6.009353565530745, 6.120756285971941, 6.230260137989044,
    6.33795775455379, 6.443934526538564, 6.548269367831731, 6.651035379893011,
    6.752300431407015, 6.852127665896068, 6.95057594791675, 7.047700256664409,
    7.14355203435219,
};

bool in_open(double a, double z, double b) {  // in_range, maxwell.cu:215-218
    return ((z > a) && (z < b)) || ((fabs(z - a) < 1e-13) && (fabs(z - b) < 1e-13));
}

}  // namespace

extern "C" {

int pic_rnd_table(double *out41) {
    if (!out41) return PIC_ERR_ARG;
    memcpy(out41, kBrent, sizeof kBrent);
    return PIC_OK;
}

void pic_rnd_init(pic_rnd *r) {
    r->ix = 1;  // cag05a, maxwell.cu:50-52
    r->iy = 255;
    r->iz = 25555;
    r->store = 1.0;  // cag05b, maxwell.cu:46-48
}

double pic_rnd_uniform(pic_rnd *r) {
    r->ix = 171 * (r->ix % 177) - 2 * (r->ix / 177);
    r->iy = 172 * (r->iy % 176) - 2 * (r->iy / 176);
    r->iz = 170 * (r->iz % 178) - 2 * (r->iz / 178);
    if (r->ix < 0) r->ix += 30269;
    if (r->iy < 0) r->iy += 30307;
    if (r->iz < 0) r->iz += 30323;
    const double s = (double)r->ix / 30269.0 + (double)r->iy / 30307.0 + (double)r->iz / 30323.0;
    return s - (double)(int)s;
}

double pic_rnd_gaussian(pic_rnd *r, double mean, double sd) {
    const double *d = kBrent;
    double u = r->store;
    int n = 1;
    while (n < 40 && !(u > 0.5)) {  // the interval [d[n-1], d[n]) of the deviate
        u += u;
        n++;
    }
    const double t = d[n - 1];
    u = pic_rnd_uniform(r);
    double w, v;
    for (;;) {
        w = (d[n] - t) * u;
        v = w * (0.5 * w + t);
        bool accept = false;
        for (;;) {
            u = pic_rnd_uniform(r);
            if (v <= u) {
                accept = true;
                break;
            }
            v = pic_rnd_uniform(r);
            if (!(u > v)) break;
        }
        if (accept) break;
        u = (v - u) / (1.0 - u);
    }
    u = (u - v) / (1.0 - v);
    if (u > 0.5) {
        r->store = u + u - 1.0;
        return mean - sd * (w + t);
    }
    r->store = u + u;
    return mean + sd * (w + t);
}

int pic_quiet_defaults(pic_quiet *q) {
    if (!q) return PIC_ERR_ARG;
    memset(q, 0, sizeof(*q));
    q->n_ions = 1600000;  // getUniformMaxwellianParticles, maxwell.cu:680-696
    q->tex0 = q->tey0 = q->tez0 = 1e-3;
    q->Tb = 0.14;
    q->rimp = 0.2;
    q->rbd = 2.0e-3;
    q->ni = 1.0;
    q->meh = 0;
    q->lp = 1000;
    q->lx = q->beam_lx = 1.1424;
    q->ly = q->beam_ly = 0.05;
    q->lz = q->beam_lz = 0.05;
    q->beamf = 1;
    return PIC_OK;
}

int pic_quiet_start(const pic_quiet *q, double *const ion[6], double *const el[6], double *const beam[6],
                    int64_t *n_beam, double *q_m3, double *m3) {
    if (!q || !ion || !el || !beam || !n_beam || q->n_ions < 0 || q->lp < 1) return PIC_ERR_ARG;
    for (int a = 0; a < 6; a++)
        if (q->n_ions > 0 && (!ion[a] || !el[a] || !beam[a])) return PIC_ERR_ARG;
    pic_rnd S;
    pic_rnd_init(&S);
    const int64_t N = q->n_ions;
    for (int64_t j = 0; j < N; j++) {
        const double z = q->lz * pic_rnd_uniform(&S);
        const double y = q->meh * q->ly + q->ly * pic_rnd_uniform(&S);
        const double x = q->lx * pic_rnd_uniform(&S);
        ion[0][j] = x; ion[1][j] = y; ion[2][j] = z;
        ion[3][j] = ion[4][j] = ion[5][j] = 0.0;
    }
    const double sh = (q->ly - q->beam_ly) / 2, y_max = q->ly - sh, y_min = sh;
    const double shz = (q->lz - q->beam_lz) / 2, z_max = q->lz - shz, z_min = shz;
    const double sb = q->Tb * q->rimp;
    int64_t nb = 0;
    for (int64_t j = 0; j < N; j++) {
        const double y = ion[1][j], z = ion[2][j];
        if (!(ion[0][j] < q->beam_lx && y < y_max && y > y_min && in_open(z_min, z, z_max))) continue;
        beam[0][nb] = ion[0][j]; beam[1][nb] = y; beam[2][nb] = z;
        const double ux = pic_rnd_gaussian(&S, 0.0, sb) + q->rimp;
        const double uy = pic_rnd_gaussian(&S, 0.0, sb);
        const double uz = pic_rnd_gaussian(&S, 0.0, sb);
        beam[3][nb] = ux; beam[4][nb] = uy; beam[5][nb] = uz;  // velocities until all are drawn
        nb++;
    }
    for (int64_t b = 0; b < nb; b++) {
        const double ux = beam[3][b], uy = beam[4][b], uz = beam[5][b];
        const double g = sqrt(1.0 - ux * ux - uy * uy - uz * uz);
        beam[3][b] = ux / g; beam[4][b] = uy / g; beam[5][b] = uz / g;
    }
    for (int64_t j = 0; j < N; j++) {
        for (int e = 0; e < 2; e++) {
            el[0][2 * j + e] = ion[0][j]; el[1][2 * j + e] = ion[1][j]; el[2][2 * j + e] = ion[2][j];
        }
        const double vy = pic_rnd_gaussian(&S, 0.0, q->tey0);
        const double vz = pic_rnd_gaussian(&S, 0.0, q->tez0);
        const double tx = pic_rnd_gaussian(&S, 0.0, q->tex0);
        // the beam's velocity at index j (the reference pairs electron pair j with beam particle j)
        const double pb = j < nb ? beam[3][j] : 0.0, qb = j < nb ? beam[4][j] : 0.0, rb = j < nb ? beam[5][j] : 0.0;
        const double vb0 = pb * pow(1.0 + pb * pb + qb * qb + rb * rb, -0.5);
        double v1, v2;
        if (q->beamf == 1 && ion[0][j] < q->beam_lx && ion[1][j] < y_max && ion[1][j] > y_min) {
            v1 = -q->rbd * vb0 + tx;
            v2 = -q->rbd * vb0 - tx;
        } else {
            v1 = tx;
            v2 = -tx;
        }
        const double k1 = pow(1.0 - v1 * v1 - vy * vy - vz * vz, -0.5);
        const double k2 = pow(1.0 - v2 * v2 - vy * vy - vz * vz, -0.5);
        el[3][2 * j] = v1 * k1;
        el[3][2 * j + 1] = v2 * k2;
        el[4][2 * j] = vy * k1;
        el[4][2 * j + 1] = -vy * k2;
        el[5][2 * j] = vz * k1;
        el[5][2 * j + 1] = -vz * k2;
    }
    *n_beam = nb;
    // getMassCharge, maxwell.cu:598-612: charge weights per lp particles of a cell
    if (q_m3) { q_m3[0] = 1.0 / 1836.0; q_m3[1] = -1.0; q_m3[2] = -1.0; }
    if (m3) {
        m3[0] = (q->ni + q->rbd) / q->lp;
        m3[1] = -q->ni / q->lp / 2.0;
        m3[2] = -q->rbd / q->lp;
    }
    return PIC_OK;
}

}  // extern "C"
