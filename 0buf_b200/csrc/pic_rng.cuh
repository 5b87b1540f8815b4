// Counter-based seeded generator of the initial particles, shared by the
// device kernel (init_species_bins) and the host function
// pic_init_species_host.  Replaces the role of the reference's quiet-start
// loader (maxwell.cu:379-757) with the synthetic inputs of the benchmark
// configurations: ppc particles per interior cell per species at uniform
// in-cell offsets, momenta drift + vth * N(0,1) per axis.
//
// The uniforms are pure integer arithmetic scaled by 2^-53, so host and device
// produce identical offsets and positions (both compiled without FMA
// contraction).  The Gaussian uses log/sqrt/cos, whose last bits differ
// between the host libm and CUDA, so parity tests always generate on the host.
#pragma once
#include <stdint.h>
#include <math.h>

#ifndef __CUDACC__
#define PIC_HD
#else
#define PIC_HD __host__ __device__
#endif

namespace pic {

PIC_HD inline uint64_t mix64(uint64_t z) {  // SplitMix64 finaliser (Steele, Lea, Flood 2014)
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return z;
}

PIC_HD inline uint64_t rng_key(uint64_t seed, int species, int64_t cell, int slot, int stream) {
    uint64_t h = mix64(seed + 0x9E3779B97F4A7C15ull);
    h = mix64(h ^ ((uint64_t)(uint32_t)species * 0xD6E8FEB86659FD93ull));
    h = mix64(h ^ ((uint64_t)cell * 0xA0761D6478BD642Full));
    h = mix64(h ^ ((uint64_t)(uint32_t)slot * 0xE7037ED1A0B428DBull));
    h = mix64(h ^ ((uint64_t)(uint32_t)stream * 0x8EBC6AF09C88C6E3ull));
    return h;
}

// uniform in [0,1): 53 random bits
PIC_HD inline double rng_uniform(uint64_t seed, int species, int64_t cell, int slot, int stream) {
    return (double)(rng_key(seed, species, cell, slot, stream) >> 11) * (1.0 / 9007199254740992.0);
}

// in-cell offset in [1e-6, 1 - 1e-6]: keeps every initial particle strictly
// inside its cell under both getPointCell and isPointInCell (cell.h:593-598, 717)
PIC_HD inline double rng_offset(uint64_t seed, int species, int64_t cell, int slot, int axis) {
    return 1e-6 + rng_uniform(seed, species, cell, slot, axis) * (1.0 - 2e-6);
}

// standard normal by Box-Muller; axis 0,1 from one pair, axis 2 from a second
PIC_HD inline double rng_normal(uint64_t seed, int species, int64_t cell, int slot, int axis) {
    int pair = axis < 2 ? 0 : 1;
    double u1 = 1.0 - rng_uniform(seed, species, cell, slot, 8 + 2 * pair);  // (0,1]
    double u2 = rng_uniform(seed, species, cell, slot, 9 + 2 * pair);
    double r = sqrt(-2.0 * log(u1));
    double a = 6.283185307179586 * u2;
    return (axis == 1) ? r * sin(a) : r * cos(a);
}

}  // namespace pic
