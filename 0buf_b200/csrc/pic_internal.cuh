// Internal definitions of the B200 PIC step: geometry, device views of the
// state, the status word and the sizes of the tile layout.
//
// Data layout in HBM
//   fields   one array per component (E, H, J, Q), (Nx+2) x (Ny+2) x Pz with
//            Pz = round_up(Nz+2, 4) so every z row starts on a 32-byte
//            boundary (TMA rows, float4/double2 access).  The caller sees the
//            reference layout (Pz = Nz+2) through pic_get_field/pic_set_field.
//   particles one SoA set per species, binned by TILE: a tile is a block of
//            tx*ty*tz interior cells; tile t owns slots
//            [tile_start[t], tile_start[t+1]) of which the first tile_count[t]
//            are live.  Each particle carries its int32 interior cell index
//            ((i*Ny + l)*Nz + k); the plain form stores global FP64 positions,
//            the mixed form FP32 in-cell offsets in [0,1).  A particle that
//            crosses a cell boundary inside its tile only rewrites its cell
//            index; only tile leavers move (outbox -> insert).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>
#include "pic0buf.h"

namespace pic {

constexpr int kMaxSpecies = PIC_MAX_SPECIES;
constexpr int kHoleMax = 1024;          // departures per tile per species handled in-kernel
constexpr int kPushThreads = 256;

// status flag bits (DevStatus::flags)
enum : unsigned {
    ST_STENCIL = 1u,     // stencil index outside the staged tile (CFL)
    ST_OUTBOX = 2u,      // outbox overflow
    ST_HOLES = 4u,       // hole list overflow
    ST_NAN = 8u,         // non-finite momentum
    ST_TILE_FULL = 16u,  // arrivals did not fit their tile (kept in the outbox, rebin needed)
    ST_BADCELL = 32u,    // a bin held a cell outside its tile, or the compaction did not pair up
    ST_TMA = 64u,        // the field tile's TMA load did not complete within the wait limit
};

struct DevStatus {
    unsigned flags;
    unsigned out_count;        // outbox entries this step
    unsigned overflow_count;   // outbox entries that did not fit their tile
    unsigned pad0;
    unsigned long long moved;  // particles written to the outbox
    unsigned long long dropped;
    unsigned long long duplicated;
    double kinetic;            // sum (m/q_m)(gamma-1) accumulated by the push
    double pad1[3];
};

struct Grid {
    int nx, ny, nz;     // interior cells
    int NX, NY, NZ;     // nx+2, ny+2, nz+2
    int pz;             // z pitch of device field arrays
    int tx, ty, tz;     // cells per tile
    int ntx, nty, ntz;  // tiles per axis
    int ntiles;
    int bz, by;         // bits of the packed cell index used by k and by l
    double lx, ly, lz, hx, hy, hz, tau;
    __host__ __device__ size_t nodes_pitched() const { return (size_t)NX * NY * pz; }
    __host__ __device__ size_t nodes_ref() const { return (size_t)NX * NY * NZ; }
    __host__ __device__ size_t node(int i, int l, int k) const { return ((size_t)i * NY + l) * pz + k; }
    __host__ __device__ int ncells() const { return nx * ny * nz; }
    // a particle's int32 cell index packs (i, l, k) as bit fields, so the hot
    // loops decode it with shifts and masks instead of integer division
    __host__ __device__ int cell_of(int i, int l, int k) const { return (i << (by + bz)) | (l << bz) | k; }
    __host__ __device__ void cell_ijk(int c, int &i, int &l, int &k) const {
        k = c & ((1 << bz) - 1);
        l = (c >> bz) & ((1 << by) - 1);
        i = c >> (by + bz);
    }
    __host__ __device__ int dense_of(int i, int l, int k) const { return (i * ny + l) * nz + k; }
    __host__ __device__ int tile_of_cell(int i, int l, int k) const {
        return ((i / tx) * nty + (l / ty)) * ntz + (k / tz);
    }
};

// The field kernels after the push (J fold, B, E, E ghosts) run as a chain
// of programmatically dependent launches: each is launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, and every CTA first
// waits in hardware for the previous grid to complete and flush
// (griddepcontrol.wait), then lets the next grid be scheduled
// (griddepcontrol.launch_dependents).  The next grid's CTAs thus take SM
// slots as this grid's retire and start the moment it is done, instead of
// after a full launch gap; every CTA of a grid has started before the next
// grid's are scheduled, so waiting CTAs never hold slots the running grid
// needs.  For a kernel launched without the attribute both are no-ops.
__device__ __forceinline__ void chain_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... P, typename... A>
inline cudaError_t launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, cudaStream_t s, A &&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Tile current accumulation in 64-bit fixed point.  Each contribution is
// rounded to the tile's quantum q = 2^(E-62), where 2^E exceeds
// bound = 2.5 * sum_s |m_s| * count_s(tile): one particle segment adds at most
// 1.03 |m| to a node (pqr, cell.h:1578-1616, with |dx| < tau and the stencil
// in range), two segments per particle, so no tile sum can overflow.  The
// sums are exact integer sums, so the tile current does not depend on the
// order in which the threads add.  Rounding: |error| <= q/2 per contribution.
//
// Every 64-bit add into shared memory goes through shared_add64: two native
// 32-bit atomics.  The add of the low halves returns the old low word, so the
// carry of each add is known exactly and goes into the high word with the
// high half.  Integer adds modulo 2^32 commute, so the pair, read as one
// little-endian 64-bit word after a barrier, is the exact sum modulo 2^64 --
// what a 64-bit atomicAdd gives -- whatever the interleaving.  Measured: a
// 64-bit shared-memory atomicAdd costs about 8 atomic instructions per add
// in the FP64 push (lanes of a warp often share a node), and the split took
// the c2 FP64 push from 106.4 to 72.4 ms.
__device__ __forceinline__ void shared_add64(unsigned long long *w, long long v) {
    unsigned *p = (unsigned *)w;  // p[0] low word, p[1] high word
    const unsigned lo = (unsigned)v;
    const unsigned old = atomicAdd(p, lo);
    const unsigned hi = (unsigned)((unsigned long long)v >> 32) + (old + lo < old ? 1u : 0u);
    if (hi) atomicAdd(p + 1, hi);
}
__device__ __forceinline__ void fx_add(unsigned long long *a, double v, double inv_q) {
    long long iv = __double2ll_rn(v * inv_q);
    if (iv) shared_add64(a, iv);
}
__device__ __forceinline__ void fx_addf(unsigned long long *a, float v, float inv_q) {
    long long iv = __float2ll_rn(v * inv_q);
    if (iv) shared_add64(a, iv);
}
// Two-word form for the FP64 plain form.  The bound above assumes every
// particle moves at c; a dense slow plasma (thousands of particles per cell at
// v ~ 1e-3, whose beam and return currents cancel) adds contributions ~1e-9 of
// the bound, which a single word rounds at ~1e-10 of their size.  The second
// word takes each contribution's remainder in units of q * 2^-40:
//   s = v / q (exact: q is a power of two), r = rint(s), s - r exact
//   (Sterbenz: |s - r| <= 1/2 and r, s within a factor 2 when r != 0),
// so the error is <= q * 2^-41 per contribution, and both adds are exact
// integer adds (order-independent).  |lo| grows by <= 2^39 per add: 2^24
// adds into one node before it could overflow, i.e. 8M particles in a tile
// (kFxMaxTileSlots guards it).
constexpr int kFxLoBits = 40;
constexpr long long kFxMaxTileSlots = 1ll << 23;
__device__ __forceinline__ void fx_split(double v, double inv_q, long long &ih, long long &il) {
    const double s = v * inv_q;
    const double r = rint(s);
    ih = (long long)r;
    il = __double2ll_rn((s - r) * 1099511627776.0);  // 2^40
}
__device__ __forceinline__ void fx_add2(unsigned long long *hi, unsigned long long *lo, double v, double inv_q) {
    long long ih, il;
    fx_split(v, inv_q, ih, il);
    if (ih) shared_add64(hi, ih);
    if (il) shared_add64(lo, il);
}
// The same split with an int32 second word (native 32-bit shared atomics: a
// c2 FP64 push takes 22 ms less than with the 64-bit word).  The remainder
// s - r (|s - r| <= 1/2) is counted in units of q * 2^-L, so one add is at
// most 2^(L-1) in magnitude.  A tile of N particles adds at most 2N times to
// one word (two zigzag segments per particle, one add per node of a segment),
// so L = 31 - bits(N), N < 2^bits(N), keeps every sum below N 2^L < 2^31:
// exact and order-independent like the 64-bit word, with |error| <=
// q * 2^-(L+1) per contribution.  The push uses it when every tile's
// capacity gives L >= kFxLo32MinBits (tiles below 2^17 particles; the
// reference's default run, 2.6e5 particles per tile, keeps the 64-bit word).
constexpr int kFxLo32MinBits = 14;
__device__ __forceinline__ int fx_lo32_bits(long long n) {
    int b = 0;
    while ((1ll << b) <= n) b++;
    return 31 - b;
}
__device__ __forceinline__ void fx_add_lo32(unsigned long long *hi, int *lo, double v, double inv_q,
                                            double lo_scale) {
    const double s = v * inv_q;
    const double r = rint(s);
    const long long ih = (long long)r;
    const int il = __double2int_rn((s - r) * lo_scale);  // lo_scale = 2^L: exact
    if (ih) shared_add64(hi, ih);
    if (il) atomicAdd(lo, il);
}

struct SpeciesView {
    // plain form
    double *x, *y, *z, *px, *py, *pz;
    // mixed form
    float *ox, *oy, *oz, *fx, *fy, *fz;
    int *cell;
    int *tile_start;  // ntiles + 1
    int *tile_count;  // ntiles
    double q_m, m;
};

// one migrating particle (plain form): 56 bytes
struct OutPlain {
    double x, y, z, px, py, pz;
    int cell, species;
};
// one migrating particle (mixed form): 32 bytes
struct OutMixed {
    float ox, oy, oz, px, py, pz;
    int cell, species;
};

struct StepParams {
    Grid g;
    int nsp;
    int mixed;
    SpeciesView sp[kMaxSpecies];
    // plain: double fields; mixed: float E/H, double J
    const void *E[3];
    const void *H[3];
    double *J[3];
    void *outbox;
    unsigned out_cap;
    DevStatus *st;
    // mixed push: per species, the largest contribution bound of the last
    // push (float, 0 = none yet) and the one this push records (float bits,
    // atomicMax); sizes the int32 tile current's quantum
    const float *lb_prev;
    unsigned *lb_cur;
    // mixed push: nonzero when H in memory is the full-step field and the
    // push forms the B half step of its staged tile itself (pic_step); zero
    // when the sub-step call pic_b_half has already advanced H
    int b_half;
};

// FP32 form: TMA descriptors of the six E/H field arrays (3D {Nz+2, Ny+2,
// Nx+2} FP32 with the pitched z row, box = one tile + halo); a kernel
// parameter (__grid_constant__), so the descriptors live in parameter space
struct MixedMaps {
    CUtensorMap m[6];
};


}  // namespace pic
