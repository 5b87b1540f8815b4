// Field-energy reduction that allocates nothing (pic_field_energy_noalloc).
//
// Some callers cannot let this library call cudaMalloc: a host framework
// that has already handed all device memory to its own pool (a PIC code with
// hundreds of GB of particles reserves HBM up front), or a timed loop that
// cannot afford cudaMalloc's implicit device synchronisation.  For them this
// entry point works on caller-owned device arrays and keeps its only scratch
// -- the per-block partial sums of a deterministic two-pass reduction -- in a
// file-scope __device__ array of fixed size, which every GPU that loads the
// library holds until the process exits.
#include <cuda_runtime.h>
#include <mutex>
#include "pic0buf.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// three partial sums per block: sum E^2 and sum H^2 over the nodes 1..N of
// every axis, sum E^2 over all nodes (the reference's GPU_getCellEnergy)
static __device__ __align__(256) double g_partials[3 * PIC_NOALLOC_MAX_BLOCKS];

// device address of g_partials per device, taken once with that device current
std::mutex g_mu;
double *g_addr[kMaxDevices] = {};

__global__ void k_energy_partials(int nx, int ny, int nz, const double *__restrict__ Ex,
                                  const double *__restrict__ Ey, const double *__restrict__ Ez,
                                  const double *__restrict__ Hx, const double *__restrict__ Hy,
                                  const double *__restrict__ Hz, long long nodes, double *partials) {
    __shared__ double red[3][kThreads / 32];
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double we = 0.0, wb = 0.0, wr = 0.0;
    if (n < nodes) {
        const int NY = ny + 2, NZ = nz + 2;
        int k = (int)(n % NZ), l = (int)((n / NZ) % NY), i = (int)(n / ((long long)NZ * NY));
        double ex = Ex[n], ey = Ey[n], ez = Ez[n];
        wr = ex * ex + ey * ey + ez * ez;
        if (i >= 1 && i <= nx && l >= 1 && l <= ny && k >= 1 && k <= nz) {
            double hx = Hx[n], hy = Hy[n], hz = Hz[n];
            we = wr;
            wb = hx * hx + hy * hy + hz * hz;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        we += __shfl_down_sync(0xffffffffu, we, o);
        wb += __shfl_down_sync(0xffffffffu, wb, o);
        wr += __shfl_down_sync(0xffffffffu, wr, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = we; red[1][w] = wb; red[2][w] = wr; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int j = 0; j < kThreads / 32; j++) s += red[threadIdx.x][j];
        // every block writes its three slots, so nothing has to start at zero
        partials[threadIdx.x * PIC_NOALLOC_MAX_BLOCKS + blockIdx.x] = s;
    }
}

// one block: fixed-order sum of the partials (deterministic result)
__global__ void k_energy_finish(const double *partials, int nblocks, double *out3) {
    __shared__ double red[3][kThreads];
    for (int c = 0; c < 3; c++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[c * PIC_NOALLOC_MAX_BLOCKS + b];
        red[c][threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int j = 0; j < kThreads; j++) s += red[threadIdx.x][j];
        out3[threadIdx.x] = threadIdx.x < 2 ? 0.5 * s : s;
    }
}

}  // namespace

extern "C" int pic_field_energy_noalloc(int nx, int ny, int nz, const double *Ex, const double *Ey, const double *Ez,
                                        const double *Hx, const double *Hy, const double *Hz, double *out3,
                                        void *stream) {
    if (nx < 1 || ny < 1 || nz < 1 || !Ex || !Ey || !Ez || !Hx || !Hy || !Hz || !out3) return PIC_ERR_ARG;
    // each extent alone must fit the scratch before any product is formed
    if (nx > PIC_NOALLOC_MAX_NODES || ny > PIC_NOALLOC_MAX_NODES || nz > PIC_NOALLOC_MAX_NODES) return PIC_ERR_ARG;
    const long long nodes = ((long long)nx + 2) * ((long long)ny + 2) * ((long long)nz + 2);
    const long long nblocks = (nodes + kThreads - 1) / kThreads;
    if (nblocks > PIC_NOALLOC_MAX_BLOCKS) return PIC_ERR_ARG;  // more than PIC_NOALLOC_MAX_NODES nodes
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= kMaxDevices) return PIC_ERR_ARG;
    double *partials;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            // first call on this device: its address of g_partials (the host-side
            // name is only a stand-in, not a device address)
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_partials);
            if (e != cudaSuccess) return (int)e;
            g_addr[dev] = (double *)p;
        }
        partials = g_addr[dev];
    }
    // an error left by the caller's own earlier work is reported as such, not
    // as a failure of these launches (cudaPeekAtLastError does not clear it)
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) return (int)e;
    cudaStream_t s = (cudaStream_t)stream;
    k_energy_partials<<<(unsigned)nblocks, kThreads, 0, s>>>(nx, ny, nz, Ex, Ey, Ez, Hx, Hy, Hz, nodes, partials);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    k_energy_finish<<<1, kThreads, 0, s>>>(partials, (int)nblocks, out3);
    return (int)cudaGetLastError();
}
