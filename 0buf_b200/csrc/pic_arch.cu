// archAPI replacement with C linkage (include/pic0buf_arch.h); the reference
// versions are archAPI.cu:16-115.
#include <cuda_runtime.h>
#include "pic0buf_arch.h"

extern "C" {

int MemoryCopy(void *dst, void *src, size_t size, int dir) {
    cudaMemcpyKind kind;
    switch (dir) {
        case HOST_TO_DEVICE: kind = cudaMemcpyHostToDevice; break;
        case HOST_TO_HOST: kind = cudaMemcpyHostToHost; break;
        case DEVICE_TO_HOST: kind = cudaMemcpyDeviceToHost; break;
        case DEVICE_TO_DEVICE: kind = cudaMemcpyDeviceToDevice; break;
        default: return (int)cudaErrorInvalidMemcpyDirection;
    }
    return (int)cudaMemcpy(dst, src, size, kind);
}

int MemoryAllocate(void **dst, size_t size) { return (int)cudaMalloc(dst, size); }

int GetDeviceMemory(size_t *m_free, size_t *m_total) { return (int)cudaMemGetInfo(m_free, m_total); }

int MemorySet(void *s, int c, size_t n) { return (int)cudaMemset(s, c, n); }

int ThreadSynchronize(void) { return (int)cudaDeviceSynchronize(); }

int DeviceSynchronize(void) { return (int)cudaDeviceSynchronize(); }

int getLastError(void) { return (int)cudaGetLastError(); }

const char *getErrorString(int err) { return cudaGetErrorString((cudaError_t)err); }

int SetDevice(int n) { return (int)cudaSetDevice(n); }

}  // extern "C"
