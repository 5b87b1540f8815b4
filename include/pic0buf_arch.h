/*
 * pic0buf_arch.h -- drop-in replacement of the reference's arch layer,
 * archAPI.h:1-127 (snytav/0buf), with C linkage.
 *
 * Same names, argument meaning and direction codes as the reference; every
 * call returns the CUDA error code as an int (archAPI.cu:39-54 does the same
 * for MemoryCopy).  Differences, all fixes of reference defects:
 *   - MemoryAllocate returns the cudaMalloc status (archAPI.cu:61-65 always
 *     returns 0);
 *   - MemoryCopy with an unknown direction returns
 *     cudaErrorInvalidMemcpyDirection instead of using an uninitialised kind
 *     (archAPI.cu:44-53);
 *   - MemorySet and DeviceSynchronize/ThreadSynchronize exist in the CUDA build
 *     (archAPI.cu:79-104 defines them only for the CPU build); MemorySet sets
 *     DEVICE memory.
 * The device-side helpers of archAPI.h (MultiThreadAdd, BlockThreadSynchronize,
 * AsyncCopy) have no host ABI: the kernels use native FP64 atomics and
 * barriers.
 */
#ifndef PIC0BUF_ARCH_H
#define PIC0BUF_ARCH_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HOST_TO_DEVICE -131313   /* archAPI.h:8 */
#define HOST_TO_HOST -131314     /* archAPI.h:9 */
#define DEVICE_TO_HOST -131315   /* archAPI.h:10 */
#define DEVICE_TO_DEVICE -131316 /* archAPI.h:11 */

int MemoryCopy(void *dst, void *src, size_t size, int dir);   /* archAPI.h:103 */
int MemoryAllocate(void **dst, size_t size);                  /* archAPI.h:107 */
int GetDeviceMemory(size_t *m_free, size_t *m_total);         /* archAPI.h:109 */
int MemorySet(void *s, int c, size_t n);                      /* archAPI.h:111 */
int ThreadSynchronize(void);                                  /* archAPI.h:114 */
int DeviceSynchronize(void);                                  /* archAPI.h:117-121 */
int getLastError(void);                                       /* archAPI.h:119-123 */
const char *getErrorString(int err);                          /* archAPI.h:92 */
int SetDevice(int n);                                         /* archAPI.h:94 */

#ifdef __cplusplus
}
#endif
#endif /* PIC0BUF_ARCH_H */
