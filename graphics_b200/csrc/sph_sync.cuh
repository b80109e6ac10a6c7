// sph_sync.cuh -- host-synchronous memory operations for the entry points.
//
// Every handle works on its own non-blocking streams, which are not ordered
// with the legacy default stream that cudaMemcpy, cudaMemcpy2D and
// cudaMemset use.  A host-to-device cudaMemcpy from pageable memory may
// return before its last bytes have reached the device, and a
// device-to-device copy or a memset may return before it has run: a kernel
// launched next on a handle's stream could read the old contents (seen as a
// boundary table whose tail was sorted from the previous contents of a
// reused allocation).  These wrappers wait for the legacy stream after the
// operation, so it has landed when they return.
#pragma once
#include <cuda_runtime.h>

inline cudaError_t copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    const cudaError_t e = cudaMemcpy(dst, src, bytes, kind);
    return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}

inline cudaError_t copy2d_sync(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                               size_t height, cudaMemcpyKind kind) {
    const cudaError_t e = cudaMemcpy2D(dst, dpitch, src, spitch, width, height, kind);
    return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}

inline cudaError_t memset_sync(void* p, int value, size_t bytes) {
    const cudaError_t e = cudaMemset(p, value, bytes);
    return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}
