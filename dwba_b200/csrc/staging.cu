// Host-to-device copies by the SMs: a kernel loads from page-locked host memory through its device
// mapping (unified addressing) and stores into device memory. A small copy made this way does not
// queue behind a large transfer that occupies the copy engines: while a batch's waves stream to the
// device, the descriptors its planning produces in the meantime arrive at once, so that kernels
// whose waves are already there can start.
#include "common.cuh"

namespace {

__global__ void copy16_kernel(uint4* __restrict__ dst, const uint4* __restrict__ src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

__global__ void copy1_kernel(unsigned char* __restrict__ dst, const unsigned char* __restrict__ src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// the device address of [p, p + n) when it lies in one allocation of the given kind, else null
const void* mapped_range(const void* p, int64_t n, cudaMemoryType kind) {
  cudaPointerAttributes a, b;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const void* last = (const char*)p + (n - 1);
  if (cudaPointerGetAttributes(&b, last) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != kind || b.type != kind || !a.devicePointer || !b.devicePointer) return nullptr;
  if ((const char*)b.devicePointer != (const char*)a.devicePointer + (n - 1)) return nullptr;
  return a.devicePointer;
}

}  // namespace

extern "C" int dwba_copy_from_host(void* dst_dev, const void* src_host, int64_t nbytes, dwba_stream_t stream) {
  if (nbytes == 0) return DWBA_OK;
  if (!dst_dev || !src_host || nbytes < 0) return DWBA_ERR_INVALID_ARG;
  const void* src = mapped_range(src_host, nbytes, cudaMemoryTypeHost);
  const void* dst = mapped_range(dst_dev, nbytes, cudaMemoryTypeDevice);
  if (!src || !dst) return DWBA_ERR_INVALID_ARG;  // not page-locked mapped host memory / device memory
  const int threads = 256;
  const bool v16 = ((uintptr_t)src % 16 == 0) && ((uintptr_t)dst % 16 == 0) && (nbytes % 16 == 0);
  const int64_t n = v16 ? nbytes / 16 : nbytes;
  const int blocks = dwba_grid_1d(n, threads, 148 * 4);
  if (v16)
    copy16_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>((uint4*)dst, (const uint4*)src, n);
  else
    copy1_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>((unsigned char*)dst, (const unsigned char*)src, n);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
