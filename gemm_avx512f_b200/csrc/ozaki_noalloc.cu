// ozaki_noalloc.cu -- the allocation-free Ozaki DGEMM entry point.
//
// Some callers cannot allocate device memory when they call the library: a
// real-time loop that must stay out of the allocator for its latency, or a
// process whose device memory another framework reserved up front, so that a
// cudaMalloc at call time would fail or stall.  b2_dgemm_ozaki_noalloc serves
// them.  It runs the same kernels as b2_dgemm(..., B2_METHOD_OZAKI, ...) but
// takes every scratch buffer (residue slices, residue products, scaling
// exponents, the kernels' error word) from the file-scope array below, and it
// calls no cudaMalloc, cudaFree or other allocating routine; it does not
// touch the per-thread library context either, whose first use allocates.
//
// The array lives in this file's own device module, so only processes that
// call this entry point pay for it: under lazy module loading (the CUDA
// default since 12.2) its B2_NOALLOC_SCRATCH_BYTES are reserved on a device
// when this module first loads there -- at the first call on that device --
// and stay reserved until the process exits.
//
// The array's name, used in host code, is only a host-side stand-in for the
// device array, not a device address: a kernel handed it would fault or, where
// the GPU can reach host memory, silently work on the wrong memory.  So the
// first call on each device (that device current) looks the real address up
// with cudaGetSymbolAddress, checks the result, and caches it.  That first
// call also uploads the Ozaki constant tables and synchronises its stream, so
// it should come before any stream capture.
//
// All calls on a device share the one array, which keeps the previous call's
// contents (only the error word is cleared at the start of each call): calls
// that overlap on the GPU -- different streams, or different host threads --
// race, and the caller must serialise them.
#include <mutex>

#include "b2_methods.cuh"

namespace b2 {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[B2_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocDevice {
  unsigned char *base = nullptr;  // device address of g_noalloc_scratch
  int sm_count = 0;
  int cc_major = 0;
};
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

// Set-up of the current device, once: the array's device address and the
// device attributes every call needs.
int noalloc_device(int dev, NoallocDevice *out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return B2_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocDevice &d = g_noalloc_dev[dev];
  if (!d.base) {
    int major = 0, sms = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      (void)cudaGetLastError();
      return B2_ERR_NO_DEVICE;
    }
    if (major < 10) return B2_ERR_NO_DEVICE;
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
    d.sm_count = sms;
    d.cc_major = major;
    d.base = (unsigned char *)p;
  }
  *out = d;
  return B2_OK;
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int b2_dgemm_ozaki_noalloc(char transa, char transb, int m, int n, int k,
                                      double alpha, const double *A, int lda, const double *B,
                                      int ldb, double beta, double *C, int ldc, int slices,
                                      void *stream) {
  int info = 0;
  int rc = check_gemm(transa, transb, m, n, k, lda, ldb, ldc, A, B, C, &info);
  if (rc != B2_OK) return rc;
  if (m == 0 || n == 0) return B2_OK;
  if (slices < 0 || slices > 16) return B2_ERR_ARG;
  const int s = slices > 0 ? slices : ozaki_auto_moduli(k);
  const bool product = k > 0 && alpha != 0.0;
  // size limit first, so an oversized call is refused before any set-up
  if (product && (k > (1 << 15) || ozaki_noalloc_bytes(m, n, k, s) > B2_NOALLOC_SCRATCH_BYTES))
    return B2_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return B2_ERR_NO_DEVICE;
  }
  NoallocDevice d;
  rc = noalloc_device(dev, &d);
  if (rc != B2_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (!is_device_ptr(C) || (product && (!is_device_ptr(A) || !is_device_ptr(B))))
    return B2_ERR_ARG;
  if (!product) {
    B2_CUDA_TRY(cudaMemsetAsync(d.base, 0, sizeof(int), st));
    return beta == 1.0 ? B2_OK : scale_matrix_d(m, n, beta, C, ldc, st);
  }
  return ozaki_noalloc_run(d.base, B2_NOALLOC_SCRATCH_BYTES, dev, d.sm_count, transa, transb, m,
                           n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, st);
}

extern "C" int b2_dgemm_ozaki_noalloc_error(int clear, void *stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return B2_ERR_NO_DEVICE;
  }
  NoallocDevice d;
  const int rc = noalloc_device(dev, &d);
  if (rc != B2_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int v = 0;
  if (cudaMemcpyAsync(&v, d.base, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    (void)cudaGetLastError();
    return B2_ERR_CUDA;
  }
  if (clear && v) {
    if (cudaMemsetAsync(d.base, 0, sizeof(int), st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      (void)cudaGetLastError();
      return B2_ERR_CUDA;
    }
  }
  return v;
}
