// api.cu -- the C ABI of libb2blas.so: per-thread context, argument checks,
// host/device pointer handling, and the drop-in Fortran-BLAS symbols.
//
// The drop-in symbols keep the reference's contract (src/gemm_driver.c:116):
// void return, everything by pointer, synchronous.  Where the reference
// allocates packing buffers per call (src/gemm_driver.c:133-140) this layer
// keeps grow-only device workspaces per host thread, and where the reference
// splits N across OpenMP threads (:136-149) the kernels' CTA grid does.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#if defined(__x86_64__)
#include <cpuid.h>
#endif

#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "b2_internal.cuh"
#include "b2_methods.cuh"

namespace b2 {

static thread_local Status g_status;
static thread_local Ctx *g_ctx = nullptr;

static void set_status(int code, int info = 0) {
  g_status.code = code;
  g_status.info = info;
}

int cuda_fail(cudaError_t e, const char *what) {
  if (getenv("B2_VERBOSE")) fprintf(stderr, "b2blas: %s failed: %s\n", what, cudaGetErrorString(e));
  (void)cudaGetLastError();  // clear sticky-free errors so the next call starts clean
  return B2_ERR_CUDA;
}

namespace {
struct CtxOwner {
  Ctx *c = nullptr;
  ~CtxOwner() {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < WS_COUNT; ++i)
      if (c->ws[i]) cudaFree(c->ws[i]);
    if (c->derr && !c->derr_host) cudaFree(c->derr);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->h2d) cudaStreamSynchronize(c->h2d), cudaStreamDestroy(c->h2d);
    if (c->d2h) cudaStreamSynchronize(c->d2h), cudaStreamDestroy(c->d2h);
    for (int i = 0; i < Ctx::PIPE_EVENTS; ++i) {
      if (c->ev_in[i]) cudaEventDestroy(c->ev_in[i]);
      if (c->ev_done[i]) cudaEventDestroy(c->ev_done[i]);
      if (c->ev_c[i]) cudaEventDestroy(c->ev_c[i]);
    }
    if (c->plan_ev) cudaEventDestroy(c->plan_ev);
    for (int i = 0; i < 2; ++i) {
      if (c->bounce_ev[i]) cudaEventSynchronize(c->bounce_ev[i]), cudaEventDestroy(c->bounce_ev[i]);
      if (c->bounce[i]) cudaFreeHost(c->bounce[i]);
    }
    for (int i = 0; i < Ctx::OZ_EVENTS; ++i)
      if (c->oz_ev[i]) cudaEventDestroy(c->oz_ev[i]);
    for (int i = 0; i < 2; ++i) {
      if (c->grp_ev[i]) cudaEventSynchronize(c->grp_ev[i]), cudaEventDestroy(c->grp_ev[i]);
      if (c->grp_host[i]) cudaFreeHost(c->grp_host[i]);
    }
    if (c->oz_gemm) cudaStreamSynchronize(c->oz_gemm), cudaStreamDestroy(c->oz_gemm);
    if (c->oz_aux) cudaStreamSynchronize(c->oz_aux), cudaStreamDestroy(c->oz_aux);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
  }
};
thread_local CtxOwner g_owner;

int method_from_env(const char *v, int dflt) {
  if (!v) return dflt;
  if (!strcmp(v, "fp64")) return B2_METHOD_FP64;
  if (!strcmp(v, "ozaki")) return B2_METHOD_OZAKI;
  if (!strcmp(v, "auto")) return B2_METHOD_AUTO;
  if (!strcmp(v, "fp32")) return B2_METHOD_FP32;
  if (!strcmp(v, "tf32")) return B2_METHOD_TF32;
  if (!strcmp(v, "tf32x3")) return B2_METHOD_TF32X3;
  if (!strcmp(v, "bf16x3")) return B2_METHOD_BF16X3;
  return dflt;
}
}  // namespace

Ctx *ctx() {
  if (g_ctx) {
    cudaSetDevice(g_ctx->device);
    return g_ctx;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { (void)cudaGetLastError(); return nullptr; }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) { (void)cudaGetLastError(); return nullptr; }
  if (prop.major < 10) return nullptr;  // sm_100a code only
  Ctx *c = new Ctx();
  c->device = dev;
  c->sm_count = prop.multiProcessorCount;
  c->cc_major = prop.major;
  c->cc_minor = prop.minor;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost(&c->pinned, 4096) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return nullptr;
  }
  for (int i = 0; i < Ctx::PIPE_EVENTS; ++i) {
    if (cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_done[i], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_c[i], cudaEventDisableTiming) != cudaSuccess) {
      (void)cudaGetLastError();
      delete c;
      return nullptr;
    }
  }
  if (cudaEventCreateWithFlags(&c->plan_ev, cudaEventDisableTiming) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return nullptr;
  }
  if (cudaHostGetDevicePointer(&c->pinned_dev, c->pinned, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    c->pinned_dev = nullptr;
  }
  // The kernels' error word: mapped pinned memory at offset 128 when the
  // device can address it (the host then reads it without a copy after a
  // synchronisation), else 64 bytes of device memory.
  if (c->pinned_dev) {
    c->derr_host = (int *)((uint8_t *)c->pinned + 128);
    c->derr = (int *)((uint8_t *)c->pinned_dev + 128);
    *c->derr_host = 0;
  } else if (cudaMalloc(&c->derr, 64) != cudaSuccess || cudaMemset(c->derr, 0, 64) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return nullptr;
  }
  c->dgemm_method = method_from_env(getenv("B2_METHOD"), B2_METHOD_FP64);
  c->sgemm_method = method_from_env(getenv("B2_SGEMM_METHOD"), B2_METHOD_FP32);
  if (const char *s = getenv("B2_SLICES")) c->dgemm_slices = atoi(s);
  g_ctx = c;
  g_owner.c = c;
  if (const char *path = getenv("B2_SELECTOR")) {  // learned selector weights for AUTO
    if (FILE *fh = fopen(path, "rb")) {
      const int np = b2_mlp_param_count();
      float *w = (float *)malloc(sizeof(float) * np);
      if (w && fread(w, sizeof(float), np, fh) == (size_t)np) b2_selector_set(w);
      free(w);
      fclose(fh);
    }
  }
  return c;
}

bool ozaki_overlap_streams(Ctx *c) {
  if (c->oz_gemm && c->oz_aux && c->oz_ev[Ctx::OZ_EVENTS - 1]) return true;
  int lo = 0, hi = 0;
  if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) {
    (void)cudaGetLastError();
    lo = hi = 0;
  }
  if (!c->oz_gemm && cudaStreamCreateWithPriority(&c->oz_gemm, cudaStreamNonBlocking, hi) != cudaSuccess) {
    (void)cudaGetLastError();
    c->oz_gemm = nullptr;
    return false;
  }
  if (!c->oz_aux && cudaStreamCreateWithPriority(&c->oz_aux, cudaStreamNonBlocking, lo) != cudaSuccess) {
    (void)cudaGetLastError();
    c->oz_aux = nullptr;
    return false;
  }
  for (int i = 0; i < Ctx::OZ_EVENTS; ++i)
    if (!c->oz_ev[i] && cudaEventCreateWithFlags(&c->oz_ev[i], cudaEventDisableTiming) != cudaSuccess) {
      (void)cudaGetLastError();
      c->oz_ev[i] = nullptr;
      return false;
    }
  return true;
}

int take_device_error(Ctx *c, int st) {
  int v = 0;
  if (c->derr_host) {
    v = *(volatile int *)c->derr_host;
    if (v) *(volatile int *)c->derr_host = 0;
  } else if (cudaMemcpy(&v, c->derr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    (void)cudaGetLastError();
    return st == B2_OK ? B2_ERR_CUDA : st;
  } else if (v && cudaMemset(c->derr, 0, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
  }
  return (st == B2_OK && v) ? B2_ERR_TIMEOUT : st;
}

void *workspace(Ctx *c, int slot, size_t bytes) {
  if (bytes == 0) bytes = 256;
  if (c->ws_bytes[slot] >= bytes) return c->ws[slot];
  if (c->ws[slot]) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->ws[slot]);
    c->ws[slot] = nullptr;
    c->ws_bytes[slot] = 0;
  }
  size_t want = bytes + bytes / 8;
  want = (want + 4095) & ~(size_t)4095;
  void *p = nullptr;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    (void)cudaGetLastError();
    if (cudaMalloc(&p, bytes) != cudaSuccess) { (void)cudaGetLastError(); return nullptr; }
    want = bytes;
  }
  c->ws[slot] = p;
  c->ws_bytes[slot] = want;
  return p;
}

cudaStream_t pick_stream(Ctx *c, void *user_stream) {
  return user_stream ? (cudaStream_t)user_stream : c->stream;
}

// ------------------------------------------------------ pointer staging --
bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { (void)cudaGetLastError(); return false; }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// ------------------------------------------------ pageable host buffers --
// A reference BLAS caller passes malloc'ed (pageable) memory.  The CUDA
// driver copies such memory through its own staging with one host thread,
// about 10 GB/s here; instead the library copies it through two pinned
// bounce buffers of its own, with up to 16 host threads doing the host-side
// copy of one buffer while the DMA engine moves the other.
bool host_pageable(const void *p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { (void)cudaGetLastError(); return true; }
  return at.type == cudaMemoryTypeUnregistered;
}

namespace {
// Persistent host threads that run the tasks of one parallel copy; the
// calling thread takes tasks too.  One parallel copy at a time.
struct CopyPool {
  std::mutex run_mu, mu;
  std::condition_variable cv, cv_done;
  const std::function<void(int)> *job = nullptr;
  int ntasks = 0, next = 0, pending = 0;
  unsigned long gen = 0;
  int workers = -1;

  void worker() {
    unsigned long seen = 0;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv.wait(lk, [&] { return gen != seen; });
      seen = gen;
      while (job && next < ntasks) {
        const int t = next++;
        const std::function<void(int)> *f = job;
        lk.unlock();
        (*f)(t);
        lk.lock();
        if (--pending == 0) cv_done.notify_all();
      }
    }
  }
  void run(int n, const std::function<void(int)> &f) {
    std::lock_guard<std::mutex> rl(run_mu);
    {
      std::lock_guard<std::mutex> lk(mu);
      if (workers < 0) {
        unsigned hw = std::thread::hardware_concurrency();
        workers = (int)(hw > 16 ? 15 : (hw > 1 ? hw - 1 : 0));
        for (int i = 0; i < workers; ++i) {
          try {
            std::thread([this] { worker(); }).detach();
          } catch (...) {
            workers = i;
            break;
          }
        }
      }
    }
    std::unique_lock<std::mutex> lk(mu);
    job = &f;
    ntasks = n;
    next = 0;
    pending = n;
    ++gen;
    cv.notify_all();
    while (next < ntasks) {
      const int t = next++;
      lk.unlock();
      f(t);
      lk.lock();
      --pending;
    }
    cv_done.wait(lk, [&] { return pending == 0; });
    job = nullptr;
  }
};
// Never destroyed: its detached workers wait on its condition variable until
// the process ends, and destroying a condition variable that threads wait on
// blocks the exit.
CopyPool &copy_pool() {
  static CopyPool *pool = new CopyPool;
  return *pool;
}

// rows x width bytes from src (pitch spitch) to dst (pitch dpitch), split over
// the pool when large.
void parallel_copy2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                     size_t rows) {
  const size_t total = width * rows;
  const int tasks = total < (size_t)(4u << 20) ? 1 : 16;
  auto body = [&](int t) {
    const size_t r0 = rows * t / tasks, r1 = rows * (t + 1) / tasks;
    for (size_t r = r0; r < r1; ++r)
      memcpy((char *)dst + r * dpitch, (const char *)src + r * spitch, width);
  };
  if (tasks == 1) {
    body(0);
    return;
  }
  const std::function<void(int)> f = body;
  copy_pool().run(tasks, f);
}

int bounce_ready(Ctx *c) {
  for (int i = 0; i < 2; ++i) {
    if (!c->bounce[i] && cudaMallocHost(&c->bounce[i], Ctx::BOUNCE_BYTES) != cudaSuccess) {
      (void)cudaGetLastError();
      c->bounce[i] = nullptr;
      return B2_ERR_NOMEM;
    }
    if (!c->bounce_ev[i] &&
        cudaEventCreateWithFlags(&c->bounce_ev[i], cudaEventDisableTiming) != cudaSuccess) {
      (void)cudaGetLastError();
      c->bounce_ev[i] = nullptr;
      return B2_ERR_CUDA;
    }
  }
  return B2_OK;
}
}  // namespace

// Host -> device 2-D copy (rows of `width` bytes), stream-ordered on s; a
// pageable source goes through the bounce buffers (the call returns once the
// host side has been copied; the DMAs stay queued on s).
int copy_h2d(Ctx *c, void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
             size_t rows, cudaStream_t s) {
  if (!rows || !width) return B2_OK;
  if (!host_pageable(src) || width > Ctx::BOUNCE_BYTES) {
    B2_CUDA_TRY(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDefault, s));
    return B2_OK;
  }
  int rc = bounce_ready(c);
  if (rc != B2_OK) return rc;
  const size_t per = Ctx::BOUNCE_BYTES / width;
  for (size_t r0 = 0, i = 0; r0 < rows; r0 += per, ++i) {
    const size_t nr = rows - r0 < per ? rows - r0 : per;
    const int slot = (int)(i & 1);
    B2_CUDA_TRY(cudaEventSynchronize(c->bounce_ev[slot]));  // its previous DMA has finished
    parallel_copy2d(c->bounce[slot], width, (const char *)src + r0 * spitch, spitch, width, nr);
    B2_CUDA_TRY(cudaMemcpy2DAsync((char *)dst + r0 * dpitch, dpitch, c->bounce[slot], width, width,
                                  nr, cudaMemcpyHostToDevice, s));
    B2_CUDA_TRY(cudaEventRecord(c->bounce_ev[slot], s));
  }
  return B2_OK;
}

// Device -> host 2-D copy after the work queued on s; synchronous (the data
// is in host memory on return).  A pageable destination is filled from the
// bounce buffers, the DMA of the next chunk overlapping the host-side copy.
int copy_d2h(Ctx *c, void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
             size_t rows, cudaStream_t s) {
  if (!rows || !width) return B2_OK;
  if (!host_pageable(dst) || width > Ctx::BOUNCE_BYTES) {
    B2_CUDA_TRY(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDefault, s));
    B2_CUDA_TRY(cudaStreamSynchronize(s));
    return B2_OK;
  }
  int rc = bounce_ready(c);
  if (rc != B2_OK) return rc;
  const size_t per = Ctx::BOUNCE_BYTES / width;
  const size_t nchunks = (rows + per - 1) / per;
  auto issue = [&](size_t i) -> cudaError_t {
    const size_t r0 = i * per, nr = rows - r0 < per ? rows - r0 : per;
    const int slot = (int)(i & 1);
    cudaError_t e = cudaEventSynchronize(c->bounce_ev[slot]);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(c->bounce[slot], width, (const char *)src + r0 * spitch, spitch, width,
                            nr, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(c->bounce_ev[slot], s);
    return e;
  };
  for (size_t i = 0; i < nchunks && i < 2; ++i) B2_CUDA_TRY(issue(i));
  for (size_t i = 0; i < nchunks; ++i) {
    const int slot = (int)(i & 1);
    B2_CUDA_TRY(cudaEventSynchronize(c->bounce_ev[slot]));
    const size_t r0 = i * per, nr = rows - r0 < per ? rows - r0 : per;
    parallel_copy2d((char *)dst + r0 * dpitch, dpitch, c->bounce[slot], width, width, nr);
    if (i + 2 < nchunks) B2_CUDA_TRY(issue(i + 2));
  }
  return B2_OK;
}

int stage_in(Ctx *c, int slot, const void *host, int rows, int cols, int ld, size_t elem,
             void **dev, int *dld, cudaStream_t s) {
  const int ldd = (rows + 1) & ~1;  // even leading dimension keeps 16-B vector loads legal
  void *d = workspace(c, slot, (size_t)(ldd > 0 ? ldd : 2) * (cols > 0 ? cols : 1) * elem);
  if (!d) return B2_ERR_NOMEM;
  *dev = d;
  *dld = ldd > 0 ? ldd : 2;
  if (rows > 0 && cols > 0)
    return copy_h2d(c, d, (size_t)ldd * elem, host, (size_t)ld * elem, (size_t)rows * elem,
                    (size_t)cols, s);
  return B2_OK;
}

int stage_out(void *host, int ld, const void *dev, int dld, int rows, int cols, size_t elem,
              cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return B2_OK;
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  return copy_d2h(c, host, (size_t)ld * elem, dev, (size_t)dld * elem, (size_t)rows * elem,
                  (size_t)cols, s);
}

static bool notrans(char c) { return c == 'N' || c == 'n'; }

// BLAS argument check for xGEMM (positions as in the Fortran interface).
int check_gemm(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc, const void *a,
               const void *b, const void *c, int *info) {
  const int nrowa = notrans(ta) ? m : k;
  const int nrowb = notrans(tb) ? k : n;
  *info = 0;
  if (m < 0) *info = 3;
  else if (n < 0) *info = 4;
  else if (k < 0) *info = 5;
  else if (lda < (nrowa > 1 ? nrowa : 1)) *info = 8;
  else if (ldb < (nrowb > 1 ? nrowb : 1)) *info = 10;
  else if (ldc < (m > 1 ? m : 1)) *info = 13;
  else if (m > 0 && n > 0 && !c) *info = 12;
  else if (m > 0 && n > 0 && k > 0 && (!a || !b)) *info = !a ? 7 : 9;
  return *info ? B2_ERR_ARG : B2_OK;
}

// ------------------------------------------------------- DGEMM dispatch --
int dgemm_device(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                 const double *B, int ldb, double beta, double *C, int ldc, int method,
                 int slices, cudaStream_t s) {
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  if (method == B2_METHOD_DEFAULT) method = c->dgemm_method;
  if (slices <= 0) slices = c->dgemm_slices;
  if (method == B2_METHOD_AUTO)
    return dgemm_auto(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, slices, s);
  if (method == B2_METHOD_OZAKI)
    return dgemm_ozaki(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, slices, s);
  return dgemm_fp64(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, nullptr);
}

int sgemm_device(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                 const float *B, int ldb, float beta, float *C, int ldc, int method,
                 cudaStream_t s) {
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  if (method == B2_METHOD_DEFAULT) method = c->sgemm_method;
  return sgemm_dispatch(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, method, s);
}

// CLFLUSHOPT on this host (CPUID leaf 7, EBX bit 23); x86-64 only.
static bool host_has_clflushopt() {
#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
  static const bool has = [] {
    unsigned a = 0, b = 0, c = 0, d = 0;
    if (!__get_cpuid_count(7, 0, &a, &b, &c, &d)) return false;
    return ((b >> 23) & 1u) != 0;
  }();
  return has;
#else
  return false;
#endif
}

// Evicts [p, p + bytes) from this core's caches (CLFLUSHOPT, line by line).
static void host_evict_lines(const void *p, size_t bytes) {
#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
  const char *q = (const char *)((uintptr_t)p & ~(uintptr_t)63);
  const char *e = (const char *)p + bytes;
  for (; q < e; q += 64) asm volatile("clflushopt (%0)" ::"r"(q) : "memory");
#else
  (void)p, (void)bytes;
#endif
}

// True when every element of the m x n column-major host block (leading
// dimension ld) is finite: the bit-level exponent test, columns split over up
// to 16 host threads (one for small blocks).  Each column is evicted from the
// scanning core's caches once read, where the CPU can: the GPU later writes C
// back into these lines, and lines still held in a core's private cache make
// those DMA writes wait on the core (on a 16-core Xeon host with 2 MB of L2
// per core, the copy-out of the last-scanned columns ran at 15-20 GB/s
// instead of 55 GB/s without the eviction).
template <typename T>
static bool host_all_finite(const T *c, int m, int n, int ld) {
  using U = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
  const U emask = sizeof(T) == 8 ? (U)0x7FF0000000000000ull : (U)0x7F800000u;
  std::atomic<bool> ok{true};
  const bool evict = host_has_clflushopt();
  auto scan = [&](int j0, int j1) {
    for (int j = j0; j < j1 && ok.load(std::memory_order_relaxed); ++j) {
      const U *col = reinterpret_cast<const U *>(c + (size_t)j * ld);
      U bad = 0;
      for (int i = 0; i < m; ++i) bad |= (U)((col[i] & emask) == emask);
      if (evict) host_evict_lines(col, (size_t)m * sizeof(T));
      if (bad) ok.store(false, std::memory_order_relaxed);
    }
  };
  unsigned nt = std::thread::hardware_concurrency();
  if (nt > 16) nt = 16;
  if (nt < 1 || (double)m * n < 4194304.0) nt = 1;
  if (nt == 1) {
    scan(0, n);
    return ok.load();
  }
  std::vector<std::thread> th;
  const int per = (n + (int)nt - 1) / (int)nt;
  for (unsigned t = 0; t < nt; ++t) {
    const int j0 = (int)t * per, j1 = j0 + per < n ? j0 + per : n;
    if (j0 < j1) th.emplace_back(scan, j0, j1);
  }
  for (auto &x : th) x.join();
  return ok.load();
}

// Column blocks of the host-operand pipeline: blocks of a multiple of 256
// columns moving about 128 MB each (A, B and C counted), 2..PIPE_MAX blocks;
// 1 (no pipeline) for products under 2^32 flops.
static int pipeline_blocks(int m, int n, int k, size_t elem, int *cols) {
  const double flops = 2.0 * m * (double)n * k;
  *cols = n;
  if (flops < 4294967296.0 || n < 512) return 1;
  const double per_col = (double)(m + k) * elem;
  int cw = (int)(134217728.0 / per_col);
  cw = (cw + 255) / 256 * 256;
  if (cw < 256) cw = 256;
  int nb = (n + cw - 1) / cw;
  if (nb < 2) { cw = ((n + 1) / 2 + 255) / 256 * 256; nb = (n + cw - 1) / cw; }
  if (nb > Ctx::PIPE_MAX) { cw = ((n + Ctx::PIPE_MAX - 1) / Ctx::PIPE_MAX + 255) / 256 * 256; nb = (n + cw - 1) / cw; }
  *cols = cw;
  return nb;
}

// Shared host-or-device driver for the real drop-in GEMMs.  run(A, lda, B,
// ldb, C, ldc, mrows, ncols, stream) computes the mrows x ncols block of C
// from the op(A) rows and B columns it is given.  Host operands of a large product go through a
// three-stream pipeline over column blocks of B and C: A is copied once, then
// block j is copied in (copy-in stream), computed (library stream) and copied
// out (copy-out stream) while block j+1 is copied in, so the PCIe transfers,
// which dominate a host-to-host product, overlap the GEMM.
// Argument-check mode of the real drop-in GEMMs (B2_ARGS_BLAS / _OPENBLAS).
static std::atomic<int> g_arg_mode{-1};
static int arg_mode() {
  int v = g_arg_mode.load();
  if (v < 0) {
    const char *e = getenv("B2_ARG_MODE");
    v = (e && !strcmp(e, "openblas")) ? B2_ARGS_OPENBLAS : B2_ARGS_BLAS;
    int expect = -1;
    g_arg_mode.compare_exchange_strong(expect, v);
    v = g_arg_mode.load();
  }
  return v;
}

// The OpenBLAS-like dgemm_ checks (OpenBLAS-like_implementation/dgemm.c:488-498).
// Returns true when the call must return now (status already set).
static bool openblas_arg_checks(char ta, char tb, int m, int n, int k, int lda, int ldb) {
  if (m < 1 || n < 1) { set_status(B2_OK); return true; }
  const char *msg = nullptr;
  int info = 0;
  if (notrans(ta)) {
    if (lda < m) msg = "ERROR: LDA < M with column-major matrix A. Please check input parameters.", info = 8;
  } else if (lda < k) {
    msg = "ERROR: LDA < K with row-major matrix A. Please check input parameters.", info = 8;
  }
  if (!msg) {
    if (notrans(tb)) {
      if (ldb < k) msg = "ERROR: LDB < K with column-major matrix B. Please check input parameters.", info = 10;
    } else if (ldb < n) {
      msg = "ERROR: LDB < N with row-major matrix B. Please check input parameters.", info = 10;
    }
  }
  if (!msg) return false;
  printf("%s\n", msg);
  fflush(stdout);
  set_status(B2_ERR_ARG, info);
  return true;
}

template <typename T, typename F>
static int gemm_dropin(char ta, char tb, int m, int n, int k, T alpha, const T *a, int lda,
                       const T *b, int ldb, T beta, T *cm, int ldc, F &&run) {
  int info = 0;
  if (arg_mode() == B2_ARGS_OPENBLAS && openblas_arg_checks(ta, tb, m, n, k, lda, ldb))
    return g_status.code;
  int st = check_gemm(ta, tb, m, n, k, lda, ldb, ldc, a, b, cm, &info);
  if (st != B2_OK) { set_status(st, info); return st; }
  if (m == 0 || n == 0) { set_status(B2_OK); return B2_OK; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  cudaStream_t s = c->stream;
  const bool need_ab = (k > 0 && alpha != (T)0);
  const bool dev = is_device_ptr(cm) && (!need_ab || (is_device_ptr(a) && is_device_ptr(b)));
  if (dev) {
    st = run(a, lda, b, ldb, cm, ldc, m, n, s);
  } else {
    const int ra = notrans(ta) ? m : k, ca = notrans(ta) ? k : m;
    const int rb = notrans(tb) ? k : n, cb = notrans(tb) ? n : k;
    void *da = nullptr, *db = nullptr, *dc = nullptr;
    int dla = 2, dlb = 2, dlc = 2;
    int cw = n;
    // Pageable operands go through the bounce buffers in one block (their
    // host-side copies keep the host busy, so the column-block pipeline,
    // which queues every copy up front, does not apply to them).
    const bool pageable = host_pageable(cm) || (need_ab && (host_pageable(a) || host_pageable(b)));
    const int nb = need_ab && !pageable ? pipeline_blocks(m, n, k, sizeof(T), &cw) : 1;
    st = B2_OK;
    if (nb == 1) {
      if (need_ab) {
        st = stage_in(c, WS_STAGE_A, a, ra, ca, lda, sizeof(T), &da, &dla, s);
        if (st == B2_OK) st = stage_in(c, WS_STAGE_B, b, rb, cb, ldb, sizeof(T), &db, &dlb, s);
      }
      // beta == 0 reads C only to keep a NaN or Inf already there: an
      // all-finite host C is zeroed on the device instead of copied in
      if (st == B2_OK && beta == (T)0 && need_ab && host_all_finite(cm, m, n, ldc)) {
        dlc = (m + 1) & ~1;
        dc = workspace(c, WS_STAGE_C, (size_t)dlc * n * sizeof(T));
        if (!dc) st = B2_ERR_NOMEM;
        else {
          cudaError_t e = cudaMemsetAsync(dc, 0, (size_t)dlc * n * sizeof(T), s);
          if (e != cudaSuccess) st = cuda_fail(e, "zero C");
        }
      } else if (st == B2_OK) {
        st = stage_in(c, WS_STAGE_C, cm, m, n, ldc, sizeof(T), &dc, &dlc, s);
      }
      if (st == B2_OK) st = run((const T *)da, dla, (const T *)db, dlb, (T *)dc, dlc, m, n, s);
      if (st == B2_OK) st = stage_out(cm, ldc, dc, dlc, m, n, sizeof(T), s);
    } else {
      // Full-size device copies (no buffer is reused, so no block waits for
      // another's copy-out); the column block j of op(B) is B's columns
      // [j0, j1) for 'N' and its rows [j0, j1) for 'T'.
      dla = (ra + 1) & ~1;
      dlb = (rb + 1) & ~1;
      dlc = (m + 1) & ~1;
      da = workspace(c, WS_STAGE_A, (size_t)dla * ca * sizeof(T));
      db = workspace(c, WS_STAGE_B, (size_t)dlb * cb * sizeof(T));
      dc = workspace(c, WS_STAGE_C, (size_t)dlc * n * sizeof(T));
      if (!da || !db || !dc) st = B2_ERR_NOMEM;
      cudaError_t e = cudaSuccess;
      // Rows [r0, r1) of op(A): rows of A for 'N', columns of A for 'T'.
      auto copy_a_rows = [&](int r0, int r1) {
        return notrans(ta)
                   ? cudaMemcpy2DAsync((T *)da + r0, (size_t)dla * sizeof(T), a + r0,
                                       (size_t)lda * sizeof(T), (size_t)(r1 - r0) * sizeof(T),
                                       ca, cudaMemcpyDefault, c->h2d)
                   : cudaMemcpy2DAsync((T *)da + (size_t)r0 * dla, (size_t)dla * sizeof(T),
                                       a + (size_t)r0 * lda, (size_t)lda * sizeof(T),
                                       (size_t)k * sizeof(T), r1 - r0, cudaMemcpyDefault, c->h2d);
      };
      auto a_rows = [&](int r0) {
        return notrans(ta) ? (const T *)da + r0 : (const T *)da + (size_t)r0 * dla;
      };
      // Block 0 is computed in two row halves: the first half starts as soon as
      // the top rows of A are in, so C starts flowing back while the rest of A
      // is still being copied (the copy-out would otherwise start only after
      // all of A and one block of B had arrived).  The last block is split the
      // same way so that only half of it is computed and copied out after the
      // copy-in has ended.
      const int mh = m >= 512 ? (m / 2) / 256 * 256 : 0;
      const bool split0 = mh > 0 && mh < m;
      auto block_cols = [&](int j, int *j0, int *nj) {
        *j0 = j * cw;
        *nj = (n - *j0 < cw) ? n - *j0 : cw;
      };
      auto b_dev = [&](int j0) {
        return notrans(tb) ? (T *)db + (size_t)j0 * dlb : (T *)db + j0;
      };
      // beta == 0 reads C only to keep a NaN or Inf already there (0 * C):
      // then the host scans C while the copies run, and an all-finite C is
      // zeroed on the device instead of copied in (a quarter of the PCIe
      // bytes).  Any other beta needs C, copied with its block of B.
      const bool scan_c = beta == (T)0 && !is_device_ptr(cm);
      auto copy_c_in = [&](int j0, int nj) {
        return cudaMemcpy2DAsync((T *)dc + (size_t)j0 * dlc, (size_t)dlc * sizeof(T),
                                 cm + (size_t)j0 * ldc, (size_t)ldc * sizeof(T),
                                 (size_t)m * sizeof(T), nj, cudaMemcpyDefault, c->h2d);
      };
      // 1. Queue the copies on the copy-in stream: A's top rows, block 0 of B
      //    (and of C), A's other rows, then the other blocks; ev_in[j] marks
      //    block j (and all of A queued before it) in device memory,
      //    ev_in[PIPE_MAX] the rest of A.
      if (st == B2_OK) e = copy_a_rows(0, split0 ? mh : m);
      for (int j = 0; j < nb && st == B2_OK && e == cudaSuccess; ++j) {
        int j0, nj;
        block_cols(j, &j0, &nj);
        const T *bh = notrans(tb) ? b + (size_t)j0 * ldb : b + j0;
        e = notrans(tb)
                ? cudaMemcpy2DAsync(b_dev(j0), (size_t)dlb * sizeof(T), bh, (size_t)ldb * sizeof(T),
                                    (size_t)k * sizeof(T), nj, cudaMemcpyDefault, c->h2d)
                : cudaMemcpy2DAsync(b_dev(j0), (size_t)dlb * sizeof(T), bh, (size_t)ldb * sizeof(T),
                                    (size_t)nj * sizeof(T), k, cudaMemcpyDefault, c->h2d);
        if (e == cudaSuccess && !scan_c) e = copy_c_in(j0, nj);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_in[j], c->h2d);
        if (j == 0 && split0 && e == cudaSuccess) {
          e = copy_a_rows(mh, m);
          if (e == cudaSuccess) e = cudaEventRecord(c->ev_in[Ctx::PIPE_MAX], c->h2d);
        }
      }
      // 2. Per block, while the copies queued above run: with beta == 0 the
      //    host scans the block's C (an all-finite block is zeroed on the
      //    device; one holding a NaN or Inf is copied in after everything
      //    queued, which is rare), then the block is computed once its copies
      //    are in and its C copied out.  Scanning block by block lets block 0
      //    start before the scan of all of C has finished.
      if (sizeof(T) == 8) ozaki_pipeline_rows(-1, nullptr, 0, 0);
      int issued = 0;
      for (int j = 0; j < nb && st == B2_OK && e == cudaSuccess; ++j) {
        int j0, nj;
        block_cols(j, &j0, &nj);
        const T *bd = b_dev(j0);
        T *cd = (T *)dc + (size_t)j0 * dlc;
        T *ch = cm + (size_t)j0 * ldc;
        if (scan_c && host_all_finite(ch, m, nj, ldc)) {
          e = cudaMemsetAsync(cd, 0, (size_t)dlc * nj * sizeof(T), s);
        } else if (scan_c) {
          e = copy_c_in(j0, nj);
          if (e == cudaSuccess) e = cudaEventRecord(c->ev_c[j], c->h2d);
          if (e == cudaSuccess) e = cudaStreamWaitEvent(s, c->ev_c[j], 0);
        }
        // rows [r0, r1) of block j once copy-in event `ev` has fired
        auto part = [&](int ev, int done, int r0, int r1) {
          cudaError_t pe = cudaStreamWaitEvent(s, c->ev_in[ev], 0);
          if (pe != cudaSuccess) return pe;
          if (sizeof(T) == 8) ozaki_pipeline_rows(j, (const double *)da, m, r0);
          st = run(a_rows(r0), dla, bd, dlb, cd + r0, dlc, r1 - r0, nj, s);
          if (st != B2_OK) return cudaSuccess;
          pe = cudaEventRecord(c->ev_done[done], s);
          if (pe == cudaSuccess) pe = cudaStreamWaitEvent(c->d2h, c->ev_done[done], 0);
          if (pe == cudaSuccess)
            pe = cudaMemcpy2DAsync(ch + r0, (size_t)ldc * sizeof(T), cd + r0,
                                   (size_t)dlc * sizeof(T), (size_t)(r1 - r0) * sizeof(T), nj,
                                   cudaMemcpyDefault, c->d2h);
          return pe;
        };
        if (e != cudaSuccess) break;
        if (j == 0 && split0) {
          e = part(0, 0, 0, mh);
          if (e == cudaSuccess && st == B2_OK) e = part(Ctx::PIPE_MAX, Ctx::PIPE_MAX, mh, m);
        } else if (j == nb - 1 && split0) {
          // the last block in two row halves as well: the first half's copy-out
          // overlaps the second half's compute, halving the exposed tail
          e = part(j, j, 0, mh);
          if (e == cudaSuccess && st == B2_OK) e = part(j, Ctx::PIPE_MAX + 1, mh, m);
        } else {
          e = part(j, j, 0, m);
        }
        if (st != B2_OK) break;
        ++issued;
      }
      if (sizeof(T) == 8) ozaki_pipeline_rows(-1, nullptr, 0, 0);
      if (st == B2_OK && e != cudaSuccess) st = cuda_fail(e, "pipelined staging");
      // Every stream drains before returning, whatever failed.
      cudaError_t e1 = cudaStreamSynchronize(c->h2d);
      cudaError_t e2 = cudaStreamSynchronize(s);
      cudaError_t e3 = cudaStreamSynchronize(c->d2h);
      if (st == B2_OK && e1 != cudaSuccess) st = cuda_fail(e1, "copy-in stream");
      if (st == B2_OK && e2 != cudaSuccess) st = cuda_fail(e2, "stream sync");
      if (st == B2_OK && e3 != cudaSuccess) st = cuda_fail(e3, "copy-out stream");
      (void)issued;
    }
  }
  if (st == B2_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "stream sync");
  }
  st = take_device_error(c, st);
  set_status(st);
  return st;
}

static bool cnotrans(char c) { return c == 'N' || c == 'n' || c == 'R' || c == 'r'; }

// Complex GEMM argument check: matrix rows follow the trans char ('N'/'R'
// keep A as m x k, 'T'/'C'/other make it k x m).
static int check_gemm3m(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc,
                        const void *a, const void *b, const void *c, int *info) {
  return check_gemm(cnotrans(ta) ? 'N' : 'T', cnotrans(tb) ? 'N' : 'T', m, n, k, lda, ldb, ldc,
                    a, b, c, info);
}

template <typename T>
static void gemm3m_dropin(const char *transa, const char *transb, const int *m, const int *n,
                          const int *k, const T *alpha, const T *a, const int *lda, const T *b,
                          const int *ldb, const T *beta, T *c, const int *ldc) {
  if (!transa || !transb || !m || !n || !k || !alpha || !lda || !ldb || !beta || !ldc) {
    set_status(B2_ERR_ARG, 0);
    return;
  }
  const char ta = *transa, tb = *transb;
  const int M = *m, N = *n, K = *k;
  int info = 0;
  int st = check_gemm3m(ta, tb, M, N, K, *lda, *ldb, *ldc, a, b, c, &info);
  if (st != B2_OK) { set_status(st, info); return; }
  if (M == 0 || N == 0) { set_status(B2_OK); return; }
  Ctx *cx = ctx();
  if (!cx) { set_status(B2_ERR_NO_DEVICE); return; }
  cudaStream_t s = cx->stream;
  const T al[2] = {alpha[0], alpha[1]}, be[2] = {beta[0], beta[1]};
  const bool need_ab = K > 0 && !(al[0] == (T)0 && al[1] == (T)0);
  const size_t esz = 2 * sizeof(T);
  if (is_device_ptr(c) && (!need_ab || (is_device_ptr(a) && is_device_ptr(b)))) {
    st = gemm3m_device<T>(ta, tb, M, N, K, al, a, *lda, b, *ldb, be, c, *ldc, s);
  } else {
    const int ra = cnotrans(ta) ? M : K, ca = cnotrans(ta) ? K : M;
    const int rb = cnotrans(tb) ? K : N, cb = cnotrans(tb) ? N : K;
    void *da = nullptr, *db = nullptr, *dc = nullptr;
    int dla = 2, dlb = 2, dlc = 2;
    st = B2_OK;
    if (need_ab) {
      st = stage_in(cx, WS_STAGE_A, a, ra, ca, *lda, esz, &da, &dla, s);
      if (st == B2_OK) st = stage_in(cx, WS_STAGE_B, b, rb, cb, *ldb, esz, &db, &dlb, s);
    }
    if (st == B2_OK) st = stage_in(cx, WS_STAGE_C, c, M, N, *ldc, esz, &dc, &dlc, s);
    if (st == B2_OK)
      st = gemm3m_device<T>(ta, tb, M, N, K, al, (const T *)da, dla, (const T *)db, dlb, be,
                            (T *)dc, dlc, s);
    if (st == B2_OK) st = stage_out(c, *ldc, dc, dlc, M, N, esz, s);
  }
  if (st == B2_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "stream sync");
  }
  st = take_device_error(cx, st);
  set_status(st);
}

template <typename T>
static int gemm3m_ext(char ta, char tb, int m, int n, int k, const T *alpha, const T *A, int lda,
                      const T *B, int ldb, const T *beta, T *C, int ldc, void *stream) {
  int info = 0;
  if (!alpha || !beta) { set_status(B2_ERR_ARG, !alpha ? 6 : 11); return B2_ERR_ARG; }
  int st = check_gemm3m(ta, tb, m, n, k, lda, ldb, ldc, A, B, C, &info);
  if (st != B2_OK) { set_status(st, info); return st; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  const bool need_ab = k > 0 && !(alpha[0] == (T)0 && alpha[1] == (T)0);
  if (m > 0 && n > 0 && (!is_device_ptr(C) || (need_ab && (!is_device_ptr(A) || !is_device_ptr(B))))) {
    set_status(B2_ERR_ARG, !is_device_ptr(C) ? 12 : (!is_device_ptr(A) ? 7 : 9));
    return B2_ERR_ARG;
  }
  st = gemm3m_device<T>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, pick_stream(c, stream));
  set_status(st);
  return st;
}

static bool lsame(char a, char b) { return a == b || a == b + 32; }

// BLAS dtrsm argument check (xerbla positions).
static int check_trsm(char side, char uplo, char transa, char diag, int m, int n, int lda,
                      int ldb, const void *a, const void *b, int *info) {
  const bool left = lsame(side, 'L');
  const int nrowa = left ? m : n;
  *info = 0;
  if (!left && !lsame(side, 'R')) *info = 1;
  else if (!lsame(uplo, 'U') && !lsame(uplo, 'L')) *info = 2;
  else if (!lsame(transa, 'N') && !lsame(transa, 'T') && !lsame(transa, 'C')) *info = 3;
  else if (!lsame(diag, 'U') && !lsame(diag, 'N')) *info = 4;
  else if (m < 0) *info = 5;
  else if (n < 0) *info = 6;
  else if (lda < (nrowa > 1 ? nrowa : 1)) *info = 9;
  else if (ldb < (m > 1 ? m : 1)) *info = 11;
  else if (m > 0 && n > 0 && (!a || !b)) *info = !a ? 8 : 10;
  return *info ? B2_ERR_ARG : B2_OK;
}

// ------------------------------------------------ sharded multi-GPU DGEMM --
// A host-operand DGEMM split over several GPUs of one node: C's columns are
// cut into one contiguous block per listed device and each block runs through
// the drop-in path (copy pipeline, method dispatch) on its own device.  There
// is no exchange between the shards: every device receives A and its columns
// of B and C, so no collective or peer memory access is involved.
//
// Each (device, occurrence) slot has one persistent host thread, so the
// library context of the shard (streams, events, grow-only workspaces) is
// created on its device at the first call and reused by later calls.  The
// threads are detached and idle on a condition variable between calls.
namespace {
struct ShardWorker {
  int device = 0;
  std::mutex mu;
  std::condition_variable cv;
  std::function<int()> task;
  bool busy = false, done = false;
  int result = B2_OK;
};
std::mutex g_shard_mu;                  // one sharded call at a time
std::vector<ShardWorker *> g_shard_workers;  // live until the process exits

void shard_worker_loop(ShardWorker *w) {
  cudaSetDevice(w->device);
  for (;;) {
    std::function<int()> t;
    {
      std::unique_lock<std::mutex> lk(w->mu);
      w->cv.wait(lk, [&] { return w->busy && !w->done; });
      t = w->task;
    }
    const int r = t();
    {
      std::lock_guard<std::mutex> lk(w->mu);
      w->result = r;
      w->done = true;
    }
    w->cv.notify_all();
  }
}

// The occurrence-th worker bound to `device` (created on first use; null
// when the host cannot start another thread).
ShardWorker *shard_worker(int device, int occurrence) {
  int seen = 0;
  for (ShardWorker *w : g_shard_workers)
    if (w->device == device && seen++ == occurrence) return w;
  ShardWorker *w = new ShardWorker();
  w->device = device;
  try {
    std::thread(shard_worker_loop, w).detach();
  } catch (...) {
    delete w;
    return nullptr;
  }
  g_shard_workers.push_back(w);
  return w;
}

// Devices listed in B2_DEVICES ("0,1,2,3"), read once; fewer than two means
// dgemm_ does not shard.
const std::vector<int> &env_devices() {
  static const std::vector<int> devs = [] {
    std::vector<int> v;
    if (const char *e = getenv("B2_DEVICES")) {
      const char *q = e;
      while (*q) {
        char *end = nullptr;
        const long d = strtol(q, &end, 10);
        if (end == q) break;
        if (d >= 0 && d < 1024) v.push_back((int)d);
        q = *end == ',' ? end + 1 : end;
        if (*end != ',') break;
      }
    }
    return v;
  }();
  return devs;
}
}  // namespace

// B2_OK when every listed device exists and is an sm_100-class GPU.
int check_shard_devices(int ndev, const int *devices) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    (void)cudaGetLastError();
    return B2_ERR_NO_DEVICE;
  }
  for (int j = 0; j < ndev; ++j) {
    cudaDeviceProp p;
    if (devices[j] < 0 || devices[j] >= count ||
        cudaGetDeviceProperties(&p, devices[j]) != cudaSuccess || p.major < 10) {
      (void)cudaGetLastError();
      return B2_ERR_ARG;
    }
  }
  return B2_OK;
}

// Runs the sharded product; arguments are already checked (host operands,
// valid devices).  Returns the first failing shard's status, in shard order,
// or B2_ERR_NOMEM when a shard's worker thread cannot be started.
int dgemm_sharded(int ndev, const int *devices, char ta, char tb, int m, int n, int k,
                  double alpha, const double *a, int lda, const double *b, int ldb, double beta,
                  double *c, int ldc, int method, int slices) {
  std::lock_guard<std::mutex> guard(g_shard_mu);
  const int shards = ndev < n ? ndev : n;
  const int base = n / shards, rem = n % shards;
  std::vector<ShardWorker *> ws;
  int st = B2_OK;
  int j0 = 0;
  for (int j = 0; j < shards; ++j) {
    int occ = 0;
    for (int i = 0; i < j; ++i) occ += devices[i] == devices[j];
    ShardWorker *w = shard_worker(devices[j], occ);
    if (!w) {  // no thread for this shard: finish the ones started, then fail
      st = B2_ERR_NOMEM;
      break;
    }
    const int nj = base + (j < rem ? 1 : 0);
    const double *bj = notrans(tb) ? b + (size_t)j0 * ldb : b + j0;
    double *cj = c + (size_t)j0 * ldc;
    {
      std::lock_guard<std::mutex> lk(w->mu);
      w->task = [=]() {
        return gemm_dropin<double>(ta, tb, m, nj, k, alpha, a, lda, bj, ldb, beta, cj, ldc,
                                   [&](const double *A, int la, const double *B, int lb,
                                       double *C, int lc, int mrows, int ncols, cudaStream_t s) {
                                     return dgemm_device(ta, tb, mrows, ncols, k, alpha, A, la,
                                                         B, lb, beta, C, lc, method, slices, s);
                                   });
      };
      w->busy = true;
      w->done = false;
    }
    w->cv.notify_all();
    ws.push_back(w);
    j0 += nj;
  }
  for (ShardWorker *w : ws) {
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [&] { return w->done; });
    w->busy = false;
    if (st == B2_OK && w->result != B2_OK) st = w->result;
  }
  return st;
}

}  // namespace b2

using namespace b2;

extern "C" {

int b2_last_error(void) { return g_status.code; }
int b2_last_info(void) { return g_status.info; }
int b2_version(void) { return 100; }

const char *b2_status_string(int s) {
  switch (s) {
    case B2_OK: return "ok";
    case B2_ERR_ARG: return "invalid argument";
    case B2_ERR_CUDA: return "CUDA runtime error";
    case B2_ERR_NOMEM: return "device allocation failed";
    case B2_ERR_TIMEOUT: return "bounded device wait gave up";
    case B2_ERR_UNSUPPORTED: return "unsupported method or shape";
    case B2_ERR_NO_DEVICE: return "no sm_100 device";
    default: return "unknown status";
  }
}

int b2_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { (void)cudaGetLastError(); return 0; }
  int ok = 0;
  for (int i = 0; i < n; ++i) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, i) == cudaSuccess && p.major >= 10) ++ok;
  }
  return ok;
}

int b2_set_dgemm_method(int method, int slices) {
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  if (!(method == B2_METHOD_FP64 || method == B2_METHOD_OZAKI || method == B2_METHOD_AUTO ||
        method == B2_METHOD_DEFAULT) || slices < 0 || slices > B2_MAX_MODULI)
    return B2_ERR_ARG;
  c->dgemm_method = method == B2_METHOD_DEFAULT ? B2_METHOD_FP64 : method;
  c->dgemm_slices = slices;
  return B2_OK;
}

int b2_set_sgemm_method(int method) {
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  if (!(method == B2_METHOD_FP32 || method == B2_METHOD_TF32 || method == B2_METHOD_TF32X3 ||
        method == B2_METHOD_BF16X3 || method == B2_METHOD_DEFAULT))
    return B2_ERR_ARG;
  c->sgemm_method = method == B2_METHOD_DEFAULT ? B2_METHOD_FP32 : method;
  return B2_OK;
}

void dgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
            const double *alpha, const double *a, const int *lda, const double *b,
            const int *ldb, const double *beta, double *c, const int *ldc) {
  if (!transa || !transb || !m || !n || !k || !alpha || !lda || !ldb || !beta || !ldc) {
    set_status(B2_ERR_ARG, 0);
    return;
  }
  const char ta = *transa, tb = *transb;
  const double al = *alpha, be = *beta;
  // B2_DEVICES lists two or more GPUs: a large product on host operands is
  // sharded over them by columns of C (checked arguments only).
  const std::vector<int> &devs = env_devices();
  if (devs.size() >= 2 && 2.0 * *m * (double)*n * *k >= 4294967296.0 && *n >= (int)devs.size() &&
      arg_mode() == B2_ARGS_BLAS) {
    int info = 0;
    if (check_gemm(ta, tb, *m, *n, *k, *lda, *ldb, *ldc, a, b, c, &info) == B2_OK &&
        !is_device_ptr(a) && !is_device_ptr(b) && !is_device_ptr(c)) {
      Ctx *cx = ctx();
      if (!cx) { set_status(B2_ERR_NO_DEVICE); return; }
      const int dst = check_shard_devices((int)devs.size(), devs.data());
      if (dst != B2_OK) {  // a device named in B2_DEVICES is missing: fail loudly
        if (getenv("B2_VERBOSE")) fprintf(stderr, "b2blas: B2_DEVICES names an unusable device\n");
        set_status(dst, 0);
        return;
      }
      set_status(dgemm_sharded((int)devs.size(), devs.data(), ta, tb, *m, *n, *k, al, a, *lda, b,
                               *ldb, be, c, *ldc, cx->dgemm_method, cx->dgemm_slices));
      return;
    }
  }
  gemm_dropin<double>(ta, tb, *m, *n, *k, al, a, *lda, b, *ldb, be, c, *ldc,
                      [&](const double *A, int la, const double *B, int lb, double *C, int lc,
                          int mrows, int ncols, cudaStream_t s) {
                        return dgemm_device(ta, tb, mrows, ncols, *k, al, A, la, B, lb, be, C, lc,
                                            B2_METHOD_DEFAULT, 0, s);
                      });
}

void sgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
            const float *alpha, const float *a, const int *lda, const float *b, const int *ldb,
            const float *beta, float *c, const int *ldc) {
  if (!transa || !transb || !m || !n || !k || !alpha || !lda || !ldb || !beta || !ldc) {
    set_status(B2_ERR_ARG, 0);
    return;
  }
  const char ta = *transa, tb = *transb;
  const float al = *alpha, be = *beta;
  gemm_dropin<float>(ta, tb, *m, *n, *k, al, a, *lda, b, *ldb, be, c, *ldc,
                     [&](const float *A, int la, const float *B, int lb, float *C, int lc,
                         int mrows, int ncols, cudaStream_t s) {
                       return sgemm_device(ta, tb, mrows, ncols, *k, al, A, la, B, lb, be, C, lc,
                                           B2_METHOD_DEFAULT, s);
                     });
}

void SGEMM_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
            const float *alpha, const float *a, const int *lda, const float *b, const int *ldb,
            const float *beta, float *c, const int *ldc) {
  sgemm_(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void zgemm3m_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
              const double *alpha, const double *a, const int *lda, const double *b,
              const int *ldb, const double *beta, double *c, const int *ldc) {
  gemm3m_dropin<double>(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void cgemm3m_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
              const float *alpha, const float *a, const int *lda, const float *b,
              const int *ldb, const float *beta, float *c, const int *ldc) {
  gemm3m_dropin<float>(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

int b2_zgemm3m(char transa, char transb, int m, int n, int k, const double *alpha,
               const double *A, int lda, const double *B, int ldb, const double *beta, double *C,
               int ldc, void *stream) {
  return gemm3m_ext<double>(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}

int b2_cgemm3m(char transa, char transb, int m, int n, int k, const float *alpha,
               const float *A, int lda, const float *B, int ldb, const float *beta, float *C,
               int ldc, void *stream) {
  return gemm3m_ext<float>(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}

void dtrsm_(const char *side, const char *uplo, const char *transa, const char *diag,
            const int *m, const int *n, const double *alpha, const double *a, const int *lda,
            double *b, const int *ldb) {
  if (!side || !uplo || !transa || !diag || !m || !n || !alpha || !lda || !ldb) {
    set_status(B2_ERR_ARG, 0);
    return;
  }
  const int M = *m, N = *n;
  int info = 0;
  int st = check_trsm(*side, *uplo, *transa, *diag, M, N, *lda, *ldb, a, b, &info);
  if (st != B2_OK) { set_status(st, info); return; }
  if (M == 0 || N == 0) { set_status(B2_OK); return; }
  Ctx *cx = ctx();
  if (!cx) { set_status(B2_ERR_NO_DEVICE); return; }
  cudaStream_t s = cx->stream;
  const int na = lsame(*side, 'L') ? M : N;
  if (is_device_ptr(b) && is_device_ptr(a)) {
    st = dtrsm_device(*side, *uplo, *transa, *diag, M, N, *alpha, a, *lda, b, *ldb,
                      cx->dgemm_method, 0, s);
  } else {
    void *da = nullptr, *db = nullptr;
    int dla = 2, dlb = 2;
    st = stage_in(cx, WS_TRSM, a, na, na, *lda, sizeof(double), &da, &dla, s);
    if (st == B2_OK) st = stage_in(cx, WS_STAGE_C, b, M, N, *ldb, sizeof(double), &db, &dlb, s);
    if (st == B2_OK)
      st = dtrsm_device(*side, *uplo, *transa, *diag, M, N, *alpha, (const double *)da, dla,
                        (double *)db, dlb, cx->dgemm_method, 0, s);
    if (st == B2_OK) st = stage_out(b, *ldb, db, dlb, M, N, sizeof(double), s);
  }
  if (st == B2_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "stream sync");
  }
  st = take_device_error(cx, st);
  set_status(st);
}

int b2_dtrsm(char side, char uplo, char transa, char diag, int m, int n, double alpha,
             const double *A, int lda, double *B, int ldb, int update_method, int block,
             void *stream) {
  int info = 0;
  int st = check_trsm(side, uplo, transa, diag, m, n, lda, ldb, A, B, &info);
  if (st != B2_OK) { set_status(st, info); return st; }
  if (m == 0 || n == 0) { set_status(B2_OK); return B2_OK; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  if (!is_device_ptr(B) || !is_device_ptr(A)) {
    set_status(B2_ERR_ARG, !is_device_ptr(A) ? 8 : 10);
    return B2_ERR_ARG;
  }
  if (!(update_method == B2_METHOD_DEFAULT || update_method == B2_METHOD_FP64 ||
        update_method == B2_METHOD_OZAKI || update_method == B2_METHOD_AUTO) ||
      block < 0 || block > 128) {
    set_status(B2_ERR_ARG, 12);
    return B2_ERR_ARG;
  }
  st = dtrsm_device(side, uplo, transa, diag, m, n, alpha, A, lda, B, ldb, update_method, block,
                    pick_stream(c, stream));
  set_status(st);
  return st;
}

int b2_gemm_grouped(int count, const b2_gemm_problem *problems, void *stream) {
  if (count < 0 || (count > 0 && !problems)) { set_status(B2_ERR_ARG, 0); return B2_ERR_ARG; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  int info = 0;
  const int st = grouped_device(count, problems, pick_stream(c, stream), &info);
  set_status(st, info);
  return st;
}

int b2_grouped_plan_create(int count, const b2_gemm_problem *problems, void **plan) {
  if (count < 0 || (count > 0 && !problems) || !plan) { set_status(B2_ERR_ARG, 0); return B2_ERR_ARG; }
  int info = 0;
  const int st = grouped_plan_create(count, problems, plan, &info);
  set_status(st, info);
  return st;
}

int b2_grouped_plan_launch(void *plan, void *stream) {
  if (!plan) { set_status(B2_ERR_ARG, 1); return B2_ERR_ARG; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  const int st = grouped_plan_launch(plan, pick_stream(c, stream));
  set_status(st);
  return st;
}

int b2_grouped_plan_destroy(void *plan) {
  if (!plan) return B2_OK;
  return grouped_plan_destroy(plan);
}

int b2_dgemm(char transa, char transb, int m, int n, int k, double alpha, const double *A,
             int lda, const double *B, int ldb, double beta, double *C, int ldc, int method,
             int slices, void *stream) {
  int info = 0;
  int st = check_gemm(transa, transb, m, n, k, lda, ldb, ldc, A, B, C, &info);
  if (st != B2_OK) { set_status(st, info); return st; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  if (m > 0 && n > 0 &&
      (!is_device_ptr(C) || (k > 0 && alpha != 0.0 && (!is_device_ptr(A) || !is_device_ptr(B))))) {
    set_status(B2_ERR_ARG, !is_device_ptr(C) ? 12 : (!is_device_ptr(A) ? 7 : 9));
    return B2_ERR_ARG;
  }
  st = dgemm_device(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, method, slices,
                    pick_stream(c, stream));
  set_status(st);
  return st;
}

int b2_dgemm_multi(int ndev, const int *devices, char transa, char transb, int m, int n, int k,
                   double alpha, const double *A, int lda, const double *B, int ldb, double beta,
                   double *C, int ldc, int method, int slices) {
  int info = 0;
  int st = check_gemm(transa, transb, m, n, k, lda, ldb, ldc, A, B, C, &info);
  if (st != B2_OK) { set_status(st, info); return st; }
  if (ndev < 1 || ndev > 64 || !devices ||
      !(method == B2_METHOD_DEFAULT || method == B2_METHOD_FP64 || method == B2_METHOD_OZAKI ||
        method == B2_METHOD_AUTO) ||
      slices < 0 || slices > B2_MAX_MODULI) {
    set_status(B2_ERR_ARG, 0);
    return B2_ERR_ARG;
  }
  st = check_shard_devices(ndev, devices);
  if (st != B2_OK) { set_status(st, 0); return st; }
  // host memory only: a shard's kernels never read another GPU's memory
  if (is_device_ptr(C) || is_device_ptr(A) || is_device_ptr(B)) {
    set_status(B2_ERR_ARG, is_device_ptr(C) ? 12 : (is_device_ptr(A) ? 7 : 9));
    return B2_ERR_ARG;
  }
  if (m == 0 || n == 0) { set_status(B2_OK); return B2_OK; }
  if (method == B2_METHOD_DEFAULT) {
    Ctx *c = ctx();
    if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
    method = c->dgemm_method;
    if (slices == 0) slices = c->dgemm_slices;
  }
  st = dgemm_sharded(ndev, devices, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                     method, slices);
  set_status(st);
  return st;
}

int b2_sgemm(char transa, char transb, int m, int n, int k, float alpha, const float *A,
             int lda, const float *B, int ldb, float beta, float *C, int ldc, int method,
             void *stream) {
  int info = 0;
  int st = check_gemm(transa, transb, m, n, k, lda, ldb, ldc, A, B, C, &info);
  if (st != B2_OK) { set_status(st, info); return st; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  if (m > 0 && n > 0 &&
      (!is_device_ptr(C) || (k > 0 && alpha != 0.0f && (!is_device_ptr(A) || !is_device_ptr(B))))) {
    set_status(B2_ERR_ARG, !is_device_ptr(C) ? 12 : (!is_device_ptr(A) ? 7 : 9));
    return B2_ERR_ARG;
  }
  st = sgemm_device(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, method,
                    pick_stream(c, stream));
  set_status(st);
  return st;
}

int b2_dgemm_dd(char transa, char transb, int m, int n, int k, double alpha, const double *A,
                int lda, const double *B, int ldb, double beta, const double *C0, int ldc,
                double *Chi, double *Clo, int ldo, void *stream) {
  int info = 0;
  int st = check_gemm(transa, transb, m, n, k, lda, ldb, C0 ? ldc : (m > 1 ? m : 1), A, B, Chi,
                      &info);
  if (st == B2_OK && ldo < (m > 1 ? m : 1)) { st = B2_ERR_ARG; info = 16; }
  if (st != B2_OK) { set_status(st, info); return st; }
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  st = dgemm_dd(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc, Chi, Clo, ldo,
                pick_stream(c, stream));
  set_status(st);
  return st;
}

int b2_dgemm_error(char transa, char transb, int m, int n, int k, double alpha,
                   const double *A, int lda, const double *B, int ldb, double beta,
                   const double *C0, const double *C, int ldc, double *normwise,
                   double *maxelem, void *stream) {
  Ctx *c = ctx();
  if (!c) { set_status(B2_ERR_NO_DEVICE); return B2_ERR_NO_DEVICE; }
  if (m <= 0 || n <= 0) {
    if (normwise) *normwise = 0.0;
    if (maxelem) *maxelem = 0.0;
    set_status(B2_OK);
    return B2_OK;
  }
  cudaStream_t s = pick_stream(c, stream);
  double *ref = (double *)workspace(c, WS_ERR, (size_t)m * n * sizeof(double) + 64);
  if (!ref) { set_status(B2_ERR_NOMEM); return B2_ERR_NOMEM; }
  double *acc = ref + (size_t)m * n;
  int st = dgemm_dd(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc, ref, nullptr, m, s);
  if (st == B2_OK) st = error_stats(m, n, C, ldc, ref, m, acc, s);
  double h[4] = {0, 0, 0, 0};
  if (st == B2_OK) {
    cudaError_t e = cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "error stats");
  }
  if (st == B2_OK) {
    if (normwise) *normwise = h[1] > 0 ? sqrt(h[0] / h[1]) : sqrt(h[0]);
    if (maxelem) *maxelem = h[3] > 0 ? h[2] / h[3] : h[2];
  }
  set_status(st);
  return st;
}

int b2_set_arg_mode(int mode) {
  if (mode != B2_ARGS_BLAS && mode != B2_ARGS_OPENBLAS) return -1;
  const int prev = arg_mode();
  g_arg_mode.store(mode);
  return prev;
}

int b2_device_error(int clear) {
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    (void)cudaGetLastError();
    return B2_ERR_CUDA;
  }
  int v = 0;
  if (c->derr_host) {
    v = *(volatile int *)c->derr_host;
    if (clear) *(volatile int *)c->derr_host = 0;
    return v;
  }
  if (cudaMemcpy(&v, c->derr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    (void)cudaGetLastError();
    return B2_ERR_CUDA;
  }
  if (clear && cudaMemset(c->derr, 0, 64) != cudaSuccess) (void)cudaGetLastError();
  return v;
}

int b2_test_bounded_wait(long long wait_ns, int withhold_launches) {
  if (withhold_launches < 0) return B2_ERR_ARG;
  unsigned long long w = wait_ns <= 0 ? umma_default_wait_ns() : (unsigned long long)wait_ns;
  if (w < 100000ull) w = 100000ull;               // 0.1 ms
  if (w > 10000000000ull) w = 10000000000ull;     // 10 s
  umma_set_wait(w, withhold_launches);
  return B2_OK;
}

}  // extern "C"
