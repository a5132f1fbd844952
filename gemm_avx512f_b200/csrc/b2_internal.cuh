// b2_internal.cuh -- shared declarations of libb2blas.so (not installed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/b2blas.h"

namespace b2 {

// ---------------------------------------------------------------- status --
struct Status {
  int code = B2_OK;
  int info = 0;
};

#define B2_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::b2::cuda_fail(_e, #expr); \
  } while (0)

int cuda_fail(cudaError_t e, const char *what);  // records, returns B2_ERR_CUDA

// ------------------------------------------------------------- context --
// One per host thread: the device, a non-blocking stream, grow-only device
// workspaces (one per slot so nested users do not alias), and the device
// error word written by kernels whose bounded waits gave up.
enum WsSlot {
  WS_STAGE_A = 0, WS_STAGE_B, WS_STAGE_C,   // host-pointer staging
  WS_OZ_X, WS_OZ_Y, WS_OZ_R, WS_OZ_SCALE,   // Ozaki slices / residues / exponents
  WS_SPLIT_X, WS_SPLIT_Y,                   // SGEMM split planes
  WS_TRSM, WS_TRSM_INV, WS_TRSM_TMP, WS_3M, WS_GROUP, WS_ERR, WS_MISC,
  WS_KABI_A, WS_KABI_B, WS_KABI_D,         // kernel-ABI unpacked panels / 3M product
  WS_GROUP2,                                // second descriptor slot of one-shot grouped calls
  WS_COUNT
};

struct Ctx {
  int device = -1;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  cudaStream_t stream = nullptr;
  void *ws[WS_COUNT] = {};
  size_t ws_bytes[WS_COUNT] = {};
  int *derr = nullptr;        // error word the kernels write (device address)
  int *derr_host = nullptr;   // the same word seen from the host when it is mapped
                              // pinned memory (then no copy is needed to read it)
  void *pinned = nullptr;     // small pinned scratch for host reads
  void *pinned_dev = nullptr; // its device address (kernels store to it directly), or null
  int dgemm_method = B2_METHOD_FP64;
  int dgemm_slices = 0;
  int sgemm_method = B2_METHOD_FP32;
  int fp64_override = 0;      // non-zero: use fp64_cfg for every FP64 GEMM
  // Host-operand pipeline of the drop-in GEMMs: copy-in and copy-out streams
  // and one (copied-in, computed) event pair per column block.
  static constexpr int PIPE_MAX = 32;
  static constexpr int PIPE_EVENTS = PIPE_MAX + 2;  // + the second row halves of the first and last blocks
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in[PIPE_EVENTS] = {}, ev_done[PIPE_EVENTS] = {}, ev_c[PIPE_EVENTS] = {};
  cudaEvent_t plan_ev = nullptr;  // marks the host store of the last Ozaki modulus count
  // Overlapped Ozaki schedule (created at its first use): the INT8 GEMMs run
  // on a high-priority stream while the slicing and reconstruction of other
  // column blocks run beside them on an auxiliary stream.
  // Pinned bounce buffers for pageable (malloc'ed) host operands, created at
  // their first use: host threads copy through them while the DMA of the
  // other one runs.
  static constexpr size_t BOUNCE_BYTES = 64ull << 20;
  void *bounce[2] = {nullptr, nullptr};
  cudaEvent_t bounce_ev[2] = {nullptr, nullptr};
  static constexpr int OZ_EVENTS = 2 * 16 + 3;  // per block: sliced, multiplied; fork, 2 joins (the last two also join the norm passes)
  cudaStream_t oz_gemm = nullptr, oz_aux = nullptr;
  cudaEvent_t oz_ev[OZ_EVENTS] = {};
  // One-shot grouped calls alternate two descriptor slots (device workspace
  // WS_GROUP / WS_GROUP2, pinned host staging, and an event after the launch
  // that last read them), so one call's descriptors are built and uploaded
  // while the previous call's kernel runs.
  void *grp_host[2] = {nullptr, nullptr};
  size_t grp_host_bytes[2] = {0, 0};
  cudaEvent_t grp_ev[2] = {nullptr, nullptr};
  int grp_next = 0;
};
// The two streams and the events of the overlapped Ozaki schedule (false when
// they cannot be created; the caller then runs the plain schedule).
bool ozaki_overlap_streams(Ctx *c);

Ctx *ctx();                          // initialises on first use; nullptr if no device
// Wait limit of the tensor-core engines' bounded waits and the number of
// launches that withhold their first copy (test hook; umma.cu).
unsigned long long umma_default_wait_ns();
void umma_set_wait(unsigned long long wait_ns, int withhold_launches);
// Reads (and clears) the error word after the caller's stream has been
// synchronised: B2_ERR_TIMEOUT when a bounded device wait gave up, else st.
int take_device_error(Ctx *c, int st);
void *workspace(Ctx *c, int slot, size_t bytes);  // nullptr on allocation failure
// At least `count` per-tile arrival counters, all zero (zeroed on `s` whenever
// the array is (re)allocated; the kernels that use them leave them at zero).
cudaStream_t pick_stream(Ctx *c, void *user_stream);

// ------------------------------------------------------------- kernels --
// Every launcher takes device pointers, enqueues on `s` and returns a
// b2_status.  Dimensions are validated by the API layer.

// Plain FP64 GEMM on the DMMA tensor-core path (dgemm_fp64.cu).
struct Fp64Cfg {
  int tile = 0;    // 0: 128x128, 1: 128x64, 2: 64x64
  int mmak = 4;    // DMMA K shape: 4, 8 or 16
  int split_k = 1; // >1: K split across CTAs, reduced in FP64 workspace
};
int dgemm_fp64(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
               const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s,
               const Fp64Cfg *cfg);
Fp64Cfg fp64_default_cfg(int m, int n, int k, int sm_count);
Fp64Cfg &fp64_override_cfg();

// C <- beta*C (reference semantics: only called when beta != 1).
int scale_matrix_d(int m, int n, double beta, double *C, int ldc, cudaStream_t s);
int scale_matrix_s(int m, int n, float beta, float *C, int ldc, cudaStream_t s);

// Double-double GEMM (dd_gemm.cu).
int dgemm_dd(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
             const double *B, int ldb, double beta, const double *C0, int ldc, double *Chi,
             double *Clo, int ldo, cudaStream_t s);
// Error reduction of C vs Chi: sums ||C-Chi||^2, ||Chi||^2, max|C-Chi|, max|Chi| into out[4].
int error_stats(int m, int n, const double *C, int ldc, const double *Ref, int ldr, double *out,
                cudaStream_t s);

}  // namespace b2
