// umma.cu -- host side of the tcgen05 engine: TMA descriptor encoding.
//
// cuTensorMapEncodeTiled is a driver API entry point; it is fetched through
// the runtime (cudaGetDriverEntryPoint) so the library needs no -lcuda.
#include <cudaTypedefs.h>

#include "umma.cuh"

namespace b2 {
namespace umma {

std::atomic<unsigned long long> g_wait_ns{B2_WAIT_NS};
std::atomic<int> g_withhold{0};

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      (void)cudaGetLastError();
  }
  return fn;
}

int make_kmajor_map(CUtensorMap *map, int kind, const void *base, long long kelems, long long rows,
                    long long nbatch, long long row_bytes, long long plane_bytes, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return B2_ERR_CUDA;
  if (((uintptr_t)base & 15) || (row_bytes & 15) || (plane_bytes & 15) || box_rows < 1 ||
      box_rows > 256)
    return B2_ERR_ARG;
  const CUtensorMapDataType dt = is_int8(kind)      ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : kind == KIND_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                     : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  cuuint64_t dims[3] = {(cuuint64_t)kelems, (cuuint64_t)rows, (cuuint64_t)nbatch};
  cuuint64_t strides[2] = {(cuuint64_t)row_bytes, (cuuint64_t)plane_bytes};
  cuuint32_t box[3] = {(cuuint32_t)(KBLOCK_BYTES / elem_bytes(kind)), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? B2_OK : B2_ERR_CUDA;
}

}  // namespace umma

unsigned long long umma_default_wait_ns() { return umma::B2_WAIT_NS; }
void umma_set_wait(unsigned long long wait_ns, int withhold_launches) {
  umma::g_wait_ns.store(wait_ns);
  umma::g_withhold.store(withhold_launches);
}

}  // namespace b2
