// screen.cu -- TMA tensor maps of the screen operands and the
// screened-values test hook.
//
// The screened pipeline of one group of jobs is (see api.cu for the order):
//   screen prep   operands + binary64 error statistics (screen_prep.cu)
//   band          keep band 2E_i per row
//   screen gemm   tcgen05 U U^T, threshold pass over a column sample
//   threshold     tau1 per row (rerank.cu)
//   screen gemm   tcgen05 U U^T, emission pass within tau1 + band
//   rerank        exact distances of the survivors + select (rerank.cu)
//   fallback      plain exact kernel over the rows the screen could not bound
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

static thread_local float *g_debug_dump = nullptr;

float *debug_dump_pointer() { return g_debug_dump; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_fn(EncodeTiledFn *out) {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (err == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    if (!fn) return set_error(HM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable (%s)", cudaGetErrorString(err));
    *out = fn;
    return HM_OK;
}

// 2-D map over a rows x kpmax operand, box = one 128-byte K slice x
// `box_rows` rows, 128-byte swizzle; rows past the end read as zeros.
int make_operand_map(CUtensorMap *m, void *base, uint64_t rows, uint32_t kpmax, uint32_t elem_bytes,
                     uint32_t kslice, uint32_t box_rows) {
    EncodeTiledFn enc;
    HM_TRY(encode_fn(&enc));
    const cuuint64_t dims[2] = {kpmax, rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kpmax * elem_bytes};
    const cuuint32_t box[2] = {kslice, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(m, elem_bytes == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                           2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(HM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return HM_OK;
}

}  // namespace hm

using namespace hm;

extern "C" {

int hm_debug_set_screen_dump(float *d_out) {
    g_debug_dump = d_out;
    return HM_OK;
}

}  // extern "C"
