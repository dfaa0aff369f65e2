// Tensor-map encoding (tmap.h).
#include "tmap.h"

#include <cudaTypedefs.h>

#include <mutex>
#include <stdexcept>
#include <string>

namespace fpm {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::string why;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
            why = std::string("cuTensorMapEncodeTiled is not available: ") + cudaGetErrorString(e);
            return;
        }
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw std::runtime_error(why);
    return fn;
}

}  // namespace

CUtensorMap make_tmap_u32(const void* base, uint64_t rows, uint64_t cols, uint64_t pitch, uint32_t box_rows,
                          uint32_t box_cols, TmaSwizzle swizzle) {
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (pitch & 3) || pitch < cols) {
        throw std::runtime_error("tensor map: base must be 16-byte aligned and the pitch a multiple of 4 words");
    }
    CUtensorMap m;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {pitch * sizeof(uint32_t)};
    const cuuint32_t box[2] = {box_cols, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 swizzle == TmaSwizzle::k128B ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        throw std::runtime_error("tensor map rejected (CUresult " + std::to_string(static_cast<int>(r)) + ") for " +
                                 std::to_string(rows) + " x " + std::to_string(cols) + " words, box " +
                                 std::to_string(box_rows) + " x " + std::to_string(box_cols));
    }
    return m;
}

}  // namespace fpm
