// Host side of the TMA helpers: tensor-map encoding through the driver entry
// point that the runtime exposes (no link against the driver library).
#include "helm_tma.cuh"

#include <mutex>

namespace helm {

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder()
{
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

}  // namespace

static bool encode_f64(CUtensorMap* m, int rank, const void* base, const uint64_t* dims, const uint64_t* strides,
                       const uint32_t* box)
{
    EncodeTiled fn = encoder();
    if (!fn || !base || (reinterpret_cast<uintptr_t>(base) & 15) || ((box[0] * 8u) & 15)) return false;
    cuuint64_t d[3], s[2];
    cuuint32_t b[3], e[3];
    for (int i = 0; i < rank; ++i) {
        if (box[i] == 0 || box[i] > 256 || dims[i] == 0) return false;
        d[i] = dims[i];
        b[i] = box[i];
        e[i] = 1;
        if (i + 1 < rank) {
            if (strides[i] & 15) return false;
            s[i] = strides[i];
        }
    }
    CUtensorMap tmp;
    const CUresult r = fn(&tmp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void*>(base), d, s, b,
                          e, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    *m = tmp;
    return true;
}

bool encode_tmap_f64_3d(CUtensorMap* m, const void* base, const uint64_t dims[3], const uint64_t strides[2],
                        const uint32_t box[3])
{
    return encode_f64(m, 3, base, dims, strides, box);
}

bool encode_tmap_f64_2d(CUtensorMap* m, const void* base, const uint64_t dims[2], const uint64_t strides[1],
                        const uint32_t box[2])
{
    return encode_f64(m, 2, base, dims, strides, box);
}

}  // namespace helm
