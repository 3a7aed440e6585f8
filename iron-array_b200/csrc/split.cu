// Split-precision forms (filled in by the Ozaki INT8 and 3xBF16 kernels).
#include "common.cuh"

namespace iab {

int gemm_f64_ozaki(int64_t, int64_t, int64_t, const double *, int64_t, const double *, int64_t, double *, int64_t, int,
                   cudaStream_t)
{
    return -1;
}

int gemm_f32_bf16x3(int64_t, int64_t, int64_t, const float *, int64_t, const float *, int64_t, float *, int64_t,
                    cudaStream_t)
{
    return -1;
}

}  // namespace iab
