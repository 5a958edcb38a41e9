// stk_umma.cuh -- host interface of the sm_100a tensor-core (tcgen05) GEMM used by
// the mixed-precision M2L: C (=|+=) A B in FP32 accuracy from TF32 tensor-core
// products (3xTF32 split with a per-K-block FP32 drain, see stk_umma.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace stk {

// A K-major operand of the 3xTF32 GEMM (tf32_split_value): hi and lo TF32 parts
// of each FP32 value, both [rows][ld] row-major with K contiguous, ld a multiple
// of 4 and rows x K the used extent.
struct Tf32Split {
    const float *hi = nullptr, *lo = nullptr;
    int ld = 0;
};

// C[m + n ldc] (beta = 0: =, 1: +=) sum_k A[m][k] B[n][k], m < M, n < N, k < K.
// A: M x K, B: N x K (K-major: B holds the columns of the product's right factor).
// Pointers 16-byte aligned, lda / ldb multiples of 4 (TMA rows).  err: device int
// set non-zero when a pipeline wait gave up (the kernel then stops early).
cudaError_t umma_gemm_3xtf32(int M, int N, int K, Tf32Split A, Tf32Split B, float *C, int ldc, int beta, int *err,
                             cudaStream_t s);

// A K-major operand as one 2-D array of rows: rows x ld floats (ld a multiple of 4),
// of which the first k columns are read (the tensor map zero-fills columns >= k and
// rows >= rows).
struct Tf32Rows {
    const float *hi = nullptr, *lo = nullptr;
    int rows = 0, k = 0, ld = 0;
};

// One 128 x 128 output tile of a grouped GEMM: out[m][n] = sum_{kk < K}
// A[a_row + m][kk] B[b_row + n][kk]; rows m < m_store, columns n < n_valid are written
// to C[c_off + n ldc + m] (0 for rows m >= m_valid), split into TF32 hi / lo parts
// (C, C_lo) when C_lo is given.
struct GroupTile {
    int a_row, b_row, K, m_valid, m_store, n_valid, ldc, pad_;
    long long c_off;
};

// Many tiles, each of its own small GEMM, in one launch (one CTA per tile; the same
// 3xTF32 pipeline as umma_gemm_3xtf32).  tiles: device array of ntiles entries.
cudaError_t umma_grouped_3xtf32(Tf32Rows A, Tf32Rows B, const GroupTile *tiles, int ntiles, float *C, float *C_lo,
                                int *err, cudaStream_t s);

// v = hi + lo to ~2^-24 relative with both parts exact in TF32: hi = v rounded to
// TF32 (to nearest, ties away), lo = (v - hi) rounded to TF32 (v - hi is exact in FP32)
__device__ __forceinline__ void tf32_split_value(float v, float &hi, float &lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
    const float r = v - __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
    hi = __uint_as_float(h);
    lo = __uint_as_float(l);
}

// hi / lo parts of x (n values), tf32_split_value
cudaError_t tf32_split(const float *x, long long n, float *hi, float *lo, cudaStream_t s);

// Whether the tensor-core path can run here (sm_100 device, driver entry point found).
bool umma_available();

}  // namespace stk
