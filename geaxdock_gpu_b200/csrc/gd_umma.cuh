/*
 * gd_umma.cuh -- BF16 tensor-core GEMM of the surrogate's training on the fifth-generation
 * tensor cores (tcgen05.mma, FP32 accumulator in tensor memory, operands staged by TMA with the
 * 128-byte swizzle), with the epilogues the network's forward and backward passes need.
 *
 *   C(m, n) = sum_k A(m, k) B(n, k),   k over one chunk of K per grid z (split-K)
 *
 * Each operand is a row-major BF16 matrix in global memory, read either K-major (its rows are
 * the output rows, its columns the reduction: X, activations, dZ, W for dZ W^T) or MN-major
 * (its rows are the reduction, its columns the output: W for X W, activations and dZ for the
 * weight gradients, where the batch is the reduction). Rows and columns past the matrix read as
 * zero (TMA out-of-bounds fill).
 */
#ifndef GD_UMMA_CUH
#define GD_UMMA_CUH

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace gd {

struct UmmaOperand {
  const __nv_bfloat16 *p;
  int rows, cols;  /* the row-major matrix in global memory (cols: the contiguous dimension) */
  int mn_major;    /* 1: rows = reduction, cols = output; 0: rows = output, cols = reduction */
};

enum UmmaEpi {
  UMMA_FWD = 0,   /* Z = C + bias[n] (stored when Z), Ob = bf16(SiLU(Z)) */
  UMMA_DGRAD = 1, /* Ob = bf16(C SiLU'(Zin)); with colsum: colsum[m tile][n] = sum of the
                     tile's rows of Ob (the bias gradient of the layer below, per 128 rows) */
  UMMA_F32 = 2    /* Of = C (trans: Of[n][m]); grid z writes Of + z split_stride */
};

struct UmmaEpilogue {
  int kind;
  const float *bias;
  float *Z;
  const float *Zin;
  __nv_bfloat16 *Ob;
  float *Of;
  float *colsum;
  int ldo;
  int trans;
  size_t split_stride;
};

/* C[M][N] over K per split (K <= 256, a multiple of 16; K-major operands are read whole, so
 * splits > 1 needs both operands MN-major), `splits` chunks of K along the reduction. err (a
 * device int) receives a nonzero code if a bounded wait of the kernel ran out. 0 on success,
 * < 0 on a launch or tensor-map error. */
int umma_gemm(const UmmaOperand &A, const UmmaOperand &B, int M, int N, int K, int splits,
              const UmmaEpilogue &e, int *err, cudaStream_t s);

}  // namespace gd

#endif
