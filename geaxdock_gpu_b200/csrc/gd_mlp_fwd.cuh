/*
 * gd_mlp_fwd.cuh -- the surrogate's forward pass over FR rows held in shared memory, as device
 * code shared by the stand-alone forward kernel (gd_mlp.cu) and the delayed-acceptance front
 * kernel (gd_da.cu).
 *
 * One CTA of 8 warps: three BF16 tensor-core layers (16 x 16 x 16 warp MMA, FP32 accumulate)
 * whose accumulators are staged through shared memory for bias + SiLU, then the output dot
 * product. Weight fragments come straight from global memory (L2-resident). Per output element
 * the MMA sequence, the bias/SiLU arithmetic and the output reduction order are those of the
 * layer-by-layer kernels, so every path gives the same bits.
 */
#ifndef GD_MLP_FWD_CUH
#define GD_MLP_FWD_CUH

#include <mma.h>

#include "gd_mlp.cuh"

namespace gd {
namespace fwd {

using bf16 = __nv_bfloat16;

constexpr int FR = 32; /* rows per CTA (a multiple of 16): short per-CTA chains, many CTAs */
constexpr int RT = FR / 16; /* 16-row tiles */

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }

template <int NT> /* 16-column tiles per warp: H = 128 * NT */
struct Dims {
  static constexpr int H = 128 * NT, LDX = GD_MLP_IN + 8, LDA = H + 8, LDS = H + 4;
  static constexpr size_t xs_bytes = (size_t)FR * LDX * 2;
  static constexpr size_t smem = xs_bytes + (size_t)FR * LDA * 2 + (size_t)FR * LDS * 4;
};

template <int NT>
__device__ __forceinline__ void layer(const bf16 *A, int lda, int K, const bf16 *__restrict__ W,
                                      const float *__restrict__ bias, bf16 *act, float *stg,
                                      int warp, int tid) {
  using namespace nvcuda;
  using D = Dims<NT>;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[RT][NT];
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) wmma::fill_fragment(acc[i][j], 0.0f);
  /* the weight fragments of KB k-steps are requested together (one L2 round trip per batch
   * instead of one per k-step); the MMA order per output element is unchanged */
  constexpr int KB = 8;
  for (int k0 = 0; k0 < K; k0 += 16 * KB) {
    wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> b[KB][NT];
#pragma unroll
    for (int kk = 0; kk < KB; ++kk)
      if (k0 + kk * 16 < K)
#pragma unroll
        for (int j = 0; j < NT; ++j)
          wmma::load_matrix_sync(b[kk][j], W + (size_t)(k0 + kk * 16) * D::H + (warp * NT + j) * 16,
                                 D::H);
#pragma unroll
    for (int kk = 0; kk < KB; ++kk) {
      if (k0 + kk * 16 >= K) break;
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> a;
        wmma::load_matrix_sync(a, A + i * 16 * lda + k0 + kk * 16, lda);
#pragma unroll
        for (int j = 0; j < NT; ++j) wmma::mma_sync(acc[i][j], a, b[kk][j], acc[i][j]);
      }
    }
  }
  __syncthreads(); /* every warp is done reading A before act is rewritten below */
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
      wmma::store_matrix_sync(stg + i * 16 * D::LDS + (warp * NT + j) * 16, acc[i][j], D::LDS,
                              wmma::mem_row_major);
  __syncthreads();
  for (int e = tid; e < FR * D::H; e += blockDim.x) {
    const int r = e / D::H, c = e - r * D::H;
    act[r * D::LDA + c] = __float2bfloat16_rn(silu(stg[r * D::LDS + c] + bias[c]));
  }
  __syncthreads();
}

/* Embedding columns of the rows whose conformer id is >= 0 (conf_smem[FR]), from the FP32
 * table; call after the rows are in xs, then __syncthreads. */
template <int NT>
__device__ __forceinline__ void fill_embedding(bf16 *xs, const int *conf_smem,
                                               const float *__restrict__ theta,
                                               const MlpLayout &L, int tid) {
  using D = Dims<NT>;
  if (!L.n_emb) return;
  for (int i = tid; i < FR * GD_MLP_EMB; i += blockDim.x) {
    const int r = i / GD_MLP_EMB, c = i - r * GD_MLP_EMB;
    const int e = conf_smem[r];
    if (e >= 0)
      xs[r * D::LDX + GD_MLP_EMB_OFF + c] =
          __float2bfloat16_rn(theta[L.emb + (size_t)e * GD_MLP_EMB + c]);
  }
}

/* y_smem[r] = network(xs row r) for all FR rows (rows past the data must hold finite values) */
template <int NT>
__device__ __forceinline__ void rows_forward(bf16 *xs, bf16 *act, float *stg,
                                             const float *__restrict__ theta,
                                             const bf16 *__restrict__ wh, const MlpLayout &L,
                                             float *y_smem, int tid) {
  using D = Dims<NT>;
  const int warp = tid >> 5, lane = tid & 31;
  layer<NT>(xs, D::LDX, GD_MLP_IN, wh + L.w1, theta + L.b1, act, stg, warp, tid);
  layer<NT>(act, D::LDA, D::H, wh + L.w2, theta + L.b2, act, stg, warp, tid);
  layer<NT>(act, D::LDA, D::H, wh + L.w3, theta + L.b3, act, stg, warp, tid);
  const float *w4 = theta + L.w4;
  for (int r = warp; r < FR; r += (blockDim.x >> 5)) {
    float s = 0.0f;
    for (int j = lane; j < D::H; j += 32) s += __bfloat162float(act[r * D::LDA + j]) * w4[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) y_smem[r] = s + theta[L.b4];
  }
  __syncthreads();
}

}  // namespace fwd
}  // namespace gd

#endif
