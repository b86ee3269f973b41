/*
 * gd_mlp_fwd.cuh -- the surrogate's forward pass over FR rows held in shared memory, as device
 * code shared by the stand-alone forward kernel (gd_mlp.cu) and the delayed-acceptance front
 * kernel (gd_da.cu).
 *
 * One CTA of 8 warps, FR = 32 rows (two 16-row MMA tiles); warp w owns output columns
 * [w H/8, (w+1) H/8) of every layer. Each layer is a chain of BF16 m16n8k16 tensor-core MMAs
 * (mma.sync, FP32 accumulate; PTX ISA "Matrix fragments for mma.m16n8k16"):
 *
 *   A  the layer's input rows, BF16 in shared memory, loaded with ldmatrix.x4;
 *   B  the weights, read straight into registers from a fragment-ordered BF16 copy in global
 *      memory (to_frag in gd_mlp.cu: one coalesced 16- or 32-byte load per lane and k-step,
 *      served by L2) through a ring of RING k-steps that runs across the three layers, so
 *      the next layer's first k-steps are in flight while this one finishes;
 *   C  bias + SiLU + BF16 rounding applied in registers to the accumulator fragments, written
 *      to the other of two activation buffers (no FP32 staging, one barrier per layer).
 *
 * The shared-memory footprint is small (about 42 KB at H = 256) so that front kernels of one
 * replica chain run on the SMs beside the exact-energy kernel of another. The output layer
 * (dot product with w4) and the bias/SiLU arithmetic are those of the layer-by-layer kernels.
 */
#ifndef GD_MLP_FWD_CUH
#define GD_MLP_FWD_CUH

#include <cstdint>

#include "gd_mlp.cuh"

namespace gd {
namespace fwd {

using bf16 = __nv_bfloat16;

constexpr int FR = 32; /* rows per CTA: short per-CTA chains, many CTAs */

__device__ __forceinline__ float silu(float z) { return mlp_silu(z); }

template <int NT> /* H = 128 * NT; a warp owns 2 NT 8-column MMA tiles */
struct Dims {
  static constexpr int H = 128 * NT, NT8 = 2 * NT, LDX = GD_MLP_IN + 8, LDA = H + 8;
  /* weight k-steps in flight per lane: 16 registers of fragments either way, which keeps the
   * kernels at <= 96 registers a thread, so they fit beside two CTAs of the exact-energy kernel */
  static constexpr int RING = 4 / NT;
  static constexpr size_t xs_bytes = (size_t)FR * LDX * 2;
  static constexpr size_t act_bytes = (size_t)FR * LDA * 2;
  static constexpr size_t par_bytes = (size_t)4 * H * 4; /* b1, b2, b3, w4 */
  static constexpr size_t smem = xs_bytes + 2 * act_bytes + par_bytes + 16;
};

/* the forward's shared-memory buffers, carved from the dynamic shared memory (row strides of
 * 144 and 2H + 16 bytes: 16-byte aligned and conflict-free for ldmatrix) */
template <int NT>
struct Smem {
  bf16 *xs, *act0, *act1;
  float *par; /* [4][H]: b1, b2, b3, w4 */
  float *b4;
  __device__ explicit Smem(unsigned char *base) {
    using D = Dims<NT>;
    xs = reinterpret_cast<bf16 *>(base);
    act0 = reinterpret_cast<bf16 *>(base + D::xs_bytes);
    act1 = reinterpret_cast<bf16 *>(base + D::xs_bytes + D::act_bytes);
    par = reinterpret_cast<float *>(base + D::xs_bytes + 2 * D::act_bytes);
    b4 = par + 4 * D::H;
  }
};

/* biases, w4 and b4 into shared memory (before the barrier that precedes rows_forward) */
template <int NT>
__device__ __forceinline__ void stage_params(const Smem<NT> &sm, const float *__restrict__ theta,
                                             const MlpLayout &L, int tid) {
  using D = Dims<NT>;
  for (int i = tid; i < 4 * D::H; i += blockDim.x) {
    const int k = i / D::H, c = i - k * D::H;
    const size_t off = k == 0 ? L.b1 : k == 1 ? L.b2 : k == 2 ? L.b3 : L.w4;
    sm.par[i] = theta[off + c];
  }
  if (tid == 0) sm.b4[0] = theta[L.b4];
}

/* this lane's weight fragments of one k-step: NT x 16 bytes = 2 NT n8 tiles x {b0b1, b2b3} */
template <int NT>
struct Ring {
  uint4 q[Dims<NT>::RING][NT];
};

/* lane `lane` of warp `warp`, k-step ks of a layer block of the fragment-ordered copy */
template <int NT>
__device__ __forceinline__ const uint4 *frag_ptr(const bf16 *__restrict__ wf, int ks, int warp,
                                                 int lane) {
  return reinterpret_cast<const uint4 *>(wf) + ((size_t)(ks * 8 + warp) * 32 + lane) * NT;
}

template <int NT>
__device__ __forceinline__ void ring_load(uint4 (&dst)[NT], const bf16 *__restrict__ wf, int ks,
                                          int warp, int lane) {
  const uint4 *p = frag_ptr<NT>(wf, ks, warp, lane);
#pragma unroll
  for (int j = 0; j < NT; ++j) dst[j] = __ldg(p + j);
}

/* the first RING k-steps of W1 (call before the barrier that precedes rows_forward, so
 * that the loads overlap the caller's own work) */
template <int NT>
__device__ __forceinline__ void prefetch_first(Ring<NT> &ring, const bf16 *__restrict__ wf,
                                               int tid) {
#pragma unroll
  for (int s = 0; s < Dims<NT>::RING; ++s) ring_load<NT>(ring.q[s], wf, s, tid >> 5, tid & 31);
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&a)[4], unsigned addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(addr)
               : "memory");
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_silu(float z0, float z1) {
  const __nv_bfloat162 h = __halves2bfloat162(__float2bfloat16_rn(silu(z0)),
                                              __float2bfloat16_rn(silu(z1)));
  return *reinterpret_cast<const uint32_t *>(&h);
}

/* one layer, K = 16 KS inputs: out = bf16(SiLU(A W + b)). G0 is the layer's first k-step in
 * the ring's sequence (slot = (G0 + ks) % RING); on entry the ring holds this layer's k-steps
 * 0..RING-1, on exit the next layer's (wf_next, when given). */
template <int NT, int KS, int G0>
__device__ __forceinline__ void layer(Ring<NT> &ring, const bf16 *A, int lda,
                                      const bf16 *__restrict__ wf, const bf16 *__restrict__ wf_next,
                                      const float *bias, bf16 *out, int warp, int lane) {
  using D = Dims<NT>;
  constexpr int NT8 = D::NT8, RING = D::RING;
  float acc[2][NT8][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int j = 0; j < NT8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.0f;
  /* ldmatrix.x4 row addresses: lanes 0-15 rows 0-15 at column 0, lanes 16-31 at column 8 */
  const unsigned a0 = (unsigned)__cvta_generic_to_shared(A + (lane & 15) * lda + (lane >> 4) * 8);
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const int slot = (G0 + ks) % RING;
    uint4 b[NT];
#pragma unroll
    for (int j = 0; j < NT; ++j) b[j] = ring.q[slot][j];
    if (ks + RING < KS)
      ring_load<NT>(ring.q[slot], wf, ks + RING, warp, lane);
    else if (wf_next)
      ring_load<NT>(ring.q[slot], wf_next, ks + RING - KS, warp, lane);
    uint32_t a[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m) ldmatrix_x4(a[m], a0 + (unsigned)((m * 16 * lda + ks * 16) * 2));
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        mma_bf16(acc[m][2 * j], a[m], b[j].x, b[j].y);
        mma_bf16(acc[m][2 * j + 1], a[m], b[j].z, b[j].w);
      }
  }
  /* accumulator fragment: c0, c1 at (row g, columns 2t, 2t+1), c2, c3 at row g + 8 */
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int j = 0; j < NT8; ++j) {
    const int col = (warp * NT8 + j) * 8 + 2 * t;
    const float bc0 = bias[col], bc1 = bias[col + 1];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int r = m * 16 + g;
      *reinterpret_cast<uint32_t *>(out + r * D::LDA + col) =
          pack_silu(acc[m][j][0] + bc0, acc[m][j][1] + bc1);
      *reinterpret_cast<uint32_t *>(out + (r + 8) * D::LDA + col) =
          pack_silu(acc[m][j][2] + bc0, acc[m][j][3] + bc1);
    }
  }
}

/* Embedding columns of the rows whose conformer id is >= 0 (theta FP32 -> BF16). */
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

/* y_smem[r] = network(xs row r) for all FR rows (rows past the data must hold finite values).
 * stage_params and prefetch_first must have been called before the last barrier; wf is the
 * fragment-ordered weight copy (W1, W2, W3 blocks; to_frag in gd_mlp.cu). */
template <int NT>
__device__ __forceinline__ void rows_forward(const Smem<NT> &sm, Ring<NT> &ring,
                                             const bf16 *__restrict__ wf, float *y_smem,
                                             int tid) {
  using D = Dims<NT>;
  constexpr int K1 = GD_MLP_IN / 16, K2 = D::H / 16;
  const int warp = tid >> 5, lane = tid & 31;
  const bf16 *wf2 = wf + (size_t)GD_MLP_IN * D::H;
  const bf16 *wf3 = wf2 + (size_t)D::H * D::H;
  layer<NT, K1, 0>(ring, sm.xs, D::LDX, wf, wf2, sm.par, sm.act0, warp, lane);
  __syncthreads();
  layer<NT, K2, K1>(ring, sm.act0, D::LDA, wf2, wf3, sm.par + D::H, sm.act1, warp, lane);
  __syncthreads();
  layer<NT, K2, K1 + K2>(ring, sm.act1, D::LDA, wf3, nullptr, sm.par + 2 * D::H, sm.act0, warp,
                         lane);
  __syncthreads();
  const float *w4 = sm.par + 3 * D::H;
  for (int r = warp; r < FR; r += (blockDim.x >> 5)) {
    float s = 0.0f;
    for (int j = lane; j < D::H; j += 32) s += __bfloat162float(sm.act0[r * D::LDA + j]) * w4[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) y_smem[r] = s + sm.b4[0];
  }
  __syncthreads();
}

}  // namespace fwd
}  // namespace gd

#endif
