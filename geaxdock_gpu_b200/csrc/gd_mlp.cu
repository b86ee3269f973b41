/*
 * gd_mlp.cu -- forward, backward and Adam kernels of the energy surrogate (gd_mlp.cuh).
 *
 * Every matrix product of training runs on the fifth-generation tensor cores through
 * umma_gemm (gd_umma.cu: TMA-staged BF16 operands, FP32 accumulator in tensor memory), with
 * the elementwise step that follows it fused into its epilogue:
 *   forward        Z = X W + b, A = bf16(SiLU(Z))         (X K-major, W MN-major)
 *   input grad     dZ' = bf16((dZ W^T) SiLU'(Z'))         (dZ K-major, W K-major)
 *   weight grad    dW = A^T dZ over chunks of 256 rows    (both MN-major, split-K partials)
 * The 256 -> 1 output layer, the loss, column sums for the bias gradients, the embedding
 * gradient (atomic scatter) and Adam are elementwise kernels. Batch reductions add per-chunk
 * partials in a fixed order. Master parameters, gradients and Adam moments are FP32; W1..W3
 * are mirrored in BF16 (row-major, and in MMA-fragment order for the one-kernel forward) after
 * every update.
 */
#include <algorithm>
#include <cmath>

#include "gd_mlp.cuh"
#include "gd_mlp_fwd.cuh"
#include "gd_numerics.h"
#include "gd_umma.cuh"

namespace gd {

using bf16 = __nv_bfloat16;

namespace {

__device__ __forceinline__ float silu(float z) { return mlp_silu(z); }
__device__ __forceinline__ float silu_grad(float z) { return mlp_silu_grad(z); }

/* y[r] = A3[r] . w4 + b4, one warp per row */
__global__ void out_layer(const bf16 *__restrict__ A3, const float *__restrict__ w4,
                          const float *__restrict__ b4, float *__restrict__ y, int rows, int h) {
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (r >= rows) return;
  float s = 0.0f;
  for (int j = lane; j < h; j += 32) s += __bfloat162float(A3[(size_t)r * h + j]) * w4[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[r] = s + b4[0];
}

/* dy = 2 (y - t) / rows; squared errors to e2 */
__global__ void mse_grad(const float *__restrict__ y, const float *__restrict__ t,
                         float *__restrict__ dy, float *__restrict__ e2, int rows) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float d = y[r] - t[r];
  dy[r] = 2.0f * d / (float)rows;
  e2[r] = d * d;
}

/* deterministic mean of e2 into out[0] (one block) */
__global__ void mean_reduce(const float *__restrict__ e2, int rows, float *out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += 256) s += e2[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = (float)(sh[0] / (double)rows);
}

/* dZ3 = (dy w4^T) * SiLU'(Z3) -> bf16 */
__global__ void out_backward(const float *__restrict__ dy, const float *__restrict__ w4,
                             const float *__restrict__ Z3, bf16 *__restrict__ D, int rows, int h) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)rows * h) return;
  const int r = (int)(i / h), j = (int)(i % h);
  D[i] = __float2bfloat16_rn(dy[r] * w4[j] * silu_grad(Z3[i]));
}

/* Reductions over the batch are split into chunks of SPLIT_ROWS rows: each chunk writes a
 * partial result, reduce_partials adds the chunks in a fixed order (deterministic). */
constexpr int SPLIT_ROWS = 256;

/* partial column sums of a [rows][n] BF16 matrix, optionally weighted per row by w; with
 * w != null an extra column n holds sum_r w[r]. Block: 32 columns x 8 row lanes; grid
 * (columns / 32, chunks). part[chunk][ncol], ncol = n + (w != null). */
__global__ void __launch_bounds__(256) colsum_split(const bf16 *__restrict__ A, const float *__restrict__ w,
                                                    int rows, int n, float *__restrict__ part) {
  __shared__ float sh[8][33];
  const int cx = threadIdx.x & 31, ry = threadIdx.x >> 5;
  const int col = blockIdx.x * 32 + cx, chunk = blockIdx.y;
  const int ncol = n + (w ? 1 : 0);
  const int r0 = chunk * SPLIT_ROWS, r1 = min(rows, r0 + SPLIT_ROWS);
  float s = 0.0f;
  if (col < ncol) {
    for (int r = r0 + ry; r < r1; r += 8) {
      const float a = col < n ? __bfloat162float(A[(size_t)r * n + col]) : 1.0f;
      s += w ? a * w[r] : a;
    }
  }
  sh[ry][cx] = s;
  __syncthreads();
  if (ry == 0 && col < ncol) {
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += sh[k][cx];
    part[(size_t)chunk * ncol + col] = t;
  }
}

/* out[i] += sum_c part[c * count + i] */
__global__ void reduce_partials(const float *__restrict__ part, int chunks, size_t count,
                                float *__restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float s = 0.0f;
  for (int c = 0; c < chunks; ++c) s += part[(size_t)c * count + i];
  out[i] += s;
}

/* embedding gradient: columns [7, 39) of dX1 scattered to the rows' conformer entries */
__global__ void emb_grad(const float *__restrict__ dX, const int *__restrict__ conf, int rows,
                         float *__restrict__ gemb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * GD_MLP_EMB) return;
  const int r = i / GD_MLP_EMB, c = i - r * GD_MLP_EMB;
  const int e = conf[r];
  if (e >= 0) atomicAdd(gemb + (size_t)e * GD_MLP_EMB + c, dX[(size_t)r * GD_MLP_IN + GD_MLP_EMB_OFF + c]);
}

/* embedding columns of X from theta (rows with conf < 0 keep their columns) */
__global__ void emb_fill(bf16 *__restrict__ X, const float *__restrict__ emb,
                         const int *__restrict__ conf, int rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * GD_MLP_EMB) return;
  const int r = i / GD_MLP_EMB, c = i - r * GD_MLP_EMB;
  const int e = conf[r];
  if (e >= 0)
    X[(size_t)r * GD_MLP_IN + GD_MLP_EMB_OFF + c] = __float2bfloat16_rn(emb[(size_t)e * GD_MLP_EMB + c]);
}

__global__ void adam_kernel(float *__restrict__ th, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  th[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

/* the Adam step with its bias corrections read from c[0], c[1] (device) */
__global__ void adam_dev_kernel(float *__restrict__ th, const float *__restrict__ g,
                                float *__restrict__ m, float *__restrict__ v, size_t n, float lr,
                                float b1, float b2, float eps, const float *__restrict__ c) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float c1 = c[0], c2 = c[1];
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  th[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

/* advances the device step count t = st[0] and writes 1 - b1^t, 1 - b2^t as floats at st[1..2] */
__global__ void adam_tick(int *st, float b1, float b2) {
  const int t = st[0] + 1;
  st[0] = t;
  float *c = reinterpret_cast<float *>(st + 1);
  c[0] = 1.0f - powf(b1, (float)t);
  c[1] = 1.0f - powf(b2, (float)t);
}

__global__ void to_bf16(const float *__restrict__ a, bf16 *__restrict__ b, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

/* Fragment-ordered BF16 copy of W1, W2, W3 for the fused forward (H = 64 NT8, NT8 = 2 or 4):
 * in each layer block, element (((ks 8 + w) 32 + lane) NT8 + j) 4 + q holds W[k][n] with
 * k = 16 ks + 2 (lane % 4) + (q % 2) + 8 (q / 2) and n = 8 (NT8 w + j) + lane / 4, the
 * m16n8k16 B-operand fragment {b0, b1, b2, b3} of lane `lane` for 8-column tile j of warp w at
 * k-step ks, so that a lane's fragments of one k-step are NT8 x 8 contiguous bytes. */
__global__ void to_frag(const float *__restrict__ theta, MlpLayout L, bf16 *__restrict__ wf) {
  const size_t H = L.hidden, n1 = (size_t)GD_MLP_IN * H, i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n1 + 2 * H * H) return;
  size_t e = i;
  const float *W = theta + L.w1;
  if (e >= n1 + H * H) {
    e -= n1 + H * H;
    W = theta + L.w3;
  } else if (e >= n1) {
    e -= n1;
    W = theta + L.w2;
  }
  const int nt8 = (int)(H / 64);
  const int q = (int)(e & 3);
  size_t t = e >> 2;
  const int j = (int)(t % nt8);
  t /= nt8;
  const int lane = (int)(t & 31);
  t >>= 5;
  const int w = (int)(t & 7);
  const size_t ks = t >> 3;
  const size_t k = 16 * ks + 2 * (lane & 3) + (q & 1) + 8 * (q >> 1);
  const size_t n = 8 * ((size_t)nt8 * w + j) + (lane >> 2);
  wf[i] = __float2bfloat16_rn(W[k * H + n]);
}

/* uniform(-scale, scale) from Philox, keyed by (seed, tensor id) */
__global__ void init_uniform(float *p, size_t n, float scale, uint32_t tensor, uint64_t seed) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const gd_u32x4 r = gd_philox4x32_10((uint32_t)i, tensor, 0x5EEDu, 7u, (uint32_t)seed,
                                      (uint32_t)(seed >> 32));
  p[i] = scale * gd_sym11(r.v[0]);
}

/* The whole forward pass of fwd::FR rows in one CTA of 8 warps (gd_mlp_fwd.cuh). */
template <int NT>
__global__ void __launch_bounds__(256) fused_forward(const bf16 *__restrict__ X,
                                                     const int *__restrict__ conf,
                                                     const float *__restrict__ theta,
                                                     const bf16 *__restrict__ wf, MlpLayout L,
                                                     int rows, float *__restrict__ y) {
  using D = fwd::Dims<NT>;
  constexpr int FR = fwd::FR;
  extern __shared__ __align__(128) unsigned char fsm[];
  __shared__ int cf[FR];
  __shared__ float ys[FR];
  const fwd::Smem<NT> sm(fsm);
  bf16 *xs = sm.xs;
  const int tid = threadIdx.x;
  const int row0 = blockIdx.x * FR;
  fwd::Ring<NT> ring;
  fwd::prefetch_first<NT>(ring, wf, tid);
  fwd::stage_params<NT>(sm, theta, L, tid);
  for (int i = tid; i < FR * 8; i += 256) {
    const int r = i >> 3, c = i & 7;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (row0 + r < rows) v = reinterpret_cast<const uint4 *>(X + (size_t)(row0 + r) * GD_MLP_IN)[c];
    *reinterpret_cast<uint4 *>(xs + r * D::LDX + c * 8) = v;
  }
  if (tid < FR) cf[tid] = row0 + tid < rows ? conf[row0 + tid] : -1;
  __syncthreads();
  fwd::fill_embedding<NT>(xs, cf, theta, L, tid);
  __syncthreads();
  fwd::rows_forward<NT>(sm, ring, wf, ys, tid);
  if (tid < FR && row0 + tid < rows) y[row0 + tid] = ys[tid];
}

constexpr int FR = fwd::FR;
template <int NT>
using FusedDims = fwd::Dims<NT>;

inline int blocks(size_t n, int t = 256) { return (int)((n + t - 1) / t); }

}  // namespace

int mlp_refresh_bf16(Mlp &n, cudaStream_t s) {
  const size_t nw = n.L.b4; /* W1..w4 region; biases converted too, unused */
  to_bf16<<<blocks(nw), 256, 0, s>>>(n.theta, n.wh, nw);
  if (n.wf) {
    const size_t H = n.L.hidden;
    to_frag<<<blocks((size_t)GD_MLP_IN * H + 2 * H * H), 256, 0, s>>>(n.theta, n.L, n.wf);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int mlp_create(Mlp &n, int hidden, int n_emb, uint64_t seed, cudaStream_t s) {
  if (hidden % 16 || hidden < 16 || hidden > 256) return -1;
  n.L.set(hidden, n_emb);
  const size_t T = n.L.total;
  if (cudaMalloc(&n.theta, T * 4) || cudaMalloc(&n.grad, T * 4) || cudaMalloc(&n.m, T * 4) ||
      cudaMalloc(&n.v, T * 4) || cudaMalloc(&n.wh, n.L.b4 * 2) || cudaMalloc(&n.loss, 16) ||
      cudaMalloc(&n.err, sizeof(int)) || cudaMalloc(&n.adam_dev, 3 * sizeof(int)))
    return -3;
  cudaMemsetAsync(n.err, 0, sizeof(int), s);
  if ((hidden == 128 || hidden == 256) &&
      cudaMalloc(&n.wf, ((size_t)GD_MLP_IN * hidden + 2 * (size_t)hidden * hidden) * 2))
    return -3;
  cudaMemsetAsync(n.theta, 0, T * 4, s);
  cudaMemsetAsync(n.m, 0, T * 4, s);
  cudaMemsetAsync(n.v, 0, T * 4, s);
  const int H = hidden;
  init_uniform<<<blocks((size_t)GD_MLP_IN * H), 256, 0, s>>>(n.theta + n.L.w1, (size_t)GD_MLP_IN * H,
                                                             1.0f / sqrtf((float)GD_MLP_IN), 1, seed);
  init_uniform<<<blocks((size_t)H * H), 256, 0, s>>>(n.theta + n.L.w2, (size_t)H * H,
                                                     1.0f / sqrtf((float)H), 2, seed);
  init_uniform<<<blocks((size_t)H * H), 256, 0, s>>>(n.theta + n.L.w3, (size_t)H * H,
                                                     1.0f / sqrtf((float)H), 3, seed);
  init_uniform<<<blocks(H), 256, 0, s>>>(n.theta + n.L.w4, H, 1.0f / sqrtf((float)H), 4, seed);
  if (n_emb)
    init_uniform<<<blocks((size_t)n_emb * GD_MLP_EMB), 256, 0, s>>>(
        n.theta + n.L.emb, (size_t)n_emb * GD_MLP_EMB, 0.3f, 5, seed);
  n.adam_t = 0;
  if (cudaFuncSetAttribute(fused_forward<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)FusedDims<1>::smem) != cudaSuccess ||
      cudaFuncSetAttribute(fused_forward<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)FusedDims<2>::smem) != cudaSuccess)
    return -2;
  return mlp_refresh_bf16(n, s);
}

void mlp_destroy(Mlp &n) {
  void *ps[] = {n.theta, n.grad, n.m, n.v, n.wh, n.wf, n.loss, n.err, n.adam_dev, n.X, n.A1, n.A2, n.A3, n.D, n.D2, n.Pb,
                n.Z1, n.Z2, n.Z3, n.C, n.y, n.dy, n.conf, n.P};
  for (void *p : ps)
    if (p) cudaFree(p);
  n = Mlp();
}

int mlp_reserve(Mlp &n, int rows) {
  rows = (rows + 15) & ~15;
  if (rows <= n.cap) return 0;
  void *ps[] = {n.X, n.A1, n.A2, n.A3, n.D, n.D2, n.Z1, n.Z2, n.Z3, n.C, n.y, n.dy, n.conf, n.Pb};
  for (void *p : ps)
    if (p) cudaFree(p);
  const size_t H = n.L.hidden, R = rows;
  if (cudaMalloc(&n.X, R * GD_MLP_IN * 2) || cudaMalloc(&n.A1, R * H * 2) ||
      cudaMalloc(&n.A2, R * H * 2) || cudaMalloc(&n.A3, R * H * 2) ||
      cudaMalloc(&n.D, R * H * 2) || cudaMalloc(&n.D2, R * H * 2) || cudaMalloc(&n.Z1, R * H * 4) ||
      cudaMalloc(&n.Z2, R * H * 4) || cudaMalloc(&n.Z3, R * H * 4) ||
      cudaMalloc(&n.C, R * (H > GD_MLP_IN ? H : GD_MLP_IN) * 4) || cudaMalloc(&n.y, R * 4) ||
      cudaMalloc(&n.dy, R * 4) || cudaMalloc(&n.conf, R * 4) ||
      cudaMalloc(&n.Pb, ((R + 127) / 128) * H * 4))
    return -3;
  cudaMemset(n.X, 0, R * GD_MLP_IN * 2);
  cudaMemset(n.conf, 0xff, R * 4);
  n.cap = (int)R;
  return 0;
}

int mlp_set_rows(Mlp &n, const float *x, const int *conf, int rows, cudaStream_t s) {
  if (rows > n.cap) return -4;
  to_bf16<<<blocks((size_t)rows * GD_MLP_IN), 256, 0, s>>>(x, n.X, (size_t)rows * GD_MLP_IN);
  cudaMemcpyAsync(n.conf, conf, sizeof(int) * rows, cudaMemcpyDeviceToDevice, s);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int mlp_embed(Mlp &n, int rows, cudaStream_t s) {
  if (!n.L.n_emb) return 0;
  emb_fill<<<blocks((size_t)rows * GD_MLP_EMB), 256, 0, s>>>(n.X, n.theta + n.L.emb, n.conf, rows);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* forward over `rows` rows of n.X; keeps Z1..Z3 when `keep` for the backward pass */
static int forward_impl(Mlp &n, int rows, bool keep, cudaStream_t s) {
  const int M = (rows + 15) & ~15, H = n.L.hidden;
  if (M > n.cap) return -4;
  /* Z_l = A_{l-1} W_l + b_l, A_l = bf16(SiLU(Z_l)) in one tensor-core kernel per layer */
  auto layer = [&](const bf16 *Ain, int K, size_t w, size_t b, float *Z, bf16 *Aout) {
    const UmmaOperand a{Ain, M, K, 0}, wt{n.wh + w, K, H, 1};
    UmmaEpilogue e{};
    e.kind = UMMA_FWD;
    e.bias = n.theta + b;
    e.Z = keep ? Z : nullptr;
    e.Ob = Aout;
    e.ldo = H;
    return umma_gemm(a, wt, M, H, K, 1, e, n.err, s);
  };
  int rc;
  if ((rc = layer(n.X, GD_MLP_IN, n.L.w1, n.L.b1, n.Z1, n.A1)) ||
      (rc = layer(n.A1, H, n.L.w2, n.L.b2, n.Z2, n.A2)) ||
      (rc = layer(n.A2, H, n.L.w3, n.L.b3, n.Z3, n.A3)))
    return rc;
  out_layer<<<blocks((size_t)rows * 32), 256, 0, s>>>(n.A3, n.theta + n.L.w4, n.theta + n.L.b4,
                                                      n.y, rows, H);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int mlp_forward(Mlp &n, int rows, cudaStream_t s) {
  const int H = n.L.hidden;
  if (rows > n.cap) return -4;
  if (rows < 1) return 0;
  if (H == 128) {
    fused_forward<1><<<(rows + FR - 1) / FR, 256, FusedDims<1>::smem, s>>>(
        n.X, n.conf, n.theta, n.wf, n.L, rows, n.y);
  } else if (H == 256) {
    fused_forward<2><<<(rows + FR - 1) / FR, 256, FusedDims<2>::smem, s>>>(
        n.X, n.conf, n.theta, n.wf, n.L, rows, n.y);
  } else {
    int rc = mlp_embed(n, rows, s);
    if (rc) return rc;
    return forward_impl(n, rows, false, s);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int mlp_loss_backward(Mlp &n, int rows, const float *t, cudaStream_t s) {
  const int M = (rows + 15) & ~15, H = n.L.hidden;
  int rc = forward_impl(n, rows, true, s);
  if (rc) return rc;
  cudaMemsetAsync(n.grad, 0, n.L.total * 4, s);
  /* padded rows (rows..M) carry zero gradient */
  cudaMemsetAsync(n.dy, 0, (size_t)M * 4, s);
  mse_grad<<<blocks(rows), 256, 0, s>>>(n.y, t, n.dy, n.C, rows);
  mean_reduce<<<1, 256, 0, s>>>(n.C, rows, n.loss);
  /* batch reductions in chunks of SPLIT_ROWS rows, partials added in a fixed order */
  const int S = (M + SPLIT_ROWS - 1) / SPLIT_ROWS;
  const size_t need = (size_t)S * (size_t)H * (size_t)(H > GD_MLP_IN ? H : GD_MLP_IN) + S;
  if (need > n.p_cap) {
    if (n.P) cudaFree(n.P);
    n.P = nullptr;
    n.p_cap = 0;
    if (cudaMalloc(&n.P, need * sizeof(float)) != cudaSuccess) return -3;
    n.p_cap = need;
  }
  auto colsum = [&](const bf16 *A, const float *w, float *g) {
    const int ncol = H + (w ? 1 : 0);
    colsum_split<<<dim3((ncol + 31) / 32, S), 256, 0, s>>>(A, w, M, H, n.P);
    reduce_partials<<<blocks(ncol), 256, 0, s>>>(n.P, S, (size_t)ncol, g);
  };
  /* dW[i][j] = sum_r Aprev[r][i] dZ[r][j] in chunks of SPLIT_ROWS rows (both operands
   * MN-major, the rows are the reduction); W1 (64 rows) is computed as dW1^T = dZ1^T X so that
   * the 128-row MMA tile runs along the hidden dimension, and stored transposed */
  auto weight_grad = [&](const bf16 *Aprev, int K, const bf16 *D, float *g) {
    UmmaEpilogue e{};
    e.kind = UMMA_F32;
    e.Of = n.P;
    e.ldo = H;
    e.split_stride = (size_t)K * H;
    int rc;
    if (K == H) {
      rc = umma_gemm(UmmaOperand{Aprev, M, K, 1}, UmmaOperand{D, M, H, 1}, K, H, SPLIT_ROWS, S,
                     e, n.err, s);
    } else {
      e.trans = 1;
      rc = umma_gemm(UmmaOperand{D, M, H, 1}, UmmaOperand{Aprev, M, K, 1}, H, K, SPLIT_ROWS, S,
                     e, n.err, s);
    }
    if (rc) return rc;
    reduce_partials<<<blocks((size_t)K * H), 256, 0, s>>>(n.P, S, (size_t)K * H, g);
    return 0;
  };
  /* dZ_{l-1} = bf16((dZ_l W_l^T) SiLU'(Z_{l-1})), and its column sums (db_{l-1}) per 128-row
   * tile, added in tile order */
  auto input_grad = [&](const bf16 *D, size_t w, const float *Zprev, bf16 *Dout, float *gb) {
    UmmaEpilogue e{};
    e.kind = UMMA_DGRAD;
    e.Zin = Zprev;
    e.Ob = Dout;
    e.colsum = n.Pb;
    e.ldo = H;
    const int rc = umma_gemm(UmmaOperand{D, M, H, 0}, UmmaOperand{n.wh + w, H, H, 0}, M, H, H, 1,
                             e, n.err, s);
    if (rc) return rc;
    reduce_partials<<<blocks(H), 256, 0, s>>>(n.Pb, (M + 127) / 128, (size_t)H, gb);
    return 0;
  };
  bf16 *Dc = n.D, *Dn = n.D2;
  /* output layer: dw4 = A3^T dy and db4 = sum dy (b4 follows w4 in theta) */
  colsum(n.A3, n.dy, n.grad + n.L.w4);
  out_backward<<<blocks((size_t)M * H), 256, 0, s>>>(n.dy, n.theta + n.L.w4, n.Z3, Dc, M, H);
  /* layer 3: dW3 = A2^T dZ3, db3, dZ2 */
  if ((rc = weight_grad(n.A2, H, Dc, n.grad + n.L.w3))) return rc;
  colsum(Dc, nullptr, n.grad + n.L.b3);
  if ((rc = input_grad(Dc, n.L.w3, n.Z2, Dn, n.grad + n.L.b2))) return rc;
  std::swap(Dc, Dn);
  /* layer 2 (db2 came with dZ2) */
  if ((rc = weight_grad(n.A1, H, Dc, n.grad + n.L.w2))) return rc;
  if ((rc = input_grad(Dc, n.L.w2, n.Z1, Dn, n.grad + n.L.b1))) return rc;
  std::swap(Dc, Dn);
  /* layer 1: dW1 = X^T dZ1 (64 x H) (db1 came with dZ1); dX = dZ1 W1^T (FP32) for the
   * embedding */
  if ((rc = weight_grad(n.X, GD_MLP_IN, Dc, n.grad + n.L.w1))) return rc;
  if (n.L.n_emb) {
    UmmaEpilogue e{};
    e.kind = UMMA_F32;
    e.Of = n.C;
    e.ldo = GD_MLP_IN;
    if ((rc = umma_gemm(UmmaOperand{Dc, M, H, 0}, UmmaOperand{n.wh + n.L.w1, GD_MLP_IN, H, 0}, M,
                        GD_MLP_IN, H, 1, e, n.err, s)))
      return rc;
    emb_grad<<<blocks((size_t)rows * GD_MLP_EMB), 256, 0, s>>>(n.C, n.conf, rows,
                                                             n.grad + n.L.emb);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int mlp_status(Mlp &n) {
  int e = 0;
  if (cudaMemcpy(&e, n.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
  if (!e) return 0;
  cudaMemset(n.err, 0, sizeof(int));
  return -6;
}

int mlp_adam(Mlp &n, float lr, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  n.adam_t += 1;
  const float c1 = 1.0f - powf(b1, (float)n.adam_t), c2 = 1.0f - powf(b2, (float)n.adam_t);
  adam_kernel<<<blocks(n.L.total), 256, 0, s>>>(n.theta, n.grad, n.m, n.v, n.L.total, lr, b1, b2,
                                               eps, c1, c2);
  return mlp_refresh_bf16(n, s);
}

int mlp_adam_dev_sync(Mlp &n, cudaStream_t s) {
  return cudaMemcpyAsync(n.adam_dev, &n.adam_t, sizeof(int), cudaMemcpyHostToDevice, s) ==
                 cudaSuccess
             ? 0
             : -2;
}

int mlp_adam_dev(Mlp &n, float lr, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  adam_tick<<<1, 1, 0, s>>>(n.adam_dev, b1, b2);
  adam_dev_kernel<<<blocks(n.L.total), 256, 0, s>>>(
      n.theta, n.grad, n.m, n.v, n.L.total, lr, b1, b2, eps,
      reinterpret_cast<const float *>(n.adam_dev + 1));
  return mlp_refresh_bf16(n, s);
}

}  // namespace gd
