/*
 * gd_umma.cu -- tcgen05 GEMM of the surrogate's training (interface and operand conventions in
 * gd_umma.cuh).
 *
 * One CTA of 8 warps computes a 128 x BN tile of C (BN = 64 or 128) over one chunk of at most
 * 256 reduction elements, so both operand tiles fit in shared memory at once (<= 128 KB) and
 * no stage is ever refilled:
 *
 *   thread 0   issues every TMA box load (2-D tiled cp.async.bulk.tensor, 128-byte swizzle,
 *              boxes 64 elements wide), each 64-wide slice of K completing on its own mbarrier,
 *              and as each slice lands (bounded wait) issues its tcgen05.mma (kind::f16, BF16 x
 *              BF16 -> FP32, M = 128, N = BN, K = 16) into a BN-column tensor-memory
 *              accumulator, so the products of the first slices run while the later ones are
 *              still in flight; the MMAs are committed to one more mbarrier;
 *   warp w     reads accumulator lanes 32 (w % 4)..+31 (rows) of column half w / 4 with
 *              tcgen05.ld.32x32b.x32, 32 columns at a time, turns the 32 x 32 block around in
 *              shared memory so that lanes run along a row (coalesced stores), and applies the
 *              epilogue (bias + SiLU into BF16 activations and FP32 pre-activations, the SiLU
 *              derivative for input gradients, or FP32 partial sums, optionally transposed).
 *              The turn-around buffer reuses the operand tiles' shared memory once the MMAs
 *              have completed, so a CTA needs only its two tiles: two BN = 64 CTAs share an SM
 *              and one's epilogue overlaps the other's loads and products.
 *
 * Shared-memory operand layouts are the canonical swizzled forms the descriptors name:
 *   K-major  per 64-wide slice of K, rows x 128 bytes, 8-row groups 1024 bytes apart
 *            (LBO 16 bytes, SBO 1024 bytes); the k-th 16-element step starts 32 k bytes in;
 *   MN-major per 64-wide block of the output dimension, K rows x 128 bytes (LBO = K x 128
 *            bytes between blocks, SBO 1024 bytes between 8-row groups of K); the k-th step
 *            starts 2048 k bytes in.
 * Every wait is bounded (globaltimer, 2 s): on a timeout the CTA records a code in err, skips
 * the work that depended on it and still frees its tensor memory.
 */
#include <cuda.h> /* CUtensorMap and its enums; the encoder is fetched from the driver at run time */

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "gd_mlp.cuh"
#include "gd_umma.cuh"

namespace gd {
namespace {

using bf16 = __nv_bfloat16;

constexpr int BM = 128;
constexpr long long WAIT_NS = 2000000000LL;
constexpr int STAGE_BYTES = 8 * 32 * 33 * 4;
constexpr int MAX_SLICES = 4; /* K <= 256 in slices of 64 */

struct UmmaArgs {
  int M, N, K, a_mn, b_mn;
  UmmaEpilogue e;
  int *err;
};

__device__ __forceinline__ uint32_t su32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ long long gtime() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool bar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
  if (bar_try(bar, parity)) return true;
  const long long deadline = gtime() + WAIT_NS;
  while (!bar_try(bar, parity))
    if (gtime() > deadline) return false;
  return true;
}
__device__ __forceinline__ void tma_2d(void *dst, const CUtensorMap *map, int x, int y,
                                       uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(su32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}
/* shared-memory matrix descriptor: start, leading / stride byte offsets (16-byte units),
 * descriptor version 1, 128-byte swizzle */
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo16, uint32_t sbo16) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo16 & 0x3FFFu) << 16) |
         ((uint64_t)(sbo16 & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
        "=r"(v[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

/* bytes of the two operand tiles in shared memory (both multiples of 1024) */
__host__ __device__ inline uint32_t tile_bytes(int mn, int rows_tile, int K) {
  return mn ? (uint32_t)(rows_tile / 64) * (uint32_t)K * 128u
            : (uint32_t)((K + 63) / 64) * (uint32_t)rows_tile * 128u;
}

/* descriptor of k-step ks of an operand tile at shared address s */
__device__ __forceinline__ uint64_t op_desc(uint32_t s, int mn, int rows_tile, int K, int ks) {
  if (mn) return sdesc(s + (uint32_t)ks * 2048u, (uint32_t)K * 8u, 64u);
  return sdesc(s + (uint32_t)(ks >> 2) * (uint32_t)rows_tile * 128u + (uint32_t)(ks & 3) * 32u,
               1u, 64u);
}

/* K slices the loads complete on: 64 wide when K is a multiple of 64 (MN-major boxes are then
 * 64 x 64 and land inside their block), else one slice with MN-major boxes K rows high */
__host__ __device__ inline int k_slices(int K) { return (K % 64 == 0) ? K / 64 : 1; }

/* bytes of slice s of an operand tile (a whole tile when there is one slice) */
__device__ __forceinline__ uint32_t slice_bytes(int mn, int rows_tile, int K, int ns) {
  if (ns == 1) return tile_bytes(mn, rows_tile, K);
  return mn ? (uint32_t)(rows_tile / 64) * 8192u : (uint32_t)rows_tile * 128u;
}

/* the boxes of slice s of one operand tile: K-major boxes are 64 (k) x rows_tile; MN-major
 * boxes 64 (mn) x 64 (k) at 64 s rows into each 64-wide block, or 64 (mn) x K for one slice */
__device__ __forceinline__ void load_slice(unsigned char *dst, const CUtensorMap *map, int mn,
                                           int rows_tile, int K, int r0, int k0, int s, int ns,
                                           uint64_t *bar) {
  if (mn) {
    for (int b = 0; b < rows_tile / 64; ++b)
      tma_2d(dst + (size_t)b * K * 128 + (size_t)s * 8192, map, r0 + 64 * b, k0 + 64 * s, bar);
  } else if (ns > 1) {
    tma_2d(dst + (size_t)s * rows_tile * 128, map, k0 + 64 * s, r0, bar);
  } else {
    for (int b = 0; b < (K + 63) / 64; ++b)
      tma_2d(dst + (size_t)b * rows_tile * 128, map, k0 + 64 * b, r0, bar);
  }
}

template <int BN>
__global__ void __launch_bounds__(256, 2)
    umma_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                UmmaArgs g) {
  extern __shared__ unsigned char dsm[];
  /* bar[0 .. MAX_SLICES - 1]: the K slices' loads; bar[MAX_SLICES]: the MMAs' commit */
  __shared__ __align__(8) uint64_t bar[MAX_SLICES + 1];
  __shared__ uint32_t tmem_sh;
  __shared__ int ok_sh;
  __shared__ float cs[4][BN]; /* per-quadrant column sums (UMMA_DGRAD with colsum) */
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  /* 1024-byte aligned operand tiles (the swizzle pattern is a function of the address) */
  unsigned char *base = dsm + ((1024u - (su32(dsm) & 1023u)) & 1023u);
  unsigned char *sa = base, *sb = base + tile_bytes(g.a_mn, BM, g.K);
  /* epilogue staging, 8 x 32 x 33 floats, over the operand tiles once the MMAs are done */
  unsigned char *sst = base;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN, k0 = blockIdx.z * g.K;
  const int ns = k_slices(g.K);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(&tmem_sh)),
                 "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int i = 0; i <= MAX_SLICES; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bar[i])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  if (tid == 0) {
    /* every slice's loads in flight first, each on its own barrier */
    for (int sl = 0; sl < ns; ++sl) {
      const uint32_t bytes =
          slice_bytes(g.a_mn, BM, g.K, ns) + slice_bytes(g.b_mn, BN, g.K, ns);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                       su32(&bar[sl])),
                   "r"(bytes)
                   : "memory");
      load_slice(sa, &ta, g.a_mn, BM, g.K, m0, k0, sl, ns, &bar[sl]);
      load_slice(sb, &tb, g.b_mn, BN, g.K, n0, k0, sl, ns, &bar[sl]);
    }
    /* kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, majors, N >> 3,
     * M >> 4 */
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)g.a_mn << 15) |
                           ((uint32_t)g.b_mn << 16) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    const uint32_t a_s = su32(sa), b_s = su32(sb);
    const int steps = g.K / 16, per = ns > 1 ? 4 : steps;
    int ok = 1;
    for (int sl = 0; sl < ns && ok; ++sl) {
      if (!bar_wait(&bar[sl], 0)) {
        ok = 0;
        break;
      }
      tc_fence_after();
      for (int ks = sl * per; ks < min(steps, (sl + 1) * per); ++ks) {
        const uint64_t ad = op_desc(a_s, g.a_mn, BM, g.K, ks);
        const uint64_t bd = op_desc(b_s, g.b_mn, BN, g.K, ks);
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(ks > 0 ? 1 : 0)
            : "memory");
      }
    }
    if (ok) {
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              su32(&bar[MAX_SLICES]))
          : "memory");
    } else {
      /* a slice never landed: let the loads still in flight finish (bounded) before the CTA
       * reuses or gives up its shared memory */
      for (int sl = 0; sl < ns; ++sl) bar_wait(&bar[sl], 0);
      atomicExch(g.err, 1);
    }
    ok_sh = ok;
  }
  __syncthreads();
  bool ok = ok_sh != 0;
  if (ok && !bar_wait(&bar[MAX_SLICES], 0)) {
    ok = false;
    if (lane == 0) atomicExch(g.err, 2);
  }
  ok = __all_sync(0xffffffffu, ok);
  tc_fence_after();
  const UmmaEpilogue &e = g.e;
  if (ok) {
    /* warp w reads accumulator lanes 32 (w % 4) .. +31 (its lane quadrant) and the columns of
     * half w / 4 of the tile, 32 at a time */
    const int q = warp & 3, c_begin = (warp >> 2) * (BN / 2);
    const int row0 = m0 + q * 32, rows = min(32, g.M - row0);
    float *of = e.Of ? e.Of + (size_t)blockIdx.z * e.split_stride : nullptr;
    float *stage = reinterpret_cast<float *>(sst) + warp * (32 * 33);
#pragma unroll 1
    for (int c0 = c_begin; c0 < c_begin + BN / 2; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
      const int nb = n0 + c0;
      float csum = 0.0f;
      if (nb < g.N && rows > 0) {
        if (e.kind == UMMA_F32 && e.trans) {
          /* lanes = consecutive rows: Of[n][row] is already coalesced */
          if (lane < rows) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (nb + j < g.N) of[(size_t)(nb + j) * e.ldo + row0 + lane] = __uint_as_float(v[j]);
          }
        } else {
          /* turn the block around in shared memory so that lanes run along a row */
#pragma unroll
          for (int j = 0; j < 32; ++j) stage[lane * 33 + j] = __uint_as_float(v[j]);
          __syncwarp();
          const int n = nb + lane;
          const bool col = n < g.N;
          const size_t o0 = (size_t)row0 * e.ldo + n;
          if (e.kind == UMMA_FWD) {
            const float bn = col ? e.bias[n] : 0.0f;
#pragma unroll 4
            for (int i = 0; i < rows; ++i) {
              const float z = stage[i * 33 + lane] + bn;
              if (col) {
                if (e.Z) e.Z[o0 + (size_t)i * e.ldo] = z;
                e.Ob[o0 + (size_t)i * e.ldo] = __float2bfloat16_rn(mlp_silu(z));
              }
            }
          } else if (e.kind == UMMA_DGRAD) {
            float zr[32]; /* every load in flight before the arithmetic */
#pragma unroll
            for (int i = 0; i < 32; ++i)
              zr[i] = (col && i < rows) ? e.Zin[o0 + (size_t)i * e.ldo] : 0.0f;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
              if (col && i < rows) {
                const bf16 d = __float2bfloat16_rn(stage[i * 33 + lane] * mlp_silu_grad(zr[i]));
                e.Ob[o0 + (size_t)i * e.ldo] = d;
                csum += __bfloat162float(d);
              }
            }
          } else {
#pragma unroll 4
            for (int i = 0; i < rows; ++i)
              if (col) of[o0 + (size_t)i * e.ldo] = stage[i * 33 + lane];
          }
          __syncwarp();
        }
      }
      if (e.colsum) cs[q][c0 + lane] = csum;
    }
  }
  tc_fence_before();
  __syncthreads();
  /* per-tile column sums of the BF16 dZ (the next layer's bias gradient), quadrants added in a
   * fixed order */
  if (e.colsum && ok_sh && tid < BN && n0 + tid < g.N)
    e.colsum[(size_t)blockIdx.x * g.N + n0 + tid] =
        ((cs[0][tid] + cs[1][tid]) + cs[2][tid]) + cs[3][tid];
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)BN)
                 : "memory");
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  /* looked up once (thread-safe static initialisation) */
  static const EncodeTiled fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiled>(p);
    return (EncodeTiled) nullptr;
  }();
  return fn;
}

/* the operand as a 2-D tensor map: dims {cols, rows}, boxes 64 x box_rows, 128-byte swizzle,
 * zero fill out of bounds */
int make_map(CUtensorMap *m, const UmmaOperand &o, int box_rows) {
  EncodeTiled fn = encoder();
  if (!fn) return -5;
  if (o.cols % 8 || o.cols < 1 || o.rows < 1 || (reinterpret_cast<uintptr_t>(o.p) & 15) ||
      box_rows < 1 || box_rows > 256)
    return -1;
  const cuuint64_t dims[2] = {(cuuint64_t)o.cols, (cuuint64_t)o.rows};
  const cuuint64_t strides[1] = {(cuuint64_t)o.cols * 2};
  const cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1u, 1u};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(o.p), dims,
            strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
             ? 0
             : -5;
}

template <int BN>
int launch(const UmmaOperand &A, const UmmaOperand &B, int M, int N, int K, int splits,
           const UmmaEpilogue &e, int *err, cudaStream_t s) {
  /* the shared-memory limit is a per-device attribute: set once per device */
  static std::atomic<unsigned long long> attr_set{0};
  const size_t smem =
      std::max<size_t>(tile_bytes(A.mn_major, BM, K) + tile_bytes(B.mn_major, BN, K),
                       (size_t)STAGE_BYTES) + 1024;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -2;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    if (cudaFuncSetAttribute(umma_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             256 * 256 + BN * 512 + 1024) != cudaSuccess)
      return -2;
    attr_set.fetch_or(bit);
  }
  CUtensorMap ta, tb;
  int rc;
  /* MN-major boxes are one K slice high (the whole chunk when it is not a multiple of 64) */
  const int mn_box = k_slices(K) > 1 ? 64 : K;
  if ((rc = make_map(&ta, A, A.mn_major ? mn_box : BM))) return rc;
  if ((rc = make_map(&tb, B, B.mn_major ? mn_box : BN))) return rc;
  UmmaArgs g;
  g.M = M;
  g.N = N;
  g.K = K;
  g.a_mn = A.mn_major;
  g.b_mn = B.mn_major;
  g.e = e;
  g.err = err;
  const dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
  umma_kernel<BN><<<grid, 256, smem, s>>>(ta, tb, g);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

int umma_gemm(const UmmaOperand &A, const UmmaOperand &B, int M, int N, int K, int splits,
              const UmmaEpilogue &e, int *err, cudaStream_t s) {
  if (M < 1 || N < 1 || K < 16 || K > 256 || K % 16 || splits < 1 || !err) return -1;
  if (splits > 1 && !(A.mn_major && B.mn_major)) return -1;
  if ((e.kind == UMMA_FWD && (!e.bias || !e.Ob)) || (e.kind == UMMA_DGRAD && (!e.Zin || !e.Ob)) ||
      (e.kind == UMMA_F32 && !e.Of))
    return -1;
  /* 64-wide tiles when 128-wide ones would leave fewer than two CTAs per SM: two 64-wide CTAs
   * share an SM, and one's epilogue overlaps the other's loads and products */
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0)
      num_sms = n;
    else
      num_sms = 148;
  }
  const long long tiles128 = (long long)((M + BM - 1) / BM) * ((N + 127) / 128) * splits;
  return (N <= 64 || tiles128 < 2LL * num_sms) ? launch<64>(A, B, M, N, K, splits, e, err, s)
                                               : launch<128>(A, B, M, N, K, splits, e, err, s);
}

}  // namespace gd
