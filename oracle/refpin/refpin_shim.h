/*
 * refpin_shim.h -- lets the reference's CUDA kernel source compile as host C++ so that its
 * own arithmetic (CalcEnergy_d, CombineEnergy_d, CalcMcc_d, InitRefMatrix_d, Move_d,
 * Accept_d, RecordLigand_d, ExchangeReplicas_d) runs on the CPU as one thread of one block.
 * TEST INFRASTRUCTURE ONLY (builds oracle/_ref/refpin from the reference tree in place).
 *
 * Block geometry seen by the reference code: blockDim = (1,1,1), blockIdx = 0; the compile-
 * time tile macros are TperB = 1 and BDx = 128 / BDy = 1 (BDx only sizes shared arrays and
 * the CalcRmsd_d loop, whose value is not used). Statements that the reference spreads over
 * threads (Move_d dims, Accept_d copies, the init energy copy) are issued by the driver once
 * per emulated thread, in an order that respects the reference's __syncthreads phases.
 */
#ifndef REFPIN_SHIM_H
#define REFPIN_SHIM_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <deque>

struct shim_dim3 { unsigned x, y, z; };
static shim_dim3 threadIdx = {0, 0, 0};
static shim_dim3 blockIdx = {0, 0, 0};
static shim_dim3 blockDim = {1, 1, 1};
static shim_dim3 gridDim = {1, 1, 1};

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static
#define __forceinline__ inline
#define __syncthreads() ((void)0)
#define CUDA_LDG_D(d) (d)
#define CUDA_LDG_P(p) (*(p))

/* scripted uniform stream standing in for curand_uniform */
struct curandState { int unused; };
static std::deque<float> g_shim_uniforms;
static long g_shim_underflow = 0;
static inline void curand_init(unsigned long long, unsigned long long, unsigned long long,
                               curandState *) {}
static inline float curand_uniform(curandState *) {
  if (g_shim_uniforms.empty()) { ++g_shim_underflow; return 0.5f; }
  const float u = g_shim_uniforms.front();
  g_shim_uniforms.pop_front();
  return u;
}

#endif
