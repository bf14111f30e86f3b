// The learned Riemann warm start on the GPU: feature extraction, FP32
// training (fused forward + backward per 64-sample tile, Adam), and BF16
// tensor-core inference (mma.sync m16n8k16, FP32 accumulation).
//
// Training: each CTA takes 64 samples of the minibatch, keeps the whole
// network (9473 FP32 parameters) and the four activation tiles in shared
// memory, runs forward and backward, and adds its parameter gradients into a
// global FP32 gradient with atomics; an Adam kernel then updates the master
// weights. Inference: each warp pushes 16 samples at a time through the three
// hidden layers as register-resident MMA fragments; the FP32 accumulator of
// one layer, after tanh, is repacked in registers as the BF16 A operand of
// the next, so activations never touch shared memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/m2c_gpu.h"
#include "mlp.cuh"

namespace m2c {

void set_last_error(const char* msg);

constexpr int TR_S = 64;        // samples per training CTA
constexpr int TR_T = 256;       // threads per training CTA
constexpr int TR_LD = MLP_H + 1;  // padded activation row (conflict-free column walks)

struct TrainSmem {
  float w[MLP_NPARAM];
  float x[TR_S][MLP_IN + 1];
  float h1[TR_S][TR_LD];
  float h2[TR_S][TR_LD];
  float h3[TR_S][TR_LD];
  float ga[TR_S][TR_LD];
  float gb[TR_S][TR_LD];
  float out[TR_S];
  float dout[TR_S];
  float red[TR_T / 32];
};

// o[s][j] = tanh(b[j] + sum_k in[s][k] W[j][k]) for the tile; lanes walk samples.
template <int K>
__device__ __forceinline__ void layer_fwd(const float* W, const float* b, const float (*in)[TR_LD], const float (*inx)[MLP_IN + 1],
                                          float (*o)[TR_LD], int ns) {
  for (int q = threadIdx.x; q < TR_S * MLP_H; q += TR_T) {
    const int s = q % TR_S, j = q / TR_S;
    float acc = b[j];
    if (s < ns) {
      for (int k = 0; k < K; k++) acc += (inx ? inx[s][k] : in[s][k]) * W[j * K + k];
    }
    o[s][j] = tanhf(acc);
  }
}

// Forward (and, if grad, backward) of one tile of the minibatch.
// mode 0: loss + gradients; mode 1: forward only, writes yhat.
__global__ void __launch_bounds__(TR_T) k_mlp_tile(const float* params, float* grad, const float* X, const float* y,
                                                   const int* idx, long long base, int count, float inv_batch,
                                                   float* loss, float* yhat, int mode) {
  extern __shared__ __align__(16) unsigned char mlp_smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(mlp_smem_raw);
  const int tid = threadIdx.x;
  const long long t0 = (long long)blockIdx.x * TR_S;
  if (t0 >= count) return;
  const int ns = (int)(count - t0 < TR_S ? count - t0 : TR_S);
  for (int q = tid; q < MLP_NPARAM; q += TR_T) S.w[q] = params[q];
  for (int q = tid; q < TR_S * MLP_IN; q += TR_T) {
    const int s = q / MLP_IN, k = q % MLP_IN;
    float v = 0.f;
    if (s < ns) {
      const long long r = idx ? idx[base + t0 + s] : base + t0 + s;
      v = X[r * MLP_IN + k];
    }
    S.x[s][k] = v;
  }
  __syncthreads();
  layer_fwd<MLP_IN>(S.w + MLP_OW1, S.w + MLP_OB1, nullptr, S.x, S.h1, ns);
  __syncthreads();
  layer_fwd<MLP_H>(S.w + MLP_OW2, S.w + MLP_OB2, S.h1, nullptr, S.h2, ns);
  __syncthreads();
  layer_fwd<MLP_H>(S.w + MLP_OW3, S.w + MLP_OB3, S.h2, nullptr, S.h3, ns);
  __syncthreads();
  for (int s = tid; s < TR_S; s += TR_T) {
    float acc = S.w[MLP_OB4];
    for (int k = 0; k < MLP_H; k++) acc += S.h3[s][k] * S.w[MLP_OW4 + k];
    S.out[s] = acc;
    float d = 0.f;
    if (s < ns) {
      const long long r = idx ? idx[base + t0 + s] : base + t0 + s;
      if (mode == 1) {
        yhat[r] = acc;
      } else {
        const float e = acc - y[r];
        d = 2.f * e * inv_batch;
        atomicAdd(loss, e * e * inv_batch);
      }
    }
    S.dout[s] = d;
  }
  if (mode == 1) return;
  __syncthreads();
  // output layer: g3 = dout w4 (1 - h3^2); dw4, db4
  for (int q = tid; q < TR_S * MLP_H; q += TR_T) {
    const int s = q % TR_S, j = q / TR_S;
    const float h = S.h3[s][j];
    S.ga[s][j] = S.dout[s] * S.w[MLP_OW4 + j] * (1.f - h * h);
  }
  for (int j = tid; j < MLP_H + 1; j += TR_T) {
    float acc = 0.f;
    for (int s = 0; s < ns; s++) acc += S.dout[s] * (j < MLP_H ? S.h3[s][j] : 1.f);
    atomicAdd(&grad[j < MLP_H ? MLP_OW4 + j : MLP_OB4], acc);
  }
  __syncthreads();
  // hidden layers 3 and 2: dW = g^T h_prev, db = sum g, g_prev = (g W) (1 - h_prev^2)
  float(*g)[TR_LD] = S.ga;
  float(*gn)[TR_LD] = S.gb;
  const float(*hprev[2])[TR_LD] = {S.h2, S.h1};
  const int ow[2] = {MLP_OW3, MLP_OW2}, ob[2] = {MLP_OB3, MLP_OB2};
  for (int L = 0; L < 2; L++) {
    const float* W = S.w + ow[L];
    for (int q = tid; q < MLP_H * (MLP_H + 1); q += TR_T) {
      const int j = q / (MLP_H + 1), k = q % (MLP_H + 1);
      float acc = 0.f;
      for (int s = 0; s < ns; s++) acc += g[s][j] * (k < MLP_H ? hprev[L][s][k] : 1.f);
      atomicAdd(&grad[k < MLP_H ? ow[L] + j * MLP_H + k : ob[L] + j], acc);
    }
    for (int q = tid; q < TR_S * MLP_H; q += TR_T) {
      const int s = q % TR_S, k = q / TR_S;
      float acc = 0.f;
      for (int j = 0; j < MLP_H; j++) acc += g[s][j] * W[j * MLP_H + k];
      const float h = hprev[L][s][k];
      gn[s][k] = acc * (1.f - h * h);
    }
    __syncthreads();
    float(*t)[TR_LD] = g;
    g = gn;
    gn = t;
  }
  // first layer: dW1 = g1^T x, db1
  for (int q = tid; q < MLP_H * (MLP_IN + 1); q += TR_T) {
    const int j = q / (MLP_IN + 1), k = q % (MLP_IN + 1);
    float acc = 0.f;
    for (int s = 0; s < ns; s++) acc += g[s][j] * (k < MLP_IN ? S.x[s][k] : 1.f);
    atomicAdd(&grad[k < MLP_IN ? MLP_OW1 + j * MLP_IN + k : MLP_OB1 + j], acc);
  }
}

__global__ void k_adam(float* w, float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.f;
  }
}

// ---------------------------------------------------------------------------
// BF16 tensor-core inference
// ---------------------------------------------------------------------------
constexpr int IN_LD1 = 24;  // bf16 row stride of W1 / X tiles (conflict-free fragment loads)
constexpr int IN_LD = 72;   // bf16 row stride of W2 / W3

struct InferSmem {
  __nv_bfloat16 w1[MLP_H][IN_LD1];
  __nv_bfloat16 w2[MLP_H][IN_LD];
  __nv_bfloat16 w3[MLP_H][IN_LD];
  float b1[MLP_H], b2[MLP_H], b3[MLP_H], w4[MLP_H];
  float b4, ymean, ystd;
  float xmean[MLP_IN], xstd[MLP_IN];
  __nv_bfloat16 x[8][16][IN_LD1];  // one 16-sample tile per warp
};

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One hidden layer on a 16-row tile: acc[j] (8 n-tiles of 8 columns) = A W^T + b.
template <int KT, int LD>
__device__ __forceinline__ void mma_layer(const unsigned (*a)[4], const __nv_bfloat16 (*W)[LD], const float* b,
                                          float (*acc)[4], int g, int t) {
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const float c0 = b[8 * j + 2 * t], c1 = b[8 * j + 2 * t + 1];
    acc[j][0] = c0; acc[j][1] = c1; acc[j][2] = c0; acc[j][3] = c1;
#pragma unroll
    for (int kk = 0; kk < KT; kk++) {
      unsigned bb[2];
      bb[0] = *reinterpret_cast<const unsigned*>(&W[8 * j + g][16 * kk + 2 * t]);
      bb[1] = *reinterpret_cast<const unsigned*>(&W[8 * j + g][16 * kk + 8 + 2 * t]);
      mma_bf16(acc[j], a[kk], bb);
    }
  }
}

// tanh of two adjacent accumulator tiles repacked as one BF16 A k-tile
__device__ __forceinline__ void to_a(float (*acc)[4], unsigned (*a)[4]) {
#pragma unroll
  for (int kk = 0; kk < 4; kk++) {
    a[kk][0] = pack_bf16(tanhf(acc[2 * kk][0]), tanhf(acc[2 * kk][1]));
    a[kk][1] = pack_bf16(tanhf(acc[2 * kk][2]), tanhf(acc[2 * kk][3]));
    a[kk][2] = pack_bf16(tanhf(acc[2 * kk + 1][0]), tanhf(acc[2 * kk + 1][1]));
    a[kk][3] = pack_bf16(tanhf(acc[2 * kk + 1][2]), tanhf(acc[2 * kk + 1][3]));
  }
}

// Network weights (FP32 master + normalisation) staged into shared memory as BF16.
__device__ void stage_weights(InferSmem& S, const float* params, const float* norm) {
  for (int q = threadIdx.x; q < MLP_H * MLP_IN; q += blockDim.x)
    S.w1[q / MLP_IN][q % MLP_IN] = __float2bfloat16_rn(params[MLP_OW1 + q]);
  for (int q = threadIdx.x; q < MLP_H * MLP_H; q += blockDim.x) {
    S.w2[q / MLP_H][q % MLP_H] = __float2bfloat16_rn(params[MLP_OW2 + q]);
    S.w3[q / MLP_H][q % MLP_H] = __float2bfloat16_rn(params[MLP_OW3 + q]);
  }
  for (int q = threadIdx.x; q < MLP_H; q += blockDim.x) {
    S.b1[q] = params[MLP_OB1 + q];
    S.b2[q] = params[MLP_OB2 + q];
    S.b3[q] = params[MLP_OB3 + q];
    S.w4[q] = params[MLP_OW4 + q];
  }
  for (int q = threadIdx.x; q < MLP_IN; q += blockDim.x) {
    S.xmean[q] = norm[q];
    S.xstd[q] = norm[MLP_IN + q];
  }
  if (threadIdx.x == 0) {
    S.b4 = params[MLP_OB4];
    S.ymean = norm[2 * MLP_IN];
    S.ystd = norm[2 * MLP_IN + 1];
  }
}

// Rows of raw features X [n][16] (valid[r] != 0) -> network output in target
// units (log(pstar / pac)), BF16 weights and activations, FP32 accumulation.
// 8 warps per CTA, 16 rows per warp per iteration.
__global__ void __launch_bounds__(256) k_mlp_infer(const float* params, const float* norm, const float* X,
                                                   const int* valid, int n, const int* ndev, float* yout) {
  __shared__ InferSmem S;
  if (ndev && *ndev < n) n = *ndev;  // rows counted on the device (n is then the capacity)
  stage_weights(S, params, norm);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int tiles = (n + 15) / 16;
  for (int tile = blockIdx.x * 8 + warp; tile < tiles; tile += gridDim.x * 8) {
    // normalised features of 16 rows, two lanes per row
    {
      const int r = lane >> 1, half = lane & 1;
      const long long row = (long long)tile * 16 + r;
      for (int k = half * 8; k < half * 8 + 8; k++) {
        float v = 0.f;
        if (row < n && valid[row]) v = (X[row * MLP_IN + k] - S.xmean[k]) / S.xstd[k];
        S.x[warp][r][k] = __float2bfloat16_rn(v);
      }
    }
    __syncwarp();
    unsigned a1[1][4];
    a1[0][0] = *reinterpret_cast<const unsigned*>(&S.x[warp][g][2 * t]);
    a1[0][1] = *reinterpret_cast<const unsigned*>(&S.x[warp][g + 8][2 * t]);
    a1[0][2] = *reinterpret_cast<const unsigned*>(&S.x[warp][g][8 + 2 * t]);
    a1[0][3] = *reinterpret_cast<const unsigned*>(&S.x[warp][g + 8][8 + 2 * t]);
    __syncwarp();
    float acc[8][4];
    unsigned a[4][4];
    mma_layer<1, IN_LD1>(a1, S.w1, S.b1, acc, g, t);
    to_a(acc, a);
    mma_layer<4, IN_LD>(a, S.w2, S.b2, acc, g, t);
    to_a(acc, a);
    mma_layer<4, IN_LD>(a, S.w3, S.b3, acc, g, t);
    // output: tanh(h3) . w4 + b4, rows g and g + 8, reduced over the quad
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const float w0 = S.w4[8 * j + 2 * t], w1 = S.w4[8 * j + 2 * t + 1];
      s0 += tanhf(acc[j][0]) * w0 + tanhf(acc[j][1]) * w1;
      s1 += tanhf(acc[j][2]) * w0 + tanhf(acc[j][3]) * w1;
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    if (t == 0) {
      const long long r0 = (long long)tile * 16 + g, r1 = r0 + 8;
      if (r0 < n) yout[r0] = (s0 + S.b4) * S.ystd + S.ymean;
      if (r1 < n) yout[r1] = (s1 + S.b4) * S.ystd + S.ymean;
    }
  }
}

// Features of per-pair problems (materials eos[2q], eos[2q+1]).
__global__ void k_mlp_features_pairs(const Eos<double>* eos, int n, const double* VL, const double* VR,
                                     const double* dir, float* X, double* P, int* valid) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    double sc[2] = {0.0, 0.0};
    const bool ok = mlp_features(eos[2 * q], eos[2 * q + 1], VL + 5 * q, VR + 5 * q, dir + 3 * q, X + (long long)q * MLP_IN, sc);
    P[2 * q] = sc[0];
    P[2 * q + 1] = sc[1];
    valid[q] = ok ? 1 : 0;
  }
}

__global__ void k_mlp_to_pressure(const float* y, const double* P, const int* valid, int n, const int* ndev,
                                  double* p) {
  if (ndev && *ndev < n) n = *ndev;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    p[q] = valid[q] ? P[2 * q] * exp((double)y[q]) - P[2 * q + 1] : NAN;
}

}  // namespace m2c

using namespace m2c;

struct m2cg_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* w = nullptr;     // [NPARAM] FP32 master weights
  float* norm = nullptr;  // [NNORM]
  std::vector<float> hnorm;
};

static m2cg_status mfail(m2cg_status st, const char* msg) {
  set_last_error(msg);
  return st;
}

static Eos<double> mlp_eos(const m2cg_material& m) {
  MatParams p;
  p.kind = m.eos; p.gam = m.gamma; p.pc = m.p_c; p.b = m.b; p.q = m.q;
  p.rhomin = m.rhomin; p.pmin = m.pmin; p.rhomax = m.rhomax; p.pmax = m.pmax;
  p.failsafe_density = m.failsafe_density;
  return make_eos<double>(p);
}

extern "C" m2cg_status m2cg_mlp_create(unsigned long long seed, m2cg_mlp** out) {
  if (!out) return mfail(M2CG_ERR_ARG, "null argument");
  m2cg_mlp* m = new m2cg_mlp;
  cudaGetDevice(&m->device);
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc((void**)&m->w, MLP_NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc((void**)&m->norm, MLP_NNORM * sizeof(float)) != cudaSuccess) {
    m2cg_mlp_destroy(m);
    return mfail(M2CG_ERR_CUDA, "m2cg_mlp_create: device allocation failed");
  }
  // Glorot-uniform weights, zero biases
  std::mt19937_64 rng(seed);
  std::vector<float> w(MLP_NPARAM, 0.f);
  auto init = [&](int off, int fan_out, int fan_in) {
    const double a = std::sqrt(6.0 / (fan_in + fan_out));
    std::uniform_real_distribution<double> U(-a, a);
    for (int i = 0; i < fan_out * fan_in; i++) w[off + i] = (float)U(rng);
  };
  init(MLP_OW1, MLP_H, MLP_IN);
  init(MLP_OW2, MLP_H, MLP_H);
  init(MLP_OW3, MLP_H, MLP_H);
  init(MLP_OW4, 1, MLP_H);
  m->hnorm.assign(MLP_NNORM, 0.f);
  for (int k = 0; k < MLP_IN; k++) m->hnorm[MLP_IN + k] = 1.f;
  m->hnorm[2 * MLP_IN + 1] = 1.f;
  if (cudaMemcpy(m->w, w.data(), MLP_NPARAM * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->norm, m->hnorm.data(), MLP_NNORM * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    m2cg_mlp_destroy(m);
    return mfail(M2CG_ERR_CUDA, "m2cg_mlp_create: upload failed");
  }
  *out = m;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_mlp_destroy(m2cg_mlp* m) {
  if (!m) return M2CG_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->w);
  cudaFree(m->norm);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_mlp_get_params(const m2cg_mlp* m, float* params, float* norm) {
  if (!m) return mfail(M2CG_ERR_ARG, "null argument");
  if (params && cudaMemcpy(params, m->w, MLP_NPARAM * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return mfail(M2CG_ERR_CUDA, "read-back failed");
  if (norm) std::copy(m->hnorm.begin(), m->hnorm.end(), norm);
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_mlp_set_params(m2cg_mlp* m, const float* params, const float* norm) {
  if (!m) return mfail(M2CG_ERR_ARG, "null argument");
  if (params && cudaMemcpy(m->w, params, MLP_NPARAM * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return mfail(M2CG_ERR_CUDA, "upload failed");
  if (norm) {
    m->hnorm.assign(norm, norm + MLP_NNORM);
    if (cudaMemcpy(m->norm, norm, MLP_NNORM * 4, cudaMemcpyHostToDevice) != cudaSuccess)
      return mfail(M2CG_ERR_CUDA, "upload failed");
  }
  return M2CG_OK;
}

static cudaError_t tile_smem_setup() {
  return cudaFuncSetAttribute(k_mlp_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
}

extern "C" m2cg_status m2cg_mlp_loss_grad(m2cg_mlp* m, const float* Xn, const float* yn, int n, float* loss,
                                          float* grad) {
  if (!m || !Xn || !yn || n < 1 || !loss || !grad) return mfail(M2CG_ERR_ARG, "null argument");
  float *dX = nullptr, *dy = nullptr, *dg = nullptr, *dl = nullptr;
  m2cg_status st = M2CG_OK;
  if (cudaMalloc((void**)&dX, (size_t)n * MLP_IN * 4) != cudaSuccess || cudaMalloc((void**)&dy, (size_t)n * 4) != cudaSuccess ||
      cudaMalloc((void**)&dg, MLP_NPARAM * 4) != cudaSuccess || cudaMalloc((void**)&dl, 4) != cudaSuccess)
    st = mfail(M2CG_ERR_NOMEM, "allocation failed");
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if (!st) {
    ck(tile_smem_setup());
    ck(cudaMemcpyAsync(dX, Xn, (size_t)n * MLP_IN * 4, cudaMemcpyHostToDevice, m->stream));
    ck(cudaMemcpyAsync(dy, yn, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    ck(cudaMemsetAsync(dg, 0, MLP_NPARAM * 4, m->stream));
    ck(cudaMemsetAsync(dl, 0, 4, m->stream));
    if (e == cudaSuccess) {
      k_mlp_tile<<<(n + TR_S - 1) / TR_S, TR_T, sizeof(TrainSmem), m->stream>>>(m->w, dg, dX, dy, nullptr, 0, n,
                                                                                 1.f / n, dl, nullptr, 0);
      ck(cudaGetLastError());
    }
    ck(cudaMemcpyAsync(grad, dg, MLP_NPARAM * 4, cudaMemcpyDeviceToHost, m->stream));
    ck(cudaMemcpyAsync(loss, dl, 4, cudaMemcpyDeviceToHost, m->stream));
    ck(cudaStreamSynchronize(m->stream));
    if (e != cudaSuccess) st = mfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaFree(dX); cudaFree(dy); cudaFree(dg); cudaFree(dl);
  return st;
}

extern "C" m2cg_status m2cg_mlp_train(m2cg_mlp* m, const float* X, const float* y, int n, int steps, int batch,
                                      float lr, unsigned long long seed, float* final_loss) {
  if (!m || !X || !y || n < 2 || steps < 1 || batch < 1) return mfail(M2CG_ERR_ARG, "bad argument");
  batch = std::min(batch, n);
  // normalisation from the data (FP64 sums)
  std::vector<double> mean(MLP_IN + 1, 0.0), var(MLP_IN + 1, 0.0);
  for (long long r = 0; r < n; r++) {
    for (int k = 0; k < MLP_IN; k++) mean[k] += X[r * MLP_IN + k];
    mean[MLP_IN] += y[r];
  }
  for (auto& v : mean) v /= n;
  for (long long r = 0; r < n; r++) {
    for (int k = 0; k < MLP_IN; k++) {
      const double d = X[r * MLP_IN + k] - mean[k];
      var[k] += d * d;
    }
    const double d = y[r] - mean[MLP_IN];
    var[MLP_IN] += d * d;
  }
  std::vector<float> hn(MLP_NNORM);
  std::vector<float> Xn((size_t)n * MLP_IN), yn(n);
  for (int k = 0; k <= MLP_IN; k++) {
    double sd = std::sqrt(var[k] / n);
    if (!(sd > 1e-12)) sd = 1.0;
    if (k < MLP_IN) {
      hn[k] = (float)mean[k];
      hn[MLP_IN + k] = (float)sd;
    } else {
      hn[2 * MLP_IN] = (float)mean[k];
      hn[2 * MLP_IN + 1] = (float)sd;
    }
  }
  for (long long r = 0; r < n; r++) {
    for (int k = 0; k < MLP_IN; k++) Xn[r * MLP_IN + k] = (X[r * MLP_IN + k] - hn[k]) / hn[MLP_IN + k];
    yn[r] = (y[r] - hn[2 * MLP_IN]) / hn[2 * MLP_IN + 1];
  }
  m->hnorm = hn;
  float *dX = nullptr, *dy = nullptr, *dg = nullptr, *dm = nullptr, *dv = nullptr, *dl = nullptr;
  int* didx = nullptr;
  m2cg_status st = M2CG_OK;
  if (cudaMalloc((void**)&dX, Xn.size() * 4) != cudaSuccess || cudaMalloc((void**)&dy, (size_t)n * 4) != cudaSuccess ||
      cudaMalloc((void**)&dg, MLP_NPARAM * 4) != cudaSuccess || cudaMalloc((void**)&dm, MLP_NPARAM * 4) != cudaSuccess ||
      cudaMalloc((void**)&dv, MLP_NPARAM * 4) != cudaSuccess || cudaMalloc((void**)&dl, 4 * (size_t)steps) != cudaSuccess ||
      cudaMalloc((void**)&didx, (size_t)n * 4) != cudaSuccess)
    st = mfail(M2CG_ERR_NOMEM, "allocation failed");
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if (!st) {
    ck(tile_smem_setup());
    ck(cudaMemcpyAsync(m->norm, hn.data(), MLP_NNORM * 4, cudaMemcpyHostToDevice, m->stream));
    ck(cudaMemcpyAsync(dX, Xn.data(), Xn.size() * 4, cudaMemcpyHostToDevice, m->stream));
    ck(cudaMemcpyAsync(dy, yn.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    ck(cudaMemsetAsync(dg, 0, MLP_NPARAM * 4, m->stream));
    ck(cudaMemsetAsync(dm, 0, MLP_NPARAM * 4, m->stream));
    ck(cudaMemsetAsync(dv, 0, MLP_NPARAM * 4, m->stream));
    ck(cudaMemsetAsync(dl, 0, 4 * (size_t)steps, m->stream));
    std::mt19937_64 rng(seed);
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    long long pos = n;  // force a shuffle on the first step
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double c1 = 1.0, c2 = 1.0;
    for (int step = 0; step < steps && e == cudaSuccess; step++) {
      if (pos + batch > n) {
        ck(cudaStreamSynchronize(m->stream));  // the previous permutation may still be read
        std::shuffle(perm.begin(), perm.end(), rng);
        ck(cudaMemcpyAsync(didx, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
        pos = 0;
      }
      k_mlp_tile<<<(batch + TR_S - 1) / TR_S, TR_T, sizeof(TrainSmem), m->stream>>>(
          m->w, dg, dX, dy, didx, pos, batch, 1.f / batch, dl + step, nullptr, 0);
      pos += batch;
      c1 *= b1;
      c2 *= b2;
      // cosine decay to lr/20
      const double frac = (double)step / std::max(1, steps - 1);
      const float lrs = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * frac))));
      k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, m->stream>>>(m->w, dg, dm, dv, MLP_NPARAM, lrs, b1, b2, eps,
                                                             (float)(1.0 - c1), (float)(1.0 - c2));
      ck(cudaGetLastError());
    }
    std::vector<float> losses(steps);
    ck(cudaMemcpyAsync(losses.data(), dl, 4 * (size_t)steps, cudaMemcpyDeviceToHost, m->stream));
    ck(cudaStreamSynchronize(m->stream));
    if (e != cudaSuccess) {
      st = mfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
    } else if (final_loss) {
      // mean of the last 5% of steps (normalised target units)
      const int w = std::max(1, steps / 20);
      double s = 0;
      for (int i = steps - w; i < steps; i++) s += losses[i];
      *final_loss = (float)(s / w);
    }
  }
  cudaFree(dX); cudaFree(dy); cudaFree(dg); cudaFree(dm); cudaFree(dv); cudaFree(dl); cudaFree(didx);
  return st;
}

// Shared by the host entry points: features -> BF16 inference -> pressure.
static cudaError_t infer_rows(m2cg_mlp* m, const float* dX, const int* dvalid, int n, float* dyout) {
  const int tiles = (n + 15) / 16;
  const int grid = std::max(1, std::min((tiles + 7) / 8, 148 * 4));
  k_mlp_infer<<<grid, 256, 0, m->stream>>>(m->w, m->norm, dX, dvalid, n, nullptr, dyout);
  return cudaGetLastError();
}

namespace m2c {
// Device-side proposals for rows of raw features (used by the batched tubes):
// warm[r] = P[2r] exp(network(X[r])) - P[2r+1] where valid[r], else NaN.
cudaError_t mlp_warm_device(const m2cg_mlp* m, cudaStream_t s, const float* X, const int* valid, const double* P,
                            int n, float* y, double* warm, const int* ndev) {
  const int tiles = (n + 15) / 16;
  const int grid = std::max(1, std::min((tiles + 7) / 8, 148 * 4));
  k_mlp_infer<<<grid, 256, 0, s>>>(m->w, m->norm, X, valid, n, ndev, y);
  k_mlp_to_pressure<<<std::max(1, std::min((n + 255) / 256, 148 * 8)), 256, 0, s>>>(y, P, valid, n, ndev, warm);
  return cudaGetLastError();
}
}  // namespace m2c

// Problems with per-pair materials: features (mode 0) or the BF16 proposal
// of p* (mode 1).
static m2cg_status pairs_common(m2cg_mlp* m, const m2cg_material* mats, int n, const double* VL, const double* VR,
                                const double* dir, float* X_out, double* P_out, int* valid_out, double* p_out,
                                int mode) {
  std::vector<Eos<double>> heos(2 * (size_t)n);
  for (int q = 0; q < 2 * n; q++) heos[q] = mlp_eos(mats[q]);
  cudaStream_t s = m ? m->stream : nullptr;
  bool own = false;
  if (!s) {
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return mfail(M2CG_ERR_CUDA, "no stream");
    own = true;
  }
  Eos<double>* deos = nullptr;
  double *dVL = nullptr, *dVR = nullptr, *ddir = nullptr, *dP = nullptr, *dp = nullptr;
  float *dX = nullptr, *dy = nullptr;
  int* dvalid = nullptr;
  const size_t nn = (size_t)n;
  m2cg_status st = M2CG_OK;
  if (cudaMalloc((void**)&deos, heos.size() * sizeof(Eos<double>)) != cudaSuccess ||
      cudaMalloc((void**)&dVL, nn * 40) != cudaSuccess || cudaMalloc((void**)&dVR, nn * 40) != cudaSuccess ||
      cudaMalloc((void**)&ddir, nn * 24) != cudaSuccess || cudaMalloc((void**)&dP, nn * 16) != cudaSuccess ||
      cudaMalloc((void**)&dp, nn * 8) != cudaSuccess || cudaMalloc((void**)&dX, nn * MLP_IN * 4) != cudaSuccess ||
      cudaMalloc((void**)&dy, nn * 4) != cudaSuccess || cudaMalloc((void**)&dvalid, nn * 4) != cudaSuccess)
    st = mfail(M2CG_ERR_NOMEM, "allocation failed");
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if (!st) {
    ck(cudaMemcpyAsync(deos, heos.data(), heos.size() * sizeof(Eos<double>), cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(dVL, VL, nn * 40, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(dVR, VR, nn * 40, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(ddir, dir, nn * 24, cudaMemcpyHostToDevice, s));
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    if (e == cudaSuccess) k_mlp_features_pairs<<<grid, 256, 0, s>>>(deos, n, dVL, dVR, ddir, dX, dP, dvalid);
    ck(cudaGetLastError());
    if (mode == 0) {
      if (X_out) ck(cudaMemcpyAsync(X_out, dX, nn * MLP_IN * 4, cudaMemcpyDeviceToHost, s));
      if (P_out) ck(cudaMemcpyAsync(P_out, dP, nn * 16, cudaMemcpyDeviceToHost, s));
      if (valid_out) ck(cudaMemcpyAsync(valid_out, dvalid, nn * 4, cudaMemcpyDeviceToHost, s));
    } else if (mode == 1) {
      if (e == cudaSuccess) ck(infer_rows(m, dX, dvalid, n, dy));
      if (e == cudaSuccess) k_mlp_to_pressure<<<grid, 256, 0, s>>>(dy, dP, dvalid, n, nullptr, dp);
      ck(cudaGetLastError());
      ck(cudaMemcpyAsync(p_out, dp, nn * 8, cudaMemcpyDeviceToHost, s));
    }
    ck(cudaStreamSynchronize(s));
    if (e != cudaSuccess) st = mfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaFree(deos); cudaFree(dVL); cudaFree(dVR); cudaFree(ddir); cudaFree(dP); cudaFree(dp);
  cudaFree(dX); cudaFree(dy); cudaFree(dvalid);
  if (own) cudaStreamDestroy(s);
  return st;
}

extern "C" m2cg_status m2cg_mlp_features_pairs(const m2cg_material* mats, int n, const double* VL, const double* VR,
                                               const double* dir, float* X, double* P, int* valid) {
  if (!mats || n < 1 || !VL || !VR || !dir || !X || !P || !valid) return mfail(M2CG_ERR_ARG, "null argument");
  return pairs_common(nullptr, mats, n, VL, VR, dir, X, P, valid, nullptr, 0);
}

extern "C" m2cg_status m2cg_mlp_predict_pairs(m2cg_mlp* m, const m2cg_material* mats, int n, const double* VL,
                                              const double* VR, const double* dir, double* p) {
  if (!m || !mats || n < 1 || !VL || !VR || !dir || !p) return mfail(M2CG_ERR_ARG, "null argument");
  return pairs_common(m, mats, n, VL, VR, dir, nullptr, nullptr, nullptr, p, 1);
}

extern "C" m2cg_status m2cg_mlp_infer(m2cg_mlp* m, const float* X, const int* valid, int n, float* y) {
  if (!m || !X || !valid || n < 1 || !y) return mfail(M2CG_ERR_ARG, "null argument");
  float *dX = nullptr, *dy = nullptr;
  int* dv = nullptr;
  m2cg_status st = M2CG_OK;
  if (cudaMalloc((void**)&dX, (size_t)n * MLP_IN * 4) != cudaSuccess || cudaMalloc((void**)&dy, (size_t)n * 4) != cudaSuccess ||
      cudaMalloc((void**)&dv, (size_t)n * 4) != cudaSuccess)
    st = mfail(M2CG_ERR_NOMEM, "allocation failed");
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if (!st) {
    ck(cudaMemcpyAsync(dX, X, (size_t)n * MLP_IN * 4, cudaMemcpyHostToDevice, m->stream));
    ck(cudaMemcpyAsync(dv, valid, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    if (e == cudaSuccess) ck(infer_rows(m, dX, dv, n, dy));
    ck(cudaMemcpyAsync(y, dy, (size_t)n * 4, cudaMemcpyDeviceToHost, m->stream));
    ck(cudaStreamSynchronize(m->stream));
    if (e != cudaSuccess) st = mfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaFree(dX); cudaFree(dy); cudaFree(dv);
  return st;
}
