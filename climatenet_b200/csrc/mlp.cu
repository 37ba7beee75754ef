// mlp.cu — learned warm start of the obstacle-contact forces (no counterpart
// in the reference): a per-contact MLP 10 -> 64 -> 64 -> 3 with ReLU, BF16
// weights and activations on the tensor cores (mma.sync m16n8k16, FP32
// accumulation), FP32 master weights, trained on the GPU with Adam on contact
// samples the solver itself logs.
//
// Parameter vector (FP32, kMlpParams values, row-major weights):
//   W1[64][10] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
// Features of obstacle contact k at vertex i (dimensionless; s_v = |g| dt,
// s_r = m_i |g| dt; B = contact basis with columns n, t, b):
//   x0..2 = B^T (t_n,i - w_k) / s_v   predictor velocity relative to the obstacle
//   x3    = gap_k / 1 cm              signed distance to the obstacle surface
//   x4..6 = B^T R_i / s_r             R_i = world-frame impulse of the contacts of
//                                     vertex i at the end of the previous step
//                                     (0 if it had none)
//   x7    = mu_k
//   x8    = n . g / |g|
//   x9    = 1
// Output y: predicted converged local force r_k / s_r.  The warm start uses
// r = cone(y s_r) instead of the projection in the first PD iteration of the
// step (the fixed point of the iteration is unchanged; only its starting
// force is).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "device.cuh"
#include "mlp.hpp"

namespace pdfb {

namespace {

constexpr int kIn = kMlpIn, kH = kMlpHidden, kOut = kMlpOut;
constexpr int OW1 = 0, OB1 = OW1 + kH * kIn, OW2 = OB1 + kH, OB2 = OW2 + kH * kH, OW3 = OB2 + kH, OB3 = OW3 + kOut * kH;
static_assert(OB3 + kOut == kMlpParams, "parameter layout");

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// D = A(16x16) B(16x8) + C, BF16 inputs, FP32 accumulate.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragment loaders from FP32 matrices in shared memory with arbitrary
// strides: element (r, c) of the logical matrix is at p[r * rs + c * cs].
// A fragment (16 x 16 at (r0, c0)):  a0 = (g, 2t..2t+1), a1 = (g+8, 2t..),
// a2 = (g, 2t+8..), a3 = (g+8, 2t+8..) with g = lane / 4, t = lane % 4.
__device__ __forceinline__ void load_a(uint32_t (&a)[4], const float* p, int rs, int cs, int r0, int c0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  auto e = [&](int r, int c) { return p[(r0 + r) * rs + (c0 + c) * cs]; };
  a[0] = pack_bf16(e(g, 2 * t), e(g, 2 * t + 1));
  a[1] = pack_bf16(e(g + 8, 2 * t), e(g + 8, 2 * t + 1));
  a[2] = pack_bf16(e(g, 2 * t + 8), e(g, 2 * t + 9));
  a[3] = pack_bf16(e(g + 8, 2 * t + 8), e(g + 8, 2 * t + 9));
}
// B fragment (16 x 8 at (k0, n0)): b0 = (k = 2t..2t+1, n = g), b1 = (k = 2t+8.., n = g).
__device__ __forceinline__ void load_b(uint32_t (&b)[2], const float* p, int ks, int ns, int k0, int n0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  auto e = [&](int k, int n) { return p[(k0 + k) * ks + (n0 + n) * ns]; };
  b[0] = pack_bf16(e(2 * t, g), e(2 * t + 1, g));
  b[1] = pack_bf16(e(2 * t + 8, g), e(2 * t + 9, g));
}
// C fragment (16 x 8 at (r0, n0)): c0 = (g, 2t), c1 = (g, 2t+1), c2 = (g+8, 2t), c3 = (g+8, 2t+1).
__device__ __forceinline__ void store_c(const float (&c)[4], float* p, int rs, int r0, int n0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  p[(r0 + g) * rs + n0 + 2 * t] = c[0];
  p[(r0 + g) * rs + n0 + 2 * t + 1] = c[1];
  p[(r0 + g + 8) * rs + n0 + 2 * t] = c[2];
  p[(r0 + g + 8) * rs + n0 + 2 * t + 1] = c[3];
}

// Shared-memory image of the parameters, zero padded for the tensor-core tiles:
//   w1[64][16] (k 10..15 zero), w2[64][64], w3[8][64] (rows 3..7 zero), b1, b2, b3[8].
struct SmemWeights {
  float w1[kH * 16];
  float w2[kH * kH];
  float w3[8 * kH];
  float b1[kH], b2[kH], b3[8];
};

__device__ void load_weights(SmemWeights& s, const float* __restrict__ prm) {
  for (int i = threadIdx.x; i < kH * 16; i += blockDim.x) {
    const int n = i / 16, k = i % 16;
    s.w1[i] = k < kIn ? prm[OW1 + n * kIn + k] : 0.f;
  }
  for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) s.w2[i] = prm[OW2 + i];
  for (int i = threadIdx.x; i < 8 * kH; i += blockDim.x) s.w3[i] = i < kOut * kH ? prm[OW3 + i] : 0.f;
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    s.b1[i] = prm[OB1 + i];
    s.b2[i] = prm[OB2 + i];
  }
  for (int i = threadIdx.x; i < 8; i += blockDim.x) s.b3[i] = i < kOut ? prm[OB3 + i] : 0.f;
}

// Per-warp activations of 16 samples.
struct WarpBuf {
  float x[16 * 16];   // inputs (cols 10..15 zero)
  float z1[16 * kH];  // pre-activations layer 1 (then gradients)
  float h1[16 * kH];  // relu(z1)
  float z2[16 * kH];
  float h2[16 * kH];
  float y[16 * 8];    // outputs (cols 3..7 zero), then output gradients
};

// Forward pass of 16 samples held by this warp.
__device__ void warp_forward(const SmemWeights& w, WarpBuf& b) {
  // layer 1: z1 = x w1^T + b1   (A = x [16 x 16], B(k, n) = w1[n][k])
  for (int nt = 0; nt < kH / 8; ++nt) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t a[4], bb[2];
    load_a(a, b.x, 16, 1, 0, 0);
    load_b(bb, w.w1, 1, 16, 0, nt * 8);
    mma16816(c, a, bb);
    store_c(c, b.z1, kH, 0, nt * 8);
  }
  __syncwarp();
  for (int i = threadIdx.x & 31; i < 16 * kH; i += 32) {
    const float z = b.z1[i] + w.b1[i % kH];
    b.z1[i] = z;
    b.h1[i] = fmaxf(z, 0.f);
  }
  __syncwarp();
  // layer 2: z2 = h1 w2^T + b2
  for (int nt = 0; nt < kH / 8; ++nt) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    for (int kt = 0; kt < kH / 16; ++kt) {
      uint32_t a[4], bb[2];
      load_a(a, b.h1, kH, 1, 0, kt * 16);
      load_b(bb, w.w2, 1, kH, kt * 16, nt * 8);
      mma16816(c, a, bb);
    }
    store_c(c, b.z2, kH, 0, nt * 8);
  }
  __syncwarp();
  for (int i = threadIdx.x & 31; i < 16 * kH; i += 32) {
    const float z = b.z2[i] + w.b2[i % kH];
    b.z2[i] = z;
    b.h2[i] = fmaxf(z, 0.f);
  }
  __syncwarp();
  // layer 3: y = h2 w3^T + b3   (N padded to 8)
  {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    for (int kt = 0; kt < kH / 16; ++kt) {
      uint32_t a[4], bb[2];
      load_a(a, b.h2, kH, 1, 0, kt * 16);
      load_b(bb, w.w3, 1, kH, kt * 16, 0);
      mma16816(c, a, bb);
    }
    store_c(c, b.y, 8, 0, 0);
  }
  __syncwarp();
  for (int i = threadIdx.x & 31; i < 16 * 8; i += 32) b.y[i] += w.b3[i % 8];
  __syncwarp();
}

// Loads up to 16 samples [s0, s0+16) of X (n x kIn) into the warp buffer.
__device__ void warp_load_x(WarpBuf& b, const float* __restrict__ X, int s0, int n) {
  for (int i = threadIdx.x & 31; i < 16 * 16; i += 32) {
    const int r = i / 16, c = i % 16;
    b.x[i] = (c < kIn && s0 + r < n) ? X[(int64_t)(s0 + r) * kIn + c] : 0.f;
  }
  __syncwarp();
}

// n samples, or min(*n_dev, n) when n_dev is given (count on the device).
__global__ void k_mlp_forward(const float* __restrict__ prm, const float* __restrict__ X, int n,
                              const int* __restrict__ n_dev, float* __restrict__ Y) {
  extern __shared__ unsigned char smem[];
  if (n_dev) n = min(n, *n_dev);
  SmemWeights& w = *reinterpret_cast<SmemWeights*>(smem);
  WarpBuf* bufs = reinterpret_cast<WarpBuf*>(smem + sizeof(SmemWeights));
  load_weights(w, prm);
  __syncthreads();
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  WarpBuf& b = bufs[warp];
  for (int s0 = (blockIdx.x * nw + warp) * 16; s0 < n; s0 += gridDim.x * nw * 16) {
    warp_load_x(b, X, s0, n);
    warp_forward(w, b);
    for (int i = threadIdx.x & 31; i < 16 * kOut; i += 32) {
      const int r = i / kOut, c = i % kOut;
      if (s0 + r < n) Y[(int64_t)(s0 + r) * kOut + c] = b.y[r * 8 + c];
    }
    __syncwarp();
  }
}

// Gradient of the mean squared error over the samples idx[0..n) (or 0..n
// when idx is null), accumulated into grad (kMlpParams) and loss.
__global__ void k_mlp_grad(const float* __restrict__ prm, const float* __restrict__ X, const float* __restrict__ T,
                           const int* __restrict__ idx, int n, float* __restrict__ grad, double* __restrict__ loss) {
  extern __shared__ unsigned char smem[];
  SmemWeights& w = *reinterpret_cast<SmemWeights*>(smem);
  float* g = reinterpret_cast<float*>(smem + sizeof(SmemWeights));  // kMlpParams gradients
  WarpBuf* bufs = reinterpret_cast<WarpBuf*>(smem + sizeof(SmemWeights) + sizeof(float) * ((kMlpParams + 63) / 64 * 64));
  load_weights(w, prm);
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) g[i] = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  WarpBuf& b = bufs[warp];
  const float inv_n = 1.f / (float)n;
  double lsum = 0.;
  for (int s0 = (blockIdx.x * nw + warp) * 16; s0 < n; s0 += gridDim.x * nw * 16) {
    for (int i = lane; i < 16 * 16; i += 32) {
      const int r = i / 16, c = i % 16;
      float v = 0.f;
      if (c < kIn && s0 + r < n) {
        const int64_t sidx = idx ? idx[s0 + r] : (s0 + r);
        v = X[sidx * kIn + c];
      }
      b.x[i] = v;
    }
    __syncwarp();
    warp_forward(w, b);
    // output gradient dL/dy = 2 (y - t) / n  (rows past n and cols >= 3 are zero)
    for (int i = lane; i < 16 * 8; i += 32) {
      const int r = i / 8, c = i % 8;
      float d = 0.f;
      if (c < kOut && s0 + r < n) {
        const int64_t sidx = idx ? idx[s0 + r] : (s0 + r);
        const float e = b.y[i] - T[sidx * kOut + c];
        lsum += (double)e * e;
        d = 2.f * e * inv_n;
      }
      b.y[i] = d;
    }
    __syncwarp();
    // dW3 += dY^T h2: A(r, k) = dY(k, r) (16 x 16, rows >= 8 read as zero via padding), B = h2 (k x n)
    for (int nt = 0; nt < kH / 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t a[4], bb[2];
      // rows 8..15 of dY^T do not exist: use a zero-padded view by reading
      // column r of dY only for r < 8
      {
        const int g2 = lane >> 2, t = lane & 3;
        auto e = [&](int r, int k) { return r < 8 ? b.y[k * 8 + r] : 0.f; };
        a[0] = pack_bf16(e(g2, 2 * t), e(g2, 2 * t + 1));
        a[1] = pack_bf16(e(g2 + 8, 2 * t), e(g2 + 8, 2 * t + 1));
        a[2] = pack_bf16(e(g2, 2 * t + 8), e(g2, 2 * t + 9));
        a[3] = pack_bf16(e(g2 + 8, 2 * t + 8), e(g2 + 8, 2 * t + 9));
      }
      load_b(bb, b.h2, kH, 1, 0, nt * 8);
      mma16816(c, a, bb);
      const int g2 = lane >> 2, t = lane & 3;
      // rows g2 (< 8) hold dW3[g2][n]; only rows < 3 are parameters
      if (g2 < kOut) {
        atomicAdd(&g[OW3 + g2 * kH + nt * 8 + 2 * t], c[0]);
        atomicAdd(&g[OW3 + g2 * kH + nt * 8 + 2 * t + 1], c[1]);
      }
    }
    for (int c = lane; c < kOut; c += 32) {
      float s = 0.f;
      for (int r = 0; r < 16; ++r) s += b.y[r * 8 + c];
      atomicAdd(&g[OB3 + c], s);
    }
    // dH2 = dY W3 (16 x 64): A = dY (16 x 16, cols >= 8 zero), B(k, n) = w3[k][n]
    for (int nt = 0; nt < kH / 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t a[4], bb[2];
      {
        const int g2 = lane >> 2, t = lane & 3;
        auto ea = [&](int r, int k) { return k < 8 ? b.y[r * 8 + k] : 0.f; };
        a[0] = pack_bf16(ea(g2, 2 * t), ea(g2, 2 * t + 1));
        a[1] = pack_bf16(ea(g2 + 8, 2 * t), ea(g2 + 8, 2 * t + 1));
        a[2] = pack_bf16(ea(g2, 2 * t + 8), ea(g2, 2 * t + 9));
        a[3] = pack_bf16(ea(g2 + 8, 2 * t + 8), ea(g2 + 8, 2 * t + 9));
        auto eb = [&](int k, int n2) { return k < 8 ? w.w3[k * kH + nt * 8 + n2] : 0.f; };
        bb[0] = pack_bf16(eb(2 * t, g2), eb(2 * t + 1, g2));
        bb[1] = pack_bf16(eb(2 * t + 8, g2), eb(2 * t + 9, g2));
      }
      mma16816(c, a, bb);
      store_c(c, b.h2, kH, 0, nt * 8);  // h2 now holds dH2
    }
    __syncwarp();
    // dZ2 = dH2 * (z2 > 0), stored in z2
    for (int i = lane; i < 16 * kH; i += 32) b.z2[i] = b.z2[i] > 0.f ? b.h2[i] : 0.f;
    __syncwarp();
    // dW2 += dZ2^T h1 (64 x 64): A(r, k) = dZ2(k, r), B(k, n) = h1(k, n)
    for (int mt = 0; mt < kH / 16; ++mt)
      for (int nt = 0; nt < kH / 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        uint32_t a[4], bb[2];
        load_a(a, b.z2, 1, kH, mt * 16, 0);
        load_b(bb, b.h1, kH, 1, 0, nt * 8);
        mma16816(c, a, bb);
        const int g2 = lane >> 2, t = lane & 3;
        atomicAdd(&g[OW2 + (mt * 16 + g2) * kH + nt * 8 + 2 * t], c[0]);
        atomicAdd(&g[OW2 + (mt * 16 + g2) * kH + nt * 8 + 2 * t + 1], c[1]);
        atomicAdd(&g[OW2 + (mt * 16 + g2 + 8) * kH + nt * 8 + 2 * t], c[2]);
        atomicAdd(&g[OW2 + (mt * 16 + g2 + 8) * kH + nt * 8 + 2 * t + 1], c[3]);
      }
    for (int c = lane; c < kH; c += 32) {
      float s = 0.f;
      for (int r = 0; r < 16; ++r) s += b.z2[r * kH + c];
      atomicAdd(&g[OB2 + c], s);
    }
    // dH1 = dZ2 W2 (16 x 64): A = dZ2 (16 x 64), B(k, n) = w2[k][n]
    for (int nt = 0; nt < kH / 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      for (int kt = 0; kt < kH / 16; ++kt) {
        uint32_t a[4], bb[2];
        load_a(a, b.z2, kH, 1, 0, kt * 16);
        load_b(bb, w.w2, kH, 1, kt * 16, nt * 8);
        mma16816(c, a, bb);
      }
      store_c(c, b.h1, kH, 0, nt * 8);  // h1 now holds dH1
    }
    __syncwarp();
    for (int i = lane; i < 16 * kH; i += 32) b.z1[i] = b.z1[i] > 0.f ? b.h1[i] : 0.f;  // dZ1
    __syncwarp();
    // dW1 += dZ1^T x (64 x 16): A(r, k) = dZ1(k, r), B(k, n) = x(k, n)
    for (int mt = 0; mt < kH / 16; ++mt)
      for (int nt = 0; nt < 2; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        uint32_t a[4], bb[2];
        load_a(a, b.z1, 1, kH, mt * 16, 0);
        load_b(bb, b.x, 16, 1, 0, nt * 8);
        mma16816(c, a, bb);
        const int g2 = lane >> 2, t = lane & 3;
        const int n0 = nt * 8 + 2 * t;
        if (n0 < kIn) {
          atomicAdd(&g[OW1 + (mt * 16 + g2) * kIn + n0], c[0]);
          atomicAdd(&g[OW1 + (mt * 16 + g2 + 8) * kIn + n0], c[2]);
        }
        if (n0 + 1 < kIn) {
          atomicAdd(&g[OW1 + (mt * 16 + g2) * kIn + n0 + 1], c[1]);
          atomicAdd(&g[OW1 + (mt * 16 + g2 + 8) * kIn + n0 + 1], c[3]);
        }
      }
    for (int c = lane; c < kH; c += 32) {
      float s = 0.f;
      for (int r = 0; r < 16; ++r) s += b.z1[r * kH + c];
      atomicAdd(&g[OB1 + c], s);
    }
    __syncwarp();
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) atomicAdd(loss, lsum * inv_n);
  __syncthreads();
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) atomicAdd(&grad[i], g[i]);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights.
__global__ void k_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float g = grad[i];
  const float a = b1 * m1[i] + (1.f - b1) * g;
  const float v = b2 * m2[i] + (1.f - b2) * g * g;
  m1[i] = a;
  m2[i] = v;
  prm[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

#define CKM(x)                                                                                      \
  do {                                                                                              \
    cudaError_t e_ = (x);                                                                           \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kMlpThreads = 128;  // 4 warps
size_t fwd_smem() { return sizeof(SmemWeights) + 4 * sizeof(WarpBuf); }
size_t grad_smem() {
  return sizeof(SmemWeights) + sizeof(float) * ((kMlpParams + 63) / 64 * 64) + 4 * sizeof(WarpBuf);
}

template <typename T>
struct DBuf {
  T* p = nullptr;
  explicit DBuf(size_t n) { CKM(cudaMalloc((void**)&p, std::max<size_t>(1, n) * sizeof(T))); }
  ~DBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

// cudaFuncSetAttribute is per device: done once per device ordinal.
static void ensure_smem_attrs() {
  static std::atomic<bool> done[64];
  int dev = 0;
  CKM(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || done[dev].load()) return;
  CKM(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem()));
  CKM(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem()));
  done[dev].store(true);
}

void mlp_forward_device(const float* prm, const float* X, int n, float* Y, cudaStream_t st) {
  if (n <= 0) return;
  ensure_smem_attrs();
  const int grid = std::min(148 * 4, (n + 63) / 64);
  k_mlp_forward<<<grid, kMlpThreads, fwd_smem(), st>>>(prm, X, n, nullptr, Y);
}

void mlp_forward_counted(const float* prm, const float* X, const int* n_dev, int cap, float* Y, cudaStream_t st) {
  if (cap <= 0) return;
  ensure_smem_attrs();
  const int grid = std::min(148 * 4, (cap + 63) / 64);
  k_mlp_forward<<<grid, kMlpThreads, fwd_smem(), st>>>(prm, X, cap, n_dev, Y);
}

void mlp_grad_device(const float* prm, const float* X, const float* T, const int* idx, int n, float* grad,
                     double* loss, cudaStream_t st) {
  if (n <= 0) return;
  ensure_smem_attrs();
  const int grid = std::min(148 * 2, (n + 63) / 64);
  k_mlp_grad<<<grid, kMlpThreads, grad_smem(), st>>>(prm, X, T, idx, n, grad, loss);
}


void mlp_adam_device(float* prm, const float* grad, float* m1, float* m2, double lr, int64_t step, cudaStream_t st) {
  const double b1 = 0.9, b2 = 0.999;
  const float c1 = (float)(1. - std::pow(b1, (double)step)), c2 = (float)(1. - std::pow(b2, (double)step));
  k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(prm, grad, m1, m2, (float)lr, (float)b1, (float)b2, 1e-8f, c1, c2);
}

double mlp_train_device(float* prm, const float* X, const float* T, int n, int epochs, int batch, double lr,
                        uint64_t seed, double* val_loss, cudaStream_t st) {
  if (n < 2 || batch <= 0 || epochs <= 0 || !(lr > 0.)) throw std::invalid_argument("invalid training arguments");
  // seeded shuffle, 90 / 10 split
  std::mt19937_64 rng(seed);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::shuffle(order.begin(), order.end(), rng);
  const int nval = std::max(1, n / 10), ntr = n - nval;
  DBuf<float> dg(kMlpParams), m1(kMlpParams), m2(kMlpParams);
  DBuf<double> dl(1);
  DBuf<int> didx(n);
  CKM(cudaMemsetAsync(m1.p, 0, kMlpParams * sizeof(float), st));
  CKM(cudaMemsetAsync(m2.p, 0, kMlpParams * sizeof(float), st));
  int64_t step = 0;
  double last = 0.;
  std::vector<int> tr(order.begin(), order.begin() + ntr);
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(tr.begin(), tr.end(), rng);
    CKM(cudaMemcpyAsync(didx.p, tr.data(), ntr * sizeof(int), cudaMemcpyHostToDevice, st));
    CKM(cudaMemsetAsync(dl.p, 0, sizeof(double), st));
    int nbatches = 0;
    for (int s0 = 0; s0 < ntr; s0 += batch) {
      const int nb = std::min(batch, ntr - s0);
      CKM(cudaMemsetAsync(dg.p, 0, kMlpParams * sizeof(float), st));
      mlp_grad_device(prm, X, T, didx.p + s0, nb, dg.p, dl.p, st);
      mlp_adam_device(prm, dg.p, m1.p, m2.p, lr, ++step, st);
      ++nbatches;
    }
    double sum = 0.;
    CKM(cudaMemcpyAsync(&sum, dl.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    CKM(cudaStreamSynchronize(st));  // also keeps `tr` alive until its copy is done
    last = sum / std::max(nbatches, 1);
  }
  // loss on the held-out part
  std::vector<int> va(order.begin() + ntr, order.end());
  CKM(cudaMemcpyAsync(didx.p, va.data(), nval * sizeof(int), cudaMemcpyHostToDevice, st));
  CKM(cudaMemsetAsync(dg.p, 0, kMlpParams * sizeof(float), st));
  CKM(cudaMemsetAsync(dl.p, 0, sizeof(double), st));
  mlp_grad_device(prm, X, T, didx.p, nval, dg.p, dl.p, st);
  double vl = 0.;
  CKM(cudaMemcpyAsync(&vl, dl.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  CKM(cudaStreamSynchronize(st));
  CKM(cudaGetLastError());
  if (val_loss) *val_loss = vl;
  return last;
}

// ---------------------------------------------------------------------------
// Standardised training: per-column mean / standard deviation of the samples
// (double accumulation), standardised copies, training, and the
// standardisation folded back into the first and last layers so that the
// network takes the raw features and returns raw forces.

__global__ void k_col_stats(const float* __restrict__ A, int64_t n, int ncol, double* __restrict__ acc) {
  // acc[2c] += sum of column c, acc[2c+1] += sum of squares (ncol <= 16)
  __shared__ double red[2 * 16];
  for (int i = threadIdx.x; i < 2 * 16; i += blockDim.x) red[i] = 0.;
  __syncthreads();
  double loc[2 * 16];
  for (int c = 0; c < 2 * ncol; ++c) loc[c] = 0.;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < ncol; ++c) {
      const double v = A[r * ncol + c];
      loc[2 * c] += v;
      loc[2 * c + 1] += v * v;
    }
  for (int c = 0; c < 2 * ncol; ++c) atomicAdd(&red[c], loc[c]);
  __syncthreads();
  for (int c = threadIdx.x; c < 2 * ncol; c += blockDim.x) atomicAdd(&acc[c], red[c]);
}

__global__ void k_standardize(const float* __restrict__ A, int64_t n, int ncol, const float* __restrict__ shift,
                              const float* __restrict__ scale, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * ncol;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % ncol);
    out[i] = (A[i] - shift[c]) / scale[c];
  }
}

double mlp_train_standardized(float* prm, const float* X, const float* T, int n, int epochs, int batch, double lr,
                              uint64_t seed, double* val_loss, cudaStream_t st) {
  if (n < 2) throw std::invalid_argument("fewer than 2 samples");
  DBuf<double> acc(2 * (kIn + kOut));
  CKM(cudaMemsetAsync(acc.p, 0, 2 * (kIn + kOut) * sizeof(double), st));
  k_col_stats<<<2 * 148, 256, 0, st>>>(X, n, kIn, acc.p);
  k_col_stats<<<2 * 148, 256, 0, st>>>(T, n, kOut, acc.p + 2 * kIn);
  std::vector<double> a(2 * (kIn + kOut));
  CKM(cudaMemcpyAsync(a.data(), acc.p, a.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CKM(cudaStreamSynchronize(st));
  std::vector<float> shift(kIn + kOut), scale(kIn + kOut);
  for (int c = 0; c < kIn + kOut; ++c) {
    const double mean = a[2 * c] / n, var = std::max(0., a[2 * c + 1] / n - mean * mean);
    double sd = std::sqrt(var), sh = mean;
    if (sd < 1e-12) {  // constant column (the bias feature): left alone
      sd = 1.;
      if (c < kIn) sh = 0.;
    }
    shift[c] = (float)sh;
    scale[c] = (float)sd;
  }
  DBuf<float> dshift(kIn + kOut), dscale(kIn + kOut), Xs((size_t)n * kIn), Ts((size_t)n * kOut);
  CKM(cudaMemcpyAsync(dshift.p, shift.data(), shift.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  CKM(cudaMemcpyAsync(dscale.p, scale.data(), scale.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  k_standardize<<<4 * 148, 256, 0, st>>>(X, n, kIn, dshift.p, dscale.p, Xs.p);
  k_standardize<<<4 * 148, 256, 0, st>>>(T, n, kOut, dshift.p + kIn, dscale.p + kIn, Ts.p);
  std::vector<float> w(kMlpParams);
  mlp_init_params(w.data(), seed);
  CKM(cudaMemcpyAsync(prm, w.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
  const double tl = mlp_train_device(prm, Xs.p, Ts.p, n, epochs, batch, lr, seed, val_loss, st);
  // fold: W1' = W1 / sigma, b1' = b1 - W1 (mu / sigma); W3' = tau W3, b3' = tau b3 + nu
  CKM(cudaMemcpyAsync(w.data(), prm, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, st));
  CKM(cudaStreamSynchronize(st));
  for (int h = 0; h < kH; ++h) {
    double b = w[OB1 + h];
    for (int i = 0; i < kIn; ++i) {
      const double wi = w[OW1 + h * kIn + i];
      b -= wi * (double)shift[i] / (double)scale[i];
      w[OW1 + h * kIn + i] = (float)(wi / (double)scale[i]);
    }
    w[OB1 + h] = (float)b;
  }
  for (int o = 0; o < kOut; ++o) {
    const double tau = scale[kIn + o], nu = shift[kIn + o];
    for (int h = 0; h < kH; ++h) w[OW3 + o * kH + h] = (float)(tau * w[OW3 + o * kH + h]);
    w[OB3 + o] = (float)(tau * w[OB3 + o] + nu);
  }
  CKM(cudaMemcpyAsync(prm, w.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
  CKM(cudaStreamSynchronize(st));
  return tl;
}

// ---------------------------------------------------------------------------
// In the step loop.  This file is compiled without FMA contraction, so the
// feature arithmetic below rounds every product and sum separately, in the
// order written (the CPU oracle evaluates the same expressions).

__device__ __forceinline__ double gnorm_of(double gx, double gy, double gz) {
  const double gn = sqrt((gx * gx + gy * gy) + gz * gz);
  return gn > 1e-12 ? gn : 1e-12;
}

// Features of every obstacle contact (definitions at the top of this file).
__global__ void k_mlp_features(DContacts c, const double* __restrict__ tn, const double* __restrict__ mass,
                               const double* __restrict__ rprev, const int* __restrict__ rprev_tag, int tag_prev,
                               double gx, double gy, double gz, double dt, float* __restrict__ X) {
  const int C = *c.n_contacts;
  const double g = gnorm_of(gx, gy, gz);
  const double sv = g * dt;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    const int v = c.c_vertex[k];
    const double* B = c.c_basis + 9 * (int64_t)k;
    const double3 w = ld3(c.c_speed, k);
    const double3 t = ld3(tn, v);
    const double dx = t.x - w.x, dy = t.y - w.y, dz = t.z - w.z;
    float* x = X + (int64_t)k * kIn;
    x[0] = (float)(((B[0] * dx + B[1] * dy) + B[2] * dz) / sv);
    x[1] = (float)(((B[3] * dx + B[4] * dy) + B[5] * dz) / sv);
    x[2] = (float)(((B[6] * dx + B[7] * dy) + B[8] * dz) / sv);
    x[3] = (float)(c.c_gap[k] / 1e-2);
    const double sr = mass[v] * sv;
    if (rprev_tag[v] == tag_prev) {
      const double3 R = ld3(rprev, v);
      x[4] = (float)(((B[0] * R.x + B[1] * R.y) + B[2] * R.z) / sr);
      x[5] = (float)(((B[3] * R.x + B[4] * R.y) + B[5] * R.z) / sr);
      x[6] = (float)(((B[6] * R.x + B[7] * R.y) + B[8] * R.z) / sr);
    } else {
      x[4] = x[5] = x[6] = 0.f;
    }
    x[7] = (float)c.c_mu[k];
    x[8] = (float)(((B[0] * gx + B[1] * gy) + B[2] * gz) / g);
    x[9] = 1.f;
  }
}

// End of step, pass 1: the r_prev memory of every contact vertex starts from zero.
__global__ void k_mlp_rprev_clear(DContacts c, double* __restrict__ rprev, int* __restrict__ rprev_tag, int tag) {
  const int C = *c.n_contacts;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    const int v = c.c_vertex[k];
    st3(rprev, v, make_double3(0., 0., 0.));
    rprev_tag[v] = tag;
  }
}

// Pass 2: world-frame impulse B r of every contact that was active in the last
// iteration, summed per vertex; with a log, (features, r / s_r) samples in
// contact order after the samples already logged (target 0 for a contact
// that took off).
__global__ void k_mlp_record(DContacts c, const double* __restrict__ mass, double* __restrict__ rprev, double gx,
                             double gy, double gz, double dt, const float* __restrict__ X, float* __restrict__ SX,
                             float* __restrict__ ST, const int* __restrict__ n_samples, int cap) {
  const int C = *c.n_contacts;
  const double sv = gnorm_of(gx, gy, gz) * dt;
  const int base = SX ? *n_samples : 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    const int v = c.c_vertex[k];
    const bool active = c.c_active[k] != 0;
    const double3 r = active ? ld3(c.c_force, k) : make_double3(0., 0., 0.);
    if (active) {
      const double* B = c.c_basis + 9 * (int64_t)k;
      atomicAdd(rprev + 3 * (int64_t)v, (B[0] * r.x + B[3] * r.y) + B[6] * r.z);
      atomicAdd(rprev + 3 * (int64_t)v + 1, (B[1] * r.x + B[4] * r.y) + B[7] * r.z);
      atomicAdd(rprev + 3 * (int64_t)v + 2, (B[2] * r.x + B[5] * r.y) + B[8] * r.z);
    }
    if (SX && (int64_t)base + k < cap) {
      const int64_t s = (int64_t)base + k;
      for (int d = 0; d < kIn; ++d) SX[s * kIn + d] = X[(int64_t)k * kIn + d];
      const double sr = mass[v] * sv;
      ST[s * kOut] = (float)(r.x / sr);
      ST[s * kOut + 1] = (float)(r.y / sr);
      ST[s * kOut + 2] = (float)(r.z / sr);
    }
  }
}

__global__ void k_mlp_count(DContacts c, int* n_samples, int cap) {
  const int64_t n = (int64_t)*n_samples + *c.n_contacts;
  *n_samples = (int)(n < cap ? n : cap);
}

void launch_mlp_features(cudaStream_t st, DContacts c, const double* tn, const double* mass, const double* rprev,
                         const int* rprev_tag, int tag_prev, const double g[3], double dt, float* X) {
  k_mlp_features<<<2 * 148, 256, 0, st>>>(c, tn, mass, rprev, rprev_tag, tag_prev, g[0], g[1], g[2], dt, X);
}

void launch_mlp_record(cudaStream_t st, DContacts c, const double* mass, double* rprev, int* rprev_tag, int tag,
                       const double g[3], double dt, const float* X, float* SX, float* ST, int* n_samples, int cap) {
  k_mlp_rprev_clear<<<2 * 148, 256, 0, st>>>(c, rprev, rprev_tag, tag);
  k_mlp_record<<<2 * 148, 256, 0, st>>>(c, mass, rprev, g[0], g[1], g[2], dt, X, SX, ST, n_samples, cap);
  if (SX) k_mlp_count<<<1, 1, 0, st>>>(c, n_samples, cap);
}

}  // namespace pdfb
