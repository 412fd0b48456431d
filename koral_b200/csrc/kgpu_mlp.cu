// The warm-start network: a 16 -> 128 -> 128 -> 5 multilayer perceptron with
// SiLU activations, BF16 weights and activations and FP32 accumulation on
// the tensor cores (mma.sync m16n8k16), trained on the device by the
// kernels below (forward, backward, Adam) and evaluated on the device to
// give every cell of a batched implicit solve its initial iterate.
//
// Tile of work: a warp carries 16 samples (the M dimension of one mma);
// a training block of four warps 64; an inference block has sixteen warps.  Weights sit in shared memory as BF16, laid
// out [output][input] so that a B fragment is two 32-bit loads.  FP32
// master weights, their gradients and Adam moments stay in global memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/koral_b200.h"
#include "kgpu_mlp.cuh"

using namespace kgpu;

int kgpu_report_cuda(const char *what, cudaError_t e);

namespace {

#define MCK(call)                                              \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return kgpu_report_cuda(#call, e_); \
  } while (0)

typedef __nv_bfloat16 bf16;

// FP32 parameter blob: W1[16][128], b1[128], W2[128][128], b2[128],
// W3[128][8] (outputs 5..7 unused, kept zero), b3[8]; then the output
// standardisation mean[8], scale[8].
constexpr int OW1 = 0;
constexpr int OB1 = OW1 + MLP_IN * MLP_H;
constexpr int OW2 = OB1 + MLP_H;
constexpr int OB2 = OW2 + MLP_H * MLP_H;
constexpr int OW3 = OB2 + MLP_H;
constexpr int OB3 = OW3 + MLP_H * MLP_OUTP;
constexpr int NPARAM = OB3 + MLP_OUTP;
constexpr int OMEAN = NPARAM, OSCALE = NPARAM + MLP_OUTP;
constexpr int NBLOB = NPARAM + 2 * MLP_OUTP;

// padded leading dimensions of the shared-memory tiles (bf16 elements)
constexpr int LDX = MLP_IN + 8;    // 24
constexpr int LDH = MLP_H + 8;     // 136

// BF16 weights in the [output][input] layout the fragments want
struct Bf16Weights {
  bf16 *w1t;   // [128][16]
  bf16 *w2t;   // [128][128]
  bf16 *w3t;   // [8][128]
};

__device__ inline int lane_id() { return threadIdx.x & 31; }

__device__ inline void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment of the 16x16 tile at column k0 of a row-major [16][lda] matrix
__device__ inline void load_a(uint32_t a[4], const bf16 *A, int lda, int k0) {
  const int g = lane_id() >> 2, t = lane_id() & 3;
  a[0] = *(const uint32_t *)(A + g * lda + k0 + 2 * t);
  a[1] = *(const uint32_t *)(A + (g + 8) * lda + k0 + 2 * t);
  a[2] = *(const uint32_t *)(A + g * lda + k0 + 2 * t + 8);
  a[3] = *(const uint32_t *)(A + (g + 8) * lda + k0 + 2 * t + 8);
}
// B fragment (k16 x n8 at n0, k0) of a matrix stored [n][ldb] (n-major)
__device__ inline void load_b_nk(uint32_t b[2], const bf16 *Bt, int ldb, int n0, int k0) {
  const int g = lane_id() >> 2, t = lane_id() & 3;
  b[0] = *(const uint32_t *)(Bt + (n0 + g) * ldb + k0 + 2 * t);
  b[1] = *(const uint32_t *)(Bt + (n0 + g) * ldb + k0 + 2 * t + 8);
}
__device__ inline uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
// B fragment of a matrix stored [k][ldb] (k-major): element pairs along k
// are a row apart, so they are packed from two 16-bit loads
__device__ inline void load_b_kn(uint32_t b[2], const bf16 *B, int ldb, int n0, int k0) {
  const int g = lane_id() >> 2, t = lane_id() & 3;
  b[0] = pack2(B[(k0 + 2 * t) * ldb + n0 + g], B[(k0 + 2 * t + 1) * ldb + n0 + g]);
  b[1] = pack2(B[(k0 + 2 * t + 8) * ldb + n0 + g], B[(k0 + 2 * t + 9) * ldb + n0 + g]);
}

__device__ inline float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ inline float dsilu(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

// shared-memory image of the weights of one block
struct SmemW {
  bf16 w1t[MLP_H * LDX];
  bf16 w2t[MLP_H * LDH];
  bf16 w3t[MLP_OUTP * LDH];
  float b1[MLP_H], b2[MLP_H], b3[MLP_OUTP];
};
// per warp: the sample tile and the activations
struct SmemWarp {
  bf16 x[16 * LDX];
  bf16 a1[16 * LDH];
  bf16 a2[16 * LDH];
  float z1[16 * MLP_H];   // pre-activations (then the layer-1 error)
  float z2[16 * MLP_H];
  float y[16 * MLP_OUTP];
  bf16 dz2[16 * LDH];
};
// per block (training): transposed activations and errors for the weight
// gradients, whose reduction dimension is the sample
struct SmemBlock {
  bf16 a1t[MLP_H * (64 + 8)];
  bf16 dz2t[MLP_H * (64 + 8)];
};

__device__ void load_weights(SmemW &w, const Bf16Weights W, const float *blob) {
  for (int i = threadIdx.x; i < MLP_H * MLP_IN; i += blockDim.x) {
    const int n = i / MLP_IN, k = i % MLP_IN;
    w.w1t[n * LDX + k] = W.w1t[i];
  }
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) {
    const int n = i / MLP_H, k = i % MLP_H;
    w.w2t[n * LDH + k] = W.w2t[i];
  }
  for (int i = threadIdx.x; i < MLP_OUTP * MLP_H; i += blockDim.x) {
    const int n = i / MLP_H, k = i % MLP_H;
    w.w3t[n * LDH + k] = W.w3t[i];
  }
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    w.b1[i] = blob[OB1 + i];
    w.b2[i] = blob[OB2 + i];
  }
  for (int i = threadIdx.x; i < MLP_OUTP; i += blockDim.x) w.b3[i] = blob[OB3 + i];
}

// forward pass of one warp's 16 samples (x already in x); leaves a1, a2,
// the standardised outputs y and, for training, the pre-activations z1, z2.
// Layer 2 keeps all 16 output tiles in flight (16 independent accumulator
// chains), so the tensor-core latency of one chain is hidden by the others.
template <bool TRAIN>
__device__ void warp_forward_t(const SmemW &w, const bf16 *x, bf16 *a1s, bf16 *a2s, float *z1s, float *z2s,
                               float *ys) {
  const int g = lane_id() >> 2, t = lane_id() & 3;
  uint32_t a[4], b[2];
  // layer 1: 16 x 16 . 16 x 128
  load_a(a, x, LDX, 0);
  for (int nt = 0; nt < MLP_H / 8; nt++) {
    const int c0 = nt * 8 + 2 * t;
    float c[4] = {w.b1[c0], w.b1[c0 + 1], w.b1[c0], w.b1[c0 + 1]};
    load_b_nk(b, w.w1t, LDX, nt * 8, 0);
    mma16816(c, a, b);
    if (TRAIN) {
      z1s[g * MLP_H + c0] = c[0];
      z1s[g * MLP_H + c0 + 1] = c[1];
      z1s[(g + 8) * MLP_H + c0] = c[2];
      z1s[(g + 8) * MLP_H + c0 + 1] = c[3];
    }
    a1s[g * LDH + c0] = __float2bfloat16(silu(c[0]));
    a1s[g * LDH + c0 + 1] = __float2bfloat16(silu(c[1]));
    a1s[(g + 8) * LDH + c0] = __float2bfloat16(silu(c[2]));
    a1s[(g + 8) * LDH + c0 + 1] = __float2bfloat16(silu(c[3]));
  }
  __syncwarp();
  // layer 2: 16 x 128 . 128 x 128
  {
    float c[MLP_H / 8][4];
#pragma unroll
    for (int nt = 0; nt < MLP_H / 8; nt++) {
      const int c0 = nt * 8 + 2 * t;
      c[nt][0] = w.b2[c0];
      c[nt][1] = w.b2[c0 + 1];
      c[nt][2] = w.b2[c0];
      c[nt][3] = w.b2[c0 + 1];
    }
#pragma unroll
    for (int ks = 0; ks < MLP_H / 16; ks++) {
      load_a(a, a1s, LDH, ks * 16);
#pragma unroll
      for (int nt = 0; nt < MLP_H / 8; nt++) {
        load_b_nk(b, w.w2t, LDH, nt * 8, ks * 16);
        mma16816(c[nt], a, b);
      }
    }
    // every lane has read its a1 fragments: a2 may overwrite a1
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < MLP_H / 8; nt++) {
      const int c0 = nt * 8 + 2 * t;
      if (TRAIN) {
        z2s[g * MLP_H + c0] = c[nt][0];
        z2s[g * MLP_H + c0 + 1] = c[nt][1];
        z2s[(g + 8) * MLP_H + c0] = c[nt][2];
        z2s[(g + 8) * MLP_H + c0 + 1] = c[nt][3];
      }
      a2s[g * LDH + c0] = __float2bfloat16(silu(c[nt][0]));
      a2s[g * LDH + c0 + 1] = __float2bfloat16(silu(c[nt][1]));
      a2s[(g + 8) * LDH + c0] = __float2bfloat16(silu(c[nt][2]));
      a2s[(g + 8) * LDH + c0 + 1] = __float2bfloat16(silu(c[nt][3]));
    }
  }
  __syncwarp();
  // layer 3: 16 x 128 . 128 x 8
  {
    const int c0 = 2 * t;
    float c[4] = {w.b3[c0], w.b3[c0 + 1], w.b3[c0], w.b3[c0 + 1]};
    for (int ks = 0; ks < MLP_H / 16; ks++) {
      load_a(a, a2s, LDH, ks * 16);
      load_b_nk(b, w.w3t, LDH, 0, ks * 16);
      mma16816(c, a, b);
    }
    ys[g * MLP_OUTP + c0] = c[0];
    ys[g * MLP_OUTP + c0 + 1] = c[1];
    ys[(g + 8) * MLP_OUTP + c0] = c[2];
    ys[(g + 8) * MLP_OUTP + c0 + 1] = c[3];
  }
  __syncwarp();
}

__device__ inline void warp_forward(const SmemW &w, SmemWarp &sw) {
  warp_forward_t<true>(w, sw.x, sw.a1, sw.a2, sw.z1, sw.z2, sw.y);
}

// per warp, inference only: no pre-activations are kept and the second
// layer's activations overwrite the first's
struct SmemWarpInfer {
  bf16 x[16 * LDX];
  bf16 a[16 * LDH];
  float y[16 * MLP_OUTP];
};
// 16 warps of 124 registers fill the register file of an SM
constexpr int kInferWarps = 16;

__device__ void load_x_tile(bf16 *x, const float *X, int n, int s0) {
  for (int i = lane_id(); i < 16 * MLP_IN; i += 32) {
    const int r = i / MLP_IN, f = i % MLP_IN;
    const int sidx = s0 + r;
    x[r * LDX + f] = __float2bfloat16(sidx < n ? X[(long)sidx * MLP_IN + f] : 0.f);
  }
  __syncwarp();
}

// inference: Y[n][8] = unstandardised outputs; the block's warps share the
// weights
__global__ void __launch_bounds__(32 * kInferWarps) k_mlp_forward(const float *blob, Bf16Weights W, const float *X,
                                                                  int n, float *Y) {
  extern __shared__ __align__(16) unsigned char smem[];
  SmemW &w = *reinterpret_cast<SmemW *>(smem);
  SmemWarpInfer &sw = reinterpret_cast<SmemWarpInfer *>(smem + sizeof(SmemW))[threadIdx.x >> 5];
  load_weights(w, W, blob);
  __syncthreads();
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int s0 = warp * 16; s0 < n; s0 += nwarps * 16) {
    load_x_tile(sw.x, X, n, s0);
    warp_forward_t<false>(w, sw.x, sw.a, sw.a, nullptr, nullptr, sw.y);
    for (int i = lane_id(); i < 16 * MLP_OUTP; i += 32) {
      const int r = i / MLP_OUTP, o = i % MLP_OUTP;
      if (s0 + r < n) Y[(long)(s0 + r) * MLP_OUTP + o] = sw.y[i] * blob[OSCALE + o] + blob[OMEAN + o];
    }
    __syncwarp();
  }
}

// One training batch: forward and backward of 64 samples per block; the
// loss is the mean over the batch of the squared error of the standardised
// outputs; gradients are added to grad (FP32, zeroed by the caller).
__global__ void __launch_bounds__(128) k_mlp_train(const float *blob, Bf16Weights W, const float *X, const float *T,
                                                   const int *order, int n, int nbatch, float *grad,
                                                   double *loss) {
  extern __shared__ __align__(16) unsigned char smem[];
  SmemW &w = *reinterpret_cast<SmemW *>(smem);
  SmemWarp *warps = reinterpret_cast<SmemWarp *>(smem + sizeof(SmemW));
  SmemBlock &sb = *reinterpret_cast<SmemBlock *>(smem + sizeof(SmemW) + 4 * sizeof(SmemWarp));
  const int wi = threadIdx.x >> 5;
  SmemWarp &sw = warps[wi];
  load_weights(w, W, blob);
  __syncthreads();
  const int g = lane_id() >> 2, t = lane_id() & 3;
  const float inv = 1.f / (float)nbatch;
  for (int b0 = blockIdx.x * 64; b0 < nbatch; b0 += gridDim.x * 64) {
    const int s0 = b0 + wi * 16;
    // gather the samples of this tile
    for (int i = lane_id(); i < 16 * MLP_IN; i += 32) {
      const int r = i / MLP_IN, f = i % MLP_IN;
      const int q = s0 + r;
      const float v = q < nbatch ? X[(long)order[q] * MLP_IN + f] : 0.f;
      sw.x[r * LDX + f] = __float2bfloat16(v);
    }
    __syncwarp();
    warp_forward(w, sw);
    // output error (standardised targets), layer-3 gradients
    float lsum = 0.f;
    for (int i = lane_id(); i < 16 * MLP_OUTP; i += 32) {
      const int r = i / MLP_OUTP, o = i % MLP_OUTP;
      const int q = s0 + r;
      float d = 0.f;
      if (q < nbatch && o < MLP_OUT) {
        const float tt = (T[(long)order[q] * MLP_OUT + o] - blob[OMEAN + o]) / blob[OSCALE + o];
        const float e = sw.y[i] - tt;
        lsum += e * e;
        d = 2.f * e * inv;
      }
      sw.y[i] = d;   // now dL/dy
    }
    __syncwarp();
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane_id() == 0 && lsum != 0.f) atomicAdd(loss, (double)(lsum * inv));
    // b3, W3 gradients and dL/da2 = dy . W3^T (SIMT: K = 8)
    if (lane_id() < MLP_OUTP) {
      float s = 0.f;
      for (int r = 0; r < 16; r++) s += sw.y[r * MLP_OUTP + lane_id()];
      atomicAdd(&grad[OB3 + lane_id()], s);
    }
    for (int i = lane_id(); i < MLP_H; i += 32) {
      float gw[MLP_OUTP];
      for (int o = 0; o < MLP_OUTP; o++) gw[o] = 0.f;
      for (int r = 0; r < 16; r++) {
        const float a2 = __bfloat162float(sw.a2[r * LDH + i]);
        float da = 0.f;
        for (int o = 0; o < MLP_OUTP; o++) {
          gw[o] += a2 * sw.y[r * MLP_OUTP + o];
          da += sw.y[r * MLP_OUTP + o] * __bfloat162float(w.w3t[o * LDH + i]);
        }
        const float dz = da * dsilu(sw.z2[r * MLP_H + i]);
        sw.dz2[r * LDH + i] = __float2bfloat16(dz);
        sb.dz2t[i * (64 + 8) + wi * 16 + r] = __float2bfloat16(dz);
        sb.a1t[i * (64 + 8) + wi * 16 + r] = sw.a1[r * LDH + i];
      }
      for (int o = 0; o < MLP_OUT; o++) atomicAdd(&grad[OW3 + i * MLP_OUTP + o], gw[o]);
    }
    __syncwarp();
    // dL/da1 = dz2 . W2 (tensor cores: B[k = out j][n = in i] = W2[i][j] =
    // w2t[j][i], k-major), then dz1 = da1 * silu'(z1) into z1
    for (int nt = 0; nt < MLP_H / 8; nt++) {
      const int c0 = nt * 8 + 2 * t;
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t a[4], bb[2];
      for (int ks = 0; ks < MLP_H / 16; ks++) {
        load_a(a, sw.dz2, LDH, ks * 16);
        load_b_kn(bb, w.w2t, LDH, nt * 8, ks * 16);
        mma16816(c, a, bb);
      }
      sw.z1[g * MLP_H + c0] = c[0] * dsilu(sw.z1[g * MLP_H + c0]);
      sw.z1[g * MLP_H + c0 + 1] = c[1] * dsilu(sw.z1[g * MLP_H + c0 + 1]);
      sw.z1[(g + 8) * MLP_H + c0] = c[2] * dsilu(sw.z1[(g + 8) * MLP_H + c0]);
      sw.z1[(g + 8) * MLP_H + c0 + 1] = c[3] * dsilu(sw.z1[(g + 8) * MLP_H + c0 + 1]);
    }
    __syncwarp();
    // b1, b2, W1 gradients (SIMT: K = 16 samples)
    for (int i = lane_id(); i < MLP_H; i += 32) {
      float s1 = 0.f, s2 = 0.f, gw[MLP_IN];
      for (int f = 0; f < MLP_IN; f++) gw[f] = 0.f;
      for (int r = 0; r < 16; r++) {
        const float dz1 = sw.z1[r * MLP_H + i];
        s1 += dz1;
        s2 += __bfloat162float(sw.dz2[r * LDH + i]);
        for (int f = 0; f < MLP_IN; f++) gw[f] += __bfloat162float(sw.x[r * LDX + f]) * dz1;
      }
      atomicAdd(&grad[OB1 + i], s1);
      atomicAdd(&grad[OB2 + i], s2);
      for (int f = 0; f < MLP_IN; f++) atomicAdd(&grad[OW1 + f * MLP_H + i], gw[f]);
    }
    __syncthreads();
    // W2 gradient = a1^T . dz2 over the block's 64 samples (tensor cores:
    // M = in i, N = out j, K = samples); each warp takes 32 of the 128 tiles
    for (int tile = wi; tile < (MLP_H / 16) * (MLP_H / 8); tile += 4) {
      const int mt = tile / (MLP_H / 8), nt = tile % (MLP_H / 8);
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t a[4], bb[2];
      for (int ks = 0; ks < 4; ks++) {
        load_a(a, sb.a1t + mt * 16 * (64 + 8), 64 + 8, ks * 16);
        load_b_nk(bb, sb.dz2t, 64 + 8, nt * 8, ks * 16);
        mma16816(c, a, bb);
      }
      const int r0 = mt * 16 + g, c0 = nt * 8 + 2 * t;
      atomicAdd(&grad[OW2 + r0 * MLP_H + c0], c[0]);
      atomicAdd(&grad[OW2 + r0 * MLP_H + c0 + 1], c[1]);
      atomicAdd(&grad[OW2 + (r0 + 8) * MLP_H + c0], c[2]);
      atomicAdd(&grad[OW2 + (r0 + 8) * MLP_H + c0 + 1], c[3]);
    }
    __syncthreads();
  }
}

// Adam on the FP32 master weights, then the BF16 copies
__global__ void k_mlp_adam(float *blob, float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const bool pad = (i >= OW3 && i < OB3 && (i - OW3) % MLP_OUTP >= MLP_OUT) || (i >= OB3 && i - OB3 >= MLP_OUT);
  const float gr = pad ? 0.f : grad[i];
  m[i] = b1 * m[i] + (1.f - b1) * gr;
  v[i] = b2 * v[i] + (1.f - b2) * gr * gr;
  if (!pad) blob[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
  grad[i] = 0.f;
}

__global__ void k_mlp_to_bf16(const float *blob, Bf16Weights W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < MLP_IN * MLP_H) {   // w1t[n][k] = W1[k][n]
    const int n = i / MLP_IN, k = i % MLP_IN;
    W.w1t[i] = __float2bfloat16(blob[OW1 + k * MLP_H + n]);
  }
  if (i < MLP_H * MLP_H) {
    const int n = i / MLP_H, k = i % MLP_H;
    W.w2t[i] = __float2bfloat16(blob[OW2 + k * MLP_H + n]);
  }
  if (i < MLP_OUTP * MLP_H) {
    const int n = i / MLP_H, k = i % MLP_H;
    W.w3t[i] = __float2bfloat16(blob[OW3 + k * MLP_OUTP + n]);
  }
}

size_t smem_forward() { return sizeof(SmemW) + kInferWarps * sizeof(SmemWarpInfer); }
size_t smem_train() { return sizeof(SmemW) + 4 * sizeof(SmemWarp) + sizeof(SmemBlock); }

int sm_count_mlp() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

}  // namespace

struct kgpu_mlp {
  float *blob = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  Bf16Weights W{};
  double *dloss = nullptr;
  int *order = nullptr;
  int order_n = 0;
  long long step = 0;
};

extern "C" int kgpu_mlp_blob_size(void) { return NBLOB; }

extern "C" int kgpu_mlp_create(kgpu_mlp **out, unsigned long long seed) {
  if (!out) return KGPU_EINVAL;
  kgpu_mlp *M = new kgpu_mlp();
  std::vector<float> h(NBLOB, 0.f);
  // He-style initialisation from a 64-bit linear congruential stream
  unsigned long long s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto unif = [&]() {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(s >> 11) / 9007199254740992.0;
  };
  auto fill = [&](int off, int fan_in, int rows, int cols, int used_cols) {
    const double a = sqrt(6.0 / fan_in);
    for (int r = 0; r < rows; r++)
      for (int c = 0; c < cols; c++) h[off + r * cols + c] = c < used_cols ? (float)((2. * unif() - 1.) * a) : 0.f;
  };
  fill(OW1, MLP_IN, MLP_IN, MLP_H, MLP_H);
  fill(OW2, MLP_H, MLP_H, MLP_H, MLP_H);
  fill(OW3, MLP_H, MLP_H, MLP_OUTP, MLP_OUT);
  for (int o = 0; o < MLP_OUTP; o++) h[OSCALE + o] = 1.f;
  cudaError_t e = cudaSuccess;
  auto al = [&](void **p, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(p, b);
  };
  al((void **)&M->blob, NBLOB * 4);
  al((void **)&M->grad, NPARAM * 4);
  al((void **)&M->m, NPARAM * 4);
  al((void **)&M->v, NPARAM * 4);
  al((void **)&M->W.w1t, MLP_IN * MLP_H * 2);
  al((void **)&M->W.w2t, MLP_H * MLP_H * 2);
  al((void **)&M->W.w3t, MLP_OUTP * MLP_H * 2);
  al((void **)&M->dloss, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(M->blob, h.data(), NBLOB * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(M->grad, 0, NPARAM * 4);
  if (e == cudaSuccess) e = cudaMemset(M->m, 0, NPARAM * 4);
  if (e == cudaSuccess) e = cudaMemset(M->v, 0, NPARAM * 4);
  if (e == cudaSuccess) {
    k_mlp_to_bf16<<<(MLP_H * MLP_H + 255) / 256, 256>>>(M->blob, M->W);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem_forward());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem_train());
  if (e != cudaSuccess) {
    kgpu_report_cuda("kgpu_mlp_create", e);
    delete M;
    return KGPU_ECUDA;
  }
  *out = M;
  return 0;
}

extern "C" int kgpu_mlp_destroy(kgpu_mlp *M) {
  if (!M) return KGPU_EINVAL;
  cudaFree(M->blob);
  cudaFree(M->grad);
  cudaFree(M->m);
  cudaFree(M->v);
  cudaFree(M->W.w1t);
  cudaFree(M->W.w2t);
  cudaFree(M->W.w3t);
  cudaFree(M->dloss);
  cudaFree(M->order);
  delete M;
  return 0;
}

extern "C" int kgpu_mlp_get(kgpu_mlp *M, float *blob) {
  if (!M || !blob) return KGPU_EINVAL;
  MCK(cudaMemcpy(blob, M->blob, NBLOB * 4, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int kgpu_mlp_set(kgpu_mlp *M, const float *blob) {
  if (!M || !blob) return KGPU_EINVAL;
  MCK(cudaMemcpy(M->blob, blob, NBLOB * 4, cudaMemcpyHostToDevice));
  k_mlp_to_bf16<<<(MLP_H * MLP_H + 255) / 256, 256>>>(M->blob, M->W);
  MCK(cudaGetLastError());
  MCK(cudaDeviceSynchronize());
  return 0;
}

extern "C" int kgpu_mlp_forward(kgpu_mlp *M, const float *X, int n, float *Y, void *stream) {
  if (!M || n < 0 || (n > 0 && (!X || !Y))) return KGPU_EINVAL;
  if (n == 0) return 0;
  const int tiles = (n + 15) / 16;
  int blocks = (tiles + kInferWarps - 1) / kInferWarps;
  const int cap = sm_count_mlp();
  if (blocks > cap) blocks = cap;
  k_mlp_forward<<<blocks, 32 * kInferWarps, smem_forward(), (cudaStream_t)stream>>>(M->blob, M->W, X, n, Y);
  MCK(cudaGetLastError());
  return 0;
}

// Gradient of the batch loss (mean over the n samples, targets
// standardised with the blob's mean and scale) at the current weights,
// without an update: for checking the backward pass.
extern "C" int kgpu_mlp_gradient(kgpu_mlp *M, const float *X, const float *T, int n, float *grad_host,
                                 double *loss) {
  if (!M || n <= 0 || !X || !T || !grad_host || !loss) return KGPU_EINVAL;
  int *order = nullptr;
  MCK(cudaMalloc(&order, (size_t)n * 4));
  std::vector<int> h(n);
  for (int i = 0; i < n; i++) h[i] = i;
  cudaError_t e = cudaMemcpy(order, h.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(M->grad, 0, NPARAM * 4);
  if (e == cudaSuccess) e = cudaMemset(M->dloss, 0, sizeof(double));
  if (e == cudaSuccess) {
    k_mlp_train<<<(n + 63) / 64, 128, smem_train()>>>(M->blob, M->W, X, T, order, n, n, M->grad, M->dloss);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(grad_host, M->grad, NPARAM * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(loss, M->dloss, sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemset(M->grad, 0, NPARAM * 4);
  cudaFree(order);
  if (e != cudaSuccess) return kgpu_report_cuda("kgpu_mlp_gradient", e);
  return 0;
}

// One epoch of Adam over n samples (X [n][16], raw targets T [n][5], both
// device pointers), shuffled with `seed`, in batches of `batch`.  The mean
// batch loss goes to *mean_loss.
extern "C" int kgpu_mlp_train_epoch(kgpu_mlp *M, const float *X, const float *T, int n, int batch, float lr,
                                    unsigned long long seed, double *mean_loss) {
  if (!M || n <= 0 || batch <= 0 || !X || !T) return KGPU_EINVAL;
  if (M->order_n < n) {
    cudaFree(M->order);
    M->order = nullptr;
    MCK(cudaMalloc(&M->order, (size_t)n * 4));
    M->order_n = n;
  }
  std::vector<int> h(n);
  for (int i = 0; i < n; i++) h[i] = i;
  unsigned long long s = seed ^ 0x9e3779b97f4a7c15ULL;
  for (int i = n - 1; i > 0; i--) {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    const int j = (int)((s >> 33) % (unsigned long long)(i + 1));
    const int tmp = h[i];
    h[i] = h[j];
    h[j] = tmp;
  }
  MCK(cudaMemcpy(M->order, h.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemset(M->dloss, 0, sizeof(double)));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int nb = 0;
  for (int b0 = 0; b0 + batch <= n; b0 += batch, nb++) {
    const int blocks = (batch + 63) / 64;
    k_mlp_train<<<blocks, 128, smem_train()>>>(M->blob, M->W, X, T, M->order + b0, n, batch, M->grad, M->dloss);
    MCK(cudaGetLastError());
    M->step++;
    const float c1 = 1.f - powf(b1, (float)M->step), c2 = 1.f - powf(b2, (float)M->step);
    k_mlp_adam<<<(NPARAM + 255) / 256, 256>>>(M->blob, M->grad, M->m, M->v, lr, b1, b2, eps, c1, c2);
    MCK(cudaGetLastError());
    k_mlp_to_bf16<<<(MLP_H * MLP_H + 255) / 256, 256>>>(M->blob, M->W);
    MCK(cudaGetLastError());
  }
  double l = 0.;
  MCK(cudaMemcpy(&l, M->dloss, sizeof(double), cudaMemcpyDeviceToHost));
  if (mean_loss) *mean_loss = nb ? l / nb : 0.;
  return 0;
}
