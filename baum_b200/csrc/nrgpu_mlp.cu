// nrgpu_mlp.cu -- the learned warm start of the puncture multigrid (sm_100a).
// No counterpart in the reference: a coordinate MLP conditioned on the
// puncture parameters predicts the conformal-factor correction u that
// PunctureData otherwise obtains from u = 0 by multigrid.
//
// Network: 32 input features -> 4 hidden layers of 128 (SiLU) -> 1 output.
// Every hidden-layer product runs on the tensor cores as BF16 x BF16 with
// FP32 accumulation (mma.sync m16n8k16); the master weights, the Adam state,
// biases, the output layer and the loss are FP32.  Training is the plain
// reverse-mode chain with the same BF16 operands as the forward pass.
//
// Kernels:
//   mlp_features_kernel   feature rows (double math, rounded to BF16)
//   gemm_bf16_kernel      C[MxN] (+)= A[MxK] B[KxN], A/B stored plain or
//                         transposed, split-K with FP32 atomics
//   bias_silu_kernel      Z += b, A = bf16(silu(Z))
//   out_layer_kernel      out = A4 w5 + b5; loss, dw5, db5, dZ4 (training)
//   silu_back_kernel      dZ = bf16(dA * silu'(Z))
//   colsum_kernel         db = sum over rows of dZ
//   adam_kernel           Adam step on the FP32 master copy + BF16 refresh
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>
#include "nrgpu_common.cuh"
#include "nrgpu_tma.cuh"

static constexpr int IN = NRGPU_MLP_IN;
static constexpr int HID = NRGPU_MLP_HIDDEN;

namespace {

// flat FP32 parameter layout: W1 [IN][HID], b1, W2 [HID][HID], b2, W3, b3,
// W4, b4, w5 [HID], b5
__host__ __device__ constexpr int off_w(int l) { return l == 0 ? 0 : IN * HID + HID + (l - 1) * (HID * HID + HID); }
constexpr int kOffW5 = IN * HID + HID + 3 * (HID * HID + HID);
constexpr int kNParams = kOffW5 + HID + 1;
__host__ __device__ constexpr int off_b(int l) { return off_w(l) + (l == 0 ? IN : HID) * HID; }
__host__ __device__ constexpr int fan_in(int l) { return l == 0 ? IN : HID; }

// ---- features ----------------------------------------------------------------
// conditioning vector of one binary: m1 m2 | pos 6 | mom 6 | spin 6
struct Feat {
  int m;
  double dx;
};

__device__ __forceinline__ __nv_bfloat16 to_bf16(double v) { return __float2bfloat16_rn((float)v); }

__global__ void mlp_features_kernel(const double *__restrict__ cond, const int *__restrict__ set,
                                    const int *__restrict__ pt, long first, int n, Feat F, __nv_bfloat16 *X) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const long p = pt ? (long)pt[r] : first + r;
  const double *c = cond + 20 * (set ? set[r] : 0);
  const int m = F.m;
  const double h0 = -0.5 * (m - 1) * F.dx;
  const int i = (int)(p % m), j = (int)((p / m) % m), k = (int)(p / ((long)m * m));
  const double x[3] = {h0 + i * F.dx, h0 + j * F.dx, h0 + k * F.dx};
  const double s = 1.0 / 8.0;
  __nv_bfloat16 *f = X + (long)r * IN;
  f[0] = to_bf16(x[0] * s);
  f[1] = to_bf16(x[1] * s);
  f[2] = to_bf16(x[2] * s);
  for (int q = 0; q < 2; ++q) {
    const double mq = c[q];
    const double d0 = x[0] - c[2 + 3 * q], d1 = x[1] - c[3 + 3 * q], d2 = x[2] - c[4 + 3 * q];
    const double rr = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    __nv_bfloat16 *g = f + 3 + 12 * q;
    g[0] = to_bf16(d0 * s);
    g[1] = to_bf16(d1 * s);
    g[2] = to_bf16(d2 * s);
    g[3] = to_bf16(rr * s);
    g[4] = to_bf16(mq / (rr + mq));
    g[5] = to_bf16(2.0 * mq);
    for (int a = 0; a < 3; ++a) {
      g[6 + a] = to_bf16(5.0 * c[8 + 3 * q + a]);
      g[9 + a] = to_bf16(5.0 * c[14 + 3 * q + a]);
    }
  }
  for (int q = 27; q < IN; ++q) f[q] = __float2bfloat16_rn(0.0f);
}

// ---- BF16 GEMM on the tensor cores --------------------------------------------
// C[M][N] (+)= A[M][K] B[K][N]; A stored [M][K] (AT = false) or [K][M] (AT =
// true), B stored [K][N] (BT = false) or [N][K] (BT = true), all row major.
// CTA tile 64 x 64, k step 32, 4 warps of 32 x 32.  M, N multiples of 16,
// K of 32 (checked by the host).  ATOMIC: split-K over gridDim.z, the
// caller zeroes C.
constexpr int TM = 64, TN = 64, TK = 32, PADK = 40;

__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// stage a 64 (outer) x 32 (k) tile into S[outer][k] from a row-major BF16
// matrix: KCONTIG = the source rows run along k (S[o][k] = G[outer0+o][k0+k]),
// otherwise along the outer index (S[o][k] = G[k0+k][outer0+o])
template <bool KCONTIG>
__device__ __forceinline__ void load_tile(__nv_bfloat16 (*S)[PADK], const __nv_bfloat16 *__restrict__ G, int ld,
                                          int outer0, int nouter, int k0) {
  const int t = threadIdx.x;
  if (KCONTIG) {
    const int o = t >> 1, kk = (t & 1) * 16;
    uint4 v0 = make_uint4(0, 0, 0, 0), v1 = v0;
    if (outer0 + o < nouter) {
      const uint4 *src = reinterpret_cast<const uint4 *>(G + (long)(outer0 + o) * ld + k0 + kk);
      v0 = __ldg(src);
      v1 = __ldg(src + 1);
    }
    // rows of S are 80 bytes: 16-byte aligned at kk = 0 and 16
    uint4 *dst = reinterpret_cast<uint4 *>(&S[o][kk]);
    dst[0] = v0;
    dst[1] = v1;
  } else {
    const int kk = t >> 2, o0 = (t & 3) * 16;
    alignas(16) __nv_bfloat16 v[16];
    if (outer0 + o0 < nouter) {
      const uint4 *src = reinterpret_cast<const uint4 *>(G + (long)(k0 + kk) * ld + outer0 + o0);
      *reinterpret_cast<uint4 *>(v) = __ldg(src);
      *reinterpret_cast<uint4 *>(v + 8) = __ldg(src + 1);
    } else {
      for (int q = 0; q < 16; ++q) v[q] = __float2bfloat16_rn(0.0f);
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) S[o0 + q][kk] = v[q];
  }
}

template <bool AT, bool BT, bool ATOMIC>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __nv_bfloat16 *__restrict__ A,
                                                        const __nv_bfloat16 *__restrict__ B, float *C, int M,
                                                        int N, int K, int kchunk) {
  __shared__ __align__(16) __nv_bfloat16 As[TM][PADK];
  __shared__ __align__(16) __nv_bfloat16 Bs[TN][PADK];
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, tg = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
  for (int k0 = kb; k0 < ke; k0 += TK) {
    load_tile<!AT>(As, A, AT ? M : K, m0, M, k0);
    load_tile<BT>(Bs, B, BT ? K : N, n0, N, k0);
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < TK; ks += 16) {
      uint32_t af[2][4], bf[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r = wm + mt * 16 + g, c = ks + tg * 2;
        af[mt][0] = *reinterpret_cast<const uint32_t *>(&As[r][c]);
        af[mt][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][c]);
        af[mt][2] = *reinterpret_cast<const uint32_t *>(&As[r][c + 8]);
        af[mt][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][c + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int n = wn + nt * 8 + g, c = ks + tg * 2;
        bf[nt][0] = *reinterpret_cast<const uint32_t *>(&Bs[n][c]);
        bf[nt][1] = *reinterpret_cast<const uint32_t *>(&Bs[n][c + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma16816(acc[mt][nt], af[mt], bf[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = m0 + wm + mt * 16 + g + 8 * h;
        const int c = n0 + wn + nt * 8 + tg * 2;
        if (r >= M) continue;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (c + e >= N) continue;
          float *dst = C + (long)r * N + c + e;
          if (ATOMIC) atomicAdd(dst, acc[mt][nt][2 * h + e]);
          else *dst = acc[mt][nt][2 * h + e];
        }
      }
}

// ---- elementwise pieces ---------------------------------------------------------
__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

__global__ void bias_silu_kernel(float *Z, const float *__restrict__ b, __nv_bfloat16 *Aout, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = Z[i] + b[i % HID];
  Z[i] = z;
  Aout[i] = __float2bfloat16_rn(z * sigm(z));
}

// one block of HID threads walks rows [r0, r1); thread k owns hidden unit k.
// Without targets (y == nullptr) only out is written.
__global__ void __launch_bounds__(HID) out_layer_kernel(const __nv_bfloat16 *__restrict__ A4,
                                                         const float *__restrict__ Z4,
                                                         const float *__restrict__ P, float *out,
                                                         const float *__restrict__ y, int n, int rows_per_block,
                                                         float *grad, __nv_bfloat16 *dZ4, float *loss) {
  __shared__ float red[HID / 32];
  __shared__ float rowsum;
  const int k = threadIdx.x;
  const float w5 = P[kOffW5 + k], b5 = P[kOffW5 + HID];
  float gw = 0.0f, gb = 0.0f, ls = 0.0f;
  const int r0 = blockIdx.x * rows_per_block, r1 = min(n, r0 + rows_per_block);
  for (int r = r0; r < r1; ++r) {
    const float a = __bfloat162float(A4[(long)r * HID + k]);
    float v = a * w5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((k & 31) == 0) red[k >> 5] = v;
    __syncthreads();
    if (k == 0) {
      float s = b5;
      for (int q = 0; q < HID / 32; ++q) s += red[q];
      rowsum = s;
      out[r] = s;
    }
    __syncthreads();
    if (y) {
      const float o = rowsum;
      const float d = 2.0f * (o - y[r]) / (float)n;
      if (k == 0) {
        ls += (o - y[r]) * (o - y[r]);
        gb += d;
      }
      gw += d * a;
      const float z = Z4[(long)r * HID + k];
      const float s = sigm(z);
      dZ4[(long)r * HID + k] = __float2bfloat16_rn(d * w5 * (s * (1.0f + z * (1.0f - s))));
    }
  }
  if (y) {
    atomicAdd(grad + kOffW5 + k, gw);
    if (k == 0) {
      atomicAdd(grad + kOffW5 + HID, gb);
      atomicAdd(loss, ls / (float)n);
    }
  }
}

__global__ void silu_back_kernel(const float *__restrict__ dA, const float *__restrict__ Z, __nv_bfloat16 *dZ,
                                 long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = Z[i];
  const float s = sigm(z);
  dZ[i] = __float2bfloat16_rn(dA[i] * (s * (1.0f + z * (1.0f - s))));
}

// db[c] += sum over rows of dZ[r][c]; block = HID threads, 256 rows each
__global__ void colsum_kernel(const __nv_bfloat16 *__restrict__ dZ, int n, float *db) {
  const int c = threadIdx.x;
  const int r0 = blockIdx.x * 256, r1 = min(n, r0 + 256);
  float s = 0.0f;
  for (int r = r0; r < r1; ++r) s += __bfloat162float(dZ[(long)r * HID + c]);
  atomicAdd(db + c, s);
}

struct AdamArgs {
  float lr, b1, b2, eps, c1, c2;  // c1 = 1/(1-b1^t), c2 = 1/(1-b2^t)
};

__global__ void adam_kernel(float *P, const float *__restrict__ G, float *Mo, float *Vo, AdamArgs a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float m = a.b1 * Mo[i] + (1.0f - a.b1) * g;
  const float v = a.b2 * Vo[i] + (1.0f - a.b2) * g * g;
  Mo[i] = m;
  Vo[i] = v;
  P[i] -= a.lr * (m * a.c1) / (sqrtf(v * a.c2) + a.eps);
}

// BF16 copies of W1..W4 in the [K][N] layout of the forward products
__global__ void refresh_bf16_kernel(const float *__restrict__ P, __nv_bfloat16 *Wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n1 = IN * HID, nh = HID * HID;
  if (i >= n1 + 3 * nh) return;
  int l, q;
  if (i < n1) { l = 0; q = i; }
  else { l = 1 + (i - n1) / nh; q = (i - n1) % nh; }
  Wb[i] = __float2bfloat16_rn(P[off_w(l) + q]);
}

// ---- FP32 inference (CUDA cores) ------------------------------------------------
// The whole forward pass for 32 grid points per block, in FP32 from the FP32
// master weights: features rounded to FP32 only (not BF16), hidden products
// as a 32 x 128 x K register-tiled SIMT product (thread: 2 rows x 8
// columns), bias + SiLU, the output layer by a warp reduction; u = s out.
// Used to evaluate the trained network without the BF16 rounding of the
// training path (whose grid-scale noise the undamped Jacobi smoother of the
// multigrid does not remove).
constexpr int kFR = 32;   // rows (grid points) per block
__global__ void __launch_bounds__(256) mlp_forward_fp32_kernel(const double *__restrict__ cond, int m, double dx,
                                                               const float *__restrict__ P, double s, double *u,
                                                               long np) {
  __shared__ float act[2][kFR][HID];
  const int t = threadIdx.x;
  const long first = (long)blockIdx.x * kFR;
  // features of the block's rows (the formulas of mlp_features_kernel)
  if (t < kFR) {
    float *f = act[0][t];
    const long p = min(first + t, np - 1);
    const double h0 = -0.5 * (m - 1) * dx;
    const int i = (int)(p % m), j = (int)((p / m) % m), k = (int)(p / ((long)m * m));
    const double x[3] = {h0 + i * dx, h0 + j * dx, h0 + k * dx};
    const double sc = 1.0 / 8.0;
    f[0] = (float)(x[0] * sc);
    f[1] = (float)(x[1] * sc);
    f[2] = (float)(x[2] * sc);
    for (int q = 0; q < 2; ++q) {
      const double mq = cond[q];
      const double d0 = x[0] - cond[2 + 3 * q], d1 = x[1] - cond[3 + 3 * q], d2 = x[2] - cond[4 + 3 * q];
      const double rr = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      float *g = f + 3 + 12 * q;
      g[0] = (float)(d0 * sc);
      g[1] = (float)(d1 * sc);
      g[2] = (float)(d2 * sc);
      g[3] = (float)(rr * sc);
      g[4] = (float)(mq / (rr + mq));
      g[5] = (float)(2.0 * mq);
      for (int a = 0; a < 3; ++a) {
        g[6 + a] = (float)(5.0 * cond[8 + 3 * q + a]);
        g[9 + a] = (float)(5.0 * cond[14 + 3 * q + a]);
      }
    }
    for (int q = 27; q < IN; ++q) f[q] = 0.0f;
  }
  __syncthreads();
  const int cg = t % 16, rg = t / 16;   // columns 8 cg .. 8 cg + 7, rows 2 rg, 2 rg + 1
  int cur = 0;
  for (int l = 0; l < 4; ++l) {
    const int K = fan_in(l);
    const float *W = P + off_w(l), *bias = P + off_b(l);
    float acc[2][8];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[r][c] = 0.0f;
    for (int k = 0; k < K; ++k) {
      float w[8], a[2];
#pragma unroll
      for (int c = 0; c < 8; ++c) w[c] = __ldg(W + (long)k * HID + 8 * cg + c);
#pragma unroll
      for (int r = 0; r < 2; ++r) a[r] = act[cur][2 * rg + r][k];
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(a[r], w[c], acc[r][c]);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float z = acc[r][c] + __ldg(bias + 8 * cg + c);
        act[cur ^ 1][2 * rg + r][8 * cg + c] = z * sigm(z);
      }
    __syncthreads();
    cur ^= 1;
  }
  // out = A4 w5 + b5: warp w reduces rows 4 w .. 4 w + 3
  const int w = t >> 5, lane = t & 31;
  const float *w5 = P + kOffW5;
  for (int r = 4 * w; r < 4 * w + 4; ++r) {
    float v = 0.0f;
    for (int k = lane; k < HID; k += 32) v = fmaf(act[cur][r][k], __ldg(w5 + k), v);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0 && first + r < np) u[first + r] = s * (double)(v + __ldg(w5 + HID));
  }
}

__global__ void scale_to_u_kernel(const float *__restrict__ o, double s, double *u, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u[i] = s * (double)o[i];
}

// ---- the forward pass on the 5th-generation tensor cores (tcgen05) ---------------
// One CTA of 512 threads per SM, two teams of 8 warps; each team walks its
// own tiles of 128 grid points with its own 128 columns of tensor memory,
// so the tensor core runs one team's layer while the other forms its
// activations.  W1..W4 sit in shared memory for the whole walk, as BF16 in
// the K-major layout without swizzle that the MMA reads through matrix
// descriptors: an operand of R rows and K columns is stored as K/8 chunks of
// R x 8 elements, each chunk row by row (16 B per row), so the 8-row core
// matrices are 128 B apart (stride byte offset) and the two 8-column chunks
// of one K = 16 step are 16 R bytes apart (leading byte offset).  Per tile:
// the features of the 128 points go into X; per layer one thread of the
// team issues the tcgen05.mma chain D[128 x 128] (FP32, tensor memory) =
// X or A (128 x K) * W^T and commits it to the team's mbarrier; thread
// (row, half) of the team then reads columns 64 half .. 64 half + 63 of its
// row of D (tcgen05.ld: warp w reaches lanes 32 (w mod 4) ..), adds the
// bias, applies SiLU, rounds to BF16 and writes the next layer's A (after
// layer 4 the two halves form out = A4 w5 + b5).  Operands BF16,
// accumulation FP32: the arithmetic of the training path.  SiLU is
// z sigm(z) = z/2 (1 + tanh(z/2)) with the hardware tanh (tanh.approx.f32,
// relative error about 2^-11, below the BF16 rounding that follows).
namespace tc {
constexpr int kRows = 128;
constexpr int kThreads = 512;                    // two teams of 256
constexpr int kChunk = kRows * 16;               // bytes of one 8-column chunk of a 128-row operand
constexpr int kOffW0 = 0;                        // W1^T: 128 x 32, 4 chunks
constexpr int kOffW = kOffW0 + 4 * kChunk;       // W2^T, W3^T, W4^T: 128 x 128, 16 chunks each
constexpr int kOffX = kOffW + 3 * 16 * kChunk;   // features, per team: 128 x 32
constexpr int kOffA = kOffX + 2 * 4 * kChunk;    // activations, per team: 128 x 128
constexpr int kOffP = kOffA + 2 * 16 * kChunk;   // b1..b4 [4][128], w5 [128], b5 (FP32)
constexpr int kOffRed = kOffP + ((4 * HID + HID + 1) * 4 + 15) / 16 * 16;   // per team: 128 partial outputs
constexpr int kOffBar = kOffRed + 2 * kRows * 4; // 2 mbarriers
constexpr int kOffTmem = kOffBar + 16;           // the tensor-memory base address; 2 timeout flags
constexpr int kSmem = kOffTmem + 16 + 128;       // + room to align the base to 128 B
static_assert(kSmem <= 227 * 1024, "shared memory of the tensor-core forward");
// the instruction descriptor of kind::f16: FP32 accumulator, A and B BF16,
// both K-major, N = 128 (bits 17-22: N/8), M = 128 (bits 24-28: M/16)
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

// byte offset of element (row, k) in a chunked K-major operand
__device__ __forceinline__ int off(int row, int k) { return (k >> 3) * kChunk + row * 16 + (k & 7) * 2; }

// shared-memory matrix descriptor (sm_100): start address >> 4 (bits 0-13),
// leading byte offset >> 4 (bits 16-29: between the two K chunks of one
// MMA), stride byte offset >> 4 (bits 32-45: between 8-row core matrices),
// version 1 (bits 46-47), base offset 0, no swizzle (bits 61-63 zero)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kChunk >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((128 >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(dtmem), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   tma::smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// barrier of one team (named barriers 1 and 2)
__device__ __forceinline__ void team_sync(int team) { asm volatile("bar.sync %0, 256;" ::"r"(team + 1) : "memory"); }

__device__ __forceinline__ float silu(float z) {
  float th;
  const float h = 0.5f * z;
  asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(h));
  return fmaf(h, th, h);
}
// two FP32 values rounded to nearest even BF16, packed (lower column low)
template <int CVT>
__device__ __forceinline__ uint32_t pack_bf16(float x0, float x1) {
  if (CVT == 0) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(x0, x1);
    return *reinterpret_cast<const uint32_t *>(&v);
  }
  // round to nearest even on the bits (finite values): add 0x7FFF plus the
  // lowest kept bit, keep the upper 16 bits
  uint32_t u0 = __float_as_uint(x0), u1 = __float_as_uint(x1);
  u0 += 0x7FFFu + ((u0 >> 16) & 1u);
  u1 += 0x7FFFu + ((u1 >> 16) & 1u);
  return __byte_perm(u0, u1, 0x7632);
}

// 32 consecutive FP32 columns of this thread's row (warp-collective); the
// caller waits (tcgen05.wait::ld) before using them
__device__ __forceinline__ void ld32(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
}  // namespace tc

template <int CVT>
__global__ void __launch_bounds__(tc::kThreads, 1) mlp_forward_tc_kernel(const double *__restrict__ cond, int m,
                                                                        double dx, const float *__restrict__ P,
                                                                        double uscale, double *u, long np,
                                                                        int *status) {
  using namespace tc;
  extern __shared__ __align__(128) unsigned char tc_raw[];
  unsigned char *sm = tc_raw + ((128 - (tma::smem_addr(tc_raw) & 127)) & 127);
  const int t = threadIdx.x, warp = t >> 5, team = t >> 8, tr = t & 255, r = tr & 127, half = tr >> 7;
  const uint32_t sbase = tma::smem_addr(sm);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kOffBar) + team;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kOffTmem);
  volatile int *failed = reinterpret_cast<volatile int *>(sm + kOffTmem + 4);
  float *par = reinterpret_cast<float *>(sm + kOffP);
  float *red = reinterpret_cast<float *>(sm + kOffRed) + team * kRows;
  // the weights, transposed to [n][k] in the chunked layout, and the biases
  for (int idx = t; idx < IN * HID; idx += kThreads) {
    const int k = idx / HID, n = idx % HID;
    *reinterpret_cast<__nv_bfloat16 *>(sm + kOffW0 + off(n, k)) = __float2bfloat16_rn(P[off_w(0) + idx]);
  }
  for (int l = 1; l < 4; ++l)
    for (int idx = t; idx < HID * HID; idx += kThreads) {
      const int k = idx / HID, n = idx % HID;
      *reinterpret_cast<__nv_bfloat16 *>(sm + kOffW + (l - 1) * 16 * kChunk + off(n, k)) =
          __float2bfloat16_rn(P[off_w(l) + idx]);
    }
  for (int idx = t; idx < 4 * HID; idx += kThreads) par[idx] = P[off_b(idx / HID) + idx % HID];
  for (int idx = t; idx <= HID; idx += kThreads) par[4 * HID + idx] = P[kOffW5 + idx];
  // 256 columns of tensor memory: the FP32 accumulators (128 x 128) of the
  // two teams
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tma::smem_addr(tslot)),
                 "r"(256u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t < 2) {
    tma::mbar_init(reinterpret_cast<uint64_t *>(sm + kOffBar) + t, 1);
    failed[t] = 0;
  }
  if (t == 0) tma::mbar_fence_init();
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t dcol = tmem + 128u * team;                                          // the team's accumulator
  const uint32_t trow = dcol + ((uint32_t)(32 * (warp & 3)) << 16) + 64u * half;     // this thread's lanes/half
  unsigned char *X = sm + kOffX + team * 4 * kChunk;
  unsigned char *A = sm + kOffA + team * 16 * kChunk;
  const float *w5 = par + 4 * HID;
  uint32_t phase = 0;
  const long ntiles = (np + kRows - 1) / kRows;
  for (long tile = 2L * blockIdx.x + team; tile < ntiles; tile += 2L * gridDim.x) {
    const long row = tile * kRows + r;
    {
      // features of this thread's point (mlp_features_kernel's formulas):
      // half 0 forms columns 0-15 (the coordinates, the first puncture's
      // twelve, the second's x offset), half 1 columns 16-31
      const long pp = row < np ? row : np - 1;
      int i, j, k;
      if (np <= 0x7FFFFFFFL) {
        const unsigned q = (unsigned)pp, um = (unsigned)m, qm = q / um;
        i = (int)(q - qm * um);
        j = (int)(qm % um);
        k = (int)(qm / um);
      } else {
        i = (int)(pp % m);
        j = (int)((pp / m) % m);
        k = (int)(pp / ((long)m * m));
      }
      const double h0 = -0.5 * (m - 1) * dx;
      const double x[3] = {h0 + i * dx, h0 + j * dx, h0 + k * dx};
      const double sc = 1.0 / 8.0;
      __align__(16) __nv_bfloat16 f[16];
      const int q = half;
      const double mq = cond[q];
      const double d0 = x[0] - cond[2 + 3 * q], d1 = x[1] - cond[3 + 3 * q], d2 = x[2] - cond[4 + 3 * q];
      const double rr = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      const double g[12] = {d0 * sc, d1 * sc, d2 * sc, rr * sc, mq / (rr + mq), 2.0 * mq,
                            5.0 * cond[8 + 3 * q], 5.0 * cond[9 + 3 * q], 5.0 * cond[10 + 3 * q],
                            5.0 * cond[14 + 3 * q], 5.0 * cond[15 + 3 * q], 5.0 * cond[16 + 3 * q]};
      if (half == 0) {
        f[0] = to_bf16(x[0] * sc);
        f[1] = to_bf16(x[1] * sc);
        f[2] = to_bf16(x[2] * sc);
#pragma unroll
        for (int c = 0; c < 12; ++c) f[3 + c] = to_bf16(g[c]);
        f[15] = to_bf16((x[0] - cond[5]) * sc);
      } else {
#pragma unroll
        for (int c = 1; c < 12; ++c) f[c - 1] = to_bf16(g[c]);
#pragma unroll
        for (int c = 11; c < 16; ++c) f[c] = __float2bfloat16_rn(0.0f);
      }
#pragma unroll
      for (int c = 0; c < 2; ++c)
        *reinterpret_cast<uint4 *>(X + off(r, 16 * half + 8 * c)) = *reinterpret_cast<const uint4 *>(f + 8 * c);
    }
    float out = 0.0f;
    for (int l = 0; l < 4; ++l) {
      // the operand was written by the threads: make it visible to the
      // tensor core, then one thread issues the layer's MMA chain
      fence_async_smem();
      fence_before();
      team_sync(team);
      fence_after();
      if (failed[team]) break;   // read after the barrier: the same in every thread of the team
      if (tr == 0) {
        const uint32_t a0 = sbase + (uint32_t)((l == 0 ? X : A) - sm);
        const uint32_t b0 = sbase + (uint32_t)(l == 0 ? kOffW0 : kOffW + (l - 1) * 16 * kChunk);
        const int ks = fan_in(l) / 16;
        for (int s = 0; s < ks; ++s)
          mma(dcol, sdesc(a0 + s * 2 * kChunk), sdesc(b0 + s * 2 * kChunk), s > 0 ? 1u : 0u);
        commit(bar);
      }
      __syncwarp();
      // a warp whose wait ran out skips the (warp-collective) tensor-memory
      // reads; the team leaves the walk at its next barrier
      if (!__all_sync(0xffffffffu, tma::mbar_wait(bar, phase))) {
        failed[team] = 1;
        continue;
      }
      phase ^= 1u;
      fence_after();
      uint32_t acc[64];
      ld32(trow, acc);
      ld32(trow + 32, acc + 32);
      ld_wait();
      const float4 *bias = reinterpret_cast<const float4 *>(par + l * HID + 64 * half);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        // the bias (and w5) as 16-byte broadcast reads of shared memory
        const float4 b0 = bias[2 * c], b1 = bias[2 * c + 1];
        const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = silu(__uint_as_float(acc[8 * c + q]) + bb[q]);
        uint4 pk;
        pk.x = pack_bf16<CVT>(v[0], v[1]);
        pk.y = pack_bf16<CVT>(v[2], v[3]);
        pk.z = pack_bf16<CVT>(v[4], v[5]);
        pk.w = pack_bf16<CVT>(v[6], v[7]);
        if (l < 3) {
          *reinterpret_cast<uint4 *>(A + off(r, 64 * half + 8 * c)) = pk;
        } else {
          const uint32_t w[4] = {pk.x, pk.y, pk.z, pk.w};
          const float4 *w5v = reinterpret_cast<const float4 *>(w5 + 64 * half + 8 * c);
          const float4 c0 = w5v[0], c1 = w5v[1];
          const float cc[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            out = fmaf(__uint_as_float(w[q] << 16), cc[2 * q], out);
            out = fmaf(__uint_as_float(w[q] & 0xFFFF0000u), cc[2 * q + 1], out);
          }
        }
      }
    }
    // out = A4 w5 + b5 from the two halves of the row
    if (half == 1) red[r] = out;
    team_sync(team);
    if (failed[team]) break;
    if (half == 0 && row < np) u[row] = uscale * (double)(out + red[r] + w5[HID]);
    // this tile's tensor-memory reads are done before the next tile's first
    // MMA overwrites the accumulator (the barrier at the next layer start)
    fence_before();
  }
  if (failed[team] && tr == 0) {
    // an MMA chain still in flight is waited for (bounded) before the
    // tensor memory is freed
    atomicOr(status, 1);
    tma::mbar_wait(bar, phase);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u) : "memory");
}

long wb_off(int l) { return l == 0 ? 0 : (long)IN * HID + (long)(l - 1) * HID * HID; }

}  // namespace

struct nrgpu_mlp {
  int device;
  int max_batch;
  float *P, *G, *Mo, *Vo;  // master params, gradients, Adam moments
  __nv_bfloat16 *Wb;       // BF16 W1..W4
  __nv_bfloat16 *X;        // [max_batch][IN]
  float *Z[4];             // [max_batch][HID] pre-activations
  __nv_bfloat16 *Ab[4];    // [max_batch][HID] activations
  float *dA;               // [max_batch][HID]
  __nv_bfloat16 *dZ;       // [max_batch][HID]
  float *out, *y, *loss;
  double *cond;            // the conditioning table
  int ncond;
  int *d_tcstatus;         // a wait of the tensor-core forward ran out
  long adam_t;
};

namespace {

int check_dims(int M, int N, int K) {
  if (M % 16 || N % 16 || K % TK || M <= 0 || N <= 0 || K <= 0)
    return nrgpu_set_error(NRGPU_ERR_ARG, "gemm dims %d x %d x %d (M, N multiples of 16, K of 32)", M, N, K);
  return NRGPU_OK;
}

template <bool AT, bool BT>
int gemm(const __nv_bfloat16 *A, const __nv_bfloat16 *B, float *C, int M, int N, int K, int splits,
         cudaStream_t st) {
  int e = check_dims(M, N, K);
  if (e) return e;
  const dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM, 1);
  if (splits > 1) {
    int kc = (K + splits - 1) / splits;
    kc = (kc + TK - 1) / TK * TK;
    NRGPU_CUDA_TRY(cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * N, st));
    gemm_bf16_kernel<AT, BT, true><<<dim3(grid.x, grid.y, (K + kc - 1) / kc), 128, 0, st>>>(A, B, C, M, N, K, kc);
  } else {
    gemm_bf16_kernel<AT, BT, false><<<grid, 128, 0, st>>>(A, B, C, M, N, K, K);
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

inline int nb(long n, int t = 256) { return (int)((n + t - 1) / t); }

// forward of n rows already featurised in M->X; fills Z, Ab
int forward(nrgpu_mlp *M, int n, cudaStream_t st) {
  const __nv_bfloat16 *in = M->X;
  for (int l = 0; l < 4; ++l) {
    int e = gemm<false, false>(in, M->Wb + wb_off(l), M->Z[l], n, HID, fan_in(l), 1, st);
    if (e) return e;
    bias_silu_kernel<<<nb((long)n * HID), 256, 0, st>>>(M->Z[l], M->P + off_b(l), M->Ab[l], (long)n * HID);
    in = M->Ab[l];
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

int set_cond(nrgpu_mlp *M, const double *host_cond, int nsets) {
  if (nsets > M->ncond) {
    cudaFree(M->cond);
    if (cudaMalloc(&M->cond, sizeof(double) * 20 * nsets) != cudaSuccess) {
      M->cond = nullptr;
      M->ncond = 0;
      cudaGetLastError();
      return nrgpu_set_error(NRGPU_ERR_NOMEM, "conditioning table");
    }
    M->ncond = nsets;
  }
  NRGPU_CUDA_TRY(cudaMemcpy(M->cond, host_cond, sizeof(double) * 20 * nsets, cudaMemcpyHostToDevice));
  return NRGPU_OK;
}

}  // namespace

extern "C" int nrgpu_mlp_nparams(void) { return kNParams; }

extern "C" int nrgpu_mlp_create(int max_batch, nrgpu_mlp **out) {
  if (!out || max_batch < 64 || max_batch % 64) return nrgpu_set_error(NRGPU_ERR_ARG, "max_batch: a multiple of 64");
  nrgpu_mlp *M = (nrgpu_mlp *)calloc(1, sizeof(nrgpu_mlp));
  if (!M) return nrgpu_set_error(NRGPU_ERR_NOMEM, "host allocation");
  cudaGetDevice(&M->device);
  M->max_batch = max_batch;
  const size_t nh = (size_t)max_batch * HID;
  bool ok = cudaMalloc(&M->P, sizeof(float) * kNParams) == cudaSuccess &&
            cudaMalloc(&M->G, sizeof(float) * kNParams) == cudaSuccess &&
            cudaMalloc(&M->Mo, sizeof(float) * kNParams) == cudaSuccess &&
            cudaMalloc(&M->Vo, sizeof(float) * kNParams) == cudaSuccess &&
            cudaMalloc(&M->Wb, sizeof(__nv_bfloat16) * (IN * HID + 3 * HID * HID)) == cudaSuccess &&
            cudaMalloc(&M->X, sizeof(__nv_bfloat16) * (size_t)max_batch * IN) == cudaSuccess &&
            cudaMalloc(&M->dA, sizeof(float) * nh) == cudaSuccess &&
            cudaMalloc(&M->dZ, sizeof(__nv_bfloat16) * nh) == cudaSuccess &&
            cudaMalloc(&M->out, sizeof(float) * max_batch) == cudaSuccess &&
            cudaMalloc(&M->y, sizeof(float) * max_batch) == cudaSuccess &&
            cudaMalloc(&M->loss, sizeof(float)) == cudaSuccess &&
            cudaMalloc(&M->d_tcstatus, sizeof(int)) == cudaSuccess &&
            cudaMemset(M->d_tcstatus, 0, sizeof(int)) == cudaSuccess;
  for (int l = 0; l < 4 && ok; ++l)
    ok = cudaMalloc(&M->Z[l], sizeof(float) * nh) == cudaSuccess &&
         cudaMalloc(&M->Ab[l], sizeof(__nv_bfloat16) * nh) == cudaSuccess;
  if (ok)
    ok = cudaMemset(M->P, 0, sizeof(float) * kNParams) == cudaSuccess &&
         cudaMemset(M->G, 0, sizeof(float) * kNParams) == cudaSuccess &&
         cudaMemset(M->Mo, 0, sizeof(float) * kNParams) == cudaSuccess &&
         cudaMemset(M->Vo, 0, sizeof(float) * kNParams) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    nrgpu_mlp_destroy(M);
    return nrgpu_set_error(NRGPU_ERR_NOMEM, "device allocation of the network (batch %d)", max_batch);
  }
  *out = M;
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_destroy(nrgpu_mlp *M) {
  if (!M) return NRGPU_OK;
  cudaFree(M->P); cudaFree(M->G); cudaFree(M->Mo); cudaFree(M->Vo); cudaFree(M->Wb); cudaFree(M->X);
  cudaFree(M->dA); cudaFree(M->dZ); cudaFree(M->out); cudaFree(M->y); cudaFree(M->loss); cudaFree(M->cond);
  cudaFree(M->d_tcstatus);
  for (int l = 0; l < 4; ++l) {
    cudaFree(M->Z[l]);
    cudaFree(M->Ab[l]);
  }
  free(M);
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_set_params(nrgpu_mlp *M, const float *host, int n) {
  if (!M || !host || n != kNParams) return nrgpu_set_error(NRGPU_ERR_ARG, "parameter count %d != %d", n, kNParams);
  NRGPU_CUDA_TRY(cudaMemcpy(M->P, host, sizeof(float) * kNParams, cudaMemcpyHostToDevice));
  NRGPU_CUDA_TRY(cudaMemset(M->Mo, 0, sizeof(float) * kNParams));
  NRGPU_CUDA_TRY(cudaMemset(M->Vo, 0, sizeof(float) * kNParams));
  M->adam_t = 0;
  refresh_bf16_kernel<<<nb(IN * HID + 3 * HID * HID), 256>>>(M->P, M->Wb);
  NRGPU_CUDA_TRY(cudaGetLastError());
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_get_params(nrgpu_mlp *M, float *host, int n) {
  if (!M || !host || n != kNParams) return nrgpu_set_error(NRGPU_ERR_ARG, "parameter count %d != %d", n, kNParams);
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  NRGPU_CUDA_TRY(cudaMemcpy(host, M->P, sizeof(float) * kNParams, cudaMemcpyDeviceToHost));
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_set_conditions(nrgpu_mlp *M, const double *host_cond, int nsets) {
  if (!M || !host_cond || nsets < 1) return nrgpu_set_error(NRGPU_ERR_ARG, "bad conditioning table");
  return set_cond(M, host_cond, nsets);
}

extern "C" int nrgpu_mlp_features(nrgpu_mlp *M, const int *d_set, const int *d_pt, int n, int m, double dx,
                                  void *stream) {
  if (!M || !d_set || !d_pt || n < 1 || n > M->max_batch || m < 2 || !M->cond)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad feature arguments (conditioning table set?)");
  mlp_features_kernel<<<nb(n), 256, 0, (cudaStream_t)stream>>>(M->cond, d_set, d_pt, 0, n, Feat{m, dx}, M->X);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_copy_features(nrgpu_mlp *M, int n, uint16_t *host) {
  if (!M || !host || n < 1 || n > M->max_batch) return nrgpu_set_error(NRGPU_ERR_ARG, "bad feature copy");
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  NRGPU_CUDA_TRY(cudaMemcpy(host, M->X, sizeof(uint16_t) * (size_t)n * IN, cudaMemcpyDeviceToHost));
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_train_step(nrgpu_mlp *M, const float *d_y, int n, float lr, int update, float *loss,
                                    void *stream) {
  if (!M || !d_y || n < 64 || n % 64 || n > M->max_batch)
    return nrgpu_set_error(NRGPU_ERR_ARG, "batch %d: a multiple of 64 up to %d", n, M ? M->max_batch : 0);
  const cudaStream_t st = (cudaStream_t)stream;
  int e = forward(M, n, st);
  if (e) return e;
  NRGPU_CUDA_TRY(cudaMemsetAsync(M->G, 0, sizeof(float) * kNParams, st));
  NRGPU_CUDA_TRY(cudaMemsetAsync(M->loss, 0, sizeof(float), st));
  const int rpb = 64;
  out_layer_kernel<<<(n + rpb - 1) / rpb, HID, 0, st>>>(M->Ab[3], M->Z[3], M->P, M->out, d_y, n, rpb, M->G, M->dZ,
                                                        M->loss);
  NRGPU_CUDA_TRY(cudaGetLastError());
  const int splits = max(1, min(64, n / 1024));
  for (int l = 3; l >= 0; --l) {
    // dW_l = A_{l-1}^T dZ_l straight into its [fan_in][HID] slot of G,
    // db_l = column sums of dZ_l
    const __nv_bfloat16 *Ain = l ? M->Ab[l - 1] : M->X;
    e = gemm<true, false>(Ain, M->dZ, M->G + off_w(l), fan_in(l), HID, n, splits, st);
    if (e) return e;
    colsum_kernel<<<(n + 255) / 256, HID, 0, st>>>(M->dZ, n, M->G + off_b(l));
    NRGPU_CUDA_TRY(cudaGetLastError());
    if (l == 0) break;
    // dA_{l-1} = dZ_l W_l^T, dZ_{l-1} = dA * silu'(Z_{l-1})
    e = gemm<false, true>(M->dZ, M->Wb + wb_off(l), M->dA, n, HID, HID, 1, st);
    if (e) return e;
    silu_back_kernel<<<nb((long)n * HID), 256, 0, st>>>(M->dA, M->Z[l - 1], M->dZ, (long)n * HID);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  if (update) {
    M->adam_t++;
    AdamArgs a;
    a.lr = lr; a.b1 = 0.9f; a.b2 = 0.999f; a.eps = 1e-8f;
    a.c1 = (float)(1.0 / (1.0 - pow(0.9, (double)M->adam_t)));
    a.c2 = (float)(1.0 / (1.0 - pow(0.999, (double)M->adam_t)));
    adam_kernel<<<nb(kNParams), 256, 0, st>>>(M->P, M->G, M->Mo, M->Vo, a, kNParams);
    refresh_bf16_kernel<<<nb(IN * HID + 3 * HID * HID), 256, 0, st>>>(M->P, M->Wb);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  if (loss) {
    NRGPU_CUDA_TRY(cudaMemcpyAsync(loss, M->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    NRGPU_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_gradients(nrgpu_mlp *M, float *host_grad, int n_params) {
  if (!M || !host_grad || n_params != kNParams) return nrgpu_set_error(NRGPU_ERR_ARG, "gradient buffer");
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  NRGPU_CUDA_TRY(cudaMemcpy(host_grad, M->G, sizeof(float) * kNParams, cudaMemcpyDeviceToHost));
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_forward(nrgpu_mlp *M, int n, float *d_out, void *stream) {
  if (!M || !d_out || n < 16 || n % 16 || n > M->max_batch)
    return nrgpu_set_error(NRGPU_ERR_ARG, "rows %d: a multiple of 16 up to %d", n, M ? M->max_batch : 0);
  const cudaStream_t st = (cudaStream_t)stream;
  int e = forward(M, n, st);
  if (e) return e;
  out_layer_kernel<<<(n + 63) / 64, HID, 0, st>>>(M->Ab[3], M->Z[3], M->P, d_out, nullptr, n, 64, nullptr, nullptr,
                                                  nullptr);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_predict_u(nrgpu_mlp *M, const double *host_cond, int m, double dx, double uscale, double *u,
                                   void *stream) {
  if (!M || !host_cond || !u || m < 2) return nrgpu_set_error(NRGPU_ERR_ARG, "bad prediction arguments");
  const cudaStream_t st = (cudaStream_t)stream;
  NRGPU_CUDA_TRY(cudaStreamSynchronize(st));  // the table is replaced below
  int e = set_cond(M, host_cond, 1);
  if (e) return e;
  const long np = (long)m * m * m;
  for (long first = 0; first < np; first += M->max_batch) {
    const int n = (int)min((long)M->max_batch, np - first);
    const int n16 = (n + 15) / 16 * 16;  // rows past np are computed and dropped
    mlp_features_kernel<<<nb(n16), 256, 0, st>>>(M->cond, nullptr, nullptr, first, n16, Feat{m, dx}, M->X);
    NRGPU_CUDA_TRY(cudaGetLastError());
    e = forward(M, n16, st);
    if (e) return e;
    out_layer_kernel<<<(n16 + 63) / 64, HID, 0, st>>>(M->Ab[3], M->Z[3], M->P, M->out, nullptr, n16, 64, nullptr,
                                                      nullptr, nullptr);
    scale_to_u_kernel<<<nb(n), 256, 0, st>>>(M->out, uscale, u + first, n);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_predict_u_fp32(nrgpu_mlp *M, const double *host_cond, int m, double dx, double uscale,
                                        double *u, void *stream) {
  if (!M || !host_cond || !u || m < 2) return nrgpu_set_error(NRGPU_ERR_ARG, "bad prediction arguments");
  const cudaStream_t st = (cudaStream_t)stream;
  NRGPU_CUDA_TRY(cudaStreamSynchronize(st));  // the table is replaced below
  int e = set_cond(M, host_cond, 1);
  if (e) return e;
  const long np = (long)m * m * m;
  mlp_forward_fp32_kernel<<<(unsigned)((np + kFR - 1) / kFR), 256, 0, st>>>(M->cond, m, dx, M->P, uscale, u, np);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_predict_u_tc(nrgpu_mlp *M, const double *host_cond, int m, double dx, double uscale,
                                      double *u, void *stream) {
  if (!M || !host_cond || !u || m < 2) return nrgpu_set_error(NRGPU_ERR_ARG, "bad prediction arguments");
  const cudaStream_t st = (cudaStream_t)stream;
  NRGPU_CUDA_TRY(cudaStreamSynchronize(st));  // the table is replaced below
  int e = set_cond(M, host_cond, 1);
  if (e) return e;
  static bool attr_set[64] = {};
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) {
    cudaGetLastError();
    nsm = 148;
  }
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    NRGPU_CUDA_TRY(cudaFuncSetAttribute(mlp_forward_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmem));
    attr_set[dev] = true;
  }
  const long np = (long)m * m * m;
  const long pairs = ((np + tc::kRows - 1) / tc::kRows + 1) / 2;
  const unsigned grid = (unsigned)(pairs < nsm ? pairs : nsm);
  NRGPU_CUDA_TRY(cudaMemsetAsync(M->d_tcstatus, 0, sizeof(int), st));
  mlp_forward_tc_kernel<0><<<grid, tc::kThreads, tc::kSmem, st>>>(M->cond, m, dx, M->P, uscale, u, np, M->d_tcstatus);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_mlp_tc_status(nrgpu_mlp *M, int *timed_out) {
  if (!M || !timed_out) return nrgpu_set_error(NRGPU_ERR_ARG, "bad status arguments");
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  NRGPU_CUDA_TRY(cudaMemcpy(timed_out, M->d_tcstatus, sizeof(int), cudaMemcpyDeviceToHost));
  return *timed_out ? nrgpu_set_error(NRGPU_ERR_TIMEOUT, "a wait of the tensor-core forward ran out") : NRGPU_OK;
}
