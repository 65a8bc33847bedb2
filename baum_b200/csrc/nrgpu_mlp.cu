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
            cudaMalloc(&M->loss, sizeof(float)) == cudaSuccess;
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
