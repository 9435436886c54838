// Learned gauge predictor: network object, training (forward, backward and
// Adam on the GPU), inference fused with the feature gather, and the
// collection of training pairs from the plain step.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "pond_internal.h"
#include "pond_mlp_kernels.cuh"

struct pond_mlp {
  int H = 64;
  int device = 0;
  int nparams = 0;
  float* P = nullptr;       // float32 master parameters
  float* M = nullptr;       // Adam first moment
  float* V = nullptr;       // Adam second moment
  float* stats = nullptr;   // xmean, xstd, ymean, ystd
  float* partials = nullptr;
  int max_cta = 0;
  float* loss_parts = nullptr;
  float* d_loss = nullptr;  // per-step loss (capacity loss_cap)
  int loss_cap = 0;
  int adam_t = 0;
  cudaStream_t stream = nullptr;
};

namespace pond {
namespace mlp {

template <int H> struct Cfg;
template <> struct Cfg<64> { static constexpr int S = 128; };   // samples per training CTA
template <> struct Cfg<128> { static constexpr int S = 64; };

template <int H> struct TrainSmem {
  static constexpr int S = Cfg<H>::S;
  WeightsSmem<H> w;
  __nv_bfloat16 X[S][K1 + PAD];
  __nv_bfloat16 XT[K1][S + PAD];
  __nv_bfloat16 H1T[H][S + PAD];
  __nv_bfloat16 H2T[H][S + PAD];
  __nv_bfloat16 D1T[H][S + PAD];
  __nv_bfloat16 D2T[H][S + PAD];
  __nv_bfloat16 D3T[OUTP][S + PAD];
  float Y[S][NOUT];
  float db[2 * H + OUTP];
  float loss;
};

// One CTA: S samples, forward + backward on tensor cores, this CTA's share of
// the parameter gradient written to partials[blockIdx.x][:] (and the summed
// squared error to loss_parts[blockIdx.x]).
template <int H>
__global__ void __launch_bounds__(128) train_kernel(const float* P, const float* stats, const float* Xr,
                                                    const float* Yr, long long n, const long long* start_ptr,
                                                    long long start_host, float inv_batch, float* partials,
                                                    float* loss_parts) {
  using Lay = Layout<H>;
  constexpr int S = Cfg<H>::S;
  constexpr int MT = S / 64;  // m16 tiles per warp (4 warps)
  extern __shared__ __align__(16) unsigned char raw[];
  TrainSmem<H>& T = *reinterpret_cast<TrainSmem<H>*>(raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  load_weights<H>(T.w, P, stats);
  for (int i = tid; i < 2 * H + OUTP; i += 128) T.db[i] = 0.f;
  for (int i = tid; i < OUTP * (S + PAD); i += 128) (&T.D3T[0][0])[i] = __float2bfloat16(0.f);
  if (tid == 0) T.loss = 0.f;
  __syncthreads();
  const long long start = start_ptr ? *start_ptr : start_host;
  for (int i = tid; i < S * K1; i += 128) {
    const int r = i / K1, k = i % K1;
    const long long s = (start + (long long)blockIdx.x * S + r) % n;
    const float v = k < NIN ? (Xr[s * NIN + k] - T.w.xmean[k]) * T.w.xistd[k] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16(v);
    T.X[r][k] = b;
    T.XT[k][r] = b;
  }
  for (int i = tid; i < S * NOUT; i += 128) {
    const int r = i / NOUT, o = i % NOUT;
    const long long s = (start + (long long)blockIdx.x * S + r) % n;
    T.Y[r][o] = (Yr[s * NOUT + o] - T.w.ymean[o]) / T.w.ystd[o];
  }
  __syncthreads();
  float lsum = 0.f;
  float dbl[2][H / 8][2];
#pragma unroll
  for (int nt = 0; nt < H / 8; nt++) dbl[0][nt][0] = dbl[0][nt][1] = dbl[1][nt][0] = dbl[1][nt][1] = 0.f;
  float db3[2] = {0.f, 0.f};
#pragma unroll
  for (int mt = 0; mt < MT; mt++) {
    const int r0 = warp * (S / 4) + mt * 16;
    float h1[H / 8][4], h2[H / 8][4], y[4];
    forward_tile<H>(T.w, &T.X[0][0], K1 + PAD, r0, lane, h1, h2, y);
    // d loss / d y (standardised), loss = sum (y - y*)^2 / batch
    float d3[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int row = r0 + g + 8 * (q >> 1), col = 2 * t + (q & 1);
      const bool valid = col < NOUT;
      const float diff = valid ? y[q] - T.Y[row][col] : 0.f;
      lsum += diff * diff;
      d3[q] = 2.f * diff * inv_batch;
      T.D3T[col][row] = __float2bfloat16(d3[q]);
    }
    db3[0] += d3[0] + d3[2];
    db3[1] += d3[1] + d3[3];
    // dH2 = dZ3 W3
    float dh2[H / 8][4];
    {
      const uint32_t a[4] = {pack_bf16(d3[0], d3[1]), pack_bf16(d3[2], d3[3]), 0u, 0u};
#pragma unroll
      for (int nt = 0; nt < H / 8; nt++) {
        dh2[nt][0] = dh2[nt][1] = dh2[nt][2] = dh2[nt][3] = 0.f;
        uint32_t b[2];
        frag_b(b, &T.w.W3T[0][0], OUTP + PAD, 0, nt * 8, lane);
        mma16816(dh2[nt], a, b);
      }
    }
    // dZ2 = dH2 (1 - h2^2); keep h2 and dZ2 (transposed) for the weight gradients
#pragma unroll
    for (int nt = 0; nt < H / 8; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int row = r0 + g + 8 * (q >> 1), col = nt * 8 + 2 * t + (q & 1);
        dh2[nt][q] *= 1.f - h2[nt][q] * h2[nt][q];
        T.H2T[col][row] = __float2bfloat16(h2[nt][q]);
        T.D2T[col][row] = __float2bfloat16(dh2[nt][q]);
        dbl[1][nt][q & 1] += dh2[nt][q];
      }
    // dH1 = dZ2 W2
    float dh1[H / 8][4];
#pragma unroll
    for (int nt = 0; nt < H / 8; nt++) dh1[nt][0] = dh1[nt][1] = dh1[nt][2] = dh1[nt][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < H / 16; kk++) {
      uint32_t a[4];
      acc_to_a(a, dh2[2 * kk], dh2[2 * kk + 1]);
#pragma unroll
      for (int nt = 0; nt < H / 8; nt++) {
        uint32_t b[2];
        frag_b(b, &T.w.W2T[0][0], H + PAD, kk * 16, nt * 8, lane);
        mma16816(dh1[nt], a, b);
      }
    }
#pragma unroll
    for (int nt = 0; nt < H / 8; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int row = r0 + g + 8 * (q >> 1), col = nt * 8 + 2 * t + (q & 1);
        dh1[nt][q] *= 1.f - h1[nt][q] * h1[nt][q];
        T.H1T[col][row] = __float2bfloat16(h1[nt][q]);
        T.D1T[col][row] = __float2bfloat16(dh1[nt][q]);
        dbl[0][nt][q & 1] += dh1[nt][q];
      }
  }
  // bias gradients: reduce over the 8 row groups of the warp, then shared atomics
#pragma unroll
  for (int L = 0; L < 2; L++)
#pragma unroll
    for (int nt = 0; nt < H / 8; nt++)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        float v = dbl[L][nt][j];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        if (g == 0) atomicAdd(&T.db[L * H + nt * 8 + 2 * t + j], v);
      }
#pragma unroll
  for (int j = 0; j < 2; j++) {
    float v = db3[j];
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    if (g == 0 && 2 * t + j < NOUT) atomicAdd(&T.db[2 * H + 2 * t + j], v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) atomicAdd(&T.loss, lsum);
  __syncthreads();
  // weight gradients dW = dZ^T A over this CTA's samples (tensor cores)
  float* out = partials + (long long)blockIdx.x * Lay::SIZE;
  constexpr int NT1 = H / 16, NT2 = H / 16, NTASK = NT1 + NT2 + 1;
  for (int task = warp; task < NTASK; task += 4) {
    const __nv_bfloat16* A;
    const __nv_bfloat16* Bt;
    int m0, ncols, ldb, off, rows_valid, ldw;
    if (task < NT1) {  // dW1 = D1T X
      A = &T.D1T[0][0]; Bt = &T.XT[0][0]; m0 = task * 16; ncols = K1; ldb = S + PAD;
      off = Lay::W1; rows_valid = H; ldw = NIN;
    } else if (task < NT1 + NT2) {  // dW2 = D2T H1
      A = &T.D2T[0][0]; Bt = &T.H1T[0][0]; m0 = (task - NT1) * 16; ncols = H; ldb = S + PAD;
      off = Lay::W2; rows_valid = H; ldw = H;
    } else {  // dW3 = D3T H2
      A = &T.D3T[0][0]; Bt = &T.H2T[0][0]; m0 = 0; ncols = H; ldb = S + PAD;
      off = Lay::W3; rows_valid = NOUT; ldw = H;
    }
    for (int n0 = 0; n0 < ncols; n0 += 8) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int k0 = 0; k0 < S; k0 += 16) {
        uint32_t a[4], b[2];
        frag_a(a, A, S + PAD, m0, k0, lane);
        frag_b(b, Bt, ldb, k0, n0, lane);
        mma16816(c, a, b);
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = m0 + g + 8 * (q >> 1), col = n0 + 2 * t + (q & 1);
        if (r < rows_valid && col < ldw) out[off + r * ldw + col] = c[q];
      }
    }
  }
  for (int i = tid; i < H; i += 128) { out[Lay::B1 + i] = T.db[i]; out[Lay::B2 + i] = T.db[H + i]; }
  for (int i = tid; i < NOUT; i += 128) out[Lay::B3 + i] = T.db[2 * H + i];
  if (tid == 0) loss_parts[blockIdx.x] = T.loss;
}

// Sum the per-CTA partials in a fixed order, then one Adam update.
__global__ void adam_kernel(float* P, float* M, float* V, const float* partials, int ncta, int np, float lr,
                            float b1, float b2, float eps, int t, float* grad_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  float gsum = 0.f;
  for (int c = 0; c < ncta; c++) gsum += partials[(long long)c * np + p];
  if (grad_out) { grad_out[p] = gsum; return; }
  const float m = b1 * M[p] + (1.f - b1) * gsum;
  const float v = b2 * V[p] + (1.f - b2) * gsum * gsum;
  M[p] = m; V[p] = v;
  const float mh = m / (1.f - powf(b1, (float)t)), vh = v / (1.f - powf(b2, (float)t));
  P[p] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void loss_kernel(const float* parts, int ncta, float inv_batch, float* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int c = 0; c < ncta; c++) s += parts[c];
    *out = s * inv_batch;
  }
}

__global__ void advance_kernel(long long* start, long long by, long long n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *start = (*start + by) % n;
}

// Inference on raw feature rows (tests and evaluation).
template <int H>
__global__ void __launch_bounds__(128) forward_rows_kernel(const float* P, const float* stats, const float* Xr,
                                                           long long n, float* Yout) {
  extern __shared__ __align__(16) unsigned char raw[];
  WeightsSmem<H>& W = *reinterpret_cast<WeightsSmem<H>*>(raw);
  __nv_bfloat16(*X)[K1 + PAD] = reinterpret_cast<__nv_bfloat16(*)[K1 + PAD]>(raw + sizeof(WeightsSmem<H>));
  float(*Y)[NOUT] = reinterpret_cast<float(*)[NOUT]>(raw + sizeof(WeightsSmem<H>) + 128 * (K1 + PAD) * 2);
  load_weights<H>(W, P, stats);
  __syncthreads();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  for (long long base = (long long)blockIdx.x * 128; base < n; base += (long long)gridDim.x * 128) {
    const long long s = base + tid;
    for (int k = 0; k < K1; k++)
      X[tid][k] = __float2bfloat16((s < n && k < NIN) ? (Xr[s * NIN + k] - W.xmean[k]) * W.xistd[k] : 0.f);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      float h1[H / 8][4], h2[H / 8][4], y[4];
      forward_tile<H>(W, &X[0][0], K1 + PAD, warp * 32 + mt * 16, lane, h1, h2, y);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int row = warp * 32 + mt * 16 + g + 8 * (q >> 1), col = 2 * t + (q & 1);
        if (col < NOUT) Y[row][col] = y[q];
      }
    }
    __syncwarp();
    if (s < n)
      for (int o = 0; o < NOUT; o++) Yout[s * NOUT + o] = Y[tid][o] * W.ystd[o] + W.ymean[o];
    __syncwarp();
  }
}

// Fused feature gather + network + starting gauge for every node of a state.
// A node whose 7-node stencil is exactly uniform, or whose predicted change
// is below `gate`, keeps its previous gauge.
template <int H, typename R>
__global__ void __launch_bounds__(128, H == 64 ? 4 : 2) predict_kernel(const float* P, const float* stats, const R* rho, const R* g,
                                                      const R* g_old, long long N, int nx, int ny, int nz, int bc0,
                                                      int bc1,
                                                      int bc2, int lattice, float gate, float* guess) {
  extern __shared__ __align__(16) unsigned char raw[];
  WeightsSmem<H>& W = *reinterpret_cast<WeightsSmem<H>*>(raw);
  __nv_bfloat16(*X)[K1 + PAD] = reinterpret_cast<__nv_bfloat16(*)[K1 + PAD]>(raw + sizeof(WeightsSmem<H>));
  float(*Y)[NOUT] = reinterpret_cast<float(*)[NOUT]>(raw + sizeof(WeightsSmem<H>) + 128 * (K1 + PAD) * 2);
  load_weights<H>(W, P, stats);
  __syncthreads();
  const int bc[3] = {bc0, bc1, bc2};
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, gg = lane >> 2, t = lane & 3;
  const double tlat = lattice == POND_D3Q27 ? 1.0 / 3.0 : 1.0;
  for (long long base = (long long)blockIdx.x * 128; base < N; base += (long long)gridDim.x * 128) {
    const long long n = base + tid;
    // activity: the largest relative last increment (features 35-38)
    float act = 0.f, c = 0.f;
    float cur[4] = {0.f, 0.f, 0.f, 0.f}, old[4] = {0.f, 0.f, 0.f, 0.f};
    if (n < N) {
      for (int k = 0; k < 4; k++) { cur[k] = g[k * N + n]; old[k] = g_old[k * N + n]; }
      c = sqrtf(fmaxf(cur[3], 0.f) * float(1.0 / tlat));
      const float ic = c > 0.f ? 1.f / c : 0.f;
      act = fmaxf(fmaxf(fabsf((cur[0] - old[0]) * ic), fabsf((cur[1] - old[1]) * ic)),
                  fmaxf(fabsf((cur[2] - old[2]) * ic), cur[3] != 0.f ? fabsf((cur[3] - old[3]) / cur[3]) : 0.f));
    }
    const bool active = n < N && act >= gate;
    float d[NOUT] = {0.f, 0.f, 0.f, 0.f};
    // a warp gathers features and runs the network only if one of its nodes is active
    if (__any_sync(0xffffffffu, active)) {
      float feat[NIN];
      bool use = false;
      if (n < N) use = node_features<R>(rho, g, g_old, N, nx, ny, nz, bc, lattice, n, feat);
#pragma unroll
      for (int k = 0; k < K1; k++)
        X[tid][k] = __float2bfloat16((n < N && k < NIN) ? (feat[k] - W.xmean[k]) * W.xistd[k] : 0.f);
      __syncwarp();
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        float h1[H / 8][4], h2[H / 8][4], y[4];
        forward_tile<H>(W, &X[0][0], K1 + PAD, warp * 32 + mt * 16, lane, h1, h2, y);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int row = warp * 32 + mt * 16 + gg + 8 * (q >> 1), col = 2 * t + (q & 1);
          if (col < NOUT) Y[row][col] = y[q];
        }
      }
      __syncwarp();
      if (active && use)
        for (int o = 0; o < NOUT; o++) d[o] = Y[tid][o] * W.ystd[o] + W.ymean[o];
    }
    if (n < N) {
      // the previous gauge, plus the predicted increment on active nodes
      float out[4];
      out[0] = cur[0] + c * d[0];
      out[1] = lattice == POND_D1Q5 ? cur[1] : cur[1] + c * d[1];
      out[2] = lattice == POND_D1Q5 ? cur[2] : cur[2] + c * d[2];
      const float Tn = cur[3] + cur[3] * d[3];
      out[3] = (Tn > 0.f && isfinite(Tn)) ? Tn : cur[3];
      for (int k = 0; k < 4; k++) guess[k * N + n] = out[k];
    }
    __syncwarp();
  }
}

// Starting gauge by linear extrapolation in time from the two stored levels:
// g* = g^n + (g^n - g^{n-1}); T keeps g^n where the extrapolation is not positive.
template <typename R>
__global__ void extrapolate_kernel(const R* g_cur, const R* g_old, long long N, float* guess) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float a = g_cur[k * N + n], b = g_old[k * N + n];
      float v = a + (a - b);
      if (k == 3 && !(v > 0.f && isfinite(v))) v = a;
      guess[k * N + n] = v;
    }
  }
}

// Training pairs from the last step: features of the pre-step state (buffer
// `prev`) and the increment to the converged gauge (buffer `cur`).  Nodes
// are sampled with a stride from a random offset; exactly uniform stencils
// (increment zero by construction) are skipped.
template <typename R>
__global__ void pairs_kernel(const R* rho_p, const R* g_p, const R* g_h, const R* g_c, long long N, int nx, int ny,
                             int nz,
                             int bc0, int bc1, int bc2, int lattice, long long offset, long long stride,
                             long long capacity, float* X, float* Y, long long* node_out,
                             unsigned long long* count) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = offset + k * stride;
  if (n >= N) return;
  const int bc[3] = {bc0, bc1, bc2};
  float feat[NIN];
  if (!node_features<R>(rho_p, g_p, g_h, N, nx, ny, nz, bc, lattice, n, feat)) return;
  const unsigned long long slot = atomicAdd(count, 1ull);
  if ((long long)slot >= capacity) return;
  for (int i = 0; i < NIN; i++) X[slot * NIN + i] = feat[i];
  if (node_out) node_out[slot] = n;
  const double tlat = lattice == POND_D3Q27 ? 1.0 / 3.0 : 1.0;
  const double T = g_p[3 * N + n];
  const double c = sqrt(fmax(T, 0.0) / tlat);
  const double ic = c > 0 ? 1.0 / c : 0.0;
  for (int k = 0; k < 4; k++) {
    const double r = double(g_c[k * N + n]) - double(g_p[k * N + n]);  // the step's increment
    Y[slot * NOUT + k] = float(k < 3 ? r * ic : (T != 0 ? r / T : 0.0));
  }
}

// Feature/target statistics (float64 sums) for the standardisation.
__global__ void stats_kernel(const float* X, const float* Y, long long n, double* acc) {
  __shared__ double s[2 * (NIN + NOUT)];
  for (int i = threadIdx.x; i < 2 * (NIN + NOUT); i += blockDim.x) s[i] = 0;
  __syncthreads();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    for (int k = 0; k < NIN; k++) {
      const double v = X[r * NIN + k];
      atomicAdd(&s[k], v);
      atomicAdd(&s[NIN + NOUT + k], v * v);
    }
    for (int o = 0; o < NOUT; o++) {
      const double v = Y[r * NOUT + o];
      atomicAdd(&s[NIN + o], v);
      atomicAdd(&s[2 * NIN + NOUT + o], v * v);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 2 * (NIN + NOUT); i += blockDim.x) atomicAdd(&acc[i], s[i]);
}

}  // namespace mlp

// ------------------------------------------------------------------ host side
static size_t train_smem(int H) { return H == 64 ? sizeof(mlp::TrainSmem<64>) : sizeof(mlp::TrainSmem<128>); }
static size_t infer_smem(int H) {
  return (H == 64 ? sizeof(mlp::WeightsSmem<64>) : sizeof(mlp::WeightsSmem<128>)) +
         128 * (mlp::K1 + mlp::PAD) * 2 + 128 * mlp::NOUT * sizeof(float);
}

static int mlp_nparams(int H) { return H == 64 ? mlp::Layout<64>::SIZE : mlp::Layout<128>::SIZE; }

static int ensure_partials(pond_mlp* m, int ncta) {
  if (ncta <= m->max_cta) return POND_OK;
  cudaFree(m->partials);
  cudaFree(m->loss_parts);
  m->partials = nullptr;
  m->loss_parts = nullptr;
  m->max_cta = 0;
  if (cudaMalloc(&m->partials, (size_t)ncta * m->nparams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->loss_parts, (size_t)ncta * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(POND_ERR_NOMEM, "gradient partials");
  }
  m->max_cta = ncta;
  return POND_OK;
}

static int launch_train(pond_mlp* m, const float* X, const float* Y, long long n, int ncta, const long long* d_start,
                        long long start, float inv_batch) {
  cudaError_t e;
  if (m->H == 64) {
    e = cudaFuncSetAttribute(mlp::train_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem(64));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    mlp::train_kernel<64><<<ncta, 128, train_smem(64), m->stream>>>(m->P, m->stats, X, Y, n, d_start, start,
                                                                     inv_batch, m->partials, m->loss_parts);
  } else {
    e = cudaFuncSetAttribute(mlp::train_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)train_smem(128));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    mlp::train_kernel<128><<<ncta, 128, train_smem(128), m->stream>>>(m->P, m->stats, X, Y, n, d_start, start,
                                                                       inv_batch, m->partials, m->loss_parts);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "train kernel launch");
}

int run_predictor(pond_ctx* c) {
  pond_mlp* m = (pond_mlp*)c->predictor;
  if (!m && !c->extrapolate) return set_error(POND_ERR_STATE, "learned step without a predictor (pond_set_predictor)");
  if (!c->guess) {
    if (cudaMalloc(&c->guess, 4 * sizeof(float) * c->N) != cudaSuccess) {
      cudaGetLastError();
      c->guess = nullptr;
      return set_error(POND_ERR_NOMEM, "predicted gauge buffer");
    }
  }
  if (!m) {
    const int cu = c->cur, od = 1 - c->cur;
    if (c->elem == 8)
      mlp::extrapolate_kernel<double><<<1184, 256, 0, c->stream>>>((const double*)c->g[cu], (const double*)c->g[od],
                                                                   c->N, c->guess);
    else
      mlp::extrapolate_kernel<float><<<1184, 256, 0, c->stream>>>((const float*)c->g[cu], (const float*)c->g[od],
                                                                  c->N, c->guess);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? POND_OK : cuda_fail(e, "extrapolation launch");
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->p.device);
  const long long tiles = (c->N + 127) / 128;
  const size_t smem = infer_smem(m->H);
  const int cu = c->cur;
  const float gate = c->gate;
  cudaError_t e;
  int grid = 0;
  // one wave: every CTA resident at once (the grid-stride loop gives each the same share)
#define POND_PREDICT(HH, RR)                                                                                       \
  e = cudaFuncSetAttribute(mlp::predict_kernel<HH, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");                                               \
  {                                                                                                                \
    int per_sm = 1;                                                                                                \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mlp::predict_kernel<HH, RR>, 128, smem);            \
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");                    \
    grid = (int)std::min<long long>(tiles, (long long)nsm * std::max(per_sm, 1));                                  \
  }                                                                                                                \
  mlp::predict_kernel<HH, RR><<<grid, 128, smem, c->stream>>>(m->P, m->stats, (const RR*)c->rho[cu],               \
                                                              (const RR*)c->g[cu], (const RR*)c->g[1 - cu], c->N,   \
                                                              (int)c->p.Nx,                                        \
                                                              (int)c->p.Ny, (int)c->p.Nz, c->p.bc[0], c->p.bc[1], \
                                                              c->p.bc[2], c->p.lattice, gate, c->guess)
  if (m->H == 64) {
    if (c->elem == 8) { POND_PREDICT(64, double); } else { POND_PREDICT(64, float); }
  } else {
    if (c->elem == 8) { POND_PREDICT(128, double); } else { POND_PREDICT(128, float); }
  }
#undef POND_PREDICT
  e = cudaGetLastError();
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "predictor launch");
}

}  // namespace pond

using namespace pond;

extern "C" {

int pond_mlp_create(int hidden, uint64_t seed, int device, pond_mlp** out) {
  if (!out) return set_error(POND_ERR_ARG, "null output");
  *out = nullptr;
  if (hidden != 64 && hidden != 128) return set_error(POND_ERR_UNSUPPORTED, "hidden width must be 64 or 128");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  pond_mlp* m = new pond_mlp();
  m->H = hidden;
  m->device = device;
  m->nparams = mlp_nparams(hidden);
  const size_t pb = (size_t)m->nparams * sizeof(float);
  if (cudaMalloc(&m->P, pb) != cudaSuccess || cudaMalloc(&m->M, pb) != cudaSuccess ||
      cudaMalloc(&m->V, pb) != cudaSuccess || cudaMalloc(&m->stats, mlp::STATS * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->d_loss, sizeof(float)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    pond_mlp_destroy(m);
    return set_error(POND_ERR_NOMEM, "network buffers");
  }
  // Xavier-uniform initialisation on the host (seeded), biases zero
  std::vector<float> P(m->nparams, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_out, int fan_in) {
    const float a = std::sqrt(6.f / float(fan_in + fan_out));
    std::uniform_real_distribution<float> U(-a, a);
    for (int i = 0; i < fan_out * fan_in; i++) P[off + i] = U(rng);
  };
  const int H = hidden;
  const int W1 = 0, B1 = W1 + H * mlp::NIN, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H;
  (void)B2;
  fill(W1, H, mlp::NIN);
  fill(W2, H, H);
  fill(W3, mlp::NOUT, H);
  std::vector<float> st(mlp::STATS, 0.f);
  for (int i = 0; i < mlp::NIN; i++) st[mlp::NIN + i] = 1.f;
  for (int o = 0; o < mlp::NOUT; o++) st[2 * mlp::NIN + mlp::NOUT + o] = 1.f;
  e = cudaMemcpy(m->P, P.data(), P.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m->stats, st.data(), st.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->M, 0, (size_t)m->nparams * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->V, 0, (size_t)m->nparams * sizeof(float));
  if (e != cudaSuccess) {
    pond_mlp_destroy(m);
    return cuda_fail(e, "network init");
  }
  *out = m;
  return POND_OK;
}

int pond_mlp_destroy(pond_mlp* m) {
  if (!m) return POND_OK;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->P); cudaFree(m->M); cudaFree(m->V); cudaFree(m->stats);
  cudaFree(m->partials); cudaFree(m->loss_parts); cudaFree(m->d_loss);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return POND_OK;
}

int pond_mlp_num_params(const pond_mlp* m) { return m ? m->nparams : 0; }

int pond_mlp_get_params(pond_mlp* m, float* params, float* stats) {
  if (!m) return set_error(POND_ERR_ARG, "null network");
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  cudaError_t e = cudaSuccess;
  if (params) e = cudaMemcpy(params, m->P, (size_t)m->nparams * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && stats) e = cudaMemcpy(stats, m->stats, mlp::STATS * sizeof(float), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_mlp_get_params");
}

int pond_mlp_set_params(pond_mlp* m, const float* params, const float* stats) {
  if (!m) return set_error(POND_ERR_ARG, "null network");
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  cudaError_t e = cudaSuccess;
  if (params) e = cudaMemcpy(m->P, params, (size_t)m->nparams * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && stats) e = cudaMemcpy(m->stats, stats, mlp::STATS * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->M, 0, (size_t)m->nparams * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->V, 0, (size_t)m->nparams * sizeof(float));
  m->adam_t = 0;
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_mlp_set_params");
}

int pond_mlp_fit_stats(pond_mlp* m, const float* X, const float* Y, int64_t n) {
  if (!m || !X || !Y || n <= 1) return set_error(POND_ERR_ARG, "pond_mlp_fit_stats: bad argument");
  cudaSetDevice(m->device);
  double* acc = nullptr;
  cudaError_t e = cudaMalloc(&acc, 2 * (mlp::NIN + mlp::NOUT) * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(e, "stats buffer");
  cudaMemsetAsync(acc, 0, 2 * (mlp::NIN + mlp::NOUT) * sizeof(double), m->stream);
  mlp::stats_kernel<<<256, 256, 0, m->stream>>>(X, Y, n, acc);
  std::vector<double> h(2 * (mlp::NIN + mlp::NOUT));
  e = cudaMemcpyAsync(h.data(), acc, h.size() * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  cudaFree(acc);
  if (e != cudaSuccess) return cuda_fail(e, "stats");
  const int C = mlp::NIN + mlp::NOUT;
  std::vector<float> st(mlp::STATS);
  for (int k = 0; k < C; k++) {
    const double mean = h[k] / n;
    const double var = std::max(h[C + k] / n - mean * mean, 0.0);
    const double sd = std::max(std::sqrt(var), 1e-12);
    if (k < mlp::NIN) { st[k] = (float)mean; st[mlp::NIN + k] = (float)sd; }
    else { st[2 * mlp::NIN + (k - mlp::NIN)] = (float)mean; st[2 * mlp::NIN + mlp::NOUT + (k - mlp::NIN)] = (float)sd; }
  }
  e = cudaMemcpy(m->stats, st.data(), st.size() * sizeof(float), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "stats upload");
}

int pond_mlp_train(pond_mlp* m, const float* X, const float* Y, int64_t n, int batch, int steps, float lr,
                   float* loss_out) {
  if (!m || !X || !Y || n <= 0 || batch <= 0 || steps < 0 || !(lr > 0))
    return set_error(POND_ERR_ARG, "pond_mlp_train: bad argument");
  cudaSetDevice(m->device);
  const int S = m->H == 64 ? 128 : 64;
  const int ncta = (batch + S - 1) / S;
  int st = ensure_partials(m, ncta);
  if (st != POND_OK) return st;
  const float inv_batch = 1.f / float(ncta * S);
  const int thr = 256, blk = (m->nparams + thr - 1) / thr;
  long long start = 0;
  for (int s = 0; s < steps; s++) {
    st = launch_train(m, X, Y, n, ncta, nullptr, start, inv_batch);
    if (st != POND_OK) return st;
    m->adam_t++;
    mlp::adam_kernel<<<blk, thr, 0, m->stream>>>(m->P, m->M, m->V, m->partials, ncta, m->nparams, lr, 0.9f, 0.999f,
                                                  1e-8f, m->adam_t, nullptr);
    if (loss_out) {
      mlp::loss_kernel<<<1, 32, 0, m->stream>>>(m->loss_parts, ncta, inv_batch, m->d_loss);
      cudaMemcpyAsync(loss_out + s, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    }
    start = (start + (long long)ncta * S) % n;
  }
  cudaError_t e = cudaStreamSynchronize(m->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_mlp_train");
}

int pond_mlp_gradients(pond_mlp* m, const float* X, const float* Y, int64_t n, float* grad, float* loss) {
  if (!m || !X || !Y || n <= 0 || !grad) return set_error(POND_ERR_ARG, "pond_mlp_gradients: bad argument");
  cudaSetDevice(m->device);
  const int S = m->H == 64 ? 128 : 64;
  if (n % S) return set_error(POND_ERR_ARG, "pond_mlp_gradients: n must be a multiple of %d", S);
  const int ncta = (int)(n / S);
  int st = ensure_partials(m, ncta);
  if (st != POND_OK) return st;
  const float inv_batch = 1.f / float(n);
  st = launch_train(m, X, Y, n, ncta, nullptr, 0, inv_batch);
  if (st != POND_OK) return st;
  float* d_grad = nullptr;
  cudaError_t e = cudaMalloc(&d_grad, (size_t)m->nparams * sizeof(float));
  if (e != cudaSuccess) return cuda_fail(e, "gradient buffer");
  const int thr = 256, blk = (m->nparams + thr - 1) / thr;
  mlp::adam_kernel<<<blk, thr, 0, m->stream>>>(m->P, m->M, m->V, m->partials, ncta, m->nparams, 0.f, 0.f, 0.f, 0.f,
                                                1, d_grad);
  mlp::loss_kernel<<<1, 32, 0, m->stream>>>(m->loss_parts, ncta, inv_batch, m->d_loss);
  e = cudaMemcpyAsync(grad, d_grad, (size_t)m->nparams * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  cudaFree(d_grad);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_mlp_gradients");
}

int pond_mlp_forward(pond_mlp* m, const float* X, float* Y, int64_t n) {
  if (!m || !X || !Y || n <= 0) return set_error(POND_ERR_ARG, "pond_mlp_forward: bad argument");
  cudaSetDevice(m->device);
  const size_t smem = infer_smem(m->H);
  const int grid = (int)std::min<long long>((n + 127) / 128, 1024);
  cudaError_t e;
  if (m->H == 64) {
    e = cudaFuncSetAttribute(mlp::forward_rows_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) mlp::forward_rows_kernel<64><<<grid, 128, smem, m->stream>>>(m->P, m->stats, X, n, Y);
  } else {
    e = cudaFuncSetAttribute(mlp::forward_rows_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) mlp::forward_rows_kernel<128><<<grid, 128, smem, m->stream>>>(m->P, m->stats, X, n, Y);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_mlp_forward");
}

int pond_collect_pairs(pond_ctx* c, float* X, float* Y, int64_t* node, int64_t capacity, int64_t stride,
                       uint64_t seed, int64_t* written) {
  if (!c || !X || !Y || capacity <= 0 || stride <= 0 || !written)
    return set_error(POND_ERR_ARG, "pond_collect_pairs: bad argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (c->istep < 1) return set_error(POND_ERR_STATE, "pond_collect_pairs needs a completed step");
  if (!c->g_hist || !c->keep_history)
    return set_error(POND_ERR_STATE, "pond_collect_pairs needs pond_keep_history(ctx, 1) before the step");
  cudaSetDevice(c->p.device);
  unsigned long long* d_count = nullptr;
  cudaError_t e = cudaMalloc(&d_count, sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "counter");
  cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), c->stream);
  const long long offset = (long long)(seed % (uint64_t)stride);
  const long long m = (c->N - offset + stride - 1) / stride;
  const int th = 256;
  const unsigned blocks = (unsigned)((m + th - 1) / th);
  const int prev = 1 - c->cur, cur = c->cur;
  if (c->elem == 8)
    mlp::pairs_kernel<double><<<blocks, th, 0, c->stream>>>(
        (const double*)c->rho[prev], (const double*)c->g[prev], (const double*)c->g_hist, (const double*)c->g[cur],
        c->N, (int)c->p.Nx,
        (int)c->p.Ny, (int)c->p.Nz, c->p.bc[0], c->p.bc[1], c->p.bc[2], c->p.lattice, offset, stride, capacity, X, Y,
        (long long*)node, d_count);
  else
    mlp::pairs_kernel<float><<<blocks, th, 0, c->stream>>>(
        (const float*)c->rho[prev], (const float*)c->g[prev], (const float*)c->g_hist, (const float*)c->g[cur],
        c->N, (int)c->p.Nx,
        (int)c->p.Ny, (int)c->p.Nz, c->p.bc[0], c->p.bc[1], c->p.bc[2], c->p.lattice, offset, stride, capacity, X, Y,
        (long long*)node, d_count);
  unsigned long long cnt = 0;
  e = cudaMemcpyAsync(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_count);
  if (e != cudaSuccess) return cuda_fail(e, "pond_collect_pairs");
  *written = (int64_t)std::min<unsigned long long>(cnt, (unsigned long long)capacity);
  return POND_OK;
}

int pond_set_predictor(pond_ctx* c, pond_mlp* m, float gate) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  if (m && m->device != c->p.device) return set_error(POND_ERR_ARG, "network and context on different devices");
  c->predictor = m;
  c->gate = gate;
  c->guess_ready = m != nullptr || c->extrapolate;
  c->p.learned = c->guess_ready ? 1 : 0;
  return POND_OK;
}

int pond_set_extrapolation(pond_ctx* c, int on) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  c->extrapolate = on != 0;
  c->guess_ready = c->predictor != nullptr || c->extrapolate;
  c->p.learned = c->guess_ready ? 1 : 0;
  return POND_OK;
}

int pond_predict(pond_ctx* c, float* guess_out) {
  if (!c || !guess_out) return set_error(POND_ERR_ARG, "null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  cudaSetDevice(c->p.device);
  int st = run_predictor(c);
  if (st != POND_OK) return st;
  cudaError_t e = cudaMemcpyAsync(guess_out, c->guess, 4 * sizeof(float) * c->N, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_predict");
}

}  // extern "C"
