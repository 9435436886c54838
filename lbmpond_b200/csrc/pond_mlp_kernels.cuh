// Learned gauge predictor: BF16 tensor-core MLP kernels (mma.sync m16n8k16,
// float32 accumulation).
//
// Network: NIN (39) -> H -> H -> NOUT (4), tanh hidden activations.
// Features of a node at time level n (the same function for training pairs
// and inference), c = sqrt(T/TLat):
//   centre  : c, u_x/c, u_y/c, u_z/c, T/TLat
//   neighbour (-x,+x,-y,+y,-z,+z): rho_m/rho - 1, (u_m - u)/c (3), T_m/T - 1
//   last increment of the centre: (u^n - u^{n-1})/c (3), (T^n - T^{n-1})/T
// Target: the step's increment (u* - u^n)/c (3), (T* - T^n)/T, with u*, T*
// the converged gauge of the step.  Inputs and targets are standardised with
// statistics kept in the network.
#pragma once
#include <cuda_bf16.h>

#include "pond_common.cuh"

namespace pond {
namespace mlp {

constexpr int NIN = 39;     // 7 nodes x (rho, u_x, u_y, u_z, T) + the centre's last increment (4)
constexpr int NOUT = 4;     // du_x, du_y, du_z, dT
constexpr int K1 = 48;      // NIN padded to a multiple of 16
constexpr int OUTP = 16;    // NOUT padded to one m16 tile (8 used as n-tile)
constexpr int PAD = 8;      // bf16 row padding against shared-memory bank conflicts

// ------------------------------------------------------------------ features
// Reads the gauge/density planes of level n (rho, g) and the gauge of level
// n-1 (g_old) and writes the raw features of node n.  Returns false when the
// node's 7-node stencil is exactly uniform in space: there the plain start
// (the previous gauge) already converges in one iteration, while a uniform
// far field still carries float32 noise of ~1e-8 from step to step, so a
// test on the time increment would not separate it.
template <typename R>
__device__ __forceinline__ bool node_features(const R* rho, const R* g, const R* g_old, long long N, int nx, int ny,
                                              int nz, const int bc[3], int lattice, long long n, float feat[NIN]) {
  const int x = n % nx, y = (n / nx) % ny, z = n / ((long long)nx * ny);
  const double tlat = lattice == POND_D3Q27 ? 1.0 / 3.0 : 1.0;
  const float rc = rho[n];
  const float ux = g[n], uy = g[N + n], uz = g[2 * N + n], T = g[3 * N + n];
  const float c = sqrtf(fmaxf(T, 0.f) * float(1.0 / tlat));
  const float ic = c > 0.f ? 1.f / c : 0.f;
  feat[0] = c; feat[1] = ux * ic; feat[2] = uy * ic; feat[3] = uz * ic; feat[4] = float(T / tlat);
  bool uniform = true;
  const int dims[3] = {nx, ny, nz};
  const int pos[3] = {x, y, z};
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const int ax = k >> 1, dir = (k & 1) ? 1 : -1;
    int p[3] = {pos[0], pos[1], pos[2]};
    bool rv = false;
    p[ax] = dims[ax] > 1 ? resolve_axis(pos[ax] + dir, dims[ax], bc[ax], rv) : pos[ax];
    const long long m = p[0] + (long long)nx * (p[1] + (long long)ny * p[2]);
    float un[3] = {float(g[m]), float(g[N + m]), float(g[2 * N + m])};
    if (rv) un[ax] = -un[ax];
    const float rn = rho[m], Tn = g[3 * N + m];
    const float d0 = rc != 0.f ? rn / rc - 1.f : 0.f;
    const float d1 = (un[0] - ux) * ic, d2 = (un[1] - uy) * ic, d3 = (un[2] - uz) * ic;
    const float d4 = T != 0.f ? Tn / T - 1.f : 0.f;
    feat[5 + 5 * k + 0] = d0; feat[5 + 5 * k + 1] = d1; feat[5 + 5 * k + 2] = d2;
    feat[5 + 5 * k + 3] = d3; feat[5 + 5 * k + 4] = d4;
    uniform = uniform && rn == rc && un[0] == ux && un[1] == uy && un[2] == uz && Tn == T;
  }
  const float ox = g_old[n], oy = g_old[N + n], oz = g_old[2 * N + n], oT = g_old[3 * N + n];
  feat[35] = (ux - ox) * ic; feat[36] = (uy - oy) * ic; feat[37] = (uz - oz) * ic;
  feat[38] = T != 0.f ? (T - oT) / T : 0.f;
  return !uniform;
}

// ------------------------------------------------------------------ mma helpers
__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }
// A fragment of rows [r0, r0+16) x cols [k0, k0+16) of a row-major bf16 matrix
__device__ __forceinline__ void frag_a(uint32_t a[4], const __nv_bfloat16* M, int ld, int r0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  a[0] = ld32(M + (r0 + g) * ld + k0 + 2 * t);
  a[1] = ld32(M + (r0 + g + 8) * ld + k0 + 2 * t);
  a[2] = ld32(M + (r0 + g) * ld + k0 + 8 + 2 * t);
  a[3] = ld32(M + (r0 + g + 8) * ld + k0 + 8 + 2 * t);
}
// B fragment (k0..k0+16) x (n0..n0+8) of B[k][n] = Mt[n][k], Mt row-major
__device__ __forceinline__ void frag_b(uint32_t b[2], const __nv_bfloat16* Mt, int ld, int k0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  b[0] = ld32(Mt + (n0 + g) * ld + k0 + 2 * t);
  b[1] = ld32(Mt + (n0 + g) * ld + k0 + 8 + 2 * t);
}
// accumulator fragments of n-tiles 2kk and 2kk+1 -> A fragment of k-step kk
__device__ __forceinline__ void acc_to_a(uint32_t a[4], const float c0[4], const float c1[4]) {
  a[0] = pack_bf16(c0[0], c0[1]);
  a[1] = pack_bf16(c0[2], c0[3]);
  a[2] = pack_bf16(c1[0], c1[1]);
  a[3] = pack_bf16(c1[2], c1[3]);
}

// Shared-memory weights of one network (bf16, padded rows):
//   W1 [H][K1+PAD], W2 [H][H+PAD], W3 [OUTP][H+PAD] (rows >= NOUT zero),
//   W2T [H][H+PAD] (W2 transposed), W3T [H][OUTP+PAD] (W3 transposed)
template <int H> struct WeightsSmem {
  __nv_bfloat16 W1[H][K1 + PAD];
  __nv_bfloat16 W2[H][H + PAD];
  __nv_bfloat16 W3[OUTP][H + PAD];
  __nv_bfloat16 W2T[H][H + PAD];
  __nv_bfloat16 W3T[H][OUTP + PAD];
  float b1[H], b2[H], b3[OUTP];
  float xmean[K1], xistd[K1];
  float ymean[OUTP], ystd[OUTP];
};

// Parameter vector layout (float32 master copy):
//   W1[H][NIN], b1[H], W2[H][H], b2[H], W3[NOUT][H], b3[NOUT]
template <int H> struct Layout {
  static constexpr int W1 = 0;
  static constexpr int B1 = W1 + H * NIN;
  static constexpr int W2 = B1 + H;
  static constexpr int B2 = W2 + H * H;
  static constexpr int W3 = B2 + H;
  static constexpr int B3 = W3 + NOUT * H;
  static constexpr int SIZE = B3 + NOUT;
};

// stats layout: xmean[NIN], xstd[NIN], ymean[NOUT], ystd[NOUT]
constexpr int STATS = 2 * NIN + 2 * NOUT;

template <int H>
__device__ void load_weights(WeightsSmem<H>& S, const float* P, const float* stats) {
  using Lay = Layout<H>;
  for (int i = threadIdx.x; i < H * (K1 + PAD); i += blockDim.x) {
    const int r = i / (K1 + PAD), k = i % (K1 + PAD);
    S.W1[r][k] = __float2bfloat16(k < NIN ? P[Lay::W1 + r * NIN + k] : 0.f);
  }
  for (int i = threadIdx.x; i < H * (H + PAD); i += blockDim.x) {
    const int r = i / (H + PAD), k = i % (H + PAD);
    S.W2[r][k] = __float2bfloat16(k < H ? P[Lay::W2 + r * H + k] : 0.f);
    S.W2T[r][k] = __float2bfloat16(k < H ? P[Lay::W2 + k * H + r] : 0.f);
  }
  for (int i = threadIdx.x; i < OUTP * (H + PAD); i += blockDim.x) {
    const int r = i / (H + PAD), k = i % (H + PAD);
    S.W3[r][k] = __float2bfloat16((r < NOUT && k < H) ? P[Lay::W3 + r * H + k] : 0.f);
  }
  for (int i = threadIdx.x; i < H * (OUTP + PAD); i += blockDim.x) {
    const int r = i / (OUTP + PAD), k = i % (OUTP + PAD);
    S.W3T[r][k] = __float2bfloat16(k < NOUT ? P[Lay::W3 + k * H + r] : 0.f);
  }
  for (int i = threadIdx.x; i < H; i += blockDim.x) { S.b1[i] = P[Lay::B1 + i]; S.b2[i] = P[Lay::B2 + i]; }
  for (int i = threadIdx.x; i < OUTP; i += blockDim.x) S.b3[i] = i < NOUT ? P[Lay::B3 + i] : 0.f;
  for (int i = threadIdx.x; i < K1; i += blockDim.x) {
    S.xmean[i] = i < NIN ? stats[i] : 0.f;
    S.xistd[i] = i < NIN ? 1.f / stats[NIN + i] : 0.f;
  }
  for (int i = threadIdx.x; i < OUTP; i += blockDim.x) {
    S.ymean[i] = i < NOUT ? stats[2 * NIN + i] : 0.f;
    S.ystd[i] = i < NOUT ? stats[2 * NIN + NOUT + i] : 1.f;
  }
}

// Forward pass of one m16 tile of standardised inputs X (bf16 rows in shared
// memory): returns the hidden activations (float, accumulator layout) and
// the standardised outputs (n-tile 0 of layer 3).
template <int H>
__device__ __forceinline__ void forward_tile(const WeightsSmem<H>& S, const __nv_bfloat16* X, int ldx, int r0,
                                             int lane, float h1[H / 8][4], float h2[H / 8][4], float y[4]) {
  const int t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < H / 8; nt++) {
    const float b0 = S.b1[nt * 8 + 2 * t], bb = S.b1[nt * 8 + 2 * t + 1];
    h1[nt][0] = b0; h1[nt][1] = bb; h1[nt][2] = b0; h1[nt][3] = bb;
  }
#pragma unroll
  for (int kk = 0; kk < K1 / 16; kk++) {
    uint32_t a[4];
    frag_a(a, X, ldx, r0, kk * 16, lane);
#pragma unroll
    for (int nt = 0; nt < H / 8; nt++) {
      uint32_t b[2];
      frag_b(b, &S.W1[0][0], K1 + PAD, kk * 16, nt * 8, lane);
      mma16816(h1[nt], a, b);
    }
  }
#pragma unroll
  for (int nt = 0; nt < H / 8; nt++)
#pragma unroll
    for (int q = 0; q < 4; q++) h1[nt][q] = tanhf(h1[nt][q]);
#pragma unroll
  for (int nt = 0; nt < H / 8; nt++) {
    const float b0 = S.b2[nt * 8 + 2 * t], bb = S.b2[nt * 8 + 2 * t + 1];
    h2[nt][0] = b0; h2[nt][1] = bb; h2[nt][2] = b0; h2[nt][3] = bb;
  }
#pragma unroll
  for (int kk = 0; kk < H / 16; kk++) {
    uint32_t a[4];
    acc_to_a(a, h1[2 * kk], h1[2 * kk + 1]);
#pragma unroll
    for (int nt = 0; nt < H / 8; nt++) {
      uint32_t b[2];
      frag_b(b, &S.W2[0][0], H + PAD, kk * 16, nt * 8, lane);
      mma16816(h2[nt], a, b);
    }
  }
#pragma unroll
  for (int nt = 0; nt < H / 8; nt++)
#pragma unroll
    for (int q = 0; q < 4; q++) h2[nt][q] = tanhf(h2[nt][q]);
  {
    const float b0 = S.b3[2 * t], bb = S.b3[2 * t + 1];
    y[0] = b0; y[1] = bb; y[2] = b0; y[3] = bb;
  }
#pragma unroll
  for (int kk = 0; kk < H / 16; kk++) {
    uint32_t a[4];
    acc_to_a(a, h2[2 * kk], h2[2 * kk + 1]);
    uint32_t b[2];
    frag_b(b, &S.W3[0][0], H + PAD, kk * 16, 0, lane);
    mma16816(y, a, b);
  }
}

}  // namespace mlp
}  // namespace pond
