// D3Q27 PonD pull step, float32, one thread per node with the stencil tile
// staged in shared memory (the hot kernel of the 256^3 benchmark).
//
// Same arithmetic as pull_point_kernel (steps.cu:356-588 LBMpull with
// propagate<N>, N = 2, 3, 4), organised for the SM:
//
//  * a CTA owns a 32 x 4 x 2 tile of nodes and stages the tile plus a halo of
//    2 nodes per side (36 x 8 x 6 nodes) once per step, node-major: a staged
//    node's 27 populations are contiguous and 16-byte aligned (a 28-float
//    stride, 189 KB), so a lane fetches a stencil node with seven 16-byte
//    loads, and the 28-word stride puts the eight lanes of every 16-byte load
//    phase on distinct banks.  Each staging thread copies whole nodes and
//    transfers them itself (no gauge planes in shared memory).  Boundary
//    resolution (periodic wrap, clamp, mirror with population reversal), the
//    reference's dropping of non-finite terms and the square root of T are
//    applied while staging;
//  * after staging, each staged node's 27 populations are replaced by their
//    transfer into a reference gauge shared by the CTA (the gauge of the
//    tile's centre node).  The transfer of a source node into a target gauge
//    (U, C), sum_b prod_ax L_i(y_b) f_b with y = (v_b - U)/C and L_i the
//    quadratic Lagrange basis over the target classes, is a quadratic in the
//    particle velocity v_b along each axis, so it equals the transfer from
//    the reference gauge to (U, C), G[i][k] = L_i((u_ref + c_ref xi_k - U)/C),
//    applied to the reference-gauge populations.  G depends on the target
//    alone: the interpolation weights and G are contracted against the
//    reference-gauge populations one axis at a time (z per stencil node, y
//    per stencil column, x per stencil row: 81 FMA each) instead of
//    transforming every stencil node into the target gauge (243 FMA);
//  * the fixed-point iteration is warp-synchronous: a warp iterates while any
//    of its lanes is unconverged and walks the union of its lanes' stencil
//    offsets, contracting every target class at every offset (a class a lane
//    does not weight there has weight 0): straight-line code the scheduler
//    interleaves;
//  * a lane whose departure points leave the +-2 halo (|u| + sqrt(T/TLat) >= 1
//    along an axis) runs that iteration from global memory instead.
#pragma once
#include "pond_step_point.cuh"

namespace pond {
namespace d27 {

constexpr int TX = 32, TY = 4, TZ = 2, H = 2;
constexpr int SX = TX + 2 * H, SY = TY + 2 * H, SZ = TZ + 2 * H;
constexpr int SN = SX * SY * SZ;  // 1728 staged nodes
constexpr int NS = 28;            // floats per staged node: its 27 R-gauge populations and a pad
constexpr int THREADS = TX * TY * TZ;
// staged nodes node-major (a node's populations contiguous, 16-byte aligned:
// seven 16-byte loads per stencil node; the 28-word stride keeps the eight
// lanes of each 16-byte load phase on distinct banks), then the iterate's
// populations of every lane
constexpr size_t SMEM_BYTES = size_t(NS) * SN * sizeof(float) + size_t(27) * THREADS * sizeof(float);

// reference population index of tensor class t = 9 cx + 3 cy + cz, for
// lookups with run-time indices (consts.h:20-30 order)
__constant__ int c_ref27[27] = {0, 3, 16, 2, 6, 18, 12, 13, 24, 1, 5, 17, 4, 7, 19, 14, 15, 25,
                                8, 10, 22, 9, 11, 23, 20, 21, 26};

// 4-byte asynchronous global -> shared copy and the wait for all of them
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// class index -> its mirror image along one axis (0 <-> 0, + <-> -)
__device__ __forceinline__ int rev3(int c) { return c == 0 ? 0 : 3 - c; }

// Quadratic Lagrange basis over the classes xi = {0, +1, -1}, evaluated at
// s + r xi_b: B[i][b] = L_i(s + r xi_b) with L_0 = 1 - y^2,
// L_+ = y (y + 1) / 2, L_- = y (y - 1) / 2.  B is the one-axis gauge
// transfer (structs.cuh:343-551) from a gauge (u, c) to (U, C) for
// s = (u - U) / C, r = c / C.
__device__ __forceinline__ void basis_rows(float s, float r, float B[3][3]) {
  const float y[3] = {s, s + r, s - r};
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const float yb = y[b], h = 0.5f * yb;
    B[0][b] = fmaf(-yb, yb, 1.f);
    B[1][b] = fmaf(h, yb, h);
    B[2][b] = fmaf(h, yb, -h);
  }
}

// Transfer of one node's 27 populations (tensor-class order), in place, into
// the gauge (u_ref, c_ref) shared by the CTA: per axis the 3x3 basis with
// s = (u - u_ref) / c_ref, r = c / c_ref.  A transfer into the target gauge
// then equals the transfer of the result from (u_ref, c_ref) to the target,
// because the basis reproduces every quadratic in the particle velocity.
__device__ __forceinline__ void node_to_ref(float v[27], const float s[3], const float r[3]) {
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    float B[3][3];
    basis_rows(s[ax], r[ax], B);
    const int st = ax == 0 ? 9 : ax == 1 ? 3 : 1;
#pragma unroll
    for (int o = 0; o < 9; o++) {
      // the two other axes' indices
      const int base = ax == 0 ? o : ax == 1 ? (o / 3) * 9 + (o % 3) : o * 3;
      const float f0 = v[base], fp = v[base + st], fm = v[base + 2 * st];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const float o3 = fmaf(B[i][2], fm, fmaf(B[i][1], fp, B[i][0] * f0));
        if (i == 0) v[base] = o3; else if (i == 1) v[base + st] = o3; else v[base + 2 * st] = o3;
      }
    }
  }
}

// Z[k1,k2,i3] += sum_k3 w_i3 Gz[i3][k3] F[k1,k2,k3] (F: reference-gauge populations) for the z-classes i3
// flagged in nz (the first contraction, one per stencil node).
template <typename LoadV>
__device__ __forceinline__ void contract_z(const float Gz[3][3], const float wz[3], const bool nz[3], LoadV loadv,
                                           float Z[27]) {
  float g[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) g[i][k] = wz[i] * Gz[i][k];
#pragma unroll
  for (int k12 = 0; k12 < 9; k12++) {
    const float v0 = loadv(k12 * 3 + 0), v1 = loadv(k12 * 3 + 1), v2 = loadv(k12 * 3 + 2);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      if (!nz[i]) continue;
      float& o = Z[k12 * 3 + i];
      o = fmaf(g[i][2], v2, fmaf(g[i][1], v1, fmaf(g[i][0], v0, o)));
    }
  }
}

// Y[k1,i2,i3] += sum_k2 w_i2 Gy[i2][k2] Z[k1,k2,i3] (one per stencil column)
__device__ __forceinline__ void contract_y(const float Gy[3][3], const float wy[3], const bool ny[3], const float Z[27],
                                           float Y[27]) {
  float g[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) g[i][k] = wy[i] * Gy[i][k];
#pragma unroll
  for (int k1 = 0; k1 < 3; k1++)
#pragma unroll
    for (int i2 = 0; i2 < 3; i2++) {
      if (!ny[i2]) continue;
#pragma unroll
      for (int i3 = 0; i3 < 3; i3++) {
        float& o = Y[(k1 * 3 + i2) * 3 + i3];
        o = fmaf(g[i2][2], Z[(k1 * 3 + 2) * 3 + i3],
                 fmaf(g[i2][1], Z[(k1 * 3 + 1) * 3 + i3], fmaf(g[i2][0], Z[k1 * 9 + i3], o)));
      }
    }
}

// acc[i1,i2,i3] += sum_k1 w_i1 Gx[i1][k1] Y[k1,i2,i3] (one per stencil row)
__device__ __forceinline__ void contract_x(const float Gx[3][3], const float wx[3], const bool nx[3], const float Y[27],
                                           float acc[27]) {
  float g[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) g[i][k] = wx[i] * Gx[i][k];
#pragma unroll
  for (int i1 = 0; i1 < 3; i1++) {
    if (!nx[i1]) continue;
#pragma unroll
    for (int i23 = 0; i23 < 9; i23++) {
      float& o = acc[i1 * 9 + i23];
      o = fmaf(g[i1][2], Y[18 + i23], fmaf(g[i1][1], Y[9 + i23], fmaf(g[i1][0], Y[i23], o)));
    }
  }
}

// interpolation weight of relative offset o for a window starting at ro
template <int N> __device__ __forceinline__ float wpick(const float w[N], int ro, int o) {
  const int j = o - ro;
  float r = 0.f;
#pragma unroll
  for (int k = 0; k < N; k++) r = (j == k) ? w[k] : r;
  return r;
}

// Per-CTA partial of the step sums, written instead of the atomic update
// when the kernel runs without a context (kPartials = true; a.sums then
// points at an array of one BlockPartial per CTA).
struct BlockPartial {
  double mass, mom[3], enrg, k;
  unsigned long long niter_sum, nonconv, work;
  int niter_max;
  int pad;
};

__device__ __forceinline__ void write_block_partial(NodeSums s, BlockPartial* out) {
  __shared__ double pd[6][THREADS / 32];
  __shared__ unsigned long long pu[3][THREADS / 32];
  __shared__ int pm[THREADS / 32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int warp = tid >> 5;
  double v[6] = {s.mass, s.m0, s.m1, s.m2, s.enrg, s.k};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 6; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    s.niter += __shfl_xor_sync(0xffffffffu, s.niter, o);
    s.nonconv += __shfl_xor_sync(0xffffffffu, s.nonconv, o);
    s.work += __shfl_xor_sync(0xffffffffu, s.work, o);
    s.nmax = max(s.nmax, __shfl_xor_sync(0xffffffffu, s.nmax, o));
  }
  if ((tid & 31) == 0) {
    for (int q = 0; q < 6; q++) pd[q][warp] = v[q];
    pu[0][warp] = s.niter; pu[1][warp] = s.nonconv; pu[2][warp] = s.work; pm[warp] = s.nmax;
  }
  __syncthreads();
  if (tid == 0) {
    BlockPartial b = {};
    for (int w = 0; w < THREADS / 32; w++) {
      b.mass += pd[0][w]; b.mom[0] += pd[1][w]; b.mom[1] += pd[2][w]; b.mom[2] += pd[3][w];
      b.enrg += pd[4][w]; b.k += pd[5][w];
      b.niter_sum += pu[0][w]; b.nonconv += pu[1][w]; b.work += pu[2][w];
      b.niter_max = max(b.niter_max, pm[w]);
    }
    out[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = b;
  }
}

template <int N, bool kPartials = false>
__global__ void __launch_bounds__(THREADS, 1) pull_d3q27_tile_kernel(StepArgs<float> a) {
  using L = Lattice<POND_D3Q27>;
  extern __shared__ __align__(16) float sm[];
  const int tid = threadIdx.x + TX * (threadIdx.y + TY * threadIdx.z);
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;

  // ---- reference gauge of the CTA: the gauge of the tile's centre node
  //      ((0, 1) if it is not finite or its c is 0)
  float uref[3], icref;
  {
    bool rv[3];
    const int gx = resolve_axis(x0 + TX / 2, a.nx, a.bc[0], rv[0]);
    const int gy = resolve_axis(y0 + TY / 2, a.ny, a.bc[1], rv[1]);
    const int gz = resolve_axis(z0 + TZ / 2, a.nz, a.bc[2], rv[2]);
    const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
    const float T = a.g_in[3 * a.N + g];
    const float cc = copysignf(sqrtf(fabsf(T) * (float)(1.0 / L::TLat)), T);
    bool ok = fabsf(cc) <= 3.0e38f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float v = a.g_in[(long long)k * a.N + g];
      uref[k] = rv[k] ? -v : v;
      ok = ok && fabsf(v) <= 3.0e38f;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) uref[k] = ok ? uref[k] : 0.f;
    icref = (ok && fabsf(cc) > 1.0e-20f) ? 1.f / cc : 1.f;
  }
  const float cref = 1.f / icref;

  // ---- stage: each thread copies whole staged nodes (27 populations in
  // tensor-class order, the mirror reversing classes) with asynchronous
  // copies, waits for its own copies and transfers its nodes into the
  // reference gauge; boundary resolution happens in the addresses, the gauge
  // comes straight from global memory (mirrored velocity components flip; a
  // node with a non-finite gauge contributes nothing, non-finite populations
  // count as 0)
  for (int i = tid; i < SN; i += THREADS) {
    const int hx = i % SX, hy = (i / SX) % SY, hz = i / (SX * SY);
    bool rv[3];
    const int gx = resolve_axis(x0 - H + hx, a.nx, a.bc[0], rv[0]);
    const int gy = resolve_axis(y0 - H + hy, a.ny, a.bc[1], rv[1]);
    const int gz = resolve_axis(z0 - H + hz, a.nz, a.bc[2], rv[2]);
    const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
#pragma unroll
    for (int t = 0; t < 27; t++) {
      int cx = t / 9, cy = (t / 3) % 3, cz = t % 3;
      if (rv[0]) cx = rev3(cx);
      if (rv[1]) cy = rev3(cy);
      if (rv[2]) cz = rev3(cz);
      cp_async4(&sm[i * NS + t], a.f_in + (long long)c_ref27[cx * 9 + cy * 3 + cz] * a.N + g);
    }
  }
  cp_async_wait_all();
  for (int i = tid; i < SN; i += THREADS) {
    const int hx = i % SX, hy = (i / SX) % SY, hz = i / (SX * SY);
    bool rv[3];
    const int gx = resolve_axis(x0 - H + hx, a.nx, a.bc[0], rv[0]);
    const int gy = resolve_axis(y0 - H + hy, a.ny, a.bc[1], rv[1]);
    const int gz = resolve_axis(z0 - H + hz, a.nz, a.bc[2], rv[2]);
    const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
    float u[3];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float v = __ldg(&a.g_in[(long long)k * a.N + g]);
      u[k] = rv[k] ? -v : v;
      ok = ok && fabsf(v) <= 3.0e38f;
    }
    const float T = __ldg(&a.g_in[3 * a.N + g]);
    const float c = copysignf(sqrtf(fabsf(T) * (float)(1.0 / L::TLat)), T);
    ok = ok && fabsf(c) <= 3.0e38f;
    float v[27];
    {
      const float4* s4 = reinterpret_cast<const float4*>(sm + i * NS);
#pragma unroll
      for (int q = 0; q < 7; q++) {
        const float4 w = s4[q];
        const float e[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (4 * q + j < 27) v[4 * q + j] = (ok && fabsf(e[j]) <= 3.402823466e38f) ? e[j] : 0.f;
      }
    }
    const float r = ok ? c * icref : 0.f;
    const float sq[3] = {ok ? (u[0] - uref[0]) * icref : 0.f, ok ? (u[1] - uref[1]) * icref : 0.f,
                         ok ? (u[2] - uref[2]) * icref : 0.f};
    const float rq[3] = {r, r, r};
    node_to_ref(v, sq, rq);
    {
      float4* s4 = reinterpret_cast<float4*>(sm + i * NS);
#pragma unroll
      for (int q = 0; q < 7; q++)
        s4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], 4 * q + 3 < 27 ? v[4 * q + 3] : 0.f);
    }
  }
  __syncthreads();

  const int lx = threadIdx.x, ly = threadIdx.y, lz = threadIdx.z;
  const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
  const bool active = x < a.nx && y < a.ny && z < a.nz;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  const long long idx = active ? x + (long long)a.nx * (y + (long long)a.ny * z) : 0;
  // the node's current populations live in shared memory between iterations,
  // which keeps them out of the loop's registers
  float* f0s = sm + NS * SN + tid;
  double rho0 = 1, U[3] = {0, 0, 0}, T = L::TLat;
  {
    float f0[27];
    if (active) load_center<POND_D3Q27, float>(a, idx, f0, rho0, U, T);
    else
#pragma unroll
      for (int t = 0; t < 27; t++) f0[t] = 0.f;
#pragma unroll
    for (int t = 0; t < 27; t++) f0s[t * THREADS] = f0[t];
  }
  const int pos[3] = {x, y, z};
  const int sbase = (lz + H) * SX * SY + (ly + H) * SX + (lx + H);
  bool done = !active;
  bool conv = false;
  int niter = 0;
  unsigned long long work = 0;
  while (__any_sync(0xffffffffu, !done)) {
    if (!done) niter++;
    const double C = sqrt(T * (1.0 / L::TLat));
    // relative window origins and Lagrange weights per axis and class
    int ro[3][3];
    float wt[3][3][N];
    int lo[3], hi[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double crd = double(pos[ax]) - (C * L::xi1(c) + U[ax]);
        const int org = window_origin<N>(crd, ax);
        ro[ax][c] = org - pos[ax];
        if (N == 2) { wt[ax][c][0] = float(1 - (crd - org)); wt[ax][c][N - 1] = float(crd - org); }
        else lagr_weights<N, float>(crd - double(org), wt[ax][c]);
      }
      lo[ax] = min(ro[ax][0], min(ro[ax][1], ro[ax][2]));
      hi[ax] = max(ro[ax][0], max(ro[ax][1], ro[ax][2])) + N - 1;
    }
    // transfer from the reference gauge to this iteration's target gauge,
    // per axis: G[i][k] = L_i(b + a xi_k), a = c_ref / C, b = (u_ref - U) / C
    const float ainv = float(double(cref) / C);
    float bq[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) bq[ax] = float((double(uref[ax]) - U[ax]) / C);
    float Gz[3][3];  // the z basis is used per stencil node; x and y are rebuilt per row and column
    basis_rows(bq[2], ainv, Gz);
    float acc[27];
#pragma unroll
    for (int t = 0; t < 27; t++) acc[t] = 0.f;
    const bool inside = lo[0] >= -H && lo[1] >= -H && lo[2] >= -H && hi[0] <= H && hi[1] <= H && hi[2] <= H;
    if (__all_sync(0xffffffffu, inside || done)) {
      // warp-uniform offsets: the union of the unconverged lanes' stencils
      int wl[3], wh[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        wl[ax] = __reduce_min_sync(0xffffffffu, done ? H : lo[ax]);
        wh[ax] = __reduce_max_sync(0xffffffffu, done ? -H : hi[ax]);
      }
      // every target class at every offset (a class a lane does not weight
      // there gets weight 0): branch-free contractions the scheduler can
      // interleave, which measured faster than skipping the classes no lane
      // of the warp weights (54.8 against 58.8 ms per 256^3 step)
      const bool all3[3] = {true, true, true};
      if (!done) {  // floating-point operations of the contractions below
        const unsigned long long ex = wh[0] - wl[0] + 1, ey = wh[1] - wl[1] + 1, ez = wh[2] - wl[2] + 1;
        work += ex * ey * ez * (54ull * 3 + 9) + ex * ey * (54ull * 3 + 9) + ex * (54ull * 3 + 9);
      }
      for (int ox = wl[0]; ox <= wh[0]; ox++) {
        float wx[3];
#pragma unroll
        for (int c = 0; c < 3; c++) wx[c] = wpick<N>(wt[0][c], ro[0][c], ox);
        float Yr[27];
#pragma unroll
        for (int t = 0; t < 27; t++) Yr[t] = 0.f;
        for (int oy = wl[1]; oy <= wh[1]; oy++) {
          float wy[3];
#pragma unroll
          for (int c = 0; c < 3; c++) wy[c] = wpick<N>(wt[1][c], ro[1][c], oy);
          float Zc[27];
#pragma unroll
          for (int t = 0; t < 27; t++) Zc[t] = 0.f;
#pragma unroll
          for (int oz = -H; oz <= H; oz++) {
            if (oz < wl[2] || oz > wh[2]) continue;
            float wz[3];
#pragma unroll
            for (int c = 0; c < 3; c++) wz[c] = wpick<N>(wt[2][c], ro[2][c], oz);
            const float4* s4 = reinterpret_cast<const float4*>(sm + (sbase + oz * SX * SY + oy * SX + ox) * NS);
            float vv[28];
#pragma unroll
            for (int q = 0; q < 7; q++) {
              const float4 w = s4[q];
              vv[4 * q] = w.x; vv[4 * q + 1] = w.y; vv[4 * q + 2] = w.z; vv[4 * q + 3] = w.w;
            }
            contract_z(Gz, wz, all3, [&](int t) { return vv[t]; }, Zc);
          }
          float Gy[3][3];
          basis_rows(bq[1], ainv, Gy);
          contract_y(Gy, wy, all3, Zc, Yr);
        }
        float Gx[3][3];
        basis_rows(bq[0], ainv, Gx);
        contract_x(Gx, wx, all3, Yr, acc);
      }
    } else if (!done) {
      // departure points beyond the staged halo: this lane reads global memory
      // and transfers each stencil node into the reference gauge itself
      const unsigned long long ex = window_positions<N, 3>(ro[0]), ey = window_positions<N, 3>(ro[1]),
                               ez = window_positions<N, 3>(ro[2]);
      work += ex * ey * ez * 171 + ex * ey * 171 + ex * 171;
      const bool all3[3] = {true, true, true};
      for (int ox = lo[0]; ox <= hi[0]; ox = window_next<N, 3>(ro[0], ox)) {
        bool rv[3] = {false, false, false};
        const int gx = resolve_axis(x + ox, a.nx, a.bc[0], rv[0]);
        float wx[3];
#pragma unroll
        for (int c = 0; c < 3; c++) wx[c] = wpick<N>(wt[0][c], ro[0][c], ox);
        float Yr[27];
#pragma unroll
        for (int t = 0; t < 27; t++) Yr[t] = 0.f;
        for (int oy = lo[1]; oy <= hi[1]; oy = window_next<N, 3>(ro[1], oy)) {
          const int gy = resolve_axis(y + oy, a.ny, a.bc[1], rv[1]);
          float wy[3];
#pragma unroll
          for (int c = 0; c < 3; c++) wy[c] = wpick<N>(wt[1][c], ro[1][c], oy);
          float Zc[27];
#pragma unroll
          for (int t = 0; t < 27; t++) Zc[t] = 0.f;
          for (int oz = lo[2]; oz <= hi[2]; oz = window_next<N, 3>(ro[2], oz)) {
            const int gz = resolve_axis(z + oz, a.nz, a.bc[2], rv[2]);
            float wz[3];
#pragma unroll
            for (int c = 0; c < 3; c++) wz[c] = wpick<N>(wt[2][c], ro[2][c], oz);
            const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
            const float un[3] = {a.g_in[g], a.g_in[a.N + g], a.g_in[2 * a.N + g]};
            const float Tn = a.g_in[3 * a.N + g];
            const bool ok = fabsf(un[0]) <= 3.0e38f && fabsf(un[1]) <= 3.0e38f && fabsf(un[2]) <= 3.0e38f &&
                            fabsf(Tn) <= 3.0e38f;
            const float cn = copysignf(sqrtf(fabsf(Tn) * (float)(1.0 / L::TLat)), Tn);
            float v[27];
#pragma unroll
            for (int t = 0; t < 27; t++)
              v[t] = ok ? finite_or_zero_f(__ldg(&a.f_in[(long long)c_ref27[t] * a.N + g])) : 0.f;
            float sq[3], rq[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
              sq[k] = ok ? ((rv[k] ? -un[k] : un[k]) - uref[k]) * icref : 0.f;
              rq[k] = ok ? (rv[k] ? -cn : cn) * icref : 0.f;
            }
            node_to_ref(v, sq, rq);
            contract_z(Gz, wz, all3, [&](int t) { return v[t]; }, Zc);
          }
          float Gy[3][3];
          basis_rows(bq[1], ainv, Gy);
          contract_y(Gy, wy, all3, Zc, Yr);
        }
        float Gx[3][3];
        basis_rows(bq[0], ainv, Gx);
        contract_x(Gx, wx, all3, Yr, acc);
      }
    }
    if (!done) {
      if (!(C >= 1.0e-300)) {  // C <= 0, NaN, or 1/C beyond 1e300
        // target T = 0: every transfer term is non-finite and dropped (structs.cuh:542)
#pragma unroll
        for (int t = 0; t < 27; t++) acc[t] = 0.f;
      }
      float f0[27];
#pragma unroll
      for (int t = 0; t < 27; t++) f0[t] = f0s[t * THREADS];
      conv = moments_and_test<POND_D3Q27, float>(a, acc, f0, C, rho0, U, T);
#pragma unroll
      for (int t = 0; t < 27; t++) f0s[t * THREADS] = f0[t];
      if (conv || niter >= a.max_iter) done = true;
    }
  }
  if (active) {
    float f0[27];
#pragma unroll
    for (int t = 0; t < 27; t++) f0[t] = f0s[t * THREADS];
    finish_node<POND_D3Q27, float>(a, idx, f0, rho0, U, T, niter, conv, ns);
    ns.work = work;
  }
  if constexpr (kPartials) write_block_partial(ns, reinterpret_cast<BlockPartial*>(a.sums));
  else reduce_and_commit(ns, a.sums);
}

}  // namespace d27
}  // namespace pond
