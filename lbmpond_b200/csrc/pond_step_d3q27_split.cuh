// D3Q27 PonD pull step, float32, three lanes per node (the benchmark kernel).
//
// The arithmetic of pull_d3q27_tile_kernel (steps.cu:356-588 LBMpull with
// propagate<N>, N = 2, 3, 4, transferred through a reference gauge shared by
// the CTA), with the node's work split by x-class over three lanes:
//
//  * lane (n, q) of a warp (lane = 3 n + q, ten nodes per warp, lanes 30 and
//    31 shadow node 9) owns reference-gauge x-class q as the source of the z
//    and y contractions and target x-class q for the x contraction and the
//    output: per stencil node it contracts the z weights and R -> target z
//    transfer against the nine R-gauge populations (q, *, *) (27 FMA), per
//    stencil column the y weights and transfer (27 FMA), and per stencil row
//    it gathers the two other source classes of its node by shuffle and adds
//    its target class's x weight and transfer (27 FMA).  A lane keeps 27
//    partial sums where one lane per node needs 81, so the kernel fits 128
//    registers;
//  * a CTA owns a 10 x 4 x 2 tile (eight warps, one x-row each) and stages it
//    with a halo of 2 (14 x 8 x 6 nodes, 27 planes, 75 KB), so two CTAs share
//    an SM and one CTA's slowest nodes overlap the other's work.  Each
//    staging thread fetches its staged nodes with asynchronous copies,
//    resolving the boundaries in the addresses, and transfers them into the
//    reference gauge itself: no barrier between staging and transfer, and no
//    gauge planes in shared memory;
//  * the plane stride of the staged populations is 26 mod 32 (9 planes =
//    10 mod 32), so the 30 addresses of a warp's load (ten nodes, three
//    x-classes) fall in distinct banks;
//  * the iteration is warp-synchronous over the union of the ten nodes'
//    stencils; a warp whose departure points leave the halo runs that
//    iteration from global memory.
#pragma once
#include "pond_step_d3q27.cuh"

namespace pond {
namespace d27s {

constexpr int TX = 10, TY = 4, TZ = 2, H = 2;
constexpr int SX = TX + 2 * H, SY = TY + 2 * H, SZ = TZ + 2 * H;
constexpr int SN = SX * SY * SZ;  // 672 staged nodes
constexpr int PS = ((SN + 31) / 32) * 32 + 26;  // plane stride, 26 mod 32: 9 * PS = 10 mod 32
static_assert((9 * PS) % 32 == 10, "three x-classes of ten nodes must hit 30 distinct banks");
constexpr int WARPS = TY * TZ;  // one x-row of ten nodes per warp
constexpr int THREADS = 32 * WARPS;
constexpr size_t SMEM_BYTES = size_t(27) * PS * sizeof(float) + size_t(9) * THREADS * sizeof(float);

// lanes of node slot n: bits 3n .. 3n+2
__device__ __forceinline__ unsigned node_mask(int n) { return 7u << (3 * n); }

// One iteration's contractions of a node whose departure points leave the
// staged halo: every stencil node is read from global memory and transferred
// into R by each of the node's three lanes (lane q keeps R x-class q).  Kept
// out of line so that the staged path's register budget does not carry it.
template <int N>
__device__ __noinline__ void global_iteration(const StepArgs<float>& a, int x, int y, int z, int q, int n,
                                          const int lo[3], const int hi[3], const int ro[3][3],
                                          const float wyz[2][3][N], const float wxq[N], int rxq,
                                          const float Gz[3][3], float bqy, float ainv, const float gxq[3],
                                          const float uref[3], float icref, float acc[9],
                                          unsigned long long& work) {
  using L = Lattice<POND_D3Q27>;
  const unsigned nmask = node_mask(n);
  if (q == 0) {
    const unsigned long long ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
    work += 3ull * (ex * ey * ez * (63 + 486) + ex * ey * 63 + ex * 57);
  }
  for (int ox = lo[0]; ox <= hi[0]; ox++) {
    bool rv[3] = {false, false, false};
    const int gx = resolve_axis(x + ox, a.nx, a.bc[0], rv[0]);
    float Yr[9];
#pragma unroll
    for (int t = 0; t < 9; t++) Yr[t] = 0.f;
    for (int oy = lo[1]; oy <= hi[1]; oy++) {
      const int gy = resolve_axis(y + oy, a.ny, a.bc[1], rv[1]);
      float Zc[9];
#pragma unroll
      for (int t = 0; t < 9; t++) Zc[t] = 0.f;
      for (int oz = lo[2]; oz <= hi[2]; oz++) {
        const int gz = resolve_axis(z + oz, a.nz, a.bc[2], rv[2]);
        const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
        const float un[3] = {a.g_in[g], a.g_in[a.N + g], a.g_in[2 * a.N + g]};
        const float Tn = a.g_in[3 * a.N + g];
        const bool ok = fabsf(un[0]) <= 3.0e38f && fabsf(un[1]) <= 3.0e38f && fabsf(un[2]) <= 3.0e38f &&
                        fabsf(Tn) <= 3.0e38f;
        const float cn = copysignf(sqrtf(fabsf(Tn) * (float)(1.0 / L::TLat)), Tn);
        float v[27];
#pragma unroll
        for (int t = 0; t < 27; t++)
          v[t] = ok ? finite_or_zero_f(__ldg(&a.f_in[(long long)d27::c_ref27[t] * a.N + g])) : 0.f;
        float sq[3], rq[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          sq[k] = ok ? ((rv[k] ? -un[k] : un[k]) - uref[k]) * icref : 0.f;
          rq[k] = ok ? (rv[k] ? -cn : cn) * icref : 0.f;
        }
        d27::node_to_ref(v, sq, rq);
        float g3[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const float w = d27::wpick<N>(wyz[1][i], ro[2][i], oz);
#pragma unroll
          for (int k = 0; k < 3; k++) g3[i][k] = w * Gz[i][k];
        }
#pragma unroll
        for (int k2 = 0; k2 < 3; k2++) {
          const float v0 = q == 0 ? v[3 * k2] : q == 1 ? v[9 + 3 * k2] : v[18 + 3 * k2];
          const float v1 = q == 0 ? v[3 * k2 + 1] : q == 1 ? v[10 + 3 * k2] : v[19 + 3 * k2];
          const float v2 = q == 0 ? v[3 * k2 + 2] : q == 1 ? v[11 + 3 * k2] : v[20 + 3 * k2];
#pragma unroll
          for (int i3 = 0; i3 < 3; i3++)
            Zc[3 * k2 + i3] = fmaf(g3[i3][2], v2, fmaf(g3[i3][1], v1, fmaf(g3[i3][0], v0, Zc[3 * k2 + i3])));
        }
      }
      float Gy[3][3];
      d27::basis_rows(bqy, ainv, Gy);
#pragma unroll
      for (int i2 = 0; i2 < 3; i2++) {
        const float w = d27::wpick<N>(wyz[0][i2], ro[1][i2], oy);
        const float g0 = w * Gy[i2][0], g1 = w * Gy[i2][1], g2 = w * Gy[i2][2];
#pragma unroll
        for (int i3 = 0; i3 < 3; i3++)
          Yr[3 * i2 + i3] = fmaf(g2, Zc[6 + i3], fmaf(g1, Zc[3 + i3], fmaf(g0, Zc[i3], Yr[3 * i2 + i3])));
      }
    }
    const float wq = d27::wpick<N>(wxq, rxq, ox);
    const int l0 = 3 * n;
#pragma unroll
    for (int t = 0; t < 9; t++) {
      const float y0v = __shfl_sync(nmask, Yr[t], l0);
      const float y1v = __shfl_sync(nmask, Yr[t], l0 + 1);
      const float y2v = __shfl_sync(nmask, Yr[t], l0 + 2);
      acc[t] = fmaf(wq, fmaf(gxq[2], y2v, fmaf(gxq[1], y1v, gxq[0] * y0v)), acc[t]);
    }
  }
}

template <int N, bool kPartials = false>
__global__ void __launch_bounds__(THREADS, 2) pull_d3q27_split_kernel(StepArgs<float> a) {
  using L = Lattice<POND_D3Q27>;
  extern __shared__ __align__(16) float sm[];
  float* f0s = sm + 27 * PS;  // the iterate's populations of each lane, [9][THREADS]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;

  // ---- reference gauge R: the gauge of tile node (5, 2, 1) ((0, 1) if not finite or c = 0)
  float uref[3], cref;
  {
    bool rv[3];
    const int gx = resolve_axis(x0 + TX / 2, a.nx, a.bc[0], rv[0]);
    const int gy = resolve_axis(y0 + TY / 2, a.ny, a.bc[1], rv[1]);
    const int gz = resolve_axis(z0 + TZ / 2, a.nz, a.bc[2], rv[2]);
    const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
    const float T = a.g_in[3 * a.N + g];
    const float cc = copysignf(sqrtf(fabsf(T) * (float)(1.0 / L::TLat)), T);
    bool ok = fabsf(cc) <= 3.0e38f && fabsf(cc) > 1.0e-20f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float v = a.g_in[(long long)k * a.N + g];
      uref[k] = rv[k] ? -v : v;
      ok = ok && fabsf(v) <= 3.0e38f;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) uref[k] = ok ? uref[k] : 0.f;
    cref = ok ? cc : 1.f;
  }
  const float icref = 1.f / cref;

  // ---- stage: each thread copies its staged nodes (27 populations in tensor-class
  //      order, the mirror reversing classes), then transfers them into R
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
      if (rv[0]) cx = d27::rev3(cx);
      if (rv[1]) cy = d27::rev3(cy);
      if (rv[2]) cz = d27::rev3(cz);
      d27::cp_async4(&sm[t * PS + i], a.f_in + (long long)d27::c_ref27[cx * 9 + cy * 3 + cz] * a.N + g);
    }
  }
  d27::cp_async_wait_all();
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
    // a node with a non-finite gauge contributes nothing (all its reference
    // terms are non-finite and dropped); non-finite populations count as 0
    float v[27];
#pragma unroll
    for (int t = 0; t < 27; t++) {
      const float x = sm[t * PS + i];
      v[t] = (ok && fabsf(x) <= 3.402823466e38f) ? x : 0.f;
    }
    const float sq[3] = {ok ? (u[0] - uref[0]) * icref : 0.f, ok ? (u[1] - uref[1]) * icref : 0.f,
                         ok ? (u[2] - uref[2]) * icref : 0.f};
    // (a mirrored axis: the classes were reversed by the copies, the velocity flips)
    const float r = ok ? c * icref : 0.f;
    const float rq[3] = {r, r, r};
    d27::node_to_ref(v, sq, rq);
#pragma unroll
    for (int t = 0; t < 27; t++) sm[t * PS + i] = v[t];
  }
  __syncthreads();

  // ---- one node per lane triple
  const bool worker = lane < 30;
  const int n = worker ? lane / 3 : 9, q = worker ? lane % 3 : lane - 30;
  const int lx = n, ly = warp % TY, lz = warp / TY;
  const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
  const bool active = worker && x < a.nx && y < a.ny && z < a.nz;
  const long long idx = active ? x + (long long)a.nx * (y + (long long)a.ny * z) : 0;
  const unsigned nmask = node_mask(n);
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  double rho0 = 1, U[3] = {0, 0, 0}, T = L::TLat;
  {  // c0.load of the centre: this lane's populations (q, i2, i3) -> f0s[(3 i2 + i3)][tid]
    float f0[9];
#pragma unroll
    for (int t = 0; t < 9; t++) f0[t] = active ? a.f_in[(long long)L::ref(q, t / 3, t % 3) * a.N + idx] : 0.f;
    if (active) {
      rho0 = a.rho_in[idx];
      U[0] = a.g_in[idx]; U[1] = a.g_in[a.N + idx]; U[2] = a.g_in[2 * a.N + idx];
      T = a.g_in[3 * a.N + idx];
      if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && T == 0) {  // set_base(1, TLat)
        rho0 = 1; T = L::TLat;
#pragma unroll
        for (int t = 0; t < 9; t++) f0[t] = float(lattice_weight_t<POND_D3Q27>(q * 9 + t));
      }
      if (a.guess) {
        U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; T = a.guess[3 * a.N + idx];
      }
    }
#pragma unroll
    for (int t = 0; t < 9; t++) f0s[t * THREADS + tid] = f0[t];
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
    // window origins (relative) and Lagrange weights: every class along y
    // and z, this lane's target class q along x
    int ro[3][3];  // [axis][class]; x: only class q is used
    float wyz[2][3][N], wxq[N];
    int lo[3], hi[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double crd = double(pos[ax]) - (C * L::xi1(c) + U[ax]);
        const int org = window_origin<N>(crd, ax);
        ro[ax][c] = org - pos[ax];
        if (ax == 0 && c != q) continue;
        float* w = ax == 0 ? wxq : wyz[ax - 1][c];
        if (N == 2) { w[0] = float(1 - (crd - org)); w[N - 1] = float(crd - org); }
        else lagr_weights<N, float>(crd - double(org), w);
      }
      lo[ax] = min(ro[ax][0], min(ro[ax][1], ro[ax][2]));
      hi[ax] = max(ro[ax][0], max(ro[ax][1], ro[ax][2])) + N - 1;
    }
    const int rxq = q == 0 ? ro[0][0] : q == 1 ? ro[0][1] : ro[0][2];
    // transfer R -> target per axis: G[i][k] = L_i(b + a xi_k), a = c_ref / C, b = (u_ref - U) / C
    const float ainv = float(double(cref) / C);
    float bq[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) bq[ax] = float((double(uref[ax]) - U[ax]) / C);
    float Gz[3][3];
    d27::basis_rows(bq[2], ainv, Gz);
    float gxq[3];  // this lane's row of the x transfer
    {
      float Gx[3][3];
      d27::basis_rows(bq[0], ainv, Gx);
#pragma unroll
      for (int k = 0; k < 3; k++) gxq[k] = q == 0 ? Gx[0][k] : q == 1 ? Gx[1][k] : Gx[2][k];
    }
    float acc[9];
#pragma unroll
    for (int t = 0; t < 9; t++) acc[t] = 0.f;
    const bool inside = lo[0] >= -H && lo[1] >= -H && lo[2] >= -H && hi[0] <= H && hi[1] <= H && hi[2] <= H;
    if (__all_sync(0xffffffffu, inside || done)) {
      int wl[3], wh[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        wl[ax] = __reduce_min_sync(0xffffffffu, done ? H : lo[ax]);
        wh[ax] = __reduce_max_sync(0xffffffffu, done ? -H : hi[ax]);
      }
      if (!done && q == 0) {  // floating-point operations of the contractions below, the node's three lanes
        const unsigned long long ex = wh[0] - wl[0] + 1, ey = wh[1] - wl[1] + 1, ez = wh[2] - wl[2] + 1;
        work += 3ull * (ex * ey * ez * 63 + ex * ey * 63 + ex * 57);
      }
      for (int ox = wl[0]; ox <= wh[0]; ox++) {
        float Yr[9];  // (i2, i3) from source x-class q
#pragma unroll
        for (int t = 0; t < 9; t++) Yr[t] = 0.f;
        for (int oy = wl[1]; oy <= wh[1]; oy++) {
          float Zc[9];  // (k2, i3)
#pragma unroll
          for (int t = 0; t < 9; t++) Zc[t] = 0.f;
#pragma unroll
          for (int oz = -H; oz <= H; oz++) {
            if (oz < wl[2] || oz > wh[2]) continue;
            float g[3][3];
#pragma unroll
            for (int i = 0; i < 3; i++) {
              const float w = d27::wpick<N>(wyz[1][i], ro[2][i], oz);
#pragma unroll
              for (int k = 0; k < 3; k++) g[i][k] = w * Gz[i][k];
            }
            const float* sv = sm + (9 * q) * PS + (sbase + oz * SX * SY + oy * SX + ox);
#pragma unroll
            for (int k2 = 0; k2 < 3; k2++) {
              const float v0 = sv[(3 * k2) * PS], v1 = sv[(3 * k2 + 1) * PS], v2 = sv[(3 * k2 + 2) * PS];
#pragma unroll
              for (int i3 = 0; i3 < 3; i3++)
                Zc[3 * k2 + i3] = fmaf(g[i3][2], v2, fmaf(g[i3][1], v1, fmaf(g[i3][0], v0, Zc[3 * k2 + i3])));
            }
          }
          float Gy[3][3];
          d27::basis_rows(bq[1], ainv, Gy);
#pragma unroll
          for (int i2 = 0; i2 < 3; i2++) {
            const float w = d27::wpick<N>(wyz[0][i2], ro[1][i2], oy);
            const float g0 = w * Gy[i2][0], g1 = w * Gy[i2][1], g2 = w * Gy[i2][2];
#pragma unroll
            for (int i3 = 0; i3 < 3; i3++)
              Yr[3 * i2 + i3] = fmaf(g2, Zc[6 + i3], fmaf(g1, Zc[3 + i3], fmaf(g0, Zc[i3], Yr[3 * i2 + i3])));
          }
        }
        // the row: this lane's target class q gathers the three source classes of its node
        const float wq = d27::wpick<N>(wxq, rxq, ox);
        const int l0 = 3 * n;
#pragma unroll
        for (int t = 0; t < 9; t++) {
          const float y0v = __shfl_sync(0xffffffffu, Yr[t], l0);
          const float y1v = __shfl_sync(0xffffffffu, Yr[t], l0 + 1);
          const float y2v = __shfl_sync(0xffffffffu, Yr[t], l0 + 2);
          acc[t] = fmaf(wq, fmaf(gxq[2], y2v, fmaf(gxq[1], y1v, gxq[0] * y0v)), acc[t]);
        }
      }
    } else if (!done) {
      // departure points beyond the staged halo: the node's lanes read global
      // memory and transfer each stencil node into R themselves
      global_iteration<N>(a, x, y, z, q, n, lo, hi, ro, wyz, wxq, rxq, Gz, bq[1], ainv, gxq, uref, icref, acc,
                          work);
    }
    // calcMoments (structs.cuh:315-342) of the node over its three lanes,
    // the T < 0 guard (steps.cu:475) and isConv (steps.cu:58-75), in float64
    if (!(C >= 1.0e-300)) {  // target T = 0: every transfer term is non-finite and dropped (structs.cuh:542)
#pragma unroll
      for (int t = 0; t < 9; t++) acc[t] = 0.f;
    }
    double mv[5] = {0, 0, 0, 0, 0};
    {
      const double vx = C * L::xi1(q) + U[0];
#pragma unroll
      for (int t = 0; t < 9; t++) {
        const double fv = acc[t], vy = C * L::xi1(t / 3) + U[1], vz = C * L::xi1(t % 3) + U[2];
        mv[0] += fv; mv[1] += fv * vx; mv[2] += fv * vy; mv[3] += fv * vz;
        mv[4] += fv * (vx * vx + vy * vy + vz * vz);
      }
    }
    // the node's sum in class order 0, 1, 2 on all three lanes (the same rounding everywhere)
    const int l0 = 3 * n;
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const double s0 = __shfl_sync(0xffffffffu, mv[k], l0), s1 = __shfl_sync(0xffffffffu, mv[k], l0 + 1),
                   s2 = __shfl_sync(0xffffffffu, mv[k], l0 + 2);
      mv[k] = (s0 + s1) + s2;
    }
    bool ok = true;
    double rho = mv[0], m[4] = {mv[1], mv[2], mv[3], mv[4]}, Tn = T;
    if (!done) {
      if (rho != 0) {
        const double ir = 1.0 / rho;
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] *= ir;
      }
      Tn = (m[3] - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) * (1.0 / L::Dim);
      if (Tn < 0) Tn = T;
#pragma unroll
      for (int k = 0; k < 3; k++) ok = ok && !(fabs(m[k] - U[k]) >= a.tolg_abs + a.tolg_rel * fabs(m[k]));
      ok = ok && !(fabs(Tn - T) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
#pragma unroll
      for (int t = 0; t < 9; t++) {
        const double nv = acc[t], ov = f0s[t * THREADS + tid];
        ok = ok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
      }
    }
    const bool node_ok = (__ballot_sync(0xffffffffu, !ok) & nmask) == 0u;
    if (!done) {
#pragma unroll
      for (int t = 0; t < 9; t++) f0s[t * THREADS + tid] = acc[t];
      rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; T = Tn;
      conv = node_ok;
      if (conv || niter >= a.max_iter) done = true;
    }
  }
  // BGK toward rho*w_i in the co-moving gauge (steps.cu:557-564) and the store
  if (active) {
    const float dtau = float(a.dtau), rr = float(rho0);
#pragma unroll
    for (int t = 0; t < 9; t++) {
      const float f0 = f0s[t * THREADS + tid];
      const float fb = f0 + dtau * (rr * float(lattice_weight_t<POND_D3Q27>(q * 9 + t)) - f0);
      a.f_out[(long long)L::ref(q, t / 3, t % 3) * a.N + idx] = fb;
    }
    if (q == 0) {
      const float u0 = float(U[0]), u1 = float(U[1]), u2 = float(U[2]), ts = float(T);
      a.rho_out[idx] = rr;
      a.g_out[idx] = u0; a.g_out[a.N + idx] = u1; a.g_out[2 * a.N + idx] = u2; a.g_out[3 * a.N + idx] = ts;
      if (a.niter_out) a.niter_out[idx] = niter;
      const double dr = rr, d0 = u0, d1 = u1, d2 = u2, dt = ts;
      const double u2s = d0 * d0 + d1 * d1 + d2 * d2;
      ns.mass = dr; ns.m0 = dr * d0; ns.m1 = dr * d1; ns.m2 = dr * d2;
      ns.enrg = dr * (u2s + L::Dim * dt);
      ns.k = a.kdx * u2s;
      ns.niter = niter; ns.nonconv = conv ? 0 : 1; ns.nmax = niter;
      ns.work = work;
    }
  }
  if constexpr (kPartials) d27::write_block_partial(ns, reinterpret_cast<d27::BlockPartial*>(a.sums));
  else reduce_and_commit(ns, a.sums);
}

}  // namespace d27s
}  // namespace pond
