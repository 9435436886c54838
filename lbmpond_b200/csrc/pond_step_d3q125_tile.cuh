// D3Q125 PonD pull step, float32 or float64: a tile of nodes per CTA, a warp
// per node.
//
// The arithmetic of steps.cu:151-250 PonDstepD3Q125 (quadratic stencil with
// its origin fixed at coord-1, gauge transfer by the 5-point Lagrange basis,
// float64 moments and convergence test), organised for the SM:
//
//  * a CTA owns a 4 x 4 x 4 tile and stages it with its +-1 halo (6 x 6 x 6
//    nodes: 125 population planes, the gauge velocities and c, 113 KB) once
//    per step, so two CTAs fit on an SM and every staged node serves up to
//    27 centres from shared memory;
//  * after staging, one thread per staged node transfers its populations
//    into a reference gauge R shared by the CTA (the gauge of a tile node):
//    three passes of the 5x5 basis.  The transfer of a source node into a
//    target gauge is, along each axis, a quartic in the particle velocity,
//    which the 5-point basis reproduces, so it equals the transfer R ->
//    target applied to the R-gauge populations; R -> target depends on the
//    target alone;
//  * each of the 8 warps takes 8 nodes of the tile in turn and iterates one
//    node at a time.  Lane 5p+q (25 lanes) owns R-class p along x and target
//    class q along z: per stencil node it contracts the z weights and
//    transfer against the R-gauge populations (p, *, *) (25 FMA), per stencil
//    column the y weights and transfer (25 FMA, coefficients from a per-warp
//    table), and per stencil row the x weights and transfer of its target
//    x-class p against the column results of the lanes (*, q) by shuffle
//    (25 FMA): 1,125 FMA per lane and iteration where the per-node transform
//    takes 2,025;
//  * the plane stride of the staged populations is 217 slots, so the five
//    R x-classes read in one instruction fall in distinct banks.
// Mirrored axes are handled as in the reference kernel: the staged node's
// velocity component and c flip sign along that axis (-c maps each
// population onto its mirror image), the populations stay in place.
#pragma once
#include "pond_common.cuh"
#include "pond_step_point.cuh"

namespace pond {
namespace d125t {

constexpr int T = 4;                // tile edge
constexpr int S = T + 2;            // staged edge (+-1 halo)
constexpr int SN = S * S * S;       // 216 staged nodes
constexpr int PS = SN + 1;          // plane stride: 25 * 217 = 17 mod 32
constexpr int WARPS = 8;
constexpr int THREADS = 32 * WARPS;

// TT: tile edge (4; 2 for the float64 tile with energy populations, whose
// two population sets of a 4^3 tile would not fit)
template <bool kE, typename Rs = float, int TT = T> struct SmemT {
  static constexpr int SNT = (TT + 2) * (TT + 2) * (TT + 2), PST = SNT + 1;
  Rs f[125 * PST];          // staged populations (non-finite values zeroed), then their transfer into R
  Rs h[kE ? 125 * PST : 1]; // the same for the energy populations (double-distribution extension)
  Rs u[3][SNT];             // staged velocities (sign-flipped on mirrored axes)
  Rs c[SNT];                // sqrts(T / TLat)
  unsigned char flags[SNT]; // mirrored axes (bits 0-2)
  Rs GY[WARPS][3][25];      // per warp and iteration: y weight x transfer entry, [n_y][5 i2 + k2]
};
using Smem = SmemT<false>;

static_assert(2 * (sizeof(SmemT<false>) + 1024) <= 233472, "two CTAs must fit in the 228 KB of an SM");
static_assert(sizeof(SmemT<true>) + 1024 <= 233472, "the energy variant must fit one CTA per SM");
static_assert(sizeof(SmemT<false, double>) <= 232448, "the float64 tile must fit one CTA");
static_assert(sizeof(SmemT<true, double, 2>) <= 232448, "the float64 energy tile must fit one CTA");

// one axis of a staged position: the index, with the inflow boundary's
// ghost below the low end (*ghost) and zero gradient above the high end
__device__ __forceinline__ int staged_axis(int p, int n, int bc, bool& rev, bool& ghost) {
  if (bc == POND_BC_INFLOW) {
    rev = false;
    if (p < 0) { ghost = true; return 0; }
    return p >= n ? n - 1 : p;
  }
  return resolve_axis(p, n, bc, rev);
}

// global node of staged node i (staged edge SS) and its mirror flags; -1 for
// the inflow ghost
template <int SS, typename Rs>
__device__ __forceinline__ int staged_global(const StepArgs<Rs>& a, int x0, int y0, int z0, int i, bool rv[3]) {
  const int hx = i % SS, hy = (i / SS) % SS, hz = i / (SS * SS);
  bool ghost = false;
  const int gx = staged_axis(x0 - 1 + hx, a.nx, a.bc[0], rv[0], ghost);
  const int gy = staged_axis(y0 - 1 + hy, a.ny, a.bc[1], rv[1], ghost);
  const int gz = staged_axis(z0 - 1 + hz, a.nz, a.bc[2], rv[2], ghost);
  if (ghost) { rv[0] = rv[1] = rv[2] = false; return -1; }
  return gx + a.nx * (gy + a.ny * gz);
}

// Row i of the 5-point Lagrange basis on {0, +EC1, -EC1, +EC2, -EC2}:
// L_i(y) = D_i (y^2 - P_i)(y^2 + s_i y - Q_i), coefficients per row
template <typename Rs> struct BasisRowT {
  Rs D, P, s, Q;
  __device__ __forceinline__ explicit BasisRowT(int i) {
    constexpr double e1s = EC1 * EC1, e2s = EC2 * EC2;
    D = i == 0 ? Rs(1.0 / (e1s * e2s))
               : (i <= 2 ? Rs(1.0 / (2.0 * e1s * (e1s - e2s))) : Rs(1.0 / (2.0 * e2s * (e2s - e1s))));
    P = (i == 1 || i == 2) ? Rs(e2s) : Rs(e1s);
    s = i == 1 ? Rs(EC1) : i == 2 ? -Rs(EC1) : i == 3 ? Rs(EC2) : i == 4 ? -Rs(EC2) : Rs(0);
    Q = i == 0 ? Rs(e2s) : Rs(0);
  }
  __device__ __forceinline__ Rs operator()(Rs y) const {
    const Rs y2 = y * y;
    return D * (y2 - P) * (fma(s, y, y2) - Q);
  }
};

__device__ __forceinline__ double xi5(int c) { return Lattice<POND_D3Q125>::xi1(c); }
template <typename Rs> __device__ __forceinline__ Rs xi5r(int c) {
  return c == 0 ? Rs(0) : c == 1 ? Rs(EC1) : c == 2 ? -Rs(EC1) : c == 3 ? Rs(EC2) : -Rs(EC2);
}

// LagrPol<3> factors of target class cls along one axis at the three stencil
// positions coord-1, coord, coord+1 (steps.cu:151-250 fixed-origin quadratic)
template <typename Rs>
__device__ __forceinline__ void stencil_weights(int pos, double C, double U, int cls, Rs w[3]) {
  const double crd = double(pos) - (C * xi5(cls) + U);
  lagr_weights<3, Rs>(crd - double(pos - 1), w);
}

// kE: with the energy populations of the double-distribution extension
// (staged, transferred and contracted like f; T from their sum; one CTA per SM).
// R: storage and transfer type (float64: one CTA per SM).
// TT: tile edge (2 for the float64 energy variant: 8 nodes, one per warp).
template <bool kE, typename R = float, int TT = T>
__global__ void __launch_bounds__(THREADS, (kE || sizeof(R) == 8) ? 1 : 2) pull_d3q125_tile_kernel(StepArgs<R> a) {
  static_assert(!(kE && sizeof(R) == 8 && TT > 2), "a float64 4^3 tile has no room for energy populations");
  constexpr int S = TT + 2, SN = S * S * S, PS = SN + 1;  // staged edge, staged nodes, plane stride
  using L = Lattice<POND_D3Q125>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemT<kE, R, TT>& sm = *reinterpret_cast<SmemT<kE, R, TT>*>(smem_raw);
  const R kFinMax = R(sizeof(R) == 8 ? 1.7976931348623157e308 : 3.402823466e38);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = blockIdx.x * TT, y0 = blockIdx.y * TT, z0 = blockIdx.z * TT;

  // ---- stage the tile (steps.cu:164-193 per node, once per CTA here)
  for (int i = tid; i < SN; i += THREADS) {
    bool rv[3];
    const int g = staged_global<S>(a, x0, y0, z0, i, rv);
    sm.flags[i] = (unsigned char)((rv[0] ? 1 : 0) | (rv[1] ? 2 : 0) | (rv[2] ? 4 : 0));
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const R v = g < 0 ? R(a.inflow[1 + k]) : a.g_in[(long long)k * a.N + g];
      sm.u[k][i] = rv[k] ? -v : v;
    }
    const R Tn = g < 0 ? R(a.inflow[4]) : a.g_in[3 * a.N + g];
    sm.c[i] = copysign(sqrt(fabs(Tn) * R(1.0 / L::TLat)), Tn);
  }
  for (int idx = tid; idx < 125 * SN; idx += THREADS) {
    const int p = idx / SN, i = idx - p * SN;
    bool rv[3];
    const int g = staged_global<S>(a, x0, y0, z0, i, rv);
    if (g < 0) {  // the inflow ghost: set_base of the inflow state (and its energy equilibrium)
      const double w = lattice_weight_t<POND_D3Q125>(p);
      sm.f[p * PS + i] = R(a.inflow[0] * w);
      if constexpr (kE) {
        const double C = sqrt(a.inflow[4] / L::TLat);
        const double vx = C * xi5(p / 25) + a.inflow[1], vy = C * xi5((p / 5) % 5) + a.inflow[2],
                     vz = C * xi5(p % 5) + a.inflow[3];
        sm.h[p * PS + i] = R(a.inflow[0] * w * (vx * vx + vy * vy + vz * vz + a.dof * a.inflow[4]));
      }
      continue;
    }
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(&sm.f[p * PS + i]));
    if constexpr (sizeof(R) == 8)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(a.f_in + (long long)p * a.N + g)
                   : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(a.f_in + (long long)p * a.N + g)
                   : "memory");
    if constexpr (kE) {
      const unsigned dh = static_cast<unsigned>(__cvta_generic_to_shared(&sm.h[p * PS + i]));
      if constexpr (sizeof(R) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dh), "l"(a.h_in + (long long)p * a.N + g)
                     : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dh), "l"(a.h_in + (long long)p * a.N + g)
                     : "memory");
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  for (int idx = tid; idx < 125 * SN; idx += THREADS) {
    const int p = idx / SN, i = idx - p * SN;
    R& v = sm.f[p * PS + i];
    v = finite_or_zero_f(v);
    if constexpr (kE) sm.h[p * PS + i] = finite_or_zero_f(sm.h[p * PS + i]);
  }
  __syncthreads();

  // ---- reference gauge R: the staged node at tile position (TT/2, TT/2, TT/2)
  //      ((0, 1) if that node's gauge is not finite or its c is 0)
  R uref[3], cref;
  {
    constexpr int cp = TT / 2 + 1, ci = (cp * S + cp) * S + cp;
    const R cc = sm.c[ci];
    bool ok = fabs(cc) <= kFinMax && fabs(cc) > 1.0e-20f;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      uref[ax] = sm.u[ax][ci];
      ok = ok && fabs(uref[ax]) <= kFinMax;
    }
#pragma unroll
    for (int ax = 0; ax < 3; ax++) uref[ax] = ok ? uref[ax] : 0.f;
    cref = ok ? cc : 1.f;
  }
  // ---- every staged node into R, one thread per node, three passes of the
  //      5x5 basis B[i][b] = L_i(s + r xi_b), s = (u - u_ref)/c_ref,
  //      r = +-c/c_ref; a node with a non-finite gauge contributes nothing
  {
    const R icref = 1.f / cref;
    for (int i = tid; i < SN; i += THREADS) {
      const unsigned fl = sm.flags[i];
      const R cn = sm.c[i];
      bool ok = fabs(cn) <= kFinMax;
      R sq[3], rq[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        const R un = sm.u[ax][i];
        ok = ok && fabs(un) <= kFinMax;
        sq[ax] = (un - uref[ax]) * icref;
        rq[ax] = ((fl >> ax) & 1 ? -cn : cn) * icref;
      }
      R* fi = sm.f + i;
      R* hi = kE ? sm.h + i : nullptr;
      if (!ok) {
        for (int pp = 0; pp < 125; pp++) fi[pp * PS] = 0.f;
        if constexpr (kE)
          for (int pp = 0; pp < 125; pp++) hi[pp * PS] = 0.f;
        continue;
      }
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        R B[5][5];
#pragma unroll
        for (int ii = 0; ii < 5; ii++) {
          const BasisRowT<R> Li(ii);
#pragma unroll
          for (int b = 0; b < 5; b++) B[ii][b] = finite_or_zero_f(Li(fma(rq[ax], xi5r<R>(b), sq[ax])));
        }
        const int st = ax == 0 ? 25 : ax == 1 ? 5 : 1;
#pragma unroll 5
        for (int o = 0; o < 25; o++) {
          const int base = ax == 0 ? o : ax == 1 ? 25 * (o / 5) + o % 5 : 5 * o;
          R v[5], w[5];
#pragma unroll
          for (int b = 0; b < 5; b++) v[b] = fi[(base + b * st) * PS];
#pragma unroll
          for (int ii = 0; ii < 5; ii++) {
            R t = B[ii][0] * v[0];
#pragma unroll
            for (int b = 1; b < 5; b++) t = fma(B[ii][b], v[b], t);
            w[ii] = t;
          }
#pragma unroll
          for (int ii = 0; ii < 5; ii++) fi[(base + ii * st) * PS] = w[ii];
          if constexpr (kE) {
#pragma unroll
            for (int b = 0; b < 5; b++) v[b] = hi[(base + b * st) * PS];
#pragma unroll
            for (int ii = 0; ii < 5; ii++) {
              R t = B[ii][0] * v[0];
#pragma unroll
              for (int b = 1; b < 5; b++) t = fma(B[ii][b], v[b], t);
              w[ii] = t;
            }
#pragma unroll
            for (int ii = 0; ii < 5; ii++) hi[(base + ii * st) * PS] = w[ii];
          }
        }
      }
    }
  }
  __syncthreads();

  // ---- one warp per node; lane 5p+q: R x-class p (target x-class p for the
  // output), target z-class q.  Idle lanes (25..31) compute like lane 20+q and
  // write nothing.
  const bool worker = lane < 25;
  const int j = worker ? lane / 5 : 4, k = lane % 5;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  for (int t = warp; t < TT * TT * TT; t += WARPS) {
    const int lx = t % TT, ly = (t / TT) % TT, lz = t / (TT * TT);
    const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
    if (x >= a.nx || y >= a.ny || z >= a.nz) continue;  // warp-uniform
    const long long idx = x + (long long)a.nx * (y + (long long)a.ny * z);
    // c0.load of the centre: this lane's populations (j, iy, k), iy = 0..4
    R f0[5], h0[5];
#pragma unroll
    for (int iy = 0; iy < 5; iy++) {
      f0[iy] = worker ? a.f_in[(long long)(25 * j + 5 * iy + k) * a.N + idx] : 0.f;
      h0[iy] = (kE && worker) ? a.h_in[(long long)(25 * j + 5 * iy + k) * a.N + idx] : 0.f;
    }
    double rho0 = a.rho_in[idx];
    double U[3] = {(double)a.g_in[idx], (double)a.g_in[a.N + idx], (double)a.g_in[2 * a.N + idx]};
    double Tc = a.g_in[3 * a.N + idx];
    if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && Tc == 0) {  // set_base(1, TLat)
      rho0 = 1;
      Tc = L::TLat;
#pragma unroll
      for (int iy = 0; iy < 5; iy++) {
        const double w = lattice_weight_t<POND_D3Q125>(25 * j + 5 * iy + k);
        f0[iy] = worker ? R(w) : 0.f;
        if constexpr (kE) {  // its energy at equilibrium: w (|xi|^2 + dof TLat)
          const double v2 = xi5(j) * xi5(j) + xi5(iy) * xi5(iy) + xi5(k) * xi5(k);
          h0[iy] = worker ? R(w * (v2 + a.dof * L::TLat)) : 0.f;
        }
      }
    }
    if (a.guess) {
      U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; Tc = a.guess[3 * a.N + idx];
    }
    const int pos[3] = {x, y, z};
    const int qc = ((lz + 1) * S + (ly + 1)) * S + (lx + 1);  // staged centre
    int niter = 0;
    bool conv = false;
    R acc[5], acch[5];
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(Tc / L::TLat);
      // transfer R -> target per axis: G[i][k] = L_i(b + a xi_k), a = c_ref/C, b = (u_ref - U)/C
      const R ga = R(double(cref) / C);
      R gb[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) gb[ax] = R((double(uref[ax]) - U[ax]) / C);
      // this lane's z (class k) and x (class j) transfer rows and stencil weights
      R tz[5], tx[5], wz[3], wx[3];
      stencil_weights(pos[2], C, U[2], k, wz);
      stencil_weights(pos[0], C, U[0], j, wx);
      const BasisRowT<R> Lj(j), Lk(k);
#pragma unroll
      for (int kk = 0; kk < 5; kk++) {
        tz[kk] = finite_or_zero_f(Lk(fma(ga, xi5r<R>(kk), gb[2])));
        tx[kk] = finite_or_zero_f(Lj(fma(ga, xi5r<R>(kk), gb[0])));
      }
      // y coefficients of every (n_y, i2, k2): three table entries per worker lane
      __syncwarp();  // the previous iteration's readers are done with the table
      if (worker) {
#pragma unroll
        for (int r = 0; r < 3; r++) {
          const int e = 3 * lane + r, ny = e / 25, i2 = (e / 5) % 5, k2 = e % 5;
          R wy[3];
          stencil_weights(pos[1], C, U[1], i2, wy);
          const R ty = finite_or_zero_f(BasisRowT<R>(i2)(fma(ga, xi5r<R>(k2), gb[1])));
          sm.GY[warp][ny][5 * i2 + k2] = (ny == 0 ? wy[0] : ny == 1 ? wy[1] : wy[2]) * ty;
        }
      }
      __syncwarp();
#pragma unroll
      for (int iy = 0; iy < 5; iy++) { acc[iy] = 0.f; acch[iy] = 0.f; }
#pragma unroll
      for (int nx = 0; nx < 3; nx++) {
        R Yr[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // (j, i2, k) of the row
        R Yh[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
        for (int ny = 0; ny < 3; ny++) {
          R Zc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // (j, k2, k) of the column
          R Zh[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
          for (int nz = 0; nz < 3; nz++) {
            const R wn = nz == 0 ? wz[0] : nz == 1 ? wz[1] : wz[2];
            R gz[5];
#pragma unroll
            for (int k3 = 0; k3 < 5; k3++) gz[k3] = wn * tz[k3];
            const R* fq = sm.f + (25 * j) * PS + qc + (nz - 1) * S * S + (ny - 1) * S + (nx - 1);
#pragma unroll
            for (int k2 = 0; k2 < 5; k2++)
#pragma unroll
              for (int k3 = 0; k3 < 5; k3++) Zc[k2] = fma(gz[k3], fq[(5 * k2 + k3) * PS], Zc[k2]);
            if constexpr (kE) {
              const R* hq = sm.h + (fq - sm.f);
#pragma unroll
              for (int k2 = 0; k2 < 5; k2++)
#pragma unroll
                for (int k3 = 0; k3 < 5; k3++) Zh[k2] = fma(gz[k3], hq[(5 * k2 + k3) * PS], Zh[k2]);
            }
          }
          const R* gy = sm.GY[warp][ny];
#pragma unroll
          for (int i2 = 0; i2 < 5; i2++)
#pragma unroll
            for (int k2 = 0; k2 < 5; k2++) {
              Yr[i2] = fma(gy[5 * i2 + k2], Zc[k2], Yr[i2]);
              if constexpr (kE) Yh[i2] = fma(gy[5 * i2 + k2], Zh[k2], Yh[i2]);
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < 5; k1++) {
          const R g = wx[nx] * tx[k1];
#pragma unroll
          for (int i2 = 0; i2 < 5; i2++) {
            acc[i2] = fma(g, __shfl_sync(0xffffffffu, Yr[i2], 5 * k1 + k), acc[i2]);
            if constexpr (kE) acch[i2] = fma(g, __shfl_sync(0xffffffffu, Yh[i2], 5 * k1 + k), acch[i2]);
          }
        }
      }
      if (!(C >= 1.0e-300)) {  // target T = 0: every transfer term is non-finite and dropped
#pragma unroll
        for (int iy = 0; iy < 5; iy++) { acc[iy] = 0.f; acch[iy] = 0.f; }
      }
      // calcMoments in float64 (structs.cuh:315-342), warp-wide
      constexpr int NM = kE ? 6 : 5;
      double mv[NM];
#pragma unroll
      for (int q = 0; q < NM; q++) mv[q] = 0;
      if (worker) {
        const double vx = C * xi5(j) + U[0], vz = C * xi5(k) + U[2];
#pragma unroll
        for (int iy = 0; iy < 5; iy++) {
          const double fv = acc[iy], vy = C * xi5(iy) + U[1];
          mv[0] += fv; mv[1] += fv * vx; mv[2] += fv * vy; mv[3] += fv * vz;
          mv[4] += fv * (vx * vx + vy * vy + vz * vz);
          if constexpr (kE) mv[NM - 1] += double(acch[iy]);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int m = 0; m < NM; m++) mv[m] += __shfl_xor_sync(0xffffffffu, mv[m], o);
      const double rho = mv[0];
      double m[4] = {mv[1], mv[2], mv[3], kE ? mv[NM - 1] : mv[4]};
      if (rho != 0) {
        const double ir = 1.0 / rho;
#pragma unroll
        for (int q = 0; q < 4; q++) m[q] *= ir;
      }
      // T from the second moment of f, or with energy populations from their sum
      double Tn = (m[3] - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) / (L::Dim + (kE ? a.dof : 0.0));
      if (Tn < 0) Tn = Tc;  // steps.cu:475
      bool ok = true;
#pragma unroll
      for (int q = 0; q < 3; q++) ok = ok && !(fabs(m[q] - U[q]) >= a.tolg_abs + a.tolg_rel * fabs(m[q]));
      ok = ok && !(fabs(Tn - Tc) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
      if (worker)
#pragma unroll
        for (int iy = 0; iy < 5; iy++) {
          const double nv = acc[iy], ov = f0[iy];
          ok = ok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
          if constexpr (kE) {
            const double nh = acch[iy], oh = h0[iy];
            ok = ok && !(fabs(nh - oh) >= a.tol_abs + a.tol_rel * fabs(nh));
          }
        }
      const bool all_ok = __all_sync(0xffffffffu, ok);
#pragma unroll
      for (int iy = 0; iy < 5; iy++) { f0[iy] = acc[iy]; h0[iy] = acch[iy]; }
      rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; Tc = Tn;
      if (all_ok) { conv = true; break; }
    }
    // BGK and store (steps.cu:230-248)
    const R rr = R(rho0), dtau = R(a.dtau);
    if (worker)
#pragma unroll
      for (int iy = 0; iy < 5; iy++) {
        const int p = 25 * j + 5 * iy + k;
        const R fb = f0[iy] + dtau * (rr * R(lattice_weight_t<POND_D3Q125>(p)) - f0[iy]);
        a.f_out[(long long)p * a.N + idx] = fb;
        if constexpr (kE) {  // h toward rho w (|v|^2 + dof T) in the final gauge
          const double Cf = sqrt(fabs(Tc) * (1.0 / L::TLat));
          const double vx = Cf * xi5(j) + U[0], vy = Cf * xi5(iy) + U[1], vz = Cf * xi5(k) + U[2];
          const R heq = R(double(rr) * lattice_weight_t<POND_D3Q125>(p) *
                                  (vx * vx + vy * vy + vz * vz + a.dof * Tc));
          a.h_out[(long long)p * a.N + idx] = h0[iy] + dtau * (heq - h0[iy]);
        }
      }
    if (lane == 0) {
      const R u0 = R(U[0]), u1 = R(U[1]), u2 = R(U[2]), ts = R(Tc);
      a.rho_out[idx] = rr;
      a.g_out[idx] = u0; a.g_out[a.N + idx] = u1; a.g_out[2 * a.N + idx] = u2; a.g_out[3 * a.N + idx] = ts;
      if (a.niter_out) a.niter_out[idx] = niter;
      const double dr = rr, d0 = u0, d1 = u1, d2 = u2, dt = ts;
      const double u2s = d0 * d0 + d1 * d1 + d2 * d2;
      ns.mass += dr; ns.m0 += dr * d0; ns.m1 += dr * d1; ns.m2 += dr * d2;
      ns.enrg += dr * (u2s + (L::Dim + (kE ? a.dof : 0.0)) * dt);
      ns.k += a.kdx * u2s;
      ns.niter += niter; ns.nonconv += conv ? 0 : 1; ns.nmax = max(ns.nmax, niter);
      ns.work += 27ull * niter;
    }
  }
  // ---- the CTA's share of the step sums, through the (now free) tile memory
  __syncthreads();
  double* pd = reinterpret_cast<double*>(sm.f);  // [WARPS][6]
  unsigned long long* pu = reinterpret_cast<unsigned long long*>(pd + 6 * WARPS);  // [WARPS][3]
  int* pm = reinterpret_cast<int*>(pu + 3 * WARPS);
  if (lane == 0) {
    pd[warp * 6 + 0] = ns.mass; pd[warp * 6 + 1] = ns.m0; pd[warp * 6 + 2] = ns.m1;
    pd[warp * 6 + 3] = ns.m2; pd[warp * 6 + 4] = ns.enrg; pd[warp * 6 + 5] = ns.k;
    pu[warp * 3 + 0] = ns.niter; pu[warp * 3 + 1] = ns.nonconv; pu[warp * 3 + 2] = ns.work;
    pm[warp] = ns.nmax;
  }
  __syncthreads();
  if (tid == 0) {
    double s6[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long s3[3] = {0, 0, 0};
    int mx = 0;
    for (int w = 0; w < WARPS; w++) {
      for (int q = 0; q < 6; q++) s6[q] += pd[w * 6 + q];
      for (int q = 0; q < 3; q++) s3[q] += pu[w * 3 + q];
      mx = max(mx, pm[w]);
    }
    atomicAdd(&a.sums->mass, s6[0]);
    atomicAdd(&a.sums->mom[0], s6[1]);
    atomicAdd(&a.sums->mom[1], s6[2]);
    atomicAdd(&a.sums->mom[2], s6[3]);
    atomicAdd(&a.sums->enrg, s6[4]);
    atomicAdd(&a.sums->k, s6[5]);
    atomicAdd(&a.sums->niter_sum, s3[0]);
    atomicAdd(&a.sums->nonconv, s3[1]);
    if (s3[2]) atomicAdd(&a.sums->work, s3[2]);
    atomicMax(&a.sums->niter_max, mx);
  }
}

}  // namespace d125t
}  // namespace pond
