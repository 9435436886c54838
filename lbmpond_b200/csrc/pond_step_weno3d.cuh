// D3Q27 / D3Q125 PonD pull step with WENO5 interpolation (steps.cu:774-825
// propagateWENO<3,5>, call site :458), float32 or float64.
//
// Per population i with departure point crd = x - v_i the reference takes
// three quadratic candidates S_s = LagrEval<3> on nodes
// (fx-2+s .. fx+s) x (fy .. fy+2) x (fz .. fz+2), fx = floor(crd.x+0.5) and
// likewise fy, fz (:776-778, the y/z windows start at the rounded
// coordinate), and blends them with Jiang-Shu weights from the smoothness
// indicators of five transferred values on one x-row (:780-815).  The
// reference reads that row at y = z = floor(crd.x+0.5) (:783), and its y/z
// windows start at the rounded coordinate, so the quadratic extrapolates
// (weights up to 1.875, -1.25, 0.375); POND_WENO5 keeps both.  POND_WENO5_ROW
// centres the y/z windows on the rounded coordinate (fy-1 .. fy+1) and reads
// the smoothness row through the departure point (y = fy, z = fz).  On 1D
// grids both are the same.
//
// Organisation: a group of Q1*Q1 lanes steps one node (D3Q125: 25 lanes, one
// node per warp; D3Q27: 9 lanes, three nodes per warp).  Lane (p, k) owns the
// target populations (p, i2, k), i2 = 0..Q1-1.  Every stencil site is
// transferred into the iterate's gauge once per iteration, shared by the
// group: lane (p, k) loads the site's populations of source x-class p,
// contracts z with row k of the z basis and y with the whole y basis, and
// the x contraction gathers the five source classes of its column by
// shuffle (the per-axis Lagrange-basis form of Cell::transfer_gauge,
// structs.cuh:343-551).  Each lane computes one entry of each basis matrix
// and shares it by shuffle.  The transferred value is then weighted into the
// three candidate sums of every population whose window holds the site.
#pragma once
#include "pond_step_point.cuh"

namespace pond {
namespace w3d {

constexpr int WARPS = 4;
constexpr int THREADS = 32 * WARPS;
constexpr int MAXOFF = 8;  // window offsets are clamped to +-MAXOFF nodes (|v| far beyond any stable step)

template <int LAT> struct Geo {
  static constexpr int Q1 = Lattice<LAT>::Q1;
  static constexpr int G = Q1 * Q1;   // lanes per node
  static constexpr int NPW = 32 / G;  // nodes per warp
};

// A stencil position resolved against the boundaries: the node index, the
// mirrored axes (the node's velocity component and c flip sign there, which
// maps each population onto its mirror image), or the inflow ghost.
struct Site {
  long long g;
  bool ghost;
  bool rev[3];
};

__device__ __forceinline__ Site resolve_site(int px, int py, int pz, int nx, int ny, int nz, const int bc[3]) {
  Site s;
  s.ghost = false;
  const int p[3] = {px, py, pz}, n[3] = {nx, ny, nz};
  int r[3];
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    if (bc[ax] == POND_BC_INFLOW) {
      s.rev[ax] = false;
      if (p[ax] < 0) s.ghost = true;
      r[ax] = p[ax] < 0 ? 0 : (p[ax] >= n[ax] ? n[ax] - 1 : p[ax]);
    } else {
      r[ax] = resolve_axis(p[ax], n[ax], bc[ax], s.rev[ax]);
    }
  }
  s.g = r[0] + (long long)nx * (r[1] + (long long)ny * r[2]);
  return s;
}

// The transfer of one site into the target gauge (U, C), shared by a group:
// lane (p, k) returns fT[i2] = f^target_(p, i2, k).  All 32 lanes must call
// it together (shuffles); `base` is the first lane of the caller's group.
template <int LAT, typename R>
__device__ __forceinline__ void site_transfer(const StepArgs<R>& a, const Site& st, int base, int p, int k,
                                              const R Uc[3], R invC, R fT[Lattice<LAT>::Q1]) {
  using L = Lattice<LAT>;
  constexpr int Q1 = L::Q1;
  R un[3], Tn, fv[Q1 * Q1];
  if (st.ghost) {
    const R rho_in = R(a.inflow[0]);
#pragma unroll
    for (int ax = 0; ax < 3; ax++) un[ax] = R(a.inflow[1 + ax]);
    Tn = R(a.inflow[4]);
#pragma unroll
    for (int b2 = 0; b2 < Q1; b2++)
#pragma unroll
      for (int b3 = 0; b3 < Q1; b3++)
        fv[b2 * Q1 + b3] = rho_in * R(lattice_weight_t<LAT>((p * Q1 + b2) * Q1 + b3));
  } else {
#pragma unroll
    for (int ax = 0; ax < 3; ax++) un[ax] = __ldg(&a.g_in[(long long)ax * a.N + st.g]);
    Tn = __ldg(&a.g_in[3 * a.N + st.g]);
#pragma unroll
    for (int b2 = 0; b2 < Q1; b2++)
#pragma unroll
      for (int b3 = 0; b3 < Q1; b3++)
        fv[b2 * Q1 + b3] = finite_or_zero_f(__ldg(&a.f_in[(long long)L::ref(p, b2, b3) * a.N + st.g]));
  }
  // sqrts(T/TLat) (params.h:110); a node with a non-finite gauge contributes nothing
  const R cn = copysign(sqrt(fabs(Tn) * R(1.0 / L::TLat)), Tn);
  R s[3], r[3];
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    const bool rv = !st.ghost && st.rev[ax];
    s[ax] = ((rv ? -un[ax] : un[ax]) - Uc[ax]) * invC;
    r[ax] = (rv ? -cn : cn) * invC;
  }
  // this lane's entries: Bz[k][p], By[p][k], Bx[p][k], B[i][b] = L_i(s + r xi_b)
  R lz[Q1], ly[Q1], lx[Q1];
  Basis<Q1, R>::eval(s[2] + r[2] * R(L::xi1(p)), lz);
  Basis<Q1, R>::eval(s[1] + r[1] * R(L::xi1(k)), ly);
  Basis<Q1, R>::eval(s[0] + r[0] * R(L::xi1(k)), lx);
  R bz = lz[0], by = ly[0], bx = lx[0];
#pragma unroll
  for (int c = 1; c < Q1; c++) {
    bz = (k == c) ? lz[c] : bz;
    by = (p == c) ? ly[c] : by;
    bx = (p == c) ? lx[c] : bx;
  }
  bz = finite_or_zero_f(bz);
  by = finite_or_zero_f(by);
  bx = finite_or_zero_f(bx);
  // z: Z[b2] = sum_b3 Bz[k][b3] f[p][b2][b3]   (Bz[k][b3] from lane (b3, k))
  R Z[Q1];
#pragma unroll
  for (int b2 = 0; b2 < Q1; b2++) Z[b2] = R(0);
#pragma unroll
  for (int b3 = 0; b3 < Q1; b3++) {
    const R w = __shfl_sync(0xffffffffu, bz, base + b3 * Q1 + k);
#pragma unroll
    for (int b2 = 0; b2 < Q1; b2++) Z[b2] = fma(w, fv[b2 * Q1 + b3], Z[b2]);
  }
  // y: Y[i2] = sum_b2 By[i2][b2] Z[b2]   (By[i2][b2] from lane (i2, b2))
  R Y[Q1];
#pragma unroll
  for (int i2 = 0; i2 < Q1; i2++) {
    R t = R(0);
#pragma unroll
    for (int b2 = 0; b2 < Q1; b2++) t = fma(__shfl_sync(0xffffffffu, by, base + i2 * Q1 + b2), Z[b2], t);
    Y[i2] = t;
  }
  // x: fT[i2] = sum_b1 Bx[p][b1] Y^(b1, k)[i2]   (Bx[p][b1] from lane (p, b1))
#pragma unroll
  for (int i2 = 0; i2 < Q1; i2++) fT[i2] = R(0);
#pragma unroll
  for (int b1 = 0; b1 < Q1; b1++) {
    const R w = __shfl_sync(0xffffffffu, bx, base + p * Q1 + b1);
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) fT[i2] = fma(w, __shfl_sync(0xffffffffu, Y[i2], base + b1 * Q1 + k), fT[i2]);
  }
}

// steps.cu:780-820: Jiang-Shu weights of the three candidates from the five
// transferred values u[0..4] on the smoothness row, eps = 1e-6, ideal weights
// d0, d2 = (c^2 -+ 3c + 2)/12 with c = crd.x - floor(crd.x+0.5)
__device__ __forceinline__ double weno5_blend(const double S[3], const double u[5], double cdist) {
  const double u1 = u[0], u2 = u[1], u3 = u[2], u4 = u[3], u5 = u[4];
  const double d0 = (cdist * cdist - 3 * cdist + 2) / 12.;
  const double d2 = (cdist * cdist + 3 * cdist + 2) / 12.;
  const double d1 = 1. - d0 - d2;
  const double b0 = (10 * u3 * u3 + (11 * u1 - 31 * u2) * u3 + 25 * u2 * u2 - 19 * u1 * u2 + 4 * u1 * u1) / 3.0;
  const double b1 = (4 * u4 * u4 + (5 * u2 - 13 * u3) * u4 + 13 * u3 * u3 - 13 * u2 * u3 + 4 * u2 * u2) / 3.0;
  const double b2 = (4 * u5 * u5 + (11 * u3 - 19 * u4) * u5 + 25 * u4 * u4 - 31 * u3 * u4 + 10 * u3 * u3) / 3.0;
  double w0 = d0 / ((1e-6 + b0) * (1e-6 + b0));
  double w1 = d1 / ((1e-6 + b1) * (1e-6 + b1));
  double w2 = d2 / ((1e-6 + b2) * (1e-6 + b2));
  const double ws = w0 + w1 + w2;
  w0 /= ws; w1 /= ws; w2 /= ws;
  return w0 * S[0] + w1 * S[1] + w2 * S[2];
}

__device__ __forceinline__ int clamp_off(int o) { return o < -MAXOFF ? -MAXOFF : (o > MAXOFF ? MAXOFF : o); }

// The three candidate sums S[s][i2] and the smoothness-row values U5[m][i2]
// of this lane's populations (p, i2, k), every stencil site read from global
// memory and transferred into the iterate's gauge (U, C) by the group.  All
// 32 lanes call it together; `done` lanes contribute no window.  Windows
// (relative offsets): x nodes bx .. bx+4 with candidate s on bx+s .. bx+s+2
// (weights LX[s]), z nodes bz .. bz+2 (WZ), y nodes by[i2] .. by[i2]+2
// (WY[i2]); the centred variant's smoothness row is the middle node of the
// y and z windows.  `work` counts the sites transferred (leader lane only).
template <int LAT, typename R, bool kCentred>
__device__ __forceinline__ void accumulate_global(const StepArgs<R>& a, int x, int y, int z, bool done, int base,
                                                  int p, int k, const R Uc[3], R invC, int bx, const R LX[3][3],
                                                  int bz, const R WZ[3], const int by[Lattice<LAT>::Q1],
                                                  const R WY[Lattice<LAT>::Q1][3], R S[3][Lattice<LAT>::Q1],
                                                  R U5[5][Lattice<LAT>::Q1], unsigned long long& work, bool leader) {
  constexpr int Q1 = Lattice<LAT>::Q1;
  // the warp's union of windows (relative offsets)
  int ylo = by[0], yhi = by[0];
#pragma unroll
  for (int i2 = 1; i2 < Q1; i2++) { ylo = min(ylo, by[i2]); yhi = max(yhi, by[i2]); }
  const int wxl = __reduce_min_sync(0xffffffffu, done ? MAXOFF : bx);
  const int wxh = __reduce_max_sync(0xffffffffu, done ? -MAXOFF : bx + 4);
  const int wyl = __reduce_min_sync(0xffffffffu, done ? MAXOFF : ylo);
  const int wyh = __reduce_max_sync(0xffffffffu, done ? -MAXOFF : yhi + 2);
  const int wzl = __reduce_min_sync(0xffffffffu, done ? MAXOFF : bz);
  const int wzh = __reduce_max_sync(0xffffffffu, done ? -MAXOFF : bz + 2);
#pragma unroll
  for (int s = 0; s < 3; s++)
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) S[s][i2] = R(0);
#pragma unroll
  for (int m = 0; m < 5; m++)
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) U5[m][i2] = R(0);
  if (!done && leader) work += (unsigned long long)(wxh - wxl + 1) * (wyh - wyl + 1) * (wzh - wzl + 1);
  for (int oz = wzl; oz <= wzh; oz++) {
    const int jz = oz - bz;
    const R wz = jz == 0 ? WZ[0] : jz == 1 ? WZ[1] : jz == 2 ? WZ[2] : R(0);
    for (int oy = wyl; oy <= wyh; oy++) {
      for (int ox = wxl; ox <= wxh; ox++) {
        const Site st = resolve_site(x + ox, y + oy, z + oz, a.nx, a.ny, a.nz, a.bc);
        R fT[Q1];
        site_transfer<LAT, R>(a, st, base, p, k, Uc, invC, fT);
        const int jx = ox - bx;
        R lxs[3];
#pragma unroll
        for (int s = 0; s < 3; s++) {
          const int j = jx - s;
          lxs[s] = j == 0 ? LX[s][0] : j == 1 ? LX[s][1] : j == 2 ? LX[s][2] : R(0);
        }
#pragma unroll
        for (int i2 = 0; i2 < Q1; i2++) {
          const int jy = oy - by[i2];
          const R wy = jy == 0 ? WY[i2][0] : jy == 1 ? WY[i2][1] : jy == 2 ? WY[i2][2] : R(0);
          const R v = wy * wz * fT[i2];
#pragma unroll
          for (int s = 0; s < 3; s++) S[s][i2] = fma(lxs[s], v, S[s][i2]);
          if (kCentred && jy == 1 && jz == 1) {
#pragma unroll
            for (int m = 0; m < 5; m++) U5[m][i2] = (jx == m) ? fT[i2] : U5[m][i2];
          }
        }
      }
    }
  }
  if (!kCentred) {
    // the reference's smoothness row (:783): nodes fx-2 .. fx+2 at y = z = fx
    // (absolute coordinates; fx = x + bx + 2 for this lane's x-class)
    const int fl = __reduce_min_sync(0xffffffffu, done ? MAXOFF : bx + 2);
    const int fh = __reduce_max_sync(0xffffffffu, done ? -MAXOFF : bx + 2);
    if (!done && leader) work += 5ull * (fh - fl + 1);
    for (int df = fl; df <= fh; df++) {
      const int F = x + df;
#pragma unroll 1
      for (int m = 0; m < 5; m++) {
        const Site st = resolve_site(F - 2 + m, F, F, a.nx, a.ny, a.nz, a.bc);
        R fT[Q1];
        site_transfer<LAT, R>(a, st, base, p, k, Uc, invC, fT);
        if (df == bx + 2) {
#pragma unroll
          for (int i2 = 0; i2 < Q1; i2++)
#pragma unroll
            for (int mm = 0; mm < 5; mm++) U5[mm][i2] = (mm == m) ? fT[i2] : U5[mm][i2];
        }
      }
    }
  }
}

// The WENO5 step.  kCentred: y/z windows centred and the smoothness row
// through the departure point (POND_WENO5_ROW).
template <int LAT, typename R, bool kCentred>
__global__ void __launch_bounds__(THREADS) pull_weno3d_kernel(StepArgs<R> a) {
  using L = Lattice<LAT>;
  constexpr int Q1 = L::Q1, G = Geo<LAT>::G, NPW = Geo<LAT>::NPW;
  __shared__ double red[WARPS][32][5];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool worker = lane < NPW * G;
  const int grp = worker ? lane / G : NPW - 1;
  const int e = worker ? lane - grp * G : G - 1;
  const int base = grp * G;
  const int p = e / Q1, k = e % Q1;  // target x-class p (and source x-class p), target z-class k
  const long long node = ((long long)blockIdx.x * WARPS + warp) * NPW + grp;
  const bool active = worker && node < a.N;
  const long long idx = active ? node : 0;
  const int x = (int)(idx % a.nx), y = (int)((idx / a.nx) % a.ny), z = (int)(idx / ((long long)a.nx * a.ny));

  // c0.load of the centre (steps.cu:360-363): this lane's populations (p, i2, k)
  R f0[Q1];
#pragma unroll
  for (int i2 = 0; i2 < Q1; i2++) f0[i2] = active ? a.f_in[(long long)L::ref(p, i2, k) * a.N + idx] : R(0);
  double rho0 = 1, U[3] = {0, 0, 0}, T = L::TLat;
  if (active) {
    rho0 = a.rho_in[idx];
    U[0] = a.g_in[idx]; U[1] = a.g_in[a.N + idx]; U[2] = a.g_in[2 * a.N + idx];
    T = a.g_in[3 * a.N + idx];
    if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && T == 0) {  // set_base(1, TLat)
      rho0 = 1; T = L::TLat;
#pragma unroll
      for (int i2 = 0; i2 < Q1; i2++) f0[i2] = R(lattice_weight_t<LAT>((p * Q1 + i2) * Q1 + k));
    }
    if (a.guess) {
      U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; T = a.guess[3 * a.N + idx];
    }
  }
  const unsigned gmask = (worker ? ((G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << base) : 0u);
  bool done = !active;
  bool conv = false;
  int niter = 0;
  unsigned long long work = 0;
  while (__any_sync(0xffffffffu, !done)) {
    if (!done) niter++;
    const double C = sqrt(T / L::TLat);
    const R Uc[3] = {R(U[0]), R(U[1]), R(U[2])};
    const R invC = R(1.0 / C);
    // departure points of this lane's classes: x-class p, z-class k, every y-class
    const double crdx = double(x) - (C * L::xi1(p) + U[0]);
    const double fxd = floor(crdx + 0.5);
    const double cdist = crdx - fxd;
    const int bx = clamp_off((int)fxd - 2 - x);  // first node of the 5-node x window, relative
    R LX[3][3];                                   // candidate s on nodes bx+s .. bx+s+2
#pragma unroll
    for (int s = 0; s < 3; s++) lagr_weights<3, R>(crdx - (fxd - 2 + s), LX[s]);
    // y/z windows from floor(c+0.5) (the reference) or floor(c+0.5)-1 (centred)
    constexpr int yz0 = kCentred ? 1 : 0;
    const double crdz = double(z) - (C * L::xi1(k) + U[2]);
    const double fzd = floor(crdz + 0.5) - yz0;
    const int bz = clamp_off((int)fzd - z);
    R WZ[3];
    lagr_weights<3, R>(crdz - fzd, WZ);
    int by[Q1];
    R WY[Q1][3];
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) {
      const double crdy = double(y) - (C * L::xi1(i2) + U[1]);
      const double fyd = floor(crdy + 0.5) - yz0;
      by[i2] = clamp_off((int)fyd - y);
      lagr_weights<3, R>(crdy - fyd, WY[i2]);
    }
    R S[3][Q1], U5[5][Q1];
    accumulate_global<LAT, R, kCentred>(a, x, y, z, done, base, p, k, Uc, invC, bx, LX, bz, WZ, by, WY, S, U5, work,
                                       lane == base);
    // blend, calcMoments (structs.cuh:315-342) and isConv (steps.cu:58-75) in float64
    R acc[Q1];
    double mv[5] = {0, 0, 0, 0, 0};
    const double vx = C * L::xi1(p) + U[0], vz = C * L::xi1(k) + U[2];
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) {
      const double Sd[3] = {double(S[0][i2]), double(S[1][i2]), double(S[2][i2])};
      const double ud[5] = {double(U5[0][i2]), double(U5[1][i2]), double(U5[2][i2]), double(U5[3][i2]),
                            double(U5[4][i2])};
      acc[i2] = (C >= 1.0e-300) ? R(weno5_blend(Sd, ud, cdist)) : R(0);  // target T = 0: terms dropped
      const double fv = acc[i2], vy = C * L::xi1(i2) + U[1];
      mv[0] += fv; mv[1] += fv * vx; mv[2] += fv * vy; mv[3] += fv * vz;
      mv[4] += fv * (vx * vx + vy * vy + vz * vz);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 5; q++) red[warp][lane][q] = worker ? mv[q] : 0.0;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 5; q++) {
      double t = 0;
      for (int l = 0; l < G; l++) t += red[warp][base + l][q];
      mv[q] = t;
    }
    const double rho = mv[0];
    double m[4] = {mv[1], mv[2], mv[3], mv[4]};
    if (rho != 0) {
      const double ir = 1.0 / rho;
#pragma unroll
      for (int q = 0; q < 4; q++) m[q] *= ir;
    }
    double Tn = (m[3] - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) * (1.0 / L::Dim);
    if (Tn < 0) Tn = T;  // steps.cu:475
    bool ok = true;
#pragma unroll
    for (int q = 0; q < 3; q++) ok = ok && !(fabs(m[q] - U[q]) >= a.tolg_abs + a.tolg_rel * fabs(m[q]));
    ok = ok && !(fabs(Tn - T) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) {
      const double nv = acc[i2], ov = f0[i2];
      ok = ok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
    }
    const unsigned bad = __ballot_sync(0xffffffffu, !ok) & gmask;
    if (!done) {
#pragma unroll
      for (int i2 = 0; i2 < Q1; i2++) f0[i2] = acc[i2];
      rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; T = Tn;
      if (bad == 0) { conv = true; done = true; }
      else if (niter >= a.max_iter) done = true;
    }
  }
  // BGK toward rho*w_i (steps.cu:557-564), store, the node's share of the sums
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (active) {
    const R dtau = R(a.dtau), rr = R(rho0);
#pragma unroll
    for (int i2 = 0; i2 < Q1; i2++) {
      const int t = (p * Q1 + i2) * Q1 + k;
      const R fb = f0[i2] + dtau * (rr * R(lattice_weight_t<LAT>(t)) - f0[i2]);
      a.f_out[(long long)L::ref(p, i2, k) * a.N + idx] = fb;
    }
    if (lane == base) {
      const R u0 = R(U[0]), u1 = R(U[1]), u2 = R(U[2]), ts = R(T);
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
  reduce_and_commit(ns, a.sums);
}

}  // namespace w3d
}  // namespace pond
