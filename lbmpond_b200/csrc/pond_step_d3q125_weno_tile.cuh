// D3Q125 PonD pull step with the centred WENO5 (POND_WENO5_ROW), float32: a
// tile of nodes per CTA, a warp per node at a time.
//
// The arithmetic is pull_weno3d_kernel's centred variant (propagateWENO<3,5>,
// steps.cu:774-825, with the y/z windows centred): three quadratic
// candidates on x nodes fx-2+s .. fx+s, y nodes fy-1 .. fy+1 and z nodes
// fz-1 .. fz+1 (fx = floor(crd.x+0.5), likewise fy, fz), blended with
// Jiang-Shu weights from five transferred values on the row
// (fx-2 .. fx+2, fy, fz).  Organised for the SM like the fixed-stencil
// D3Q125 tile kernel:
//
//  * a CTA owns a 4 x 2 x 2 tile and stages it once per step with the halo
//    the windows reach while |v| < 1.5 along every axis: 3 nodes on both
//    sides in x, 2 in y and z (10 x 6 x 6 nodes, 125 population planes and
//    the gauge, 186 KB);
//  * every staged node is transferred into the tile's reference gauge R
//    once (three passes of the 5x5 basis); the transfer of a source node into
//    a target gauge equals R -> target applied to its R-gauge populations,
//    since the 5-point basis reproduces every quartic in the particle
//    velocity;
//  * eight warps step the 16 tile nodes, one node at a time; lane 5p+q owns
//    R x-class p and target z-class q.  Per
//    stencil node it contracts the R -> target z transfer against the
//    R-gauge populations (p, *, *) (25 FMA) and scales the result by its z
//    weight; per stencil column it applies the y weights and transfer of
//    every target y-class (a per-warp table); per stencil row it gathers the
//    five R x-classes of its column by shuffle, applies its target x-class
//    transfer and adds the row into the three candidate sums.  The
//    smoothness row is the same contraction with unit weights on the middle
//    window node in y and z;
//  * a warp whose node's windows leave the staged halo runs that iteration
//    from global memory (the group transfer of pull_weno3d_kernel).
#pragma once
#include "pond_step_d3q125_tile.cuh"
#include "pond_step_weno3d.cuh"

namespace pond {
namespace d125w {

constexpr int TX = 4, TY = 2, TZ = 2;      // tile
constexpr int HXL = 3, HXH = 3, HL = 2, HH = 2;  // halo: x both sides; y and z below / above
constexpr int SX = TX + HXL + HXH, SY = TY + HL + HH, SZ = TZ + HL + HH;
constexpr int SN = SX * SY * SZ;  // 360 staged nodes
constexpr int PS = SN + 1;        // plane stride: odd, so the five R x-classes of a load hit distinct banks
constexpr int NODES = TX * TY * TZ;
constexpr int WARPS = 8;  // each warp steps NODES / WARPS tile nodes in turn
constexpr int THREADS = 32 * WARPS;

struct Smem {
  float f[125 * PS];          // staged populations, then their transfer into R
  float u[3][SN];             // staged velocities (sign-flipped on mirrored axes)
  float c[SN];                // sqrts(T / TLat)
  unsigned char flags[SN];    // mirrored axes (bits 0-2)
  float GY[WARPS][5][25];     // per warp: y weight x transfer entry, [oy + HL][5 i2 + k2]
  float GD[WARPS][25];        // per warp: the y transfer itself, [5 i2 + k2]
};
static_assert(sizeof(Smem) + 4096 <= 232448, "the tile must fit one CTA");

// staged node i -> global node (-1: the inflow ghost) and mirror flags
__device__ __forceinline__ int staged_global(const StepArgs<float>& a, int x0, int y0, int z0, int i, bool rv[3]) {
  const int hx = i % SX, hy = (i / SX) % SY, hz = i / (SX * SY);
  bool ghost = false;
  const int gx = d125t::staged_axis(x0 - HXL + hx, a.nx, a.bc[0], rv[0], ghost);
  const int gy = d125t::staged_axis(y0 - HL + hy, a.ny, a.bc[1], rv[1], ghost);
  const int gz = d125t::staged_axis(z0 - HL + hz, a.nz, a.bc[2], rv[2], ghost);
  if (ghost) { rv[0] = rv[1] = rv[2] = false; return -1; }
  return gx + a.nx * (gy + a.ny * gz);
}

__global__ void __launch_bounds__(THREADS, 1) pull_d3q125_weno_tile_kernel(StepArgs<float> a) {
  using L = Lattice<POND_D3Q125>;
  using R = float;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;

  // ---- stage the tile
  for (int i = tid; i < SN; i += THREADS) {
    bool rv[3];
    const int g = staged_global(a, x0, y0, z0, i, rv);
    sm.flags[i] = (unsigned char)((rv[0] ? 1 : 0) | (rv[1] ? 2 : 0) | (rv[2] ? 4 : 0));
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const R v = g < 0 ? R(a.inflow[1 + k]) : a.g_in[(long long)k * a.N + g];
      sm.u[k][i] = rv[k] ? -v : v;
    }
    const R Tn = g < 0 ? R(a.inflow[4]) : a.g_in[3 * a.N + g];
    sm.c[i] = copysignf(sqrtf(fabsf(Tn) * R(1.0 / L::TLat)), Tn);
  }
  for (int idx = tid; idx < 125 * SN; idx += THREADS) {
    const int p = idx / SN, i = idx - p * SN;
    bool rv[3];
    const int g = staged_global(a, x0, y0, z0, i, rv);
    if (g < 0) {  // the inflow ghost: set_base of the inflow state
      sm.f[p * PS + i] = R(a.inflow[0] * lattice_weight_t<POND_D3Q125>(p));
      continue;
    }
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(&sm.f[p * PS + i]));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(a.f_in + (long long)p * a.N + g)
                 : "memory");
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();

  // ---- reference gauge R: the staged gauge of tile node (2, 1, 1)
  //      ((0, 1) if that gauge is not finite or its c is 0)
  R uref[3], cref;
  {
    constexpr int ci = ((1 + HL) * SY + (1 + HL)) * SX + (2 + HXL);
    const R cc = sm.c[ci];
    bool ok = fabsf(cc) <= 3.402823466e38f && fabsf(cc) > 1.0e-20f;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      uref[ax] = sm.u[ax][ci];
      ok = ok && fabsf(uref[ax]) <= 3.402823466e38f;
    }
#pragma unroll
    for (int ax = 0; ax < 3; ax++) uref[ax] = ok ? uref[ax] : 0.f;
    cref = ok ? cc : 1.f;
  }
  // ---- every staged node into R, one thread per node; non-finite
  //      populations count as 0, a node with a non-finite gauge as all 0
  {
    const R icref = 1.f / cref;
    for (int i = tid; i < SN; i += THREADS) {
      const unsigned fl = sm.flags[i];
      const R cn = sm.c[i];
      bool ok = fabsf(cn) <= 3.402823466e38f;
      R sq[3], rq[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        const R un = sm.u[ax][i];
        ok = ok && fabsf(un) <= 3.402823466e38f;
        sq[ax] = (un - uref[ax]) * icref;
        rq[ax] = ((fl >> ax) & 1 ? -cn : cn) * icref;
      }
      R* fi = sm.f + i;
      if (!ok) {
        for (int pp = 0; pp < 125; pp++) fi[pp * PS] = 0.f;
        continue;
      }
#pragma unroll 1
      for (int ax = 0; ax < 3; ax++) {
        R B[5][5];
#pragma unroll
        for (int ii = 0; ii < 5; ii++) {
          const d125t::BasisRowT<R> Li(ii);
#pragma unroll
          for (int b = 0; b < 5; b++) B[ii][b] = finite_or_zero_f(Li(fmaf(rq[ax], d125t::xi5r<R>(b), sq[ax])));
        }
        const int st = ax == 0 ? 25 : ax == 1 ? 5 : 1;
#pragma unroll 5
        for (int o = 0; o < 25; o++) {
          const int base = ax == 0 ? o : ax == 1 ? 25 * (o / 5) + o % 5 : 5 * o;
          R v[5], w[5];
#pragma unroll
          for (int b = 0; b < 5; b++) v[b] = finite_or_zero_f(fi[(base + b * st) * PS]);
#pragma unroll
          for (int ii = 0; ii < 5; ii++) {
            R t = B[ii][0] * v[0];
#pragma unroll
            for (int b = 1; b < 5; b++) t = fmaf(B[ii][b], v[b], t);
            w[ii] = t;
          }
#pragma unroll
          for (int ii = 0; ii < 5; ii++) fi[(base + ii * st) * PS] = w[ii];
        }
      }
    }
  }
  __syncthreads();

  // ---- one warp per tile node; lane 5p+q: R x-class p (target x-class p
  //      for the output), target z-class q.  Idle lanes (25..31) compute like
  //      lane 20+q and write nothing.
  const bool worker = lane < 25;
  const int j = worker ? lane / 5 : 4, k = lane % 5;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  for (int t = warp; t < NODES; t += WARPS) {
    const int lx = t % TX, ly = (t / TX) % TY, lz = t / (TX * TY);
    const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
    if (x < a.nx && y < a.ny && z < a.nz) {  // warp-uniform
      const long long idx = x + (long long)a.nx * (y + (long long)a.ny * z);
      R f0[5];
#pragma unroll
      for (int iy = 0; iy < 5; iy++) f0[iy] = worker ? a.f_in[(long long)(25 * j + 5 * iy + k) * a.N + idx] : 0.f;
      double rho0 = a.rho_in[idx];
      double U[3] = {(double)a.g_in[idx], (double)a.g_in[a.N + idx], (double)a.g_in[2 * a.N + idx]};
      double Tc = a.g_in[3 * a.N + idx];
      if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && Tc == 0) {  // set_base(1, TLat)
        rho0 = 1; Tc = L::TLat;
#pragma unroll
        for (int iy = 0; iy < 5; iy++) f0[iy] = worker ? R(lattice_weight_t<POND_D3Q125>(25 * j + 5 * iy + k)) : 0.f;
      }
      if (a.guess) {
        U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; Tc = a.guess[3 * a.N + idx];
      }
      const int qc = ((lz + HL) * SY + (ly + HL)) * SX + (lx + HXL);  // staged centre
      int niter = 0;
      bool conv = false;
      unsigned long long work = 0;
      while (niter < a.max_iter) {
        niter++;
        const double C = sqrt(Tc / L::TLat);
        // windows of this lane's classes (relative offsets) and their weights
        const double crdx = double(x) - (C * L::xi1(j) + U[0]);
        const double fxd = floor(crdx + 0.5);
        const double cdist = crdx - fxd;
        const int bx = w3d::clamp_off((int)fxd - 2 - x);
        R LX[3][3];
#pragma unroll
        for (int s = 0; s < 3; s++) lagr_weights<3, R>(crdx - (fxd - 2 + s), LX[s]);
        const double crdz = double(z) - (C * L::xi1(k) + U[2]);
        const double fzd = floor(crdz + 0.5) - 1;  // centred window: fz-1 .. fz+1
        const int bz = w3d::clamp_off((int)fzd - z);
        R WZ[3];
        lagr_weights<3, R>(crdz - fzd, WZ);
        int by[5];
        R WY[5][3];
#pragma unroll
        for (int i2 = 0; i2 < 5; i2++) {
          const double crdy = double(y) - (C * L::xi1(i2) + U[1]);
          const double fyd = floor(crdy + 0.5) - 1;
          by[i2] = w3d::clamp_off((int)fyd - y);
          lagr_weights<3, R>(crdy - fyd, WY[i2]);
        }
        bool inside = bx >= -HXL && bx + 4 <= HXH && bz >= -HL && bz + 2 <= HH;
#pragma unroll
        for (int i2 = 0; i2 < 5; i2++) inside = inside && by[i2] >= -HL && by[i2] + 2 <= HH;
        R S[3][5], U5[5][5];
        if (__all_sync(0xffffffffu, inside)) {
          // transfer R -> target per axis: G[i][k] = L_i(b + a xi_k), a = c_ref/C, b = (u_ref - U)/C
          const R ga = R(double(cref) / C);
          R gb[3];
#pragma unroll
          for (int ax = 0; ax < 3; ax++) gb[ax] = R((double(uref[ax]) - U[ax]) / C);
          R tz[5], tx[5];
          {
            const d125t::BasisRowT<R> Lj(j), Lk(k);
#pragma unroll
            for (int kk = 0; kk < 5; kk++) {
              tz[kk] = finite_or_zero_f(Lk(fmaf(ga, d125t::xi5r<R>(kk), gb[2])));
              tx[kk] = finite_or_zero_f(Lj(fmaf(ga, d125t::xi5r<R>(kk), gb[0])));
            }
          }
          // the warp's y tables: lane e = 5 i2 + k2 writes its entry for every stencil row oy
          __syncwarp();  // readers of the previous iteration are done
          if (worker) {
            const int i2 = lane / 5, k2 = lane % 5;
            const R gy = finite_or_zero_f(d125t::BasisRowT<R>(i2)(fmaf(ga, d125t::xi5r<R>(k2), gb[1])));
            int byi = by[0];
            R w0 = WY[0][0], w1 = WY[0][1], w2 = WY[0][2];
#pragma unroll
            for (int c = 1; c < 5; c++)
              if (i2 == c) { byi = by[c]; w0 = WY[c][0]; w1 = WY[c][1]; w2 = WY[c][2]; }
#pragma unroll
            for (int oyi = 0; oyi < 5; oyi++) {
              const int jy = oyi - HL - byi;
              sm.GY[warp][oyi][lane] = (jy == 0 ? w0 : jy == 1 ? w1 : jy == 2 ? w2 : 0.f) * gy;
            }
            sm.GD[warp][lane] = gy;
          }
          __syncwarp();
          // union of the windows over the worker lanes
          int ylo = by[0], yhi = by[0];
#pragma unroll
          for (int i2 = 1; i2 < 5; i2++) { ylo = min(ylo, by[i2]); yhi = max(yhi, by[i2]); }
          const int wxl = __reduce_min_sync(0xffffffffu, worker ? bx : HXH);
          const int wxh = __reduce_max_sync(0xffffffffu, worker ? bx + 4 : -HXL);
          const int wzl = __reduce_min_sync(0xffffffffu, worker ? bz : HH);
          const int wzh = __reduce_max_sync(0xffffffffu, worker ? bz + 2 : -HL);
          work += (unsigned long long)(wxh - wxl + 1) * (yhi - ylo + 3) * (wzh - wzl + 1);
#pragma unroll
          for (int s = 0; s < 3; s++)
#pragma unroll
            for (int i2 = 0; i2 < 5; i2++) S[s][i2] = 0.f;
#pragma unroll
          for (int m = 0; m < 5; m++)
#pragma unroll
            for (int i2 = 0; i2 < 5; i2++) U5[m][i2] = 0.f;
#pragma unroll 1
          for (int ox = wxl; ox <= wxh; ox++) {
            R Yr[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, Yd[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
            for (int oy = ylo; oy <= yhi + 2; oy++) {
              R Zc[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, Zd[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
              for (int oz = wzl; oz <= wzh; oz++) {
                const int jz = oz - bz;
                const R wz = jz == 0 ? WZ[0] : jz == 1 ? WZ[1] : jz == 2 ? WZ[2] : 0.f;
                const R* fq = sm.f + (25 * j) * PS + qc + oz * SX * SY + oy * SX + ox;
#pragma unroll
                for (int k2 = 0; k2 < 5; k2++) {
                  R zr = 0.f;
#pragma unroll
                  for (int k3 = 0; k3 < 5; k3++) zr = fmaf(tz[k3], fq[(5 * k2 + k3) * PS], zr);
                  Zc[k2] = fmaf(wz, zr, Zc[k2]);
                  Zd[k2] = jz == 1 ? zr : Zd[k2];
                }
              }
              const R* gy = sm.GY[warp][oy + HL];
              const R* gd = sm.GD[warp];
#pragma unroll
              for (int i2 = 0; i2 < 5; i2++) {
                R t = Yr[i2], td = 0.f;
#pragma unroll
                for (int k2 = 0; k2 < 5; k2++) {
                  t = fmaf(gy[5 * i2 + k2], Zc[k2], t);
                  td = fmaf(gd[5 * i2 + k2], Zd[k2], td);
                }
                Yr[i2] = t;
                Yd[i2] = oy == by[i2] + 1 ? td : Yd[i2];
              }
            }
            // the row: gather the five R x-classes of this lane's column
            const int jx = ox - bx;
            R lxs[3];
#pragma unroll
            for (int s = 0; s < 3; s++) {
              const int jj = jx - s;
              lxs[s] = jj == 0 ? LX[s][0] : jj == 1 ? LX[s][1] : jj == 2 ? LX[s][2] : 0.f;
            }
#pragma unroll
            for (int i2 = 0; i2 < 5; i2++) {
              R t = 0.f, td = 0.f;
#pragma unroll
              for (int k1 = 0; k1 < 5; k1++) {
                t = fmaf(tx[k1], __shfl_sync(0xffffffffu, Yr[i2], 5 * k1 + k), t);
                td = fmaf(tx[k1], __shfl_sync(0xffffffffu, Yd[i2], 5 * k1 + k), td);
              }
#pragma unroll
              for (int s = 0; s < 3; s++) S[s][i2] = fmaf(lxs[s], t, S[s][i2]);
#pragma unroll
              for (int m = 0; m < 5; m++) U5[m][i2] = jx == m ? td : U5[m][i2];
            }
          }
        } else {
          // a window leaves the staged halo: this iteration from global memory
          const R Uc[3] = {R(U[0]), R(U[1]), R(U[2])};
          w3d::accumulate_global<POND_D3Q125, R, true>(a, x, y, z, !worker, 0, j, k, Uc, R(1.0 / C), bx, LX, bz, WZ,
                                                       by, WY, S, U5, work, true);
        }
        // blend, calcMoments (structs.cuh:315-342) in float64, warp-wide
        R acc[5];
        double mv[5] = {0, 0, 0, 0, 0};
        const double vx = C * L::xi1(j) + U[0], vz = C * L::xi1(k) + U[2];
#pragma unroll
        for (int i2 = 0; i2 < 5; i2++) {
          const double Sd[3] = {double(S[0][i2]), double(S[1][i2]), double(S[2][i2])};
          const double ud[5] = {double(U5[0][i2]), double(U5[1][i2]), double(U5[2][i2]), double(U5[3][i2]),
                                double(U5[4][i2])};
          acc[i2] = (C >= 1.0e-300) ? R(w3d::weno5_blend(Sd, ud, cdist)) : 0.f;  // target T = 0: terms dropped
          if (worker) {
            const double fv = acc[i2], vy = C * L::xi1(i2) + U[1];
            mv[0] += fv; mv[1] += fv * vx; mv[2] += fv * vy; mv[3] += fv * vz;
            mv[4] += fv * (vx * vx + vy * vy + vz * vz);
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
          for (int q = 0; q < 5; q++) mv[q] += __shfl_xor_sync(0xffffffffu, mv[q], o);
        const double rho = mv[0];
        double m[4] = {mv[1], mv[2], mv[3], mv[4]};
        if (rho != 0) {
          const double ir = 1.0 / rho;
#pragma unroll
          for (int q = 0; q < 4; q++) m[q] *= ir;
        }
        double Tn = (m[3] - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) * (1.0 / L::Dim);
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
          }
        const bool all_ok = __all_sync(0xffffffffu, ok);
#pragma unroll
        for (int iy = 0; iy < 5; iy++) f0[iy] = acc[iy];
        rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; Tc = Tn;
        if (all_ok) { conv = true; break; }
      }
      // BGK toward rho*w_i (steps.cu:557-564) and store
      const R rr = R(rho0), dtau = R(a.dtau);
      if (worker)
#pragma unroll
        for (int iy = 0; iy < 5; iy++) {
          const int p = 25 * j + 5 * iy + k;
          a.f_out[(long long)p * a.N + idx] = f0[iy] + dtau * (rr * R(lattice_weight_t<POND_D3Q125>(p)) - f0[iy]);
        }
      if (lane == 0) {
        const R u0 = R(U[0]), u1 = R(U[1]), u2 = R(U[2]), ts = R(Tc);
        a.rho_out[idx] = rr;
        a.g_out[idx] = u0; a.g_out[a.N + idx] = u1; a.g_out[2 * a.N + idx] = u2; a.g_out[3 * a.N + idx] = ts;
        if (a.niter_out) a.niter_out[idx] = niter;
        const double dr = rr, d0 = u0, d1 = u1, d2 = u2, dt = ts;
        const double u2s = d0 * d0 + d1 * d1 + d2 * d2;
        ns.mass += dr; ns.m0 += dr * d0; ns.m1 += dr * d1; ns.m2 += dr * d2;
        ns.enrg += dr * (u2s + L::Dim * dt);
        ns.k += a.kdx * u2s;
        ns.niter += niter; ns.nonconv += conv ? 0 : 1; ns.nmax = max(ns.nmax, niter);
        ns.work += work;
      }
    }
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace d125w
}  // namespace pond
