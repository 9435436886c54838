// D1Q5 pull step with the reference's limited interpolations, one thread per
// node on 1D grids:
//
//  TVD   steps.cu:447 -- f_i = propagate<4>(x) - FluxTVDdif(x-2v, x-v, x, x+v)
//        with FluxTVDdif (steps.cu:118-124) built from minmod (:113-117):
//        four cubic evaluations per population plus a limited correction;
//  WENO5 steps.cu:774-825 propagateWENO<3,5> -- three quadratic candidates on
//        the five nodes round(x-v)-2 .. round(x-v)+2, Jiang-Shu smoothness
//        indicators of the transformed node values, eps = 1e-6.
//
// As in the point kernel, each stencil node is transformed once per
// iteration (5x5 Lagrange-basis matrix) and scattered into the slots of the
// populations that use it.  The nonlinear WENO/TVD combination is evaluated
// in float64 from the float32 (or float64) slot values.
#pragma once
#include "pond_step_point.cuh"

namespace pond {

__device__ __forceinline__ double minmod_d(double a, double b) {  // steps.cu:113-117
  if (a * b <= 0) return 0;
  if (fabs(a) < fabs(b)) return a;
  return b;
}

// steps.cu:447 with FluxTVDdif (:118-124): the cubic value at x minus the
// minmod-limited flux difference, from the slots F(x-2v), F(x-v), F(x), F(x+v)
__device__ __forceinline__ double tvd_combine(double Fm2, double Fm1, double F0, double Fp1, double v) {
  const int sg = (0.0 < v) - (v < 0.0);
  const double flux = F0 - Fm1 + sg * 0.5 * minmod_d(F0 - Fm1, Fp1 - F0) - sg * 0.5 * minmod_d(F0 - Fm1, Fm1 - Fm2);
  return F0 - flux;
}

// steps.cu:774-825 propagateWENO<3,5>: three quadratic candidates on the five
// transformed values u[0..4] at round(crd)-2 .. round(crd)+2, Jiang-Shu
// smoothness indicators, eps = 1e-6
__device__ __forceinline__ double weno5_combine(const double u[5], double crd) {
  const double u1 = u[0], u2 = u[1], u3 = u[2], u4 = u[3], u5 = u[4];
  const double fx = floor(crd + 0.5);
  double S[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {  // LagrEval<3> with origins fx-2, fx-1, fx
    double w3[3];
    lagr_weights<3, double>(crd - (fx - 2 + j), w3);
    S[j] = w3[0] * u[j] + w3[1] * u[j + 1] + w3[2] * u[j + 2];
  }
  const double cd = crd - (int)fx;
  const double d0 = (cd * cd - 3 * cd + 2) / 12.;
  const double d2 = (cd * cd + 3 * cd + 2) / 12.;
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

template <int SCHEME, typename R>
__global__ void __launch_bounds__(128) pull_1d_scheme_kernel(StepArgs<R> a) {
  using L = Lattice<POND_D1Q5>;
  constexpr int Q = 5;
  constexpr int NS = SCHEME == POND_TVD ? 4 : 5;  // slots per population
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = x < a.nx;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (active) {
    const long long idx = x;
    R f0[Q];
    double rho0, U[3], T;
    load_center<POND_D1Q5, R>(a, idx, f0, rho0, U, T);
    int niter = 0;
    bool conv = false;
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(T / L::TLat);
      // TVD: window origins/weights of the four evaluation points x-2v, x-v,
      // x, x+v (propagate<4>); WENO5: first node round(x-v)-2 of the 5 nodes
      int org[Q][NS];
      R wt[Q][NS][4];
      int base[Q];
      double vk[Q];
      int lo = 1 << 30, hi = -(1 << 30);
#pragma unroll
      for (int k = 0; k < Q; k++) {
        vk[k] = C * L::xi1(k) + U[0];
        if (SCHEME == POND_TVD) {
          const double mult[4] = {-2.0, -1.0, 0.0, 1.0};
#pragma unroll
          for (int m = 0; m < 4; m++) {
            const double crd = double(x) + vk[k] * mult[m];
            org[k][m] = window_origin<4>(crd, 0);
            lagr_weights<4, R>(crd - double(org[k][m]), wt[k][m]);
            lo = min(lo, org[k][m]);
            hi = max(hi, org[k][m] + 3);
          }
        } else {
          const double crd = held_coordinate(double(x) - vk[k]);
          base[k] = (int)(floor(crd + 0.5) - 2);
          lo = min(lo, base[k]);
          hi = max(hi, base[k] + 4);
        }
      }
      const R Uc = R(U[0]);
      const R invC = R(1.0 / C);
      R acc[Q][NS];
#pragma unroll
      for (int k = 0; k < Q; k++)
#pragma unroll
        for (int m = 0; m < NS; m++) acc[k][m] = R(0);
      ns.work += (unsigned long long)(hi - lo + 1);
      // the positions inside some window, in increasing order (gaps skipped)
      for (int p = lo; p <= hi;
           p = SCHEME == POND_TVD ? windows_next<Q * NS, 4, 1>(&org[0][0], p) : windows_next<Q, 5, 1>(base, p)) {
        bool rv[3] = {false, false, false};
        const int rx = resolve_axis(p, a.nx, a.bc[0], rv[0]);
        R fn[Q], s[3], r[3];
        const R Ucs[3] = {Uc, R(0), R(0)};
        load_node<POND_D1Q5, R>(a, rx, rv, Ucs, invC, fn, s, r);
        R Lm[Q][Q];
#pragma unroll
        for (int b = 0; b < Q; b++) Basis<5, R>::eval(s[0] + r[0] * R(L::xi1(b)), Lm[b]);
#pragma unroll
        for (int i = 0; i < Q; i++) {
          R g = R(0);
#pragma unroll
          for (int b = 0; b < Q; b++) g += finite_or_zero_f(Lm[b][i]) * fn[b];
          if (SCHEME == POND_TVD) {
#pragma unroll
            for (int m = 0; m < 4; m++) acc[i][m] += pick<4, R>(wt[i][m], org[i][m], p) * g;
          } else {
            const int j = p - base[i];
#pragma unroll
            for (int m = 0; m < 5; m++) acc[i][m] = (j == m) ? g : acc[i][m];
          }
        }
      }
      R fnew[Q];
#pragma unroll
      for (int k = 0; k < Q; k++) {
        if constexpr (SCHEME == POND_TVD) {
          fnew[k] = R(tvd_combine(acc[k][0], acc[k][1], acc[k][2], acc[k][3], vk[k]));
        } else {
          const double uu[5] = {acc[k][0], acc[k][1], acc[k][2], acc[k][3], acc[k][4]};
          fnew[k] = R(weno5_combine(uu, double(x) - vk[k]));
        }
      }
      if (moments_and_test<POND_D1Q5, R>(a, fnew, f0, C, rho0, U, T)) { conv = true; break; }
    }
    finish_node<POND_D1Q5, R>(a, idx, f0, rho0, U, T, niter, conv, ns);
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace pond
