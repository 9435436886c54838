// D1Q5 pull step with the double-distribution extension: a second set of
// populations h carries the total energy, so the gas has dof extra degrees
// of freedom and gamma = (Dim + dof + 2) / (Dim + dof) instead of 3.
//
// The reference has only non-compiling scaffolding for it (Cell::h,
// structs.cuh:37-39; T from sum h, :336-341; h transferred like f, :391-394;
// its set_base and BGK, lbpack.cu:18-20, steps.cu:233-236).  This kernel
// completes it:
//  * h is transferred to the iterate's gauge with the same 5x5 basis as f
//    and interpolated with the same scheme (Lagrange 2..5, TVD or WENO5,
//    as in pull_point_kernel and pull_1d_scheme_kernel);
//  * the iterate's temperature comes from h: T = (sum h / rho - |u|^2) /
//    (Dim + dof), with the reference's T < 0 guard (steps.cu:475);
//  * the convergence test covers u, T, every f and every h;
//  * h relaxes with the same rate as f to h_eq,i = rho w_i (|v_i|^2 + dof T),
//    v_i = U + C xi_i, whose zeroth moment is twice the total energy and whose
//    first moment is twice the enthalpy flux (the scaffolding's
//    rho w_i (Dim T + |u|^2) lacks the pressure work in the energy flux).
// One thread per node, float32 or float64 storage, float64 moments and tests.
#pragma once
#include "pond_step_1d.cuh"

namespace pond {

template <int SCHEME, typename R>
__global__ void __launch_bounds__(128) pull_1d_energy_kernel(StepArgs<R> a) {
  using L = Lattice<POND_D1Q5>;
  constexpr int Q = 5;
  constexpr bool kLagr = SCHEME >= POND_LAGR2 && SCHEME <= POND_LAGR5;
  constexpr int NL = kLagr ? SCHEME : 4;                                     // Lagrange order
  constexpr int NS = SCHEME == POND_TVD ? 4 : SCHEME == POND_WENO5 ? 5 : 1;  // slots per population
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = x < a.nx;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (active) {
    const long long idx = x;
    R f0[Q], h0[Q];
    double rho0, U[3], T;
    load_center<POND_D1Q5, R>(a, idx, f0, rho0, U, T);
    const bool base = a.rho_in[idx] == R(0) && a.g_in[idx] == R(0) && a.g_in[a.N + idx] == R(0) &&
                      a.g_in[2 * a.N + idx] == R(0) && a.g_in[3 * a.N + idx] == R(0);
    if (base) energy_equilibrium<POND_D1Q5, R>(rho0, U, T, a.dof, h0);  // set_base(1, TLat) with its energy
    else
#pragma unroll
      for (int k = 0; k < Q; k++) h0[k] = a.h_in[(long long)L::ref(k, 0, 0) * a.N + idx];
    int niter = 0;
    bool conv = false;
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(T / L::TLat);
      // per population: windows and weights (Lagrange: the departure point;
      // TVD: x-2v, x-v, x, x+v; WENO5: first node round(x-v)-2)
      int org[Q][NS];
      R wt[Q][NS][NL];
      int wb[Q];
      double vk[Q];
      int lo = 1 << 30, hi = -(1 << 30);
#pragma unroll
      for (int k = 0; k < Q; k++) {
        vk[k] = C * L::xi1(k) + U[0];
        if (kLagr) {
          const double crd = double(x) - vk[k];
          org[k][0] = window_origin<NL>(crd, 0);
          const double sh = crd - double(org[k][0]);
          if (NL == 2) { wt[k][0][0] = R(1 - sh); wt[k][0][NL - 1] = R(sh); }
          else lagr_weights<NL, R>(sh, wt[k][0]);
          lo = min(lo, org[k][0]);
          hi = max(hi, org[k][0] + NL - 1);
        } else if (SCHEME == POND_TVD) {
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
          wb[k] = (int)(floor(crd + 0.5) - 2);
          lo = min(lo, wb[k]);
          hi = max(hi, wb[k] + 4);
        }
      }
      const R Uc = R(U[0]);
      const R invC = R(1.0 / C);
      R accf[Q][NS], acch[Q][NS];
#pragma unroll
      for (int k = 0; k < Q; k++)
#pragma unroll
        for (int m = 0; m < NS; m++) { accf[k][m] = R(0); acch[k][m] = R(0); }
      ns.work += (unsigned long long)(hi - lo + 1);
      // the positions inside some window, in increasing order (gaps skipped)
      for (int p = lo; p <= hi;
           p = kLagr ? windows_next<Q, NL, NS>(&org[0][0], p)
                     : SCHEME == POND_TVD ? windows_next<Q * NS, 4, 1>(&org[0][0], p) : windows_next<Q, 5, 1>(wb, p)) {
        bool rv[3] = {false, false, false};
        const int rx = resolve_axis(p, a.nx, a.bc[0], rv[0]);
        R fn[Q], s[3], r[3];
        const R Ucs[3] = {Uc, R(0), R(0)};
        load_node<POND_D1Q5, R>(a, rx, rv, Ucs, invC, fn, s, r);
        R hn[Q];
#pragma unroll
        for (int c = 0; c < Q; c++) hn[c] = finite_or_zero_f(__ldg(&a.h_in[(long long)L::ref(c, 0, 0) * a.N + rx]));
        R Lm[Q][Q];
#pragma unroll
        for (int b = 0; b < Q; b++) Basis<5, R>::eval(s[0] + r[0] * R(L::xi1(b)), Lm[b]);
#pragma unroll
        for (int i = 0; i < Q; i++) {
          R gf = R(0), gh = R(0);
#pragma unroll
          for (int b = 0; b < Q; b++) {
            const R lb = finite_or_zero_f(Lm[b][i]);
            gf += lb * fn[b];
            gh += lb * hn[b];
          }
          if (kLagr) {
            const R w = pick<NL, R>(wt[i][0], org[i][0], p);
            accf[i][0] += w * gf;
            acch[i][0] += w * gh;
          } else if (SCHEME == POND_TVD) {
#pragma unroll
            for (int m = 0; m < NS; m++) {
              const R w = pick<4, R>(wt[i][m], org[i][m], p);
              accf[i][m] += w * gf;
              acch[i][m] += w * gh;
            }
          } else {
            const int j = p - wb[i];
#pragma unroll
            for (int m = 0; m < NS; m++) {
              accf[i][m] = (j == m) ? gf : accf[i][m];
              acch[i][m] = (j == m) ? gh : acch[i][m];
            }
          }
        }
      }
      // the scheme's combination of the slots, for f and for h alike
      R fnew[Q], hnew[Q];
#pragma unroll
      for (int e = 0; e < 2; e++)
#pragma unroll
        for (int k = 0; k < Q; k++) {
          const R* sl = e == 0 ? accf[k] : acch[k];
          double val;
          if constexpr (kLagr) {
            val = sl[0];
          } else if constexpr (SCHEME == POND_TVD) {
            val = tvd_combine(sl[0], sl[1], sl[2], sl[3], vk[k]);
          } else {
            const double uu[5] = {sl[0], sl[1], sl[2], sl[3], sl[4]};
            val = weno5_combine(uu, double(x) - vk[k]);
          }
          if (e == 0) fnew[k] = R(val); else hnew[k] = R(val);
        }
      // calcMoments (structs.cuh:315-342) for rho and u, T from h, in float64
      double rho = 0, m0 = 0, esum = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) {
        const double fv = fnew[k];
        rho += fv;
        m0 += fv * (C * L::xi1(k) + U[0]);
        esum += double(hnew[k]);
      }
      double m1 = rho * U[1], m2 = rho * U[2];
      if (rho != 0) {
        const double ir = 1.0 / rho;
        m0 *= ir; m1 *= ir; m2 *= ir; esum *= ir;
      }
      double Tn = (esum - m0 * m0 - m1 * m1 - m2 * m2) / (L::Dim + a.dof);
      if (Tn < 0) Tn = T;  // steps.cu:475
      bool ok = !(fabs(m0 - U[0]) >= a.tolg_abs + a.tolg_rel * fabs(m0)) &&
                !(fabs(m1 - U[1]) >= a.tolg_abs + a.tolg_rel * fabs(m1)) &&
                !(fabs(m2 - U[2]) >= a.tolg_abs + a.tolg_rel * fabs(m2)) &&
                !(fabs(Tn - T) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
#pragma unroll
      for (int k = 0; k < Q; k++) {
        const double nf = fnew[k], of = f0[k], nh = hnew[k], oh = h0[k];
        ok = ok && !(fabs(nf - of) >= a.tol_abs + a.tol_rel * fabs(nf)) &&
             !(fabs(nh - oh) >= a.tol_abs + a.tol_rel * fabs(nh));
        f0[k] = fnew[k];
        h0[k] = hnew[k];
      }
      rho0 = rho; U[0] = m0; U[1] = m1; U[2] = m2; T = Tn;
      if (ok) { conv = true; break; }
    }
    // h relaxes toward its equilibrium in the final gauge (the BGK of f in finish_node)
    R heq[Q];
    energy_equilibrium<POND_D1Q5, R>(double(R(rho0)), U, T, a.dof, heq);
    const R dtau = R(a.dtau);
#pragma unroll
    for (int k = 0; k < Q; k++) a.h_out[(long long)L::ref(k, 0, 0) * a.N + idx] = h0[k] + dtau * (heq[k] - h0[k]);
    finish_node<POND_D1Q5, R>(a, idx, f0, rho0, U, T, niter, conv, ns);
    // total energy with the extra degrees of freedom
    const double dr = R(rho0), d0 = R(U[0]), d1 = R(U[1]), d2 = R(U[2]), dt = R(T);
    ns.enrg = dr * (d0 * d0 + d1 * d1 + d2 * d2 + (L::Dim + a.dof) * dt);
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace pond
