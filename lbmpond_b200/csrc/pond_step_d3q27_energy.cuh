// D3Q27 pull step with the double-distribution extension (energy populations
// h beside f; gamma = (3 + dof + 2) / (3 + dof)), one thread per node, Lagrange
// interpolation of order N, float32 or float64 storage, float64 moments and
// tests.  The same completion of the reference's DDF scaffolding as the D1Q5
// kernel (pond_step_1d_energy.cuh): h is transferred and interpolated like f,
// the iterate's temperature is (sum h / rho - |u|^2) / (3 + dof), the
// convergence test covers every h, and h relaxes to rho w_i (|v_i|^2 + dof T).
//
// The arithmetic of f is that of pull_point_kernel (steps.cu:356-588 LBMpull
// with propagate<N>): per stencil node three 1D passes of the 3x3 basis with
// the interpolation weights folded into the rows, here applied to f and h.
// The node reads its stencil from global memory (L1/L2): the staged tile
// kernel of the plain step has no shared memory left for a second set of 27
// planes.
#pragma once
#include "pond_step_point.cuh"

namespace pond {

// acc[ix,iy,iz] += sum_j Mx[ix][jx] My[iy][jy] Mz[iz][jz] v[jx,jy,jz]
template <typename R>
__device__ __forceinline__ void transform_add3(const R v[27], const R Mx[3][3], const R My[3][3], const R Mz[3][3],
                                               R acc[27]) {
  R t1[3][3][3];
#pragma unroll
  for (int jx = 0; jx < 3; jx++)
#pragma unroll
    for (int jy = 0; jy < 3; jy++)
#pragma unroll
      for (int iz = 0; iz < 3; iz++) {
        R t = R(0);
#pragma unroll
        for (int jz = 0; jz < 3; jz++) t += Mz[iz][jz] * v[(jx * 3 + jy) * 3 + jz];
        t1[jx][jy][iz] = t;
      }
  R t2[3][3][3];
#pragma unroll
  for (int jx = 0; jx < 3; jx++)
#pragma unroll
    for (int iy = 0; iy < 3; iy++)
#pragma unroll
      for (int iz = 0; iz < 3; iz++) {
        R t = R(0);
#pragma unroll
        for (int jy = 0; jy < 3; jy++) t += My[iy][jy] * t1[jx][jy][iz];
        t2[jx][iy][iz] = t;
      }
#pragma unroll
  for (int ix = 0; ix < 3; ix++)
#pragma unroll
    for (int iy = 0; iy < 3; iy++)
#pragma unroll
      for (int iz = 0; iz < 3; iz++) {
        R t = acc[(ix * 3 + iy) * 3 + iz];
#pragma unroll
        for (int jx = 0; jx < 3; jx++) t += Mx[ix][jx] * t2[jx][iy][iz];
        acc[(ix * 3 + iy) * 3 + iz] = t;
      }
}

template <int N, typename R>
__global__ void __launch_bounds__(128) pull_d3q27_energy_kernel(StepArgs<R> a) {
  using L = Lattice<POND_D3Q27>;
  constexpr int Q = 27, Q1 = 3;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  const bool active = x < a.nx && y < a.ny && z < a.nz;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (active) {
    const long long idx = x + (long long)a.nx * (y + (long long)a.ny * z);
    R f0[Q], h0[Q];
    double rho0, U[3], T;
    load_center<POND_D3Q27, R>(a, idx, f0, rho0, U, T);
    const bool base = a.rho_in[idx] == R(0) && a.g_in[idx] == R(0) && a.g_in[a.N + idx] == R(0) &&
                      a.g_in[2 * a.N + idx] == R(0) && a.g_in[3 * a.N + idx] == R(0);
    if (base) energy_equilibrium<POND_D3Q27, R>(rho0, U, T, a.dof, h0);  // set_base(1, TLat) with its energy
    else
#pragma unroll
      for (int t = 0; t < Q; t++) h0[t] = a.h_in[(long long)L::ref(t / 9, (t / 3) % 3, t % 3) * a.N + idx];
    const int pos[3] = {x, y, z};
    const int dims[3] = {a.nx, a.ny, a.nz};
    int niter = 0;
    bool conv = false;
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(T / L::TLat);
      int org[3][Q1];
      R wt[3][Q1][N];
#pragma unroll
      for (int ax = 0; ax < 3; ax++)
#pragma unroll
        for (int c = 0; c < Q1; c++) {
          const double crd = double(pos[ax]) - (C * L::xi1(c) + U[ax]);
          org[ax][c] = window_origin<N>(crd, ax);
          const double sh = crd - double(org[ax][c]);
          if (N == 2) { wt[ax][c][0] = R(1 - sh); wt[ax][c][N - 1] = R(sh); }
          else lagr_weights<N, R>(sh, wt[ax][c]);
        }
      const R Uc[3] = {R(U[0]), R(U[1]), R(U[2])};
      const R invC = R(1.0 / C);
      R acc[Q], acch[Q];
#pragma unroll
      for (int t = 0; t < Q; t++) { acc[t] = R(0); acch[t] = R(0); }
      int lo[3], hi[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        lo[ax] = min(org[ax][0], min(org[ax][1], org[ax][2]));
        hi[ax] = max(org[ax][0], max(org[ax][1], org[ax][2])) + N - 1;
      }
      ns.work += (unsigned long long)window_positions<N, Q1>(org[0]) * window_positions<N, Q1>(org[1]) *
                 window_positions<N, Q1>(org[2]);
      for (int px = lo[0]; px <= hi[0]; px = window_next<N, Q1>(org[0], px)) {
        bool rv[3] = {false, false, false};
        const int rx = resolve_axis(px, dims[0], a.bc[0], rv[0]);
        R wx[Q1];
#pragma unroll
        for (int c = 0; c < Q1; c++) wx[c] = pick<N, R>(wt[0][c], org[0][c], px);
        for (int py = lo[1]; py <= hi[1]; py = window_next<N, Q1>(org[1], py)) {
          const int ry = resolve_axis(py, dims[1], a.bc[1], rv[1]);
          R wy[Q1];
#pragma unroll
          for (int c = 0; c < Q1; c++) wy[c] = pick<N, R>(wt[1][c], org[1][c], py);
          for (int pz = lo[2]; pz <= hi[2]; pz = window_next<N, Q1>(org[2], pz)) {
            const int rz = resolve_axis(pz, dims[2], a.bc[2], rv[2]);
            R wz[Q1];
#pragma unroll
            for (int c = 0; c < Q1; c++) wz[c] = pick<N, R>(wt[2][c], org[2][c], pz);
            const long long nidx = rx + (long long)a.nx * (ry + (long long)a.ny * rz);
            R fn[Q], s[3], r[3];
            load_node<POND_D3Q27, R>(a, nidx, rv, Uc, invC, fn, s, r);
            R hn[Q];
#pragma unroll
            for (int t = 0; t < Q; t++)
              hn[t] = finite_or_zero_f(__ldg(&a.h_in[(long long)L::ref(t / 9, (t / 3) % 3, t % 3) * a.N + nidx]));
            R Mx[Q1][Q1], My[Q1][Q1], Mz[Q1][Q1];  // M[i][b] = w_i * L_i(y_b)
#pragma unroll
            for (int b = 0; b < Q1; b++) {
              R lx[Q1], ly[Q1], lz[Q1];
              Basis<Q1, R>::eval(s[0] + r[0] * R(L::xi1(b)), lx);
              Basis<Q1, R>::eval(s[1] + r[1] * R(L::xi1(b)), ly);
              Basis<Q1, R>::eval(s[2] + r[2] * R(L::xi1(b)), lz);
#pragma unroll
              for (int i = 0; i < Q1; i++) {
                Mx[i][b] = wx[i] * finite_or_zero_f(lx[i]);
                My[i][b] = wy[i] * finite_or_zero_f(ly[i]);
                Mz[i][b] = wz[i] * finite_or_zero_f(lz[i]);
              }
            }
            transform_add3<R>(fn, Mx, My, Mz, acc);
            transform_add3<R>(hn, Mx, My, Mz, acch);
          }
        }
      }
      if (!(C >= 1.0e-300)) {  // target T = 0: every transfer term is non-finite and dropped
#pragma unroll
        for (int t = 0; t < Q; t++) { acc[t] = R(0); acch[t] = R(0); }
      }
      // calcMoments (structs.cuh:315-342) for rho and u, T from h, in float64
      double rho = 0, m[3] = {0, 0, 0}, esum = 0;
#pragma unroll
      for (int t = 0; t < Q; t++) {
        const double fv = acc[t];
        rho += fv;
        m[0] += fv * (C * L::xi1(t / 9) + U[0]);
        m[1] += fv * (C * L::xi1((t / 3) % 3) + U[1]);
        m[2] += fv * (C * L::xi1(t % 3) + U[2]);
        esum += double(acch[t]);
      }
      if (rho != 0) {
        const double ir = 1.0 / rho;
        m[0] *= ir; m[1] *= ir; m[2] *= ir; esum *= ir;
      }
      double Tn = (esum - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) / (L::Dim + a.dof);
      if (Tn < 0) Tn = T;  // steps.cu:475
      bool ok = !(fabs(Tn - T) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
#pragma unroll
      for (int k = 0; k < 3; k++) ok = ok && !(fabs(m[k] - U[k]) >= a.tolg_abs + a.tolg_rel * fabs(m[k]));
#pragma unroll
      for (int t = 0; t < Q; t++) {
        const double nf = acc[t], of = f0[t], nh = acch[t], oh = h0[t];
        ok = ok && !(fabs(nf - of) >= a.tol_abs + a.tol_rel * fabs(nf)) &&
             !(fabs(nh - oh) >= a.tol_abs + a.tol_rel * fabs(nh));
        f0[t] = acc[t];
        h0[t] = acch[t];
      }
      rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; T = Tn;
      if (ok) { conv = true; break; }
    }
    // h relaxes toward its equilibrium in the final gauge (the BGK of f in finish_node)
    R heq[Q];
    energy_equilibrium<POND_D3Q27, R>(double(R(rho0)), U, T, a.dof, heq);
    const R dtau = R(a.dtau);
#pragma unroll
    for (int t = 0; t < Q; t++)
      a.h_out[(long long)L::ref(t / 9, (t / 3) % 3, t % 3) * a.N + idx] = h0[t] + dtau * (heq[t] - h0[t]);
    finish_node<POND_D3Q27, R>(a, idx, f0, rho0, U, T, niter, conv, ns);
    const double dr = R(rho0), d0 = R(U[0]), d1 = R(U[1]), d2 = R(U[2]), dt = R(T);
    ns.enrg = dr * (d0 * d0 + d1 * d1 + d2 * d2 + (L::Dim + a.dof) * dt);
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace pond
