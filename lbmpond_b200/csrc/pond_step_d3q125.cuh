// D3Q125 PonD pull step: one 128-thread CTA per node, quadratic stencil with
// its origin fixed at coord-1 (steps.cu:151-250 PonDstepD3Q125, launched by
// update.cu:98; the same arithmetic as LBMpull's D3Q125 branch :366-420).
//
// The reference gives each of its 125 threads one target population and
// evaluates a 125-term transfer_gauge for each of the 27 stencil nodes.  Here
// the 27 nodes are staged once per step in shared memory and every iteration
// applies the separable transform (three 5x5 passes per node, interpolation
// weights folded into the basis rows), so a step costs 3*27*125*5 multiply-
// adds per iteration instead of 27*125*125 transfer terms.
#pragma once
#include "pond_common.cuh"
#include "pond_step_point.cuh"

namespace pond {

constexpr int D125_THREADS = 128;

template <typename R> struct D125Smem {
  R f[27][125];      // staged stencil populations (non-finite zeroed)
  R t1[27][125];     // pass-z output [node][jx][jy][iz]
  R t2[27][125];     // pass-y output [node][jx][iy][iz]
  R M[27][3][5][5];  // weighted basis rows per node and axis: M[i][b]
  R un[27][3];       // stencil gauge velocities (sign-flipped on mirrored axes)
  R cn[27][3];       // sqrts(T/TLat) (sign-flipped on mirrored axes)
  double red[4][5];  // per-warp partial moment sums
};

template <typename R>
__global__ void __launch_bounds__(D125_THREADS) pull_d3q125_kernel(StepArgs<R> a) {
  using L = Lattice<POND_D3Q125>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  D125Smem<R>& S = *reinterpret_cast<D125Smem<R>*>(smem_raw);
  const int tid = threadIdx.x;
  const long long node = blockIdx.x;
  const int x = node % a.nx, y = (node / a.nx) % a.ny, z = node / ((long long)a.nx * a.ny);
  const long long idx = node;
  const bool own = tid < 125;

  // ---- stage the 3x3x3 stencil (steps.cu:164-193)
  for (int n = 0; n < 27; n++) {
    bool rv[3];
    const int px = resolve_axis(x - 1 + n / 9, a.nx, a.bc[0], rv[0]);
    const int py = resolve_axis(y - 1 + (n / 3) % 3, a.ny, a.bc[1], rv[1]);
    const int pz = resolve_axis(z - 1 + n % 3, a.nz, a.bc[2], rv[2]);
    const long long nidx = px + (long long)a.nx * (py + (long long)a.ny * pz);
    if (own) S.f[n][tid] = finite_or_zero_f(a.f_in[(long long)tid * a.N + nidx]);
    if (tid < 3) {
      const R u = a.g_in[(long long)tid * a.N + nidx];
      const R T = a.g_in[3 * a.N + nidx];
      const R c = copysign(sqrt(fabs(T) * R(1.0 / L::TLat)), T);
      S.un[n][tid] = rv[tid] ? -u : u;
      S.cn[n][tid] = rv[tid] ? -c : c;
    }
  }
  // ---- c0.load of the centre node (every thread keeps a copy of the gauge)
  R f0 = own ? a.f_in[(long long)tid * a.N + idx] : R(0);
  double rho0 = a.rho_in[idx];
  double U[3] = {(double)a.g_in[idx], (double)a.g_in[a.N + idx], (double)a.g_in[2 * a.N + idx]};
  double T = a.g_in[3 * a.N + idx];
  if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && T == 0) {
    rho0 = 1; T = L::TLat;
    f0 = own ? R(lattice_weight_t<POND_D3Q125>(tid)) : R(0);
  }
  if (a.guess) {
    U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; T = a.guess[3 * a.N + idx];
  }
  __syncthreads();
  const int pos[3] = {x, y, z};
  const int ix = tid / 25, iy = (tid / 5) % 5, iz = tid % 5;
  int niter = 0;
  bool conv = false;
  while (niter < a.max_iter) {
    niter++;
    const double C = sqrt(T / L::TLat);
    // basis rows with the quadratic interpolation weights of class i folded in
    if (tid < 81) {
      const int n = tid / 3, ax = tid % 3;
      const int na = ax == 0 ? n / 9 : ax == 1 ? (n / 3) % 3 : n % 3;  // stencil position on this axis
      const R invC = R(1.0 / C);
      const R s = (S.un[n][ax] - R(U[ax])) * invC;
      const R r = S.cn[n][ax] * invC;
      R Lb[5][5];
#pragma unroll
      for (int b = 0; b < 5; b++) Basis<5, R>::eval(s + r * R(L::xi1(b)), Lb[b]);
#pragma unroll
      for (int i = 0; i < 5; i++) {
        // LagrPol<3> factor of class i on this axis at shift = crd - (coord-1)
        const double crd = double(pos[ax]) - (C * L::xi1(i) + U[ax]);
        const double sh = crd - double(pos[ax] - 1);
        R w3[3];
        lagr_weights<3, R>(sh, w3);
        const R wi = na == 0 ? w3[0] : na == 1 ? w3[1] : w3[2];
#pragma unroll
        for (int b = 0; b < 5; b++) S.M[n][ax][i][b] = wi * finite_or_zero_f(Lb[b][i]);
      }
    }
    __syncthreads();
    // pass z: t1[n][jx][jy][iz] = sum_jz Mz[iz][jz] f[n][jx][jy][jz]
    for (int line = tid; line < 27 * 25; line += D125_THREADS) {
      const int n = line / 25, jxy = line % 25;
      R fin[5];
#pragma unroll
      for (int jz = 0; jz < 5; jz++) fin[jz] = S.f[n][jxy * 5 + jz];
#pragma unroll
      for (int oz = 0; oz < 5; oz++) {
        R t = R(0);
#pragma unroll
        for (int jz = 0; jz < 5; jz++) t += S.M[n][2][oz][jz] * fin[jz];
        S.t1[n][jxy * 5 + oz] = t;
      }
    }
    __syncthreads();
    // pass y: t2[n][jx][iy][iz] = sum_jy My[iy][jy] t1[n][jx][jy][iz]
    for (int line = tid; line < 27 * 25; line += D125_THREADS) {
      const int n = line / 25, jx = (line % 25) / 5, oz = line % 5;
      R tin[5];
#pragma unroll
      for (int jy = 0; jy < 5; jy++) tin[jy] = S.t1[n][jx * 25 + jy * 5 + oz];
#pragma unroll
      for (int oy = 0; oy < 5; oy++) {
        R t = R(0);
#pragma unroll
        for (int jy = 0; jy < 5; jy++) t += S.M[n][1][oy][jy] * tin[jy];
        S.t2[n][jx * 25 + oy * 5 + oz] = t;
      }
    }
    __syncthreads();
    // pass x and the sum over the 27 stencil nodes: population tid
    R fnew = R(0);
    if (own) {
      for (int n = 0; n < 27; n++) {
#pragma unroll
        for (int jx = 0; jx < 5; jx++) fnew += S.M[n][0][ix][jx] * S.t2[n][jx * 25 + iy * 5 + iz];
      }
    }
    // ---- calcMoments in float64 (thread 0's role in the reference)
    double mv[5] = {0, 0, 0, 0, 0};
    if (own) {
      const double fv = fnew;
      const double vx = C * L::xi1(ix) + U[0], vy = C * L::xi1(iy) + U[1], vz = C * L::xi1(iz) + U[2];
      mv[0] = fv; mv[1] = fv * vx; mv[2] = fv * vy; mv[3] = fv * vz; mv[4] = fv * (vx * vx + vy * vy + vz * vz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int q = 0; q < 5; q++) mv[q] += __shfl_xor_sync(0xffffffffu, mv[q], o);
    if ((tid & 31) == 0)
#pragma unroll
      for (int q = 0; q < 5; q++) S.red[tid >> 5][q] = mv[q];
    __syncthreads();
    double rho = 0, m[4] = {0, 0, 0, 0};
#pragma unroll
    for (int w = 0; w < 4; w++) {
      rho += S.red[w][0];
#pragma unroll
      for (int k = 0; k < 4; k++) m[k] += S.red[w][k + 1];
    }
    if (rho != 0)
#pragma unroll
      for (int k = 0; k < 4; k++) m[k] /= rho;
    double Tn = (m[3] - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) * (1.0 / L::Dim);
    if (Tn < 0) Tn = T;
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; k++) ok = ok && !(fabs(m[k] - U[k]) >= a.tol_abs + a.tol_rel * fabs(m[k]));
    ok = ok && !(fabs(Tn - T) >= a.tol_abs + a.tol_rel * fabs(Tn));
    if (own) {
      const double nv = fnew, ov = f0;
      ok = ok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
    }
    const bool all_ok = __syncthreads_and(ok);
    f0 = fnew;
    rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; T = Tn;
    if (all_ok) { conv = true; break; }
  }
  // ---- BGK and store (steps.cu:230-248)
  if (own) {
    const R feq = R(rho0) * R(lattice_weight_t<POND_D3Q125>(tid));
    f0 += R(a.dtau) * (feq - f0);
    a.f_out[(long long)tid * a.N + idx] = f0;
  }
  const R rs = R(rho0), u0 = R(U[0]), u1 = R(U[1]), u2 = R(U[2]), ts = R(T);
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (tid == 0) {
    a.rho_out[idx] = rs;
    a.g_out[idx] = u0; a.g_out[a.N + idx] = u1; a.g_out[2 * a.N + idx] = u2; a.g_out[3 * a.N + idx] = ts;
    if (a.niter_out) a.niter_out[idx] = niter;
    const double dr = rs, d0 = u0, d1 = u1, d2 = u2, dt = ts;
    const double u2s = d0 * d0 + d1 * d1 + d2 * d2;
    ns.mass = dr; ns.m0 = dr * d0; ns.m1 = dr * d1; ns.m2 = dr * d2;
    ns.enrg = dr * (u2s + L::Dim * dt);
    ns.k = a.kdx * u2s;
    ns.niter = niter; ns.nonconv = conv ? 0 : 1; ns.nmax = niter;
    ns.work = 27ull * niter;
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace pond
