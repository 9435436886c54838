// D3Q27 pull step with energy populations (double-distribution extension,
// gamma = (3 + dof + 2) / (3 + dof)), float32, Lagrange order N = 2..4: the
// staged-tile form of pull_d3q27_energy_kernel (same arithmetic as the D1Q5
// and D3Q27 energy kernels: h is transferred and interpolated like f, the
// iterate's temperature is (sum h / rho - |u|^2) / (3 + dof), the convergence
// test covers every f and h, and h relaxes to rho w_i (|v_i|^2 + dof T)).
//
// Organised like the plain tile kernel (pond_step_d3q27.cuh), with two
// threads per node:
//
//  * a CTA owns an 8 x 4 x 4 tile (128 nodes) and stages it with its +-2 halo
//    (12 x 8 x 8 nodes) twice, node-major: the 27 f and the 27 h of a staged
//    node each contiguous at a 28-float stride (2 x 84 KB), transferred into
//    the reference gauge of the tile's centre node once per step;
//  * warps 0-3 iterate the f of the tile's nodes and warps 4-7 the h of the
//    same nodes in the same lane order (warp w and w + 4 form a pair).  Both
//    threads of a node evaluate the same target gauge, weights and
//    reference -> target transfer, and each contracts its own staged array.
//    Per iteration the f thread publishes rho and the momentum sums and the
//    verdict of its population test, the h thread the energy sum and its
//    verdict, through a per-pair slot in shared memory (double-buffered by
//    iteration parity, one 64-thread named barrier per iteration); both
//    threads then form the new gauge with the same float64 operations, so
//    the pair stays in lockstep and leaves the loop together;
//  * a lane whose departure points leave the halo runs that iteration from
//    global memory (f_in or h_in), transferring each stencil node itself.
// The node's previous iterate (f or h) lives in shared memory between
// iterations.
#pragma once
#include "pond_step_d3q27.cuh"

namespace pond {
namespace d27e {

using d27::basis_rows;
using d27::contract_x;
using d27::contract_y;
using d27::contract_z;
using d27::cp_async4;
using d27::cp_async_wait_all;
using d27::c_ref27;
using d27::node_to_ref;
using d27::rev3;
using d27::wpick;

constexpr int TX = 8, TY = 4, TZ = 4, H = 2;
constexpr int SX = TX + 2 * H, SY = TY + 2 * H, SZ = TZ + 2 * H;
constexpr int SN = SX * SY * SZ;  // 768 staged nodes
constexpr int NS = 28;            // floats per staged node and distribution (27 and a pad)
constexpr int NODES = TX * TY * TZ;
constexpr int THREADS = 2 * NODES;
// float offsets: staged f, staged h, the iterates (27 per thread), then the
// exchange slots (float64 [2][5][NODES], int [2][2][NODES])
constexpr int OFF_H = NS * SN;
constexpr int OFF_OWN = 2 * NS * SN;
constexpr int OFF_X = OFF_OWN + 27 * THREADS;
constexpr size_t SMEM_BYTES =
    size_t(OFF_X) * sizeof(float) + size_t(2 * 5 * NODES) * sizeof(double) + size_t(2 * 2 * NODES) * sizeof(int);
static_assert(OFF_X % 2 == 0, "the float64 exchange slots must be 8-byte aligned");
static_assert(SMEM_BYTES + 3 * 1024 <= 232448, "the tile must fit one CTA per SM");

__device__ __forceinline__ void pair_barrier(int pair) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(1 + pair), "r"(64) : "memory");
}

template <int N>
__global__ void __launch_bounds__(THREADS, 1) pull_d3q27_energy_tile_kernel(StepArgs<float> a) {
  using L = Lattice<POND_D3Q27>;
  extern __shared__ __align__(16) float sm[];
  const int tid = threadIdx.x;
  const int role = tid / NODES;  // 0: f, 1: h
  const int node = tid % NODES;
  const int pair = (tid >> 5) & 3;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;

  // ---- reference gauge of the CTA: the gauge of the tile's centre node
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

  // ---- stage f and h of every staged node, then transfer both into the
  //      reference gauge (boundary resolution, mirror reversal and the
  //      dropping of non-finite values as in the plain tile kernel)
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
      const long long src = (long long)c_ref27[cx * 9 + cy * 3 + cz] * a.N + g;
      cp_async4(&sm[i * NS + t], a.f_in + src);
      cp_async4(&sm[OFF_H + i * NS + t], a.h_in + src);
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
    const float r = ok ? c * icref : 0.f;
    const float sq[3] = {ok ? (u[0] - uref[0]) * icref : 0.f, ok ? (u[1] - uref[1]) * icref : 0.f,
                         ok ? (u[2] - uref[2]) * icref : 0.f};
    const float rq[3] = {r, r, r};
#pragma unroll 1
    for (int d = 0; d < 2; d++) {
      float* p = sm + d * OFF_H + i * NS;
      float v[27];
      {
        const float4* s4 = reinterpret_cast<const float4*>(p);
#pragma unroll
        for (int q = 0; q < 7; q++) {
          const float4 w = s4[q];
          const float e[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (4 * q + j < 27) v[4 * q + j] = (ok && fabsf(e[j]) <= 3.402823466e38f) ? e[j] : 0.f;
        }
      }
      node_to_ref(v, sq, rq);
      float4* s4 = reinterpret_cast<float4*>(p);
#pragma unroll
      for (int q = 0; q < 7; q++)
        s4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], 4 * q + 3 < 27 ? v[4 * q + 3] : 0.f);
    }
  }
  __syncthreads();

  const int lx = node % TX, ly = (node / TX) % TY, lz = node / (TX * TY);
  const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
  const bool active = x < a.nx && y < a.ny && z < a.nz;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  const long long idx = active ? x + (long long)a.nx * (y + (long long)a.ny * z) : 0;
  const float* sd = sm + role * OFF_H;       // this thread's staged distribution
  const float* gsrc = role ? a.h_in : a.f_in; // and its global copy
  float* own = sm + OFF_OWN + tid;            // the iterate of this thread's distribution
  double* xd = reinterpret_cast<double*>(sm + OFF_X);
  int* xf = reinterpret_cast<int*>(xd + 2 * 5 * NODES);
  double rho0 = 1, U[3] = {0, 0, 0}, T = L::TLat;
  {
    float f0[27];
    if (active) {
      load_center<POND_D3Q27, float>(a, idx, f0, rho0, U, T);
      if (role) {
        const bool base = a.rho_in[idx] == 0.f && a.g_in[idx] == 0.f && a.g_in[a.N + idx] == 0.f &&
                          a.g_in[2 * a.N + idx] == 0.f && a.g_in[3 * a.N + idx] == 0.f;
        if (base) energy_equilibrium<POND_D3Q27, float>(rho0, U, T, a.dof, f0);  // set_base with its energy
        else
#pragma unroll
          for (int t = 0; t < 27; t++) f0[t] = a.h_in[(long long)c_ref27[t] * a.N + idx];
      }
    } else {
#pragma unroll
      for (int t = 0; t < 27; t++) f0[t] = 0.f;
    }
#pragma unroll
    for (int t = 0; t < 27; t++) own[t * THREADS] = f0[t];
  }
  const int pos[3] = {x, y, z};
  const int sbase = (lz + H) * SX * SY + (ly + H) * SX + (lx + H);
  bool done = !active;
  bool conv = false;
  int niter = 0, it = 0;
  unsigned long long work = 0;
  while (__any_sync(0xffffffffu, !done)) {
    if (!done) niter++;
    const double C = sqrt(T * (1.0 / L::TLat));
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
    const float ainv = float(double(cref) / C);
    float bq[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) bq[ax] = float((double(uref[ax]) - U[ax]) / C);
    float Gz[3][3];
    basis_rows(bq[2], ainv, Gz);
    float acc[27];
#pragma unroll
    for (int t = 0; t < 27; t++) acc[t] = 0.f;
    const bool all3[3] = {true, true, true};
    const bool inside = lo[0] >= -H && lo[1] >= -H && lo[2] >= -H && hi[0] <= H && hi[1] <= H && hi[2] <= H;
    if (__all_sync(0xffffffffu, inside || done)) {
      int wl[3], wh[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        wl[ax] = __reduce_min_sync(0xffffffffu, done ? H : lo[ax]);
        wh[ax] = __reduce_max_sync(0xffffffffu, done ? -H : hi[ax]);
      }
      if (!done) {
        const unsigned long long ex = wh[0] - wl[0] + 1, ey = wh[1] - wl[1] + 1, ez = wh[2] - wl[2] + 1;
        work += ex * ey * ez * 171 + ex * ey * 171 + ex * 171;
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
            const float4* s4 = reinterpret_cast<const float4*>(sd + (sbase + oz * SX * SY + oy * SX + ox) * NS);
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
      // departure points beyond the staged halo: global memory, each stencil
      // node transferred into the reference gauge by this lane
      const unsigned long long ex = window_positions<N, 3>(ro[0]), ey = window_positions<N, 3>(ro[1]),
                               ez = window_positions<N, 3>(ro[2]);
      work += ex * ey * ez * 171 + ex * ey * 171 + ex * 171;
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
            for (int t = 0; t < 27; t++) v[t] = ok ? finite_or_zero_f(__ldg(&gsrc[(long long)c_ref27[t] * a.N + g])) : 0.f;
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
    // ---- moments of this thread's distribution and its population test,
    //      published to the partner thread of the node
    double* xs = xd + (it & 1) * 5 * NODES + node;
    int* xfl = xf + (it & 1) * 2 * NODES + node;
    if (!done) {
      if (!(C >= 1.0e-300)) {  // target T = 0: every transfer term is non-finite and dropped
#pragma unroll
        for (int t = 0; t < 27; t++) acc[t] = 0.f;
      }
      bool pok = true;
#pragma unroll
      for (int t = 0; t < 27; t++) {
        const double nv = acc[t], ov = own[t * THREADS];
        pok = pok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
        own[t * THREADS] = acc[t];
      }
      if (role == 0) {
        double rho = 0, m[3] = {0, 0, 0};
#pragma unroll
        for (int t = 0; t < 27; t++) {
          const double fv = acc[t];
          rho += fv;
          m[0] += fv * (C * L::xi1(t / 9) + U[0]);
          m[1] += fv * (C * L::xi1((t / 3) % 3) + U[1]);
          m[2] += fv * (C * L::xi1(t % 3) + U[2]);
        }
        xs[0] = rho; xs[NODES] = m[0]; xs[2 * NODES] = m[1]; xs[3 * NODES] = m[2];
      } else {
        double esum = 0;
#pragma unroll
        for (int t = 0; t < 27; t++) esum += double(acc[t]);
        xs[4 * NODES] = esum;
      }
      xfl[role * NODES] = pok ? 1 : 0;
    }
    pair_barrier(pair);
    if (!done) {
      // calcMoments (structs.cuh:315-342) with T from h, the T < 0 guard
      // (steps.cu:475) and isConv (steps.cu:58-75), in float64, identical in
      // both threads of the node
      const double rho = xs[0];
      double m[3] = {xs[NODES], xs[2 * NODES], xs[3 * NODES]}, esum = xs[4 * NODES];
      if (rho != 0) {
        const double ir = 1.0 / rho;
        m[0] *= ir; m[1] *= ir; m[2] *= ir; esum *= ir;
      }
      double Tn = (esum - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) / (L::Dim + a.dof);
      if (Tn < 0) Tn = T;
      bool ok = !(fabs(Tn - T) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
#pragma unroll
      for (int k = 0; k < 3; k++) ok = ok && !(fabs(m[k] - U[k]) >= a.tolg_abs + a.tolg_rel * fabs(m[k]));
      ok = ok && xfl[0] != 0 && xfl[NODES] != 0;
      rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; T = Tn;
      conv = ok;
      if (conv || niter >= a.max_iter) done = true;
    }
    it++;
  }
  if (active) {
    float f0[27];
#pragma unroll
    for (int t = 0; t < 27; t++) f0[t] = own[t * THREADS];
    if (role == 0) {
      finish_node<POND_D3Q27, float>(a, idx, f0, rho0, U, T, niter, conv, ns);
      const double dr = float(rho0), d0 = float(U[0]), d1 = float(U[1]), d2 = float(U[2]), dt = float(T);
      ns.enrg = dr * (d0 * d0 + d1 * d1 + d2 * d2 + (L::Dim + a.dof) * dt);
    } else {
      // h relaxes toward its equilibrium in the final gauge
      float heq[27];
      energy_equilibrium<POND_D3Q27, float>(double(float(rho0)), U, T, a.dof, heq);
      const float dtau = float(a.dtau);
#pragma unroll
      for (int t = 0; t < 27; t++) a.h_out[(long long)c_ref27[t] * a.N + idx] = f0[t] + dtau * (heq[t] - f0[t]);
    }
    ns.work = work;
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace d27e
}  // namespace pond
