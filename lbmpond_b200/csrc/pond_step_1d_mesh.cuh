// D1Q5 pull step on a one-dimensional mesh with a node mask (the reference's
// Cinfo::set) and, for the non-uniform scheme, node positions (Cell::p.x
// under NRMESH).  One thread per node, periodic in x, Ny = Nz = 1.
//
//  GAP2         steps.cu:1122-1149 propagate_nonequal_1D<2>: population i is
//               interpolated linearly at x - v_i between the nearest ACTIVE
//               nodes left and right of it, the shifts growing by one per
//               inactive node passed;
//  NONUNIFORM3  steps.cu:882-908 propagateNR_1D: quadratic Lagrange
//               interpolation (LagrPolNR_1D, :590-594) at p_x - v_i on the
//               positions of nodes x-1, x, x+1, abscissae relative to the
//               first node and lifted by Nx across the periodic seam.
//
// An inactive node is skipped by the reference's step (steps.cu:359) and left
// unwritten; here it is carried over unchanged so that the output buffer is
// always a complete state.  Each CTA takes a window of 128 consecutive nodes
// and hands its threads the window's active nodes first and then its inactive
// ones (each in node order), so a warp mostly either steps active nodes or
// copies inactive ones whatever the mask's pattern, and both halves of every
// 32-byte sector of the output are written by one CTA within microseconds
// (an L2 line that two far-apart launches half-write costs DRAM read-modify-
// write traffic).  The gauge iteration, moments, convergence test and BGK are
// those of the other kernels (moments_and_test / finish_node); the
// conservation sums cover active nodes, weighted under NONUNIFORM3 by half
// the distance between the node's neighbours (update.cu:52-69).
#pragma once
#include "pond_step_point.cuh"

namespace pond {

// Population k of the node at index n, transferred into the target gauge
// (Uc, C): the k-th row of the 5x5 Lagrange-basis matrix of the node.
template <typename R>
__device__ __forceinline__ R transfer_one_1d(const StepArgs<R>& a, int n, int k, R Uc, R invC) {
  using L = Lattice<POND_D1Q5>;
  const bool rv[3] = {false, false, false};
  const R Ucs[3] = {Uc, R(0), R(0)};
  R fn[5], s[3], r[3];
  load_node<POND_D1Q5, R>(a, n, rv, Ucs, invC, fn, s, r);
  R v = R(0);
#pragma unroll
  for (int b = 0; b < 5; b++) {
    R Lb[5];
    Basis<5, R>::eval(s[0] + r[0] * R(L::xi1(b)), Lb);
    R lk = Lb[0];
#pragma unroll
    for (int j = 1; j < 5; j++) lk = (j == k) ? Lb[j] : lk;
    v += finite_or_zero_f(lk) * fn[b];
  }
  return v;
}

__device__ __forceinline__ bool mesh_active(const uint8_t* mask, int n) { return mask == nullptr || mask[n] != 0; }

// periodic index of an integer-valued coordinate (a 64-bit remainder only
// for coordinates outside [-n, 2n), which no finite gauge of the step reaches
// in practice)
__device__ __forceinline__ int wrap_node(double fl, int n) {
  if (fl >= 0.0 && fl < double(n)) return int(fl);
  if (fl >= -double(n) && fl < 0.0) return int(fl) + n;
  if (fl >= double(n) && fl < 2.0 * double(n)) return int(fl) - n;
  long long q = (long long)fl % n;
  return int(q < 0 ? q + n : q);
}

template <int SCHEME, typename R>
__global__ void __launch_bounds__(128) pull_1d_mesh_kernel(StepArgs<R> a) {
  using L = Lattice<POND_D1Q5>;
  constexpr int Q = 5;
  // the window's nodes, active ones first (stable), then inactive ones
  __shared__ int wnode[128];
  __shared__ int wcount[2][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = blockIdx.x * 128 + threadIdx.x;
  bool act = false;
  {
    const bool mine = x < a.nx;
    const bool a_me = mine && mesh_active(a.mask, x);
    const unsigned ba = __ballot_sync(0xffffffffu, a_me), bi = __ballot_sync(0xffffffffu, mine && !a_me);
    if (lane == 0) { wcount[0][warp] = __popc(ba); wcount[1][warp] = __popc(bi); }
    __syncthreads();
    int na = 0, ni = 0, pa = 0, pi = 0;
#pragma unroll
    for (int w = 0; w < 4; w++) {
      if (w < warp) { pa += wcount[0][w]; pi += wcount[1][w]; }
      na += wcount[0][w]; ni += wcount[1][w];
    }
    const unsigned below = (1u << lane) - 1u;
    if (a_me) wnode[pa + __popc(ba & below)] = x;
    else if (mine) wnode[na + pi + __popc(bi & below)] = x;
    __syncthreads();
    act = (int)threadIdx.x < na;
    x = (int)threadIdx.x < na + ni ? wnode[threadIdx.x] : a.nx;
  }
  const int t = x;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (t < a.nx && !act) {
#pragma unroll
    for (int q = 0; q < Q; q++) a.f_out[(long long)q * a.N + x] = a.f_in[(long long)q * a.N + x];
    a.rho_out[x] = a.rho_in[x];
#pragma unroll
    for (int k = 0; k < 4; k++) a.g_out[(long long)k * a.N + x] = a.g_in[(long long)k * a.N + x];
    if (a.niter_out) a.niter_out[x] = 0;
  } else if (t < a.nx) {
    const int nx = a.nx;
    R f0[Q];
    double rho0, U[3], T;
    load_center<POND_D1Q5, R>(a, x, f0, rho0, U, T);
    // NONUNIFORM3: the three stencil nodes and their abscissae are fixed for the step
    const int first = x == 0 ? nx - 1 : x - 1;
    int nodes[3] = {first, x, x + 1 == nx ? 0 : x + 1};
    double bp[3] = {0, 0, 0}, p_first = 0, p_x = double(x);
    double inv[3][3];  // 1 / (bp[j] - bp[m]): the basis denominators, fixed for the step
    const double lift = double((-nx) / 2);  // -pars.Nx/2 with integer division
    if (SCHEME == POND_NONUNIFORM3) {
      p_first = a.pos ? a.pos[first] : double(first);
      p_x = a.pos ? a.pos[x] : double(x);
#pragma unroll
      for (int j = 0; j < 3; j++) {
        bp[j] = (a.pos ? a.pos[nodes[j]] : double(nodes[j])) - p_first;
        if (bp[j] < lift) bp[j] += nx;
      }
#pragma unroll
      for (int j = 0; j < 3; j++)
#pragma unroll
        for (int m = 0; m < 3; m++) inv[j][m] = m == j ? 0.0 : 1.0 / (bp[j] - bp[m]);
    }
    int niter = 0;
    bool conv = false;
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(T / L::TLat);
      const R Uc = R(U[0]);
      const R invC = R(1.0 / C);
      R acc[Q];
      if constexpr (SCHEME == POND_GAP2) {
#pragma unroll
        for (int k = 0; k < Q; k++) {
          const double crd = double(x) - (C * L::xi1(k) + U[0]);
          const double fl = floor(crd);
          int pl = wrap_node(fl, nx);
          int pr = pl + 1 == nx ? 0 : pl + 1;
          double sL = crd - fl, sR = (fl + 1) - crd;
          // each walk ends at the latest on node x, which is active
          for (int w = 0; w < nx && !mesh_active(a.mask, pl); w++) { pl = pl == 0 ? nx - 1 : pl - 1; sL += 1; }
          for (int w = 0; w < nx && !mesh_active(a.mask, pr); w++) { pr = pr + 1 == nx ? 0 : pr + 1; sR += 1; }
          const double isum = 1.0 / (sL + sR);
          const R wl = R(sR * isum), wr = R(sL * isum);
          acc[k] = wl * transfer_one_1d<R>(a, pl, k, Uc, invC) + wr * transfer_one_1d<R>(a, pr, k, Uc, invC);
        }
        ns.work += 2 * Q;
      } else {
        // each stencil node transferred once into the target gauge (all five rows)
        R gt[3][Q];
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const bool rv[3] = {false, false, false};
          const R Ucs[3] = {Uc, R(0), R(0)};
          R fn[Q], s[3], r[3];
          load_node<POND_D1Q5, R>(a, nodes[j], rv, Ucs, invC, fn, s, r);
          R Lm[Q][Q];
#pragma unroll
          for (int b = 0; b < Q; b++) Basis<5, R>::eval(s[0] + r[0] * R(L::xi1(b)), Lm[b]);
#pragma unroll
          for (int i = 0; i < Q; i++) {
            R g = R(0);
#pragma unroll
            for (int b = 0; b < Q; b++) g += finite_or_zero_f(Lm[b][i]) * fn[b];
            gt[j][i] = g;
          }
        }
#pragma unroll
        for (int k = 0; k < Q; k++) {
          const double crd = p_x - (C * L::xi1(k) + U[0]);
          double sh = crd - p_first;
          if (sh < lift) sh += nx;
          R v = R(0);
#pragma unroll
          for (int j = 0; j < 3; j++) {
            double wj = 1;
#pragma unroll
            for (int m = 0; m < 3; m++)
              if (m != j) wj *= (sh - bp[m]) * inv[j][m];
            v += R(wj) * gt[j][k];
          }
          acc[k] = v;
        }
        ns.work += 3;
      }
      if (moments_and_test<POND_D1Q5, R>(a, acc, f0, C, rho0, U, T)) { conv = true; break; }
    }
    finish_node<POND_D1Q5, R>(a, x, f0, rho0, U, T, niter, conv, ns);
    if (SCHEME == POND_NONUNIFORM3 && a.pos) {  // calcTotMoments' cell width (update.cu:59-62)
      const double pm = a.pos[first];
      double pp = a.pos[nodes[2]];
      if (pp < pm) pp += nx;
      const double dstep = 0.5 * (pp - pm);
      ns.mass *= dstep; ns.m0 *= dstep; ns.m1 *= dstep; ns.m2 *= dstep; ns.enrg *= dstep;
    }
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace pond
