// One-thread-per-node PonD pull step for the D1Q5 and D3Q27 lattices.
//
// Restates steps.cu:356-588 (LBMpull) with propagate<N> (steps.cu:986-1036),
// and for 1D grids also the TVD (steps.cu:118-124, call :447) and WENO5
// (steps.cu:774-825) variants.  The arithmetic is reorganised for the GPU:
//
//  * the gauge transform of a stencil node (structs.cuh:343-551, one Q-term
//    sum per (node, population) pair) is applied as three 1D passes of the
//    per-axis Lagrange-basis matrix, because every lattice here is a tensor
//    product (D3Q27 = D1Q3^3): 3*Q*Q1 multiply-adds per node instead of Q*Q;
//  * each stencil node is transformed once per iteration and scattered, with
//    its Lagrange interpolation weights folded into the basis rows, into the
//    accumulators of every population whose stencil contains it;
//  * non-finite terms are dropped as in the reference (:390,:516,:542) by
//    zeroing non-finite populations and basis entries before the passes.
//
// The conserved-moment sums (Cell::calcMoments, structs.cuh:315-342) and the
// convergence test (isConv, steps.cu:58-75) are evaluated in float64.
#pragma once
#include "pond_common.cuh"

namespace pond {

__device__ __forceinline__ float finite_or_zero_f(float v) { return fabsf(v) <= 3.402823466e38f ? v : 0.f; }
__device__ __forceinline__ double finite_or_zero_f(double v) { return fabs(v) <= 1.7976931348623157e308 ? v : 0.0; }

// Lagrange interpolation weights on N nodes at offset s from the first node
// (steps.cu:595-601 LagrPol per axis, :602-608 LinPol for N = 2).  The node
// spacings j - p are compile-time constants, so each factor multiplies by a
// folded reciprocal instead of dividing (within one float64 ulp of the
// quotient; a float64 division is a long instruction sequence).
template <int N, typename R> __device__ __forceinline__ void lagr_weights(double s, R w[N]) {
#pragma unroll
  for (int j = 0; j < N; j++) {
    double a = 1.0;
#pragma unroll
    for (int p = 0; p < N; p++)
      if (p != j) a *= (s - p) * (1.0 / double(j - p));
    w[j] = R(a);
  }
}

// Window origin of propagate<N> along one axis (steps.cu:996-997: even N use
// floor(c)-N/2+1; odd N use floor(c+0.5)-(N-1)/2 in x and floor(c)-(N-1)/2
// in y and z).
// A coordinate beyond +-2^29 (a diverged gauge) is held there, so origins,
// offsets and the positions built from them stay inside int; a NaN stays NaN.
template <int N> __device__ __forceinline__ int window_origin(double c, int axis) {
  if (fabs(c) > 536870912.0) c = copysign(536870912.0, c);
  if (N % 2 == 0) return (int)(floor(c) - N / 2 + 1);
  if (axis == 0) return (int)(floor(c + 0.5) - (N - 1) / 2);
  return (int)(floor(c) - (N - 1) / 2);
}

// The stencil positions of one axis are the union of the Q1 class windows
// [org[c], org[c] + N), walked in increasing order from the lowest origin:
// the position after p is p + 1 when a window holds it, else the next origin
// above p (INT_MAX past the last window).  The walk visits at most Q1 N
// positions however far a hot or fast node's gauge spreads the windows,
// where a sweep over every position between the lowest and the highest
// window would grow with the spread.
template <int N, int Q1> __device__ __forceinline__ int window_next(const int org[Q1], int p) {
  const int q = p + 1;
  bool in = false;
  int nxt = 0x7fffffff;
#pragma unroll
  for (int c = 0; c < Q1; c++) {
    in = in || (q - org[c] >= 0 && q - org[c] < N);
    nxt = org[c] > p ? min(nxt, org[c]) : nxt;
  }
  return in ? q : nxt;
}
// The same walk over NW windows of LEN positions whose starts lie STRIDE
// ints apart (the 1D schemes' per-population windows).
template <int NW, int LEN, int STRIDE> __device__ __forceinline__ int windows_next(const int* start, int p) {
  const int q = p + 1;
  bool in = false;
  int nxt = 0x7fffffff;
#pragma unroll
  for (int w = 0; w < NW; w++) {
    const int st = start[w * STRIDE];
    in = in || (q - st >= 0 && q - st < LEN);
    nxt = st > p ? min(nxt, st) : nxt;
  }
  return in ? q : nxt;
}
// a departure coordinate held within +-2^29 (a NaN stays NaN), for windows
// placed without window_origin
__device__ __forceinline__ double held_coordinate(double c) {
  return fabs(c) > 536870912.0 ? copysign(536870912.0, c) : c;
}

// number of positions the walk visits
template <int N, int Q1> __device__ __forceinline__ int window_positions(const int org[Q1]) {
  int n = 0;
#pragma unroll
  for (int k = 0; k < Q1 * N; k++) {
    const int c = k / N, p = org[c] + k % N;
    bool seen = false;
#pragma unroll
    for (int c2 = 0; c2 < c; c2++) seen = seen || (p - org[c2] >= 0 && p - org[c2] < N);
    n += seen ? 0 : 1;
  }
  return n;
}

// weight of window position j for a node at coordinate p (0 outside the window)
template <int N, typename R> __device__ __forceinline__ R pick(const R w[N], int org, int p) {
  const int j = p - org;
  R r = R(0);
#pragma unroll
  for (int k = 0; k < N; k++) r = (j == k) ? w[k] : r;
  return r;
}

// Block-wide float64/int64 reduction of the per-node diagnostics into the
// context's StepSums (one atomic per block and quantity).
struct NodeSums {
  double mass, m0, m1, m2, enrg, k;
  unsigned long long niter, nonconv, work;
  int nmax;
};
__device__ __forceinline__ void reduce_and_commit(NodeSums s, StepSums* out) {
  __shared__ double sd[6][32];
  __shared__ unsigned long long su[3][32];
  __shared__ int si[32];
  const int lane = threadIdx.x & 31;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int warp = tid >> 5;
  const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  double v[6] = {s.mass, s.m0, s.m1, s.m2, s.enrg, s.k};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 6; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    s.niter += __shfl_xor_sync(0xffffffffu, s.niter, o);
    s.nonconv += __shfl_xor_sync(0xffffffffu, s.nonconv, o);
    s.work += __shfl_xor_sync(0xffffffffu, s.work, o);
    s.nmax = max(s.nmax, __shfl_xor_sync(0xffffffffu, s.nmax, o));
  }
  if ((tid & 31) == 0) {
    for (int q = 0; q < 6; q++) sd[q][warp] = v[q];
    su[0][warp] = s.niter; su[1][warp] = s.nonconv; su[2][warp] = s.work; si[warp] = s.nmax;
  }
  __syncthreads();
  if (tid == 0) {
    double t[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long a = 0, b = 0, c = 0;
    int m = 0;
    for (int w = 0; w < nwarps; w++) {
      for (int q = 0; q < 6; q++) t[q] += sd[q][w];
      a += su[0][w]; b += su[1][w]; c += su[2][w]; m = max(m, si[w]);
    }
    atomicAdd(&out->mass, t[0]);
    atomicAdd(&out->mom[0], t[1]);
    atomicAdd(&out->mom[1], t[2]);
    atomicAdd(&out->mom[2], t[3]);
    atomicAdd(&out->enrg, t[4]);
    atomicAdd(&out->k, t[5]);
    atomicAdd(&out->niter_sum, a);
    atomicAdd(&out->nonconv, b);
    if (c) atomicAdd(&out->work, c);
    atomicMax(&out->niter_max, m);
  }
  (void)lane;
}

// Load one stencil node: populations in tensor-class order with non-finite
// values zeroed, and the per-axis transform parameters s = (u_n - U)/C and
// r = c_n / C (negated on a mirrored axis, which reverses the populations
// along that axis and flips u_n there: structs.cuh:552-578).
template <int LAT, typename R>
__device__ __forceinline__ void load_node(const StepArgs<R>& a, long long idx, const bool rev[3], const R Uc[3],
                                          R invC, R fn[Lattice<LAT>::Q], R s[3], R r[3]) {
  using L = Lattice<LAT>;
  constexpr int Q1 = L::Q1;
  if (L::D == 1) {
#pragma unroll
    for (int c = 0; c < Q1; c++) fn[c] = finite_or_zero_f(__ldg(&a.f_in[(long long)L::ref(c, 0, 0) * a.N + idx]));
  } else {
#pragma unroll
    for (int cx = 0; cx < Q1; cx++)
#pragma unroll
      for (int cy = 0; cy < Q1; cy++)
#pragma unroll
        for (int cz = 0; cz < Q1; cz++)
          fn[(cx * Q1 + cy) * Q1 + cz] =
              finite_or_zero_f(__ldg(&a.f_in[(long long)L::ref(cx, cy, cz) * a.N + idx]));
  }
  const R Tn = __ldg(&a.g_in[3 * a.N + idx]);
  // sqrts(T/TLat) of params.h:110 (sign-preserving square root)
  const R cn = copysign(sqrt(fabs(Tn) * R(1.0 / L::TLat)), Tn);
#pragma unroll
  for (int ax = 0; ax < L::D; ax++) {
    const R un = __ldg(&a.g_in[(long long)ax * a.N + idx]);
    s[ax] = ((rev[ax] ? -un : un) - Uc[ax]) * invC;
    r[ax] = (rev[ax] ? -cn : cn) * invC;
  }
}

// c0.load of the centre node (steps.cu:360-363) into tensor-class order, with
// the reference's set_base(1, TLat) for an all-zero record and the optional
// predicted starting gauge of the learned path.
template <int LAT, typename R>
__device__ __forceinline__ void load_center(const StepArgs<R>& a, long long idx, R f0[Lattice<LAT>::Q],
                                            double& rho0, double U[3], double& T) {
  using L = Lattice<LAT>;
  constexpr int Q = L::Q, Q1 = L::Q1;
  if (L::D == 1) {
#pragma unroll
    for (int c = 0; c < Q1; c++) f0[c] = a.f_in[(long long)L::ref(c, 0, 0) * a.N + idx];
  } else {
#pragma unroll
    for (int cx = 0; cx < Q1; cx++)
#pragma unroll
      for (int cy = 0; cy < Q1; cy++)
#pragma unroll
        for (int cz = 0; cz < Q1; cz++)
          f0[(cx * Q1 + cy) * Q1 + cz] = a.f_in[(long long)L::ref(cx, cy, cz) * a.N + idx];
  }
  rho0 = a.rho_in[idx];
  U[0] = a.g_in[idx]; U[1] = a.g_in[a.N + idx]; U[2] = a.g_in[2 * a.N + idx];
  T = a.g_in[3 * a.N + idx];
  if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && T == 0) {
    rho0 = 1; T = L::TLat;
#pragma unroll
    for (int t = 0; t < Q; t++) f0[t] = R(lattice_weight_t<LAT>(t));
  }
  if (a.guess) {
    U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; T = a.guess[3 * a.N + idx];
  }
}

// cnew.calcMoments(vi) (structs.cuh:315-342), the T < 0 guard (steps.cu:475)
// and isConv (steps.cu:58-75), all in float64; then c0 = cnew.
// Returns true when the iteration has converged.
template <int LAT, typename R>
__device__ __forceinline__ bool moments_and_test(const StepArgs<R>& a, const R acc[Lattice<LAT>::Q],
                                                 R f0[Lattice<LAT>::Q], double C, double& rho0, double U[3],
                                                 double& T) {
  using L = Lattice<LAT>;
  constexpr int Q = L::Q, Q1 = L::Q1;
  double m[4] = {0, 0, 0, 0}, rho = 0;
  if (L::D == 1) {
#pragma unroll
    for (int c = 0; c < Q1; c++) {
      const double fv = acc[c];
      const double vx = C * L::xi1(c) + U[0];
      rho += fv;
      m[0] += fv * vx; m[1] += fv * U[1]; m[2] += fv * U[2];
      m[3] += fv * (vx * vx + U[1] * U[1] + U[2] * U[2]);
    }
  } else {
#pragma unroll
    for (int cx = 0; cx < Q1; cx++)
#pragma unroll
      for (int cy = 0; cy < Q1; cy++)
#pragma unroll
        for (int cz = 0; cz < Q1; cz++) {
          const double fv = acc[(cx * Q1 + cy) * Q1 + cz];
          const double vx = C * L::xi1(cx) + U[0], vy = C * L::xi1(cy) + U[1], vz = C * L::xi1(cz) + U[2];
          rho += fv;
          m[0] += fv * vx; m[1] += fv * vy; m[2] += fv * vz;
          m[3] += fv * (vx * vx + vy * vy + vz * vz);
        }
  }
  if (rho != 0) {
    const double ir = 1.0 / rho;
#pragma unroll
    for (int k = 0; k < 4; k++) m[k] *= ir;
  }
  double Tn = (m[3] - m[0] * m[0] - m[1] * m[1] - m[2] * m[2]) * (1.0 / L::Dim);
  if (Tn < 0) Tn = T;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; k++) ok = ok && !(fabs(m[k] - U[k]) >= a.tolg_abs + a.tolg_rel * fabs(m[k]));
  ok = ok && !(fabs(Tn - T) >= a.tolg_abs + a.tolg_rel * fabs(Tn));
#pragma unroll
  for (int t = 0; t < Q; t++) {
    const double nv = acc[t], ov = f0[t];
    ok = ok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
  }
#pragma unroll
  for (int t = 0; t < Q; t++) f0[t] = acc[t];
  rho0 = rho; U[0] = m[0]; U[1] = m[1]; U[2] = m[2]; T = Tn;
  return ok;
}

// BGK toward rho*w_i in the co-moving gauge (steps.cu:557-564), c0.save
// (:582) and the node's share of the conservation sums (:583-585).
template <int LAT, typename R>
__device__ __forceinline__ void finish_node(const StepArgs<R>& a, long long idx, R f0[Lattice<LAT>::Q],
                                            double rho0, const double U[3], double T, int niter, bool conv,
                                            NodeSums& ns) {
  using L = Lattice<LAT>;
  constexpr int Q = L::Q, Q1 = L::Q1;
  const R dtau = R(a.dtau);
  const R rr = R(rho0);
#pragma unroll
  for (int t = 0; t < Q; t++) {
    const R feq = rr * R(lattice_weight_t<LAT>(t));
    f0[t] += dtau * (feq - f0[t]);
  }
  if (L::D == 1) {
#pragma unroll
    for (int c = 0; c < Q1; c++) a.f_out[(long long)L::ref(c, 0, 0) * a.N + idx] = f0[c];
  } else {
#pragma unroll
    for (int cx = 0; cx < Q1; cx++)
#pragma unroll
      for (int cy = 0; cy < Q1; cy++)
#pragma unroll
        for (int cz = 0; cz < Q1; cz++)
          a.f_out[(long long)L::ref(cx, cy, cz) * a.N + idx] = f0[(cx * Q1 + cy) * Q1 + cz];
  }
  const R rs = R(rho0), u0 = R(U[0]), u1 = R(U[1]), u2 = R(U[2]), ts = R(T);
  a.rho_out[idx] = rs;
  a.g_out[idx] = u0; a.g_out[a.N + idx] = u1; a.g_out[2 * a.N + idx] = u2; a.g_out[3 * a.N + idx] = ts;
  if (a.niter_out) a.niter_out[idx] = niter;
  const double dr = rs, d0 = u0, d1 = u1, d2 = u2, dt = ts;
  const double u2s = d0 * d0 + d1 * d1 + d2 * d2;
  ns.mass = dr; ns.m0 = dr * d0; ns.m1 = dr * d1; ns.m2 = dr * d2;
  ns.enrg = dr * (u2s + L::Dim * dt);
  ns.k = a.kdx * u2s;
  ns.niter = niter; ns.nonconv = conv ? 0 : 1; ns.nmax = niter;
}

// One pull step, one thread per node, D1Q5 (1D lines) or D3Q27, Lagrange
// interpolation of order N (steps.cu:986 propagate<N>).
template <int LAT, int N, typename R>
__global__ void __launch_bounds__(128) pull_point_kernel(StepArgs<R> a) {
  using L = Lattice<LAT>;
  constexpr int Q = L::Q, Q1 = L::Q1, D = L::D;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  const bool active = x < a.nx && y < a.ny && z < a.nz;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (active) {
    const long long idx = x + (long long)a.nx * (y + (long long)a.ny * z);
    R f0[Q];
    double rho0, U[3], T;
    load_center<LAT, R>(a, idx, f0, rho0, U, T);
    const int pos[3] = {x, y, z};
    const int dims[3] = {a.nx, a.ny, a.nz};
    int niter = 0;
    bool conv = false;
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(T / L::TLat);
      // departure windows and interpolation weights per axis and class
      int org[3][Q1];
      R wt[3][Q1][N];
#pragma unroll
      for (int ax = 0; ax < D; ax++)
#pragma unroll
        for (int c = 0; c < Q1; c++) {
          const double v = C * (D == 1 && ax > 0 ? 0.0 : L::xi1(c)) + U[ax];
          const double crd = double(pos[ax]) - v;
          org[ax][c] = window_origin<N>(crd, ax);
          const double sh = crd - double(org[ax][c]);
          if (N == 2) {  // LinPol
            wt[ax][c][0] = R(1 - sh);
            wt[ax][c][N - 1] = R(sh);
          } else {
            lagr_weights<N, R>(sh, wt[ax][c]);
          }
        }
      const R Uc[3] = {R(U[0]), R(U[1]), R(U[2])};
      const R invC = R(1.0 / C);
      R acc[Q];
#pragma unroll
      for (int t = 0; t < Q; t++) acc[t] = R(0);

      int lo[3], hi[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        if (ax < D) {
          lo[ax] = org[ax][0]; hi[ax] = org[ax][0];
#pragma unroll
          for (int c = 1; c < Q1; c++) { lo[ax] = min(lo[ax], org[ax][c]); hi[ax] = max(hi[ax], org[ax][c]); }
          hi[ax] += N - 1;
        } else {
          lo[ax] = hi[ax] = pos[ax];
        }
      }
      ns.work += (unsigned long long)window_positions<N, Q1>(org[0]) *
                 (D == 3 ? window_positions<N, Q1>(org[1]) * window_positions<N, Q1>(org[2]) : 1);
      for (int px = lo[0]; px <= hi[0]; px = window_next<N, Q1>(org[0], px)) {
        bool rv[3] = {false, false, false};
        const int rx = resolve_axis((int)px, dims[0], a.bc[0], rv[0]);
        R wx[Q1];
#pragma unroll
        for (int c = 0; c < Q1; c++) wx[c] = pick<N, R>(wt[0][c], org[0][c], px);
        for (int py = lo[1]; py <= hi[1]; py = D == 3 ? window_next<N, Q1>(org[1], py) : py + 1) {
          const int ry = (D == 3) ? resolve_axis((int)py, dims[1], a.bc[1], rv[1]) : (int)py;
          R wy[Q1];
          if (D == 3) {
#pragma unroll
            for (int c = 0; c < Q1; c++) wy[c] = pick<N, R>(wt[1][c], org[1][c], py);
          }
          for (int pz = lo[2]; pz <= hi[2]; pz = D == 3 ? window_next<N, Q1>(org[2], pz) : pz + 1) {
            const int rz = (D == 3) ? resolve_axis((int)pz, dims[2], a.bc[2], rv[2]) : (int)pz;
            const long long nidx = rx + (long long)a.nx * (ry + (long long)a.ny * rz);
            R fn[Q], s[3], r[3];
            load_node<LAT, R>(a, nidx, rv, Uc, invC, fn, s, r);
            if (D == 1) {
              R Lm[Q1][Q1];  // Lm[b][i] = L_i(y_b)
#pragma unroll
              for (int b = 0; b < Q1; b++) Basis<Q1, R>::eval(s[0] + r[0] * R(L::xi1(b)), Lm[b]);
#pragma unroll
              for (int i = 0; i < Q1; i++) {
                R t = R(0);
#pragma unroll
                for (int b = 0; b < Q1; b++) t += finite_or_zero_f(Lm[b][i]) * fn[b];
                acc[i] += wx[i] * t;
              }
            } else {
              R wz[Q1];
#pragma unroll
              for (int c = 0; c < Q1; c++) wz[c] = pick<N, R>(wt[2][c], org[2][c], pz);
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
              // pass z: t1[jx][jy][iz]
              R t1[Q1][Q1][Q1];
#pragma unroll
              for (int jx = 0; jx < Q1; jx++)
#pragma unroll
                for (int jy = 0; jy < Q1; jy++)
#pragma unroll
                  for (int iz = 0; iz < Q1; iz++) {
                    R t = R(0);
#pragma unroll
                    for (int jz = 0; jz < Q1; jz++) t += Mz[iz][jz] * fn[(jx * Q1 + jy) * Q1 + jz];
                    t1[jx][jy][iz] = t;
                  }
              // pass y: t2[jx][iy][iz]
              R t2[Q1][Q1][Q1];
#pragma unroll
              for (int jx = 0; jx < Q1; jx++)
#pragma unroll
                for (int iy = 0; iy < Q1; iy++)
#pragma unroll
                  for (int iz = 0; iz < Q1; iz++) {
                    R t = R(0);
#pragma unroll
                    for (int jy = 0; jy < Q1; jy++) t += My[iy][jy] * t1[jx][jy][iz];
                    t2[jx][iy][iz] = t;
                  }
              // pass x, accumulated into the interpolated populations
#pragma unroll
              for (int ix = 0; ix < Q1; ix++)
#pragma unroll
                for (int iy = 0; iy < Q1; iy++)
#pragma unroll
                  for (int iz = 0; iz < Q1; iz++) {
                    R t = acc[(ix * Q1 + iy) * Q1 + iz];
#pragma unroll
                    for (int jx = 0; jx < Q1; jx++) t += Mx[ix][jx] * t2[jx][iy][iz];
                    acc[(ix * Q1 + iy) * Q1 + iz] = t;
                  }
            }
          }
        }
      }
      if (moments_and_test<LAT, R>(a, acc, f0, C, rho0, U, T)) { conv = true; break; }
    }
    finish_node<LAT, R>(a, idx, f0, rho0, U, T, niter, conv, ns);
  }
  reduce_and_commit(ns, a.sums);
}

}  // namespace pond
