// Shared device-side definitions of the PonD step library: lattice traits,
// the 1D Lagrange basis used by the separable gauge transform, boundary
// resolution and the step-kernel argument block.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pond.h"

namespace pond {

// consts.h:117-118: the positive roots of the 5-velocity Hermite set
constexpr double EC1 = 1.3556261799742657;
constexpr double EC2 = 2.8569700138728056;

// Lattice traits.  Every lattice of the reference step is a tensor product
// of a 1D velocity set (D1Q5: 5 speeds in x; D3Q27 = D1Q3^3; D3Q125 =
// D1Q5^3), so a population is addressed by its per-axis class index
// c in [0, Q1): class velocities are XI1[c] * sqrt(T/TLat).
// Class order {0, +a, -a, +b, -b} follows the reference's ef tables.
template <int LAT> struct Lattice;

template <> struct Lattice<POND_D1Q5> {
  static constexpr int D = 1, Q1 = 5, Q = 5;
  static constexpr double TLat = 1.0, Dim = 1.0;
  __host__ __device__ static constexpr double xi1(int c) {
    return c == 0 ? 0.0 : c == 1 ? EC1 : c == 2 ? -EC1 : c == 3 ? EC2 : -EC2;
  }
  // reference population index of tensor class (cx, cy, cz)
  __host__ __device__ static constexpr int ref(int cx, int, int) { return cx; }
};

template <> struct Lattice<POND_D3Q27> {
  static constexpr int D = 3, Q1 = 3, Q = 27;
  static constexpr double TLat = 1.0 / 3.0, Dim = 3.0;
  __host__ __device__ static constexpr double xi1(int c) { return c == 0 ? 0.0 : c == 1 ? 1.0 : -1.0; }
  // consts.h:20-30 lists the 27 directions in its own order; this table maps
  // a class triple (0, +1, -1 per axis) to that order
  __host__ __device__ static constexpr int ref(int cx, int cy, int cz) {
    constexpr int T[27] = {
        /* cx=0 */ 0, 3, 16, 2, 6, 18, 12, 13, 24,
        /* cx=+ */ 1, 5, 17, 4, 7, 19, 14, 15, 25,
        /* cx=- */ 8, 10, 22, 9, 11, 23, 20, 21, 26};
    return T[9 * cx + 3 * cy + cz];
  }
};

template <> struct Lattice<POND_D3Q125> {
  static constexpr int D = 3, Q1 = 5, Q = 125;
  static constexpr double TLat = 1.0, Dim = 3.0;
  __host__ __device__ static constexpr double xi1(int c) {
    return c == 0 ? 0.0 : c == 1 ? EC1 : c == 2 ? -EC1 : c == 3 ? EC2 : -EC2;
  }
  // consts.h:146-199: index = 25*cx + 5*cy + cz
  __host__ __device__ static constexpr int ref(int cx, int cy, int cz) { return 25 * cx + 5 * cy + cz; }
};

// Lattice weight of tensor class t = (cx*Q1 + cy)*Q1 + cz, with the
// reference's expressions (consts.h:34-47 for D3Q27 with TLat = 1/3,
// :127-130 for D1Q5, :200-229 for D3Q125 as W[cx]*W[cy]*W[cz]).
template <int LAT> __host__ __device__ constexpr double lattice_weight_t(int t);
template <> __host__ __device__ constexpr double lattice_weight_t<POND_D1Q5>(int t) {
  constexpr double TLat = 1.0, ec1d = EC1 * EC1, ec2d = EC2 * EC2;
  constexpr double W0 = (3 * TLat * TLat - (ec1d + ec2d) * TLat + ec1d * ec2d) / (ec1d * ec2d);
  constexpr double W1 = TLat * (ec2d - 3 * TLat) / (2 * ec1d * (ec2d - ec1d));
  constexpr double W2 = TLat * (ec1d - 3 * TLat) / (2 * ec2d * (ec1d - ec2d));
  return t == 0 ? W0 : (t <= 2 ? W1 : W2);
}
template <> __host__ __device__ constexpr double lattice_weight_t<POND_D3Q27>(int t) {
  constexpr double TLat = 1. / 3.;
  constexpr double W0 = (1 - TLat) * (1 - TLat) * (1 - TLat);
  constexpr double W1 = (1 - TLat) * (1 - TLat) * TLat / 2.0;
  constexpr double W2 = (1 - TLat) * TLat * TLat / 4.0;
  constexpr double W3 = TLat * TLat * TLat / 8.;
  const int nz = (t / 9 != 0) + ((t / 3) % 3 != 0) + (t % 3 != 0);
  return nz == 0 ? W0 : nz == 1 ? W1 : nz == 2 ? W2 : W3;
}
template <> __host__ __device__ constexpr double lattice_weight_t<POND_D3Q125>(int t) {
  return lattice_weight_t<POND_D1Q5>(t / 25) * lattice_weight_t<POND_D1Q5>((t / 5) % 5) *
         lattice_weight_t<POND_D1Q5>(t % 5);
}

// Lagrange basis of the Q1-point normalised speed set, evaluated at y:
// L_a(y) = prod_{k != a} (y - xi_k) / (xi_a - xi_k).
// This is the matrix of Cell::transfer_gauge (structs.cuh:343-551): the
// population b of a source node, sitting at normalised velocity
// y_b = (u_src - u_dst)/c_dst + (c_src/c_dst) xi_b, contributes L_a(y_b) to
// population a of the target gauge, per axis.
template <int Q1, typename R> struct Basis;

template <typename R> struct Basis<3, R> {
  __device__ __forceinline__ static void eval(R y, R L[3]) {
    const R h = R(0.5) * y;
    L[0] = R(1) - y * y;   // (y-1)(y+1)/(-1)
    L[1] = h * y + h;      // y(y+1)/2
    L[2] = h * y - h;      // y(y-1)/2
  }
};

template <typename R> struct Basis<5, R> {
  __device__ __forceinline__ static void eval(R y, R L[5]) {
    constexpr double e1s = EC1 * EC1, e2s = EC2 * EC2;
    constexpr double D0 = 1.0 / (e1s * e2s);
    constexpr double D1 = 1.0 / (2.0 * e1s * (e1s - e2s));
    constexpr double D2 = 1.0 / (2.0 * e2s * (e2s - e1s));
    const R y2 = y * y;
    const R p1 = y2 - R(e1s);
    const R p2 = y2 - R(e2s);
    const R a = R(D1) * p2;
    const R b = R(D2) * p1;
    L[0] = R(D0) * p1 * p2;
    L[1] = a * (y2 + R(EC1) * y);
    L[2] = a * (y2 - R(EC1) * y);
    L[3] = b * (y2 + R(EC2) * y);
    L[4] = b * (y2 - R(EC2) * y);
  }
};

// Boundary resolution of a stencil coordinate along one axis.  Returns the
// in-range index and sets *rev when the mirror boundary reflected it.
__device__ __forceinline__ int resolve_axis(int p, int n, int bc, bool& rev) {
  rev = false;
  if (p >= 0 && p < n) return p;
  if (bc == POND_BC_CLAMP) return p < 0 ? 0 : n - 1;
  if (bc == POND_BC_MIRROR) {
    if (p < 0) { p = -1 - p; rev = true; }
    if (p >= n) { p = n - 1 - p + n; rev = true; }
  }
  p %= n;
  return p < 0 ? p + n : p;
}

// Per-step reduction slots (float64 sums and int64 counters), one set per
// context in device memory.
struct StepSums {
  double mass, mom[3], enrg, k;
  unsigned long long niter_sum, nonconv;
  unsigned long long work;  // stencil nodes transformed (summed over nodes and iterations)
  int niter_max;
  int pad;
};

// Equilibrium energy populations of one node in the gauge (U, T) for the
// double-distribution extension, in tensor-class order t = (cx Q1 + cy) Q1 + cz
// (for D1Q5 the class order is the population order):
// h_t = rho w_t (|v_t|^2 + dof T), v_t = U + sqrt(T/TLat) xi_t.
template <int LAT, typename R>
__host__ __device__ inline void energy_equilibrium(double rho, const double U[3], double T, double dof, R* h) {
  using L = Lattice<LAT>;
  const double C = sqrt(fabs(T) * (1.0 / L::TLat));
#pragma unroll
  for (int t = 0; t < L::Q; t++) {
    const int cx = L::D == 1 ? t : t / (L::Q1 * L::Q1);
    const double vx = C * L::xi1(cx) + U[0];
    const double vy = (L::D == 1 ? 0.0 : C * L::xi1((t / L::Q1) % L::Q1)) + U[1];
    const double vz = (L::D == 1 ? 0.0 : C * L::xi1(t % L::Q1)) + U[2];
    h[t] = R(rho * lattice_weight_t<LAT>(t) * (vx * vx + vy * vy + vz * vz + dof * T));
  }
}

// Arguments of the step kernels.
template <typename R> struct StepArgs {
  const R* f_in;   // [Q][N]
  const R* rho_in; // [N]
  const R* g_in;   // [4][N]
  R* f_out;
  R* rho_out;
  R* g_out;
  const float* guess;  // [4][N] predicted starting gauge, or null
  int* niter_out;      // [N] or null
  StepSums* sums;
  int nx, ny, nz;
  long long N;
  int bc[3];
  double dtau;
  double tol_abs, tol_rel;    // isConv on every population
  double tolg_abs, tolg_rel;  // isConv on the gauge u, T (the reference uses tol_abs, tol_rel for both)
  int max_iter;
  double kdx;  // 0.5 * dx*dy*dz / (8 pi^3) with dx = 2 pi / Nx (diagn.cu:14-18)
  // energy populations of the double-distribution extension (D1Q5), or null
  const R* h_in = nullptr;  // [Q][N]
  R* h_out = nullptr;
  double dof = 0;           // extra degrees of freedom
  // one-dimensional mesh schemes: node mask (nonzero = active) and node positions, or null
  const uint8_t* mask = nullptr;  // [N]
  const double* pos = nullptr;    // [N]
  // state of the inflow ghost node of POND_BC_INFLOW axes: rho, u_x, u_y, u_z, T
  double inflow[5] = {1, 0, 0, 0, 1};
};

}  // namespace pond
