// D3Q125 PonD pull step, float32: a tile of nodes per CTA, a warp per node.
//
// Same arithmetic as pull_d3q125_kernel (steps.cu:151-250 PonDstepD3Q125:
// quadratic stencil with its origin fixed at coord-1, separable gauge
// transform with the interpolation weights folded into the basis rows,
// float64 moments and convergence test), organised for the SM:
//
//  * a CTA owns a 4 x 4 x 4 tile and stages it with its +-1 halo (6 x 6 x 6
//    nodes: 125 population planes, the gauge velocities and c, 113 KB) once
//    per step, so two CTAs fit on an SM and every staged node serves up to
//    27 centres from shared memory;
//  * each of the 8 warps takes 8 nodes of the tile in turn and iterates one
//    node at a time, so a warp never waits for another node's iterations;
//  * lane 5j+k (25 lanes) owns source x-class j and target z-class k: per
//    stencil node it runs the z pass (t1[j][*][k], 25 FMA) and the y pass
//    (t2[j][*][k], 25 FMA) on its own data, then takes t2 of the lanes with
//    the same k by shuffle and accumulates target populations (j, *, k) of
//    the x pass (25 FMA); the 75 weighted basis entries of the stencil node
//    are computed three per lane into a per-warp table;
//  * the plane stride of the staged populations is 217 slots, so the five
//    source x-classes read in one instruction fall in distinct banks.
// Mirrored axes are handled as in the reference kernel: the staged node's
// velocity component and c flip sign along that axis (-c maps each
// population onto its mirror image), the populations stay in place.
#pragma once
#include "pond_common.cuh"
#include "pond_step_point.cuh"

namespace pond {
namespace d125t {

constexpr int T = 4;                // tile edge
constexpr int S = T + 2;            // staged edge (+-1 halo)
constexpr int SN = S * S * S;       // 216 staged nodes
constexpr int PS = SN + 1;          // plane stride: 25 * 217 = 17 mod 32
constexpr int WARPS = 8;
constexpr int THREADS = 32 * WARPS;

struct Smem {
  float f[125 * PS];       // staged populations, non-finite values zeroed
  float u[3][SN];          // staged velocities (sign-flipped on mirrored axes)
  float c[SN];             // sqrts(T / TLat)
  unsigned char flags[SN]; // mirrored axes (bits 0-2)
  float M[WARPS][3][6][5]; // per-warp weighted basis rows of the current stencil node (row 5: idle lanes)
};

static_assert(2 * (sizeof(Smem) + 1024) <= 233472, "two CTAs must fit in the 228 KB of an SM");

// global node of staged node i and its mirror flags
__device__ __forceinline__ int staged_global(const StepArgs<float>& a, int x0, int y0, int z0, int i, bool rv[3]) {
  const int hx = i % S, hy = (i / S) % S, hz = i / (S * S);
  const int gx = resolve_axis(x0 - 1 + hx, a.nx, a.bc[0], rv[0]);
  const int gy = resolve_axis(y0 - 1 + hy, a.ny, a.bc[1], rv[1]);
  const int gz = resolve_axis(z0 - 1 + hz, a.nz, a.bc[2], rv[2]);
  return gx + a.nx * (gy + a.ny * gz);
}

// Row i of the 5-point Lagrange basis on {0, +EC1, -EC1, +EC2, -EC2}:
// L_i(y) = D_i (y^2 - P_i)(y^2 + s_i y - Q_i), coefficients per row
struct BasisRow {
  float D, P, s, Q;
  __device__ __forceinline__ explicit BasisRow(int i) {
    constexpr double e1s = EC1 * EC1, e2s = EC2 * EC2;
    D = i == 0 ? float(1.0 / (e1s * e2s))
               : (i <= 2 ? float(1.0 / (2.0 * e1s * (e1s - e2s))) : float(1.0 / (2.0 * e2s * (e2s - e1s))));
    P = (i == 1 || i == 2) ? float(e2s) : float(e1s);
    s = i == 1 ? float(EC1) : i == 2 ? -float(EC1) : i == 3 ? float(EC2) : i == 4 ? -float(EC2) : 0.f;
    Q = i == 0 ? float(e2s) : 0.f;
  }
  __device__ __forceinline__ float operator()(float y) const {
    const float y2 = y * y;
    return D * (y2 - P) * (fmaf(s, y, y2) - Q);
  }
};

__device__ __forceinline__ double xi5(int c) { return Lattice<POND_D3Q125>::xi1(c); }

__global__ void __launch_bounds__(THREADS, 2) pull_d3q125_tile_kernel(StepArgs<float> a) {
  using L = Lattice<POND_D3Q125>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = blockIdx.x * T, y0 = blockIdx.y * T, z0 = blockIdx.z * T;

  // ---- stage the tile (steps.cu:164-193 per node, once per CTA here)
  for (int i = tid; i < SN; i += THREADS) {
    bool rv[3];
    const int g = staged_global(a, x0, y0, z0, i, rv);
    sm.flags[i] = (unsigned char)((rv[0] ? 1 : 0) | (rv[1] ? 2 : 0) | (rv[2] ? 4 : 0));
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float v = a.g_in[(long long)k * a.N + g];
      sm.u[k][i] = rv[k] ? -v : v;
    }
    const float Tn = a.g_in[3 * a.N + g];
    sm.c[i] = copysignf(sqrtf(fabsf(Tn) * float(1.0 / L::TLat)), Tn);
  }
  for (int idx = tid; idx < 125 * SN; idx += THREADS) {
    const int p = idx / SN, i = idx - p * SN;
    bool rv[3];
    const int g = staged_global(a, x0, y0, z0, i, rv);
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(&sm.f[p * PS + i]));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(a.f_in + (long long)p * a.N + g)
                 : "memory");
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  for (int idx = tid; idx < 125 * SN; idx += THREADS) {
    const int p = idx / SN, i = idx - p * SN;
    float& v = sm.f[p * PS + i];
    v = finite_or_zero_f(v);
  }
  __syncthreads();

  // ---- one warp per node; lane 5j+k: source / target x-class j, z-class k
  // idle lanes (25..31) compute like lane 20+k and write table row 5, which nobody reads
  const bool worker = lane < 25;
  const int j = worker ? lane / 5 : 4, k = lane % 5, jrow = worker ? j : 5;
  const BasisRow Lj(j);
  const float xik = float(xi5(k));
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  for (int t = warp; t < T * T * T; t += WARPS) {
    const int lx = t % T, ly = (t / T) % T, lz = t / (T * T);
    const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
    if (x >= a.nx || y >= a.ny || z >= a.nz) continue;  // warp-uniform
    const long long idx = x + (long long)a.nx * (y + (long long)a.ny * z);
    // c0.load of the centre: this lane's populations (j, iy, k), iy = 0..4
    float f0[5];
#pragma unroll
    for (int iy = 0; iy < 5; iy++) f0[iy] = worker ? a.f_in[(long long)(25 * j + 5 * iy + k) * a.N + idx] : 0.f;
    double rho0 = a.rho_in[idx];
    double U[3] = {(double)a.g_in[idx], (double)a.g_in[a.N + idx], (double)a.g_in[2 * a.N + idx]};
    double Tc = a.g_in[3 * a.N + idx];
    if (rho0 == 0 && U[0] == 0 && U[1] == 0 && U[2] == 0 && Tc == 0) {  // set_base(1, TLat)
      rho0 = 1;
      Tc = L::TLat;
#pragma unroll
      for (int iy = 0; iy < 5; iy++) f0[iy] = worker ? float(lattice_weight_t<POND_D3Q125>(25 * j + 5 * iy + k)) : 0.f;
    }
    if (a.guess) {
      U[0] = a.guess[idx]; U[1] = a.guess[a.N + idx]; U[2] = a.guess[2 * a.N + idx]; Tc = a.guess[3 * a.N + idx];
    }
    const int pos[3] = {x, y, z};
    const int qc = ((lz + 1) * S + (ly + 1)) * S + (lx + 1);  // staged centre
    int niter = 0;
    bool conv = false;
    float acc[5];
    while (niter < a.max_iter) {
      niter++;
      const double C = sqrt(Tc / L::TLat);
      const float invC = __frcp_rn(float(C));
      // LagrPol<3> factors of target class j (this lane's basis row) per
      // axis at the three stencil positions: shift = crd - (coord - 1)
      float w3[3][3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        const double crd = double(pos[ax]) - (C * xi5(j) + U[ax]);
        lagr_weights<3, float>(crd - double(pos[ax] - 1), w3[ax]);
      }
      const float Uf[3] = {float(U[0]), float(U[1]), float(U[2])};
#pragma unroll
      for (int iy = 0; iy < 5; iy++) acc[iy] = 0.f;
      for (int n = 0; n < 27; n++) {
        const int na[3] = {n / 9, (n / 3) % 3, n % 3};
        const int q = qc + (na[2] - 1) * S * S + (na[1] - 1) * S + (na[0] - 1);
        // this lane's three basis entries M[ax][j][k] = w_j L_j(s + r xi_k)
        {
          const float cq = sm.c[q] * invC;
          const unsigned fl = sm.flags[q];
#pragma unroll
          for (int ax = 0; ax < 3; ax++) {
            const float s = (sm.u[ax][q] - Uf[ax]) * invC;
            const float r = (fl >> ax) & 1 ? -cq : cq;
            const float wj = na[ax] == 0 ? w3[ax][0] : na[ax] == 1 ? w3[ax][1] : w3[ax][2];
            sm.M[warp][ax][jrow][k] = wj * finite_or_zero_f(Lj(fmaf(r, xik, s)));
          }
        }
        __syncwarp();
        // z pass: t1[jy] = sum_jz Mz[k][jz] f[j][jy][jz]
        float mz[5];
#pragma unroll
        for (int jz = 0; jz < 5; jz++) mz[jz] = sm.M[warp][2][k][jz];
        float t1[5];
        const float* fq = sm.f + (25 * j) * PS + q;
#pragma unroll
        for (int jy = 0; jy < 5; jy++) {
          float v = 0.f;
#pragma unroll
          for (int jz = 0; jz < 5; jz++) v += mz[jz] * fq[(5 * jy + jz) * PS];
          t1[jy] = v;
        }
        // y pass: t2[iy] = sum_jy My[iy][jy] t1[jy]
        float t2[5];
#pragma unroll
        for (int iy = 0; iy < 5; iy++) {
          float v = 0.f;
#pragma unroll
          for (int jy = 0; jy < 5; jy++) v += sm.M[warp][1][iy][jy] * t1[jy];
          t2[iy] = v;
        }
        // x pass: acc[iy] += sum_jx Mx[j][jx] t2 of lane (jx, k)
        float mxr[5];
#pragma unroll
        for (int jx = 0; jx < 5; jx++) mxr[jx] = sm.M[warp][0][j][jx];
#pragma unroll
        for (int jx = 0; jx < 5; jx++) {
          const float mx = mxr[jx];
#pragma unroll
          for (int iy = 0; iy < 5; iy++) acc[iy] += mx * __shfl_sync(0xffffffffu, t2[iy], 5 * jx + k);
        }
        __syncwarp();  // the table is rewritten for the next stencil node
      }
      // calcMoments in float64 (structs.cuh:315-342), warp-wide
      double mv[5] = {0, 0, 0, 0, 0};
      if (worker) {
        const double vx = C * xi5(j) + U[0], vz = C * xi5(k) + U[2];
#pragma unroll
        for (int iy = 0; iy < 5; iy++) {
          const double fv = acc[iy], vy = C * xi5(iy) + U[1];
          mv[0] += fv; mv[1] += fv * vx; mv[2] += fv * vy; mv[3] += fv * vz;
          mv[4] += fv * (vx * vx + vy * vy + vz * vz);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int m = 0; m < 5; m++) mv[m] += __shfl_xor_sync(0xffffffffu, mv[m], o);
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
      for (int q = 0; q < 3; q++) ok = ok && !(fabs(m[q] - U[q]) >= a.tol_abs + a.tol_rel * fabs(m[q]));
      ok = ok && !(fabs(Tn - Tc) >= a.tol_abs + a.tol_rel * fabs(Tn));
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
    // BGK and store (steps.cu:230-248)
    const float rr = float(rho0), dtau = float(a.dtau);
    if (worker)
#pragma unroll
      for (int iy = 0; iy < 5; iy++) {
        const int p = 25 * j + 5 * iy + k;
        const float fb = f0[iy] + dtau * (rr * float(lattice_weight_t<POND_D3Q125>(p)) - f0[iy]);
        a.f_out[(long long)p * a.N + idx] = fb;
      }
    if (lane == 0) {
      const float u0 = float(U[0]), u1 = float(U[1]), u2 = float(U[2]), ts = float(Tc);
      a.rho_out[idx] = rr;
      a.g_out[idx] = u0; a.g_out[a.N + idx] = u1; a.g_out[2 * a.N + idx] = u2; a.g_out[3 * a.N + idx] = ts;
      if (a.niter_out) a.niter_out[idx] = niter;
      const double dr = rr, d0 = u0, d1 = u1, d2 = u2, dt = ts;
      const double u2s = d0 * d0 + d1 * d1 + d2 * d2;
      ns.mass += dr; ns.m0 += dr * d0; ns.m1 += dr * d1; ns.m2 += dr * d2;
      ns.enrg += dr * (u2s + L::Dim * dt);
      ns.k += a.kdx * u2s;
      ns.niter += niter; ns.nonconv += conv ? 0 : 1; ns.nmax = max(ns.nmax, niter);
      ns.work += 27ull * niter;
    }
  }
  // ---- the CTA's share of the step sums, through the (now free) tile memory
  __syncthreads();
  double* pd = reinterpret_cast<double*>(sm.f);  // [WARPS][6]
  unsigned long long* pu = reinterpret_cast<unsigned long long*>(pd + 6 * WARPS);  // [WARPS][3]
  int* pm = reinterpret_cast<int*>(pu + 3 * WARPS);
  if (lane == 0) {
    pd[warp * 6 + 0] = ns.mass; pd[warp * 6 + 1] = ns.m0; pd[warp * 6 + 2] = ns.m1;
    pd[warp * 6 + 3] = ns.m2; pd[warp * 6 + 4] = ns.enrg; pd[warp * 6 + 5] = ns.k;
    pu[warp * 3 + 0] = ns.niter; pu[warp * 3 + 1] = ns.nonconv; pu[warp * 3 + 2] = ns.work;
    pm[warp] = ns.nmax;
  }
  __syncthreads();
  if (tid == 0) {
    double s6[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long s3[3] = {0, 0, 0};
    int mx = 0;
    for (int w = 0; w < WARPS; w++) {
      for (int q = 0; q < 6; q++) s6[q] += pd[w * 6 + q];
      for (int q = 0; q < 3; q++) s3[q] += pu[w * 3 + q];
      mx = max(mx, pm[w]);
    }
    atomicAdd(&a.sums->mass, s6[0]);
    atomicAdd(&a.sums->mom[0], s6[1]);
    atomicAdd(&a.sums->mom[1], s6[2]);
    atomicAdd(&a.sums->mom[2], s6[3]);
    atomicAdd(&a.sums->enrg, s6[4]);
    atomicAdd(&a.sums->k, s6[5]);
    atomicAdd(&a.sums->niter_sum, s3[0]);
    atomicAdd(&a.sums->nonconv, s3[1]);
    if (s3[2]) atomicAdd(&a.sums->work, s3[2]);
    atomicMax(&a.sums->niter_max, mx);
  }
}

}  // namespace d125t
}  // namespace pond
