// D3Q27 PonD pull step, float32, one thread per node with the stencil tile
// staged in shared memory (the hot kernel of the 256^3 benchmark).
//
// Same arithmetic as pull_point_kernel (steps.cu:356-588 LBMpull with
// propagate<N>, N = 2, 3, 4), organised for the SM:
//
//  * a CTA owns a 32 x 4 x 2 tile of nodes and stages the tile plus a halo of
//    2 nodes per side (36 x 8 x 6 nodes, 31 float planes: 27 populations,
//    u_x, u_y, u_z and c = sqrts(T/TLat), 214 KB) once per step.  Boundary
//    resolution (periodic wrap, clamp, mirror with population reversal), the
//    reference's dropping of non-finite terms and the square root of T are
//    applied while staging, so the iteration loop reads plain SoA planes;
//  * the fixed-point iteration is warp-synchronous: a warp iterates while any
//    of its lanes is unconverged, and walks the stencil offsets common to its
//    lanes, so a warp's shared-memory loads hit 32 consecutive addresses;
//  * per stencil node the gauge transform is three 1D passes of the 3x3
//    Lagrange-basis matrix with the interpolation weights folded into the
//    rows (243 FMA), accumulated straight into the 27 populations;
//  * a lane whose departure points leave the +-2 halo (|u| + sqrt(T/TLat) >= 1
//    along an axis) runs that iteration from global memory instead.
#pragma once
#include "pond_step_point.cuh"

namespace pond {
namespace d27 {

constexpr int TX = 32, TY = 4, TZ = 2, H = 2;
constexpr int SX = TX + 2 * H, SY = TY + 2 * H, SZ = TZ + 2 * H;
constexpr int SN = SX * SY * SZ;  // 1728 staged nodes
constexpr int NPL = 31;           // planes: 27 f, u_x, u_y, u_z, c
// + a global node index (int32) and a flag byte per staged node
constexpr size_t SMEM_BYTES = size_t(NPL) * SN * sizeof(float) + size_t(SN) * sizeof(int) + SN;
constexpr int THREADS = TX * TY * TZ;

// reference population index of tensor class t = 9 cx + 3 cy + cz, for
// lookups with run-time indices (consts.h:20-30 order)
__constant__ int c_ref27[27] = {0, 3, 16, 2, 6, 18, 12, 13, 24, 1, 5, 17, 4, 7, 19, 14, 15, 25,
                                8, 10, 22, 9, 11, 23, 20, 21, 26};

// 4-byte asynchronous global -> shared copy and the wait for all of them
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// class index -> its mirror image along one axis (0 <-> 0, + <-> -)
__device__ __forceinline__ int rev3(int c) { return c == 0 ? 0 : 3 - c; }

// Weighted basis rows of one axis: M[i][b] = w_i * L_i(s + r*xi_b) for the
// three classes i of the target gauge, xi = {0, +1, -1}.
__device__ __forceinline__ void weighted_rows(float s, float r, const float w[3], float M[3][3]) {
  const float y[3] = {s, s + r, s - r};
  const float hw1 = 0.5f * w[1], hw2 = 0.5f * w[2];
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const float t = w[0] * y[b];
    M[0][b] = fmaf(-t, y[b], w[0]);      // w0 (1 - y^2)
    const float u = hw1 * y[b];
    M[1][b] = fmaf(u, y[b], u);          // w1 y (y + 1) / 2
    const float v = hw2 * y[b];
    M[2][b] = fmaf(v, y[b], -v);         // w2 y (y - 1) / 2
  }
}

// acc[ix,iy,iz] += sum_j Mx[ix][jx] My[iy][jy] Mz[iz][jz] f[jx,jy,jz]
__device__ __forceinline__ void transform_accumulate(const float fn[27], const float Mx[3][3], const float My[3][3],
                                                     const float Mz[3][3], float acc[27]) {
  float t1[3][3][3];
#pragma unroll
  for (int jx = 0; jx < 3; jx++)
#pragma unroll
    for (int jy = 0; jy < 3; jy++)
#pragma unroll
      for (int iz = 0; iz < 3; iz++)
        t1[jx][jy][iz] = fmaf(Mz[iz][2], fn[jx * 9 + jy * 3 + 2],
                              fmaf(Mz[iz][1], fn[jx * 9 + jy * 3 + 1], Mz[iz][0] * fn[jx * 9 + jy * 3]));
  float t2[3][3][3];
#pragma unroll
  for (int jx = 0; jx < 3; jx++)
#pragma unroll
    for (int iy = 0; iy < 3; iy++)
#pragma unroll
      for (int iz = 0; iz < 3; iz++)
        t2[jx][iy][iz] = fmaf(My[iy][2], t1[jx][2][iz], fmaf(My[iy][1], t1[jx][1][iz], My[iy][0] * t1[jx][0][iz]));
#pragma unroll
  for (int ix = 0; ix < 3; ix++)
#pragma unroll
    for (int iy = 0; iy < 3; iy++)
#pragma unroll
      for (int iz = 0; iz < 3; iz++) {
        float& o = acc[ix * 9 + iy * 3 + iz];
        o = fmaf(Mx[ix][2], t2[2][iy][iz], fmaf(Mx[ix][1], t2[1][iy][iz], fmaf(Mx[ix][0], t2[0][iy][iz], o)));
      }
}

// As transform_accumulate, restricted to the target classes each axis needs
// at this stencil node (nx/ny/nz: warp-uniform, a class is skipped when its
// interpolation weight is zero for every lane of the warp).
__device__ __forceinline__ void transform_accumulate_sel(const float fn[27], const float Mx[3][3],
                                                         const float My[3][3], const float Mz[3][3],
                                                         const bool nx[3], const bool ny[3], const bool nz[3],
                                                         float acc[27]) {
  float t1[3][3][3];
#pragma unroll
  for (int iz = 0; iz < 3; iz++) {
    if (!nz[iz]) continue;
#pragma unroll
    for (int jx = 0; jx < 3; jx++)
#pragma unroll
      for (int jy = 0; jy < 3; jy++)
        t1[jx][jy][iz] = fmaf(Mz[iz][2], fn[jx * 9 + jy * 3 + 2],
                              fmaf(Mz[iz][1], fn[jx * 9 + jy * 3 + 1], Mz[iz][0] * fn[jx * 9 + jy * 3]));
  }
  float t2[3][3][3];
#pragma unroll
  for (int iy = 0; iy < 3; iy++) {
    if (!ny[iy]) continue;
#pragma unroll
    for (int iz = 0; iz < 3; iz++) {
      if (!nz[iz]) continue;
#pragma unroll
      for (int jx = 0; jx < 3; jx++)
        t2[jx][iy][iz] = fmaf(My[iy][2], t1[jx][2][iz], fmaf(My[iy][1], t1[jx][1][iz], My[iy][0] * t1[jx][0][iz]));
    }
  }
#pragma unroll
  for (int ix = 0; ix < 3; ix++) {
    if (!nx[ix]) continue;
#pragma unroll
    for (int iy = 0; iy < 3; iy++) {
      if (!ny[iy]) continue;
#pragma unroll
      for (int iz = 0; iz < 3; iz++) {
        if (!nz[iz]) continue;
        float& o = acc[ix * 9 + iy * 3 + iz];
        o = fmaf(Mx[ix][2], t2[2][iy][iz], fmaf(Mx[ix][1], t2[1][iy][iz], fmaf(Mx[ix][0], t2[0][iy][iz], o)));
      }
    }
  }
}

// interpolation weight of relative offset o for a window starting at ro
template <int N> __device__ __forceinline__ float wpick(const float w[N], int ro, int o) {
  const int j = o - ro;
  float r = 0.f;
#pragma unroll
  for (int k = 0; k < N; k++) r = (j == k) ? w[k] : r;
  return r;
}

// Per-CTA partial of the step sums, written instead of the atomic update
// when the kernel runs without a context (kPartials = true; a.sums then
// points at an array of one BlockPartial per CTA).
struct BlockPartial {
  double mass, mom[3], enrg, k;
  unsigned long long niter_sum, nonconv, work;
  int niter_max;
  int pad;
};

__device__ __forceinline__ void write_block_partial(NodeSums s, BlockPartial* out) {
  __shared__ double pd[6][THREADS / 32];
  __shared__ unsigned long long pu[3][THREADS / 32];
  __shared__ int pm[THREADS / 32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int warp = tid >> 5;
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
    for (int q = 0; q < 6; q++) pd[q][warp] = v[q];
    pu[0][warp] = s.niter; pu[1][warp] = s.nonconv; pu[2][warp] = s.work; pm[warp] = s.nmax;
  }
  __syncthreads();
  if (tid == 0) {
    BlockPartial b = {};
    for (int w = 0; w < THREADS / 32; w++) {
      b.mass += pd[0][w]; b.mom[0] += pd[1][w]; b.mom[1] += pd[2][w]; b.mom[2] += pd[3][w];
      b.enrg += pd[4][w]; b.k += pd[5][w];
      b.niter_sum += pu[0][w]; b.nonconv += pu[1][w]; b.work += pu[2][w];
      b.niter_max = max(b.niter_max, pm[w]);
    }
    out[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = b;
  }
}

template <int N, bool kPartials = false>
__global__ void __launch_bounds__(THREADS, 1) pull_d3q27_tile_kernel(StepArgs<float> a) {
  using L = Lattice<POND_D3Q27>;
  extern __shared__ __align__(16) float sm[];
  int* gidx = reinterpret_cast<int*>(sm + NPL * SN);
  unsigned char* flags = reinterpret_cast<unsigned char*>(gidx + SN);
  const int tid = threadIdx.x + TX * (threadIdx.y + TY * threadIdx.z);
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;

  // ---- stage the tile: every value is fetched with an asynchronous copy
  // (cp.async, no register round trip), so a thread has all of its ~210
  // copies in flight at once; boundary resolution happens in the addresses.
  // 1) per staged node: global index, mirror flags, the four gauge planes
  for (int i = tid; i < SN; i += THREADS) {
    const int hx = i % SX, hy = (i / SX) % SY, hz = i / (SX * SY);
    bool rv[3];
    const int gx = resolve_axis(x0 - H + hx, a.nx, a.bc[0], rv[0]);
    const int gy = resolve_axis(y0 - H + hy, a.ny, a.bc[1], rv[1]);
    const int gz = resolve_axis(z0 - H + hz, a.nz, a.bc[2], rv[2]);
    const int g = gx + a.nx * (gy + a.ny * gz);
    gidx[i] = g;
    flags[i] = (unsigned char)((rv[0] ? 1 : 0) | (rv[1] ? 2 : 0) | (rv[2] ? 4 : 0));
#pragma unroll
    for (int k = 0; k < 4; k++) cp_async4(&sm[(27 + k) * SN + i], a.g_in + (long long)k * a.N + g);
  }
  __syncthreads();
  // 2) populations in tensor-class order (the mirror reverses classes)
  for (int idx = tid; idx < 27 * SN; idx += THREADS) {
    const int p = idx / SN, i = idx - p * SN;
    const unsigned fl = flags[i];
    int cx = p / 9, cy = (p / 3) % 3, cz = p % 3;
    if (fl & 1) cx = rev3(cx);
    if (fl & 2) cy = rev3(cy);
    if (fl & 4) cz = rev3(cz);
    cp_async4(&sm[idx], a.f_in + (long long)c_ref27[cx * 9 + cy * 3 + cz] * a.N + gidx[i]);
  }
  cp_async_wait_all();
  __syncthreads();
  // 3) gauge post-pass: mirrored velocity components flip sign, c = sqrts(T/TLat);
  //    a node with a non-finite gauge contributes nothing (all its transfer
  //    terms are non-finite in the reference and dropped)
  for (int i = tid; i < SN; i += THREADS) {
    const unsigned fl = flags[i];
    float u[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float v = sm[(27 + k) * SN + i];
      u[k] = (fl >> k) & 1 ? -v : v;
    }
    const float T = sm[30 * SN + i];
    const float c = copysignf(sqrtf(fabsf(T) * (float)(1.0 / L::TLat)), T);
    const bool ok = fabsf(u[0]) <= 3.0e38f && fabsf(u[1]) <= 3.0e38f && fabsf(u[2]) <= 3.0e38f && fabsf(c) <= 3.0e38f;
    sm[27 * SN + i] = ok ? u[0] : 0.f;
    sm[28 * SN + i] = ok ? u[1] : 0.f;
    sm[29 * SN + i] = ok ? u[2] : 0.f;
    sm[30 * SN + i] = ok ? c : 1.f;
    flags[i] = (unsigned char)(fl | (ok ? 0 : 8));
  }
  __syncthreads();
  // 4) populations post-pass: non-finite values and invalid nodes -> 0
  for (int idx = tid; idx < 27 * SN; idx += THREADS) {
    const int i = idx % SN;
    const float v = sm[idx];
    sm[idx] = (!(flags[i] & 8) && fabsf(v) <= 3.402823466e38f) ? v : 0.f;
  }
  __syncthreads();

  const int lx = threadIdx.x, ly = threadIdx.y, lz = threadIdx.z;
  const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
  const bool active = x < a.nx && y < a.ny && z < a.nz;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  const long long idx = active ? x + (long long)a.nx * (y + (long long)a.ny * z) : 0;
  float f0[27];
  double rho0 = 1, U[3] = {0, 0, 0}, T = L::TLat;
  if (active) load_center<POND_D3Q27, float>(a, idx, f0, rho0, U, T);
  else
#pragma unroll
    for (int t = 0; t < 27; t++) f0[t] = 0.f;
  const int pos[3] = {x, y, z};
  const int sbase = (lz + H) * SX * SY + (ly + H) * SX + (lx + H);
  bool done = !active;
  bool conv = false;
  int niter = 0;
  unsigned long long work = 0;
  while (__any_sync(0xffffffffu, !done)) {
    if (!done) niter++;
    const double C = sqrt(T * (1.0 / L::TLat));
    // relative window origins and Lagrange weights per axis and class
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
    const float invC = __frcp_rn(float(C));
    const float Us[3] = {float(U[0]) * invC, float(U[1]) * invC, float(U[2]) * invC};
    float acc[27];
#pragma unroll
    for (int t = 0; t < 27; t++) acc[t] = 0.f;
    const bool inside = lo[0] >= -H && lo[1] >= -H && lo[2] >= -H && hi[0] <= H && hi[1] <= H && hi[2] <= H;
    if (__all_sync(0xffffffffu, inside || done)) {
      // warp-uniform offsets: the union of the unconverged lanes' stencils
      int wl[3], wh[3];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        wl[ax] = __reduce_min_sync(0xffffffffu, done ? H : lo[ax]);
        wh[ax] = __reduce_max_sync(0xffffffffu, done ? -H : hi[ax]);
      }
      if (!done) work += (unsigned long long)(wh[0] - wl[0] + 1) * (wh[1] - wl[1] + 1) * (wh[2] - wl[2] + 1);
      for (int ox = wl[0]; ox <= wh[0]; ox++) {
        float wx[3];
        bool nx[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          wx[c] = wpick<N>(wt[0][c], ro[0][c], ox);
          nx[c] = __any_sync(0xffffffffu, !done && wx[c] != 0.f);
        }
        for (int oy = wl[1]; oy <= wh[1]; oy++) {
          float wy[3];
          bool ny[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            wy[c] = wpick<N>(wt[1][c], ro[1][c], oy);
            ny[c] = __any_sync(0xffffffffu, !done && wy[c] != 0.f);
          }
#pragma unroll
          for (int oz = -H; oz <= H; oz++) {
            if (oz < wl[2] || oz > wh[2]) continue;
            float wz[3];
            bool nz[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
              wz[c] = wpick<N>(wt[2][c], ro[2][c], oz);
              nz[c] = __any_sync(0xffffffffu, !done && wz[c] != 0.f);
            }
            const int si = sbase + oz * SX * SY + oy * SX + ox;
            float fn[27];
#pragma unroll
            for (int t = 0; t < 27; t++) fn[t] = sm[t * SN + si];
            const float cn = sm[30 * SN + si];
            const float r = cn * invC;
            float Mx[3][3], My[3][3], Mz[3][3];
            weighted_rows(fmaf(sm[27 * SN + si], invC, -Us[0]), r, wx, Mx);
            weighted_rows(fmaf(sm[28 * SN + si], invC, -Us[1]), r, wy, My);
            weighted_rows(fmaf(sm[29 * SN + si], invC, -Us[2]), r, wz, Mz);
            transform_accumulate_sel(fn, Mx, My, Mz, nx, ny, nz, acc);
          }
        }
      }
    } else if (!done) {
      // departure points beyond the staged halo: this lane reads global memory
      if (!done) work += (unsigned long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
      for (int ox = lo[0]; ox <= hi[0]; ox++) {
        bool rv[3] = {false, false, false};
        const int gx = resolve_axis(x + ox, a.nx, a.bc[0], rv[0]);
        float wx[3];
#pragma unroll
        for (int c = 0; c < 3; c++) wx[c] = wpick<N>(wt[0][c], ro[0][c], ox);
        for (int oy = lo[1]; oy <= hi[1]; oy++) {
          const int gy = resolve_axis(y + oy, a.ny, a.bc[1], rv[1]);
          float wy[3];
#pragma unroll
          for (int c = 0; c < 3; c++) wy[c] = wpick<N>(wt[1][c], ro[1][c], oy);
          for (int oz = lo[2]; oz <= hi[2]; oz++) {
            const int gz = resolve_axis(z + oz, a.nz, a.bc[2], rv[2]);
            float wz[3];
#pragma unroll
            for (int c = 0; c < 3; c++) wz[c] = wpick<N>(wt[2][c], ro[2][c], oz);
            const long long g = gx + (long long)a.nx * (gy + (long long)a.ny * gz);
            float fn[27], s[3], r[3];
            const float Uc[3] = {float(U[0]), float(U[1]), float(U[2])};
            load_node<POND_D3Q27, float>(a, g, rv, Uc, invC, fn, s, r);
            const float Tn = a.g_in[3 * a.N + g];
            const float un0 = a.g_in[g], un1 = a.g_in[a.N + g], un2 = a.g_in[2 * a.N + g];
            const bool ok = fabsf(un0) <= 3.0e38f && fabsf(un1) <= 3.0e38f && fabsf(un2) <= 3.0e38f &&
                            fabsf(Tn) <= 3.0e38f;
            float Mx[3][3], My[3][3], Mz[3][3];
            weighted_rows(s[0], r[0], wx, Mx);
            weighted_rows(s[1], r[1], wy, My);
            weighted_rows(s[2], r[2], wz, Mz);
            if (ok) transform_accumulate(fn, Mx, My, Mz, acc);
          }
        }
      }
    }
    if (!done) {
      if (!(C >= 1.0e-300)) {  // C <= 0, NaN, or 1/C beyond 1e300
        // target T = 0: every transfer term is non-finite and dropped (structs.cuh:542)
#pragma unroll
        for (int t = 0; t < 27; t++) acc[t] = 0.f;
      }
      conv = moments_and_test<POND_D3Q27, float>(a, acc, f0, C, rho0, U, T);
      if (conv || niter >= a.max_iter) done = true;
    }
  }
  if (active) {
    finish_node<POND_D3Q27, float>(a, idx, f0, rho0, U, T, niter, conv, ns);
    ns.work = work;
  }
  if constexpr (kPartials) write_block_partial(ns, reinterpret_cast<BlockPartial*>(a.sums));
  else reduce_and_commit(ns, a.sums);
}

}  // namespace d27
}  // namespace pond
