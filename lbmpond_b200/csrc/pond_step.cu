// Step dispatch, buffer management and host<->device conversion.
#include <cuda_runtime.h>

#include <cstring>
#include <type_traits>
#include <vector>

#include "pond_internal.h"
#include "pond_step_1d.cuh"
#include "pond_step_1d_energy.cuh"
#include "pond_step_1d_mesh.cuh"
#include "pond_step_d3q27_energy.cuh"
#include "pond_step_d3q27_energy_tile.cuh"
#include "pond_step_d3q125_tile.cuh"
#include "pond_step_d3q27.cuh"
#include "pond_step_point.cuh"
#include "pond_step_weno3d.cuh"
#include "pond_step_d3q125_weno_tile.cuh"

namespace pond {

int ctx_alloc(pond_ctx* c) {
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
  if ((e = cudaEventCreate(&c->ev1)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
  const size_t N = (size_t)c->N;
  for (int b = 0; b < 2; b++) {
    if (cudaMalloc(&c->f[b], (size_t)c->Q * N * c->elem) != cudaSuccess ||
        cudaMalloc(&c->rho[b], N * c->elem) != cudaSuccess || cudaMalloc(&c->g[b], 4 * N * c->elem) != cudaSuccess ||
        (c->p.ddf && cudaMalloc(&c->h[b], (size_t)c->Q * N * c->elem) != cudaSuccess)) {
      cudaGetLastError();
      return set_error(POND_ERR_NOMEM, "state buffers (%zu bytes each)",
                       (size_t)(c->Q * (c->p.ddf ? 2 : 1) + 5) * N * c->elem);
    }
  }
  if (cudaMalloc(&c->d_sums, sizeof(StepSums)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(POND_ERR_NOMEM, "step sums");
  }
  if ((e = cudaMallocHost(&c->h_sums, sizeof(StepSums))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
  std::memset(c->h_sums, 0, sizeof(StepSums));
  return mesh_alloc(c);
}

void ctx_free(pond_ctx* c) {
  pipe_free(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  mesh_free(c);
  for (int b = 0; b < 2; b++) {
    cudaFree(c->f[b]); cudaFree(c->rho[b]); cudaFree(c->g[b]); cudaFree(c->h[b]);
    c->f[b] = c->rho[b] = c->g[b] = c->h[b] = nullptr;
  }
  cudaFree(c->d_sums); c->d_sums = nullptr;
  cudaFree(c->niter); c->niter = nullptr;
  cudaFree(c->guess); c->guess = nullptr;
  cudaFree(c->g_hist); c->g_hist = nullptr;
  if (c->h_sums) cudaFreeHost(c->h_sums);
  c->h_sums = nullptr;
  if (c->staging) cudaFreeHost(c->staging);
  c->staging = nullptr;
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->ev0 = c->ev1 = nullptr;
  c->stream = nullptr;
}

static int ensure_staging(pond_ctx* c, size_t bytes) {
  if (c->staging_bytes >= bytes) return POND_OK;
  if (c->staging) cudaFreeHost(c->staging);
  c->staging = nullptr;
  c->staging_bytes = 0;
  cudaError_t e = cudaMallocHost(&c->staging, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost staging");
  c->staging_bytes = bytes;
  return POND_OK;
}

static constexpr size_t CHUNK = size_t(1) << 22;  // elements per staged copy

int upload(pond_ctx* c, const double* src, size_t count, void* dst) {
  if (c->elem == 8) {
    cudaError_t e = cudaMemcpyAsync(dst, src, count * 8, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? POND_OK : cuda_fail(e, "upload");
  }
  int st = ensure_staging(c, CHUNK * 4);
  if (st != POND_OK) return st;
  float* stg = (float*)c->staging;
  for (size_t o = 0; o < count; o += CHUNK) {
    const size_t n = count - o < CHUNK ? count - o : CHUNK;
    for (size_t i = 0; i < n; i++) stg[i] = (float)src[o + i];
    cudaError_t e = cudaMemcpyAsync((float*)dst + o, stg, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload");
  }
  return POND_OK;
}

int download(pond_ctx* c, const void* src, size_t count, double* dst) {
  if (c->elem == 8) {
    cudaError_t e = cudaMemcpyAsync(dst, src, count * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? POND_OK : cuda_fail(e, "download");
  }
  int st = ensure_staging(c, CHUNK * 4);
  if (st != POND_OK) return st;
  float* stg = (float*)c->staging;
  for (size_t o = 0; o < count; o += CHUNK) {
    const size_t n = count - o < CHUNK ? count - o : CHUNK;
    cudaError_t e = cudaMemcpyAsync(stg, (const float*)src + o, n * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "download");
    for (size_t i = 0; i < n; i++) dst[o + i] = stg[i];
  }
  return POND_OK;
}

// ---------------------------------------------------------------- sums of a state
// calcTotMoments (update.cu:52-69): active nodes only when a mask is given,
// weighted by half the distance between the node's neighbours (1D, periodic)
// when positions are given
template <typename R>
__global__ void state_sums_kernel(const R* rho, const R* g, long long N, double dim, double kdx, StepSums* out,
                                  const uint8_t* mask, const double* pos) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  NodeSums ns = {0, 0, 0, 0, 0, 0, 0ull, 0ull, 0ull, 0};
  if (n < N && (mask == nullptr || mask[n] != 0)) {
    const double r = rho[n], u0 = g[n], u1 = g[N + n], u2 = g[2 * N + n], T = g[3 * N + n];
    const double u2s = u0 * u0 + u1 * u1 + u2 * u2;
    double d = 1.0;
    if (pos) {
      const double pm = pos[n == 0 ? N - 1 : n - 1];
      double pp = pos[n + 1 == N ? 0 : n + 1];
      if (pp < pm) pp += double(N);
      d = 0.5 * (pp - pm);
    }
    ns.mass = r * d; ns.m0 = r * u0 * d; ns.m1 = r * u1 * d; ns.m2 = r * u2 * d;
    ns.enrg = r * (u2s + dim * T) * d;
    ns.k = kdx * u2s;
  }
  reduce_and_commit(ns, out);
}

static double kdx_of(const pond_ctx* c) {
  const double PI = 3.14159265358979323846;
  return 0.5 / (8 * PI * PI * PI) * (2 * PI / c->p.Nx) * (2 * PI / c->p.Ny) * (2 * PI / c->p.Nz);
}

int state_sums(pond_ctx* c, pond_diag* out) {
  cudaError_t e = cudaMemsetAsync(c->d_sums, 0, sizeof(StepSums), c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "memset");
  const int th = 256;
  const unsigned blocks = (unsigned)((c->N + th - 1) / th);
  const double dim = lattice_dim(c->p.lattice) + (c->p.ddf ? c->p.ddf_dof : 0);  // total energy's degrees
  const uint8_t* mask = c->mask[0] ? c->mask[c->mask_cur] : nullptr;
  if (c->elem == 8)
    state_sums_kernel<double><<<blocks, th, 0, c->stream>>>((const double*)c->rho[c->cur], (const double*)c->g[c->cur],
                                                            c->N, dim, kdx_of(c), c->d_sums, mask, c->pos);
  else
    state_sums_kernel<float><<<blocks, th, 0, c->stream>>>((const float*)c->rho[c->cur], (const float*)c->g[c->cur],
                                                           c->N, dim, kdx_of(c), c->d_sums, mask, c->pos);
  StepSums s;
  e = cudaMemcpyAsync(&s, c->d_sums, sizeof(s), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "state sums");
  out->mass = s.mass;
  out->moment[0] = s.mom[0]; out->moment[1] = s.mom[1]; out->moment[2] = s.mom[2];
  out->enrg = s.enrg;
  out->k = s.k;
  return POND_OK;
}

// ---------------------------------------------------------------- dispatch
template <int LAT, int N, typename R> static void launch_point(const StepArgs<R>& a, cudaStream_t s) {
  if (Lattice<LAT>::D == 1) {
    dim3 blk(128, 1, 1), grd((a.nx + 127) / 128, a.ny, a.nz);
    pull_point_kernel<LAT, N, R><<<grd, blk, 0, s>>>(a);
  } else {
    dim3 blk(32, 4, 1), grd((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
    pull_point_kernel<LAT, N, R><<<grd, blk, 0, s>>>(a);
  }
}

// One step from in[] = {f, rho, g} to out[] (device buffers of the context's
// precision); with in == nullptr the context's own double buffer is used.
template <typename R> static int launch_typed(pond_ctx* c, const void* const* in = nullptr, void* const* out = nullptr) {
  StepArgs<R> a;
  const int i = c->cur, o = 1 - c->cur;
  if (in) {
    a.f_in = (const R*)in[0]; a.rho_in = (const R*)in[1]; a.g_in = (const R*)in[2];
    a.f_out = (R*)out[0]; a.rho_out = (R*)out[1]; a.g_out = (R*)out[2];
  } else {
    a.f_in = (const R*)c->f[i]; a.rho_in = (const R*)c->rho[i]; a.g_in = (const R*)c->g[i];
    a.f_out = (R*)c->f[o]; a.rho_out = (R*)c->rho[o]; a.g_out = (R*)c->g[o];
  }
  a.guess = (c->p.learned && !in) ? c->guess : nullptr;
  a.niter_out = c->keep_niter ? c->niter : nullptr;
  a.sums = c->d_sums;
  a.nx = (int)c->p.Nx; a.ny = (int)c->p.Ny; a.nz = (int)c->p.Nz;
  a.N = c->N;
  for (int k = 0; k < 3; k++) a.bc[k] = c->p.bc[k];
  a.dtau = 1.0 / c->p.tau;
  a.tol_abs = c->p.tol_abs; a.tol_rel = c->p.tol_rel;
  a.tolg_abs = c->tolg_abs >= 0 ? c->tolg_abs : c->p.tol_abs;
  a.tolg_rel = c->tolg_rel >= 0 ? c->tolg_rel : c->p.tol_rel;
  a.max_iter = c->p.max_iter;
  a.kdx = kdx_of(c);
  a.mask = c->mask[0] ? c->mask[c->mask_cur] : nullptr;
  a.pos = c->pos;
  for (int k = 0; k < 3; k++)
    if (c->p.bc[k] == POND_BC_INFLOW && !c->have_inflow)
      return set_error(POND_ERR_STATE, "an inflow boundary needs pond_set_inflow before stepping");
  for (int k = 0; k < 5; k++) a.inflow[k] = c->inflow[k];
  cudaError_t e = cudaMemsetAsync(c->d_sums, 0, sizeof(StepSums), c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "memset sums");
  cudaStream_t s = c->stream;
  if (c->p.ddf) {  // energy populations: D1Q5 and D3Q27 (pond_create checks), context buffers only
    if (in) return set_error(POND_ERR_UNSUPPORTED, "explicit step buffers carry no energy populations");
    a.h_in = (const R*)c->h[i];
    a.h_out = (R*)c->h[o];
    a.dof = c->p.ddf_dof;
    if (c->p.lattice == POND_D3Q125) {
      if constexpr (std::is_same<R, float>::value) {
        const size_t smem = sizeof(d125t::SmemT<true>);
        e = cudaFuncSetAttribute(d125t::pull_d3q125_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        const dim3 grd((a.nx + d125t::T - 1) / d125t::T, (a.ny + d125t::T - 1) / d125t::T,
                       (a.nz + d125t::T - 1) / d125t::T);
        d125t::pull_d3q125_tile_kernel<true><<<grd, d125t::THREADS, smem, s>>>(a);
        e = cudaGetLastError();
        return e == cudaSuccess ? POND_OK : cuda_fail(e, "step kernel launch");
      } else {  // float64: 2^3 tiles, the two population sets of a 4^3 tile would not fit
        constexpr int TT = 2;
        const size_t smem = sizeof(d125t::SmemT<true, double, TT>);
        e = cudaFuncSetAttribute(d125t::pull_d3q125_tile_kernel<true, double, TT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        const dim3 grd((a.nx + TT - 1) / TT, (a.ny + TT - 1) / TT, (a.nz + TT - 1) / TT);
        d125t::pull_d3q125_tile_kernel<true, double, TT><<<grd, d125t::THREADS, smem, s>>>(a);
        e = cudaGetLastError();
        return e == cudaSuccess ? POND_OK : cuda_fail(e, "step kernel launch");
      }
    }
    if (c->p.lattice == POND_D3Q27) {
      if constexpr (std::is_same<R, float>::value) {
        if (c->p.interp == POND_LAGR2 || c->p.interp == POND_LAGR3 || c->p.interp == POND_LAGR4) {
          const dim3 grd((a.nx + d27e::TX - 1) / d27e::TX, (a.ny + d27e::TY - 1) / d27e::TY,
                         (a.nz + d27e::TZ - 1) / d27e::TZ);
          auto kern = c->p.interp == POND_LAGR2   ? d27e::pull_d3q27_energy_tile_kernel<2>
                      : c->p.interp == POND_LAGR3 ? d27e::pull_d3q27_energy_tile_kernel<3>
                                                  : d27e::pull_d3q27_energy_tile_kernel<4>;
          e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d27e::SMEM_BYTES);
          if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
          kern<<<grd, d27e::THREADS, d27e::SMEM_BYTES, s>>>(a);
          e = cudaGetLastError();
          return e == cudaSuccess ? POND_OK : cuda_fail(e, "step kernel launch");
        }
      }
      const dim3 blk(32, 4, 1), grd((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
      switch (c->p.interp) {
        case POND_LAGR2: pull_d3q27_energy_kernel<2, R><<<grd, blk, 0, s>>>(a); break;
        case POND_LAGR3: pull_d3q27_energy_kernel<3, R><<<grd, blk, 0, s>>>(a); break;
        case POND_LAGR4: pull_d3q27_energy_kernel<4, R><<<grd, blk, 0, s>>>(a); break;
        case POND_LAGR5: pull_d3q27_energy_kernel<5, R><<<grd, blk, 0, s>>>(a); break;
        default: return set_error(POND_ERR_UNSUPPORTED, "scheme");
      }
      e = cudaGetLastError();
      return e == cudaSuccess ? POND_OK : cuda_fail(e, "step kernel launch");
    }
    const unsigned g1 = (unsigned)((a.nx + 127) / 128);
    switch (c->p.interp) {
      case POND_LAGR2: pull_1d_energy_kernel<POND_LAGR2, R><<<g1, 128, 0, s>>>(a); break;
      case POND_LAGR3: pull_1d_energy_kernel<POND_LAGR3, R><<<g1, 128, 0, s>>>(a); break;
      case POND_LAGR4: pull_1d_energy_kernel<POND_LAGR4, R><<<g1, 128, 0, s>>>(a); break;
      case POND_LAGR5: pull_1d_energy_kernel<POND_LAGR5, R><<<g1, 128, 0, s>>>(a); break;
      case POND_TVD: pull_1d_energy_kernel<POND_TVD, R><<<g1, 128, 0, s>>>(a); break;
      case POND_WENO5:
      case POND_WENO5_ROW: pull_1d_energy_kernel<POND_WENO5, R><<<g1, 128, 0, s>>>(a); break;
      default: return set_error(POND_ERR_UNSUPPORTED, "scheme");
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? POND_OK : cuda_fail(e, "step kernel launch");
  }
  if (c->p.lattice != POND_D1Q5 && (c->p.interp == POND_WENO5 || c->p.interp == POND_WENO5_ROW)) {
    const bool fix = c->p.interp == POND_WENO5_ROW;
    if (c->p.lattice == POND_D3Q27) {
      const long long per = (long long)w3d::WARPS * w3d::Geo<POND_D3Q27>::NPW;
      const unsigned grd = (unsigned)((a.N + per - 1) / per);
      if (fix) w3d::pull_weno3d_kernel<POND_D3Q27, R, true><<<grd, w3d::THREADS, 0, s>>>(a);
      else w3d::pull_weno3d_kernel<POND_D3Q27, R, false><<<grd, w3d::THREADS, 0, s>>>(a);
    } else if (std::is_same<R, float>::value && fix) {  // staged tile (float32, row through the departure point)
      if constexpr (std::is_same<R, float>::value) {
        const size_t smem = sizeof(d125w::Smem);
        e = cudaFuncSetAttribute(d125w::pull_d3q125_weno_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        const dim3 grd((a.nx + d125w::TX - 1) / d125w::TX, (a.ny + d125w::TY - 1) / d125w::TY,
                       (a.nz + d125w::TZ - 1) / d125w::TZ);
        d125w::pull_d3q125_weno_tile_kernel<<<grd, d125w::THREADS, smem, s>>>(a);
      }
    } else {
      const long long per = (long long)w3d::WARPS * w3d::Geo<POND_D3Q125>::NPW;
      const unsigned grd = (unsigned)((a.N + per - 1) / per);
      if (fix) w3d::pull_weno3d_kernel<POND_D3Q125, R, true><<<grd, w3d::THREADS, 0, s>>>(a);
      else w3d::pull_weno3d_kernel<POND_D3Q125, R, false><<<grd, w3d::THREADS, 0, s>>>(a);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? POND_OK : cuda_fail(e, "step kernel launch");
  }
  switch (c->p.lattice) {
    case POND_D1Q5:
      switch (c->p.interp) {
        case POND_LAGR2: launch_point<POND_D1Q5, 2, R>(a, s); break;
        case POND_LAGR3: launch_point<POND_D1Q5, 3, R>(a, s); break;
        case POND_LAGR4: launch_point<POND_D1Q5, 4, R>(a, s); break;
        case POND_LAGR5: launch_point<POND_D1Q5, 5, R>(a, s); break;
        case POND_TVD:
          pull_1d_scheme_kernel<POND_TVD, R><<<(a.nx + 127) / 128, 128, 0, s>>>(a);
          break;
        case POND_WENO5:
        case POND_WENO5_ROW:  // one row on a 1D grid: both read row 0
          pull_1d_scheme_kernel<POND_WENO5, R><<<(a.nx + 127) / 128, 128, 0, s>>>(a);
          break;
        case POND_GAP2:
          pull_1d_mesh_kernel<POND_GAP2, R><<<(a.nx + 127) / 128, 128, 0, s>>>(a);
          break;
        case POND_NONUNIFORM3:
          pull_1d_mesh_kernel<POND_NONUNIFORM3, R><<<(a.nx + 127) / 128, 128, 0, s>>>(a);
          break;
        default: return set_error(POND_ERR_UNSUPPORTED, "scheme");
      }
      break;
    case POND_D3Q27:
      if constexpr (std::is_same<R, float>::value) {
        if (c->p.interp >= POND_LAGR2 && c->p.interp <= POND_LAGR4) {
          dim3 blk(d27::TX, d27::TY, d27::TZ);
          dim3 grd((a.nx + d27::TX - 1) / d27::TX, (a.ny + d27::TY - 1) / d27::TY, (a.nz + d27::TZ - 1) / d27::TZ);
          void (*kern)(StepArgs<float>) = c->p.interp == POND_LAGR2   ? d27::pull_d3q27_tile_kernel<2>
                                          : c->p.interp == POND_LAGR3 ? d27::pull_d3q27_tile_kernel<3>
                                                                      : d27::pull_d3q27_tile_kernel<4>;
          e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d27::SMEM_BYTES);
          if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
          kern<<<grd, blk, d27::SMEM_BYTES, s>>>(a);
          break;
        }
      }
      switch (c->p.interp) {
        case POND_LAGR2: launch_point<POND_D3Q27, 2, R>(a, s); break;
        case POND_LAGR3: launch_point<POND_D3Q27, 3, R>(a, s); break;
        case POND_LAGR4: launch_point<POND_D3Q27, 4, R>(a, s); break;
        case POND_LAGR5: launch_point<POND_D3Q27, 5, R>(a, s); break;
        default: return set_error(POND_ERR_UNSUPPORTED, "scheme");
      }
      break;
    case POND_D3Q125: {  // staged tile, reference-gauge transfer (float64: one CTA per SM)
      const size_t smem = sizeof(d125t::SmemT<false, R>);
      e = cudaFuncSetAttribute(d125t::pull_d3q125_tile_kernel<false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
      const dim3 grd((a.nx + d125t::T - 1) / d125t::T, (a.ny + d125t::T - 1) / d125t::T,
                     (a.nz + d125t::T - 1) / d125t::T);
      d125t::pull_d3q125_tile_kernel<false, R><<<grd, d125t::THREADS, smem, s>>>(a);
      break;
    }
    default: return set_error(POND_ERR_UNSUPPORTED, "lattice");
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "step kernel launch");
  return POND_OK;
}

int launch_step_io(pond_ctx* c, const void* const in[3], void* const out[3]) {
  return c->elem == 8 ? launch_typed<double>(c, in, out) : launch_typed<float>(c, in, out);
}

int launch_step(pond_ctx* c) {
  if (c->keep_history && c->g_hist) {  // g^{n-1}, before this step overwrites it
    cudaError_t e = cudaMemcpyAsync(c->g_hist, c->g[1 - c->cur], 4 * (size_t)c->N * c->elem,
                                    cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "history copy");
  }
  if (c->p.learned) {
    int st = run_predictor(c);
    if (st != POND_OK) return st;
  }
  return c->elem == 8 ? launch_typed<double>(c) : launch_typed<float>(c);
}

}  // namespace pond
