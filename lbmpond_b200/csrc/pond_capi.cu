// C ABI of the PonD step library: context lifetime, state upload/download,
// built-in initial conditions, the step driver and diagnostics.
// The reference keeps this state in globals (parsHost, __constant__ pars,
// structs.cuh:150-151) and exits on any CUDA error (params.h:74-81); here a
// context owns it and every entry point returns a status.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pond_internal.h"

namespace pond {

thread_local std::string g_last_error;

int set_error(int status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(POND_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int lattice_q(int lattice) {
  switch (lattice) {
    case POND_D1Q5: return 5;
    case POND_D3Q27: return 27;
    case POND_D3Q125: return 125;
    default: return 0;
  }
}

double lattice_weight_host(int lattice, int ref_index) {
  // population weights in reference order
  switch (lattice) {
    case POND_D1Q5: return lattice_weight_t<POND_D1Q5>(ref_index);
    case POND_D3Q125: return lattice_weight_t<POND_D3Q125>(ref_index);
    case POND_D3Q27: {
      for (int t = 0; t < 27; t++)
        if (Lattice<POND_D3Q27>::ref(t / 9, (t / 3) % 3, t % 3) == ref_index) return lattice_weight_t<POND_D3Q27>(t);
      return 0;
    }
    default: return 0;
  }
}

double lattice_tlat(int lattice) { return lattice == POND_D3Q27 ? 1.0 / 3.0 : 1.0; }

// velocities and weights of every population in the reference's order
template <int LAT> static void tables_of(double* xi, double* w) {
  using L = Lattice<LAT>;
  for (int t = 0; t < L::Q; t++) {  // tensor class t -> reference population ref(cx, cy, cz)
    const int cx = L::D == 1 ? t : t / (L::Q1 * L::Q1);
    const int cy = L::D == 1 ? 0 : (t / L::Q1) % L::Q1, cz = L::D == 1 ? 0 : t % L::Q1;
    const int q = L::ref(cx, cy, cz);
    if (xi) {
      xi[3 * q] = L::xi1(cx);
      xi[3 * q + 1] = L::D == 1 ? 0.0 : L::xi1(cy);
      xi[3 * q + 2] = L::D == 1 ? 0.0 : L::xi1(cz);
    }
    if (w) w[q] = lattice_weight_t<LAT>(t);
  }
}
double lattice_dim(int lattice) { return lattice == POND_D1Q5 ? 1.0 : 3.0; }

// Checks shared by every entry point that runs a step from a pond_params:
// boundaries, tau, the iteration cap and the tolerances.  The cap bounds the
// length of one step launch on a shared GPU.
int check_step_params(const pond_params* p) {
  for (int a = 0; a < 3; a++)
    if (p->bc[a] < POND_BC_PERIODIC || p->bc[a] > POND_BC_INFLOW) return set_error(POND_ERR_ARG, "bad bc[%d]", a);
  if (!(p->tau > 0.5) || !std::isfinite(p->tau)) return set_error(POND_ERR_ARG, "tau must be a finite value > 0.5");
  if (p->max_iter < 1 || p->max_iter > 100000) return set_error(POND_ERR_ARG, "max_iter out of range (1..100000)");
  if (!(p->tol_abs >= 0) || !(p->tol_rel >= 0) || !std::isfinite(p->tol_abs) || !std::isfinite(p->tol_rel))
    return set_error(POND_ERR_ARG, "tolerances must be finite and >= 0");
  return POND_OK;
}

bool scheme_supported(int lattice, int interp) {
  switch (lattice) {
    case POND_D1Q5:
      return (interp >= POND_LAGR2 && interp <= POND_LAGR5) || interp == POND_TVD || interp == POND_WENO5 ||
             interp == POND_WENO5_ROW || interp == POND_GAP2 || interp == POND_NONUNIFORM3;
    case POND_D3Q27: return (interp >= POND_LAGR2 && interp <= POND_LAGR5) || interp == POND_WENO5 ||
                            interp == POND_WENO5_ROW;
    case POND_D3Q125: return interp == POND_FIXED3 || interp == POND_WENO5 || interp == POND_WENO5_ROW;
    default: return false;
  }
}

// ---------------------------------------------------------------- fill kernel
// init.cu:2-108 (fill) + lbpack.cu:15-21 (Cell::set_base): rho, u, T from
// the chosen initial condition, f_i = w_i * rho, written to both buffers.
struct FillArgs {
  int ic;
  double p[8];
  int nx, ny, nz;
  long long N;
  int Q;
  double dim;
  double dof;  // extra degrees of freedom of the energy populations
  double w[125];
};

template <typename R>
__global__ void fill_kernel(FillArgs a, R* f0, R* rho0, R* g0, R* f1, R* rho1, R* g1, R* h0, R* h1) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  const int x = n % a.nx, y = (n / a.nx) % a.ny, z = n / ((long long)a.nx * a.ny);
  double rho = 1, ux = 0, uy = 0, uz = 0, T = 1;
  const double PI = 3.14159265358979323846;
  switch (a.ic) {
    case POND_IC_ACOUSTIC: {  // init.cu:43-50, centred at x = 0, one wavelength over Nx
      const double T0 = a.p[0], Ampl = a.p[1], gamma = a.p[2], P0 = 1;
      const double sn = sin(x * 2 * PI / a.nx);
      const double P = P0 + Ampl * sn;
      T = T0 * pow(P, (gamma - 1) / gamma);
      rho = P / T;
      ux = Ampl * sn / P0 * T0 / sqrt(gamma * T0);
      break;
    }
    case POND_IC_SOD_X: {
      const bool left = x < a.p[0] * a.nx;
      rho = left ? a.p[1] : a.p[4];
      ux = left ? a.p[2] : a.p[5];
      T = left ? a.p[3] : a.p[6];
      break;
    }
    case POND_IC_SPHERE: {  // unit box, cell-centred coordinates
      const double px = (x + 0.5) / a.nx - a.p[0], py = (y + 0.5) / a.ny - a.p[1], pz = (z + 0.5) / a.nz - a.p[2];
      const bool in = px * px + py * py + pz * pz < a.p[3] * a.p[3];
      rho = in ? a.p[4] : a.p[6];
      T = in ? a.p[5] : a.p[7];
      break;
    }
    case POND_IC_TGV: {  // compressible Taylor-Green vortex on [0, 2pi)^3
      const double U0 = a.p[0], T0 = a.p[1], r0 = a.p[2];
      const double X = x * 2 * PI / a.nx, Y = y * 2 * PI / a.ny, Z = z * 2 * PI / a.nz;
      ux = U0 * sin(X) * cos(Y) * cos(Z);
      uy = -U0 * cos(X) * sin(Y) * cos(Z);
      uz = 0;
      rho = r0;
      const double P = r0 * T0 + r0 * U0 * U0 / 16. * (cos(2 * X) + cos(2 * Y)) * (cos(2 * Z) + 2);
      T = P / rho;
      break;
    }
    default: {
      rho = a.p[0]; ux = a.p[1]; uy = a.p[2]; uz = a.p[3]; T = a.p[4];
      break;
    }
  }
  if (a.dim == 1) { uy = 0; uz = 0; }
  for (int q = 0; q < a.Q; q++) {
    const R fv = R(a.w[q] * rho);
    f0[(long long)q * a.N + n] = fv;
    f1[(long long)q * a.N + n] = fv;
  }
  rho0[n] = R(rho); rho1[n] = R(rho);
  const R gv[4] = {R(ux), R(uy), R(uz), R(T)};
  for (int k = 0; k < 4; k++) { g0[k * a.N + n] = gv[k]; g1[k * a.N + n] = gv[k]; }
  if (h0) {  // equilibrium energy populations, class order -> reference order
    const double U[3] = {ux, uy, uz};
    R h[125];
    if (a.Q == 5) {
      energy_equilibrium<POND_D1Q5, R>(rho, U, T, a.dof, h);
      for (int q = 0; q < 5; q++) { h0[(long long)q * a.N + n] = h[q]; h1[(long long)q * a.N + n] = h[q]; }
    } else if (a.Q == 125) {  // class order is the population order
      energy_equilibrium<POND_D3Q125, R>(rho, U, T, a.dof, h);
      for (int q = 0; q < 125; q++) { h0[(long long)q * a.N + n] = h[q]; h1[(long long)q * a.N + n] = h[q]; }
    } else {
      energy_equilibrium<POND_D3Q27, R>(rho, U, T, a.dof, h);
      for (int t = 0; t < 27; t++) {
        const long long q = Lattice<POND_D3Q27>::ref(t / 9, (t / 3) % 3, t % 3);
        h0[q * a.N + n] = h[t];
        h1[q * a.N + n] = h[t];
      }
    }
  }
}

}  // namespace pond

using namespace pond;

extern "C" {

int pond_abi_version(void) { return POND_ABI_VERSION; }

const char* pond_status_string(int s) {
  switch (s) {
    case POND_OK: return "ok";
    case POND_ERR_ARG: return "invalid argument";
    case POND_ERR_CUDA: return "CUDA runtime error";
    case POND_ERR_NOMEM: return "out of device memory";
    case POND_ERR_STATE: return "call out of order";
    case POND_ERR_UNSUPPORTED: return "unsupported lattice/scheme/precision";
    case POND_ERR_NOT_CONVERGED: return "iteration did not converge";
    default: return "unknown status";
  }
}

const char* pond_last_error_string(void) { return g_last_error.c_str(); }

int pond_q(int lattice) { return lattice_q(lattice); }

int pond_lattice_tables(int lattice, double* xi, double* w, double* tlat_dim) {
  switch (lattice) {
    case POND_D1Q5: tables_of<POND_D1Q5>(xi, w); break;
    case POND_D3Q27: tables_of<POND_D3Q27>(xi, w); break;
    case POND_D3Q125: tables_of<POND_D3Q125>(xi, w); break;
    default: return set_error(POND_ERR_ARG, "unknown lattice %d", lattice);
  }
  if (tlat_dim) { tlat_dim[0] = lattice_tlat(lattice); tlat_dim[1] = lattice_dim(lattice); }
  return POND_OK;
}

int pond_params_default(int lattice, pond_params* out) {
  if (!out) return set_error(POND_ERR_ARG, "pond_params_default: null output");
  if (!lattice_q(lattice)) return set_error(POND_ERR_ARG, "unknown lattice %d", lattice);
  std::memset(out, 0, sizeof(*out));
  out->lattice = lattice;
  out->Nx = lattice == POND_D1Q5 ? 128 : 32;
  out->Ny = lattice == POND_D1Q5 ? 1 : 32;
  out->Nz = lattice == POND_D1Q5 ? 1 : 32;
  out->interp = lattice == POND_D3Q125 ? POND_FIXED3 : POND_LAGR4;
  out->precision = POND_FP32;
  out->tau = 0.9;       // structs.cuh:98
  out->dt = 1.0;
  out->tol_abs = 1e-7;  // float32 accumulation noise is ~2e-8 at rho~1; the reference's 1e-12 suits float64 only
  out->tol_rel = 1e-6;
  out->max_iter = 100;  // steps.cu:422
  out->device = 0;
  return POND_OK;
}

int pond_create(const pond_params* p, pond_ctx** out) {
  if (!p || !out) return set_error(POND_ERR_ARG, "pond_create: null argument");
  *out = nullptr;
  const int Q = lattice_q(p->lattice);
  if (!Q) return set_error(POND_ERR_ARG, "unknown lattice %d", p->lattice);
  if (p->Nx <= 0 || p->Ny <= 0 || p->Nz <= 0 || p->Nx > (1 << 30) || p->Ny > (1 << 30) || p->Nz > (1 << 30))
    return set_error(POND_ERR_ARG, "grid %lldx%lldx%lld out of range", (long long)p->Nx, (long long)p->Ny,
                     (long long)p->Nz);
  const long long N = p->Nx * p->Ny * p->Nz;
  if (N > (1LL << 31) - 1) return set_error(POND_ERR_ARG, "grid has more than 2^31-1 nodes");
  if (p->precision != POND_FP32 && p->precision != POND_FP64)
    return set_error(POND_ERR_ARG, "unknown precision %d", p->precision);
  if (!scheme_supported(p->lattice, p->interp))
    return set_error(POND_ERR_UNSUPPORTED, "interpolation %d is not available for lattice %d", p->interp, p->lattice);
  const int vst = check_step_params(p);
  if (vst != POND_OK) return vst;
  {
    bool inflow = false;
    for (int a = 0; a < 3; a++) inflow = inflow || p->bc[a] == POND_BC_INFLOW;
    const bool weno3d = p->lattice != POND_D1Q5 && (p->interp == POND_WENO5 || p->interp == POND_WENO5_ROW);
    if (inflow && !weno3d && !(p->lattice == POND_D3Q125 && p->interp == POND_FIXED3))
      return set_error(POND_ERR_UNSUPPORTED,
                       "the inflow boundary runs with the D3Q27/D3Q125 WENO5 schemes and the D3Q125 fixed-origin quadratic");
    if (weno3d && p->ddf)
      return set_error(POND_ERR_UNSUPPORTED, "WENO5 on the 3D lattices carries no energy populations");
  }
  if (p->lattice == POND_D1Q5 && (p->interp == POND_TVD || p->interp == POND_WENO5 || p->interp == POND_WENO5_ROW) &&
      (p->Ny != 1 || p->Nz != 1))
    return set_error(POND_ERR_UNSUPPORTED, "TVD/WENO5 run on 1D grids (Ny = Nz = 1)");
  if (p->lattice == POND_D1Q5 && mesh_scheme(p->interp)) {
    if (p->Ny != 1 || p->Nz != 1 || p->Nx < 3) return set_error(POND_ERR_UNSUPPORTED, "mesh schemes run on 1D grids, Nx >= 3");
    if (p->bc[0] != POND_BC_PERIODIC) return set_error(POND_ERR_UNSUPPORTED, "mesh schemes are periodic");
    if (p->ddf || p->learned) return set_error(POND_ERR_UNSUPPORTED, "mesh schemes carry neither energy populations nor the learned start");
  }
  if (p->ddf != 0 && p->ddf != 1) return set_error(POND_ERR_ARG, "ddf must be 0 or 1");
  if (p->ddf) {
    const bool d1 = p->lattice == POND_D1Q5 && p->Ny == 1 && p->Nz == 1;
    const bool d27 = p->lattice == POND_D3Q27 && p->interp >= POND_LAGR2 && p->interp <= POND_LAGR5;
    const bool d125 = p->lattice == POND_D3Q125;
    if (!d1 && !d27 && !d125)
      return set_error(POND_ERR_UNSUPPORTED, "energy populations run on D1Q5 1D grids, D3Q27 (Lagrange 2-5) and D3Q125");
    if (p->ddf_dof < 0 || p->ddf_dof > 1000) return set_error(POND_ERR_ARG, "ddf_dof must be in 0..1000");
    if (p->learned) return set_error(POND_ERR_UNSUPPORTED, "the learned start does not carry energy populations");
  }

  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (p->device < 0 || p->device >= ndev) return set_error(POND_ERR_ARG, "device %d not present", p->device);
  e = cudaSetDevice(p->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");

  pond_ctx* c = new (std::nothrow) pond_ctx();
  if (!c) return set_error(POND_ERR_NOMEM, "host allocation failed");
  c->p = *p;
  c->Q = Q;
  c->N = N;
  c->elem = p->precision == POND_FP64 ? 8 : 4;
  int st = ctx_alloc(c);
  if (st != POND_OK) {
    ctx_free(c);
    delete c;
    return st;
  }
  *out = c;
  return POND_OK;
}

int pond_destroy(pond_ctx* c) {
  if (!c) return POND_OK;
  cudaSetDevice(c->p.device);
  ctx_free(c);
  delete c;
  return POND_OK;
}

int pond_get_params(const pond_ctx* c, pond_params* out) {
  if (!c || !out) return set_error(POND_ERR_ARG, "null argument");
  *out = c->p;
  return POND_OK;
}

void* pond_stream(pond_ctx* c) { return c ? (void*)c->stream : nullptr; }

int pond_device_state(pond_ctx* c, void** f, void** rho, void** g) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (f) *f = c->f[c->cur];
  if (rho) *rho = c->rho[c->cur];
  if (g) *g = c->g[c->cur];
  return POND_OK;
}

int pond_init(pond_ctx* c, int ic, const double* prm, int nprm) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (ic < POND_IC_ACOUSTIC || ic > POND_IC_UNIFORM) return set_error(POND_ERR_ARG, "unknown initial condition %d", ic);
  if (nprm < 0 || nprm > 8 || (nprm > 0 && !prm)) return set_error(POND_ERR_ARG, "bad initial-condition parameters");
  cudaSetDevice(c->p.device);
  FillArgs a;
  std::memset(&a, 0, sizeof(a));
  a.ic = ic;
  const double dim = lattice_dim(c->p.lattice);
  // defaults: the reference's shipped acoustic wave (init.cu:8-9,44-45)
  const double defaults[5][8] = {
      {0.1, 0.02, (dim + 2.0) / dim, 0, 0, 0, 0, 0},
      {0.5, 1.0, 0.0, 0.01, 0.125, 0.0, 0.008, 0},
      {0.5, 0.5, 0.5, 0.2, 1.0, 0.0625, 0.125, 0.05},
      {0.05, 0.1, 1.0, (dim + 2.0) / dim, 0, 0, 0, 0},
      {1.0, 0.0, 0.0, 0.0, 0.1, 0, 0, 0}};
  for (int k = 0; k < 8; k++) a.p[k] = k < nprm ? prm[k] : defaults[ic][k];
  a.nx = (int)c->p.Nx; a.ny = (int)c->p.Ny; a.nz = (int)c->p.Nz;
  a.N = c->N;
  a.Q = c->Q;
  a.dim = dim;
  a.dof = c->p.ddf_dof;
  for (int q = 0; q < c->Q; q++) a.w[q] = lattice_weight_host(c->p.lattice, q);
  const int th = 256;
  const unsigned blocks = (unsigned)((c->N + th - 1) / th);
  const int o = c->cur, n = 1 - c->cur;
  if (c->elem == 8)
    fill_kernel<double><<<blocks, th, 0, c->stream>>>(a, (double*)c->f[o], (double*)c->rho[o], (double*)c->g[o],
                                                       (double*)c->f[n], (double*)c->rho[n], (double*)c->g[n],
                                                       (double*)c->h[o], (double*)c->h[n]);
  else
    fill_kernel<float><<<blocks, th, 0, c->stream>>>(a, (float*)c->f[o], (float*)c->rho[o], (float*)c->g[o],
                                                      (float*)c->f[n], (float*)c->rho[n], (float*)c->g[n],
                                                      (float*)c->h[o], (float*)c->h[n]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fill kernel launch");
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "fill kernel");
  { const int ms = mesh_reset(c); if (ms != POND_OK) return ms; }  // fill sets every Cinfo::set (init.cu:106)
  c->initialized = true;
  c->istep = 0;
  c->curtime = 0;
  c->have_sums = false;
  return POND_OK;
}

int pond_set_state(pond_ctx* c, const double* f, const double* rho, const double* g) {
  if (!c || !rho || !g) return set_error(POND_ERR_ARG, "pond_set_state: null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  cudaSetDevice(c->p.device);
  const long long N = c->N;
  const int Q = c->Q;
  std::vector<double> fb;
  if (!f) {  // Cell::set_base (lbpack.cu:15-21)
    fb.resize((size_t)Q * N);
    for (int q = 0; q < Q; q++) {
      const double wq = lattice_weight_host(c->p.lattice, q);
      for (long long n = 0; n < N; n++) fb[(size_t)q * N + n] = wq * rho[n];
    }
    f = fb.data();
  }
  int st = upload(c, f, (size_t)Q * N, c->f[c->cur]);
  if (st == POND_OK) st = upload(c, rho, (size_t)N, c->rho[c->cur]);
  if (st == POND_OK) st = upload(c, g, (size_t)4 * N, c->g[c->cur]);
  if (st == POND_OK && c->p.ddf) {  // energy populations at equilibrium in every node's gauge
    std::vector<double> hb((size_t)Q * N);
    for (long long n = 0; n < N; n++) {
      const double U[3] = {g[n], g[N + n], g[2 * N + n]};
      double h[125];
      if (c->p.lattice == POND_D1Q5) {
        energy_equilibrium<POND_D1Q5, double>(rho[n], U, g[3 * N + n], c->p.ddf_dof, h);
        for (int q = 0; q < Q; q++) hb[(size_t)q * N + n] = h[q];
      } else if (c->p.lattice == POND_D3Q125) {
        energy_equilibrium<POND_D3Q125, double>(rho[n], U, g[3 * N + n], c->p.ddf_dof, h);
        for (int q = 0; q < Q; q++) hb[(size_t)q * N + n] = h[q];
      } else {
        energy_equilibrium<POND_D3Q27, double>(rho[n], U, g[3 * N + n], c->p.ddf_dof, h);
        for (int t = 0; t < 27; t++) hb[(size_t)Lattice<POND_D3Q27>::ref(t / 9, (t / 3) % 3, t % 3) * N + n] = h[t];
      }
    }
    st = upload(c, hb.data(), (size_t)Q * N, c->h[c->cur]);
  }
  if (st != POND_OK) return st;
  // the reference fills both buffers (init.cu:104-105)
  const size_t bytes[4] = {(size_t)Q * N * c->elem, (size_t)N * c->elem, (size_t)4 * N * c->elem,
                           (size_t)Q * N * c->elem};
  void* src[4] = {c->f[c->cur], c->rho[c->cur], c->g[c->cur], c->h[c->cur]};
  void* dst[4] = {c->f[1 - c->cur], c->rho[1 - c->cur], c->g[1 - c->cur], c->h[1 - c->cur]};
  for (int k = 0; k < (c->p.ddf ? 4 : 3); k++) {
    cudaError_t e = cudaMemcpyAsync(dst[k], src[k], bytes[k], cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync D2D");
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_set_state");
  c->initialized = true;
  c->have_sums = false;
  return POND_OK;
}

int pond_get_state(pond_ctx* c, double* f, double* rho, double* g) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  cudaSetDevice(c->p.device);
  int st = POND_OK;
  if (f) st = download(c, c->f[c->cur], (size_t)c->Q * c->N, f);
  if (st == POND_OK && rho) st = download(c, c->rho[c->cur], (size_t)c->N, rho);
  if (st == POND_OK && g) st = download(c, c->g[c->cur], (size_t)4 * c->N, g);
  return st;
}

int pond_set_energy(pond_ctx* c, const double* h) {
  if (!c || !h) return set_error(POND_ERR_ARG, "pond_set_energy: null argument");
  if (!c->p.ddf) return set_error(POND_ERR_STATE, "the context has no energy populations (ddf = 0)");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->initialized) return set_error(POND_ERR_STATE, "set the state before its energy populations");
  cudaSetDevice(c->p.device);
  const size_t cnt = (size_t)c->Q * c->N;
  int st = upload(c, h, cnt, c->h[c->cur]);
  if (st != POND_OK) return st;
  cudaError_t e = cudaMemcpyAsync(c->h[1 - c->cur], c->h[c->cur], cnt * c->elem, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_set_energy");
}

int pond_get_energy(pond_ctx* c, double* h) {
  if (!c || !h) return set_error(POND_ERR_ARG, "pond_get_energy: null argument");
  if (!c->p.ddf) return set_error(POND_ERR_STATE, "the context has no energy populations (ddf = 0)");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  cudaSetDevice(c->p.device);
  return download(c, c->h[c->cur], (size_t)c->Q * c->N, h);
}

int pond_get_fields(pond_ctx* c, double* rho, double* ux, double* uy, double* uz, double* T) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  cudaSetDevice(c->p.device);
  int st = POND_OK;
  const size_t N = (size_t)c->N;
  char* g = (char*)c->g[c->cur];
  double* outs[4] = {ux, uy, uz, T};
  if (rho) st = download(c, c->rho[c->cur], N, rho);
  for (int k = 0; k < 4 && st == POND_OK; k++)
    if (outs[k]) st = download(c, g + k * N * c->elem, N, outs[k]);
  return st;
}

int pond_keep_niter(pond_ctx* c, int on) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  cudaSetDevice(c->p.device);
  if (on && !c->niter) {
    cudaError_t e = cudaMalloc(&c->niter, sizeof(int) * c->N);
    if (e != cudaSuccess) { c->niter = nullptr; return set_error(POND_ERR_NOMEM, "niter buffer"); }
    cudaMemsetAsync(c->niter, 0, sizeof(int) * c->N, c->stream);
  }
  c->keep_niter = on != 0;
  return POND_OK;
}

int pond_keep_history(pond_ctx* c, int on) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  cudaSetDevice(c->p.device);
  if (on && !c->g_hist) {
    if (cudaMalloc(&c->g_hist, 4 * (size_t)c->N * c->elem) != cudaSuccess) {
      cudaGetLastError();
      c->g_hist = nullptr;
      return set_error(POND_ERR_NOMEM, "history buffer");
    }
  }
  c->keep_history = on != 0;
  return POND_OK;
}

int pond_get_niter(pond_ctx* c, int32_t* out) {
  if (!c || !out) return set_error(POND_ERR_ARG, "null argument");
  if (!c->niter) return set_error(POND_ERR_STATE, "call pond_keep_niter(ctx, 1) before the step");
  cudaSetDevice(c->p.device);
  cudaError_t e = cudaMemcpyAsync(out, c->niter, sizeof(int) * c->N, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_get_niter");
  return POND_OK;
}

int pond_set_inflow(pond_ctx* c, double rho, double ux, double uy, double uz, double T) {
  if (!c) return set_error(POND_ERR_ARG, "null argument");
  if (!(rho > 0) || !(T > 0) || !std::isfinite(rho) || !std::isfinite(T) || !std::isfinite(ux) ||
      !std::isfinite(uy) || !std::isfinite(uz))
    return set_error(POND_ERR_ARG, "inflow state needs finite rho > 0, u and T > 0");
  const double v[5] = {rho, ux, uy, uz, T};
  for (int k = 0; k < 5; k++) c->inflow[k] = v[k];
  c->have_inflow = true;
  return POND_OK;
}

int pond_set_gauge_tolerance(pond_ctx* c, double tol_abs, double tol_rel) {
  if (!c) return set_error(POND_ERR_ARG, "null argument");
  if (std::isnan(tol_abs) || std::isnan(tol_rel) || std::isinf(tol_abs) || std::isinf(tol_rel))
    return set_error(POND_ERR_ARG, "gauge tolerances must be finite");
  const bool off = tol_abs < 0 || tol_rel < 0;
  c->tolg_abs = off ? -1 : tol_abs;
  c->tolg_rel = off ? -1 : tol_rel;
  return POND_OK;
}

int pond_step(pond_ctx* c, int nsteps) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (nsteps < 0) return set_error(POND_ERR_ARG, "nsteps < 0");
  if (!c->initialized) return set_error(POND_ERR_STATE, "pond_step before pond_init/pond_set_state");
  if (c->p.learned && !c->guess_ready) return set_error(POND_ERR_STATE, "learned step without a predictor");
  cudaSetDevice(c->p.device);
  cudaError_t e = cudaEventRecord(c->ev0, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  for (int s = 0; s < nsteps; s++) {
    int st = launch_step(c);
    if (st != POND_OK) return st;
    c->cur = 1 - c->cur;  // LBMParamsHost::swapLS (structs.cuh:148)
    c->istep++;
    c->curtime += c->p.dt;
    if (c->dt_adapt) {  // update.cu:121-123, after curtime advanced by the old dt
      st = dt_adapt_after_step(c);
      if (st != POND_OK) return st;
    }
    if (c->strict) {
      e = cudaMemcpyAsync(c->h_sums, c->d_sums, sizeof(StepSums), cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) return cuda_fail(e, "sums download");
      c->have_sums = true;
      if (c->h_sums->nonconv) {
        cudaEventRecord(c->ev1, c->stream);
        return set_error(POND_ERR_NOT_CONVERGED, "step %lld: %llu nodes reached max_iter = %d", c->istep,
                         (unsigned long long)c->h_sums->nonconv, c->p.max_iter);
      }
    }
  }
  e = cudaEventRecord(c->ev1, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  if (nsteps > 0) {
    e = cudaMemcpyAsync(c->h_sums, c->d_sums, sizeof(StepSums), cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "sums download");
    c->have_sums = true;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "step launch");
  return POND_OK;
}

int pond_last_step_ms(pond_ctx* c, float* ms) {
  if (!c || !ms) return set_error(POND_ERR_ARG, "null argument");
  cudaError_t e = cudaEventSynchronize(c->ev1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, c->ev0, c->ev1);
  if (e != cudaSuccess) return cuda_fail(e, "pond_last_step_ms");
  return POND_OK;
}

int pond_upload_state(pond_ctx* c, const void* f, const void* rho, const void* g) {
  if (!c || !f || !rho || !g) return set_error(POND_ERR_ARG, "pond_upload_state: null argument");
  if (c->p.ddf) return set_error(POND_ERR_UNSUPPORTED, "pond_upload_state carries no energy populations");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  cudaSetDevice(c->p.device);
  const size_t N = (size_t)c->N;
  cudaError_t e = cudaMemcpyAsync(c->f[c->cur], f, (size_t)c->Q * N * c->elem, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->rho[c->cur], rho, N * c->elem, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->g[c->cur], g, 4 * N * c->elem, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_upload_state");
  c->initialized = true;
  c->have_sums = false;
  return POND_OK;
}

int pond_download_state(pond_ctx* c, void* f, void* rho, void* g) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  cudaSetDevice(c->p.device);
  const size_t N = (size_t)c->N;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMemcpyAsync(f, c->f[c->cur], (size_t)c->Q * N * c->elem, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, c->rho[c->cur], N * c->elem, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && g) e = cudaMemcpyAsync(g, c->g[c->cur], 4 * N * c->elem, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_download_state");
  return POND_OK;
}

}  // extern "C"

namespace pond {
template <typename S, typename D> __global__ void convert_kernel(const S* src, D* dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = D(src[i]);
}
}  // namespace pond

extern "C" {

int pond_copy_state(pond_ctx* dst, pond_ctx* src) {
  if (!dst || !src) return set_error(POND_ERR_ARG, "null context");
  for (pond_ctx* x : {dst, src}) { const int ps = pipe_drain(x); if (ps != POND_OK) return ps; }
  if (dst->p.lattice != src->p.lattice || dst->N != src->N || dst->p.Nx != src->p.Nx || dst->p.Ny != src->p.Ny)
    return set_error(POND_ERR_ARG, "pond_copy_state: lattice or grid differ");
  if (dst->p.device != src->p.device) return set_error(POND_ERR_ARG, "pond_copy_state: contexts on different devices");
  if (dst->p.ddf != src->p.ddf) return set_error(POND_ERR_ARG, "pond_copy_state: one context has energy populations");
  if (!src->initialized) return set_error(POND_ERR_STATE, "source state not initialised");
  cudaSetDevice(dst->p.device);
  cudaError_t e = cudaStreamSynchronize(src->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_copy_state");
  const long long cnt[4] = {(long long)dst->Q * dst->N, dst->N, 4 * dst->N, (long long)dst->Q * dst->N};
  for (int b = 0; b < 2; b++) {  // both time levels: the current one and the one before it
    const int sb = b == 0 ? src->cur : 1 - src->cur, db = b == 0 ? dst->cur : 1 - dst->cur;
    void* d[4] = {dst->f[db], dst->rho[db], dst->g[db], dst->h[db]};
    const void* s3[4] = {src->f[sb], src->rho[sb], src->g[sb], src->h[sb]};
    for (int k = 0; k < (dst->p.ddf ? 4 : 3); k++) {
      if (dst->elem == src->elem) {
        e = cudaMemcpyAsync(d[k], s3[k], cnt[k] * dst->elem, cudaMemcpyDeviceToDevice, dst->stream);
      } else if (dst->elem == 8) {
        convert_kernel<float, double><<<1024, 256, 0, dst->stream>>>((const float*)s3[k], (double*)d[k], cnt[k]);
        e = cudaGetLastError();
      } else {
        convert_kernel<double, float><<<1024, 256, 0, dst->stream>>>((const double*)s3[k], (float*)d[k], cnt[k]);
        e = cudaGetLastError();
      }
      if (e != cudaSuccess) return cuda_fail(e, "pond_copy_state");
    }
  }
  e = cudaStreamSynchronize(dst->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_copy_state");
  if (dst->mask[0] && src->mask[0]) {  // the mesh of the source goes with its state
    e = cudaMemcpyAsync(dst->mask[dst->mask_cur], src->mask[src->mask_cur], (size_t)dst->N, cudaMemcpyDeviceToDevice,
                        dst->stream);
    if (e == cudaSuccess && dst->pos && src->pos)
      e = cudaMemcpyAsync(dst->pos, src->pos, (size_t)dst->N * sizeof(double), cudaMemcpyDeviceToDevice, dst->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(dst->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pond_copy_state");
    dst->n_active = src->n_active;
  }
  dst->initialized = true;
  dst->have_sums = false;
  dst->istep = src->istep;
  dst->curtime = src->curtime;
  return POND_OK;
}

int pond_last_step_work(pond_ctx* c, int64_t* work) {
  if (!c || !work) return set_error(POND_ERR_ARG, "null argument");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_last_step_work");
  *work = c->have_sums ? (int64_t)c->h_sums->work : 0;
  return POND_OK;
}

int pond_set_strict(pond_ctx* c, int strict) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  c->strict = strict != 0;
  return POND_OK;
}

int pond_set_clock(pond_ctx* c, int64_t istep, double curtime, double dt) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  if (istep < 0 || !std::isfinite(curtime) || !std::isfinite(dt))
    return set_error(POND_ERR_ARG, "pond_set_clock: istep >= 0, finite time and dt");
  c->istep = istep;
  c->curtime = curtime;
  if (dt > 0) c->p.dt = dt;
  return POND_OK;
}

int pond_diagnostics(pond_ctx* c, pond_diag* out) {
  if (!c || !out) return set_error(POND_ERR_ARG, "null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  cudaSetDevice(c->p.device);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_diagnostics");
  std::memset(out, 0, sizeof(*out));
  out->istep = c->istep;
  out->curtime = c->curtime;
  if (c->have_sums) {
    const StepSums& s = *c->h_sums;
    out->mass = s.mass;
    out->moment[0] = s.mom[0]; out->moment[1] = s.mom[1]; out->moment[2] = s.mom[2];
    out->enrg = s.enrg;
    out->k = s.k;
    out->niter_max = s.niter_max;
    out->niter_sum = (int64_t)s.niter_sum;
    const long long nodes = c->mask[0] ? c->n_active : c->N;  // nodes the step visited
    out->niter_mean = nodes ? double(s.niter_sum) / double(nodes) : 0.0;
    out->nonconverged = (int64_t)s.nonconv;
    return POND_OK;
  }
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  // no step yet: sums of the current state (calcTotMoments, update.cu:52-69)
  return state_sums(c, out);
}

}  // extern "C"
