// One-dimensional mesh support of the PonD step library: the node mask
// (Cinfo::set) and node positions (Cell::p.x under NRMESH) of the
// POND_GAP2 / POND_NONUNIFORM3 schemes, AMR refinement (AMR_add) and
// coarsening (AMR_remove), and time-step rescaling (TimeCorr) with the
// reference's NiterMax policy.
//
// Coarsening.  The reference's AMR_remove (amr.cu:28-55) is one serial pass
// <<<1,1>>> over the nodes in order, each decision reading the mask as the
// pass has left it.  A node can only be removed when its nearest active
// neighbours are both within 3 nodes, so the decision at x depends on the
// pass so far only through s[x-1], s[x-2], s[x-3]: an automaton with 8
// states.  Each node's transition is fixed by the old mask and the data (the
// nodes to its right are not yet visited; the wrap-around of the last three
// nodes onto the first three is resolved separately), so the pass is a
// prefix composition of 8-entry maps: per-node codes, per-chunk composed
// maps, one block-wide scan, and a replay of every chunk from its entry
// state.  The result equals the serial pass bit for bit; grids of fewer than
// 8 nodes run the serial pass itself.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pond_internal.h"

namespace pond {

bool mesh_scheme(int interp) { return interp == POND_GAP2 || interp == POND_NONUNIFORM3; }

namespace mesh {

constexpr int CHUNK = 64;           // nodes per thread in the coarsening scan
constexpr int SCAN_THREADS = 1024;  // the single block of the scan
constexpr int SERIAL_MAX = 8;       // grids below this size run the serial pass

__global__ void init_kernel(uint8_t* mask, double* pos, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    mask[i] = 1;
    if (pos) pos[i] = double(i);
  }
}

// ---------------------------------------------------------------- refinement
// AMR_add (amr.cu:1-27): reads the old mask `set`, activates midpoints in
// `setnew` (a copy of it).  Each thread's reads are of active nodes and its
// writes of an inactive node strictly inside its own gap, so the threads
// never touch the same node.
template <typename R>
__global__ void refine_kernel(const uint8_t* set, uint8_t* setnew, R* f0, R* r0, R* g0, R* f1, R* r1, R* g1, int nx,
                              double tol, unsigned long long* counts) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nx || !set[x]) return;
  int xp = x, dist = 0;
  do {  // ends at x itself at the latest (amr.cu:8-12)
    xp = xp + 1 == nx ? 0 : xp + 1;
    dist++;
  } while (!set[xp]);
  const long long N = nx;
  const double vdif = double(g0[xp]) - double(g0[x]);
  const double rm = r0[x], rp = r0[xp];
  if (vdif * vdif / fmin(double(g0[3 * N + x]), double(g0[3 * N + xp])) > tol || fabs(1 - rm / rp) > tol) {
    if (dist <= 1) atomicAdd(&counts[1], 1ull);
    if (dist % 2 == 0) {  // amr.cu:18-25: the average record, saved to both time levels (save_12)
      const long long mid = ((long long)x + dist / 2) % nx;
      const R rv = R(0.5 * (rm + rp));
      r0[mid] = rv;
      r1[mid] = rv;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const R v = R(0.5 * (double(g0[k * N + x]) + double(g0[k * N + xp])));
        g0[k * N + mid] = v;
        g1[k * N + mid] = v;
      }
#pragma unroll
      for (int q = 0; q < 5; q++) {
        const R v = R(0.5 * (double(f0[q * N + x]) + double(f0[q * N + xp])));
        f0[q * N + mid] = v;
        f1[q * N + mid] = v;
      }
      setnew[mid] = 1;
      atomicAdd(&counts[0], 1ull);
    }
  }
}

// ---------------------------------------------------------------- coarsening
// amr.cu:50: the removal test of node x between its nearest active
// neighbours cm and cp (operand order of the reference, in float64)
template <typename R>
__device__ __forceinline__ bool coarsen_cond(const R* rho, const R* g, long long N, int x, int cm, int cp, double tol) {
  const double T0 = g[3 * N + x];
  const double u0 = g[x];
  const double vdifm = double(g[cm]) - u0;
  const double vdifp = double(g[cp]) - u0;
  const double r0 = rho[x];
  return vdifm * vdifm / T0 < tol && vdifp * vdifp / T0 < tol && fabs(double(rho[cp]) / r0 - 1) < tol &&
         fabs(double(rho[cm]) / r0 - 1) < tol;
}

// Automaton state sigma = s[x-1] | s[x-2] << 1 | s[x-3] << 2 (the mask as
// the pass has left it).  A node's code: bit 3 = old s[x]; bit d-1 = removal
// when the nearest active left neighbour is at distance d (d = 1..3; the
// right side and its distance limit are already folded in).
__device__ __forceinline__ int coarsen_next(int code, int sigma) {
  int keep = (code >> 3) & 1;
  const int d = (sigma & 1) ? 0 : (sigma & 2) ? 1 : (sigma & 4) ? 2 : 3;
  if (keep && d < 3 && ((code >> d) & 1)) keep = 0;
  return keep | ((sigma << 1) & 6);
}

// 8-entry maps of states, 3 bits per entry
__device__ __forceinline__ int map_get(uint32_t m, int e) { return (m >> (3 * e)) & 7; }
__device__ __forceinline__ uint32_t map_ident() {
  uint32_t m = 0;
#pragma unroll
  for (int e = 0; e < 8; e++) m |= uint32_t(e) << (3 * e);
  return m;
}
// the map "second after first"
__device__ __forceinline__ uint32_t map_then(uint32_t first, uint32_t second) {
  uint32_t m = 0;
#pragma unroll
  for (int e = 0; e < 8; e++) m |= uint32_t(map_get(second, map_get(first, e))) << (3 * e);
  return m;
}

// codes of nodes 0 .. nx-4 (their right neighbours x+1..x+3 are all in range
// and not yet visited by the pass, so the old mask decides them)
template <typename R>
__global__ void codes_kernel(const uint8_t* set, const R* rho, const R* g, int nx, double tol, uint8_t* code) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int M = nx - 3;
  if (x >= M) return;
  int c = 0;
  if (set[x]) {
    c = 8;
    int cp = -1;
    for (int k = 1; k <= 3; k++)
      if (set[x + k]) { cp = x + k; break; }
    if (cp >= 0)
      for (int d = 1; d <= 3; d++) {
        const int cm = x - d < 0 ? x - d + nx : x - d;
        if (coarsen_cond<R>(rho, g, nx, x, cm, cp, tol)) c |= 1 << (d - 1);
      }
  }
  code[x] = (uint8_t)c;
}

__global__ void chunk_maps_kernel(const uint8_t* code, int M, int nch, uint32_t* maps) {
  const int ch = blockIdx.x * blockDim.x + threadIdx.x;
  if (ch >= nch) return;
  int st[8];
#pragma unroll
  for (int e = 0; e < 8; e++) st[e] = e;
  const int x1 = min((ch + 1) * CHUNK, M);
  for (int x = ch * CHUNK; x < x1; x++) {
    const int cd = code[x];
#pragma unroll
    for (int e = 0; e < 8; e++) st[e] = coarsen_next(cd, st[e]);
  }
  uint32_t m = 0;
#pragma unroll
  for (int e = 0; e < 8; e++) m |= uint32_t(st[e]) << (3 * e);
  maps[ch] = m;
}

// One block: scan of the chunk maps into each chunk's entry state, then the
// last three nodes (whose right neighbours wrap onto the already visited
// first three) in order.  Grids below SERIAL_MAX run the reference's serial
// pass here instead.
template <typename R>
__global__ void __launch_bounds__(SCAN_THREADS)
    scan_kernel(const uint8_t* set, uint8_t* setnew, const R* rho, const R* g, int nx, double tol,
                const uint8_t* code, const uint32_t* maps, int nch, uint8_t* sigma_in, unsigned long long* counts) {
  const int t = threadIdx.x;
  if (nx < SERIAL_MAX) {
    if (t == 0) {
      for (int i = 0; i < nx; i++) setnew[i] = set[i];
      unsigned long long removed = 0;
      for (int ix = 0; ix < nx; ix++) {
        if (!setnew[ix]) continue;
        int xm = ix, xp = ix, dM = 0, dP = 0;
        do { xm = xm == 0 ? nx - 1 : xm - 1; dM++; } while (!setnew[xm]);  // ends at ix at the latest
        do { xp = xp + 1 == nx ? 0 : xp + 1; dP++; } while (!setnew[xp]);
        if (coarsen_cond<R>(rho, g, nx, ix, xm, xp, tol) && dM < 4 && dP < 4) {
          setnew[ix] = 0;
          removed++;
        }
      }
      counts[0] += removed;
    }
    return;
  }
  __shared__ uint32_t sm[SCAN_THREADS];
  const uint32_t ident = map_ident();
  const int per = (nch + SCAN_THREADS - 1) / SCAN_THREADS;
  const int c0 = min(t * per, nch), c1 = min(c0 + per, nch);
  uint32_t run = ident;
  for (int ch = c0; ch < c1; ch++) run = map_then(run, maps[ch]);
  sm[t] = run;
  __syncthreads();
  for (int off = 1; off < SCAN_THREADS; off <<= 1) {  // inclusive prefix: sm[t] = run_0 .. run_t in order
    const uint32_t before = t >= off ? sm[t - off] : ident;
    __syncthreads();
    sm[t] = map_then(before, sm[t]);
    __syncthreads();
  }
  const int s0 = set[nx - 1] | (set[nx - 2] << 1) | (set[nx - 3] << 2);
  int st = t == 0 ? s0 : map_get(sm[t - 1], s0);
  for (int ch = c0; ch < c1; ch++) {
    sigma_in[ch] = (uint8_t)st;
    st = map_get(maps[ch], st);
  }
  if (t == 0) {
    int head[3];  // the new values of nodes 0..2, which the tail's right neighbours reach
    int sg = s0;
    for (int x = 0; x < 3; x++) {
      sg = coarsen_next(code[x], sg);
      head[x] = sg & 1;
    }
    int sigma = map_get(sm[SCAN_THREADS - 1], s0);  // state entering node nx-3
    unsigned long long removed = 0;
    for (int x = nx - 3; x < nx; x++) {
      int keep = set[x];
      if (keep) {
        const int d = (sigma & 1) ? 1 : (sigma & 2) ? 2 : (sigma & 4) ? 3 : 0;
        int cp = -1;
        for (int k = 1; k <= 3 && cp < 0; k++) {
          const int j = x + k;
          if (j < nx ? set[j] != 0 : head[j - nx] != 0) cp = j < nx ? j : j - nx;
        }
        if (d > 0 && cp >= 0 && coarsen_cond<R>(rho, g, nx, x, x - d, cp, tol)) {
          keep = 0;
          removed++;
        }
      }
      setnew[x] = (uint8_t)keep;
      sigma = keep | ((sigma << 1) & 6);
    }
    atomicAdd(&counts[0], removed);
  }
}

__global__ void apply_kernel(const uint8_t* code, const uint8_t* sigma_in, int M, int nch, uint8_t* setnew,
                             unsigned long long* counts) {
  const int ch = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long removed = 0;
  if (ch < nch) {
    int st = sigma_in[ch];
    const int x1 = min((ch + 1) * CHUNK, M);
    for (int x = ch * CHUNK; x < x1; x++) {
      const int cd = code[x];
      st = coarsen_next(cd, st);
      setnew[x] = (uint8_t)(st & 1);
      removed += ((cd >> 3) & 1) && !(st & 1);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) removed += __shfl_xor_sync(0xffffffffu, removed, o);
  if ((threadIdx.x & 31) == 0 && removed) atomicAdd(&counts[0], removed);
}

// ---------------------------------------------------------------- TimeCorr
// update.cu:15-28: u *= s, T *= s*s in the context's precision (dtscale is
// an ftype there); the step's sums follow (mass unchanged, momentum by s,
// energy and kinetic energy by s*s).
template <typename R> __global__ void rescale_kernel(R* g, long long N, double s, StepSums* sums) {
  const R sr = R(s);
  const R s2 = sr * sr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    g[i] *= sr;
    g[N + i] *= sr;
    g[2 * N + i] *= sr;
    g[3 * N + i] *= s2;
  }
  if (sums && blockIdx.x == 0 && threadIdx.x == 0) {
    sums->mom[0] *= s; sums->mom[1] *= s; sums->mom[2] *= s;
    sums->enrg *= s * s;
    sums->k *= s * s;
  }
}

}  // namespace mesh

int mesh_alloc(pond_ctx* c) {
  if (!mesh_scheme(c->p.interp)) return POND_OK;
  const size_t N = (size_t)c->N;
  if (cudaMalloc(&c->mask[0], N) != cudaSuccess || cudaMalloc(&c->mask[1], N) != cudaSuccess ||
      (c->p.interp == POND_NONUNIFORM3 && cudaMalloc(&c->pos, N * sizeof(double)) != cudaSuccess)) {
    cudaGetLastError();
    return set_error(POND_ERR_NOMEM, "node mask / positions");
  }
  return mesh_reset(c);
}

int mesh_reset(pond_ctx* c) {
  if (!c->mask[0]) return POND_OK;
  const size_t N = (size_t)c->N;
  mesh::init_kernel<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(c->mask[0], c->pos, (long long)N);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->mask[1], c->mask[0], N, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "mesh init");
  c->mask_cur = 0;
  c->n_active = c->N;
  return POND_OK;
}

void mesh_free(pond_ctx* c) {
  cudaFree(c->mask[0]); cudaFree(c->mask[1]); cudaFree(c->pos);
  cudaFree(c->amr_code); cudaFree(c->amr_maps); cudaFree(c->amr_sigma); cudaFree(c->amr_counts);
  if (c->amr_counts_h) cudaFreeHost(c->amr_counts_h);
  c->mask[0] = c->mask[1] = nullptr;
  c->pos = nullptr;
  c->amr_code = nullptr; c->amr_maps = nullptr; c->amr_sigma = nullptr;
  c->amr_counts = nullptr; c->amr_counts_h = nullptr;
}

static int amr_counts(pond_ctx* c) {
  if (c->amr_counts && c->amr_counts_h) return POND_OK;
  if (!c->amr_counts && cudaMalloc(&c->amr_counts, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    c->amr_counts = nullptr;
    return set_error(POND_ERR_NOMEM, "AMR counters");
  }
  cudaError_t e = cudaMallocHost(&c->amr_counts_h, 4 * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    c->amr_counts_h = nullptr;
    return cuda_fail(e, "cudaMallocHost");
  }
  return POND_OK;
}

static int read_counts(pond_ctx* c) {
  cudaError_t e = cudaMemcpyAsync(c->amr_counts_h, c->amr_counts, 4 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "AMR counters");
}

template <typename R> static int refine_typed(pond_ctx* c, double tol) {
  const int i = c->cur, o = 1 - c->cur, m = c->mask_cur;
  const int nx = (int)c->p.Nx;
  cudaError_t e = cudaMemcpyAsync(c->mask[1 - m], c->mask[m], (size_t)c->N, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->amr_counts, 0, 4 * sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "refine");
  mesh::refine_kernel<R><<<(nx + 127) / 128, 128, 0, c->stream>>>(
      c->mask[m], c->mask[1 - m], (R*)c->f[i], (R*)c->rho[i], (R*)c->g[i], (R*)c->f[o], (R*)c->rho[o], (R*)c->g[o],
      nx, tol, c->amr_counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "refine kernel launch");
  return read_counts(c);
}

template <typename R> static int coarsen_typed(pond_ctx* c, double tol) {
  const int i = c->cur, m = c->mask_cur;
  const int nx = (int)c->p.Nx;
  const int M = nx >= mesh::SERIAL_MAX ? nx - 3 : 0;
  const int nch = (M + mesh::CHUNK - 1) / mesh::CHUNK;
  cudaError_t e = cudaMemsetAsync(c->amr_counts, 0, 4 * sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "coarsen");
  const R* rho = (const R*)c->rho[i];
  const R* g = (const R*)c->g[i];
  if (nch > 0) {
    mesh::codes_kernel<R><<<(M + 255) / 256, 256, 0, c->stream>>>(c->mask[m], rho, g, nx, tol, c->amr_code);
    mesh::chunk_maps_kernel<<<(nch + 127) / 128, 128, 0, c->stream>>>(c->amr_code, M, nch, c->amr_maps);
  }
  mesh::scan_kernel<R><<<1, mesh::SCAN_THREADS, 0, c->stream>>>(c->mask[m], c->mask[1 - m], rho, g, nx, tol,
                                                                c->amr_code, c->amr_maps, nch, c->amr_sigma,
                                                                c->amr_counts);
  if (nch > 0)
    mesh::apply_kernel<<<(nch + 127) / 128, 128, 0, c->stream>>>(c->amr_code, c->amr_sigma, M, nch, c->mask[1 - m],
                                                                 c->amr_counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "coarsen kernel launch");
  return read_counts(c);
}

static int rescale(pond_ctx* c, double s) {
  const long long N = c->N;
  const unsigned blocks = (unsigned)std::min<long long>((N + 255) / 256, 148 * 8);
  StepSums* sums = c->have_sums ? c->d_sums : nullptr;
  if (c->elem == 8)
    mesh::rescale_kernel<double><<<blocks, 256, 0, c->stream>>>((double*)c->g[c->cur], N, s, sums);
  else
    mesh::rescale_kernel<float><<<blocks, 256, 0, c->stream>>>((float*)c->g[c->cur], N, s, sums);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "rescale kernel launch");
  c->p.dt *= s;  // update.cu:128
  return POND_OK;
}

int dt_adapt_after_step(pond_ctx* c) {
  cudaError_t e = cudaMemcpyAsync(c->h_sums, c->d_sums, sizeof(StepSums), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "NiterMax read-back");
  const int nmax = c->h_sums->niter_max;
  const double s = nmax >= c->adapt_hi ? 0.5 : nmax <= c->adapt_lo ? 2.0 : 1.0;  // update.cu:121-122
  if (s == 1.0) return POND_OK;
  c->have_sums = true;  // the step's sums are rescaled with the state
  return rescale(c, s);
}

}  // namespace pond

using namespace pond;

extern "C" {

int pond_set_mask(pond_ctx* c, const uint8_t* mask) {
  if (!c || !mask) return set_error(POND_ERR_ARG, "pond_set_mask: null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->mask[0]) return set_error(POND_ERR_UNSUPPORTED, "the node mask belongs to POND_GAP2 / POND_NONUNIFORM3");
  cudaSetDevice(c->p.device);
  std::vector<uint8_t> m((size_t)c->N);
  long long active = 0;
  for (long long i = 0; i < c->N; i++) {
    m[i] = mask[i] ? 1 : 0;
    active += m[i];
  }
  cudaError_t e = cudaMemcpyAsync(c->mask[c->mask_cur], m.data(), (size_t)c->N, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_set_mask");
  c->n_active = active;
  return POND_OK;
}

int pond_get_mask(pond_ctx* c, uint8_t* mask) {
  if (!c || !mask) return set_error(POND_ERR_ARG, "pond_get_mask: null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->mask[0]) return set_error(POND_ERR_UNSUPPORTED, "the node mask belongs to POND_GAP2 / POND_NONUNIFORM3");
  cudaSetDevice(c->p.device);
  cudaError_t e = cudaMemcpyAsync(mask, c->mask[c->mask_cur], (size_t)c->N, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_get_mask");
}

int pond_set_positions(pond_ctx* c, const double* x) {
  if (!c || !x) return set_error(POND_ERR_ARG, "pond_set_positions: null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->pos) return set_error(POND_ERR_UNSUPPORTED, "node positions belong to POND_NONUNIFORM3");
  const long long N = c->N;
  for (long long i = 0; i < N; i++) {
    if (!std::isfinite(x[i])) return set_error(POND_ERR_ARG, "position %lld is not finite", i);
    if (i > 0 && !(x[i] > x[i - 1])) return set_error(POND_ERR_ARG, "positions must increase (node %lld)", i);
  }
  if (!(x[N - 1] - x[0] < double(c->p.Nx))) return set_error(POND_ERR_ARG, "positions span Nx or more");
  cudaSetDevice(c->p.device);
  cudaError_t e = cudaMemcpyAsync(c->pos, x, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_set_positions");
}

int pond_get_positions(pond_ctx* c, double* x) {
  if (!c || !x) return set_error(POND_ERR_ARG, "pond_get_positions: null argument");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->pos) return set_error(POND_ERR_UNSUPPORTED, "node positions belong to POND_NONUNIFORM3");
  cudaSetDevice(c->p.device);
  cudaError_t e = cudaMemcpyAsync(x, c->pos, (size_t)c->N * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_get_positions");
}

int pond_amr_refine(pond_ctx* c, double tol, int64_t* added, int64_t* limit_hits) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->mask[0]) return set_error(POND_ERR_UNSUPPORTED, "AMR needs POND_GAP2 / POND_NONUNIFORM3");
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  if (!(tol > 0) || !std::isfinite(tol)) return set_error(POND_ERR_ARG, "tol must be a finite value > 0");
  cudaSetDevice(c->p.device);
  int st = amr_counts(c);
  if (st == POND_OK) st = c->elem == 8 ? refine_typed<double>(c, tol) : refine_typed<float>(c, tol);
  if (st != POND_OK) return st;
  c->mask_cur = 1 - c->mask_cur;
  c->n_active += (long long)c->amr_counts_h[0];
  if (added) *added = (int64_t)c->amr_counts_h[0];
  if (limit_hits) *limit_hits = (int64_t)c->amr_counts_h[1];
  return POND_OK;
}

int pond_amr_coarsen(pond_ctx* c, double tol, int64_t* removed) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!c->mask[0]) return set_error(POND_ERR_UNSUPPORTED, "AMR needs POND_GAP2 / POND_NONUNIFORM3");
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  if (!(tol > 0) || !std::isfinite(tol)) return set_error(POND_ERR_ARG, "tol must be a finite value > 0");
  cudaSetDevice(c->p.device);
  int st = amr_counts(c);
  if (st != POND_OK) return st;
  if (!c->amr_code || !c->amr_maps || !c->amr_sigma) {
    const size_t N = (size_t)c->N, nch = (N + mesh::CHUNK - 1) / mesh::CHUNK;
    cudaFree(c->amr_code); cudaFree(c->amr_maps); cudaFree(c->amr_sigma);
    c->amr_code = nullptr; c->amr_maps = nullptr; c->amr_sigma = nullptr;
    if (cudaMalloc(&c->amr_code, N) != cudaSuccess || cudaMalloc(&c->amr_maps, nch * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&c->amr_sigma, nch) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(c->amr_code); cudaFree(c->amr_maps); cudaFree(c->amr_sigma);
      c->amr_code = nullptr; c->amr_maps = nullptr; c->amr_sigma = nullptr;
      return set_error(POND_ERR_NOMEM, "coarsening scratch");
    }
  }
  st = c->elem == 8 ? coarsen_typed<double>(c, tol) : coarsen_typed<float>(c, tol);
  if (st != POND_OK) return st;
  c->mask_cur = 1 - c->mask_cur;
  c->n_active -= (long long)c->amr_counts_h[0];
  if (removed) *removed = (int64_t)c->amr_counts_h[0];
  return POND_OK;
}

int pond_rescale_time(pond_ctx* c, double s) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  { const int ps = pipe_drain(c); if (ps != POND_OK) return ps; }
  if (!(s > 0) || !std::isfinite(s)) return set_error(POND_ERR_ARG, "the time-step factor must be finite and > 0");
  if (!c->initialized) return set_error(POND_ERR_STATE, "state not initialised");
  cudaSetDevice(c->p.device);
  int st = rescale(c, s);
  if (st != POND_OK) return st;
  cudaError_t e = cudaSuccess;
  if (c->have_sums)
    e = cudaMemcpyAsync(c->h_sums, c->d_sums, sizeof(StepSums), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_rescale_time");
}

int pond_set_dt_adapt(pond_ctx* c, int on, int niter_hi, int niter_lo) {
  if (!c) return set_error(POND_ERR_ARG, "null context");
  if (on && !(niter_lo < niter_hi)) return set_error(POND_ERR_ARG, "niter_lo must be below niter_hi");
  c->dt_adapt = on != 0;
  c->adapt_hi = niter_hi;
  c->adapt_lo = niter_lo;
  return POND_OK;
}

}  // extern "C"
