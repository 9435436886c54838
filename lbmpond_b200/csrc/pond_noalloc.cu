// pond_step_noalloc: one D3Q27 float32 PonD step that allocates no memory.
//
// Some callers cannot let a library allocate device memory: an application
// that owns every device buffer through its own pool or a memory budget
// fixed at start-up (as the reference's lbm.cu does with its global
// buffers), a host that must not stall on cudaMalloc/cudaFree inside its time
// loop, or a runtime that hands out device memory only through its own
// allocator.  The context API allocates its double buffers and reduction
// slots in pond_create; this entry point takes the caller's input and output
// buffers and keeps its only scratch -- one partial-sum record per CTA of the
// step kernel -- in a fixed array in this file's device memory.
//
// The scratch array is a file-scope __device__ variable: every GPU that
// loads the library holds POND_NOALLOC_SCRATCH_BYTES of it until the process
// exits.  Host code cannot use its name as a device address, so the first
// call on each device looks the address up with cudaGetSymbolAddress (with
// that device current) and keeps it; that first call should come before any
// stream capture.  All calls share the one array, so calls whose kernels
// overlap on a GPU (different streams, or threads) race on it.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "pond_internal.h"
#include "pond_step_d3q27.cuh"

namespace pond {
namespace noalloc {

constexpr int kMaxBlocks = 65536;  // CTAs of the step kernel: 256^3 nodes at 32x4x2 per CTA
constexpr size_t kScratchBytes = size_t(kMaxBlocks) * sizeof(d27::BlockPartial);
static_assert(kScratchBytes == POND_NOALLOC_SCRATCH_BYTES, "pond.h states the scratch size");

static __device__ __align__(256) unsigned char g_partials[kScratchBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_setup_mutex;
static void* g_partials_addr[kMaxDevices] = {};

// Sum the per-CTA records in a fixed order (the result does not depend on
// CTA scheduling) and write the step's diagnostics to the caller's buffer.
__global__ void __launch_bounds__(256) reduce_partials_kernel(const d27::BlockPartial* part, int nblocks,
                                                              long long N, pond_diag* out) {
  __shared__ double sd[6][256];
  __shared__ unsigned long long su[2][256];
  __shared__ int sm[256];
  const int t = threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long ni = 0, nc = 0;
  int mx = 0;
  for (int b = t; b < nblocks; b += 256) {
    const d27::BlockPartial& p = part[b];
    v[0] += p.mass; v[1] += p.mom[0]; v[2] += p.mom[1]; v[3] += p.mom[2]; v[4] += p.enrg; v[5] += p.k;
    ni += p.niter_sum; nc += p.nonconv; mx = max(mx, p.niter_max);
  }
  for (int q = 0; q < 6; q++) sd[q][t] = v[q];
  su[0][t] = ni; su[1][t] = nc; sm[t] = mx;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) {
      for (int q = 0; q < 6; q++) sd[q][t] += sd[q][t + w];
      su[0][t] += su[0][t + w]; su[1][t] += su[1][t + w]; sm[t] = max(sm[t], sm[t + w]);
    }
    __syncthreads();
  }
  if (t == 0) {
    pond_diag d = {};
    d.mass = sd[0][0];
    d.moment[0] = sd[1][0]; d.moment[1] = sd[2][0]; d.moment[2] = sd[3][0];
    d.enrg = sd[4][0];
    d.k = sd[5][0];
    d.niter_max = sm[0];
    d.niter_sum = (int64_t)su[0][0];
    d.niter_mean = N ? double(su[0][0]) / double(N) : 0.0;
    d.nonconverged = (int64_t)su[1][0];
    *out = d;
  }
}

// The step reads neighbouring nodes of f_in/rho_in/g_in while other CTAs
// write f_out/rho_out/g_out, so every output range (27 N, N and 4 N floats)
// must be disjoint from every input range and from the other outputs.
static bool any_overlap(long long N, const float* fi, const float* ri, const float* gi, const float* fo,
                        const float* ro, const float* go) {
  struct Range { uintptr_t lo, hi; };
  auto rg = [](const float* p, long long n) { return Range{(uintptr_t)p, (uintptr_t)p + (uintptr_t)n * 4u}; };
  const Range in[3] = {rg(fi, 27 * N), rg(ri, N), rg(gi, 4 * N)};
  const Range out[3] = {rg(fo, 27 * N), rg(ro, N), rg(go, 4 * N)};
  auto meet = [](Range a, Range b) { return a.lo < b.hi && b.lo < a.hi; };
  for (int o = 0; o < 3; o++) {
    for (int i = 0; i < 3; i++)
      if (meet(out[o], in[i])) return true;
    for (int j = o + 1; j < 3; j++)
      if (meet(out[o], out[j])) return true;
  }
  return false;
}

// Once per device: the scratch array's device address and the step kernels'
// shared-memory opt-in.  Called with the target device current.
static int setup_device(void** addr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return set_error(POND_ERR_UNSUPPORTED, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
    e = cudaFuncSetAttribute(d27::pull_d3q27_tile_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)d27::SMEM_BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(d27::pull_d3q27_tile_kernel<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)d27::SMEM_BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(d27::pull_d3q27_tile_kernel<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)d27::SMEM_BYTES);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    g_partials_addr[dev] = p;
  }
  *addr = g_partials_addr[dev];
  return POND_OK;
}

}  // namespace noalloc
}  // namespace pond

using namespace pond;

extern "C" int pond_step_noalloc(const pond_params* p, const float* f_in, const float* rho_in, const float* g_in,
                                 float* f_out, float* rho_out, float* g_out, pond_diag* diag_out, void* stream) {
  if (!p || !f_in || !rho_in || !g_in || !f_out || !rho_out || !g_out || !diag_out)
    return set_error(POND_ERR_ARG, "pond_step_noalloc: null argument");
  if (p->lattice != POND_D3Q27 || p->precision != POND_FP32 || p->interp < POND_LAGR2 || p->interp > POND_LAGR4)
    return set_error(POND_ERR_UNSUPPORTED, "pond_step_noalloc runs D3Q27, float32, Lagrange order 2-4 only");
  if (p->ddf) return set_error(POND_ERR_UNSUPPORTED, "pond_step_noalloc carries no energy populations");
  if (p->learned) return set_error(POND_ERR_UNSUPPORTED, "pond_step_noalloc has no learned start (learned = 0)");
  if (p->Nx <= 0 || p->Ny <= 0 || p->Nz <= 0 || p->Nx > (1 << 30) || p->Ny > (1 << 30) || p->Nz > (1 << 30))
    return set_error(POND_ERR_ARG, "grid out of range");
  const long long N = p->Nx * p->Ny * p->Nz;
  if (N > (1LL << 31) - 1) return set_error(POND_ERR_ARG, "grid has more than 2^31-1 nodes");
  const int vst = check_step_params(p);
  if (vst != POND_OK) return vst;
  for (int k = 0; k < 3; k++)
    if (p->bc[k] == POND_BC_INFLOW) return set_error(POND_ERR_UNSUPPORTED, "pond_step_noalloc has no inflow boundary");
  const dim3 grd((unsigned)((p->Nx + d27::TX - 1) / d27::TX), (unsigned)((p->Ny + d27::TY - 1) / d27::TY),
                 (unsigned)((p->Nz + d27::TZ - 1) / d27::TZ));
  const long long nblocks = (long long)grd.x * grd.y * grd.z;
  if (nblocks > noalloc::kMaxBlocks)
    return set_error(POND_ERR_ARG,
                     "pond_step_noalloc: grid %lldx%lldx%lld needs %lld step CTAs; its fixed scratch holds %d "
                     "(at most %d nodes, e.g. 256^3)",
                     (long long)p->Nx, (long long)p->Ny, (long long)p->Nz, nblocks, noalloc::kMaxBlocks,
                     noalloc::kMaxBlocks * d27::THREADS);
  if (noalloc::any_overlap(N, f_in, rho_in, g_in, f_out, rho_out, g_out))
    return set_error(POND_ERR_ARG, "pond_step_noalloc: an output buffer overlaps an input or another output");
  void* scratch = nullptr;
  int st = noalloc::setup_device(&scratch);
  if (st != POND_OK) return st;

  StepArgs<float> a;
  a.f_in = f_in; a.rho_in = rho_in; a.g_in = g_in;
  a.f_out = f_out; a.rho_out = rho_out; a.g_out = g_out;
  a.guess = nullptr;
  a.niter_out = nullptr;
  a.sums = reinterpret_cast<StepSums*>(scratch);  // the per-CTA partial records
  a.nx = (int)p->Nx; a.ny = (int)p->Ny; a.nz = (int)p->Nz;
  a.N = N;
  for (int k = 0; k < 3; k++) a.bc[k] = p->bc[k];
  a.dtau = 1.0 / p->tau;
  a.tol_abs = p->tol_abs; a.tol_rel = p->tol_rel;
  a.tolg_abs = p->tol_abs; a.tolg_rel = p->tol_rel;
  a.max_iter = p->max_iter;
  const double PI = 3.14159265358979323846;
  a.kdx = 0.5 / (8 * PI * PI * PI) * (2 * PI / p->Nx) * (2 * PI / p->Ny) * (2 * PI / p->Nz);
  cudaStream_t s = (cudaStream_t)stream;
  const dim3 blk(d27::TX, d27::TY, d27::TZ);
  if (p->interp == POND_LAGR2) d27::pull_d3q27_tile_kernel<2, true><<<grd, blk, d27::SMEM_BYTES, s>>>(a);
  else if (p->interp == POND_LAGR3) d27::pull_d3q27_tile_kernel<3, true><<<grd, blk, d27::SMEM_BYTES, s>>>(a);
  else d27::pull_d3q27_tile_kernel<4, true><<<grd, blk, d27::SMEM_BYTES, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "pond_step_noalloc step launch");
  noalloc::reduce_partials_kernel<<<1, 256, 0, s>>>(reinterpret_cast<const d27::BlockPartial*>(scratch),
                                                      (int)nblocks, N, diag_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "pond_step_noalloc reduction launch");
  return POND_OK;
}
