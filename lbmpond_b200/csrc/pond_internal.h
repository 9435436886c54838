// Host-side internals shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include "pond_common.cuh"

struct pond_ctx {
  pond_params p;
  int Q = 0;
  long long N = 0;
  size_t elem = 4;           // bytes per stored value (float or double)
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // double-buffered SoA state: f[Q][N], rho[N], g[4][N]; cur is the latest
  void* f[2] = {nullptr, nullptr};
  void* rho[2] = {nullptr, nullptr};
  void* g[2] = {nullptr, nullptr};
  void* h[2] = {nullptr, nullptr};  // energy populations h[Q][N] (double-distribution extension)
  int cur = 0;
  pond::StepSums* d_sums = nullptr;
  pond::StepSums* h_sums = nullptr;  // pinned
  bool have_sums = false;
  int* niter = nullptr;
  bool keep_niter = false;
  float* guess = nullptr;  // [4][N] predicted starting gauge (learned path)
  bool guess_ready = false;
  void* predictor = nullptr;  // learned-gauge network bound to this context
  float gate = 0.f;           // minimum predicted change that replaces the previous gauge
  bool extrapolate = false;   // start from g^n + (g^n - g^{n-1}) when no network is bound
  void* g_hist = nullptr;     // gauge of the level before the last step's input (training pairs)
  bool keep_history = false;
  bool initialized = false;
  long long istep = 0;
  double curtime = 0;
  void* staging = nullptr;  // pinned host staging for conversions
  size_t staging_bytes = 0;
  // host-buffer pipeline (pond_step_host): two input slots, copy streams, events
  void* in_f[2] = {nullptr, nullptr};
  void* in_rho[2] = {nullptr, nullptr};
  void* in_g[2] = {nullptr, nullptr};
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in_ready[2] = {nullptr, nullptr}, ev_step_done[2] = {nullptr, nullptr},
              ev_out_free[2] = {nullptr, nullptr};
  long long pipe_k = 0;
  bool pipe_pending = false;
  // one-dimensional mesh schemes (POND_GAP2, POND_NONUNIFORM3)
  uint8_t* mask[2] = {nullptr, nullptr};  // node mask and the scratch copy AMR writes into
  int mask_cur = 0;
  long long n_active = 0;                 // active nodes in mask[mask_cur]
  double* pos = nullptr;                  // node positions (POND_NONUNIFORM3)
  uint8_t* amr_code = nullptr;            // coarsening: per-node transition codes [N]
  uint32_t* amr_maps = nullptr;           // coarsening: per-chunk composed transitions
  uint8_t* amr_sigma = nullptr;           // coarsening: automaton state entering each chunk
  unsigned long long* amr_counts = nullptr;  // [4] device counters
  unsigned long long* amr_counts_h = nullptr;  // pinned copy
  bool strict = false;  // pond_step stops with POND_ERR_NOT_CONVERGED after a step with nodes at max_iter
  // ghost state of POND_BC_INFLOW axes (pond_set_inflow): rho, u_x, u_y, u_z, T
  double inflow[5] = {1, 0, 0, 0, 1};
  bool have_inflow = false;
  // separate convergence tolerance on the gauge u, T (pond_set_gauge_tolerance); < 0: params' tol_abs / tol_rel
  double tolg_abs = -1, tolg_rel = -1;
  // time-step adaptation after every step (update.cu:121-123)
  bool dt_adapt = false;
  int adapt_hi = 1000, adapt_lo = 4;
};

namespace pond {
int set_error(int status, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
int lattice_q(int lattice);
// boundaries, tau, max_iter and tolerances of a step's parameters (POND_OK or POND_ERR_ARG)
int check_step_params(const pond_params* p);
double lattice_weight_host(int lattice, int ref_index);
double lattice_tlat(int lattice);
double lattice_dim(int lattice);

int ctx_alloc(pond_ctx* c);
void ctx_free(pond_ctx* c);
// float64 host array -> device array of the context's precision (and back)
int upload(pond_ctx* c, const double* src, size_t count, void* dst);
int download(pond_ctx* c, const void* src, size_t count, double* dst);
int launch_step(pond_ctx* c);
// one plain step between explicit device buffers {f, rho, g} (no predictor)
int launch_step_io(pond_ctx* c, const void* const in[3], void* const out[3]);
// wait for the host-buffer pipeline (pond_step_host) if one is in flight
int pipe_drain(pond_ctx* c);
void pipe_free(pond_ctx* c);
int state_sums(pond_ctx* c, pond_diag* out);
// learned path: run the bound predictor on the current state into c->guess
int run_predictor(pond_ctx* c);
bool mesh_scheme(int interp);
// allocate and initialise the mask (all active) and positions (p_x = x) of a mesh context
int mesh_alloc(pond_ctx* c);
// every node active, positions p_x = x (fill, init.cu:100-106)
int mesh_reset(pond_ctx* c);
void mesh_free(pond_ctx* c);
// the adaptation policy after one step: rescale the new state when NiterMax crosses a threshold
int dt_adapt_after_step(pond_ctx* c);
}  // namespace pond
