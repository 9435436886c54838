/*
 * pond.h -- C ABI of the B200 (sm_100a) Particles-on-Demand step library
 * (lbmpond_b200/libpond_b200.so).
 *
 * Drop-in boundary for the reference's step entry points (engrab6/lbmPonD):
 *
 *   reference (global state, exit() on error)        this ABI (explicit context, status codes)
 *   ------------------------------------------------  ----------------------------------------
 *   LBMParamsHost::set      lbm.cu:134-168           pond_params_default + pond_create
 *   copy2dev(tables)        lbm.cu:201-250           pond_create (tables live in the library)
 *   void init()             init.cu:109-128          pond_init (built-in initial conditions)
 *   fill / Cell::set_base   init.cu:2-108,           pond_set_state (host arrays; f = NULL
 *                           lbpack.cu:15-21            means set_base from rho, u, T)
 *   void calcStep()         update.cu:86-142         pond_step (minus file I/O and printf)
 *   calcTotMoments/diagn    update.cu:52-69,         pond_diagnostics
 *                           diagn.cu:1-30
 *   void drop(string*)      drop.cu:2-34             pond_get_fields / pond_get_state
 *   LBMParamsHost::swapLS   structs.cuh:148          done inside pond_step
 *
 * Every function returns POND_OK (0) or a negative pond_status; none exits
 * the process.  A context belongs to one device and one CUDA stream; calls on
 * one context must not overlap from several threads, while separate contexts
 * are independent.  Host arrays are float64 in the layout
 *   f[q*N + n], rho[n], g[k*N + n] (k: 0,1,2 = u_x,u_y,u_z; 3 = T),
 *   n = x + Nx*(y + Ny*z), populations in the reference's order (consts.h).
 */
#ifndef POND_H
#define POND_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define POND_ABI_VERSION 1

typedef enum {
  POND_OK = 0,
  POND_ERR_ARG = -1,          /* bad argument or parameter combination */
  POND_ERR_CUDA = -2,         /* a CUDA runtime call failed (see pond_last_error_string) */
  POND_ERR_NOMEM = -3,        /* device allocation failed */
  POND_ERR_STATE = -4,        /* call out of order (e.g. step before init) */
  POND_ERR_UNSUPPORTED = -5,  /* lattice / scheme / precision combination not built */
  POND_ERR_NOT_CONVERGED = -6 /* a node reached max_iter (only with pond_set_strict) */
} pond_status;

/* lattices: consts.h:6-12 picks one at compile time; here it is a parameter */
enum { POND_D1Q5 = 0, POND_D3Q27 = 1, POND_D3Q125 = 2 };
/* interpolation at the departure point (steps.cu:444-463 call sites) */
enum {
  POND_LAGR2 = 2, POND_LAGR3 = 3, POND_LAGR4 = 4, POND_LAGR5 = 5, /* propagate<N>, steps.cu:986 */
  POND_FIXED3 = 6, /* quadratic, origin fixed at coord-1: PonDstepD3Q125 steps.cu:151 */
  POND_TVD = 7,    /* flux-difference minmod form, steps.cu:118-124 with call site :447 */
  POND_WENO5 = 8,  /* propagateWENO<3,5>, steps.cu:774-825 (call site :458); in 3D the smoothness
                      indicators read the row y = z = floor(crd.x+0.5) as the reference does (:783) */
  /* one-dimensional meshes (D1Q5, Ny = Nz = 1, periodic), with a node mask: */
  POND_GAP2 = 9,        /* linear between the nearest active nodes, propagate_nonequal_1D<2>,
                           steps.cu:1122-1149 (call site :449) */
  POND_NONUNIFORM3 = 10, /* quadratic Lagrange on the node positions of x-1, x, x+1,
                           propagateNR_1D + LagrPolNR_1D, steps.cu:882-908,590-594 (call site :453) */
  /* centred WENO5: the candidates' y and z windows centred on the departure
     point (nodes floor(c+0.5)-1 .. floor(c+0.5)+1; the reference's start at
     floor(c+0.5) and extrapolate, steps.cu:776-778) and the smoothness row
     through it (y = floor(crd.y+0.5), z = floor(crd.z+0.5) instead of the
     reference's y = z = floor(crd.x+0.5)); the same as POND_WENO5 on 1D grids */
  POND_WENO5_ROW = 11
};
/* boundaries per axis: periodic is the reference (steps.cu:1015-1017); mirror
   is its disabled outflow reflection (steps.cu:1004-1013); clamp = zero gradient;
   inflow = below the low end a ghost node at equilibrium in the state set by
   pond_set_inflow (Dirichlet inflow), above the high end zero gradient
   (outflow).  The reference has no inflow boundary.  Inflow runs with the
   D3Q27/D3Q125 WENO5 schemes and the D3Q125 fixed-origin quadratic. */
enum { POND_BC_PERIODIC = 0, POND_BC_CLAMP = 1, POND_BC_MIRROR = 2, POND_BC_INFLOW = 3 };
/* arithmetic of populations, interpolation and collision; conserved-moment
   sums and the convergence test are float64 in both */
enum { POND_FP32 = 0, POND_FP64 = 1 };
/* built-in initial conditions for pond_init (init.cu:2-108 keeps its library
   of ICs as overwritten assignments; each is a separate choice here) */
enum {
  POND_IC_ACOUSTIC = 0,  /* small-amplitude isentropic wave, init.cu:43-50 (the shipped IC) */
  POND_IC_SOD_X = 1,     /* planar Riemann problem along x */
  POND_IC_SPHERE = 2,    /* spherical Riemann problem */
  POND_IC_TGV = 3,       /* compressible Taylor-Green vortex, init.cu:54-65 */
  POND_IC_UNIFORM = 4    /* rho, u, T constant */
};

/* LBMParams (structs.cuh:100-122) + PhysPars (:96-99) + the compile-time
   switches of consts.h / params.h, as runtime fields */
typedef struct {
  int64_t Nx, Ny, Nz;
  int lattice;
  int interp;
  int precision;
  int bc[3];
  double tau;      /* relaxation time; the step uses dtau = 1/tau */
  double dt;       /* time advanced per step (bookkeeping, LBMParams::dt) */
  double tol_abs;  /* isConv: |new-old| < tol_abs + tol_rel*|new| on u, T and every f */
  double tol_rel;
  int max_iter;    /* fixed-point iteration cap (steps.cu:422: 100) */
  int device;      /* CUDA device ordinal */
  int learned;     /* 1: start each node's iteration from the predictor's gauge */
  int ddf;         /* 1: energy populations (double-distribution extension; D1Q5 on 1D grids,
                      D3Q27 with Lagrange 2-5, D3Q125 fixed-origin quadratic): a second
                      population set carries the total energy, gamma = (Dim+dof+2)/(Dim+dof);
                      completes the reference's DDF scaffolding (structs.cuh:37-39,336-341,391-394,
                      lbpack.cu:18-20, steps.cu:233-236) */
  int ddf_dof;     /* extra degrees of freedom dof >= 0 of the extension (4: gamma = 1.4 in 1D) */
  int reserved[3];
} pond_params;

/* diagnostics of the last completed step (update.cu:124-135, diagn.cu:24-30) */
typedef struct {
  double mass;        /* sum rho */
  double moment[3];   /* sum rho*u (the reference prints the x component) */
  double enrg;        /* sum rho*(u.u + Dim*T)  (update.cu:67) */
  double k;           /* sum 0.5|u|^2 dx dy dz/(8 pi^3), dx = 2pi/Nx (diagn.cu:18) */
  int32_t niter_max;  /* LBMParams::NiterMax */
  int32_t pad;
  double niter_mean;
  int64_t niter_sum;
  int64_t nonconverged; /* nodes that reached max_iter without meeting the tolerance */
  int64_t istep;
  double curtime;
} pond_diag;

typedef struct pond_ctx pond_ctx;

int pond_abi_version(void);
const char* pond_status_string(int status);
/* message of the last failing call on this thread */
const char* pond_last_error_string(void);

int pond_params_default(int lattice, pond_params* out);
int pond_create(const pond_params* params, pond_ctx** out);
int pond_destroy(pond_ctx* ctx);
int pond_get_params(const pond_ctx* ctx, pond_params* out);
int pond_q(int lattice);
/* lattice tables in the reference's population order (consts.h): xi[3*Q]
   velocity components of each population at T = TLat (ef, or e for D3Q27),
   w[Q] weights, tlat_dim[2] = {TLat, Dim}; any pointer may be NULL.  Host only. */
int pond_lattice_tables(int lattice, double* xi, double* w, double* tlat_dim);

/* ic_params: ACOUSTIC {T0, amplitude, gamma}; SOD_X {x0, rhoL, uL, TL, rhoR, uR, TR};
   SPHERE {cx, cy, cz, radius, rho_in, T_in, rho_out, T_out};
   TGV {U0, T0, rho0, gamma}; UNIFORM {rho, ux, uy, uz, T} */
int pond_init(pond_ctx* ctx, int ic, const double* ic_params, int n_params);
/* upload a state from host memory; f == NULL applies set_base (f_i = w_i*rho);
   a context with energy populations (ddf = 1) also gets them at equilibrium,
   h_i = rho w_i (|v_i|^2 + ddf_dof T) */
int pond_set_state(pond_ctx* ctx, const double* f, const double* rho, const double* g);
int pond_get_state(pond_ctx* ctx, double* f, double* rho, double* g);
/* energy populations h[Q*N] (reference population order) of a ddf = 1 context:
   the reference's Cell::h (structs.cuh:37-39), which its scaffolding never
   initialises or stores; set after pond_set_state / pond_init */
int pond_set_energy(pond_ctx* ctx, const double* h);
int pond_get_energy(pond_ctx* ctx, double* h);
/* any pointer may be NULL; each receives N values */
int pond_get_fields(pond_ctx* ctx, double* rho, double* ux, double* uy, double* uz, double* T);
/* state of the inflow ghost node of POND_BC_INFLOW axes: rho > 0, u, T > 0
   (finite); needed before the first step of such a context.  Its populations
   are f_i = rho w_i in the gauge (u, T) (set_base, lbpack.cu:15-21), with
   energy populations at their equilibrium when the context carries them. */
int pond_set_inflow(pond_ctx* ctx, double rho, double ux, double uy, double uz, double T);
/* Convergence tolerance of the gauge alone: the iteration's test on u and T
   uses |new-old| < tol_abs + tol_rel*|new| with these values, the test on
   every population keeps params.tol_abs / tol_rel.  The reference uses one
   pair for both (isConv, steps.cu:58-75); a float32 context can so test the
   float64 gauge residual below the float32 rounding floor of the
   populations.  A negative value restores the params' pair.  Not used by the
   batched 1D mode. */
int pond_set_gauge_tolerance(pond_ctx* ctx, double tol_abs, double tol_rel);
/* advance nsteps steps (calcStep without drop/diagnostics printing) */
int pond_step(pond_ctx* ctx, int nsteps);
int pond_diagnostics(pond_ctx* ctx, pond_diag* out);
/* strict = 1: pond_step reads each step's counters back and returns
   POND_ERR_NOT_CONVERGED after the first step that left a node at max_iter
   (that step is complete and counted; the reference prints NiterMax and goes
   on, update.cu:131).  strict = 0 (default): the count is in pond_diagnostics. */
int pond_set_strict(pond_ctx* ctx, int strict);
/* the step counter, simulated time and dt of a resumed run (LBMParamsHost
   iStep / curtime / dt); dt <= 0 keeps the current dt.  Host bookkeeping only. */
int pond_set_clock(pond_ctx* ctx, int64_t istep, double curtime, double dt);
/* per-node iteration counts of the last step (int32[N]); needs pond_keep_niter(ctx, 1) before the step */
int pond_keep_niter(pond_ctx* ctx, int on);
int pond_get_niter(pond_ctx* ctx, int32_t* niter);
/* keep the gauge of one more time level (needed by pond_collect_pairs) */
int pond_keep_history(pond_ctx* ctx, int on);

/* the context's CUDA stream (a cudaStream_t) */
void* pond_stream(pond_ctx* ctx);
/* device pointers of the current state (for zero-copy callers on the same device):
   f[Q*N], rho[N], g[4*N] in the context's precision (float or double) */
int pond_device_state(pond_ctx* ctx, void** f, void** rho, void** g);
/* synchronous device-time of the last pond_step call's step kernels, in ms */
int pond_last_step_ms(pond_ctx* ctx, float* ms);
/* host transfers in the context's own precision (float for POND_FP32, double
   for POND_FP64), no conversion: f[Q*N], rho[N], g[4*N]; pinned host memory
   gives full PCIe bandwidth.  pond_upload_state writes the current buffer only. */
int pond_upload_state(pond_ctx* ctx, const void* f, const void* rho, const void* g);
/* any of f, rho, g may be NULL */
int pond_download_state(pond_ctx* ctx, void* f, void* rho, void* g);
/* copy the state of src into dst (same lattice and grid; the precision is
   converted on the device): both stored time levels and the step counter */
int pond_copy_state(pond_ctx* dst, pond_ctx* src);
/* work of the last step, summed over nodes and iterations (the count behind
   the compute roofline): for the D3Q27 float32 kernel the floating-point
   operations of its basis contractions (a multiply-add counts 2), for the
   other kernels the stencil nodes transformed */
int pond_last_step_work(pond_ctx* ctx, int64_t* work);

/* ---- one-dimensional mesh: node mask, AMR, node positions -------------
   A context made with POND_GAP2 or POND_NONUNIFORM3 owns a node mask (the
   reference's Cinfo::set, structs.cuh:89-94; every node active after
   pond_create and after pond_init, whose fill sets it, init.cu:106).  The
   step skips inactive nodes (steps.cu:359) and carries them over unchanged;
   diagnostics sum active nodes only (update.cu:56-69).  A POND_NONUNIFORM3
   context also owns node positions (Cell::p.x under NRMESH,
   structs.cuh:40-42; p_x = x after pond_create and pond_init,
   init.cu:100-103) and weights the diagnostics by half the distance between
   each node's neighbours (update.cu:59-62). */
/* mask[N] bytes, nonzero = active */
int pond_set_mask(pond_ctx* ctx, const uint8_t* mask);
int pond_get_mask(pond_ctx* ctx, uint8_t* mask);
/* positions[N]: finite, strictly increasing, last - first < Nx (node units) */
int pond_set_positions(pond_ctx* ctx, const double* positions);
int pond_get_positions(pond_ctx* ctx, double* positions);
/* AMR_add (amr.cu:1-27, with cinfo_setnew_reset / cinfo_set_new of
   update.cu:30-39) on the current state: every active node whose next active
   node (periodic) differs from it by (du_x)^2 / min(T) > tol or
   |1 - rho/rho_next| > tol activates the midpoint of an even gap between
   them, holding the average of the two records in both time levels (the
   reference's tol is 0.01).  *added = nodes activated; *limit_hits = nodes
   over the threshold with an adjacent neighbour (the reference prints
   "limit of cells division exceeded").  Either output may be NULL. */
int pond_amr_refine(pond_ctx* ctx, double tol, int64_t* added, int64_t* limit_hits);
/* AMR_remove (amr.cu:28-55): deactivates, in one pass in node order over
   the mask as it changes, each active node whose nearest active neighbours
   are both within 3 nodes and within tol in (du_x)^2 / T and density ratio.
   The result equals the reference's serial pass; it is computed as a
   parallel prefix over the pass's 8-state automaton. */
int pond_amr_coarsen(pond_ctx* ctx, double tol, int64_t* removed);

/* ---- time-step rescaling (TimeCorr, update.cu:15-28) ------------------
   Multiplies every node's u by s and T by s*s in the current state (lattice
   velocities are displacements per step) and the context's dt by s; any
   lattice.  pond_set_dt_adapt applies the reference's disabled policy after
   every step (update.cu:121-123): s = 1/2 when the step's NiterMax >= niter_hi,
   s = 2 when it is <= niter_lo (the reference's values: 1000 and 4); on = 0
   turns it off.  The step's diagnostics are rescaled with the state. */
int pond_rescale_time(pond_ctx* ctx, double s);
int pond_set_dt_adapt(pond_ctx* ctx, int on, int niter_hi, int niter_lo);

/* ---- learned starting gauge ------------------------------------------
   A small network (39 -> H -> H -> 4, tanh, H = 64 or 128; BF16 tensor-core
   GEMMs with float32 accumulation, float32 master weights, Adam) predicts
   each node's converged gauge from the pre-step (rho, u, T) of the node and
   its six face neighbours and the node's last gauge increment.  The
   prediction only replaces the starting gauge of the unchanged fixed-point
   iteration, which still runs to the same tolerance.
   Features (39), c = sqrt(T/TLat): centre c, u/c (3), T/TLat; per neighbour
   (-x,+x,-y,+y,-z,+z) rho_m/rho-1, (u_m-u)/c (3), T_m/T-1; the centre's last
   increment (u^n-u^{n-1})/c (3), (T^n-T^{n-1})/T.
   Targets (4): the step's increment of the gauge, (u*-u)/c (3), (T*-T)/T.
   Feature/target rows are float32 in device memory, row-major.  No
   counterpart in the reference (whose iteration starts from the previous
   gauge, steps.cu:360). */
typedef struct pond_mlp pond_mlp;
int pond_mlp_create(int hidden, uint64_t seed, int device, pond_mlp** out);
int pond_mlp_destroy(pond_mlp* net);
int pond_mlp_num_params(const pond_mlp* net);
/* params: W1[H][39], b1[H], W2[H][H], b2[H], W3[4][H], b3[4];
   stats: xmean[39], xstd[39], ymean[4], ystd[4] (either pointer may be NULL) */
int pond_mlp_get_params(pond_mlp* net, float* params, float* stats);
int pond_mlp_set_params(pond_mlp* net, const float* params, const float* stats);
/* standardisation statistics from n device rows X[n][39], Y[n][4] */
int pond_mlp_fit_stats(pond_mlp* net, const float* X, const float* Y, int64_t n);
/* `steps` Adam steps (beta 0.9/0.999) of mean-squared error on standardised
   targets, minibatches of `batch` rows taken cyclically; loss_out (host,
   `steps` floats) may be NULL */
int pond_mlp_train(pond_mlp* net, const float* X, const float* Y, int64_t n, int batch, int steps, float lr,
                   float* loss_out);
/* full-batch gradient (host, num_params floats) and loss; n must be a
   multiple of the training tile (128 rows for H = 64, 64 for H = 128) */
int pond_mlp_gradients(pond_mlp* net, const float* X, const float* Y, int64_t n, float* grad, float* loss);
/* de-standardised outputs Y[n][4] for raw feature rows X[n][39] (device) */
int pond_mlp_forward(pond_mlp* net, const float* X, float* Y, int64_t n);
/* training pairs from the last step (needs pond_keep_history(ctx, 1) before
   it): pre-step features and the increment target, for nodes offset +
   k*stride (offset = seed % stride) whose 7-node stencil is not exactly
   uniform in space; *written rows (<= capacity),
   in no particular order; node (device int64[capacity], may be NULL)
   receives each row's node index */
int pond_collect_pairs(pond_ctx* ctx, float* X, float* Y, int64_t* node, int64_t capacity, int64_t stride,
                       uint64_t seed, int64_t* written);
/* bind a network to a context (NULL detaches): every following pond_step
   first predicts each node's starting gauge: the previous gauge plus the
   network's increment on active nodes, i.e. nodes whose 7-node stencil is
   not exactly uniform and whose last increment (largest of the 4 temporal
   features) is at least `gate`; other nodes start from the previous gauge. */
int pond_set_predictor(pond_ctx* ctx, pond_mlp* net, float gate);
/* without a bound network: start each node from the linear extrapolation
   g^n + (g^n - g^{n-1}) of its last two gauges (on = 1) or from g^n (on = 0,
   the reference) */
int pond_set_extrapolation(pond_ctx* ctx, int on);
/* the starting gauge the bound network predicts for the current state
   (device float[4*N], planes u_x, u_y, u_z, T) */
int pond_predict(pond_ctx* ctx, float* guess);

/* Allocation-free step.  This entry point has no counterpart in the
   reference, which only steps its own global buffers.

   One D3Q27 float32 step (Lagrange order 2-4, params->interp) from the
   caller's device buffers f_in/rho_in/g_in into f_out/rho_out/g_out (layout
   as above, float, N = Nx*Ny*Nz nodes), with the step's diagnostics written
   to diag_out, a pond_diag in DEVICE memory; istep and curtime are left 0.
   Work is queued on `stream` (a cudaStream_t, 0 = legacy default stream); the
   call does not synchronise.  params->device is ignored: the current device
   is used.  The six state buffers must be pairwise disjoint (an output that
   overlaps an input or another output is rejected with POND_ERR_ARG: the
   step reads neighbours of the input while other CTAs write the output).
   params->learned and params->ddf must be 0 (POND_ERR_UNSUPPORTED); tau,
   max_iter (1..100000) and the tolerances are checked as in pond_create.

   It is meant for callers that cannot let a library call cudaMalloc: code
   that owns all device memory through its own pool or a budget fixed at
   start-up, or that must not stall on an allocation inside its time loop.
   It calls no cudaMalloc, cudaFree or allocating library routine.  Its only
   scratch, one partial-sum record per step CTA, lives in a fixed
   POND_NOALLOC_SCRATCH_BYTES array in the library's device memory, which
   every GPU that loads the library holds until the process exits.  Grids that
   need more than 65536 step CTAs (more than 256^3 nodes, counted in 32x4x2
   tiles) are rejected with POND_ERR_ARG.  The first call on each device looks
   up that array's device address (and opts the kernel into its shared
   memory); make that first call before any stream capture.  All calls share
   the array and every call rewrites it: calls whose kernels overlap on a GPU
   (other streams, other threads) race on it, so serialise them on one stream.
   The looked-up address is kept for the life of the process: do not call
   cudaDeviceReset on a device between calls of this entry point. */
#define POND_NOALLOC_SCRATCH_BYTES 5242880
int pond_step_noalloc(const pond_params* params, const float* f_in, const float* rho_in, const float* g_in,
                      float* f_out, float* rho_out, float* g_out, pond_diag* diag_out, void* stream);

/* Pipelined step from host buffers.  No counterpart in the reference, whose
   state never leaves the device; this is calcStep plus the two PCIe copies a
   caller with host-resident states would otherwise issue around it.

   Queues the copy of an input state (f[Q*N], rho[N], g[4*N] in the
   context's precision, pinned host memory for full PCIe speed) to the
   device, one plain step from it (no predictor: POND_ERR_STATE while one is
   bound), and the copy of the result's rho and g to rho_out / g_out (either
   may be NULL); returns without waiting.  Uploads and read-backs run on two
   copy streams of the context, so consecutive calls overlap their copies with
   the neighbouring steps.  The host buffers of a call must stay untouched
   until pond_sync; the last result is the context's current state.  Any
   other call on the context waits for the queued work first.  The first call
   allocates two input slots of one state each on the device. */
int pond_step_host(pond_ctx* ctx, const void* f_in, const void* rho_in, const void* g_in, void* rho_out,
                   void* g_out);
/* wait for all queued pond_step_host work */
int pond_sync(pond_ctx* ctx);

/* ---- Batched 1D mode.  No counterpart in the reference, which steps one
   grid per process (lbm.cu:179-298); the per-node arithmetic is the D1Q5
   step above (LBMpull, steps.cu:356-588), float32 populations with float64
   moments and convergence test.

   A batch holds independent D1Q5 problems of 1..4096 nodes each with
   zero-gradient (clamped) ends.  Problems are packed into bins of up to 6144
   nodes; one persistent kernel launch advances every bin K steps, each CTA
   holding its bin in shared memory, and the launch sequence is captured once
   in a CUDA graph and replayed.  Host arrays are float64 in the caller's
   problem order, problems concatenated (f: 5 planes of pond_batch_nodes()). */
typedef struct pond_batch pond_batch;
/* interp: POND_WENO5 or POND_LAGR4; tau > 0.5 */
int pond_batch_create(int nproblems, const int32_t* lengths, int interp, double tau, double tol_abs,
                      double tol_rel, int max_iter, int device, pond_batch** out);
int pond_batch_destroy(pond_batch* batch);
int64_t pond_batch_nodes(const pond_batch* batch);
int32_t pond_batch_bins(const pond_batch* batch);
/* macroscopic state per node (rho, u finite, T > 0); populations become
   w_i*rho in each node's own gauge; resets the step counter */
int pond_batch_set_state(pond_batch* batch, const double* rho, const double* u, const double* T);
/* any pointer may be NULL */
int pond_batch_get_state(pond_batch* batch, double* f, double* rho, double* u, double* T);
/* training pairs, written during pond_batch_run: every `every` steps (0 =
   off) at local coordinates x % stride == 0, X[capacity][21] (device) gets
   the pre-step rho, u, T at x-3..x+3 (clamped), Y[capacity][2] the converged
   u, T of that step; rows in no particular order, the row count restarts at
   0 with each call */
int pond_batch_set_pairs(pond_batch* batch, float* X, float* Y, int64_t capacity, int every, int stride);
int pond_batch_pairs_written(pond_batch* batch, int64_t* rows);
/* advance every problem nsteps steps, k steps per persistent launch; *ms
   (may be NULL) receives the device time of the call (CUDA events) */
int pond_batch_run(pond_batch* batch, int nsteps, int k, float* ms);
/* iteration statistics of the last pond_batch_run */
int pond_batch_stats(pond_batch* batch, int64_t* niter_sum, int64_t* nonconverged, int32_t* niter_max);
/* Tile of the persistent kernel: threads per CTA (256, 512, 768 or 1024)
   and lane_cap, the iterations a node runs on one lane before it is handed
   to a whole warp (>= 1; >= max_iter keeps every node on one lane). */
int pond_batch_set_tile(pond_batch* batch, int threads, int lane_cap);
int pond_batch_get_tile(const pond_batch* batch, int* threads, int* lane_cap);
/* time probe_steps steps with each of ncand candidate tiles (int32 pairs
   threads, lane_cap) on the current state, keep the fastest, restore the
   state; ms_out (ncand floats) and best (its index) may be NULL */
int pond_batch_autotune(pond_batch* batch, int probe_steps, const int32_t* tiles, int ncand, float* ms_out,
                        int* best);

#ifdef __cplusplus
}
#endif
#endif
