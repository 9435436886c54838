/*
 * FP64 CPU oracle for the Particles-on-Demand (PonD) pull step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, in plain C++ with OpenMP,
 * the reference's per-node PonD step (engrab6/lbmPonD: steps.cu LBMpull /
 * PonDstepD3Q125, structs.cuh Cell::transfer_gauge / calcMoments, consts.h
 * lattice tables).  It is the checker for the CUDA path and the timed CPU
 * baseline; the product library never links, loads or calls it.
 *
 * Layout of every state array (the same as the CUDA library's host view):
 *   f[q * N + n]      populations, q < Q, n = x + nx*(y + ny*z)
 *   rho[n]            density
 *   g[k * N + n]      gauge: k = 0,1,2 -> u_x,u_y,u_z ; k = 3 -> T
 * Population order is the reference's (consts.h e_host order).
 */
#ifndef POND_ORACLE_H
#define POND_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_D1Q5 = 0, ORC_D3Q27 = 1, ORC_D3Q125 = 2 };
/* interpolation schemes; numbers 2..5 are Lagrange orders (steps.cu:986 propagate<N>) */
enum { ORC_LAGR2 = 2, ORC_LAGR3 = 3, ORC_LAGR4 = 4, ORC_LAGR5 = 5,
       ORC_FIXED3 = 6,   /* quadratic, stencil origin fixed at coord-1 (steps.cu:151 PonDstepD3Q125) */
       ORC_TVD = 7,      /* flux-difference minmod form (steps.cu:118 FluxTVDdif, call site :447) */
       ORC_WENO5 = 8,    /* propagateWENO<3,5> (steps.cu:774) */
       ORC_GAP2 = 9,     /* linear between the nearest active nodes, propagate_nonequal_1D<2> (steps.cu:1122) */
       ORC_NONUNIFORM3 = 10, /* quadratic on node positions, propagateNR_1D (steps.cu:882) */
       ORC_WENO5_ROW = 11 }; /* propagateWENO<3,5> centred: y, z windows floor(c+0.5)-1 .. +1 (the
                                reference's :776-778 start at floor(c+0.5)) and the smoothness row
                                through the departure point (the reference's :783 reads row y = z = x) */
/* INFLOW: a ghost node below the low end holding the equilibrium of
   orc_params.inflow (rho, u_x, u_y, u_z, T), zero gradient above the high end */
enum { ORC_BC_PERIODIC = 0, ORC_BC_CLAMP = 1, ORC_BC_MIRROR = 2, ORC_BC_INFLOW = 3 };

typedef struct {
  int lattice;
  int interp;
  int64_t nx, ny, nz;
  int bc[3];          /* per axis */
  double tau;         /* BGK relaxation time; dtau = 1/tau (structs.cuh:98) */
  double tol_abs;     /* isConv absolute tolerance (steps.cu:62) */
  double tol_rel;     /* isConv relative tolerance (steps.cu:63) */
  int max_iter;       /* iteration cap (steps.cu:422) */
  int nthreads;       /* 0 = OpenMP default */
  double dof;         /* double-distribution extension: extra degrees of freedom (orc_step_ddf) */
  double inflow[5];   /* state of the ORC_BC_INFLOW ghost node: rho, u_x, u_y, u_z, T */
  double tolg[2];     /* abs, rel tolerance of the test on u, T; negative: tol_abs, tol_rel */
} orc_params;

int    orc_q(int lattice);
/* xi[3*Q] real lattice directions (ef, or e for D3Q27), e[3*Q] integer
   directions, w[Q] weights, out[0]=TLat, out[1]=Dim */
int    orc_tables(int lattice, double* xi, int* e, double* w, double* tlat_dim);
/* reference-order reverse maps per axis (consts.h / lbm.cu:206-244) */
int    orc_reverse(int lattice, int* rev_x, int* rev_y, int* rev_z);
void   orc_set_base(int lattice, double rho, const double* uT, double* f);
double orc_transfer_gauge(int lattice, const double* f, const double* uT_src,
                          const double* uT_dst, int inew);
void   orc_calc_moments(int lattice, const double* f, const double* vi,
                        double* rho, double* uT);
double orc_lagr_pol(int n, int ix, int iy, int iz, double sx, double sy, double sz);
/* one pull step; guess (4*N, optional) replaces each node's starting gauge;
   niter (N, optional) receives each node's iteration count.
   Returns the number of nodes that hit max_iter without converging. */
int64_t orc_step(const orc_params* p,
                 const double* f_in, const double* rho_in, const double* g_in,
                 const double* guess,
                 double* f_out, double* rho_out, double* g_out, int* niter);
/* Double-distribution extension (energy populations h, same layout as f):
   gamma = (Dim + dof + 2) / (Dim + dof).  orc_set_energy gives the
   equilibrium h of one node; orc_step_ddf is orc_step carrying h. */
void   orc_set_energy(int lattice, double rho, const double* uT, double dof, double* h);
int64_t orc_step_ddf(const orc_params* p,
                     const double* f_in, const double* h_in, const double* rho_in, const double* g_in,
                     const double* guess,
                     double* f_out, double* h_out, double* rho_out, double* g_out, int* niter);
/* One-dimensional mesh (D1Q5, nx x 1 x 1, periodic): orc_step with a node
   mask (Cinfo::set, structs.cuh:92; NULL = every node active) and node
   positions (Cell::p under NRMESH, structs.cuh:40-42; NULL = p_x = x).
   An inactive node is skipped by the step (steps.cu:359) and copied through.
   Schemes ORC_GAP2 and ORC_NONUNIFORM3 read the mask / the positions. */
int64_t orc_step_mesh(const orc_params* p, const double* f_in, const double* rho_in, const double* g_in,
                      const uint8_t* mask, const double* pos,
                      double* f_out, double* rho_out, double* g_out, int* niter);
/* AMR_add (amr.cu:1-27) with cinfo_setnew_reset / cinfo_set_new
   (update.cu:30-39): every active node whose next active node to the right
   (periodic) differs by (du)^2/min(T) > tol or |1 - rho/rho_next| > tol gets
   the midpoint of an even gap activated, holding the average of the two
   records (written to the state in place).  Decisions read the mask as it
   was on entry.  Returns the nodes added; *limit_hits counts the nodes whose
   neighbour is adjacent (the reference's "limit of cells division exceeded"). */
int64_t orc_amr_refine(const orc_params* p, double* f, double* rho, double* g, uint8_t* mask, double tol,
                       int64_t* limit_hits);
/* AMR_remove (amr.cu:28-55): one serial pass in node order deactivating
   every active node whose nearest active neighbours (in the mask as updated
   so far) are both within 3 nodes and within tol of it in (du)^2/T and
   density ratio.  Returns the nodes removed. */
int64_t orc_amr_coarsen(const orc_params* p, const double* rho, const double* g, uint8_t* mask, double tol);
int    orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
