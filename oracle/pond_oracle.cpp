// FP64 CPU oracle for the PonD pull step -- TEST INFRASTRUCTURE ONLY.
//
// A plain restatement of the reference step (engrab6/lbmPonD), used by the
// tests as the correctness checker and by bench.py as the timed CPU baseline.
// Every function cites the reference lines it restates.  Arithmetic follows
// the reference expression by expression (same operand order), in double,
// so that it agrees with the reference's USE_DOUBLE build to rounding.
#include "pond_oracle.h"

#include <cmath>
#include <cstring>
#include <cstdlib>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int QMAX = 125;
// consts.h:117-118 / :142-143: the two positive roots scaled lattice speeds
constexpr double EC1 = 1.3556261799742657;
constexpr double EC2 = 2.8569700138728056;

struct Lattice {
  int kind = -1;
  int Q = 0;
  double TLat = 1, Dim = 1;
  double xi[QMAX][3];  // ef (D1Q5, D3Q125) or double(e) (D3Q27)
  int e[QMAX][3];
  double w[QMAX];
  int rev[3][QMAX];
};

Lattice make_lattice(int kind) {
  Lattice L;
  L.kind = kind;
  std::memset(L.xi, 0, sizeof(L.xi));
  std::memset(L.e, 0, sizeof(L.e));
  const double ec1d = EC1 * EC1, ec2d = EC2 * EC2;
  if (kind == ORC_D1Q5) {  // consts.h:111-134
    L.Q = 5; L.TLat = 1; L.Dim = 1;
    const double TLat = L.TLat;
    const double C[5] = {0, EC1, -EC1, EC2, -EC2};
    const int CI[5] = {0, int(EC1), -int(EC1), int(EC2), -int(EC2)};
    const double W0 = (3 * TLat * TLat - (ec1d + ec2d) * TLat + ec1d * ec2d) / (ec1d * ec2d);
    const double W1 = TLat * (ec2d - 3 * TLat) / (2 * ec1d * (ec2d - ec1d));
    const double W2 = TLat * (ec1d - 3 * TLat) / (2 * ec2d * (ec1d - ec2d));
    const double W[5] = {W0, W1, W1, W2, W2};
    for (int i = 0; i < 5; i++) { L.xi[i][0] = C[i]; L.e[i][0] = CI[i]; L.w[i] = W[i]; }
  } else if (kind == ORC_D3Q27) {  // consts.h:14-65
    L.Q = 27; L.TLat = 1. / 3.; L.Dim = 3;
    static const int E[27][3] = {
        {0, 0, 0},
        {1, 0, 0},  {0, 1, 0},  {0, 0, 1},  {1, 1, 0},  {1, 0, 1},  {0, 1, 1},  {1, 1, 1},
        {-1, 0, 0}, {-1, 1, 0}, {-1, 0, 1}, {-1, 1, 1},
        {0, -1, 0}, {0, -1, 1}, {1, -1, 0}, {1, -1, 1},
        {0, 0, -1}, {1, 0, -1}, {0, 1, -1}, {1, 1, -1},
        {-1, -1, 0}, {-1, -1, 1},
        {-1, 0, -1}, {-1, 1, -1},
        {0, -1, -1}, {1, -1, -1},
        {-1, -1, -1}};
    const double TLat = L.TLat;
    const double W0 = (1 - TLat) * (1 - TLat) * (1 - TLat);
    const double W1 = (1 - TLat) * (1 - TLat) * TLat / 2.0;
    const double W2 = (1 - TLat) * TLat * TLat / 4.0;
    const double W3 = TLat * TLat * TLat / 8.;
    const double Wn[4] = {W0, W1, W2, W3};
    for (int i = 0; i < 27; i++) {
      int nz = 0;
      for (int a = 0; a < 3; a++) { L.e[i][a] = E[i][a]; L.xi[i][a] = E[i][a]; nz += E[i][a] != 0; }
      L.w[i] = Wn[nz];
    }
  } else if (kind == ORC_D3Q125) {  // consts.h:136-245 (index = 25*a + 5*b + c)
    L.Q = 125; L.TLat = 1; L.Dim = 3;
    const double TLat = L.TLat;
    const double C[5] = {0, EC1, -EC1, EC2, -EC2};
    const int CI[5] = {0, int(EC1), -int(EC1), int(EC2), -int(EC2)};
    const double W0 = (3 * TLat * TLat - (ec1d + ec2d) * TLat + ec1d * ec2d) / (ec1d * ec2d);
    const double W1 = TLat * (ec2d - 3 * TLat) / (2 * ec1d * (ec2d - ec1d));
    const double W2 = TLat * (ec1d - 3 * TLat) / (2 * ec2d * (ec1d - ec2d));
    const double W[5] = {W0, W1, W1, W2, W2};
    for (int a = 0; a < 5; a++)
      for (int b = 0; b < 5; b++)
        for (int c = 0; c < 5; c++) {
          const int i = 25 * a + 5 * b + c;
          L.xi[i][0] = C[a]; L.xi[i][1] = C[b]; L.xi[i][2] = C[c];
          L.e[i][0] = CI[a]; L.e[i][1] = CI[b]; L.e[i][2] = CI[c];
          L.w[i] = W[a] * W[b] * W[c];
        }
  } else {
    return L;
  }
  // reverse maps: the direction mirrored in one axis (consts.h:62-64 for
  // D3Q27, computed the same way for D3Q125 at lbm.cu:206-244)
  for (int ax = 0; ax < 3; ax++)
    for (int i = 0; i < L.Q; i++) {
      L.rev[ax][i] = i;
      if (L.xi[i][ax] == 0) continue;
      for (int j = 0; j < L.Q; j++) {
        bool ok = true;
        for (int b = 0; b < 3; b++) {
          const double want = (b == ax) ? -L.xi[i][b] : L.xi[i][b];
          if (L.xi[j][b] != want) ok = false;
        }
        if (ok) { L.rev[ax][i] = j; break; }
      }
    }
  return L;
}

const Lattice& lattice(int kind) {
  static const Lattice L0 = make_lattice(ORC_D1Q5);
  static const Lattice L1 = make_lattice(ORC_D3Q27);
  static const Lattice L2 = make_lattice(ORC_D3Q125);
  static const Lattice Lbad = make_lattice(-1);
  switch (kind) {
    case ORC_D1Q5: return L0;
    case ORC_D3Q27: return L1;
    case ORC_D3Q125: return L2;
    default: return Lbad;
  }
}

// params.h:101-112
inline int sign_i(double v) { return (0.0 < v) - (v < 0.0); }
inline double sqrts(double v) { return std::sqrt(std::fabs(v)) * sign_i(v); }
inline bool finite(double v) { return !std::isnan(v) && !std::isinf(v); }

struct Cell {
  double f[QMAX];
  double h[QMAX];  // energy populations of the double-distribution extension (unused otherwise)
  double rho;
  double uT[4];
};

// lbpack.cu:15-21 Cell::set_base
void set_base(const Lattice& L, Cell& c, double r, const double* uT) {
  c.rho = r;
  for (int k = 0; k < 4; k++) c.uT[k] = uT[k];
  for (int i = 0; i < L.Q; i++) c.f[i] = L.w[i] * c.rho;
}

// Equilibrium energy populations of the double-distribution extension in the
// gauge uT: h_i = rho w_i (|v_i|^2 + dof T), v_i = sqrt(T/TLat) xi_i + u, so
// that sum_i h_i = rho (|u|^2 + (Dim + dof) T) (twice the total energy) and
// sum_i h_i v_i = rho u (|u|^2 + (Dim + 2 + dof) T) (twice the enthalpy flux).
// The reference's scaffolding (lbpack.cu:18-20, steps.cu:233-236) uses
// rho w_i (Dim T + |u|^2), whose flux lacks the pressure work.
void set_energy(const Lattice& L, Cell& c, double dof) {
  const double s = std::sqrt(std::fabs(c.uT[3]) / L.TLat);
  for (int i = 0; i < L.Q; i++) {
    double v2 = 0;
    for (int a = 0; a < 3; a++) {
      const double v = s * L.xi[i][a] + c.uT[a];
      v2 += v * v;
    }
    c.h[i] = c.rho * L.w[i] * (v2 + dof * c.uT[3]);
  }
}

// structs.cuh:343-551 Cell::transfer_gauge: population inew of cell c
// re-expressed in the gauge `base` = (u1, T1).  Non-finite terms are dropped
// (:390, :516, :542).  `energy` transfers the energy populations h instead of
// f (the reference's DDF branch, structs.cuh:391-394, applies the same
// transfer to h).
double transfer_gauge(const Lattice& L, const Cell& c, const double* base, int inew, bool energy = false) {
  const double* src = energy ? c.h : c.f;
  const double Tbase = L.TLat;
  const double u0x = c.uT[0], u0y = c.uT[1], u0z = c.uT[2];
  const double T0 = c.uT[3];
  const double u1x = base[0], u1y = base[1], u1z = base[2];
  const double T1 = base[3];
  double fnew = 0;
  double wk = 1. / (2 * T1), wl = wk, wm = wk;
  if (L.kind == ORC_D1Q5) {  // :352-395
    const double e1_to = L.xi[1][0] * sqrts(T1 / Tbase);
    const double e2_to = L.xi[3][0] * sqrts(T1 / Tbase);
    double e_fr[5], e_to[5];
    for (int i = 0; i < 5; i++) {
      e_fr[i] = L.xi[i][0] * sqrts(T0 / Tbase);
      e_to[i] = L.xi[i][0] * sqrts(T1 / Tbase);
    }
    if (L.xi[inew][0] == 0) wk = 1. / (e1_to * e1_to * e2_to * e2_to);
    else if (std::fabs(L.xi[inew][0]) == EC1) wk = 1. / (2 * e1_to * e1_to * (e1_to * e1_to - e2_to * e2_to));
    else wk = 1. / (2 * e2_to * e2_to * (e2_to * e2_to - e1_to * e1_to));
    const double M4moment = 0;
    fnew = wk * M4moment;
    for (int iold = 0; iold < 5; iold++) {
      double K0, K1, K2, K3, K4;
      K4 = 1;
      K3 = -4 * e_fr[iold] - e_to[inew];
      if (inew == 0) {
        K2 = 6 * e_fr[iold] * e_fr[iold] - (e1_to * e1_to + e2_to * e2_to);
        K1 = 2 * e_fr[iold] * (e1_to * e1_to + e2_to * e2_to - 2 * e_fr[iold] * e_fr[iold]);
        K0 = (e1_to * e1_to - e_fr[iold] * e_fr[iold]) * (e2_to * e2_to - e_fr[iold] * e_fr[iold]);
      } else {
        K2 = 6 * e_fr[iold] * e_fr[iold] + 3 * e_fr[iold] * e_to[inew] -
             (e1_to * e1_to + e2_to * e2_to - e_to[inew] * e_to[inew]);
        K1 = (2 * e_fr[iold] + e_to[inew]) * (e1_to * e1_to + e2_to * e2_to - e_to[inew] * e_to[inew]) -
             e_fr[iold] * e_fr[iold] * (4 * e_fr[iold] + 3 * e_to[inew]);
        K0 = e_fr[iold] * (e_fr[iold] * e_fr[iold] - (e1_to * e1_to + e2_to * e2_to) + e_to[inew] * e_to[inew]) *
             (e_fr[iold] + e_to[inew]);
      }
      const double difu = u1x - u0x;
      double difM4moment = u0x + e_fr[iold];
      difM4moment = difM4moment * difM4moment * difM4moment * difM4moment;
      difM4moment *= 0;
      const double gx = K4 * difu * difu * difu * difu + K3 * difu * difu * difu + K2 * difu * difu +
                        K1 * difu + K0 - difM4moment;
      const double fadd = wk * gx * src[iold];
      if (finite(fadd)) fnew += fadd;
    }
  } else if (L.kind == ORC_D3Q125) {  // :396-524
    const double S0 = sqrts(T0 / Tbase);
    const double S1 = sqrts(T1 / Tbase);
    const double e1_to = EC1 * S1;
    const double e2_to = EC2 * S1;
    auto wclass = [&](double v) {
      if (v == 0) return 1. / (e1_to * e1_to * e2_to * e2_to);
      if (std::fabs(v) == EC1) return 1. / (2 * e1_to * e1_to * (e1_to * e1_to - e2_to * e2_to));
      return 1. / (2 * e2_to * e2_to * (e2_to * e2_to - e1_to * e1_to));
    };
    wk = wclass(L.xi[inew][0]);
    wl = wclass(L.xi[inew][1]);
    wm = wclass(L.xi[inew][2]);
    const double dux = u0x - u1x, duy = u0y - u1y, duz = u0z - u1z;
    auto cls = [](double v) {
      if (v == +EC1) return 1;
      if (v == -EC1) return 2;
      if (v == +EC2) return 3;
      if (v == -EC2) return 4;
      return 0;
    };
    const int Xi = cls(L.xi[inew][0]), Yi = cls(L.xi[inew][1]), Zi = cls(L.xi[inew][2]);
    for (int iold = 0; iold < 125; iold++) {
      const double efx = L.xi[iold][0] * S0, efy = L.xi[iold][1] * S0, efz = L.xi[iold][2] * S0;
      const double fX[5] = {(dux + efx), (dux + efx - e1_to), (dux + efx + e1_to), (dux + efx - e2_to), (dux + efx + e2_to)};
      const double fY[5] = {(duy + efy), (duy + efy - e1_to), (duy + efy + e1_to), (duy + efy - e2_to), (duy + efy + e2_to)};
      const double fZ[5] = {(duz + efz), (duz + efz - e1_to), (duz + efz + e1_to), (duz + efz - e2_to), (duz + efz + e2_to)};
      const double gx = fX[(Xi + 1) % 5] * fX[(Xi + 2) % 5] * fX[(Xi + 3) % 5] * fX[(Xi + 4) % 5];
      const double gy = fY[(Yi + 1) % 5] * fY[(Yi + 2) % 5] * fY[(Yi + 3) % 5] * fY[(Yi + 4) % 5];
      const double gz = fZ[(Zi + 1) % 5] * fZ[(Zi + 2) % 5] * fZ[(Zi + 3) % 5] * fZ[(Zi + 4) % 5];
      const double gxyz = gx * gy * gz;
      const double fadd = wk * wl * wm * gxyz * src[iold];
      if (finite(fadd)) fnew += fadd;
    }
  } else {  // generic branch :525-548 (D3Q27)
    const int* en = L.e[inew];
    if (en[0] == 0) wk = -1. / T1;
    if (en[1] == 0) wl = -1. / T1;
    if (en[2] == 0) wm = -1. / T1;
    const double sT0 = std::sqrt(std::fabs(T0)), sT1 = std::sqrt(std::fabs(T1));
    const int sg0 = sign_i(T0), sg1 = sign_i(T1);
    for (int iold = 0; iold < L.Q; iold++) {
      const int* eo = L.e[iold];
      const double Ax_i = (u1x - u0x) * std::sqrt(Tbase) - eo[0] * sT0 * sg0;
      const double Ay_j = (u1y - u0y) * std::sqrt(Tbase) - eo[1] * sT0 * sg0;
      const double Az_p = (u1z - u0z) * std::sqrt(Tbase) - eo[2] * sT0 * sg0;
      double Bx_ik = T1; if (en[0] != 0) Bx_ik = en[0] * sT1 * sg1 * Ax_i;
      double By_jl = T1; if (en[1] != 0) By_jl = en[1] * sT1 * sg1 * Ay_j;
      double Bz_pm = T1; if (en[2] != 0) Bz_pm = en[2] * sT1 * sg1 * Az_p;
      const double gx = Ax_i * Ax_i - Bx_ik;
      const double gy = Ay_j * Ay_j - By_jl;
      const double gz = Az_p * Az_p - Bz_pm;
      double fadd = 0;
      if (L.Dim == 1) fadd = wk * gx * src[iold];
      else fadd = wk * wl * wm * gx * gy * gz * src[iold];
      if (finite(fadd)) fnew += fadd;
    }
  }
  return fnew;
}

// structs.cuh:315-342 Cell::calcMoments (M3 side computations are unused)
void calc_moments(const Lattice& L, Cell& c, const double (*vi)[3]) {
  c.rho = 0;
  double u[4] = {0, 0, 0, 0};
  for (int i = 0; i < L.Q; i++) {
    c.rho += c.f[i];
    const double dot = vi[i][0] * vi[i][0] + vi[i][1] * vi[i][1] + vi[i][2] * vi[i][2];
    u[0] += c.f[i] * vi[i][0];
    u[1] += c.f[i] * vi[i][1];
    u[2] += c.f[i] * vi[i][2];
    u[3] += c.f[i] * dot;
  }
  if (c.rho != 0) for (int k = 0; k < 4; k++) u[k] /= c.rho;
  u[3] = (u[3] - u[0] * u[0] - u[1] * u[1] - u[2] * u[2]) * (1. / L.Dim);
  for (int k = 0; k < 4; k++) c.uT[k] = u[k];
}

// steps.cu:58-75 isConv
// (ga, gr: the gauge's own tolerance, an extension; the reference tests u, T
// with ea, er like the populations)
bool is_conv(const Lattice& L, const Cell& cnew, const Cell& cold, double ea, double er, bool ddf, double ga,
             double gr) {
  for (int k = 0; k < 4; k++)
    if (std::fabs(cnew.uT[k] - cold.uT[k]) >= ga + gr * std::fabs(cnew.uT[k])) return false;
  for (int i = 0; i < L.Q; i++)
    if (std::fabs(cnew.f[i] - cold.f[i]) >= ea + er * std::fabs(cnew.f[i])) return false;
  if (ddf)  // the energy populations converge like the others
    for (int i = 0; i < L.Q; i++)
      if (std::fabs(cnew.h[i] - cold.h[i]) >= ea + er * std::fabs(cnew.h[i])) return false;
  return true;
}

// steps.cu:595-601 LagrPol<N>
double lagr_pol(int N, int ix, int iy, int iz, double sx, double sy, double sz) {
  double a = 1;
  for (int p = 0; p < N; p++) if (p != ix) a *= (sx - p) / double(ix - p);
  for (int p = 0; p < N; p++) if (p != iy) a *= (sy - p) / double(iy - p);
  for (int p = 0; p < N; p++) if (p != iz) a *= (sz - p) / double(iz - p);
  return a;
}
// steps.cu:602-608 LinPol
double lin_pol(int ix, int iy, int iz, double sx, double sy, double sz) {
  double a = 1;
  if (ix == 0) a *= 1 - sx; else if (ix == 1) a *= sx;
  if (iy == 0) a *= 1 - sy; else if (iy == 1) a *= sy;
  if (iz == 0) a *= 1 - sz; else if (iz == 1) a *= sz;
  return a;
}

struct Domain {
  const Lattice* L;
  const double* f;
  const double* h;  // energy populations (nullptr without the double-distribution extension)
  const double* rho;
  const double* g;
  int64_t n[3];
  int64_t N;
  int bc[3];
  const uint8_t* mask = nullptr;  // Cinfo::set per node (nullptr: every node active)
  const double* pos = nullptr;    // Cell::p.x per node under NRMESH (nullptr: p_x = x)
  double inflow[5] = {1, 0, 0, 0, 1};  // ghost state of ORC_BC_INFLOW axes: rho, u, T
  double dof = 0;                      // energy populations of the ghost (double-distribution extension)
};

inline int64_t wrapi(int64_t p, int64_t n) { return ((p % n) + n) % n; }

// Resolve a stencil position to a node and load it.  Periodic is the
// reference's modulo wrap (steps.cu:1015-1017); MIRROR is its disabled
// outflow reflection (steps.cu:1004-1013 with Cell::mirrX/Y/Z,
// structs.cuh:552-578); CLAMP is a zero-gradient extension.
void load_cell(const Domain& D, int64_t px, int64_t py, int64_t pz, Cell& c) {
  int64_t p[3] = {px, py, pz};
  bool rev[3] = {false, false, false};
  for (int a = 0; a < 3; a++) {
    const int64_t n = D.n[a];
    if (D.bc[a] == ORC_BC_INFLOW && p[a] < 0) {  // the inflow ghost: set_base of the inflow state
      set_base(*D.L, c, D.inflow[0], D.inflow + 1);
      if (D.h) set_energy(*D.L, c, D.dof);
      return;
    }
    if (D.bc[a] == ORC_BC_INFLOW) {  // outflow end: zero gradient
      if (p[a] >= n) p[a] = n - 1;
    } else if (D.bc[a] == ORC_BC_MIRROR) {
      if (p[a] < 0) { p[a] = -1 - p[a]; rev[a] = true; }
      if (p[a] >= n) { p[a] = n - 1 - p[a] + n; rev[a] = true; }
      p[a] = wrapi(p[a], n);
    } else if (D.bc[a] == ORC_BC_CLAMP) {
      if (p[a] < 0) p[a] = 0;
      if (p[a] >= n) p[a] = n - 1;
    } else {
      p[a] = wrapi(p[a], n);
    }
  }
  const int64_t idx = p[0] + D.n[0] * (p[1] + D.n[1] * p[2]);
  const Lattice& L = *D.L;
  for (int i = 0; i < L.Q; i++) c.f[i] = D.f[(int64_t)i * D.N + idx];
  if (D.h) for (int i = 0; i < L.Q; i++) c.h[i] = D.h[(int64_t)i * D.N + idx];
  c.rho = D.rho[idx];
  for (int k = 0; k < 4; k++) c.uT[k] = D.g[(int64_t)k * D.N + idx];
  for (int a = 0; a < 3; a++) {
    if (!rev[a]) continue;
    c.uT[a] = -c.uT[a];
    double fn[QMAX];
    for (int i = 0; i < L.Q; i++) fn[i] = (L.e[i][a] == 0) ? c.f[i] : c.f[L.rev[a][i]];
    for (int i = 0; i < L.Q; i++) c.f[i] = fn[i];
    if (D.h) {
      for (int i = 0; i < L.Q; i++) fn[i] = (L.e[i][a] == 0) ? c.h[i] : c.h[L.rev[a][i]];
      for (int i = 0; i < L.Q; i++) c.h[i] = fn[i];
    }
  }
}

// steps.cu:986-1036 propagate<N> (N = 2..5) -- Lagrange interpolation of the
// gauge-transformed stencil at the departure point crd.
double propagate(const Domain& D, int N, const double crd[3], int i, const double* base, bool energy = false) {
  int64_t cl[3];
  if (N % 2 == 0) {
    for (int a = 0; a < 3; a++) cl[a] = (int64_t)(std::floor(crd[a]) - N / 2 + 1);
  } else {  // :997 -- x rounds to nearest, y and z use floor
    cl[0] = (int64_t)(std::floor(crd[0] + 0.5) - (N - 1) / 2);
    cl[1] = (int64_t)(std::floor(crd[1]) - (N - 1) / 2);
    cl[2] = (int64_t)(std::floor(crd[2]) - (N - 1) / 2);
  }
  const double sx = crd[0] - cl[0], sy = crd[1] - cl[1], sz = crd[2] - cl[2];
  double fpr = 0;
  Cell c;
  for (int ix = 0; ix < N; ix++)
    for (int iy = 0; iy < N; iy++)
      for (int iz = 0; iz < N; iz++) {
        const double a = (N == 2) ? lin_pol(ix, iy, iz, sx, sy, sz) : lagr_pol(N, ix, iy, iz, sx, sy, sz);
        // a zero weight contributes +-0 (the transferred value is finite, or
        // NaN for every stencil cell alike), so skipping it is exact
        if (a == 0) continue;
        load_cell(D, cl[0] + ix, cl[1] + iy, cl[2] + iz, c);
        fpr += a * transfer_gauge(*D.L, c, base, i, energy);
      }
  return fpr;
}

// steps.cu:924-937 LagrEval<N> (explicit stencil origin)
double lagr_eval(const Domain& D, int N, const double crd[3], const int64_t cl[3], int i, const double* base,
                 bool energy = false) {
  const double sx = crd[0] - cl[0], sy = crd[1] - cl[1], sz = crd[2] - cl[2];
  double fpr = 0;
  Cell c;
  for (int ix = 0; ix < N; ix++)
    for (int iy = 0; iy < N; iy++)
      for (int iz = 0; iz < N; iz++) {
        const double a = (N == 2) ? lin_pol(ix, iy, iz, sx, sy, sz) : lagr_pol(N, ix, iy, iz, sx, sy, sz);
        if (a == 0) continue;
        load_cell(D, cl[0] + ix, cl[1] + iy, cl[2] + iz, c);
        fpr += a * transfer_gauge(*D.L, c, base, i, energy);
      }
  return fpr;
}

// steps.cu:774-825 propagateWENO<3,5>.  centred: the variant with the
// candidates' y and z windows centred on the departure point (nodes
// floor(c+0.5)-1 .. floor(c+0.5)+1 instead of the reference's floor(c+0.5) ..
// floor(c+0.5)+2, :776-778, which extrapolate) and the smoothness indicators
// read on the row through the departure point (y = floor(crd.y+0.5), z =
// floor(crd.z+0.5)) instead of the reference's y = z = floor(crd.x+0.5)
// (:783), which in 3D lies elsewhere in the domain; on 1D grids both are the
// same.
double propagate_weno5(const Domain& D, const double crd[3], int i, const double* base, bool energy = false,
                       bool centred = false) {
  const double fx = std::floor(crd[0] + 0.5), fy = std::floor(crd[1] + 0.5), fz = std::floor(crd[2] + 0.5);
  const double oy = centred ? fy - 1 : fy, oz = centred ? fz - 1 : fz;
  const int64_t c0[3] = {(int64_t)(fx - 2), (int64_t)oy, (int64_t)oz};
  const int64_t c1[3] = {(int64_t)(fx - 1), (int64_t)oy, (int64_t)oz};
  const int64_t c2[3] = {(int64_t)(fx), (int64_t)oy, (int64_t)oz};
  const double S0 = lagr_eval(D, 3, crd, c0, i, base, energy);
  const double S1 = lagr_eval(D, 3, crd, c1, i, base, energy);
  const double S2 = lagr_eval(D, 3, crd, c2, i, base, energy);
  const double cdist = crd[0] - (int)(std::floor(crd[0] + 0.5));
  const double d0 = (cdist * cdist - 3 * cdist + 2) / 12.;
  const double d2 = (cdist * cdist + 3 * cdist + 2) / 12.;
  const double d1 = 1. - d0 - d2;
  // :783 -- the smoothness row uses y = z = floor(crd.x+0.5) (wrapped)
  const int64_t lx = (int64_t)(fx - 2), ly = (int64_t)(centred ? fy : fx), lz = (int64_t)(centred ? fz : fx);
  double u[6];
  Cell c;
  for (int k = 1; k <= 5; k++) {
    load_cell(D, lx + (k - 1), ly, lz, c);
    u[k] = transfer_gauge(*D.L, c, base, i, energy);
  }
  const double u1 = u[1], u2 = u[2], u3 = u[3], u4 = u[4], u5 = u[5];
  const double beta0 = (10 * u3 * u3 + (11 * u1 - 31 * u2) * u3 + 25 * u2 * u2 - 19 * u1 * u2 + 4 * u1 * u1) / 3.0;
  const double beta1 = (4 * u4 * u4 + (5 * u2 - 13 * u3) * u4 + 13 * u3 * u3 - 13 * u2 * u3 + 4 * u2 * u2) / 3.0;
  const double beta2 = (4 * u5 * u5 + (11 * u3 - 19 * u4) * u5 + 25 * u4 * u4 - 31 * u3 * u4 + 10 * u3 * u3) / 3.0;
  double w0 = d0, w1 = d1, w2 = d2;
  const double sc = 1e-6;
  w0 /= (sc + beta0) * (sc + beta0);
  w1 /= (sc + beta1) * (sc + beta1);
  w2 /= (sc + beta2) * (sc + beta2);
  const double wsum = w0 + w1 + w2;
  w0 /= wsum; w1 /= wsum; w2 /= wsum;
  return w0 * S0 + w1 * S1 + w2 * S2;
}

inline bool node_active(const Domain& D, int64_t idx) { return D.mask == nullptr || D.mask[idx] != 0; }
inline double node_pos(const Domain& D, int64_t idx) { return D.pos ? D.pos[idx] : (double)idx; }

// steps.cu:1122-1149 propagate_nonequal_1D<2>: linear interpolation at crd.x
// between the nearest active nodes left and right of it, each found by
// walking over inactive nodes (periodic), the shifts growing by one per node
// passed.  1D grids (y = z = 0).
double propagate_gap2(const Domain& D, const double crd[3], int i, const double* base, bool energy = false) {
  const int64_t n = D.n[0];
  const double fl = std::floor(crd[0]);
  int64_t posL = wrapi((int64_t)fl, n), posR = wrapi((int64_t)fl + 1, n);
  double shiftL = crd[0] - fl, shiftR = (fl + 1) - crd[0];
  // the walks end at the latest on the (active) node being updated
  for (int64_t k = 0; k < n && !node_active(D, posL); k++) { posL = wrapi(posL - 1, n); shiftL++; }
  for (int64_t k = 0; k < n && !node_active(D, posR); k++) { posR = wrapi(posR + 1, n); shiftR++; }
  Cell cl, cr;
  load_cell(D, posL, 0, 0, cl);
  load_cell(D, posR, 0, 0, cr);
  return shiftR / (shiftL + shiftR) * transfer_gauge(*D.L, cl, base, i, energy) +
         shiftL / (shiftL + shiftR) * transfer_gauge(*D.L, cr, base, i, energy);
}

// steps.cu:590-594 LagrPolNR_1D<N>: Lagrange basis on the abscissae bp[]
double lagr_pol_nr(int N, int ix, double sx, const double* bp) {
  double a = 1;
  for (int ixp = 0; ixp < N; ixp++)
    if (ixp != ix) a *= (sx - bp[ixp]) / (bp[ix] - bp[ixp]);
  return a;
}

// steps.cu:882-908 propagateNR_1D: quadratic Lagrange interpolation at the
// position crd_x on the node positions of x-1, x, x+1 (periodic), abscissae
// relative to the first; a relative coordinate below -Nx/2 (integer
// division) is lifted by Nx.
double propagate_nonuniform3(const Domain& D, int64_t x, double crd_x, int i, const double* base,
                             bool energy = false) {
  const int64_t n = D.n[0];
  const double lift = (double)((-n) / 2);
  const int N = 3;
  Cell c[N];
  double bp[N];
  const int64_t first = wrapi(x - 1, n);
  for (int ix = 0; ix < N; ix++) {
    const int64_t pos = wrapi(x - 1 + ix, n);
    load_cell(D, pos, 0, 0, c[ix]);
    bp[ix] = node_pos(D, pos) - node_pos(D, first);
    if (bp[ix] < lift) bp[ix] += n;
  }
  double shift = crd_x - node_pos(D, first);
  if (shift < lift) shift += n;
  double fpr = 0;
  for (int ix = 0; ix < N; ix++) fpr += lagr_pol_nr(N, ix, shift, bp) * transfer_gauge(*D.L, c[ix], base, i, energy);
  return fpr;
}

// steps.cu:113-117 minmod
double minmod(double a, double b) {
  if (a * b <= 0) return 0;
  if (std::fabs(a) < std::fabs(b)) return a;
  return b;
}

// steps.cu:447 with FluxTVDdif (:118-124): plain cubic value at x-v plus a
// minmod-limited flux-difference correction
double propagate_tvd(const Domain& D, const double coord[3], const double v[3], int i, const double* base,
                     bool energy = false) {
  double cM2[3], cM1[3], cC[3], cP1[3];
  for (int a = 0; a < 3; a++) {
    cM2[a] = coord[a] - v[a] * 2;
    cM1[a] = coord[a] - v[a] * 1;
    cC[a] = coord[a] + v[a] * 0;
    cP1[a] = coord[a] + v[a] * 1;
  }
  const double Fm1 = propagate(D, 4, cM1, i, base, energy);
  const double Fm2 = propagate(D, 4, cM2, i, base, energy);
  const double F0 = propagate(D, 4, cC, i, base, energy);
  const double Fp1 = propagate(D, 4, cP1, i, base, energy);
  const int sg = sign_i(v[0]);
  const double flux = F0 - Fm1 + sg * 0.5 * minmod(F0 - Fm1, Fp1 - F0) - sg * 0.5 * minmod(F0 - Fm1, Fm1 - Fm2);
  const double fc = propagate(D, 4, coord, i, base, energy);
  return fc - flux;
}

// steps.cu:356-588 LBMpull (and :151-250 PonDstepD3Q125 for FIXED3): the
// fixed-point gauge iteration, BGK relaxation and store for one node.
//
// With the double-distribution extension (D.h set), the energy populations h
// are transferred and interpolated exactly as f, the temperature of each
// iterate comes from their sum, T = (sum h / rho - |u|^2) / (Dim + dof), the
// convergence test covers them too, and they relax to the equilibrium of
// set_energy.  The model's heat-capacity ratio is (Dim + dof + 2)/(Dim + dof).
int pull_node(const Domain& D, const orc_params& P, int64_t x, int64_t y, int64_t z,
              const double* guess, double* f_out, double* h_out, double* rho_out, double* g_out, int* niter_out) {
  const Lattice& L = *D.L;
  const bool ddf = D.h != nullptr;
  const double dof = P.dof;
  const int64_t idx = x + D.n[0] * (y + D.n[1] * z);
  Cell c0, cnew;
  load_cell(D, x, y, z, c0);
  if (!node_active(D, idx)) {  // steps.cu:359: the step skips it; here it is carried over unchanged
    for (int i = 0; i < L.Q; i++) f_out[(int64_t)i * D.N + idx] = c0.f[i];
    rho_out[idx] = c0.rho;
    for (int k = 0; k < 4; k++) g_out[(int64_t)k * D.N + idx] = c0.uT[k];
    if (niter_out) niter_out[idx] = 0;
    return 0;
  }
  if (c0.rho == 0 && c0.uT[0] == 0 && c0.uT[1] == 0 && c0.uT[2] == 0 && c0.uT[3] == 0) {
    const double b[4] = {0, 0, 0, L.TLat};
    set_base(L, c0, 1, b);
    if (ddf) set_energy(L, c0, dof);
  }
  if (guess) for (int k = 0; k < 4; k++) c0.uT[k] = guess[(int64_t)k * D.N + idx];
  const double coord[3] = {(double)x, (double)y, (double)z};
  std::vector<Cell> cfix;
  if (P.interp == ORC_FIXED3) {  // stencil staged once (steps.cu:164-193)
    cfix.resize(27);
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) load_cell(D, x - 1 + a, y - 1 + b, z - 1 + c, cfix[9 * a + 3 * b + c]);
  }
  int Niter = 0;
  bool conv = false;
  double vi[QMAX][3];
  while (Niter < P.max_iter) {
    Niter++;
    const double uT[4] = {c0.uT[0], c0.uT[1], c0.uT[2], c0.uT[3]};
    const double s = std::sqrt(uT[3] / L.TLat);
    for (int i = 0; i < L.Q; i++)
      for (int a = 0; a < 3; a++) vi[i][a] = s * L.xi[i][a] + uT[a];
    for (int i = 0; i < L.Q; i++) {
      double crd[3];
      for (int a = 0; a < 3; a++) crd[a] = coord[a] - vi[i][a];
      double val = 0;
      switch (P.interp) {
        case ORC_FIXED3: {
          for (int e = 0; e < (ddf ? 2 : 1); e++) {
            double newval[27];
            for (int k = 0; k < 27; k++) newval[k] = transfer_gauge(L, cfix[k], uT, i, e == 1);
            const double sx = crd[0] - (x - 1), sy = crd[1] - (y - 1), sz = crd[2] - (z - 1);
            double fpr = 0;
            for (int a = 0; a < 3; a++)
              for (int b = 0; b < 3; b++)
                for (int c = 0; c < 3; c++) fpr += lagr_pol(3, a, b, c, sx, sy, sz) * newval[9 * a + 3 * b + c];
            if (e == 0) val = fpr; else cnew.h[i] = fpr;
          }
          break;
        }
        case ORC_TVD:
          val = propagate_tvd(D, coord, vi[i], i, uT);
          if (ddf) cnew.h[i] = propagate_tvd(D, coord, vi[i], i, uT, true);
          break;
        case ORC_WENO5:
        case ORC_WENO5_ROW: {
          const bool fix = P.interp == ORC_WENO5_ROW;
          val = propagate_weno5(D, crd, i, uT, false, fix);
          if (ddf) cnew.h[i] = propagate_weno5(D, crd, i, uT, true, fix);
          break;
        }
        case ORC_GAP2:  // call site steps.cu:449
          val = propagate_gap2(D, crd, i, uT);
          break;
        case ORC_NONUNIFORM3:  // call site steps.cu:453: departure point c0_st.p - v_i
          val = propagate_nonuniform3(D, x, node_pos(D, idx) - vi[i][0], i, uT);
          break;
        default:
          val = propagate(D, P.interp, crd, i, uT);
          if (ddf) cnew.h[i] = propagate(D, P.interp, crd, i, uT, true);
          break;
      }
      cnew.f[i] = val;
    }
    calc_moments(L, cnew, vi);
    if (ddf) {  // the temperature of the iterate from its energy populations
      double e = 0;
      for (int i = 0; i < L.Q; i++) e += cnew.h[i];
      if (cnew.rho != 0) e /= cnew.rho;
      cnew.uT[3] = (e - cnew.uT[0] * cnew.uT[0] - cnew.uT[1] * cnew.uT[1] - cnew.uT[2] * cnew.uT[2]) / (L.Dim + dof);
    }
    if (cnew.uT[3] < 0) cnew.uT[3] = c0.uT[3];  // steps.cu:475-478
    const bool gsep = P.tolg[0] >= 0 && P.tolg[1] >= 0;
    if (is_conv(L, cnew, c0, P.tol_abs, P.tol_rel, ddf, gsep ? P.tolg[0] : P.tol_abs, gsep ? P.tolg[1] : P.tol_rel)) {
      c0 = cnew;
      conv = true;
      break;
    }
    c0 = cnew;
  }
  const double dtau = 1.0 / P.tau;
  for (int i = 0; i < L.Q; i++) {  // steps.cu:557-564
    const double feq = c0.rho * L.w[i];
    c0.f[i] += dtau * (feq - c0.f[i]);
  }
  if (ddf) {
    Cell eq = c0;
    set_energy(L, eq, dof);
    for (int i = 0; i < L.Q; i++) {
      c0.h[i] += dtau * (eq.h[i] - c0.h[i]);
      h_out[(int64_t)i * D.N + idx] = c0.h[i];
    }
  }
  for (int i = 0; i < L.Q; i++) f_out[(int64_t)i * D.N + idx] = c0.f[i];
  rho_out[idx] = c0.rho;
  for (int k = 0; k < 4; k++) g_out[(int64_t)k * D.N + idx] = c0.uT[k];
  if (niter_out) niter_out[idx] = Niter;
  return conv ? 0 : 1;
}

}  // namespace

extern "C" {

int orc_q(int lattice_kind) { return lattice(lattice_kind).Q; }

int orc_tables(int lattice_kind, double* xi, int* e, double* w, double* tlat_dim) {
  const Lattice& L = lattice(lattice_kind);
  if (L.Q == 0) return -1;
  for (int i = 0; i < L.Q; i++) {
    for (int a = 0; a < 3; a++) {
      if (xi) xi[3 * i + a] = L.xi[i][a];
      if (e) e[3 * i + a] = L.e[i][a];
    }
    if (w) w[i] = L.w[i];
  }
  if (tlat_dim) { tlat_dim[0] = L.TLat; tlat_dim[1] = L.Dim; }
  return L.Q;
}

int orc_reverse(int lattice_kind, int* rx, int* ry, int* rz) {
  const Lattice& L = lattice(lattice_kind);
  if (L.Q == 0) return -1;
  for (int i = 0; i < L.Q; i++) { rx[i] = L.rev[0][i]; ry[i] = L.rev[1][i]; rz[i] = L.rev[2][i]; }
  return L.Q;
}

void orc_set_base(int lattice_kind, double rho, const double* uT, double* f) {
  const Lattice& L = lattice(lattice_kind);
  Cell c;
  set_base(L, c, rho, uT);
  for (int i = 0; i < L.Q; i++) f[i] = c.f[i];
}

double orc_transfer_gauge(int lattice_kind, const double* f, const double* uT_src, const double* uT_dst, int inew) {
  const Lattice& L = lattice(lattice_kind);
  Cell c;
  for (int i = 0; i < L.Q; i++) c.f[i] = f[i];
  c.rho = 0;
  for (int k = 0; k < 4; k++) c.uT[k] = uT_src[k];
  return transfer_gauge(L, c, uT_dst, inew);
}

void orc_calc_moments(int lattice_kind, const double* f, const double* vi, double* rho, double* uT) {
  const Lattice& L = lattice(lattice_kind);
  Cell c;
  double v[QMAX][3];
  for (int i = 0; i < L.Q; i++) {
    c.f[i] = f[i];
    for (int a = 0; a < 3; a++) v[i][a] = vi[3 * i + a];
  }
  calc_moments(L, c, v);
  *rho = c.rho;
  for (int k = 0; k < 4; k++) uT[k] = c.uT[k];
}

double orc_lagr_pol(int n, int ix, int iy, int iz, double sx, double sy, double sz) {
  return n == 2 ? lin_pol(ix, iy, iz, sx, sy, sz) : lagr_pol(n, ix, iy, iz, sx, sy, sz);
}

void orc_set_energy(int lattice_kind, double rho, const double* uT, double dof, double* h) {
  const Lattice& L = lattice(lattice_kind);
  Cell c;
  c.rho = rho;
  for (int k = 0; k < 4; k++) c.uT[k] = uT[k];
  set_energy(L, c, dof);
  for (int i = 0; i < L.Q; i++) h[i] = c.h[i];
}

int64_t orc_step(const orc_params* p, const double* f_in, const double* rho_in, const double* g_in,
                 const double* guess, double* f_out, double* rho_out, double* g_out, int* niter) {
  return orc_step_ddf(p, f_in, nullptr, rho_in, g_in, guess, f_out, nullptr, rho_out, g_out, niter);
}

int64_t orc_step_ddf(const orc_params* p, const double* f_in, const double* h_in, const double* rho_in,
                     const double* g_in, const double* guess, double* f_out, double* h_out, double* rho_out,
                     double* g_out, int* niter) {
  const Lattice& L = lattice(p->lattice);
  if (L.Q == 0 || p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->max_iter <= 0) return -1;
  if ((h_in == nullptr) != (h_out == nullptr) || (h_in && !(p->dof >= 0))) return -1;
  Domain D;
  D.L = &L;
  D.f = f_in; D.h = h_in; D.rho = rho_in; D.g = g_in;
  D.n[0] = p->nx; D.n[1] = p->ny; D.n[2] = p->nz;
  D.N = p->nx * p->ny * p->nz;
  for (int a = 0; a < 3; a++) D.bc[a] = p->bc[a];
  for (int k = 0; k < 5; k++) D.inflow[k] = p->inflow[k];
  D.dof = p->dof;
  const orc_params P = *p;
  int64_t nonconv = 0;
  const int64_t N = D.N;
#ifdef _OPENMP
  const int nth = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : nonconv) num_threads(nth)
#endif
  for (int64_t n = 0; n < N; n++) {
    const int64_t x = n % p->nx, y = (n / p->nx) % p->ny, z = n / (p->nx * p->ny);
    nonconv += pull_node(D, P, x, y, z, guess, f_out, h_out, rho_out, g_out, niter);
  }
  return nonconv;
}

int64_t orc_step_mesh(const orc_params* p, const double* f_in, const double* rho_in, const double* g_in,
                      const uint8_t* mask, const double* pos, double* f_out, double* rho_out, double* g_out,
                      int* niter) {
  const Lattice& L = lattice(p->lattice);
  if (L.Q == 0 || p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->max_iter <= 0) return -1;
  const bool mesh_scheme = p->interp == ORC_GAP2 || p->interp == ORC_NONUNIFORM3;
  if (mesh_scheme && (p->lattice != ORC_D1Q5 || p->ny != 1 || p->nz != 1 || p->bc[0] != ORC_BC_PERIODIC)) return -1;
  Domain D;
  D.L = &L;
  D.f = f_in; D.h = nullptr; D.rho = rho_in; D.g = g_in;
  D.n[0] = p->nx; D.n[1] = p->ny; D.n[2] = p->nz;
  D.N = p->nx * p->ny * p->nz;
  for (int a = 0; a < 3; a++) D.bc[a] = p->bc[a];
  D.mask = mask;
  D.pos = pos;
  const orc_params P = *p;
  int64_t nonconv = 0;
  const int64_t N = D.N;
#ifdef _OPENMP
  const int nth = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : nonconv) num_threads(nth)
#endif
  for (int64_t n = 0; n < N; n++) {
    const int64_t x = n % p->nx, y = (n / p->nx) % p->ny, z = n / (p->nx * p->ny);
    nonconv += pull_node(D, P, x, y, z, nullptr, f_out, nullptr, rho_out, g_out, niter);
  }
  return nonconv;
}

int64_t orc_amr_refine(const orc_params* p, double* f, double* rho, double* g, uint8_t* mask, double tol,
                       int64_t* limit_hits) {
  const Lattice& L = lattice(p->lattice);
  if (L.Q == 0 || p->ny != 1 || p->nz != 1 || p->nx <= 0 || !mask) return -1;
  const int64_t nx = p->nx, N = nx;
  const std::vector<uint8_t> set(mask, mask + nx);  // cinfo_setnew_reset: decisions read the old mask
  int64_t added = 0, limits = 0;
  for (int64_t x = 0; x < nx; x++) {
    if (!set[x]) continue;
    int64_t xp = x, dist = 0;
    do {  // amr.cu:8-12
      xp = (xp + 1) % nx;
      dist++;
    } while (!set[xp]);
    const double vdif = g[xp] - g[x];
    const int64_t mid = (x + dist / 2) % nx;
    if (vdif * vdif / std::fmin(g[3 * N + x], g[3 * N + xp]) > tol || std::fabs(1 - rho[x] / rho[xp]) > tol) {
      if (dist <= 1) limits++;
      if (dist % 2 == 0) {  // amr.cu:18-25: the record average, saved to both time levels
        rho[mid] = 0.5 * (rho[x] + rho[xp]);
        for (int k = 0; k < 4; k++) g[k * N + mid] = 0.5 * (g[k * N + x] + g[k * N + xp]);
        for (int i = 0; i < L.Q; i++) f[i * N + mid] = 0.5 * (f[i * N + x] + f[i * N + xp]);
        if (!mask[mid]) added++;
        mask[mid] = 1;
      }
    }
  }
  if (limit_hits) *limit_hits = limits;
  return added;
}

int64_t orc_amr_coarsen(const orc_params* p, const double* rho, const double* g, uint8_t* mask, double tol) {
  if (p->ny != 1 || p->nz != 1 || p->nx <= 0 || !mask) return -1;
  const int64_t nx = p->nx, N = nx;
  int64_t removed = 0;
  for (int64_t ix = 0; ix < nx; ix++) {  // amr.cu:29-54, in node order, on the mask as it changes
    if (!mask[ix]) continue;
    int64_t xm = ix, xp = ix, distM = 0, distP = 0;
    do { xm = (xm - 1 + nx) % nx; distM++; } while (!mask[xm]);
    do { xp = (xp + 1) % nx; distP++; } while (!mask[xp]);
    const double T0 = g[3 * N + ix];
    const double vdifm = g[xm] - g[ix];
    const double vdifp = g[xp] - g[ix];
    if (vdifm * vdifm / T0 < tol && vdifp * vdifp / T0 < tol && std::fabs(rho[xp] / rho[ix] - 1) < tol &&
        std::fabs(rho[xm] / rho[ix] - 1) < tol && (distM < 4 && distP < 4)) {
      mask[ix] = 0;
      removed++;
    }
  }
  return removed;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
