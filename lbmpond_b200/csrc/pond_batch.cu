// Batched 1D PonD: thousands of independent D1Q5 problems of uneven length
// advanced by persistent kernel launches replayed from a CUDA graph.
//
// Layout.  At creation the problems are packed (best fit, longest first)
// into bins of at most BIN_CAP = 6144 nodes and BIN_SEGS problems; the
// device state is stored bin after bin, SoA: f[5][S], rho, u, T (float32),
// every bin starting on a 4-node (16-byte) boundary, S the padded total.
// Host set/get calls translate to and from the caller's problem order.
//
// Kernel.  Each CTA takes bins from a queue, holds one bin in shared memory
// (populations, u, T, c = sqrt(T): 8 planes, 196 KB; rho is the sum of the
// populations) and advances it K steps
// before taking the next.  A step computes every node of the bin from the
// shared copy and writes the new level to the bin's global arrays (L2
// resident); after a barrier the shared copy is restaged.  Staging is seven
// bulk copies (cp.async.bulk, the TMA engine) issued by one thread and
// completed on an mbarrier whose wait is bounded.  The per-node step
// is LBMpull (steps.cu:356-588) on D1Q5 with WENO5 (propagateWENO<3,5>,
// steps.cu:774-825) or cubic Lagrange (propagate<4>, steps.cu:986):
// float32 populations, transforms and interpolation, float64 moments
// (structs.cuh:315-342), T < 0 guard (steps.cu:475) and convergence test
// (isConv, steps.cu:58-75).  Each population reads only its own 5 (or 4)
// window nodes, so the work per iteration does not grow with the sound
// speed.  Stencil coordinates are clamped at each problem's ends
// (zero-gradient boundaries).
//
// Two phases per step.  Iteration counts are very uneven: most nodes
// converge in 1-3 iterations, a few on each jump run to max_iter.  Phase 1
// gives every lane one node at a time (a lane whose node is done takes the
// next unclaimed node) and stops a node after `lane_cap` iterations,
// parking it in a shared-memory list.  Phase 2 gives each parked node a
// whole warp: lane 5k+m evaluates window node m of population k, so one
// iteration takes about the latency of one transfer row instead of 25.  The
// arithmetic of an iteration is the same in both phases.
//
// Training pairs: every `every` steps, nodes at local coordinate
// x % stride == 0 write their pre-step 7-node (rho, u, T) stencil and the
// converged (u, T) of that step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <set>
#include <utility>
#include <vector>

#include "pond_internal.h"

namespace pond {
namespace batch {

constexpr int BIN_CAP = 6144;  // nodes per bin (problems are at most MAX_LEN)
constexpr int MAX_LEN = 4096;
constexpr int BIN_SEGS = 64;
constexpr int HARD_MAX = 192;  // parked nodes per bin and step
constexpr int NPAIR_IN = 21;   // rho, u, T at x-3 .. x+3
constexpr int NPAIR_OUT = 2;   // converged u, T
constexpr size_t SMEM = size_t(8) * BIN_CAP * sizeof(float);  // f x5, u, T, c

struct Args {
  float* f;    // [5][stride], bin order
  float* rho;  // [stride]
  float* u;
  float* T;
  long long stride;          // plane length: the node count with every bin start padded to 4 nodes
  const long long* bin_off;  // [B+1] first node of each bin (a multiple of 4)
  const int* seg_first;      // [B+1] into segs
  const int* segs;           // per bin: local problem starts, then the fill
  int B;
  int* queue;
  const int* istep;  // device step counter (pair sampling)
  int nsteps;
  float dtau;
  double tol_abs, tol_rel;
  int max_iter;
  int lane_cap;  // phase-1 iterations before a node is parked
  unsigned long long* stats;  // niter_sum, nonconv, niter_max (as int)
  float* px;
  float* py;
  unsigned long long* pcount;
  long long pcap;
  int pair_every, pair_stride;
  int* err;  // set when a staging copy did not complete in time
};

// One node's iteration state.
struct Node {
  double rho0, U, T;
  float f0[5];
  int x, niter;
};

__device__ __forceinline__ float finite_or_zero(float v) { return fabsf(v) <= 3.402823466e38f ? v : 0.f; }

// Row k of the 5-point Lagrange basis on the normalised speeds
// {0, +EC1, -EC1, +EC2, -EC2} at y (the transfer_gauge matrix entry,
// structs.cuh:343-551, for D1Q5):
//   L_k(y) = D_k (y^2 - P_k)(y^2 + s_k y - Q_k).
__device__ __forceinline__ float basis5_row(int k, float y) {
  constexpr double e1s = EC1 * EC1, e2s = EC2 * EC2;
  const float D = k == 0 ? float(1.0 / (e1s * e2s))
                         : (k <= 2 ? float(1.0 / (2.0 * e1s * (e1s - e2s))) : float(1.0 / (2.0 * e2s * (e2s - e1s))));
  const float P = (k == 1 || k == 2) ? float(e2s) : float(e1s);
  const float S = k == 1 ? float(EC1) : k == 2 ? -float(EC1) : k == 3 ? float(EC2) : k == 4 ? -float(EC2) : 0.f;
  const float Q = k == 0 ? float(e2s) : 0.f;
  const float y2 = y * y;
  return D * (y2 - P) * (fmaf(S, y, y2) - Q);
}

// Population k of the guessed gauge (U, 1/C) at shared-memory node q: the
// gauge transform of node q's five populations, non-finite terms dropped
// (steps.cu:390).
__device__ __forceinline__ float transfer_row(int k, const float* sf, const float* su, const float* sc, int q,
                                              float Uf, float invC) {
  const float s = (su[q] - Uf) * invC, r = sc[q] * invC;
  float g = 0.f;
  if (fabsf(s) < 1e8f && fabsf(r) < 1e8f) {  // every |y| < 3e8: each basis value is finite
#pragma unroll
    for (int b = 0; b < 5; b++)
      g = fmaf(basis5_row(k, fmaf(r, float(Lattice<POND_D1Q5>::xi1(b)), s)), sf[b * BIN_CAP + q], g);
  } else {
#pragma unroll
    for (int b = 0; b < 5; b++)
      g = fmaf(finite_or_zero(basis5_row(k, fmaf(r, float(Lattice<POND_D1Q5>::xi1(b)), s))), sf[b * BIN_CAP + q], g);
  }
  return g;
}

// WENO5 smoothness indicators in Jiang-Shu difference form: algebraically
// the quadratic forms of steps.cu:803-805, without their cancellation in
// float32.
__device__ __forceinline__ float beta_js(float a, float b, float c, float d1, float d2, float d3) {
  const float s = a - 2.f * b + c;
  const float t = d1 * a + d2 * b + d3 * c;
  return (13.f / 12.f) * s * s + 0.25f * t * t;
}

// propagateWENO<3,5> (steps.cu:774-825) on the five transformed window
// values w (nodes fx-2 .. fx+2) at offset d = crd - fx in [-0.5, 0.5).
__device__ __forceinline__ float weno5(const float w[5], float d) {
  float S[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const float t = d + float(2 - j);  // crd - (fx - 2 + j)
    const float l0 = 0.5f * (t - 1.f) * (t - 2.f), l1 = -t * (t - 2.f), l2 = 0.5f * t * (t - 1.f);
    S[j] = l0 * w[j] + l1 * w[j + 1] + l2 * w[j + 2];
  }
  const float d0 = (d * d - 3.f * d + 2.f) * (1.f / 12.f), d2 = (d * d + 3.f * d + 2.f) * (1.f / 12.f);
  const float d1 = 1.f - d0 - d2;
  const float b0 = beta_js(w[0], w[1], w[2], 1.f, -4.f, 3.f);
  const float b1 = beta_js(w[1], w[2], w[3], 1.f, 0.f, -1.f);
  const float b2 = beta_js(w[2], w[3], w[4], 3.f, -4.f, 1.f);
  // the nonlinear weights only scale the candidates: 2-ulp divisions
  const float a0 = __fdividef(d0, (1e-6f + b0) * (1e-6f + b0));
  const float a1 = __fdividef(d1, (1e-6f + b1) * (1e-6f + b1));
  const float a2 = __fdividef(d2, (1e-6f + b2) * (1e-6f + b2));
  return __fdividef(a0 * S[0] + a1 * S[1] + a2 * S[2], a0 + a1 + a2);
}

// cubic Lagrange weights (propagate<4>) at offset t in [1, 2) from the first
// of the four window nodes
__device__ __forceinline__ void lagr4(float t, float l[4]) {
  l[0] = -(t - 1.f) * (t - 2.f) * (t - 3.f) * (1.f / 6.f);
  l[1] = t * (t - 2.f) * (t - 3.f) * 0.5f;
  l[2] = -t * (t - 1.f) * (t - 3.f) * 0.5f;
  l[3] = t * (t - 1.f) * (t - 2.f) * (1.f / 6.f);
}

// Window of population k: first node o (before clamping) and the offset
// of the departure point crd = xl - v_k inside it.
template <int SCHEME> __device__ __forceinline__ int window(double crd, float& off) {
  if (SCHEME == POND_WENO5) {
    const double fx = floor(crd + 0.5);
    off = float(crd - fx);
    return int(fx) - 2;
  }
  const double fl = floor(crd);
  off = float(crd - fl) + 1.f;
  return int(fl) - 1;
}

// New value of population k, one lane (phase 1).
template <int SCHEME>
__device__ __forceinline__ float pull_population(int k, const float* sf, const float* su, const float* sc, int ps,
                                                 int n, int xl, double vK, float Uf, float invC) {
  float off;
  const int o = window<SCHEME>(double(xl) - vK, off);
  if (SCHEME == POND_WENO5) {
    float w[5];
#pragma unroll
    for (int m = 0; m < 5; m++) w[m] = transfer_row(k, sf, su, sc, ps + min(max(o + m, 0), n - 1), Uf, invC);
    return weno5(w, off);
  }
  float l[4];
  lagr4(off, l);
  float g = 0.f;
#pragma unroll
  for (int m = 0; m < 4; m++) g = fmaf(l[m], transfer_row(k, sf, su, sc, ps + min(max(o + m, 0), n - 1), Uf, invC), g);
  return g;
}

// cnew.calcMoments (float64), the T < 0 guard and isConv; then c0 = cnew.
// Returns true when the iteration has converged.
__device__ __forceinline__ bool moments_and_test(const Args& a, const float fn[5], const double vk[5], Node& s) {
  double rho = 0, m1 = 0, m2 = 0;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const double fv = fn[k];
    rho += fv; m1 += fv * vk[k]; m2 += fv * vk[k] * vk[k];
  }
  if (rho != 0) {
    const double ir = 1.0 / rho;
    m1 *= ir;
    m2 *= ir;
  }
  double Tn = m2 - m1 * m1;
  if (Tn < 0) Tn = s.T;
  bool ok = !(fabs(m1 - s.U) >= a.tol_abs + a.tol_rel * fabs(m1)) &&
            !(fabs(Tn - s.T) >= a.tol_abs + a.tol_rel * fabs(Tn));
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const double nv = fn[k], ov = s.f0[k];
    ok = ok && !(fabs(nv - ov) >= a.tol_abs + a.tol_rel * fabs(nv));
    s.f0[k] = fn[k];
  }
  s.rho0 = rho; s.U = m1; s.T = Tn;
  return ok;
}

// The problem holding bin node x: s_seg[j] <= x < s_seg[j + 1].
__device__ __forceinline__ void locate(const int* s_seg, int nseg, int x, int& ps, int& n) {
  int lo = 0, hi = nseg;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s_seg[mid] <= x) lo = mid; else hi = mid;
  }
  ps = s_seg[lo];
  n = s_seg[lo + 1] - ps;
}

// rho of staged node q: the sum of its populations (the stored rho is that
// sum after the collision, which conserves it; shared memory holds f, u, T, c)
__device__ __forceinline__ float rho_of(const float* sf, int q) {
  float r = sf[q];
#pragma unroll
  for (int k = 1; k < 5; k++) r += sf[k * BIN_CAP + q];
  return r;
}

// c0.load of bin node x from the shared copy (steps.cu:360-363), with
// set_base(1, TLat) for an empty record.
__device__ __forceinline__ void load_node(const float* sf, const float* su, const float* sT, int x, Node& s) {
#pragma unroll
  for (int k = 0; k < 5; k++) s.f0[k] = sf[k * BIN_CAP + x];
  s.rho0 = rho_of(sf, x); s.U = su[x]; s.T = sT[x];
  if (s.rho0 == 0 && s.U == 0 && s.T == 0) {
    s.rho0 = 1; s.T = Lattice<POND_D1Q5>::TLat;
#pragma unroll
    for (int k = 0; k < 5; k++) s.f0[k] = float(lattice_weight_t<POND_D1Q5>(k));
  }
  s.x = x;
  s.niter = 0;
}

// BGK toward rho w_i in the co-moving gauge (steps.cu:557-564), the new
// level to global memory and the node's training pair.
__device__ __forceinline__ void finish_node(const Args& a, Node& s, long long off, int ps, int n, bool sample,
                                            const float* sf, const float* su, const float* sT) {
  const float rr = float(s.rho0);
  const long long g = off + s.x;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const float fk = s.f0[k] + a.dtau * (rr * float(lattice_weight_t<POND_D1Q5>(k)) - s.f0[k]);
    a.f[k * a.stride + g] = fk;
  }
  a.rho[g] = rr;
  a.u[g] = float(s.U);
  a.T[g] = float(s.T);
  const int xl = s.x - ps;
  if (sample && (xl % a.pair_stride) == 0) {
    const unsigned long long slot = atomicAdd(a.pcount, 1ull);
    if ((long long)slot < a.pcap) {
      float* X = a.px + slot * NPAIR_IN;
#pragma unroll
      for (int o = -3; o <= 3; o++) {
        const int q = ps + min(max(xl + o, 0), n - 1);
        X[o + 3] = rho_of(sf, q);
        X[7 + o + 3] = su[q];
        X[14 + o + 3] = sT[q];
      }
      a.py[slot * NPAIR_OUT + 0] = float(s.U);
      a.py[slot * NPAIR_OUT + 1] = float(s.T);
    }
  }
}

// ---- bin staging with the bulk-copy (TMA) engine: thread 0 posts the byte
// count on an mbarrier and issues one cp.async.bulk per plane; every thread
// waits on the barrier's phase.  Plane segments start 16-byte aligned (bin
// starts and the plane stride are multiples of 4 nodes).
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// true once the barrier has completed the phase with this parity (bounded poll)
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (int spin = 0; spin < (1 << 22); spin++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <int SCHEME, int NT>
__global__ void __launch_bounds__(NT, 1) batch_kernel(Args a) {
  using L = Lattice<POND_D1Q5>;
  constexpr int GROUP = SCHEME == POND_WENO5 ? 5 : 4;  // lanes per population in phase 2
  extern __shared__ __align__(16) float sm[];
  float* sf = sm;                // [5][BIN_CAP]
  float* su = sm + 5 * BIN_CAP;  // u
  float* sT = sm + 6 * BIN_CAP;  // T
  float* sc = sm + 7 * BIN_CAP;  // c = sqrts(T / TLat)
  __shared__ int s_seg[BIN_SEGS + 1];
  __shared__ Node s_hard[HARD_MAX];
  __shared__ int s_bin, s_next, s_nhard, s_hnext;
  __shared__ __align__(8) unsigned long long s_bar;
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) mbar_init(&s_bar);
  __syncthreads();
  unsigned phase = 0;
  const int step0 = *a.istep;
  unsigned long long it_sum = 0, nc = 0;
  int it_max = 0;
  for (;;) {
    if (tid == 0) s_bin = atomicAdd(a.queue, 1);
    __syncthreads();
    const int bin = s_bin;
    if (bin >= a.B) break;
    const long long off = a.bin_off[bin];
    const int sf0 = a.seg_first[bin];
    const int nseg = a.seg_first[bin + 1] - sf0 - 1;
    const int fill = a.segs[sf0 + nseg];
    for (int i = tid; i <= nseg; i += NT) s_seg[i] = a.segs[sf0 + i];
    for (int step = 0; step < a.nsteps; step++) {
      // stage the bin's current level (first from HBM, then from L2) by bulk copies
      if (tid == 0) {  // bins are never empty; fill <= BIN_CAP, a multiple of 4
        const unsigned bytes = unsigned((fill + 3) & ~3) * sizeof(float);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier generic use of the buffer
        mbar_expect(&s_bar, 7 * bytes);
#pragma unroll
        for (int k = 0; k < 5; k++) bulk_g2s(sf + k * BIN_CAP, a.f + k * a.stride + off, bytes, &s_bar);
        bulk_g2s(su, a.u + off, bytes, &s_bar);
        bulk_g2s(sT, a.T + off, bytes, &s_bar);
      }
      const bool staged = mbar_wait(&s_bar, phase & 1u);
      phase++;
      if (__syncthreads_or(!staged)) {  // a copy did not land: report, give it one more bounded wait, leave
        if (tid == 0) {
          atomicExch(a.err, 1);
          mbar_wait(&s_bar, (phase - 1) & 1u);
        }
        return;
      }
      for (int i = tid; i < fill; i += NT) {
#pragma unroll
        for (int k = 0; k < 5; k++) sf[k * BIN_CAP + i] = finite_or_zero(sf[k * BIN_CAP + i]);
        const float T = sT[i];
        sc[i] = copysignf(sqrtf(fabsf(T) * float(1.0 / L::TLat)), T);
      }
      if (tid == 0) { s_next = NT; s_nhard = 0; s_hnext = 0; }
      __syncthreads();
      const bool sample = a.px && ((step0 + step) % a.pair_every) == 0;
      // phase 1: one lane per node
      Node s;
      int ps = 0, n = 1;
      if (tid < fill) {
        load_node(sf, su, sT, tid, s);
        locate(s_seg, nseg, tid, ps, n);
      } else {
        s.x = fill;
      }
      while (s.x < fill) {
        s.niter++;
        const double C = sqrt(s.T / L::TLat);
        const float Uf = float(s.U), invC = __frcp_rn(float(C));
        double vk[5];
        float fn[5];
#pragma unroll
        for (int k = 0; k < 5; k++) vk[k] = C * L::xi1(k) + s.U;
#pragma unroll
        for (int k = 0; k < 5; k++) fn[k] = pull_population<SCHEME>(k, sf, su, sc, ps, n, s.x - ps, vk[k], Uf, invC);
        const bool ok = moments_and_test(a, fn, vk, s);
        if (!ok && s.niter < a.max_iter) {
          if (s.niter != a.lane_cap) continue;
          const int slot = atomicAdd(&s_nhard, 1);
          if (slot >= HARD_MAX) continue;  // list full: keep iterating here
          s_hard[slot] = s;
        } else {
          it_sum += s.niter;
          nc += ok ? 0 : 1;
          it_max = max(it_max, s.niter);
          finish_node(a, s, off, ps, n, sample, sf, su, sT);
        }
        const int x = atomicAdd(&s_next, 1);
        if (x < fill) {
          load_node(sf, su, sT, x, s);
          locate(s_seg, nseg, x, ps, n);
        } else {
          s.x = fill;
        }
      }
      __syncthreads();
      // phase 2: one warp per parked node
      const int nh = min(s_nhard, HARD_MAX);
      for (;;) {
        int h = 0;
        if (lane == 0) h = atomicAdd(&s_hnext, 1);
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h >= nh) break;
        Node w = s_hard[h];
        locate(s_seg, nseg, w.x, ps, n);
        const int xl = w.x - ps;
        const int k = min(lane / GROUP, 4), m = lane - k * GROUP;  // lanes past 5*GROUP repeat group 4
        bool ok = false;
        while (w.niter < a.max_iter) {
          w.niter++;
          const double C = sqrt(w.T / L::TLat);
          const float Uf = float(w.U), invC = __frcp_rn(float(C));
          double vk[5];
#pragma unroll
          for (int j = 0; j < 5; j++) vk[j] = C * L::xi1(j) + w.U;
          float offk;
          const int o = window<SCHEME>(double(xl) - (C * L::xi1(k) + w.U), offk);  // vk[k] without a dynamic index
          const float t = transfer_row(k, sf, su, sc, ps + min(max(o + min(m, GROUP - 1), 0), n - 1), Uf, invC);
          float g[GROUP];
#pragma unroll
          for (int j = 0; j < GROUP; j++) g[j] = __shfl_sync(0xffffffffu, t, k * GROUP + j);
          float mine;
          if (SCHEME == POND_WENO5) {
            mine = weno5(g, offk);
          } else {
            float l[4];
            lagr4(offk, l);
            mine = 0.f;
#pragma unroll
            for (int j = 0; j < 4; j++) mine = fmaf(l[j], g[j], mine);
          }
          float fn[5];
#pragma unroll
          for (int j = 0; j < 5; j++) fn[j] = __shfl_sync(0xffffffffu, mine, j * GROUP);
          ok = moments_and_test(a, fn, vk, w);
          if (ok) break;
        }
        if (lane == 0) {
          it_sum += w.niter;
          nc += ok ? 0 : 1;
          it_max = max(it_max, w.niter);
          finish_node(a, w, off, ps, n, sample, sf, su, sT);
        }
      }
      // this thread's global writes of the new level, before the next bulk copy reads them
      asm volatile("fence.proxy.async.global;\n" ::: "memory");
      __syncthreads();  // the new level is in global memory; the shared copy is free
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    it_sum += __shfl_xor_sync(0xffffffffu, it_sum, o);
    nc += __shfl_xor_sync(0xffffffffu, nc, o);
    it_max = max(it_max, __shfl_xor_sync(0xffffffffu, it_max, o));
  }
  if (lane == 0) {
    atomicAdd(&a.stats[0], it_sum);
    if (nc) atomicAdd(&a.stats[1], nc);
    atomicMax(reinterpret_cast<int*>(&a.stats[2]), it_max);
  }
}

__global__ void advance_kernel(int* istep, int k) { *istep += k; }

}  // namespace batch
}  // namespace pond

struct pond_batch {
  int device = 0;
  int P = 0;
  int B = 0;
  long long Ltot = 0;    // nodes of all problems
  long long stride = 0;  // device plane length: bins start on 4-node (16-byte) boundaries
  int interp = POND_WENO5;
  double tau = 0.9, tol_abs = 1e-7, tol_rel = 1e-6;
  int max_iter = 100;
  int threads = 768;   // threads per CTA (autotuned)
  int lane_cap = 4;    // phase-1 iterations per node (autotuned)
  int grid = 0;
  cudaStream_t stream = nullptr;
  float* f = nullptr;
  float* rho = nullptr;
  float* u = nullptr;
  float* T = nullptr;
  long long* bin_off = nullptr;
  int* seg_first = nullptr;
  int* segs = nullptr;
  int* queue = nullptr;
  int* istep_dev = nullptr;
  unsigned long long* stats = nullptr;
  unsigned long long* pcount = nullptr;
  int* err = nullptr;
  float* px = nullptr;
  float* py = nullptr;
  long long pcap = 0;
  int pair_every = 0, pair_stride = 1;
  std::vector<long long> pos;  // first node of each problem in bin order
  std::vector<int> len;
  long long istep = 0;
  cudaGraphExec_t exec = nullptr;
  int exec_k = -1, exec_threads = -1, exec_cap = -1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace pond {
namespace batch {

static void* kernel_for(int interp, int threads) {
  if (interp == POND_WENO5) {
    switch (threads) {
      case 256: return (void*)batch_kernel<POND_WENO5, 256>;
      case 512: return (void*)batch_kernel<POND_WENO5, 512>;
      case 768: return (void*)batch_kernel<POND_WENO5, 768>;
      default: return (void*)batch_kernel<POND_WENO5, 1024>;
    }
  }
  switch (threads) {
    case 256: return (void*)batch_kernel<POND_LAGR4, 256>;
    case 512: return (void*)batch_kernel<POND_LAGR4, 512>;
    case 768: return (void*)batch_kernel<POND_LAGR4, 768>;
    default: return (void*)batch_kernel<POND_LAGR4, 1024>;
  }
}

// Enqueue one K-step chunk: queue reset, the persistent kernel, step counter.
static int enqueue_chunk(pond_batch* b, int k, cudaStream_t s) {
  Args a;
  a.f = b->f; a.rho = b->rho; a.u = b->u; a.T = b->T; a.stride = b->stride;
  a.bin_off = b->bin_off; a.seg_first = b->seg_first; a.segs = b->segs; a.B = b->B;
  a.queue = b->queue; a.istep = b->istep_dev; a.nsteps = k;
  a.dtau = float(1.0 / b->tau); a.tol_abs = b->tol_abs; a.tol_rel = b->tol_rel; a.max_iter = b->max_iter;
  a.lane_cap = b->lane_cap;
  a.stats = b->stats;
  a.px = b->pair_every > 0 ? b->px : nullptr; a.py = b->py; a.pcount = b->pcount; a.pcap = b->pcap;
  a.pair_every = b->pair_every > 0 ? b->pair_every : 1; a.pair_stride = b->pair_stride;
  a.err = b->err;
  void* kern = kernel_for(b->interp, b->threads);
  cudaError_t e = cudaMemsetAsync(b->queue, 0, sizeof(int), s);
  if (e != cudaSuccess) return cuda_fail(e, "batch queue reset");
  void* args[] = {&a};
  e = cudaLaunchKernel(kern, dim3(b->grid), dim3(b->threads), args, SMEM, s);
  if (e != cudaSuccess) return cuda_fail(e, "batch kernel launch");
  advance_kernel<<<1, 1, 0, s>>>(b->istep_dev, k);
  e = cudaGetLastError();
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "batch step counter");
}

static void drop_graph(pond_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->exec_k = b->exec_threads = b->exec_cap = -1;
}

// Capture one chunk of k steps as a CUDA graph (kept until k, the tile or
// the pair settings change).
static int chunk_graph(pond_batch* b, int k) {
  if (b->exec && b->exec_k == k && b->exec_threads == b->threads && b->exec_cap == b->lane_cap) return POND_OK;
  drop_graph(b);
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
  const int st = enqueue_chunk(b, k, b->stream);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->stream, &g);
  if (st != POND_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->exec = nullptr;
    return cuda_fail(e, "cudaGraphInstantiate");
  }
  b->exec_k = k;
  b->exec_threads = b->threads;
  b->exec_cap = b->lane_cap;
  return POND_OK;
}

// Best-fit packing of the problems, longest first, into bins of at most
// BIN_CAP nodes and BIN_SEGS problems.
static void pack(const int32_t* lengths, int P, std::vector<std::vector<int>>& bins) {
  std::vector<int> order(P);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return lengths[x] > lengths[y]; });
  std::set<std::pair<int, int>> room;  // (free nodes, bin) of bins with a free problem slot
  std::vector<int> free_nodes;
  for (int p : order) {
    const int l = lengths[p];
    auto it = room.lower_bound({l, -1});
    int bi;
    if (it == room.end()) {
      bi = (int)bins.size();
      bins.emplace_back();
      free_nodes.push_back(BIN_CAP);
    } else {
      bi = it->second;
      room.erase(it);
    }
    bins[bi].push_back(p);
    free_nodes[bi] -= l;
    if ((int)bins[bi].size() < BIN_SEGS && free_nodes[bi] > 0) room.insert({free_nodes[bi], bi});
  }
}

}  // namespace batch
}  // namespace pond

using namespace pond;

extern "C" {

int pond_batch_destroy(pond_batch* b) {
  if (!b) return POND_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch::drop_graph(b);
  cudaFree(b->f); cudaFree(b->rho); cudaFree(b->u); cudaFree(b->T);
  cudaFree(b->bin_off); cudaFree(b->seg_first); cudaFree(b->segs);
  cudaFree(b->queue); cudaFree(b->istep_dev); cudaFree(b->stats); cudaFree(b->pcount); cudaFree(b->err);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return POND_OK;
}

int pond_batch_create(int nproblems, const int32_t* lengths, int interp, double tau, double tol_abs,
                      double tol_rel, int max_iter, int device, pond_batch** out) {
  if (!out) return set_error(POND_ERR_ARG, "pond_batch_create: null output");
  *out = nullptr;
  if (!lengths || nproblems <= 0) return set_error(POND_ERR_ARG, "pond_batch_create: no problems");
  if (interp != POND_WENO5 && interp != POND_LAGR4)
    return set_error(POND_ERR_UNSUPPORTED, "batched D1Q5 runs WENO5 (8) or cubic Lagrange (4), not %d", interp);
  if (!(tau > 0.5) || max_iter < 1 || !(tol_abs >= 0) || !(tol_rel >= 0))
    return set_error(POND_ERR_ARG, "bad tau, max_iter or tolerance");
  long long Ltot = 0;
  for (int p = 0; p < nproblems; p++) {
    if (lengths[p] < 1 || lengths[p] > batch::MAX_LEN)
      return set_error(POND_ERR_ARG, "problem %d has length %d (allowed 1..%d)", p, lengths[p], batch::MAX_LEN);
    Ltot += lengths[p];
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  std::vector<std::vector<int>> bins;
  batch::pack(lengths, nproblems, bins);
  pond_batch* b = new pond_batch();
  b->device = device; b->P = nproblems; b->B = (int)bins.size(); b->Ltot = Ltot; b->interp = interp;
  b->tau = tau; b->tol_abs = tol_abs; b->tol_rel = tol_rel; b->max_iter = max_iter;
  b->len.assign(lengths, lengths + nproblems);
  b->pos.assign(nproblems, 0);
  std::vector<long long> bin_off(b->B + 1, 0);
  std::vector<int> seg_first(b->B + 1, 0), segs;
  for (int bi = 0; bi < b->B; bi++) {
    int local = 0;
    seg_first[bi] = (int)segs.size();
    for (int p : bins[bi]) {
      segs.push_back(local);
      b->pos[p] = bin_off[bi] + local;
      local += lengths[p];
    }
    segs.push_back(local);
    bin_off[bi + 1] = (bin_off[bi] + local + 3) & ~3LL;  // bulk copies start 16-byte aligned
  }
  seg_first[b->B] = (int)segs.size();
  const long long S = bin_off[b->B];
  b->stride = S;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  b->grid = std::min(b->B, nsm);  // one resident CTA per SM (a bin fills most of shared memory)
  bool ok = cudaMalloc(&b->f, 5 * S * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&b->rho, S * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&b->u, S * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&b->T, S * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&b->bin_off, bin_off.size() * sizeof(long long)) == cudaSuccess &&
            cudaMalloc(&b->seg_first, seg_first.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&b->segs, segs.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&b->queue, sizeof(int)) == cudaSuccess && cudaMalloc(&b->istep_dev, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&b->stats, 3 * sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc(&b->pcount, sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc(&b->err, sizeof(int)) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    pond_batch_destroy(b);
    return set_error(POND_ERR_NOMEM, "batch buffers (%lld nodes)", Ltot);
  }
  e = cudaMemcpy(b->bin_off, bin_off.data(), bin_off.size() * sizeof(long long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->seg_first, seg_first.data(), seg_first.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->segs, segs.data(), segs.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->istep_dev, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->pcount, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->stats, 0, 3 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->err, 0, sizeof(int));
  // padding nodes between bins are copied along with the bins but never read
  if (e == cudaSuccess) e = cudaMemset(b->f, 0, 5 * S * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(b->rho, 0, S * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(b->u, 0, S * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(b->T, 0, S * sizeof(float));
  for (int t : {256, 512, 768, 1024})
    for (int s : {POND_WENO5, POND_LAGR4})
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(batch::kernel_for(s, t), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)batch::SMEM);
  if (e != cudaSuccess) {
    pond_batch_destroy(b);
    return cuda_fail(e, "batch set-up");
  }
  *out = b;
  return POND_OK;
}

int64_t pond_batch_nodes(const pond_batch* b) { return b ? b->Ltot : 0; }
int32_t pond_batch_bins(const pond_batch* b) { return b ? b->B : 0; }

int pond_batch_set_state(pond_batch* b, const double* rho, const double* u, const double* T) {
  if (!b || !rho || !u || !T) return set_error(POND_ERR_ARG, "pond_batch_set_state: null argument");
  const long long n = b->stride;
  std::vector<float> fb(5 * n), rb(n), ub(n), tb(n);
  long long src = 0;
  for (int p = 0; p < b->P; p++) {
    const long long dst = b->pos[p];
    for (int i = 0; i < b->len[p]; i++, src++) {
      const double r = rho[src], v = u[src], t = T[src];
      if (!(std::isfinite(r) && std::isfinite(v) && t > 0 && std::isfinite(t)))
        return set_error(POND_ERR_ARG, "problem %d node %d: rho and u must be finite and T > 0", p, i);
      rb[dst + i] = (float)r; ub[dst + i] = (float)v; tb[dst + i] = (float)t;
      for (int k = 0; k < 5; k++) fb[k * n + dst + i] = (float)(lattice_weight_t<POND_D1Q5>(k) * r);
    }
  }
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(b->f, fb.data(), fb.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->rho, rb.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->u, ub.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->T, tb.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->istep_dev, 0, sizeof(int));
  b->istep = 0;
  return e == cudaSuccess ? POND_OK : cuda_fail(e, "pond_batch_set_state");
}

int pond_batch_get_state(pond_batch* b, double* f, double* rho, double* u, double* T) {
  if (!b) return set_error(POND_ERR_ARG, "pond_batch_get_state: null batch");
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "pond_batch_get_state");
  const long long n = b->stride, nu = b->Ltot;
  std::vector<float> tmp(5 * n);
  struct Item {
    double* dst;
    const float* src;
    int comps;
  } items[4] = {{f, b->f, 5}, {rho, b->rho, 1}, {u, b->u, 1}, {T, b->T, 1}};
  for (const Item& it : items) {
    if (!it.dst) continue;
    e = cudaMemcpy(tmp.data(), it.src, it.comps * n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "pond_batch_get_state");
    for (int k = 0; k < it.comps; k++) {
      long long dst = (long long)k * nu;
      for (int p = 0; p < b->P; p++) {
        const float* s = tmp.data() + (long long)k * n + b->pos[p];
        for (int i = 0; i < b->len[p]; i++) it.dst[dst++] = s[i];
      }
    }
  }
  return POND_OK;
}

int pond_batch_set_pairs(pond_batch* b, float* X, float* Y, int64_t capacity, int every, int stride) {
  if (!b || every < 0 || stride < 1 || (every > 0 && (!X || !Y || capacity <= 0)))
    return set_error(POND_ERR_ARG, "pond_batch_set_pairs: bad argument");
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemset(b->pcount, 0, sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "pond_batch_set_pairs");
  b->px = X; b->py = Y; b->pcap = capacity; b->pair_every = every; b->pair_stride = stride;
  batch::drop_graph(b);
  return POND_OK;
}

int pond_batch_pairs_written(pond_batch* b, int64_t* n) {
  if (!b || !n) return set_error(POND_ERR_ARG, "pond_batch_pairs_written: null argument");
  cudaSetDevice(b->device);
  unsigned long long c = 0;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&c, b->pcount, sizeof(c), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "pond_batch_pairs_written");
  *n = (int64_t)std::min<unsigned long long>(c, (unsigned long long)b->pcap);
  return POND_OK;
}

int pond_batch_run(pond_batch* b, int nsteps, int k, float* ms) {
  if (!b || nsteps < 0 || k < 1) return set_error(POND_ERR_ARG, "pond_batch_run: bad argument");
  cudaSetDevice(b->device);
  cudaError_t e = cudaMemsetAsync(b->stats, 0, 3 * sizeof(unsigned long long), b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch statistics reset");
  e = cudaEventRecord(b->ev0, b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  int done = 0;
  while (done < nsteps) {
    const int kk = std::min(k, nsteps - done);
    const int st = batch::chunk_graph(b, kk);
    if (st != POND_OK) return st;
    e = cudaGraphLaunch(b->exec, b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    done += kk;
  }
  e = cudaEventRecord(b->ev1, b->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(b->ev1);
  if (e != cudaSuccess) return cuda_fail(e, "pond_batch_run");
  int err = 0;
  e = cudaMemcpy(&err, b->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "pond_batch_run");
  if (err) {
    cudaMemset(b->err, 0, sizeof(int));
    return set_error(POND_ERR_CUDA, "pond_batch_run: a bin staging copy did not complete; the state is undefined");
  }
  float t = 0;
  cudaEventElapsedTime(&t, b->ev0, b->ev1);
  if (ms) *ms = t;
  b->istep += nsteps;
  return POND_OK;
}

int pond_batch_stats(pond_batch* b, int64_t* niter_sum, int64_t* nonconverged, int32_t* niter_max) {
  if (!b) return set_error(POND_ERR_ARG, "pond_batch_stats: null batch");
  cudaSetDevice(b->device);
  unsigned long long h[3] = {0, 0, 0};
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(h, b->stats, sizeof(h), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "pond_batch_stats");
  int mx;
  std::memcpy(&mx, &h[2], sizeof(int));
  if (niter_sum) *niter_sum = (int64_t)h[0];
  if (nonconverged) *nonconverged = (int64_t)h[1];
  if (niter_max) *niter_max = mx;
  return POND_OK;
}

int pond_batch_set_tile(pond_batch* b, int threads, int lane_cap) {
  if (!b || (threads != 256 && threads != 512 && threads != 768 && threads != 1024) || lane_cap < 1)
    return set_error(POND_ERR_ARG, "tile: threads per CTA 256, 512, 768 or 1024 and lane_cap >= 1");
  b->threads = threads;
  b->lane_cap = lane_cap;
  return POND_OK;
}

int pond_batch_get_tile(const pond_batch* b, int* threads, int* lane_cap) {
  if (!b) return set_error(POND_ERR_ARG, "pond_batch_get_tile: null batch");
  if (threads) *threads = b->threads;
  if (lane_cap) *lane_cap = b->lane_cap;
  return POND_OK;
}

int pond_batch_autotune(pond_batch* b, int probe_steps, const int32_t* tiles, int ncand, float* ms_out, int* best) {
  if (!b || probe_steps < 1 || !tiles || ncand < 1) return set_error(POND_ERR_ARG, "pond_batch_autotune: bad argument");
  for (int c = 0; c < ncand; c++) {
    const int t = tiles[2 * c], l = tiles[2 * c + 1];
    if ((t != 256 && t != 512 && t != 768 && t != 1024) || l < 1)
      return set_error(POND_ERR_ARG, "autotune candidate %d is not a valid tile", c);
  }
  cudaSetDevice(b->device);
  const long long n = b->stride;
  float* snap = nullptr;
  int istep_dev = 0;
  cudaError_t e = cudaMalloc(&snap, 8 * n * sizeof(float));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(POND_ERR_NOMEM, "autotune snapshot");
  }
  float* parts[4] = {b->f, b->rho, b->u, b->T};
  const long long cnt[4] = {5 * n, n, n, n};
  const long long at[4] = {0, 5 * n, 6 * n, 7 * n};
  e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&istep_dev, b->istep_dev, sizeof(int), cudaMemcpyDeviceToHost);
  for (int i = 0; i < 4 && e == cudaSuccess; i++)
    e = cudaMemcpyAsync(snap + at[i], parts[i], cnt[i] * sizeof(float), cudaMemcpyDeviceToDevice, b->stream);
  const int saved_every = b->pair_every, saved[2] = {b->threads, b->lane_cap};
  b->pair_every = 0;
  batch::drop_graph(b);
  float best_ms = 1e30f;
  int best_c = -1;
  int st = e == cudaSuccess ? POND_OK : cuda_fail(e, "autotune snapshot");
  for (int c = 0; c < ncand && st == POND_OK; c++) {
    b->threads = tiles[2 * c];
    b->lane_cap = tiles[2 * c + 1];
    float ms = 0;
    st = pond_batch_run(b, probe_steps, probe_steps, &ms);
    if (ms_out) ms_out[c] = ms;
    if (st == POND_OK && ms < best_ms) {
      best_ms = ms;
      best_c = c;
    }
    for (int i = 0; i < 4 && st == POND_OK; i++) {
      e = cudaMemcpyAsync(parts[i], snap + at[i], cnt[i] * sizeof(float), cudaMemcpyDeviceToDevice, b->stream);
      if (e != cudaSuccess) st = cuda_fail(e, "autotune restore");
    }
    if (st == POND_OK) {
      e = cudaMemcpyAsync(b->istep_dev, &istep_dev, sizeof(int), cudaMemcpyHostToDevice, b->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
      if (e != cudaSuccess) st = cuda_fail(e, "autotune restore");
    }
    b->istep -= probe_steps;
  }
  cudaStreamSynchronize(b->stream);
  cudaFree(snap);
  b->pair_every = saved_every;
  const bool ok = st == POND_OK && best_c >= 0;
  b->threads = ok ? tiles[2 * best_c] : saved[0];
  b->lane_cap = ok ? tiles[2 * best_c + 1] : saved[1];
  batch::drop_graph(b);
  if (best) *best = best_c;
  return st;
}

}  // extern "C"
