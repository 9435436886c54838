// Headless driver for the reference's own CUDA step kernels (TEST
// INFRASTRUCTURE ONLY).  oracle/build_ref.sh compiles it together with the
// reference's update.cu / init.cu / lbpack.cu / diagn.cu / drop.cu, taken
// from patched copies of engrab6/lbmPonD, into oracle/_ref/.  It replaces the
// GL application (lbm.cu) with a file-in / file-out loop:
//
//   ref_pond <in.state> <out.state> <nsteps> <tau> [<in.mesh> <out.mesh> <amr>]
//
// It uploads the lattice tables as lbm.cu:201-250 does, calls the reference
// init() (init.cu:109), overwrites both population buffers with the state read
// from <in.state>, then runs the kernel-launch part of calcStep
// (update.cu:92-100 and :138-141: reset accumulators, launch PonDstep or
// PonDstepD3Q125, swap buffers, refresh the constant parameters) <nsteps>
// times and writes the final state.  Each step's kernel time is measured with
// CUDA events around the step launch only.
//
// State file (little endian): int32 magic 0x504f4e44, int32 Q, int64 nx, ny,
// nz, then float64 f[Q*N], rho[N], g[4*N] (u_x,u_y,u_z,T), x fastest.  The
// output file appends int32 NiterMax of the last step, int32 nsteps,
// float32 kernel milliseconds per step and the float64 mean of the last
// step's per-node iteration counts.
//
// Mesh mode (the 1D adaptive-mesh code the reference's calcStep leaves
// commented, enabled by build_ref.sh's gap2 / nu3 schemes): <in.mesh> holds
// the node mask (Cinfo::set) and, for an NRMESH build, the node positions
// (Cell::p.x); after every step with <amr> = 1 the driver runs
// cinfo_setnew_reset, AMR_add, cinfo_set_new and AMR_remove in calcStep's
// order (update.cu:102-105) before the swap.  <out.mesh> receives the final
// mask and positions.  Mesh file: uint32 magic 0x4d455348, int64 N, uint8
// mask[N], float64 pos[N].
//
// A D3Q125 build with -DPOND_REF_D3Q125_PULL launches PonDstep (LBMpull)
// instead of PonDstepD3Q125, as the reference's calcStep does once its
// `#if defined D3Q125 && 1` (update.cu:97) reads `&& 0`.
//
// With POND_REF_TIMECORR=s in the environment the driver also runs the
// reference's TimeCorr(s) (update.cu:15-28: u *= s, T *= s*s, its call
// commented at update.cu:123) after every step, before the swap, and scales
// dt by s (update.cu:128).
#include "structs.cuh"
#include <cstdint>
#include <cstdlib>
#include <vector>

// Globals that lbm.cu:13-24 normally defines.
im3D_pars im3DHost;
LBMParamsHost parsHost;
__constant__ LBMParams pars;
__constant__ int3 e[Qn];
__constant__ ftype3 ef[Qn];
__constant__ ftype w[Qn];
__constant__ int reverseX[Qn];
__constant__ int reverseY[Qn];
__constant__ int reverseZ[Qn];
__constant__ int reverseXYZ[Qn];
image2D im2D;
int maxR = 1;
float calcTime, calcPerf;
int TimeStep;
bool recalc_at_once;
const char* FuncStr[] = {"Rho"};

void init();
__global__ void PonDstep();
__global__ void PonDstepD3Q125();
__global__ void cinfo_setnew_reset();
__global__ void cinfo_set_new();
__global__ void AMR_add();
__global__ void AMR_remove();
__global__ void TimeCorr(ftype dtscale);

static const uint32_t MAGIC = 0x504f4e44u;
static const uint32_t MESH_MAGIC = 0x4d455348u;

static bool read_mesh(const char* fn, int64_t N, std::vector<uint8_t>& mask, std::vector<double>& pos) {
  FILE* fp = fopen(fn, "rb");
  if (!fp) return false;
  uint32_t magic; int64_t n;
  bool ok = fread(&magic, 4, 1, fp) == 1 && fread(&n, 8, 1, fp) == 1 && magic == MESH_MAGIC && n == N;
  if (ok) {
    mask.resize(N); pos.resize(N);
    ok = fread(mask.data(), 1, N, fp) == (size_t)N && fread(pos.data(), 8, N, fp) == (size_t)N;
  }
  fclose(fp);
  return ok;
}

static bool write_mesh(const char* fn, const std::vector<uint8_t>& mask, const std::vector<double>& pos) {
  FILE* fp = fopen(fn, "wb");
  if (!fp) return false;
  const int64_t n = (int64_t)mask.size();
  fwrite(&MESH_MAGIC, 4, 1, fp); fwrite(&n, 8, 1, fp);
  fwrite(mask.data(), 1, mask.size(), fp); fwrite(pos.data(), 8, pos.size(), fp);
  fclose(fp);
  return true;
}

static bool read_state(const char* fn, int64_t n[3], std::vector<double>& f, std::vector<double>& rho,
                       std::vector<double>& g) {
  FILE* fp = fopen(fn, "rb");
  if (!fp) return false;
  uint32_t magic; int32_t q;
  bool ok = fread(&magic, 4, 1, fp) == 1 && fread(&q, 4, 1, fp) == 1 && fread(n, 8, 3, fp) == 3;
  ok = ok && magic == MAGIC && q == Qn;
  if (ok) {
    const int64_t N = n[0] * n[1] * n[2];
    f.resize((size_t)Qn * N); rho.resize(N); g.resize(4 * (size_t)N);
    ok = fread(f.data(), 8, f.size(), fp) == f.size() && fread(rho.data(), 8, rho.size(), fp) == rho.size() &&
         fread(g.data(), 8, g.size(), fp) == g.size();
  }
  fclose(fp);
  return ok;
}

int main(int argc, char** argv) {
  if (argc < 5 || (argc > 5 && argc != 8)) {
    fprintf(stderr, "usage: %s in.state out.state nsteps tau [in.mesh out.mesh amr]\n", argv[0]);
    return 2;
  }
  const bool mesh = argc == 8;
  const char* tc = getenv("POND_REF_TIMECORR");
  const double dtscale = tc ? atof(tc) : 0.0;
  const bool amr = mesh && atoi(argv[7]) != 0;
  const int nsteps = atoi(argv[3]);
  const double tau = atof(argv[4]);
  int64_t n[3];
  std::vector<double> f, rho, g;
  if (!read_state(argv[1], n, f, rho, g)) { fprintf(stderr, "bad state file %s\n", argv[1]); return 3; }

  // lattice tables to constant memory (lbm.cu:201-250)
  CHECK_ERROR(cudaMemcpyToSymbol(e, e_host, sizeof(e_host)));
  CHECK_ERROR(cudaMemcpyToSymbol(w, w_host, sizeof(w_host)));
#if !(defined D1Q3 || defined D3Q27)
  CHECK_ERROR(cudaMemcpyToSymbol(ef, ef_host, sizeof(ef_host)));
#endif
  int rx[Qn], ry[Qn], rz[Qn];
  for (int i = 0; i < Qn; i++) { rx[i] = reverseX_host[i]; ry[i] = reverseY_host[i]; rz[i] = reverseZ_host[i]; }
#ifdef D3Q125
  // lbm.cu:206-244 builds the mirrored-direction maps for D3Q125
  for (int i = 0; i < Qn; i++)
    for (int ax = 0; ax < 3; ax++) {
      const double c[3] = {ef_host[i].x, ef_host[i].y, ef_host[i].z};
      if (c[ax] == 0) continue;
      for (int j = 0; j < Qn; j++) {
        const double d[3] = {ef_host[j].x, ef_host[j].y, ef_host[j].z};
        bool same = true;
        for (int b = 0; b < 3; b++) if (d[b] != (b == ax ? -c[b] : c[b])) same = false;
        if (same) { (ax == 0 ? rx : ax == 1 ? ry : rz)[i] = j; break; }
      }
    }
#endif
  CHECK_ERROR(cudaMemcpyToSymbol(reverseX, rx, sizeof(rx)));
  CHECK_ERROR(cudaMemcpyToSymbol(reverseY, ry, sizeof(ry)));
  CHECK_ERROR(cudaMemcpyToSymbol(reverseZ, rz, sizeof(rz)));
  CHECK_ERROR(cudaMemcpyToSymbol(reverseXYZ, reverseXYZ_host, sizeof(reverseXYZ_host)));

  // the GL-free part of LBMParamsHost::set (lbm.cu:134-168)
  parsHost.nFunc = 0;
  parsHost.Nx = LSizeX * brick.x; parsHost.Ny = LSizeY * brick.y; parsHost.Nz = LSizeZ * brick.z;
  if (parsHost.Nx != n[0] || parsHost.Ny != n[1] || parsHost.Nz != n[2]) {
    fprintf(stderr, "state is %ldx%ldx%ld but the binary was compiled for %ldx%ldx%ld\n", (long)n[0], (long)n[1], (long)n[2],
            parsHost.Nx, parsHost.Ny, parsHost.Nz);
    return 4;
  }
  CHECK_ERROR(cudaMallocManaged((void**)&parsHost.NiterMax, sizeof(int)));
  CHECK_ERROR(cudaMallocManaged((void**)&parsHost.mass, sizeof(ftype)));
  CHECK_ERROR(cudaMallocManaged((void**)&parsHost.enrg, sizeof(ftype)));
  CHECK_ERROR(cudaMallocManaged((void**)&parsHost.moment, sizeof(ftype3)));
  parsHost.dt = 1;
  parsHost.iStep = 0;
  parsHost.pc.dtau = 1.0 / tau;
  copy2dev(parsHost, pars);
  init();
  CHECK_ERROR(cudaDeviceSynchronize());

  const int64_t N = n[0] * n[1] * n[2];
  std::vector<uint8_t> mask(N, 1);
  std::vector<double> pos(N);
  for (int64_t i = 0; i < N; i++) pos[i] = double(i % n[0]);  // init.cu:102
  if (mesh) {
    if (!read_mesh(argv[5], N, mask, pos)) { fprintf(stderr, "bad mesh file %s\n", argv[5]); return 3; }
    std::vector<Cinfo> ci(N);
    for (int64_t i = 0; i < N; i++) {
      const int x = i % n[0], y = (i / n[0]) % n[1], z = i / (n[0] * n[1]);
      Cinfo& c = ci[Cinfo::ind_zip(x, y, z)];
      c.ctype = 0; c.niter = 0;
      c.set = c.setnew = mask[i] ? 1 : 0;
    }
    CHECK_ERROR(cudaMemcpy(parsHost.cinfo, ci.data(), N * sizeof(Cinfo), cudaMemcpyHostToDevice));
  }
  std::vector<Group> gh(N);
  for (int64_t i = 0; i < N; i++) {
    Cell c;
    for (int q = 0; q < Qn; q++) c.f[q] = (ftype)f[(size_t)q * N + i];
    c.rho = (ftype)rho[i];
    c.uT = make_ftype4((ftype)g[i], (ftype)g[N + i], (ftype)g[2 * N + i], (ftype)g[3 * N + i]);
    const int x = i % n[0], y = (i / n[0]) % n[1], z = i / (n[0] * n[1]);
#ifdef NRMESH
    c.p = make_ftype3((ftype)pos[i], (ftype)y, (ftype)z);
#endif
    const int2 gc = Group::ind_conv(x, y, z);
    gh[gc.x].pack(c, gc.y);
  }
  CHECK_ERROR(cudaMemcpy(parsHost.loadGroups, gh.data(), N * sizeof(Group), cudaMemcpyHostToDevice));
  CHECK_ERROR(cudaMemcpy(parsHost.storeGroups, gh.data(), N * sizeof(Group), cudaMemcpyHostToDevice));

  cudaEvent_t t0, t1;
  CHECK_ERROR(cudaEventCreate(&t0));
  CHECK_ERROR(cudaEventCreate(&t1));
  std::vector<float> ms(nsteps > 0 ? nsteps : 1, 0.f);
  int niter_max = 0;
  for (int s = 0; s < nsteps; s++) {
    CHECK_ERROR(cudaMemset(parsHost.NiterMax, 0, sizeof(int)));
    CHECK_ERROR(cudaMemset(parsHost.mass, 0, sizeof(ftype)));
    CHECK_ERROR(cudaMemset(parsHost.enrg, 0, sizeof(ftype)));
    CHECK_ERROR(cudaMemset(parsHost.moment, 0, sizeof(ftype3)));
    CHECK_ERROR(cudaEventRecord(t0));
    const dim3 block(parsHost.Nx / brick.x, parsHost.Ny / brick.y, parsHost.Nz / brick.z);
#if defined D3Q125 && !defined POND_REF_D3Q125_PULL
    PonDstepD3Q125<<<dim3(parsHost.Nx, parsHost.Ny, parsHost.Nz), Qn>>>();
#else  // (with POND_REF_D3Q125_PULL a D3Q125 build takes calcStep's other branch, update.cu:99)
    PonDstep<<<block, brick>>>();
#endif
    CHECK_ERROR(cudaEventRecord(t1));
    CHECK_ERROR(cudaDeviceSynchronize());
    CHECK_ERROR(cudaGetLastError());
    CHECK_ERROR(cudaEventElapsedTime(&ms[s], t0, t1));
    niter_max = *parsHost.NiterMax;
    if (amr) {  // update.cu:102-105 with the AMR lines enabled, on the store buffer before the swap
      cinfo_setnew_reset<<<block, brick>>>();
      AMR_add<<<block, brick>>>();
      cinfo_set_new<<<block, brick>>>();
      AMR_remove<<<1, 1>>>();
      CHECK_ERROR(cudaDeviceSynchronize());
      CHECK_ERROR(cudaGetLastError());
    }
    if (dtscale > 0) {  // update.cu:121-128 with the TimeCorr line enabled
      TimeCorr<<<block, brick>>>((ftype)dtscale);
      CHECK_ERROR(cudaDeviceSynchronize());
      CHECK_ERROR(cudaGetLastError());
      parsHost.dt *= dtscale;
    }
    parsHost.iStep++;
    parsHost.swapLS();
    copy2dev(parsHost, pars);
  }
  CHECK_ERROR(cudaMemcpy(gh.data(), parsHost.loadGroups, N * sizeof(Group), cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < N; i++) {
    const int x = i % n[0], y = (i / n[0]) % n[1], z = i / (n[0] * n[1]);
    const int2 gc = Group::ind_conv(x, y, z);
    Cell c;
    gh[gc.x].unpack(c, gc.y);
    for (int q = 0; q < Qn; q++) f[(size_t)q * N + i] = c.f[q];
    rho[i] = c.rho;
    g[i] = c.uT.x; g[N + i] = c.uT.y; g[2 * N + i] = c.uT.z; g[3 * N + i] = c.uT.w;
#ifdef NRMESH
    pos[i] = c.p.x;
#endif
  }
  if (mesh) {
    std::vector<Cinfo> ci(N);
    CHECK_ERROR(cudaMemcpy(ci.data(), parsHost.cinfo, N * sizeof(Cinfo), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < N; i++) {
      const int x = i % n[0], y = (i / n[0]) % n[1], z = i / (n[0] * n[1]);
      mask[i] = ci[Cinfo::ind_zip(x, y, z)].set ? 1 : 0;
    }
    if (!write_mesh(argv[6], mask, pos)) { fprintf(stderr, "cannot write %s\n", argv[6]); return 5; }
  }
  FILE* fp = fopen(argv[2], "wb");
  if (!fp) { fprintf(stderr, "cannot write %s\n", argv[2]); return 5; }
  const uint32_t magic = MAGIC; const int32_t q = Qn;
  fwrite(&magic, 4, 1, fp); fwrite(&q, 4, 1, fp); fwrite(n, 8, 3, fp);
  fwrite(f.data(), 8, f.size(), fp); fwrite(rho.data(), 8, rho.size(), fp); fwrite(g.data(), 8, g.size(), fp);
  const int32_t ns = nsteps;
  fwrite(&niter_max, 4, 1, fp); fwrite(&ns, 4, 1, fp); fwrite(ms.data(), 4, ms.size(), fp);
  {  // mean of the per-node iteration counts of the last step (Cinfo::niter, steps.cu:417,508)
    std::vector<Cinfo> ci(N);
    CHECK_ERROR(cudaMemcpy(ci.data(), parsHost.cinfo, N * sizeof(Cinfo), cudaMemcpyDeviceToHost));
    double sum = 0;
    for (int64_t i = 0; i < N; i++) sum += ci[i].niter;
    const double mean = N ? sum / double(N) : 0.0;
    fwrite(&mean, 8, 1, fp);
  }
  fclose(fp);
  printf("ref_pond: Q=%d %ldx%ldx%ld steps=%d NiterMax=%d ms/step(last)=%.3f\n", Qn, (long)n[0], (long)n[1],
         (long)n[2], nsteps, niter_max, ms.empty() ? 0.f : ms.back());
  return 0;
}
