// C ABI of libturbid_gpu.so and the orchestration of the RK3 substep.
//
// One context = one case on one GPU.  The phase methods below follow the
// reference's FlatCarrierPhase / FlatScalarPhase call sequence
// (src/phase_carrier_flat.cc:272-709, src/phase_scalar_flat.cc:245-533) but
// keep every field resident in HBM in the z-slab spectral layout, fold the
// boundary fix rows into the two Helmholtz matrices, fuse the elementwise
// Armadillo expressions into GEMM epilogues, and skip the transforms whose
// results the reference never reads (only the bottom plane of du/dz, dv/dz
// feeds the erosion flux; the scalar phase's physical velocity is the
// carrier's plus a constant settling shift).
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <regex>
#include <sstream>
#include <stdexcept>
#include <string>

#include "fields.cuh"
#include "setup.h"
#include "tg_common.cuh"

namespace tg {

thread_local std::string g_err;
long long g_launches = 0;
void set_error(const std::string& m) { g_err = m; }

// columns: stage; rows: c1, c2, c3 (src/stepper_time_rk3.cc:28-31)
static const double RK3[3][3] = {{0.0 / 1.0, -5.0 / 9.0, -153.0 / 128.0},
                                 {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0},
                                 {1.0 / 6.0, 5.0 / 24.0, 1.0 / 8.0}};
static const double kSmall = 10e-12;   // COMPARE_NUMBER_SMALL, src/common.h:42

void fft_init();

// ---------------------------------------------------------------------------
// profiler: CUDA events around every instrumented launch, grouped by class
// ---------------------------------------------------------------------------
struct Profiler {
  struct Rec {
    int cat;
    double bytes, flops, xflops;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  double last_x[TG_PROF_NCAT] = {0};  // executed flops of the window tg_profile_end closed
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  cudaEvent_t get() {
    if (used < pool.size()) return pool[used++];
    cudaEvent_t e;
    TG_CUDA(cudaEventCreate(&e));
    pool.push_back(e);
    ++used;
    return e;
  }
  void reset() {
    recs.clear();
    used = 0;
  }
  ~Profiler() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};
thread_local Profiler* g_prof = nullptr;

void prof_begin(cudaStream_t s, int cat, double bytes, double flops, double xflops) {
  if (!g_prof) return;
  Profiler::Rec r{cat, bytes, flops, xflops < 0 ? flops : xflops, g_prof->get(), g_prof->get()};
  TG_CUDA(cudaEventRecord(r.a, s));
  g_prof->recs.push_back(r);
}
void prof_end(cudaStream_t s) {
  if (!g_prof || g_prof->recs.empty()) return;
  TG_CUDA(cudaEventRecord(g_prof->recs.back().b, s));
}

struct Ctx {
  tg_case c{};
  int nx = 0, ny = 0, nz = 0, nxc = 0, nyc = 0, nxh = 0, M = 0;
  size_t S = 0, P = 0;
  bool mixed = false, scalar = false, opentop = false;
  cudaStream_t s = nullptr;
  bool own_stream = false;
  std::vector<double> gridz, gridzc, gridlenz, D1h, D2h;
  double lmx = 0, lmy = 0;
  Decomposition dec[5];
  // device constants
  double *kx = nullptr, *ky = nullptr, *dx2 = nullptr, *dy2 = nullptr, *k2 = nullptr;
  double *gz = nullptr, *glz = nullptr, *d1r0 = nullptr, *d1rn = nullptr;
  int* yidx = nullptr;
  ZOperator opD1, opD2, opTmp, opEinv[5], opE[5];
  // z-solver of the dense Helmholtz solves in mixed precision: FP64 DMMA
  // (TG_ZSOLVER_DMMA) or the int8-slice tensor-core product (TG_ZSOLVER_ISLICE,
  // the default of the mixed mode)
  int zsolver = TG_ZSOLVER_DMMA;
  IsliceOp* islTmp = nullptr;
  // the flag of the int8-slice products' bounded waits (device), copied to
  // err_h[slot] with every step's features and checked with them
  int* isl_err = nullptr;
  int* err_h = nullptr;   // pinned [2]
  double* lamd[5] = {nullptr};
  FftPlan px, py;
  TransformDims td{};
  // device fields
  double2 *U = nullptr, *PR = nullptr, *H = nullptr, *DP = nullptr, *SU = nullptr, *RHS = nullptr, *TMP = nullptr;
  double2 *ADV = nullptr, *DU = nullptr, *F6 = nullptr, *PHI = nullptr, *HPHI = nullptr, *ADVPHI = nullptr;
  double2 *RHSPHI = nullptr, *hist = nullptr, *ero = nullptr, *REF = nullptr;
  void *UNL = nullptr, *DUP = nullptr, *PRD = nullptr, *PHIP = nullptr, *PLN = nullptr, *work = nullptr;
  int work_planes = 0;  // planes one transform launch pair handles
  double* feat = nullptr;
  unsigned long long* bits = nullptr;
  double* feat_h = nullptr;   // pinned [2][100]
  cudaEvent_t fev[2] = {nullptr, nullptr};
  // whole RK3 steps replayed as CUDA graphs (one per alternation parity): the
  // only per-step kernel argument, the mean-mode forcing, goes through
  // force_d, copied from the pinned slot force_h[parity] by the graph itself
  bool graphs = true, capturing = false;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  long long gkernels[2] = {0, 0};
  cudaStream_t cap_s = nullptr;
  double* force_d = nullptr;  // device [2]
  double* force_h = nullptr;  // pinned [2 parities][2]
  // The scalar phase's Correct of stage s runs on a second stream s2 while the
  // carrier's next Predict computes its nonlinear term on s; the carrier waits
  // for the scalar (sc_done) only where it needs phi (the buoyancy term of the
  // H update).  The scalar phase then works in its own scratch fields; the
  // erosion planes alternate between two buffers by stage parity.
  double *post_buf = nullptr, *post_out = nullptr;  // post-processor, allocated on first use
  int post_planes = 0;
  bool overlap = true, overlap_active = false, sc_pending = false;
  cudaStream_t s2 = nullptr;
  cudaEvent_t cc_done = nullptr, sc_done = nullptr;
  // The w solve of the carrier Predict, when it is split (folded kernel), runs
  // on a third stream beside the u and v solves (dense kernel), so that the
  // two launches fill each other's tails; same conditions as the overlap.
  bool fork_active = false;
  cudaStream_t s3 = nullptr;
  cudaEvent_t w_fork = nullptr, w_join = nullptr;
  double2 *TMP_s = nullptr, *F6_s = nullptr;
  void *PRD_s = nullptr, *DUP_s = nullptr, *work_s = nullptr, *PLN2 = nullptr, *PLN1 = nullptr;
  std::vector<void*> allocs;
  Profiler prof;
  // time / phase state
  int step = 0;
  double time = 0, dt = 0, olddt = 0, cfl = 0;
  bool alternation = false, isforward = true, loaded = false;
  double sig_u[3] = {0, 0, 0}, sig_s[3] = {0, 0, 0};
  double shift[3] = {0, 0, 0};

  template <typename X>
  X* dalloc(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(X));
    if (e != cudaSuccess) {
      (void)cudaGetLastError();   // not left for the next launch check
      throw Error{TG_ERR_NOMEM, std::string("tg_create > cudaMalloc > ") + cudaGetErrorString(e)};
    }
    allocs.push_back(p);
    TG_CUDA(cudaMemset(p, 0, n * sizeof(X)));
    return reinterpret_cast<X*>(p);
  }
  void release_overlap() {
    if (s2) cudaStreamDestroy(s2);
    if (cc_done) cudaEventDestroy(cc_done);
    if (sc_done) cudaEventDestroy(sc_done);
    if (s3) cudaStreamDestroy(s3);
    if (w_fork) cudaEventDestroy(w_fork);
    if (w_join) cudaEventDestroy(w_join);
    s2 = s3 = nullptr;
    cc_done = sc_done = w_fork = w_join = nullptr;
  }
  void drop_graphs() {
    for (auto& g : gexec) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
  }
  ~Ctx() {
    for (int i = 0; i < 5; ++i) {
      islice_destroy(opEinv[i].isl);
      islice_destroy(opE[i].isl);
    }
    islice_destroy(islTmp);
    drop_graphs();
    release_overlap();
    if (cap_s) cudaStreamDestroy(cap_s);
    for (void* p : allocs) cudaFree(p);
    if (feat_h) cudaFreeHost(feat_h);
    if (err_h) cudaFreeHost(err_h);
    if (force_h) cudaFreeHost(force_h);
    for (auto& e : fev)
      if (e) cudaEventDestroy(e);
    fft_plan_destroy(px);
    fft_plan_destroy(py);
    if (own_stream && s) cudaStreamDestroy(s);
  }
  size_t psize() const { return mixed ? sizeof(float) : sizeof(double); }
};

// ---------------------------------------------------------------------------
// construction
// ---------------------------------------------------------------------------
static std::function<double*(size_t)> allocator(Ctx& x) {
  return [&x](size_t n) { return x.dalloc<double>(n); };
}

// The solve's two GEMMs: dense (E^-1 with the forward fix folded in, E with
// the backward fix rows), or, for a decomposition whose eigenvectors have
// parity (w and the pressure: the same condition on both walls), the split
// pair of half-size products of the folded-operator kernel (half the flops).
static void install_decomposition(Ctx& x, int which) {
  std::vector<double> Ei, E;
  double quirk = 0.0;
  if (split_operators(x.dec[which], which == 3, Ei, E, quirk)) {
    zop_build_split(x.opEinv[which], Ei, x.nz, 1, 0.0, allocator(x));
    zop_build_split(x.opE[which], E, x.nz, 2, quirk, allocator(x));
  } else {
    fold_decomposition(x.dec[which], which == 3, Ei, E);
    zop_build(x.opEinv[which], Ei, x.nz, false, allocator(x));
    zop_build(x.opE[which], E, x.nz, false, allocator(x));
    // the int8-slice form of the two products (mixed precision, interior of
    // at most 256 rows); used while the z-solver selects it
    if (x.mixed && x.nz - 2 <= 256) {
      auto bytes = [&x](size_t n) -> void* { return x.dalloc<unsigned char>(n); };
      islice_build(x.opEinv[which].isl, Ei, x.nz, x.nz, 5, x.M, bytes, x.isl_err);
      islice_build(x.opE[which].isl, E, x.nz, x.nz, 5, x.M, bytes, x.isl_err);
    }
  }
  x.opEinv[which].use_isl = x.opE[which].use_isl = x.zsolver == TG_ZSOLVER_ISLICE;
  if (!x.lamd[which]) x.lamd[which] = x.dalloc<double>(x.nz);
  TG_CUDA(cudaMemcpy(x.lamd[which], x.dec[which].lam.data(), sizeof(double) * x.nz, cudaMemcpyHostToDevice));
}

static Ctx* create(const tg_case& c) {
  if (c.nx < 1 || c.ny < 1 || c.nz < 3) throw Error{TG_ERR_SHAPE, "DomainDecomposition::Configure > Empty Data Dimension is not Supported!"};
  if (c.nphase < 1 || c.nphase > 2) throw Error{TG_ERR_ARG, "tg_create > total_phase_number must be 1 or 2"};
  if (c.precision != TG_PREC_FP64 && c.precision != TG_PREC_MIXED) throw Error{TG_ERR_ARG, "tg_create > unknown precision"};
  std::unique_ptr<Ctx> px(new Ctx);
  Ctx& x = *px;
  x.c = c;
  x.nx = c.nx;
  x.ny = c.ny;
  x.nz = c.nz;
  x.nxc = c.nx / 3 * 2;   // src/base.cc:233-234
  x.nyc = c.ny / 3 * 2;
  x.nxh = x.nxc / 2 + 1;
  x.M = x.nyc * x.nxh;
  if (x.nyc < 1) throw Error{TG_ERR_SHAPE, "DomainDecomposition::Configure > Ny too small for the 2/3 cut"};
  x.S = (size_t)x.nz * x.M;
  x.P = (size_t)x.nx * x.ny * x.nz;
  x.mixed = c.precision == TG_PREC_MIXED;
  // mixed precision: the dense solves on the int8-slice tensor-core product
  x.zsolver = x.mixed ? TG_ZSOLVER_ISLICE : TG_ZSOLVER_DMMA;
  x.isl_err = x.dalloc<int>(1);
  x.scalar = c.nphase > 1;
  x.opentop = std::fabs(c.bc_u[2] - 0) <= kSmall && std::fabs(c.bc_u[3] - 1) <= kSmall;  // boundary.cc:59-71
  x.dt = c.dt;
  x.olddt = c.dt;
  TG_CUDA(cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking));
  x.own_stream = true;
  zgemm_init();
  fft_init();

  // grids (src/domain.cc:304-332) and operators (stepper_space_chebyshev.cc)
  chebyshev_operators(x.nz, c.mapping, c.mapping_coef, x.gridz, x.D1h, x.D2h, x.gridzc);
  {
    std::vector<double> gx(x.nx), gy(x.ny);
    for (int i = 0; i < x.nx; ++i) gx[i] = c.lx / x.nx * i;
    for (int i = 0; i < x.ny; ++i) gy[i] = c.ly / x.ny * i;
    x.lmx = c.lx;
    for (int i = 0; i + 1 < x.nx; ++i) x.lmx = std::min(x.lmx, gx[i + 1] - gx[i]);
    x.lmy = c.ly;
    for (int i = 0; i + 1 < x.ny; ++i) x.lmy = std::min(x.lmy, gy[i + 1] - gy[i]);
    const std::vector<double>& g = x.gridzc;
    x.gridlenz.assign(x.nz, 0.0);
    for (int k = 0; k < x.nz; ++k) {
      if (k == 0)
        x.gridlenz[k] = (g[1] - g[0]) / 2;
      else if (k == x.nz - 1)
        x.gridlenz[k] = (g[x.nz - 1] - g[x.nz - 2]) / 2;
      else
        x.gridlenz[k] = std::min(g[k + 1] - g[k], g[k] - g[k - 1]);
    }
  }
  // wavenumbers per column m = iy + nyc*ix (src/stepper_space.cc:196-213)
  {
    const double pi = 3.141592653589793238462643383279502884;
    const double kx1 = 2 * pi / c.lx, ky1 = 2 * pi / c.ly;
    std::vector<double> kx(x.M), ky(x.M), dx2(x.M), dy2(x.M), k2(x.M);
    for (int ix = 0; ix < x.nxh; ++ix)
      for (int iy = 0; iy < x.nyc; ++iy) {
        const int m = iy + x.nyc * ix;
        double kxn = kx1 * (ix - 0);
        double kym = (iy <= x.nyc / 2) ? +ky1 * (iy - 0) : -ky1 * (x.nyc - iy);
        kx[m] = kxn;
        ky[m] = kym;
        dx2[m] = -std::pow(kxn, 2);
        dy2[m] = -std::pow(kym, 2);
        k2[m] = dx2[m] + dy2[m];
      }
    std::vector<int> yidx(x.nyc);
    const int h = x.nyc / 2;
    for (int iy = 0; iy < x.nyc; ++iy) yidx[iy] = iy < h ? iy : x.ny - (x.nyc - iy);
    x.kx = x.dalloc<double>(x.M);
    x.ky = x.dalloc<double>(x.M);
    x.dx2 = x.dalloc<double>(x.M);
    x.dy2 = x.dalloc<double>(x.M);
    x.k2 = x.dalloc<double>(x.M);
    x.yidx = x.dalloc<int>(x.nyc);
    TG_CUDA(cudaMemcpy(x.kx, kx.data(), sizeof(double) * x.M, cudaMemcpyHostToDevice));
    TG_CUDA(cudaMemcpy(x.ky, ky.data(), sizeof(double) * x.M, cudaMemcpyHostToDevice));
    TG_CUDA(cudaMemcpy(x.dx2, dx2.data(), sizeof(double) * x.M, cudaMemcpyHostToDevice));
    TG_CUDA(cudaMemcpy(x.dy2, dy2.data(), sizeof(double) * x.M, cudaMemcpyHostToDevice));
    TG_CUDA(cudaMemcpy(x.k2, k2.data(), sizeof(double) * x.M, cudaMemcpyHostToDevice));
    TG_CUDA(cudaMemcpy(x.yidx, yidx.data(), sizeof(int) * x.nyc, cudaMemcpyHostToDevice));
  }
  x.gz = x.dalloc<double>(x.nz);
  x.glz = x.dalloc<double>(x.nz);
  x.d1r0 = x.dalloc<double>(x.nz);
  x.d1rn = x.dalloc<double>(x.nz);
  TG_CUDA(cudaMemcpy(x.gz, x.gridz.data(), sizeof(double) * x.nz, cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(x.glz, x.gridlenz.data(), sizeof(double) * x.nz, cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(x.d1r0, x.D1h.data(), sizeof(double) * x.nz, cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(x.d1rn, x.D1h.data() + (size_t)(x.nz - 1) * x.nz, sizeof(double) * x.nz,
                     cudaMemcpyHostToDevice));

  // operators: dense copies, plus folded halves for the centro-(anti)symmetric
  // derivative matrices (the Chebyshev grid is symmetric about z = 0)
  zop_build(x.opD1, x.D1h, x.nz, true, allocator(x));
  zop_build(x.opD2, x.D2h, x.nz, true, allocator(x));
  // decompositions: u, v, w, p (phase_carrier_flat.cc:186-201), scalar (phase_scalar_flat.cc:186-200)
  const double* bcs[4] = {c.bc_u, c.bc_v, c.bc_w, c.bc_p};
  for (int s = 0; s < 3; ++s) x.sig_u[s] = -c.reynolds / c.dt / RK3[2][s];
  const int ndec = x.scalar ? 5 : 4;
  for (int w = 0; w < ndec; ++w) {
    double bc[4];
    if (w < 4) {
      for (int k = 0; k < 4; ++k) bc[k] = bcs[w][k];
    } else {
      const double rsw = c.reynolds * c.schmidt * c.settling;
      bc[0] = rsw * 10e6;   // BOUNDARY_COEF_SCALE, src/common.h:55
      bc[1] = 1 * 10e6;
      bc[2] = rsw * 10e6;
      bc[3] = 1 * 10e6;
      for (int s = 0; s < 3; ++s) x.sig_s[s] = -c.reynolds * c.schmidt / c.dt / RK3[2][s];
    }
    try {
      build_decomposition(x.nz, x.D1h, x.D2h, bc, x.dec[w]);
    } catch (std::exception& e) {
      throw Error{TG_ERR_SETUP, std::string("CmDz2DecompositionCplx::Construct > ") + e.what()};
    }
    install_decomposition(x, w);
  }

  // transforms
  fft_plan_create(x.px, x.nx);
  fft_plan_create(x.py, x.ny);
  x.td.nx = x.nx;
  x.td.ny = x.ny;
  x.td.nz = x.nz;
  x.td.nxh = x.nxh;
  x.td.nyc = x.nyc;
  x.td.M = x.M;
  x.td.yidx = x.yidx;

  // fields
  const size_t S = x.S, P = x.P;
  x.U = x.dalloc<double2>(3 * S);
  x.PR = x.dalloc<double2>(S);
  x.H = x.dalloc<double2>(3 * S);
  x.DP = x.dalloc<double2>(3 * S);
  x.SU = x.dalloc<double2>(3 * S);
  x.RHS = x.dalloc<double2>(3 * S);
  x.TMP = x.dalloc<double2>(3 * S);
  x.ADV = x.dalloc<double2>(3 * S);
  x.DU = x.dalloc<double2>(9 * S);
  x.F6 = x.dalloc<double2>(6 * S);
  x.REF = x.dalloc<double2>(3 * S);
  x.hist = x.dalloc<double2>(24 * (size_t)x.M);
  if (x.scalar) {
    x.PHI = x.dalloc<double2>(S);
    x.HPHI = x.dalloc<double2>(S);
    x.ADVPHI = x.dalloc<double2>(S);
    x.RHSPHI = x.dalloc<double2>(S);
    x.ero = x.dalloc<double2>(x.M);
  }
  const size_t ps = x.psize();
  x.UNL = x.dalloc<unsigned char>(3 * P * ps);
  x.DUP = x.dalloc<unsigned char>(9 * P * ps);
  x.PRD = x.dalloc<unsigned char>(6 * P * ps);
  x.PHIP = x.dalloc<unsigned char>(P * ps);
  x.PLN = x.dalloc<unsigned char>(3 * (size_t)x.nx * x.ny * ps);
  // whole-batch transforms (up to nine fields per launch pair): splitting a
  // batch so its intermediate stays in L2 measured slower (partial last waves)
  x.work_planes = 9 * x.nz;
  x.work = x.dalloc<double2>((size_t)x.work_planes * x.nxh * x.ny);
  x.PLN1 = x.PLN;
  if (x.scalar) {  // the scalar phase's own scratch for the overlapped Correct
    x.TMP_s = x.dalloc<double2>(3 * S);
    x.F6_s = x.dalloc<double2>(3 * S);
    x.PRD_s = x.dalloc<unsigned char>(3 * P * ps);
    x.DUP_s = x.dalloc<unsigned char>(3 * P * ps);
    x.work_s = x.dalloc<double2>((size_t)3 * x.nz * x.nxh * x.ny);
    x.PLN2 = x.dalloc<unsigned char>(3 * (size_t)x.nx * x.ny * ps);
    TG_CUDA(cudaStreamCreateWithFlags(&x.s2, cudaStreamNonBlocking));
    TG_CUDA(cudaEventCreateWithFlags(&x.cc_done, cudaEventDisableTiming));
    TG_CUDA(cudaEventCreateWithFlags(&x.sc_done, cudaEventDisableTiming));
  }
  x.feat = x.dalloc<double>(100);
  x.bits = x.dalloc<unsigned long long>(16);
  TG_CUDA(cudaMallocHost(&x.feat_h, 2 * 100 * sizeof(double)));
  std::memset(x.feat_h, 0, 2 * 100 * sizeof(double));
  TG_CUDA(cudaMallocHost(&x.err_h, 2 * sizeof(int)));
  x.err_h[0] = x.err_h[1] = 0;
  x.force_d = x.dalloc<double>(2);
  TG_CUDA(cudaMallocHost(&x.force_h, 4 * sizeof(double)));
  std::memset(x.force_h, 0, 4 * sizeof(double));
  TG_CUDA(cudaEventCreateWithFlags(&x.fev[0], cudaEventDisableTiming));
  TG_CUDA(cudaEventCreateWithFlags(&x.fev[1], cudaEventDisableTiming));
  TG_CUDA(cudaStreamCreateWithFlags(&x.s3, cudaStreamNonBlocking));
  TG_CUDA(cudaEventCreateWithFlags(&x.w_fork, cudaEventDisableTiming));
  TG_CUDA(cudaEventCreateWithFlags(&x.w_join, cudaEventDisableTiming));
  return px.release();
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static void gemm(Ctx& x, const ZOperator& A, const double2* in, long long sin, double2* out, long long sout,
                 int batch, EpiParams ep) {
  ep.nz = x.nz;
  ep.M = x.M;
  zgemm(A, in, sin, out, sout, x.M, batch, ep, x.s);
}

template <typename T>
static void fwd(Ctx& x, const void* phys, double2* spec, int planes) {
  for (int p0 = 0; p0 < planes; p0 += x.work_planes) {
    int np = std::min(planes - p0, x.work_planes);
    dft_forward<T>(x.td, x.px, x.py, (const T*)phys + (size_t)p0 * x.nx * x.ny, spec + (size_t)p0 * x.M, np,
                   x.work, x.s);
  }
}
template <typename T>
static void bwd(Ctx& x, const double2* spec, void* phys, int planes) {
  for (int p0 = 0; p0 < planes; p0 += x.work_planes) {
    int np = std::min(planes - p0, x.work_planes);
    dft_backward<T>(x.td, x.px, x.py, spec + (size_t)p0 * x.M, (T*)phys + (size_t)p0 * x.nx * x.ny, np, x.work,
                    x.s);
  }
}

// Backward transforms of ncomp groups of three gradient fields (spectral
// sources, x/y derivatives formed on load) reduced on the x pass to the
// advection terms (u+su) d/dx + (v+sv) d/dy + (w+sw) d/dz of each group; false
// when the grid or the scratch does not allow it.
template <typename T>
static bool bwd_advection(Ctx& x, const double2* const* src, const int* deriv, int ncomp, const T* unl, T* out,
                          double su, double sv, double sw) {
  const int nf = 3 * ncomp;
  if (nf * x.nz > x.work_planes || !dft_backward_adv_ok<T>(x.td, x.px, x.py, unl, out)) return false;
  SpecGather g{};
  for (int f = 0; f < nf; ++f) {
    g.src[f] = src[f];
    g.deriv[f] = deriv[f];
  }
  g.kx = x.kx;
  g.ky = x.ky;
  g.nf = nf;
  g.plane0 = 0;
  dft_backward_adv<T>(x.td, x.px, x.py, g, ncomp, unl, out, su, sv, sw, x.work, x.s);
  return true;
}

// Forward transform of nf products a[f] * (b[f] + sh[f]) of physical fields,
// formed as the x pass loads its rows (one launch pair); false when the grid or
// the scratch does not allow it (the caller then forms the products itself).
template <typename T>
static bool fwd_products(Ctx& x, const PhysProduct& pp, double2* spec) {
  if (pp.nf * x.nz > x.work_planes || !dft_forward_products_ok<T>(x.td, x.px, pp)) return false;
  dft_forward<T>(x.td, x.px, x.py, nullptr, spec, pp.nf * x.nz, x.work, x.s, &pp);
  return true;
}

// Backward transforms of nf fields gathered from their own spectral sources,
// the x and y derivatives (deriv 1, 2) formed as the coefficients are loaded:
// the spectral derivative fields are never written.
template <typename T>
static void bwd_gather(Ctx& x, const double2* const* src, const int* deriv, int nf, void* phys) {
  if (nf < 1 || nf > kMaxGather) throw Error{TG_ERR_ARG, "bwd_gather > bad field count"};
  SpecGather g{};
  for (int f = 0; f < nf; ++f) {
    g.src[f] = src[f];
    g.deriv[f] = deriv[f];
  }
  g.kx = x.kx;
  g.ky = x.ky;
  g.nf = nf;
  const int planes = nf * x.nz;
  for (int p0 = 0; p0 < planes; p0 += x.work_planes) {
    const int np = std::min(planes - p0, x.work_planes);
    g.plane0 = p0;
    dft_backward<T>(x.td, x.px, x.py, nullptr, (T*)phys + (size_t)p0 * x.nx * x.ny, np, x.work, x.s, &g);
  }
}

// driving force of the mean mode (src/phase_carrier_flat.cc:365-501)
static void mean_force(const Ctx& x, double& f1, double& f2) {
  const tg_case& c = x.c;
  const double dt = x.dt, t = x.time;
  const double tt = c.output_based_on_step ? t - dt / 2 : t + dt / 2;
  f1 = f2 = 0;
  const int* fd = c.force_direction;
  const double* fa = c.force_amplitude;
  switch (c.force_type) {
    case 0:
      break;
    case 1:
      if (fd[0] == 1) f1 = fa[0];
      if (fd[0] == 2) f2 = fa[0];
      break;
    case 2: {
      double a = fa[1];
      if (fd[1] == 1) f1 = a * std::cos(a * tt);
      if (fd[1] == 2) f2 = a * std::cos(a * tt);
    } break;
    case 3: {
      if (fd[0] == 1) f1 = fa[0];
      if (fd[0] == 2) f2 = fa[0];
      double a = fa[1];
      if (fd[1] == 1) f1 = f1 + a * std::cos(a * tt);
      if (fd[1] == 2) f2 = f2 + a * std::cos(a * tt);
    } break;
    case 4: {
      if (fd[0] == 1) f1 = fa[0];
      if (fd[0] == 2) f2 = fa[0];
      double a = fa[1];
      const double T = fa[0], t0 = fa[1], lastp = fa[2], tarp = fa[3];
      const double damp = -std::log(tarp) / (lastp + 0.25) / T;
      double v = (a * std::cos(a * tt) - damp * std::sin(a * tt)) * std::exp(-damp * (t - t0));
      if (fd[1] == 1) f1 = f1 + v;
      if (fd[1] == 2) f2 = f2 + v;
    } break;
    default:
      throw Error{TG_ERR_ARG, "FlatCarrierPhase::Predict() > Not Supported Force Type!"};
  }
}

// ---------------------------------------------------------------------------
// FlatCarrierPhase::Predict
// ---------------------------------------------------------------------------
template <typename T>
static void carrier_predict(Ctx& x, int stage) {
  const double dt = x.dt, c1 = RK3[0][stage], c2 = RK3[1][stage], c3 = RK3[2][stage];
  const size_t S = x.S, P = x.P;
  T* unl = (T*)x.UNL;
  T* prd = (T*)x.PRD;
  T* dup = (T*)x.DUP;
  auto grad_u = [&]() {  // SpaceStepper::Gradient(uvw, d*dxyz, i) for i = 0..2: d/dz here, d/dx and d/dy
    gemm(x, x.opD1, x.U, S, x.DU + 2 * S, 3 * S, 3, EpiParams());   // are formed by the transform's loads
  };
  // NonlinearVelocity (phase_carrier_flat.cc:716-813)
  if (x.alternation) {
    {  // the six products u_i u_j, formed as the forward transform loads its rows
      PhysProduct pp{};
      const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
      for (int f = 0; f < 6; ++f) {
        pp.a[f] = unl + ia[f] * P;
        pp.b[f] = unl + ib[f] * P;
        pp.sh[f] = 0.0;
      }
      pp.nf = 6;
      if (!fwd_products<T>(x, pp, x.F6)) {
        products6<T>(unl, prd, P, x.s);
        fwd<T>(x, prd, x.F6, 6 * x.nz);
      }
    }
    // adv_i = d/dx(u_i u) + d/dy(u_i v) + d/dz(u_i w): GradientTmp + sum
    const int inI[3] = {2, 4, 5}, x0I[3] = {0, 1, 2}, x1I[3] = {1, 3, 4};
    ZProblem pr[3];
    for (int i = 0; i < 3; ++i) {
      EpiParams ep;
      ep.mode = EPI_DIV;
      ep.kx = x.kx;
      ep.ky = x.ky;
      ep.X0 = x.F6 + x0I[i] * S;
      ep.X1 = x.F6 + x1I[i] * S;
      ep.s = 1.0;
      pr[i] = ZProblem{&x.opD1, x.F6 + inI[i] * S, (long long)S, x.ADV + i * S, (long long)S, 1, ep};
    }
    zgemm_group(pr, 3, x.M, x.s);
    // only the wall rows of du_i/dz are read in this form
    wall_dz(x.U, x.DU, S, x.M, x.nz, x.d1r0, x.d1rn, x.s);
  } else {
    grad_u();
    const double2* src[9];
    int der[9];
    for (int i = 0; i < 3; ++i) {  // field 3i+j: d u_i / d x_j
      src[3 * i + 0] = src[3 * i + 1] = x.U + i * S;
      der[3 * i + 0] = 1;
      der[3 * i + 1] = 2;
      src[3 * i + 2] = x.DU + (3 * i + 2) * S;
      der[3 * i + 2] = 0;
    }
    if (!bwd_advection<T>(x, src, der, 3, unl, prd, 0.0, 0.0, 0.0)) {
      bwd_gather<T>(x, src, der, 9, dup);
      adv_products<T>(unl, dup, prd, P, 3, 0.0, 0.0, 0.0, x.s);
    }
    fwd<T>(x, prd, x.ADV, 3 * x.nz);
  }
  if (x.scalar && x.c.scalar_bc == 1) {
    // bottom plane of du/dz, dv/dz in physical space for the erosion flux
    // (one gathered transform of the two planes: the gather takes plane f of
    // its sources as field f when the dimensions say one plane per field)
    SpecGather g{};
    g.src[0] = x.DU + 2 * S;
    g.src[1] = x.DU + 5 * S;
    g.kx = x.kx;
    g.ky = x.ky;
    g.nf = 2;
    TransformDims d1 = x.td;
    d1.nz = 1;
    dft_backward<T>(d1, x.px, x.py, nullptr, (T*)x.PLN, 2, x.work, x.s, &g);
  }
  // H = c1 H - dt adv; buoyancy; mean-mode force
  double bcoef = 0.0;
  const double2* phi = nullptr;
  if (x.scalar && x.c.affected_by_scalar) {
    bcoef = dt * x.c.averaged_concentration / std::pow(x.c.froude, 2) * (x.c.specific_gravity - 1);
    phi = x.PHI;
  }
  double f1, f2;
  mean_force(x, f1, f2);
  // The buoyancy term needs phi from the previous stage's scalar Correct
  // (possibly still running on the second stream): it is added after the
  // right-hand side, just before the solves of the components it enters, so
  // that the H update, the Laplacian and the u/v solves do not wait for it.
  h_update(x.H, x.ADV, nullptr, S, x.M, c1, dt, 0.0, 0.0, 0.0, 0, dt * f1, dt * f2,
           x.capturing ? x.force_d : nullptr, x.s);
  // Laplacian and rhs (phase_carrier_flat.cc:517-536)
  {
    const double redtc3 = -x.c.reynolds / dt / c3;
    EpiParams ep;
    ep.mode = EPI_LAPRHS;
    ep.H = x.H;
    ep.sH = S;
    ep.U = x.U;
    ep.sU = S;
    ep.dx2 = x.dx2;
    ep.dy2 = x.dy2;
    ep.a = redtc3;
    ep.c2 = c2;
    gemm(x, x.opD2, x.U, S, x.RHS, S, 3, ep);
  }
  // FlatCarrierBoundary::Apply (boundary_carrier_flat.cc:185-246) + top mean values
  {
    const double c3m0 = RK3[2][stage], c3m1 = RK3[2][(stage + 2) % 3], c3m2 = RK3[2][(stage + 1) % 3];
    double xm0 = 0, xm1 = 0, xm2 = 0;
    switch (stage) {
      case 0:
        xm0 = 2 * (0 + c3m0) * dt;
        xm1 = 0;
        xm2 = 2 * (0 - c3m1) * x.olddt;
        break;
      case 1:
        xm0 = 2 * (c3m0 + c3m1 + 0) * dt;
        xm1 = 2 * (0 + c3m1 + 0) * dt;
        xm2 = 0;
        break;
      default:
        xm0 = 2 * (c3m0 + c3m1 + c3m2) * dt;
        xm1 = 2 * (0 + c3m1 + c3m2) * dt;
        xm2 = 2 * (0 + +0 + c3m2) * dt;
        break;
    }
    const double r = (xm0 - xm1) / (xm1 - xm2);
    boundary_apply(x.RHS, x.hist, S, x.M, x.nz, 2 * dt * c3m0, r, x.opentop ? 1 : 0, x.c.bc_u[4], x.c.bc_v[4],
                   x.c.bc_w[4], x.s);
  }
  // Helmholtz, predict branch (phase_carrier_flat.cc:861-931): the three
  // components' E^-1 products in one launch, then their E products
  {
    ZProblem fwd[3], bwd[3];
    for (int i = 0; i < 3; ++i) {
      EpiParams ep;
      ep.mode = EPI_RSCALE;
      ep.lam = x.lamd[i];
      ep.k2 = x.k2;
      ep.sigma = x.sig_u[stage];
      ep.null_mode = std::fabs(ep.sigma) < kSmall;
      fwd[i] = ZProblem{&x.opEinv[i], x.RHS + i * S, (long long)S, x.TMP + i * S, (long long)S, 1, ep};
      bwd[i] = ZProblem{&x.opE[i], x.TMP + i * S, (long long)S, x.SU + i * S, (long long)S, 1, EpiParams()};
    }
    // buoyancy: w always (-cos of the slope), u or v along a sloped bed (+sin)
    const int sdir = x.c.slope_direction;
    const double ac2 = (-x.c.reynolds / dt / c3) * c2;   // coefficient of H in the rhs
    auto add_buoyancy = [&](int c, cudaStream_t st) {
      if (!phi) return;
      if (c == 2)
        buoyancy(x.H + 2 * S, x.RHS + 2 * S, phi, x.M, x.nz, bcoef, std::cos(x.c.slope), -1, ac2, st);
      else if ((sdir == 1 && c == 0) || (sdir == 2 && c == 1))
        buoyancy(x.H + c * S, x.RHS + c * S, phi, x.M, x.nz, bcoef, std::sin(x.c.slope), +1, ac2, st);
    };
    if (x.fork_active && x.opEinv[2].sym && x.opE[2].sym) {
      TG_CUDA(cudaEventRecord(x.w_fork, x.s));
      TG_CUDA(cudaStreamWaitEvent(x.s3, x.w_fork, 0));
      if (x.sc_pending) TG_CUDA(cudaStreamWaitEvent(x.s3, x.sc_done, 0));
      add_buoyancy(2, x.s3);
      zgemm_group(&fwd[2], 1, x.M, x.s3);
      zgemm_group(&bwd[2], 1, x.M, x.s3);
      TG_CUDA(cudaEventRecord(x.w_join, x.s3));
      if (phi && sdir != 0) {  // a sloped bed: u or v waits for phi too
        if (x.sc_pending) TG_CUDA(cudaStreamWaitEvent(x.s, x.sc_done, 0));
        add_buoyancy(0, x.s);
        add_buoyancy(1, x.s);
      }
      zgemm_group(fwd, 2, x.M, x.s);
      zgemm_group(bwd, 2, x.M, x.s);
      TG_CUDA(cudaStreamWaitEvent(x.s, x.w_join, 0));   // also after the scalar Correct
      x.sc_pending = false;
    } else {
      if (x.sc_pending) {
        TG_CUDA(cudaStreamWaitEvent(x.s, x.sc_done, 0));
        x.sc_pending = false;
      }
      for (int c = 0; c < 3; ++c) add_buoyancy(c, x.s);
      zgemm_group(fwd, 3, x.M, x.s);
      zgemm_group(bwd, 3, x.M, x.s);
    }
  }
}

// ---------------------------------------------------------------------------
// FlatCarrierPhase::Correct
// ---------------------------------------------------------------------------
template <typename T>
static void carrier_correct(Ctx& x, int stage) {
  const double dt = x.dt, c3 = RK3[2][stage];
  const size_t S = x.S;
  {  // divergence of u* and pressure rhs (phase_carrier_flat.cc:586-589)
    EpiParams ep;
    ep.mode = EPI_DIV;
    ep.kx = x.kx;
    ep.ky = x.ky;
    ep.X0 = x.SU;
    ep.X1 = x.SU + S;
    ep.s = 0.5 / dt / c3;
    gemm(x, x.opD1, x.SU + 2 * S, S, x.TMP, S, 1, ep);
  }
  {  // Helmholtz, correction branch (phase_carrier_flat.cc:933-987)
    EpiParams ep;
    ep.mode = EPI_RSCALE;
    ep.lam = x.lamd[3];
    ep.k2 = x.k2;
    ep.sigma = 0.0;
    ep.null_mode = 1;
    gemm(x, x.opEinv[3], x.TMP, S, x.TMP + S, S, 1, ep);
    gemm(x, x.opE[3], x.TMP + S, S, x.PR, S, 1, EpiParams());
  }
  // grad p (phase_carrier_flat.cc:597): dp/dz here; dp/dx, dp/dy = i kx p, i ky p
  // are formed from p by the two kernels that read them
  gemm(x, x.opD1, x.PR, S, x.DP + 2 * S, S, 1, EpiParams());
  if (stage == 2) x.olddt = dt;   // boundary_carrier_flat.cc:140-142
  boundary_update(x.hist, x.PR, x.DP + 2 * S, x.M, x.nz, x.opentop ? 1 : 0, x.kx, x.ky, x.d1r0, x.d1rn, x.s);
  project(x.U, x.SU, x.PR, x.DP + 2 * S, S, x.M, x.kx, x.ky, 2 * dt * c3, x.s);
  bwd<T>(x, x.U, x.UNL, 3 * x.nz);
  if (stage == 2)
    features<T>((const T*)x.UNL, x.nx, x.ny, x.nz, x.glz, x.lmx, x.lmy, x.bits, x.feat, x.DU, S, x.M, x.s);
}

// ---------------------------------------------------------------------------
// FlatScalarPhase::Predict / Correct
// ---------------------------------------------------------------------------
static void scalar_predict(Ctx& x, int) {
  // u_phi = u with the settling shift of the mean mode (phase_scalar_flat.cc:258-279);
  // its physical field is the carrier's plus this constant.
  const tg_case& c = x.c;
  x.shift[0] = x.shift[1] = 0.0;
  if (c.slope_direction == 1) x.shift[0] = c.settling * std::sin(c.slope);
  if (c.slope_direction == 2) x.shift[1] = c.settling * std::sin(c.slope);
  x.shift[2] = -(c.settling * std::cos(c.slope));
}

template <typename T>
static void scalar_correct(Ctx& x, int stage) {
  const tg_case& c = x.c;
  const double dt = x.dt, c1 = RK3[0][stage], c2 = RK3[1][stage], c3 = RK3[2][stage];
  const size_t S = x.S, P = x.P, pl = (size_t)x.nx * x.ny;
  T* unl = (T*)x.UNL;
  T* prd = (T*)x.PRD;
  T* dup = (T*)x.DUP;
  T* phip = (T*)x.PHIP;
  T* pln = (T*)x.PLN;
  const double s0 = x.shift[0], s1 = x.shift[1], s2 = x.shift[2];
  // NonlinearPressure (phase_scalar_flat.cc:552-599)
  if (x.alternation) {
    bwd<T>(x, x.PHI, phip, x.nz);
    PhysProduct pp{};  // phi (u_j + shift_j), formed as the forward transform loads its rows
    const double shj[3] = {s0, s1, s2};
    for (int f = 0; f < 3; ++f) {
      pp.a[f] = phip;
      pp.b[f] = unl + f * P;
      pp.sh[f] = shj[f];
    }
    pp.nf = 3;
    if (!fwd_products<T>(x, pp, x.F6)) {
      phi_products<T>(phip, unl, prd, P, s0, s1, s2, x.s);
      fwd<T>(x, prd, x.F6, 3 * x.nz);
    }
    EpiParams ep;
    ep.mode = EPI_DIV;
    ep.kx = x.kx;
    ep.ky = x.ky;
    ep.X0 = x.F6;
    ep.X1 = x.F6 + S;
    ep.s = 1.0;
    gemm(x, x.opD1, x.F6 + 2 * S, S, x.ADVPHI, S, 1, ep);
  } else {
    gemm(x, x.opD1, x.PHI, S, x.TMP + 2 * S, S, 1, EpiParams());   // d(phi)/dz; x and y on load
    const double2* src[3] = {x.PHI, x.PHI, x.TMP + 2 * S};
    const int der[3] = {1, 2, 0};
    if (!bwd_advection<T>(x, src, der, 1, unl, prd, s0, s1, s2)) {
      bwd_gather<T>(x, src, der, 3, dup);
      adv_products<T>(unl, dup, prd, P, 1, s0, s1, s2, x.s);
    }
    fwd<T>(x, prd, x.ADVPHI, x.nz);
  }
  axmby(x.HPHI, x.ADVPHI, S, c1, dt, x.s);
  {  // lap phi and rhs (phase_scalar_flat.cc:313-329)
    const double redtc3 = -c.reynolds * c.schmidt / dt / c3;
    EpiParams ep;
    ep.mode = EPI_LAPRHS;
    ep.H = x.HPHI;
    ep.U = x.PHI;
    ep.dx2 = x.dx2;
    ep.dy2 = x.dy2;
    ep.a = redtc3;
    ep.c2 = c2;
    gemm(x, x.opD2, x.PHI, S, x.RHSPHI, S, 1, ep);
  }
  zero_rows(x.RHSPHI, x.M, x.nz, x.s);   // FlatScalarBoundary::Apply
  if (c.scalar_bc == 1) {                 // erosion / deposition row (phase_scalar_flat.cc:340-384)
    erosion_tau<T>(pln, pln + pl, pln + 2 * pl, pl, c.reynolds, c.critical_shear, c.erosion_rate, x.s);
    fwd<T>(x, pln + 2 * pl, x.ero, 1);
    erosion_row(x.RHSPHI, x.ero, x.PHI, x.M, c.settling * std::cos(c.slope), c.averaged_concentration,
                c.reynolds * c.schmidt, x.feat, x.s);
  }
  {  // Helmholtz (phase_scalar_flat.cc:635-667)
    EpiParams ep;
    ep.mode = EPI_RSCALE;
    ep.lam = x.lamd[4];
    ep.k2 = x.k2;
    ep.sigma = x.sig_s[stage];
    ep.null_mode = std::fabs(ep.sigma) < kSmall;
    gemm(x, x.opEinv[4], x.RHSPHI, S, x.TMP, S, 1, ep);
    gemm(x, x.opE[4], x.TMP, S, x.PHI, S, 1, EpiParams());
  }
  // Bartnicki positivity filter (phase_scalar_flat.cc:419-478)
  bwd<T>(x, x.PHI, phip, x.nz);
  positivity_filter<T>(phip, (int)pl, x.nz, x.s);
  fwd<T>(x, phip, x.PHI, x.nz);
  trapz_mean(x.PHI, x.M, x.nz, x.gz, 0.0, x.feat, 21, x.s);
  if (stage == 2 && c.slope_direction > 0) {
    trapz_mean(x.U, x.M, x.nz, x.gz, s0, x.feat, 22, x.s);
    trapz_mean(x.U + S, x.M, x.nz, x.gz, s1, x.feat, 24, x.s);
    set_feat(x.feat, 23, 0.0, x.s);
    set_feat(x.feat, 25, 0.0, x.s);
    if (x.step % 10 == 0) {
      mul_shift<T>(phip, unl, prd, P, s0, x.s);
      fwd<T>(x, prd, x.TMP, x.nz);
      trapz_mean(x.TMP, x.M, x.nz, x.gz, 0.0, x.feat, 23, x.s);
      mul_shift<T>(phip, unl + P, prd, P, s1, x.s);
      fwd<T>(x, prd, x.TMP, x.nz);
      trapz_mean(x.TMP, x.M, x.nz, x.gz, 0.0, x.feat, 25, x.s);
    }
  }
}

template <typename T>
static void run_stage(Ctx& x, int stage) {
  const bool ov = x.overlap_active && x.scalar;
  if (ov) x.PLN = (stage & 1) ? x.PLN2 : x.PLN1;  // erosion planes of this stage
  carrier_predict<T>(x, stage);
  carrier_correct<T>(x, stage);
  if (x.scalar) {
    scalar_predict(x, stage);
    if (!ov) {
      scalar_correct<T>(x, stage);
    } else {
      // fork: the scalar Correct on s2, in its own scratch fields
      TG_CUDA(cudaEventRecord(x.cc_done, x.s));
      TG_CUDA(cudaStreamWaitEvent(x.s2, x.cc_done, 0));
      cudaStream_t s1 = x.s;
      double2 *tmp = x.TMP, *f6 = x.F6;
      void *prd = x.PRD, *dup = x.DUP, *work = x.work;
      const int wp = x.work_planes;
      x.s = x.s2;
      x.TMP = x.TMP_s;
      x.F6 = x.F6_s;
      x.PRD = x.PRD_s;
      x.DUP = x.DUP_s;
      x.work = x.work_s;
      x.work_planes = 3 * x.nz;
      try {
        scalar_correct<T>(x, stage);
      } catch (...) {
        x.s = s1, x.TMP = tmp, x.F6 = f6, x.PRD = prd, x.DUP = dup, x.work = work, x.work_planes = wp;
        throw;
      }
      x.s = s1, x.TMP = tmp, x.F6 = f6, x.PRD = prd, x.DUP = dup, x.work = work, x.work_planes = wp;
      TG_CUDA(cudaEventRecord(x.sc_done, x.s2));
      x.sc_pending = true;
    }
  }
}

// After the last stage of a step: the second stream rejoins the first.
static void join_scalar(Ctx& x) {
  if (x.sc_pending) {
    TG_CUDA(cudaStreamWaitEvent(x.s, x.sc_done, 0));
    x.sc_pending = false;
  }
  x.PLN = x.PLN1;
}

static void upload_state(Ctx& x, const double* uvw, const double* p, const double* phi, int start_step) {
  const size_t S = x.S;
  TG_CUDA(cudaMemcpyAsync(x.REF, uvw, 3 * S * sizeof(double2), cudaMemcpyHostToDevice, x.s));
  ref_to_slab(x.REF, x.U, x.M, x.nz, 3, x.s);
  TG_CUDA(cudaMemcpyAsync(x.REF, p, S * sizeof(double2), cudaMemcpyHostToDevice, x.s));
  ref_to_slab(x.REF, x.PR, x.M, x.nz, 1, x.s);
  if (x.scalar) {
    if (!phi) throw Error{TG_ERR_ARG, "FlatScalarVariable::Load > phi is required when nphase == 2"};
    TG_CUDA(cudaMemcpyAsync(x.REF, phi, S * sizeof(double2), cudaMemcpyHostToDevice, x.s));
    ref_to_slab(x.REF, x.PHI, x.M, x.nz, 1, x.s);
    TG_CUDA(cudaMemsetAsync(x.HPHI, 0, S * sizeof(double2), x.s));
  }
  // FlatCarrierVariable::Configure: grad p (its z component; x and y are
  // formed from p where they are read), physical velocity; fresh registers
  gemm(x, x.opD1, x.PR, S, x.DP + 2 * S, S, 1, EpiParams());
  TG_CUDA(cudaMemsetAsync(x.H, 0, 3 * S * sizeof(double2), x.s));
  TG_CUDA(cudaMemsetAsync(x.hist, 0, 24 * (size_t)x.M * sizeof(double2), x.s));
  TG_CUDA(cudaMemsetAsync(x.DU, 0, 9 * S * sizeof(double2), x.s));
  TG_CUDA(cudaMemsetAsync(x.feat, 0, 100 * sizeof(double), x.s));
  if (x.mixed)
    bwd<float>(x, x.U, x.UNL, 3 * x.nz);
  else
    bwd<double>(x, x.U, x.UNL, 3 * x.nz);
  x.olddt = x.dt;
  x.step = std::max(0, start_step);
  x.time = x.step * x.dt;
  x.isforward = true;
  x.alternation = false;
  x.cfl = 0.0;
  std::memset(x.feat_h, 0, 2 * 100 * sizeof(double));
  x.loaded = true;
}

static void download_state(Ctx& x, double* uvw, double* p, double* phi) {
  const size_t S = x.S;
  slab_to_ref(x.U, x.REF, x.M, x.nz, 3, x.s);
  TG_CUDA(cudaMemcpyAsync(uvw, x.REF, 3 * S * sizeof(double2), cudaMemcpyDeviceToHost, x.s));
  TG_CUDA(cudaStreamSynchronize(x.s));
  slab_to_ref(x.PR, x.REF, x.M, x.nz, 1, x.s);
  TG_CUDA(cudaMemcpyAsync(p, x.REF, S * sizeof(double2), cudaMemcpyDeviceToHost, x.s));
  TG_CUDA(cudaStreamSynchronize(x.s));
  if (x.scalar && phi) {
    slab_to_ref(x.PHI, x.REF, x.M, x.nz, 1, x.s);
    TG_CUDA(cudaMemcpyAsync(phi, x.REF, S * sizeof(double2), cudaMemcpyDeviceToHost, x.s));
  }
  TG_CUDA(cudaStreamSynchronize(x.s));
}

// FlatChannelSolver::Execute loop body; the CFL guard of TimeStepper::Update
// for step n+1 uses the features of step n, read back while step n+1 runs.
// A whole step can be replayed from a graph when none of its kernel arguments
// changes from step to step except the forcing: a fixed dt (changing dt drops
// the graphs), no sloped bed (its flux features run every tenth step only),
// no active profiler, and a stream other than the legacy default stream.
static bool graph_eligible(const Ctx& x) {
  return x.graphs && x.c.slope_direction == 0 && !g_prof && x.s != nullptr;
}

template <typename T>
static void record_step(Ctx& x) {
  x.overlap_active = x.overlap && x.scalar && !g_prof;  // profiled steps run sequentially
  x.fork_active = x.overlap && !g_prof;
  try {
    for (int st = 0; st < 3; ++st) run_stage<T>(x, st);
    join_scalar(x);  // a captured step ends joined
  } catch (...) {
    x.overlap_active = x.fork_active = false;
    x.sc_pending = false;
    x.PLN = x.PLN1;
    throw;
  }
  x.overlap_active = x.fork_active = false;
}

static void run_step_graph(Ctx& x) {
  const int par = x.alternation ? 1 : 0;
  double f1, f2;
  mean_force(x, f1, f2);  // the same forcing for the three stages
  // this pinned slot was last read two steps ago, which has completed
  x.force_h[2 * par] = x.dt * f1;
  x.force_h[2 * par + 1] = x.dt * f2;
  if (!x.gexec[par]) {
    if (!x.cap_s) TG_CUDA(cudaStreamCreateWithFlags(&x.cap_s, cudaStreamNonBlocking));
    cudaStream_t user = x.s;
    x.s = x.cap_s;
    x.capturing = true;
    cudaGraph_t g = nullptr;
    try {
      TG_CUDA(cudaStreamBeginCapture(x.s, cudaStreamCaptureModeThreadLocal));
      TG_CUDA(cudaMemcpyAsync(x.force_d, x.force_h + 2 * par, 2 * sizeof(double), cudaMemcpyHostToDevice, x.s));
      if (x.mixed)
        record_step<float>(x);
      else
        record_step<double>(x);
      TG_CUDA(cudaStreamEndCapture(x.s, &g));
    } catch (...) {
      cudaGraph_t dead = nullptr;
      cudaStreamEndCapture(x.s, &dead);
      if (dead) cudaGraphDestroy(dead);
      x.s = user;
      x.capturing = false;
      throw;
    }
    x.s = user;
    x.capturing = false;
    size_t nn = 0;
    TG_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    TG_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    long long kernels = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      TG_CUDA(cudaGraphNodeGetType(nd, &t));
      if (t == cudaGraphNodeTypeKernel) ++kernels;
    }
    const cudaError_t e = cudaGraphInstantiate(&x.gexec[par], g, 0);
    cudaGraphDestroy(g);
    TG_CUDA(e);
    x.gkernels[par] = kernels;
    // the kernels recorded during capture were counted; they run with the launch below
    g_launches -= kernels;
  }
  TG_CUDA(cudaGraphLaunch(x.gexec[par], x.s));
  g_launches += x.gkernels[par];
}

// One step of the Execute loop body, enqueued: TimeStepper::Update's time
// advance, three stages of both phases, alternation flip, and the feature
// copy into pinned slot `slot`.
static void enqueue_step(Ctx& x, int slot) {
  x.step += 1;
  x.time = x.time + x.dt;
  if (graph_eligible(x)) {
    run_step_graph(x);
  } else {
    x.overlap_active = x.overlap && x.scalar && !g_prof;  // profiled steps run sequentially
    x.fork_active = x.overlap && !g_prof;
    try {
      if (x.mixed)
        for (int st = 0; st < 3; ++st) run_stage<float>(x, st);
      else
        for (int st = 0; st < 3; ++st) run_stage<double>(x, st);
      join_scalar(x);
    } catch (...) {
      x.overlap_active = x.fork_active = false;
      throw;
    }
    x.overlap_active = x.fork_active = false;
  }
  x.alternation = !x.alternation;
  TG_CUDA(cudaMemcpyAsync(x.feat_h + slot * 100, x.feat, 100 * sizeof(double), cudaMemcpyDeviceToHost, x.s));
  if (x.zsolver == TG_ZSOLVER_ISLICE)
    TG_CUDA(cudaMemcpyAsync(x.err_h + slot, x.isl_err, sizeof(int), cudaMemcpyDeviceToHost, x.s));
  TG_CUDA(cudaEventRecord(x.fev[slot], x.s));
}

// Per-case state of the pipelined step loop: the CFL guard of step k uses the
// features of step k-1, which are read only after step k has been enqueued.
struct StepLoop {
  int done = 0, pending = -1;
  double prev_f19 = 0.0;
};

// the int8-slice products of a step reported a bounded wait that gave up
static void check_islice_flag(const Ctx& x, int slot) {
  if (x.zsolver == TG_ZSOLVER_ISLICE && x.err_h[slot])
    throw Error{TG_ERR_TIMEOUT, "FlatCarrierPhase::Helmholtz > a bounded wait of the int8-slice product gave up"};
}

static void check_step(Ctx& x, StepLoop& L, int maxstep, double maxcfl) {
  bool fwd_flag = x.step < maxstep;
  if (L.pending >= 0) {
    TG_CUDA(cudaEventSynchronize(x.fev[L.pending]));
    L.prev_f19 = x.feat_h[L.pending * 100 + 50 + 19];
    check_islice_flag(x, L.pending);
  }
  x.cfl = L.prev_f19 * x.dt;
  if (!std::isfinite(L.prev_f19)) throw Error{TG_ERR_NAN, "TimeStepper::Update > non-finite CFL feature"};
  if (x.cfl > maxcfl) fwd_flag = false;
  x.isforward = fwd_flag;
  L.pending = L.done & 1;
  ++L.done;
}

static void finish_steps(Ctx& x, StepLoop& L, double* feat_out) {
  TG_CUDA(cudaStreamSynchronize(x.s));
  if (L.pending >= 0) {
    std::memcpy(x.feat_h + 100 * (L.pending ^ 1), x.feat_h + 100 * L.pending, 100 * sizeof(double));
    if (feat_out) std::memcpy(feat_out, x.feat_h + L.pending * 100 + 50, 50 * sizeof(double));
    check_islice_flag(x, L.pending);
    if (!std::isfinite(x.feat_h[L.pending * 100 + 50 + 19]))
      throw Error{TG_ERR_NAN, "FlatCarrierPhase::Correct > non-finite velocity features"};
  }
}

static int run_steps(Ctx& x, int nsteps, int maxstep, double maxcfl, double* feat_out) {
  if (!x.loaded) throw Error{TG_ERR_STATE, "FlatChannelSolver::Execute > state not loaded"};
  StepLoop L;
  L.prev_f19 = x.feat_h[50 + 19];
  for (int k = 0; k < nsteps && x.isforward; ++k) {
    enqueue_step(x, L.done & 1);
    check_step(x, L, maxstep, maxcfl);
  }
  finish_steps(x, L, feat_out);
  return L.done;
}

// Independent cases stepped together: each step of every case is enqueued on
// its own stream before the previous step's features of any case are awaited,
// so the cases' kernels (or step graphs) overlap on the GPU.
static void run_ensemble(std::vector<Ctx*>& xs, int nsteps, int maxstep, double maxcfl, int* done) {
  std::vector<StepLoop> L(xs.size());
  for (size_t i = 0; i < xs.size(); ++i) {
    if (!xs[i]->loaded) throw Error{TG_ERR_STATE, "FlatChannelSolver::Execute > state not loaded"};
    L[i].prev_f19 = xs[i]->feat_h[50 + 19];
  }
  for (int k = 0; k < nsteps; ++k) {
    bool any = false;
    std::vector<char> stepped(xs.size(), 0);
    for (size_t i = 0; i < xs.size(); ++i)
      if (xs[i]->isforward) {
        enqueue_step(*xs[i], L[i].done & 1);
        stepped[i] = 1;
        any = true;
      }
    if (!any) break;
    for (size_t i = 0; i < xs.size(); ++i)
      if (stepped[i]) check_step(*xs[i], L[i], maxstep, maxcfl);
  }
  for (size_t i = 0; i < xs.size(); ++i) {
    finish_steps(*xs[i], L[i], nullptr);
    if (done) done[i] = L[i].done;
  }
}

// ---------------------------------------------------------------------------
// row-tiling autotuner of the z-operator GEMMs
// ---------------------------------------------------------------------------
// The row tiling (m-tiles of 8 output rows per CTA) sets how often each CTA
// column re-reads its input from L2 against how evenly the grid fills the
// SMs; the best choice depends on Nz, M and the GPU.  The tuner times the
// store-epilogue product of three components for each distinct tiling of the
// dense and the folded kernel and keeps the fastest; the choice is cached in a
// flat JSON object {"<Nx>x<Ny>x<Nz>:<precision>:sm<cc>x<SMs>": [dense, folded]}
// of the two preferences (most m-tiles per CTA).
using TuneCache = std::map<std::string, std::pair<int, int>>;

static std::string tune_key(const Ctx& x) {
  int dev = 0;
  TG_CUDA(cudaGetDevice(&dev));
  int major = 0, minor = 0, sms = 0;
  TG_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  TG_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
  TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  char buf[128];
  snprintf(buf, sizeof buf, "%dx%dx%d:%s:sm%d%dx%d", x.nx, x.ny, x.nz, x.mixed ? "mixed" : "fp64", major, minor,
           sms);
  return buf;
}

static TuneCache read_tune_cache(const char* path) {
  TuneCache m;
  std::ifstream f(path);
  if (!f) return m;   // no cache yet
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string t = ss.str();
  const size_t a = t.find_first_not_of(" \t\r\n"), b = t.find_last_not_of(" \t\r\n");
  if (a != std::string::npos && (t[a] != '{' || t[b] != '}'))
    throw Error{TG_ERR_ARG, std::string("tg_autotune > ") + path + " is not a tiling cache"};
  static const std::regex entry("\"([^\"]+)\"\\s*:\\s*\\[\\s*(-?\\d+)\\s*,\\s*(-?\\d+)\\s*\\]");
  for (std::sregex_iterator it(t.begin(), t.end(), entry), end; it != end; ++it)
    m[(*it)[1].str()] = {std::stoi((*it)[2].str()), std::stoi((*it)[3].str())};
  return m;
}

static void write_tune_cache(const char* path, const TuneCache& m) {
  // whole file to a neighbour, then renamed over the cache: readers never
  // see a partial file
  const std::string tmp = std::string(path) + ".tmp" + std::to_string((long long)getpid());
  {
    std::ofstream f(tmp, std::ios::trunc);
    if (!f) throw Error{TG_ERR_ARG, std::string("tg_autotune > cannot write ") + tmp};
    f << "{\n";
    size_t i = 0;
    for (const auto& kv : m)
      f << "  \"" << kv.first << "\": [" << kv.second.first << ", " << kv.second.second << "]"
        << (++i < m.size() ? ",\n" : "\n");
    f << "}\n";
    if (!f) throw Error{TG_ERR_ARG, std::string("tg_autotune > cannot write ") + tmp};
  }
  if (std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    throw Error{TG_ERR_ARG, std::string("tg_autotune > cannot write ") + path};
  }
}

// device milliseconds of one launch: the least mean over three runs of five
static float time_gemm(Ctx& x, const ZOperator& op, const double2* in, double2* out, int batch) {
  cudaEvent_t a = nullptr, b = nullptr;
  TG_CUDA(cudaEventCreate(&a));
  TG_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  try {
    for (int w = 0; w < 2; ++w) gemm(x, op, in, x.S, out, x.S, batch, EpiParams());
    for (int r = 0; r < 3; ++r) {
      TG_CUDA(cudaEventRecord(a, x.s));
      for (int i = 0; i < 5; ++i) gemm(x, op, in, x.S, out, x.S, batch, EpiParams());
      TG_CUDA(cudaEventRecord(b, x.s));
      TG_CUDA(cudaEventSynchronize(b));
      float ms = 0.f;
      TG_CUDA(cudaEventElapsedTime(&ms, a, b));
      best = std::min(best, ms / 5);
    }
  } catch (...) {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    throw;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

// distinct tilings of `rows` rows, from the fewest row tiles up
static std::vector<int> tiling_candidates(int rows, int maxmt, int count) {
  std::vector<int> prefs;
  int last_tiles = -1;
  for (int p = maxmt; p >= 1 && (int)prefs.size() < count; --p) {
    int mt = 0, tiles = 0;
    row_tiling(rows, p, mt, tiles);
    if (tiles != last_tiles) prefs.push_back(p);
    last_tiles = tiles;
  }
  return prefs;
}

static void apply_tiling(Ctx& x, int pd, int ps) {
  zop_set_tiling(x.opD1, pd, ps);
  zop_set_tiling(x.opD2, pd, ps);
  zop_set_tiling(x.opTmp, pd, ps);
  for (int i = 0; i < 5; ++i) {
    zop_set_tiling(x.opEinv[i], pd, ps);
    zop_set_tiling(x.opE[i], pd, ps);
  }
  x.drop_graphs();   // the recorded launches carry the old grids
}

static void autotune(Ctx& x, const char* cache_path, int* tiling) {
  int maxd = 0, maxs = 0;
  zop_tiling_limits(maxd, maxs);
  const std::string key = tune_key(x);
  TuneCache cache;
  if (cache_path) cache = read_tune_cache(cache_path);
  int pd = 0, ps = 0;
  auto hit = cache.find(key);
  if (hit != cache.end()) {
    pd = hit->second.first;
    ps = hit->second.second;
    if (pd < 1 || pd > maxd || ps < 1 || ps > maxs)
      throw Error{TG_ERR_ARG, "tg_autotune > cache entry " + key + " out of range"};
  } else {
    TG_CUDA(cudaStreamSynchronize(x.s));
    if (x.s2) TG_CUDA(cudaStreamSynchronize(x.s2));
    if (x.s3) TG_CUDA(cudaStreamSynchronize(x.s3));
    Profiler* saved = g_prof;   // tuning launches stay out of a profiling window
    g_prof = nullptr;
    const size_t n = 3 * x.S;
    double2 *in = nullptr, *out = nullptr;
    cudaError_t e1 = cudaMalloc(&in, n * sizeof(double2));
    cudaError_t e2 = cudaMalloc(&out, n * sizeof(double2));
    try {
      if (e1 != cudaSuccess || e2 != cudaSuccess) {
        (void)cudaGetLastError();   // not left for the next launch check
        throw Error{TG_ERR_NOMEM, "tg_autotune > cudaMalloc"};
      }
      if (x.loaded)
        TG_CUDA(cudaMemcpyAsync(in, x.U, n * sizeof(double2), cudaMemcpyDeviceToDevice, x.s));
      else
        TG_CUDA(cudaMemsetAsync(in, 0x3f, n * sizeof(double2), x.s));   // finite non-zero values
      // the dense kernel on the dense copy of D1, the folded kernel on D1 itself
      ZOperator dense = x.opD1, folded = x.opD1;
      dense.sym = false;
      dense.split = 0;
      float best = 1e30f;
      for (int p : tiling_candidates(x.nz, maxd, 6)) {
        zop_set_tiling(dense, p, 0);
        const float ms = time_gemm(x, dense, in, out, 3);
        if (ms < best) best = ms, pd = p;
      }
      best = 1e30f;
      if (folded.sym) {
        for (int p : tiling_candidates(folded.rows, maxs, 4)) {
          zop_set_tiling(folded, 0, p);
          const float ms = time_gemm(x, folded, in, out, 3);
          if (ms < best) best = ms, ps = p;
        }
      } else {
        ps = maxs;   // no folded operator on this grid (even Nz)
      }
    } catch (...) {
      cudaFree(in);
      cudaFree(out);
      g_prof = saved;
      throw;
    }
    TG_CUDA(cudaFree(in));
    TG_CUDA(cudaFree(out));
    g_prof = saved;
    if (cache_path) {
      cache[key] = {pd, ps};
      write_tune_cache(cache_path, cache);
    }
  }
  apply_tiling(x, pd, ps);
  if (tiling) {
    int mt = 0, tiles = 0;
    row_tiling(x.nz, pd, mt, tiles);
    tiling[0] = mt;
    tiling[1] = tiles;
    row_tiling((x.nz - 1) / 2 + 1, ps, mt, tiles);
    tiling[2] = mt;
    tiling[3] = tiles;
  }
}

}  // namespace tg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace tg;

#define TG_TRY(...)                                          \
  try {                                                      \
    __VA_ARGS__;                                             \
    return TG_OK;                                            \
  } catch (const Error& e) {                                 \
    set_error(e.msg);                                        \
    return e.code;                                           \
  } catch (const std::exception& e) {                        \
    set_error(e.what());                                     \
    return TG_ERR_SETUP;                                     \
  }

#define TG_CHECK_CTX(x) \
  if (!(x)) { set_error("null context"); return TG_ERR_ARG; }

extern "C" {

const char* tg_last_error(void) { return g_err.c_str(); }
int tg_version(void) { return 1; }
long long tg_launch_count(void) { return g_launches; }

tg_status tg_create(const tg_case* c, tg_ctx** out) {
  if (!c || !out) {
    set_error("tg_create > null argument");
    return TG_ERR_ARG;
  }
  TG_TRY(*out = reinterpret_cast<tg_ctx*>(create(*c)));
}

tg_status tg_destroy(tg_ctx* ctx) {
  TG_CHECK_CTX(ctx);
  TG_TRY(delete reinterpret_cast<Ctx*>(ctx));
}

tg_status tg_get_dims(const tg_ctx* ctx, int dims[6]) {
  TG_CHECK_CTX(ctx);
  const Ctx& x = *reinterpret_cast<const Ctx*>(ctx);
  dims[0] = x.nx;
  dims[1] = x.ny;
  dims[2] = x.nz;
  dims[3] = x.nxh;
  dims[4] = x.nyc;
  dims[5] = x.M;
  return TG_OK;
}

tg_status tg_set_stream(tg_ctx* ctx, void* stream) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    if (x.own_stream) TG_CUDA(cudaStreamDestroy(x.s));
    x.s = reinterpret_cast<cudaStream_t>(stream);
    x.own_stream = false;
  });
}

tg_status tg_synchronize(tg_ctx* ctx) {
  TG_CHECK_CTX(ctx);
  TG_TRY(TG_CUDA(cudaStreamSynchronize(reinterpret_cast<Ctx*>(ctx)->s)));
}

tg_status tg_set_decomposition(tg_ctx* ctx, int which, const double* E, const double* Einv, const double* lam,
                               const double* fbb, const double* ftb, const double* fbf, const double* ftf) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (which < 0 || which > 4 || (which == 4 && !x.scalar) || !E || !Einv || !lam || !fbb || !ftb || !fbf || !ftf) {
    set_error("tg_set_decomposition > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    const size_t nn = (size_t)x.nz * x.nz;
    Decomposition& d = x.dec[which];
    d.n = x.nz;
    d.E.assign(E, E + nn);
    d.Einv.assign(Einv, Einv + nn);
    d.lam.assign(lam, lam + x.nz);
    d.fbb.assign(fbb, fbb + x.nz);
    d.ftb.assign(ftb, ftb + x.nz);
    d.fbf.assign(fbf, fbf + x.nz);
    d.ftf.assign(ftf, ftf + x.nz);
    d.parity = false;   // caller's eigenvectors: no parity order assumed, dense solve
    TG_CUDA(cudaStreamSynchronize(x.s));
    install_decomposition(x, which);
  });
}

tg_status tg_get_decomposition(const tg_ctx* ctx, int which, double* E, double* Einv, double* lam, double* fbb,
                               double* ftb, double* fbf, double* ftf) {
  TG_CHECK_CTX(ctx);
  const Ctx& x = *reinterpret_cast<const Ctx*>(ctx);
  if (which < 0 || which > 4 || (which == 4 && !x.scalar)) {
    set_error("tg_get_decomposition > bad argument");
    return TG_ERR_ARG;
  }
  const Decomposition& d = x.dec[which];
  auto cp = [](double* dst, const std::vector<double>& v) {
    if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
  };
  cp(E, d.E);
  cp(Einv, d.Einv);
  cp(lam, d.lam);
  cp(fbb, d.fbb);
  cp(ftb, d.ftb);
  cp(fbf, d.fbf);
  cp(ftf, d.ftf);
  return TG_OK;
}

tg_status tg_get_operators(const tg_ctx* ctx, double* D1, double* D2) {
  TG_CHECK_CTX(ctx);
  const Ctx& x = *reinterpret_cast<const Ctx*>(ctx);
  if (D1) std::memcpy(D1, x.D1h.data(), x.D1h.size() * sizeof(double));
  if (D2) std::memcpy(D2, x.D2h.data(), x.D2h.size() * sizeof(double));
  return TG_OK;
}

tg_status tg_operators_host(int nz, int mapping, double mapping_coef, double* D1, double* D2) {
  if (nz < 3 || !D1 || !D2) {
    set_error("tg_operators_host > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    std::vector<double> gz, d1, d2, gzc;
    chebyshev_operators(nz, mapping, mapping_coef, gz, d1, d2, gzc);
    std::memcpy(D1, d1.data(), d1.size() * sizeof(double));
    std::memcpy(D2, d2.data(), d2.size() * sizeof(double));
  });
}

tg_status tg_decomposition_host(int nz, int mapping, double mapping_coef, const double* bc, double* E, double* Einv,
                                double* lam, double* fbb, double* ftb, double* fbf, double* ftf) {
  if (nz < 3 || !bc) {
    set_error("tg_decomposition_host > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    std::vector<double> gz, d1, d2, gzc;
    chebyshev_operators(nz, mapping, mapping_coef, gz, d1, d2, gzc);
    Decomposition d;
    build_decomposition(nz, d1, d2, bc, d);
    auto cp = [](double* dst, const std::vector<double>& v) {
      if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    cp(E, d.E);
    cp(Einv, d.Einv);
    cp(lam, d.lam);
    cp(fbb, d.fbb);
    cp(ftb, d.ftb);
    cp(fbf, d.fbf);
    cp(ftf, d.ftf);
  });
}

tg_status tg_upload_state(tg_ctx* ctx, const double* uvw, const double* p, const double* phi, int start_step) {
  TG_CHECK_CTX(ctx);
  if (!uvw || !p) {
    set_error("FlatCarrierVariable::Load > null state pointer");
    return TG_ERR_ARG;
  }
  TG_TRY(upload_state(*reinterpret_cast<Ctx*>(ctx), uvw, p, phi, start_step));
}

tg_status tg_download_state(tg_ctx* ctx, double* uvw, double* p, double* phi) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!uvw || !p) {
    set_error("FlatCarrierVariable::Save > null state pointer");
    return TG_ERR_ARG;
  }
  if (!x.loaded) {
    set_error("FlatCarrierVariable::Save > state not loaded");
    return TG_ERR_STATE;
  }
  TG_TRY(download_state(x, uvw, p, phi));
}

tg_status tg_set_time(tg_ctx* ctx, int step, double time, double dt, int alternation) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!(dt > 0.0)) {
    set_error("TimeStepper::Update > dt must be positive");
    return TG_ERR_ARG;
  }
  if (dt != x.dt) {
    x.drop_graphs();  // dt is an argument of the recorded kernels
    // FlatCarrierPhase::Update / FlatScalarPhase::Update: the reciprocals of
    // the velocity and scalar solves follow dt (the GEMM epilogue forms them
    // from sigma); the pressure solve does not depend on dt
    x.dt = dt;
    for (int s = 0; s < 3; ++s) x.sig_u[s] = -x.c.reynolds / dt / RK3[2][s];
    if (x.scalar)
      for (int s = 0; s < 3; ++s) x.sig_s[s] = -x.c.reynolds * x.c.schmidt / dt / RK3[2][s];
  }
  x.step = step;
  x.time = time;
  x.alternation = alternation != 0;
  return TG_OK;
}

tg_status tg_get_time(const tg_ctx* ctx, int* step, double* time, double* dt, int* alternation, int* isforward,
                      double* cfl) {
  TG_CHECK_CTX(ctx);
  const Ctx& x = *reinterpret_cast<const Ctx*>(ctx);
  if (step) *step = x.step;
  if (time) *time = x.time;
  if (dt) *dt = x.dt;
  if (alternation) *alternation = x.alternation;
  if (isforward) *isforward = x.isforward;
  if (cfl) *cfl = x.cfl;
  return TG_OK;
}

#define TG_STAGE_CALL(fn_f32, fn_f64)                                     \
  TG_CHECK_CTX(ctx);                                                      \
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);                                  \
  if (stage < 0 || stage > 2) {                                           \
    set_error("Phase > stage must be 0, 1 or 2");                         \
    return TG_ERR_ARG;                                                    \
  }                                                                       \
  if (!x.loaded) {                                                        \
    set_error("Phase > state not loaded");                                \
    return TG_ERR_STATE;                                                  \
  }                                                                       \
  TG_TRY(if (x.mixed) fn_f32; else fn_f64;)

tg_status tg_carrier_predict(tg_ctx* ctx, int stage) {
  TG_STAGE_CALL(carrier_predict<float>(x, stage), carrier_predict<double>(x, stage));
}
tg_status tg_carrier_correct(tg_ctx* ctx, int stage) {
  TG_STAGE_CALL(carrier_correct<float>(x, stage), carrier_correct<double>(x, stage));
}
static bool has_scalar(tg_ctx* ctx) {
  if (ctx && reinterpret_cast<Ctx*>(ctx)->scalar) return true;
  set_error("FlatScalarPhase > case has no scalar phase");
  return false;
}
tg_status tg_scalar_predict(tg_ctx* ctx, int stage) {
  if (ctx && !has_scalar(ctx)) return TG_ERR_STATE;
  TG_STAGE_CALL(scalar_predict(x, stage), scalar_predict(x, stage));
}
tg_status tg_scalar_correct(tg_ctx* ctx, int stage) {
  if (ctx && !has_scalar(ctx)) return TG_ERR_STATE;
  TG_STAGE_CALL(scalar_correct<float>(x, stage), scalar_correct<double>(x, stage));
}

// FlatChannelPostprocessor::Execute (src/postprocessor_channel_flat.cc:195-236)
// for the current state: the velocity gradients (SpaceStepper::Gradient, the
// GEMM with the gradient epilogue), their FP64 c2r in chunks of z planes, and
// lambda_ci per point.
static void swirling_strength(Ctx& x, double* out_host) {
  if (!x.loaded) throw Error{TG_ERR_STATE, "FlatChannelPostprocessor::Execute > state not loaded"};
  const size_t S = x.S, plane = (size_t)x.nx * x.ny;
  if (!x.post_buf) {
    x.post_planes = std::min(x.nz, 16);
    x.post_buf = x.dalloc<double>(9 * (size_t)x.post_planes * plane);
    x.post_out = x.dalloc<double>(x.P);
  }
  EpiParams ep;
  ep.mode = EPI_GRAD;
  ep.kx = x.kx;
  ep.ky = x.ky;
  ep.X0 = x.U;
  ep.sX = S;
  ep.aux0 = x.DU;
  ep.aux1 = x.DU + S;
  ep.sAux = 3 * S;
  gemm(x, x.opD1, x.U, S, x.DU + 2 * S, 3 * S, 3, ep);
  const size_t fstride = (size_t)x.post_planes * plane;
  for (int z0 = 0; z0 < x.nz; z0 += x.post_planes) {
    const int np = std::min(x.post_planes, x.nz - z0);
    for (int f = 0; f < 9; ++f)
      dft_backward<double>(x.td, x.px, x.py, x.DU + (size_t)f * S + (size_t)z0 * x.M, x.post_buf + f * fstride, np,
                           x.work, x.s);
    swirling(x.post_buf, fstride, (size_t)np * plane, x.post_out + (size_t)z0 * plane, x.s);
  }
  TG_CUDA(cudaMemcpyAsync(out_host, x.post_out, x.P * sizeof(double), cudaMemcpyDeviceToHost, x.s));
  TG_CUDA(cudaStreamSynchronize(x.s));
}

tg_status tg_swirling_strength(tg_ctx* ctx, double* vortex) {
  TG_CHECK_CTX(ctx);
  if (!vortex) {
    set_error("FlatChannelPostprocessor::Execute > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY(swirling_strength(*reinterpret_cast<Ctx*>(ctx), vortex));
}

tg_status tg_set_graphs(tg_ctx* ctx, int enable) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  x.graphs = enable != 0;
  if (!x.graphs) x.drop_graphs();
  return TG_OK;
}

tg_status tg_autotune(tg_ctx* ctx, const char* cache_path, int* tiling) {
  TG_CHECK_CTX(ctx);
  TG_TRY(autotune(*reinterpret_cast<Ctx*>(ctx), cache_path, tiling));
}

tg_status tg_run_ensemble(tg_ctx** ctxs, int n, int nsteps, int maxstep, double maxcfl, int* done) {
  if (!ctxs || n < 1) {
    set_error("tg_run_ensemble > bad argument");
    return TG_ERR_ARG;
  }
  std::vector<Ctx*> xs(n);
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) {
      set_error("tg_run_ensemble > null context");
      return TG_ERR_ARG;
    }
    xs[i] = reinterpret_cast<Ctx*>(ctxs[i]);
  }
  TG_TRY(run_ensemble(xs, nsteps, maxstep, maxcfl, done));
}

tg_status tg_run_steps(tg_ctx* ctx, int nsteps, int maxstep, double maxcfl, double* features, int* done) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  int d = 0;
  tg_status st;
  try {
    d = run_steps(x, nsteps, maxstep, maxcfl, features);
    st = TG_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    st = e.code;
  }
  if (done) *done = d;
  return st;
}

tg_status tg_profile_begin(tg_ctx* ctx) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    x.prof.reset();
    g_prof = &x.prof;
  });
}

tg_status tg_profile_end(tg_ctx* ctx, int ncat, double* ms, double* bytes, double* flops, int* count) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  TG_TRY({
    g_prof = nullptr;
    TG_CUDA(cudaStreamSynchronize(x.s));
    for (int c = 0; c < ncat; ++c) {
      if (ms) ms[c] = 0;
      if (bytes) bytes[c] = 0;
      if (flops) flops[c] = 0;
      if (count) count[c] = 0;
    }
    for (double& v : x.prof.last_x) v = 0.0;
    for (auto& r : x.prof.recs) {
      if (r.cat >= 0 && r.cat < TG_PROF_NCAT) x.prof.last_x[r.cat] += r.xflops;
      if (r.cat < 0 || r.cat >= ncat) continue;
      float t = 0.f;
      TG_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
      if (ms) ms[r.cat] += t;
      if (bytes) bytes[r.cat] += r.bytes;
      if (flops) flops[r.cat] += r.flops;
      if (count) count[r.cat] += 1;
    }
    x.prof.reset();
  });
}

tg_status tg_profile_executed(const tg_ctx* ctx, int ncat, double* flops) {
  TG_CHECK_CTX(ctx);
  const Ctx& x = *reinterpret_cast<const Ctx*>(ctx);
  if (!flops || ncat < 0) {
    set_error("tg_profile_executed > bad argument");
    return TG_ERR_ARG;
  }
  for (int c = 0; c < ncat; ++c) flops[c] = c < TG_PROF_NCAT ? x.prof.last_x[c] : 0.0;
  return TG_OK;
}

tg_status tg_features(tg_ctx* ctx, double* out) {
  TG_CHECK_CTX(ctx);
  if (!out) {
    set_error("tg_features > null output");
    return TG_ERR_ARG;
  }
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  TG_TRY({
    TG_CUDA(cudaMemcpyAsync(x.feat_h, x.feat, 100 * sizeof(double), cudaMemcpyDeviceToHost, x.s));
    TG_CUDA(cudaStreamSynchronize(x.s));
    std::memcpy(out, x.feat_h + 50, 50 * sizeof(double));
  });
}

tg_status tg_dft_forward_f64(tg_ctx* ctx, const double* phys, double* spec, int dim) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!phys || !spec || dim < 1) {
    set_error("RealCplxCube::DftForward > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY(fwd<double>(x, phys, reinterpret_cast<double2*>(spec), dim * x.nz));
}
tg_status tg_dft_forward_f32(tg_ctx* ctx, const float* phys, double* spec, int dim) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!phys || !spec || dim < 1) {
    set_error("RealCplxCube::DftForward > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY(fwd<float>(x, phys, reinterpret_cast<double2*>(spec), dim * x.nz));
}
tg_status tg_dft_forward_planes(tg_ctx* ctx, const void* phys, double* spec, int planes, int fp32) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!phys || !spec || planes < 1) {
    set_error("RealCplxCube::DftForward > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    if (fp32)
      fwd<float>(x, phys, reinterpret_cast<double2*>(spec), planes);
    else
      fwd<double>(x, phys, reinterpret_cast<double2*>(spec), planes);
  });
}
tg_status tg_dft_backward_planes(tg_ctx* ctx, const double* spec, void* phys, int planes, int fp32) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!phys || !spec || planes < 1) {
    set_error("RealCplxCube::DftBackward > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    if (fp32)
      bwd<float>(x, reinterpret_cast<const double2*>(spec), phys, planes);
    else
      bwd<double>(x, reinterpret_cast<const double2*>(spec), phys, planes);
  });
}
tg_status tg_dft_backward_f64(tg_ctx* ctx, const double* spec, double* phys, int dim) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!phys || !spec || dim < 1) {
    set_error("RealCplxCube::DftBackward > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY(bwd<double>(x, reinterpret_cast<const double2*>(spec), phys, dim * x.nz));
}
tg_status tg_dft_backward_f32(tg_ctx* ctx, const double* spec, float* phys, int dim) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!phys || !spec || dim < 1) {
    set_error("RealCplxCube::DftBackward > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY(bwd<float>(x, reinterpret_cast<const double2*>(spec), phys, dim * x.nz));
}

tg_status tg_multiply(tg_ctx* ctx, const double* A_host, const double* in, double* out, int dim) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!A_host || !in || !out || dim < 1) {
    set_error("RealCplxCube::Multiply > bad argument");
    return TG_ERR_ARG;
  }
  if (in == out) {
    set_error("RealCplxCube::Multiply(cmat,RealCplxCube) > Can not Do In-place Multiplication!");
    return TG_ERR_ARG;
  }
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    std::vector<double> A(A_host, A_host + (size_t)x.nz * x.nz);
    zop_build(x.opTmp, A, x.nz, true, allocator(x));
    gemm(x, x.opTmp, reinterpret_cast<const double2*>(in), x.S, reinterpret_cast<double2*>(out), x.S, dim,
         EpiParams());
  });
}

tg_status tg_multiply_islice(tg_ctx* ctx, const double* A_host, const double* in, double* out, int dim) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!A_host || !in || !out || dim < 1) {
    set_error("RealCplxCube::Multiply > bad argument");
    return TG_ERR_ARG;
  }
  if (in == out) {
    set_error("RealCplxCube::Multiply(cmat,RealCplxCube) > Can not Do In-place Multiplication!");
    return TG_ERR_ARG;
  }
  if (x.nz - 2 > 256) {
    set_error("RealCplxCube::Multiply > the int8-slice product needs nz <= 258");
    return TG_ERR_SHAPE;
  }
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    std::vector<double> A(A_host, A_host + (size_t)x.nz * x.nz);
    auto bytes = [&x](size_t n) -> void* { return x.dalloc<unsigned char>(n); };
    islice_build(x.islTmp, A, x.nz, x.nz, 5, x.M, bytes);
    EpiParams ep;
    ep.nz = x.nz;
    ep.M = x.M;
    islice_apply(*x.islTmp, reinterpret_cast<const double2*>(in), x.S, reinterpret_cast<double2*>(out), x.S, x.M,
                 dim, ep, x.s);
    TG_CUDA(cudaStreamSynchronize(x.s));
    if (islice_error(*x.islTmp)) throw Error{TG_ERR_TIMEOUT, "RealCplxCube::Multiply > a bounded device wait gave up"};
  });
}

tg_status tg_islice_selftest(tg_ctx* ctx) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (x.nz - 2 > 256) {
    set_error("tg_islice_selftest > the int8-slice product needs nz <= 258");
    return TG_ERR_SHAPE;
  }
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    // a product of the identity whose operator copies are withheld: its
    // bounded wait for them gives up, the kernel drains, frees its tensor
    // memory, sets the flag and returns
    std::vector<double> A((size_t)x.nz * x.nz, 0.0);
    for (int i = 0; i < x.nz; ++i) A[(size_t)i * x.nz + i] = 1.0;
    auto bytes = [&x](size_t n) -> void* { return x.dalloc<unsigned char>(n); };
    islice_build(x.islTmp, A, x.nz, x.nz, 5, x.M, bytes);
    islice_clear_error(*x.islTmp);
    EpiParams ep;
    ep.nz = x.nz;
    ep.M = x.M;
    const IsliceOp* o = x.islTmp;
    const double2* in = x.U;
    double2* out = x.TMP;
    islice_group(&o, &in, &out, &ep, 1, x.M, x.s, true);
    TG_CUDA(cudaStreamSynchronize(x.s));
    const int flag = islice_error(*x.islTmp);
    islice_clear_error(*x.islTmp);
    if (flag) throw Error{TG_ERR_TIMEOUT, "tg_islice_selftest > a bounded wait of the int8-slice product gave up"};
  });
}

tg_status tg_set_zsolver(tg_ctx* ctx, int solver) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (solver != TG_ZSOLVER_DMMA && solver != TG_ZSOLVER_ISLICE) {
    set_error("tg_set_zsolver > unknown z-solver");
    return TG_ERR_ARG;
  }
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    x.zsolver = solver;
    for (int i = 0; i < 5; ++i)
      x.opEinv[i].use_isl = x.opE[i].use_isl = solver == TG_ZSOLVER_ISLICE && x.opEinv[i].isl && x.opE[i].isl;
    x.drop_graphs();
  });
}

tg_status tg_zsolver_error(tg_ctx* ctx, int* flag) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (!flag) {
    set_error("tg_zsolver_error > null argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    TG_CUDA(cudaStreamSynchronize(x.s));
    int f = 0;
    TG_CUDA(cudaMemcpy(&f, x.isl_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (x.islTmp) f |= islice_error(*x.islTmp);
    *flag = f;
  });
}

tg_status tg_helmholtz(tg_ctx* ctx, int which, int stage, const double* rhs, double* out) {
  TG_CHECK_CTX(ctx);
  Ctx& x = *reinterpret_cast<Ctx*>(ctx);
  if (which < 0 || which > 4 || (which == 4 && !x.scalar) || stage < 0 || stage > 2 || !rhs || !out) {
    set_error("Phase::Helmholtz > bad argument");
    return TG_ERR_ARG;
  }
  TG_TRY({
    EpiParams ep;
    ep.mode = EPI_RSCALE;
    ep.lam = x.lamd[which];
    ep.k2 = x.k2;
    ep.sigma = which < 3 ? x.sig_u[stage] : (which == 3 ? 0.0 : x.sig_s[stage]);
    ep.null_mode = std::fabs(ep.sigma) < kSmall;
    gemm(x, x.opEinv[which], reinterpret_cast<const double2*>(rhs), x.S, x.TMP, x.S, 1, ep);
    gemm(x, x.opE[which], x.TMP, x.S, reinterpret_cast<double2*>(out), x.S, 1, EpiParams());
  });
}

}  // extern "C"
