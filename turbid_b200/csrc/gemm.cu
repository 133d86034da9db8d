// Dense z-operators of the Chebyshev space stepper and of the Helmholtz
// decompositions (reference src/cube_real_cplx.cc:461-513 Multiply, applied by
// src/stepper_space.cc:265-408 and src/phase_carrier_flat.cc:861-994).
//
// In the z-slab layout a spectral component is a row-major (Nz x 2M) real
// matrix (row = z plane, column = re/im of mode m), so applying a real Nz x Nz
// operator along z is the plain GEMM  out = A * in  with a K dimension of Nz.
// Tiles run on the FP64 tensor-core path (mma.sync m8n8k4 f64), operands
// staged through shared memory with double buffering.  Each accumulator pair
// of a thread is one complex number (re, im) of mode m, so the epilogues that
// follow the reference's Armadillo expressions (reciprocal scaling,
// divergence, Laplacian + right-hand side, gradient) run per element on the
// accumulators before the single store.
//
// Two kernels:
//   dense: CTA = MT*8 output rows x 128 reals; 8 warps, each all MT m-tiles x
//          2 n-tiles; MT chosen per Nz so the row tiles cover Nz with little
//          padding (257 rows = 3 tiles of 88).
//   sym:   operators with A[n-1-i][n-1-j] = s*A[i][j] (s = +1 for D2, -1 for
//          D1 on the Chebyshev-Gauss-Lobatto grid).  With h = (n-1)/2 and the
//          folded input  xe[k] = x[k] + x[n-1-k] (k < h), xe[h] = x[h],
//          xo[k] = x[k] - x[n-1-k]  the product is P = Ae*xe, Q = Ao*xo with
//          Ae[i][j] = (A[i][j] + A[i][n-1-j])/2, Ao[i][j] = (A[i][j] - A[i][n-1-j])/2
//          (j < h), Ae[i][h] = A[i][h], and  y[i] = P + Q, y[n-1-i] = s (P - Q)
//          for i <= h: half the flops of the dense product.  CTA = MT*8 folded
//          rows x 64 reals; each warp holds P and Q of one n-tile.
//
// A launch may carry up to kMaxGroup problems (different operators, inputs,
// outputs and epilogues of the same kernel shape): blockIdx.z enumerates the
// components of all of them, so independent z-solves share one grid and one
// tail.
#include <algorithm>
#include <cmath>

#include "tg_common.cuh"

namespace tg {

namespace {
constexpr int BK = 16;          // K per pipeline stage
constexpr int AST = BK + 4;     // smem row stride of A tiles (doubles): conflict-free fragments
constexpr int kThreads = 256;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Epilogue in two phases: the operands of several outputs are loaded first
// (the output stores may alias them as far as the compiler knows, so loads
// issued after a store would each wait for it), then combined and stored.
struct EpiIn {
  double2 a, c;   // DIV: X0, X1; LAPRHS: H, U; GRAD: X
  double s0, s1;  // DIV/GRAD: kx, ky; LAPRHS: dx2, dy2; RSCALE: k2 + lam (+ sigma), lam
};

template <int MODE>
__device__ __forceinline__ EpiIn epi_load(const EpiParams& ep, int b, int r, int m) {
  // read-only operands (never the launch's output: every caller passes
  // separate buffers), loaded through the non-coherent path so that the
  // compiler may move them ahead of the epilogue's stores
  EpiIn in;
  switch (MODE) {
    case EPI_RSCALE:
      if (r != 0 && r != ep.nz - 1) {
        in.s1 = __ldg(ep.lam + r);
        in.s0 = (__ldg(ep.k2 + m) + in.s1) + ep.sigma;
      }
      break;
    case EPI_DIV: {
      const size_t o = (size_t)b * ep.sX + (size_t)r * ep.M + m;
      in.a = __ldg(ep.X0 + o);
      in.c = __ldg(ep.X1 + o);
      in.s0 = __ldg(ep.kx + m);
      in.s1 = __ldg(ep.ky + m);
      break;
    }
    case EPI_LAPRHS:
      in.a = __ldg(ep.H + (size_t)b * ep.sH + (size_t)r * ep.M + m);
      in.c = __ldg(ep.U + (size_t)b * ep.sU + (size_t)r * ep.M + m);
      in.s0 = __ldg(ep.dx2 + m);
      in.s1 = __ldg(ep.dy2 + m);
      break;
    case EPI_GRAD:
      in.a = __ldg(ep.X0 + (size_t)b * ep.sX + (size_t)r * ep.M + m);
      in.s0 = __ldg(ep.kx + m);
      in.s1 = __ldg(ep.ky + m);
      break;
    default:
      break;
  }
  return in;
}

// Every rounding step of the epilogues is explicit (__fma_rn, __dmul_rn,
// __dadd_rn): plain a * b + c may be fused or not by the code generator,
// differently in each tile-shape instantiation, and the results are meant to be
// bit-identical for every row tiling.
template <int MODE>
__device__ __forceinline__ double2 epi_apply(const EpiParams& ep, int b, int r, int m, double2 acc, const EpiIn& in) {
  switch (MODE) {
    case EPI_RSCALE: {
      double R = 1.0;
      if (r != 0 && r != ep.nz - 1) {
        R = 1.0 / in.s0;
        if (ep.null_mode && m == 0 && fabs(in.s1) < 10e-12) R = 0.0;
      }
      return make_double2(__dmul_rn(acc.x, R), __dmul_rn(acc.y, R));
    }
    case EPI_DIV: {
      const double2 x0 = in.a, x1 = in.c;
      const double kx = in.s0, ky = in.s1;
      const double re = __dadd_rn(__dadd_rn(acc.x, __fma_rn(-kx, x0.y, __dmul_rn(0.0, x0.x))),
                                  __fma_rn(-ky, x1.y, __dmul_rn(0.0, x1.x)));
      const double im = __dadd_rn(__dadd_rn(acc.y, __fma_rn(kx, x0.x, __dmul_rn(0.0, x0.y))),
                                  __fma_rn(ky, x1.x, __dmul_rn(0.0, x1.y)));
      return make_double2(__dmul_rn(ep.s, re), __dmul_rn(ep.s, im));
    }
    case EPI_LAPRHS: {
      const double2 h = in.a, u = in.c;
      const double dx2 = in.s0, dy2 = in.s1;
      const double lre = __fma_rn(dy2, u.x, __fma_rn(dx2, u.x, acc.x));
      const double lim = __fma_rn(dy2, u.y, __fma_rn(dx2, u.y, acc.y));
      const double ac2 = __dmul_rn(ep.a, ep.c2);
      return make_double2(__fma_rn(ac2, h.x, __fma_rn(ep.a, u.x, -lre)), __fma_rn(ac2, h.y, __fma_rn(ep.a, u.y, -lim)));
    }
    case EPI_GRAD: {
      const double2 x = in.a;
      const double kx = in.s0, ky = in.s1;
      const size_t oa = (size_t)b * ep.sAux + (size_t)r * ep.M + m;
      ep.aux0[oa] = make_double2(__fma_rn(-kx, x.y, __dmul_rn(0.0, x.x)), __fma_rn(kx, x.x, __dmul_rn(0.0, x.y)));
      ep.aux1[oa] = make_double2(__fma_rn(-ky, x.y, __dmul_rn(0.0, x.x)), __fma_rn(ky, x.x, __dmul_rn(0.0, x.y)));
      return acc;
    }
    default:
      return acc;
  }
}

struct GemmArgs {
  const double* A;    // dense: A; sym: Ae      (rows padded x lda, zero padded)
  const double* Ao;   // sym: Ao
  int lda;
  int rows;           // dense: output rows; sym: folded rows h+1
  int K;              // dense: Nz; sym: h+1
  int nz;             // physical rows
  int sgn;            // sym: +1 / -1
  const double* B;
  long long in_stride;   // complex elements between batch components
  double* C;
  long long out_stride;
  int M;
  int batch;          // components of this problem
  int split;          // sym: ZOperator::split
  double quirk;       // sym, split 2: x[n-1] += quirk * x[0]
  EpiParams ep;
};

constexpr int kMaxGroup = 3;

// output of a dense tile through the epilogue MODE, one m-tile at a time
template <int MT, int MODE>
__device__ __forceinline__ void dense_store(const GemmArgs& g, int b, int r0, int j0, const double (&acc)[MT][2][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* Cb = reinterpret_cast<double2*>(g.C) + (size_t)b * g.out_stride;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt) {
    const int r = r0 + mt * 8 + (lane >> 2);
    EpiIn in[2];
    bool ok[2];
    int m[2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      m[nt] = (j0 + warp * 16 + nt * 8) / 2 + (lane & 3);
      ok[nt] = r < g.rows && m[nt] < g.M;
      if (ok[nt]) in[nt] = epi_load<MODE>(g.ep, b, r, m[nt]);
    }
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
      if (ok[nt])
        Cb[(size_t)r * g.M + m[nt]] =
            epi_apply<MODE>(g.ep, b, r, m[nt], make_double2(acc[mt][nt][0], acc[mt][nt][1]), in[nt]);
  }
}

// output of a folded tile (rows i and n-1-i) through the epilogue MODE
template <int MT, int MODE>
__device__ __forceinline__ void sym_store(const GemmArgs& g, int b, int r0, int j0, const double (&accE)[MT][2][2],
                                          const double (&accO)[MT][2][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = g.nz, h = (g.nz - 1) / 2;
  const double s = (double)g.sgn;
  double2* Cb = reinterpret_cast<double2*>(g.C) + (size_t)b * g.out_stride;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt) {
    const int i = r0 + mt * 8 + (lane >> 2);
    const int j = n - 1 - i;
    bool ok[2];
    int m[2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      m[nt] = (j0 + warp * 16 + nt * 8) / 2 + (lane & 3);
      ok[nt] = m[nt] < g.M;
    }
    // split 1: row i = P, row h+1+i = Q; otherwise row i = P + Q, row n-1-i = s (P - Q)
    const bool sp1 = g.split == 1;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int r = half == 0 ? i : (sp1 ? h + 1 + i : j);
      const bool row_ok = half == 0 ? i <= h : i < h;
      // one n-tile at a time: the operand loads of both n-tiles at once
      // spill the folded kernel's registers at MT = 6
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        if (!(row_ok && ok[nt])) continue;
        const EpiIn in = epi_load<MODE>(g.ep, b, r, m[nt]);
        const double pe = accE[mt][nt][0], pi = accE[mt][nt][1], qe = accO[mt][nt][0], qi = accO[mt][nt][1];
        double2 v;
        if (sp1)
          v = half == 0 ? make_double2(pe, pi) : make_double2(qe, qi);
        else if (half == 0)
          v = make_double2(__dadd_rn(pe, qe), __dadd_rn(pi, qi));
        else {
          v = make_double2(__dmul_rn(s, __dsub_rn(pe, qe)), __dmul_rn(s, __dsub_rn(pi, qi)));
          if (i == 0 && g.quirk != 0.0) {  // top row after the bottom one (x[0] = P + Q)
            v.x = __fma_rn(g.quirk, __dadd_rn(pe, qe), v.x);
            v.y = __fma_rn(g.quirk, __dadd_rn(pi, qi), v.y);
          }
        }
        Cb[(size_t)r * g.M + m[nt]] = epi_apply<MODE>(g.ep, b, r, m[nt], v, in);
      }
    }
  }
}


// ---------------------------------------------------------------------------
// dense: out rows [r0, r0 + 8*MT), columns [j0, j0 + 128) reals
// ---------------------------------------------------------------------------
template <int MT>
__device__ __forceinline__ void dense_body(const GemmArgs& g, const int b) {
  constexpr int BM = 8 * MT, BN = 128, BST = BN + 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* As = reinterpret_cast<double*>(smem_raw);   // [2][BM][AST]
  double* Bs = As + 2 * BM * AST;                      // [2][BK][BST]
  const int ncol = 2 * g.M;
  const int r0 = blockIdx.x * BM;
  const int j0 = blockIdx.y * BN;
  const double* Bb = g.B + (size_t)b * g.in_stride * 2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nkt = (g.K + BK - 1) / BK;
  int mt_valid = (g.rows - r0 + 7) / 8;
  mt_valid = mt_valid > MT ? MT : mt_valid;

  auto load_tile = [&](int kt, int buf) {
    const int k0 = kt * BK;
    double* as = As + buf * BM * AST;
    for (int c = tid; c < BM * (BK / 2); c += kThreads) {
      int row = c / (BK / 2), kk = (c % (BK / 2)) * 2;
      cp_async16(as + row * AST + kk, g.A + (size_t)(r0 + row) * g.lda + k0 + kk, true);
    }
    double* bs = Bs + buf * BK * BST;
#pragma unroll
    for (int i = 0; i < (BK * BN / 2) / kThreads; ++i) {
      int c = tid + i * kThreads;
      int kr = c / (BN / 2), jj = (c % (BN / 2)) * 2;
      int k = k0 + kr, j = j0 + jj;
      bool ok = (k < g.K) && (j < ncol);
      const double* src = ok ? (Bb + (size_t)k * ncol + j) : Bb;
      cp_async16(bs + kr * BST + jj, src, ok);
    }
  };

  double acc[MT][2][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  load_tile(0, 0);
  cp_async_commit();
  for (int kt = 0; kt < nkt; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < nkt) {
      load_tile(kt + 1, buf ^ 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* as = As + buf * BM * AST;
    const double* bs = Bs + buf * BK * BST;
    const int ksteps = min(BK / 4, (g.K - kt * BK + 3) / 4);   // skip the zero K tail
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      if (ks < ksteps) {
        double bf[2];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) bf[nt] = bs[(ks * 4 + (lane & 3)) * BST + warp * 16 + nt * 8 + (lane >> 2)];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          if (mt < mt_valid) {
            double af = as[(mt * 8 + (lane >> 2)) * AST + ks * 4 + (lane & 3)];
            dmma(acc[mt][0][0], acc[mt][0][1], af, bf[0]);
            dmma(acc[mt][1][0], acc[mt][1][1], af, bf[1]);
          }
        }
      }
    }
    __syncthreads();
  }

  switch (g.ep.mode) {
    case EPI_RSCALE: dense_store<MT, EPI_RSCALE>(g, b, r0, j0, acc); break;
    case EPI_DIV: dense_store<MT, EPI_DIV>(g, b, r0, j0, acc); break;
    case EPI_LAPRHS: dense_store<MT, EPI_LAPRHS>(g, b, r0, j0, acc); break;
    case EPI_GRAD: dense_store<MT, EPI_GRAD>(g, b, r0, j0, acc); break;
    default: dense_store<MT, EPI_STORE>(g, b, r0, j0, acc); break;
  }
}

// ---------------------------------------------------------------------------
// sym: folded rows [r0, r0 + 8*MT) of P and Q, columns [j0, j0 + 128) reals
// ---------------------------------------------------------------------------
template <int MT, bool SPLIT_IN>
__device__ __forceinline__ void sym_body(const GemmArgs& g, const int b) {
  constexpr int BM = 8 * MT, BN = 128, BST = BN + 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* Ae = reinterpret_cast<double*>(smem_raw);   // [2][BM][AST]
  double* Ao = Ae + 2 * BM * AST;                      // [2][BM][AST]
  double* Bt = Ao + 2 * BM * AST;                      // [2][BK][BST] input rows k (k <= h)
  double* Bb = Bt + 2 * BK * BST;                      // [2][BK][BST] input rows n-1-k (k < h, else 0)
  const int ncol = 2 * g.M;
  const int n = g.nz, h = (g.nz - 1) / 2;
  const int r0 = blockIdx.x * BM;
  const int j0 = blockIdx.y * BN;
  const double* Bsrc = g.B + (size_t)b * g.in_stride * 2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nkt = (g.K + BK - 1) / BK;
  int mt_valid = (g.rows - r0 + 7) / 8;
  mt_valid = mt_valid > MT ? MT : mt_valid;
  constexpr bool split_in = SPLIT_IN;   // input already even rows 0..h, odd rows h+1..n-1 (split 2)

  auto load_tile = [&](int kt, int buf) {
    const int k0 = kt * BK;
    double* ae = Ae + buf * BM * AST;
    double* ao = Ao + buf * BM * AST;
    for (int c = tid; c < BM * (BK / 2); c += kThreads) {
      const int row = c / (BK / 2), kk = (c % (BK / 2)) * 2;
      cp_async16(ae + row * AST + kk, g.A + (size_t)(r0 + row) * g.lda + k0 + kk, true);
      cp_async16(ao + row * AST + kk, g.Ao + (size_t)(r0 + row) * g.lda + k0 + kk, true);
    }
    double* bt = Bt + buf * BK * BST;
    double* bb = Bb + buf * BK * BST;
#pragma unroll
    for (int i = 0; i < (BK * BN / 2) / kThreads; ++i) {
      const int c = tid + i * kThreads;
      const int kr = c / (BN / 2), jj = (c % (BN / 2)) * 2;
      const int k = k0 + kr, j = j0 + jj;
      const bool okt = (k <= h) && (j < ncol);
      const bool okb = (k < h) && (j < ncol);
      const int kb = split_in ? h + 1 + k : n - 1 - k;   // odd half: split rows or mirrored rows
      cp_async16(bt + kr * BST + jj, okt ? Bsrc + (size_t)k * ncol + j : Bsrc, okt);
      cp_async16(bb + kr * BST + jj, okb ? Bsrc + (size_t)kb * ncol + j : Bsrc, okb);
    }
  };

  double accE[MT][2][2], accO[MT][2][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) accE[i][j][0] = accE[i][j][1] = accO[i][j][0] = accO[i][j][1] = 0.0;

  load_tile(0, 0);
  cp_async_commit();
  for (int kt = 0; kt < nkt; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < nkt) {
      load_tile(kt + 1, buf ^ 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* ae = Ae + buf * BM * AST;
    const double* ao = Ao + buf * BM * AST;
    const double* bt = Bt + buf * BK * BST;
    const double* bb = Bb + buf * BK * BST;
    const int ksteps = min(BK / 4, (g.K - kt * BK + 3) / 4);
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      if (ks < ksteps) {
        double be[2], bo[2];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const int bi = (ks * 4 + (lane & 3)) * BST + warp * 16 + nt * 8 + (lane >> 2);
          const double top = bt[bi], bot = bb[bi];
          be[nt] = split_in ? top : top + bot;
          bo[nt] = split_in ? bot : top - bot;
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          if (mt < mt_valid) {
            const int ai = (mt * 8 + (lane >> 2)) * AST + ks * 4 + (lane & 3);
            const double fe = ae[ai], fo = ao[ai];
            dmma(accE[mt][0][0], accE[mt][0][1], fe, be[0]);
            dmma(accE[mt][1][0], accE[mt][1][1], fe, be[1]);
            dmma(accO[mt][0][0], accO[mt][0][1], fo, bo[0]);
            dmma(accO[mt][1][0], accO[mt][1][1], fo, bo[1]);
          }
        }
      }
    }
    __syncthreads();
  }

  switch (g.ep.mode) {
    case EPI_RSCALE: sym_store<MT, EPI_RSCALE>(g, b, r0, j0, accE, accO); break;
    case EPI_DIV: sym_store<MT, EPI_DIV>(g, b, r0, j0, accE, accO); break;
    case EPI_LAPRHS: sym_store<MT, EPI_LAPRHS>(g, b, r0, j0, accE, accO); break;
    case EPI_GRAD: sym_store<MT, EPI_GRAD>(g, b, r0, j0, accE, accO); break;
    default: sym_store<MT, EPI_STORE>(g, b, r0, j0, accE, accO); break;
  }
}

// blockIdx.z runs over the components of all problems of the launch (NP = 1
// or kMaxGroup; unused trailing problems have batch 0).  The problems are
// separate by-value parameters so that each body reads its arguments as
// constant-bank operands.
#define TG_GROUP_DISPATCH(BODY)               \
  int z = blockIdx.z;                         \
  if (NP == 1 || z < g0.batch) {              \
    BODY(g0, z);                              \
    return;                                   \
  }                                           \
  z -= g0.batch;                              \
  if (z < g1.batch) {                         \
    BODY(g1, z);                              \
    return;                                   \
  }                                           \
  z -= g1.batch;                              \
  BODY(g2, z);

template <int MT, int NP>
__global__ void __launch_bounds__(kThreads) zgemm_dense_kernel(GemmArgs g0, GemmArgs g1, GemmArgs g2) {
#define TG_BODY(G, Z) dense_body<MT>(G, Z)
  TG_GROUP_DISPATCH(TG_BODY)
#undef TG_BODY
}

template <int MT, int NP, bool SPLIT_IN>
__global__ void __launch_bounds__(kThreads, 2) zgemm_sym_kernel(GemmArgs g0, GemmArgs g1, GemmArgs g2) {
#define TG_BODY(G, Z) sym_body<MT, SPLIT_IN>(G, Z)
  TG_GROUP_DISPATCH(TG_BODY)
#undef TG_BODY
}

template <int MT>
size_t dense_smem() {
  return 2 * (8 * MT * AST + BK * (128 + 4)) * sizeof(double);
}
template <int MT>
size_t sym_smem() {
  return 2 * (2 * 8 * MT * AST + 2 * BK * (128 + 4)) * sizeof(double);
}

constexpr int kMaxMtDense = 16, kMaxMtSym = 6;
#define TG_MT_LIST(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)
#define TG_MT_SYM_LIST(X) X(1) X(2) X(3) X(4) X(5) X(6)

}  // namespace

void zgemm_init() {
#define TG_SET(MT)                                                                                           \
  TG_CUDA(cudaFuncSetAttribute(zgemm_dense_kernel<MT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                               (int)dense_smem<MT>()));                                                      \
  TG_CUDA(cudaFuncSetAttribute(zgemm_dense_kernel<MT, kMaxGroup>,                                           \
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dense_smem<MT>()));
  TG_MT_LIST(TG_SET)
#undef TG_SET
#define TG_SET_ONE(MT, NP, SI)                                                                           \
  TG_CUDA(cudaFuncSetAttribute(zgemm_sym_kernel<MT, NP, SI>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                               (int)sym_smem<MT>()));
#define TG_SET(MT)                      \
  TG_SET_ONE(MT, 1, false)              \
  TG_SET_ONE(MT, kMaxGroup, false)      \
  TG_SET_ONE(MT, 1, true)               \
  TG_SET_ONE(MT, kMaxGroup, true)
  TG_MT_SYM_LIST(TG_SET)
#undef TG_SET
#undef TG_SET_ONE
}

// m-tiles per CTA for `rows` rows: as few row tiles as possible with at most
// maxmt m-tiles each, then the tiles as even as possible
void row_tiling(int rows, int maxmt, int& mt, int& tiles) {
  const int need = (rows + 7) / 8;
  tiles = (need + maxmt - 1) / maxmt;
  mt = (need + tiles - 1) / tiles;
}

// Rows of the padded operator buffers of an n x n operator: enough for every
// tiling that a preference in [1, kMaxMtDense] (dense kernel, n rows) or
// [1, kMaxMtSym] (folded kernel, h+1 rows) selects, so that re-tiling a built
// operator needs no new buffers.
static int rows_alloc(int n) {
  const int hr = (n - 1) / 2 + 1;
  int r = 0, mt = 0, tiles = 0;
  for (int p = 1; p <= kMaxMtDense; ++p) {
    row_tiling(n, p, mt, tiles);
    r = std::max(r, mt * tiles * 8);
  }
  for (int p = 1; p <= kMaxMtSym; ++p) {
    row_tiling(hr, p, mt, tiles);
    r = std::max(r, mt * tiles * 8);
  }
  return r;
}

void zop_tiling_limits(int& max_dense, int& max_sym) {
  max_dense = kMaxMtDense;
  max_sym = kMaxMtSym;
}

void zop_set_tiling(ZOperator& op, int pref_dense, int pref_sym) {
  if (pref_dense < 0 || pref_dense > kMaxMtDense || pref_sym < 0 || pref_sym > kMaxMtSym)
    throw Error{TG_ERR_ARG, "zop_set_tiling > tiling out of range"};
  op.pref_dense = pref_dense;
  op.pref_sym = pref_sym;
  if (op.n == 0) return;   // not built yet: zop_build applies the preferences
  row_tiling(op.n, pref_dense ? pref_dense : kMaxMtDense, op.mt_dense, op.tiles_dense);
  int need = op.mt_dense * op.tiles_dense * 8;
  if (op.sym) {
    row_tiling(op.rows, pref_sym ? pref_sym : kMaxMtSym, op.mt, op.tiles);
    need = std::max(need, op.mt * op.tiles * 8);
  } else {
    op.mt = op.mt_dense;
    op.tiles = op.tiles_dense;
  }
  if (op.rowsPad < need) throw Error{TG_ERR_ARG, "zop_set_tiling > operator buffer too small"};
}

static void zgemm_launch(const ZProblem* probs, int nprob, int M, cudaStream_t s);

// Problems of one kernel shape share a launch; a group that mixes dense,
// folded and split-input operators runs as one launch per shape.
// Dense operators with an int8-slice form (use_isl) take the tensor-core
// slice product for single-component problems with a STORE or RSCALE
// epilogue, grouped when their operators differ (each owns its scratch).
void zgemm_group(const ZProblem* probs, int nprob, int M, cudaStream_t s) {
  if (nprob < 1 || nprob > kMaxGroup) throw Error{TG_ERR_ARG, "zgemm > bad group size"};
  ZProblem part[3][kMaxGroup];
  int np[3] = {0, 0, 0};
  const IsliceOp* iops[kMaxGroup];
  const double2* iins[kMaxGroup];
  double2* iouts[kMaxGroup];
  EpiParams ieps[kMaxGroup];
  int ni = 0;
  for (int i = 0; i < nprob; ++i) {
    const ZOperator& op = *probs[i].op;
    const bool isl = op.isl && op.use_isl && !op.sym && probs[i].batch == 1 &&
                     (probs[i].ep.mode == EPI_STORE || probs[i].ep.mode == EPI_RSCALE);
    bool shared_op = false;
    for (int k = 0; k < ni; ++k) shared_op |= iops[k] == op.isl;
    if (isl && !shared_op) {
      iops[ni] = op.isl;
      iins[ni] = probs[i].in;
      iouts[ni] = probs[i].out;
      ieps[ni] = probs[i].ep;
      ieps[ni].nz = op.n;
      ieps[ni].M = M;
      ++ni;
      continue;
    }
    const int k = !op.sym ? 0 : (op.split == 2 ? 2 : 1);
    part[k][np[k]++] = probs[i];
  }
  if (ni) islice_group(iops, iins, iouts, ieps, ni, M, s);
  for (int k = 0; k < 3; ++k)
    if (np[k]) zgemm_launch(part[k], np[k], M, s);
}

static void zgemm_launch(const ZProblem* probs, int nprob, int M, cudaStream_t s) {
  const ZOperator& op0 = *probs[0].op;
  GemmArgs grp[kMaxGroup];
  int total = 0;
  double fl = 0.0, xfl = 0.0, by = 0.0;
  for (int i = 0; i < nprob; ++i) {
    const ZProblem& pr = probs[i];
    const ZOperator& op = *pr.op;
    if (op.sym != op0.sym || op.mt != op0.mt || op.tiles != op0.tiles || op.n != op0.n ||
        (op.split == 2) != (op0.split == 2))
      throw Error{TG_ERR_ARG, "zgemm > operators of one launch differ in shape"};
    GemmArgs& g = grp[i];
    g.lda = op.lda;
    g.nz = op.n;
    g.B = reinterpret_cast<const double*>(pr.in);
    g.in_stride = pr.in_stride;
    g.C = reinterpret_cast<double*>(pr.out);
    g.out_stride = pr.out_stride;
    g.M = M;
    g.batch = pr.batch;
    g.ep = pr.ep;
    g.ep.nz = op.n;
    g.ep.M = M;
    if (op.sym) {
      g.A = op.Ae;
      g.Ao = op.Ao;
      g.rows = op.rows;
      g.K = op.rows;
      g.sgn = op.sgn;
      g.split = op.split;
      g.quirk = op.quirk;
    } else {
      g.A = op.A;
      g.Ao = nullptr;
      g.rows = op.n;
      g.K = op.n;
      g.sgn = 1;
      g.split = 0;
      g.quirk = 0.0;
    }
    total += pr.batch;
    // flops executed (the folded product does two (h+1)^2 halves), bytes in + out + operator
    fl += 4.0 * op.n * op.n * (double)M * pr.batch;   // algorithmic: the dense product
    xfl += (op.sym ? 2.0 * 4.0 * op.rows * op.rows : 4.0 * op.n * op.n) * (double)M * pr.batch;
    by += (double)pr.batch * 16.0 * M * 2 * op.n + 8.0 * op.n * op.n;
  }
  for (int i = nprob; i < kMaxGroup; ++i) {
    grp[i] = grp[0];
    grp[i].batch = 0;
  }
  prof_begin(s, PC_GEMM, by, fl, xfl);
  if (op0.sym) {
    const bool split_in = op0.split == 2;
    dim3 grid(op0.tiles, (2 * M + 127) / 128, total);
#define TG_SYM(MT, NP, SI) zgemm_sym_kernel<MT, NP, SI><<<grid, kThreads, sym_smem<MT>(), s>>>(grp[0], grp[1], grp[2])
#define TG_CASE(MT)                                              \
  case MT:                                                       \
    if (nprob == 1)                                              \
      split_in ? TG_SYM(MT, 1, true) : TG_SYM(MT, 1, false);     \
    else                                                         \
      split_in ? TG_SYM(MT, kMaxGroup, true) : TG_SYM(MT, kMaxGroup, false); \
    break;
    switch (op0.mt) { TG_MT_SYM_LIST(TG_CASE) default: throw Error{TG_ERR_ARG, "zgemm > bad tiling"}; }
#undef TG_CASE
#undef TG_SYM
  } else {
    dim3 grid(op0.tiles, (2 * M + 127) / 128, total);
#define TG_CASE(MT)                                                                                       \
  case MT:                                                                                                \
    if (nprob == 1)                                                                                       \
      zgemm_dense_kernel<MT, 1><<<grid, kThreads, dense_smem<MT>(), s>>>(grp[0], grp[1], grp[2]);        \
    else                                                                                                  \
      zgemm_dense_kernel<MT, kMaxGroup><<<grid, kThreads, dense_smem<MT>(), s>>>(grp[0], grp[1], grp[2]); \
    break;
    switch (op0.mt) { TG_MT_LIST(TG_CASE) default: throw Error{TG_ERR_ARG, "zgemm > bad tiling"}; }
#undef TG_CASE
  }
  prof_end(s);
  TG_LAUNCH_CHECK("zgemm kernel");
}

void zgemm(const ZOperator& op, const double2* in, long long in_stride, double2* out, long long out_stride, int M,
           int batch, const EpiParams& ep, cudaStream_t s) {
  if (op.isl && op.use_isl && !op.sym && batch > 1 && (ep.mode == EPI_STORE || ep.mode == EPI_RSCALE)) {
    EpiParams e = ep;
    e.nz = op.n;
    e.M = M;
    islice_apply(*op.isl, in, in_stride, out, out_stride, M, batch, e, s);
    return;
  }
  ZProblem p{&op, in, in_stride, out, out_stride, batch, ep};
  zgemm_group(&p, 1, M, s);
}

// Upload an nz x nz operator: the dense copy always; the folded halves when
// the operator is centro-symmetric (sgn = +1) or centro-antisymmetric
// (sgn = -1) to within 1e-12 of its largest entry and allow_sym is set.
void zop_build(ZOperator& op, const std::vector<double>& A, int n, bool allow_sym,
               const std::function<double*(size_t)>& alloc) {
  op.n = n;
  op.lda = (n + 15) / 16 * 16;
  row_tiling(n, op.pref_dense ? op.pref_dense : kMaxMtDense, op.mt_dense, op.tiles_dense);
  const int h = (n - 1) / 2;
  const int hr = h + 1;   // folded rows
  int mts, ts;
  row_tiling(hr, op.pref_sym ? op.pref_sym : kMaxMtSym, mts, ts);
  const int rowsAlloc = rows_alloc(n);
  if (op.rowsPad == 0) op.rowsPad = rowsAlloc;
  if (op.rowsPad < rowsAlloc) throw Error{TG_ERR_ARG, "zop_build > operator buffer too small"};
  const size_t sz = (size_t)op.rowsPad * op.lda;
  if (!op.A) op.A = alloc(sz);
  std::vector<double> pad(sz, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) pad[(size_t)i * op.lda + j] = A[(size_t)i * n + j];
  TG_CUDA(cudaMemcpy(op.A, pad.data(), sz * sizeof(double), cudaMemcpyHostToDevice));
  op.sym = false;
  op.split = 0;
  op.quirk = 0.0;
  if (allow_sym && (n & 1) && n >= 5) {
    double amax = 0.0;
    for (double v : A) amax = std::max(amax, std::fabs(v));
    for (int sgn : {+1, -1}) {
      double dev = 0.0;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          dev = std::max(dev, std::fabs(A[(size_t)(n - 1 - i) * n + (n - 1 - j)] - sgn * A[(size_t)i * n + j]));
      if (dev <= 1e-12 * amax) {
        op.sym = true;
        op.sgn = sgn;
        break;
      }
    }
  }
  if (op.sym) {
    op.rows = hr;
    op.mt = mts;
    op.tiles = ts;
    if (!op.Ae) op.Ae = alloc(sz);
    if (!op.Ao) op.Ao = alloc(sz);
    std::vector<double> ae(sz, 0.0), ao(sz, 0.0);
    for (int i = 0; i < hr; ++i) {
      for (int j = 0; j < h; ++j) {
        const double a = A[(size_t)i * n + j], c = A[(size_t)i * n + (n - 1 - j)];
        ae[(size_t)i * op.lda + j] = (a + c) / 2;
        ao[(size_t)i * op.lda + j] = (a - c) / 2;
      }
      ae[(size_t)i * op.lda + h] = A[(size_t)i * n + h];
    }
    TG_CUDA(cudaMemcpy(op.Ae, ae.data(), sz * sizeof(double), cudaMemcpyHostToDevice));
    TG_CUDA(cudaMemcpy(op.Ao, ao.data(), sz * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    op.rows = n;
    op.mt = op.mt_dense;
    op.tiles = op.tiles_dense;
  }
}

// One step of a split Helmholtz solve on the folded-operator kernel.
//   split 1 (A = Einvs, rows 0..h even and h+1..n-1 odd in the column index):
//     Ae = rows 0..h folded over the columns, Ao = rows h+1..n-1 folded;
//     the kernel stores P at rows 0..h and Q at rows h+1..n-1.
//   split 2 (A = Es, columns 0..h even and h+1..n-1 odd in the row index):
//     Ae = A[0..h][0..h], Ao = A[0..h][h+1..n-1]; the kernel reads the even
//     and odd halves of its input as they are and unfolds the output.
void zop_build_split(ZOperator& op, const std::vector<double>& A, int n, int split, double quirk,
                     const std::function<double*(size_t)>& alloc) {
  if (!(n & 1) || n < 5 || (split != 1 && split != 2)) throw Error{TG_ERR_ARG, "zop_build_split > bad shape"};
  op.n = n;
  op.lda = (n + 15) / 16 * 16;
  row_tiling(n, op.pref_dense ? op.pref_dense : kMaxMtDense, op.mt_dense, op.tiles_dense);
  const int h = (n - 1) / 2, hr = h + 1;
  int mts, ts;
  row_tiling(hr, op.pref_sym ? op.pref_sym : kMaxMtSym, mts, ts);
  const int rowsAlloc = rows_alloc(n);
  if (op.rowsPad == 0) op.rowsPad = rowsAlloc;
  if (op.rowsPad < rowsAlloc) throw Error{TG_ERR_ARG, "zop_build_split > operator buffer too small"};
  const size_t sz = (size_t)op.rowsPad * op.lda;
  if (!op.A) op.A = alloc(sz);
  if (!op.Ae) op.Ae = alloc(sz);
  if (!op.Ao) op.Ao = alloc(sz);
  std::vector<double> ae(sz, 0.0), ao(sz, 0.0);
  auto a = [&](int i, int j) { return A[(size_t)i * n + j]; };
  if (split == 1) {
    for (int i = 0; i < hr; ++i) {
      for (int j = 0; j < h; ++j) ae[(size_t)i * op.lda + j] = 0.5 * (a(i, j) + a(i, n - 1 - j));
      ae[(size_t)i * op.lda + h] = a(i, h);
    }
    for (int i = 0; i < h; ++i)
      for (int j = 0; j < h; ++j) ao[(size_t)i * op.lda + j] = 0.5 * (a(h + 1 + i, j) - a(h + 1 + i, n - 1 - j));
  } else {
    for (int i = 0; i < hr; ++i) {
      for (int j = 0; j < hr; ++j) ae[(size_t)i * op.lda + j] = a(i, j);
      for (int j = 0; j < h; ++j) ao[(size_t)i * op.lda + j] = a(i, h + 1 + j);
    }
  }
  TG_CUDA(cudaMemcpy(op.Ae, ae.data(), sz * sizeof(double), cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(op.Ao, ao.data(), sz * sizeof(double), cudaMemcpyHostToDevice));
  op.sym = true;
  op.sgn = 1;
  op.split = split;
  op.quirk = split == 2 ? quirk : 0.0;
  op.rows = hr;
  op.mt = mts;
  op.tiles = ts;
}

}  // namespace tg
