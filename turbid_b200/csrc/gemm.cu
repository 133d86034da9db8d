// Dense z-operators of the Chebyshev space stepper and of the Helmholtz
// decompositions (reference src/cube_real_cplx.cc:461-513 Multiply, applied by
// src/stepper_space.cc:265-408 and src/phase_carrier_flat.cc:861-994).
//
// In the z-slab layout a spectral component is a row-major (Nz x 2M) real
// matrix (row = z plane, column = re/im of mode m), so applying a real Nz x Nz
// operator along z is the plain GEMM  out = A * in  with a K dimension of Nz.
// FP64 tiles run on the FP64 tensor-core path (mma.sync m8n8k4 f64), operands
// staged through shared memory with cp.async double buffering.  Each
// accumulator pair of a thread is one complex number (re, im) of mode m, so
// the epilogues that follow the reference's Armadillo expressions (reciprocal
// scaling, divergence, Laplacian + right-hand side, gradient) run per element
// on the accumulators before the single store.
#include "tg_common.cuh"

namespace tg {

namespace {
constexpr int BM = 64;    // rows (output z) per CTA
constexpr int BN = 128;   // columns (reals = 64 complex modes) per CTA
constexpr int BK = 16;    // K (input z) per pipeline stage
constexpr int AST = BK + 4;   // smem row stride of A (doubles): conflict-free fragments
constexpr int BST = BN + 4;   // smem row stride of B
constexpr int kThreads = 256;
constexpr size_t kSmem = 2 * (BM * AST + BK * BST) * sizeof(double);

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

__device__ __forceinline__ double2 epilogue(const EpiParams& ep, int b, int r, int m, double2 acc) {
  switch (ep.mode) {
    case EPI_RSCALE: {
      double R = 1.0;
      if (r != 0 && r != ep.nz - 1) {
        R = 1.0 / ((ep.k2[m] + ep.lam[r]) + ep.sigma);
        if (ep.null_mode && m == 0 && fabs(ep.lam[r]) < 10e-12) R = 0.0;
      }
      return make_double2(acc.x * R, acc.y * R);
    }
    case EPI_DIV: {
      const size_t o = (size_t)b * ep.sX + (size_t)r * ep.M + m;
      double2 x0 = ep.X0[o], x1 = ep.X1[o];
      double kx = ep.kx[m], ky = ep.ky[m];
      double re = (acc.x + (0.0 * x0.x - kx * x0.y)) + (0.0 * x1.x - ky * x1.y);
      double im = (acc.y + (0.0 * x0.y + kx * x0.x)) + (0.0 * x1.y + ky * x1.x);
      return make_double2(ep.s * re, ep.s * im);
    }
    case EPI_LAPRHS: {
      const size_t oh = (size_t)b * ep.sH + (size_t)r * ep.M + m;
      const size_t ou = (size_t)b * ep.sU + (size_t)r * ep.M + m;
      double2 h = ep.H[oh], u = ep.U[ou];
      double dx2 = ep.dx2[m], dy2 = ep.dy2[m];
      double lre = (acc.x + dx2 * u.x) + dy2 * u.x;
      double lim = (acc.y + dx2 * u.y) + dy2 * u.y;
      double ac2 = ep.a * ep.c2;
      return make_double2((ac2 * h.x + ep.a * u.x) - lre, (ac2 * h.y + ep.a * u.y) - lim);
    }
    case EPI_GRAD: {
      const size_t o = (size_t)b * ep.sX + (size_t)r * ep.M + m;
      const size_t oa = (size_t)b * ep.sAux + (size_t)r * ep.M + m;
      double2 x = ep.X0[o];
      double kx = ep.kx[m], ky = ep.ky[m];
      ep.aux0[oa] = make_double2(0.0 * x.x - kx * x.y, 0.0 * x.y + kx * x.x);
      ep.aux1[oa] = make_double2(0.0 * x.x - ky * x.y, 0.0 * x.y + ky * x.x);
      return acc;
    }
    default:
      return acc;
  }
}

// A: padded (rowsPad x lda) zero-filled beyond (rows x K); lda % BK == 0.
__global__ void __launch_bounds__(kThreads) zgemm64_kernel(const double* __restrict__ A, int lda, int rows, int K,
                                                           const double* __restrict__ Bm, long long in_stride,
                                                           double* __restrict__ Cm, long long out_stride, int M,
                                                           EpiParams ep) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* As = reinterpret_cast<double*>(smem_raw);       // [2][BM][AST]
  double* Bs = As + 2 * BM * AST;                           // [2][BK][BST]
  const int ncol = 2 * M;
  const int r0 = blockIdx.x * BM;
  const int j0 = blockIdx.y * BN;
  const int b = blockIdx.z;
  const double* Bb = Bm + (size_t)b * in_stride * 2;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wr = warp >> 2, wc = warp & 3;
  const int nkt = (K + BK - 1) / BK;

  auto load_tile = [&](int kt, int buf) {
    const int k0 = kt * BK;
    // A: BM x BK doubles = 512 double2 chunks, 2 per thread
    double* as = As + buf * BM * AST;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      int c = tid + i * kThreads;        // 0..511
      int row = c >> 3, kk = (c & 7) * 2;
      cp_async16(as + row * AST + kk, A + (size_t)(r0 + row) * lda + k0 + kk, true);
    }
    // B: BK x BN doubles = 1024 double2 chunks, 4 per thread
    double* bs = Bs + buf * BK * BST;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int c = tid + i * kThreads;        // 0..1023
      int kr = c >> 6, jj = (c & 63) * 2;
      int k = k0 + kr, j = j0 + jj;
      bool ok = (k < K) && (j < ncol);
      const double* src = ok ? (Bb + (size_t)k * ncol + j) : Bb;
      cp_async16(bs + kr * BST + jj, src, ok);
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // rows of this warp that exist (ragged last row tile): skip empty m-tiles
  const int wrow0 = r0 + wr * 32;
  int mtiles = (rows - wrow0 + 7) / 8;
  mtiles = mtiles < 0 ? 0 : (mtiles > 4 ? 4 : mtiles);

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
    if (mtiles > 0) {
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks) {
        double af[4], bf[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) af[mt] = as[(wr * 32 + mt * 8 + (lane >> 2)) * AST + ks * 4 + (lane & 3)];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) bf[nt] = bs[(ks * 4 + (lane & 3)) * BST + wc * 32 + nt * 8 + (lane >> 2)];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          if (mt < mtiles) {
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt][0], acc[mt][nt][1], af[mt], bf[nt]);
          }
        }
      }
    }
    __syncthreads();
  }

  // epilogue: thread holds (re, im) of one complex mode per (mt, nt)
  double2* Cb = reinterpret_cast<double2*>(Cm) + (size_t)b * out_stride;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int r = wrow0 + mt * 8 + (lane >> 2);
    if (r >= rows) continue;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int m = (j0 + wc * 32 + nt * 8) / 2 + (lane & 3);
      if (m >= M) continue;
      double2 v = epilogue(ep, b, r, m, make_double2(acc[mt][nt][0], acc[mt][nt][1]));
      Cb[(size_t)r * M + m] = v;
    }
  }
}
}  // namespace

void zgemm_init() {
  TG_CUDA(cudaFuncSetAttribute(zgemm64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
}

void zgemm(const double* A, int lda, int rows, int K, const double2* in, long long in_stride, double2* out,
           long long out_stride, int M, int batch, const EpiParams& ep, cudaStream_t s) {
  if (lda % BK != 0) throw Error{TG_ERR_ARG, "zgemm > lda must be a multiple of 16"};
  dim3 grid((rows + BM - 1) / BM, (2 * M + BN - 1) / BN, batch);
  const double fl = 4.0 * rows * K * (double)M * batch;
  const double by = (double)batch * 16.0 * M * (K + rows) + 8.0 * rows * K;
  prof_begin(s, PC_GEMM, by, fl);
  zgemm64_kernel<<<grid, kThreads, kSmem, s>>>(A, lda, rows, K, reinterpret_cast<const double*>(in), in_stride,
                                               reinterpret_cast<double*>(out), out_stride, M, ep);
  prof_end(s);
  TG_LAUNCH_CHECK("zgemm64_kernel");
}

}  // namespace tg
