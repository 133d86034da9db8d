// Shared definitions of the sm_100a kernels of libturbid_gpu.so.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "../../include/turbid_gpu.h"

namespace tg {

// ---------------------------------------------------------------------------
// error handling: the C ABI returns codes, the message is kept per thread
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);

struct Error {
  int code;
  std::string msg;
};

// A failed runtime call also records its error as the thread's last error;
// a non-sticky one (out of memory, invalid argument) is cleared here, so that
// the next TG_LAUNCH_CHECK does not report it against an unrelated launch.
#define TG_CUDA(call)                                                           \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      (void)cudaGetLastError();                                                 \
      throw ::tg::Error{TG_ERR_CUDA, std::string(#call) + " > " +               \
                                         cudaGetErrorString(e_)};               \
    }                                                                           \
  } while (0)

extern long long g_launches;   // kernel launches issued by this library (host thread count)

#define TG_LAUNCH_CHECK(name)                                                   \
  do {                                                                          \
    ++::tg::g_launches;                                                         \
    cudaError_t e_ = cudaGetLastError();                                        \
    if (e_ != cudaSuccess)                                                      \
      throw ::tg::Error{TG_ERR_CUDA, std::string(name) + " launch > " +         \
                                         cudaGetErrorString(e_)};               \
  } while (0)

// ---------------------------------------------------------------------------
// per-kernel-class timing with CUDA events (enabled by tg_profile_begin)
// ---------------------------------------------------------------------------
enum ProfCat { PC_GEMM = 0, PC_FFT_FX, PC_FFT_FY, PC_FFT_BY, PC_FFT_BX, PC_ELEM, PC_FILTER, PC_FEAT, PC_ADV, PC_ISLICE, PC_N };
// flops: algorithmic; xflops: executed (< 0: the same)
void prof_begin(cudaStream_t s, int cat, double bytes, double flops, double xflops = -1.0);
void prof_end(cudaStream_t s);

// ---------------------------------------------------------------------------
// complex helpers (device)
// ---------------------------------------------------------------------------
template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mkc(decltype(C::x) a, decltype(C::x) b) {
  C r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
// complex<float> sums as one packed FP32x2 instruction (sm_100); IEEE
// round-to-nearest per lane, so the results equal the two scalar operations
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<unsigned long long*>(&a)),
      "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<unsigned long long*>(&a)),
      "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
#endif
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mkc<C>(a.x * s, a.y * s); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return mkc<C>(a.x, -a.y); }

// ---------------------------------------------------------------------------
// FFT plan for one length (host-owned, device twiddles)
// ---------------------------------------------------------------------------
constexpr int kMaxPasses = 24;
struct FftPlan {
  int L = 0;
  int npass = 0;
  int rad[kMaxPasses] = {0};
  double2* tw64 = nullptr;   // exp(-2 pi i k / L), k < L
  float2* tw32 = nullptr;
};
void fft_plan_create(FftPlan& p, int L);
void fft_plan_destroy(FftPlan& p);

// Grid description the transform kernels need.
struct TransformDims {
  int nx, ny, nz, nxh, nyc, M;
  const int* yidx;   // device: spectral iy -> FFT y index (P3DFFT pruning)
};

// Transforms (fft.cu).  planes = dim * nz; work = Nxh*Ny complex per plane
// of the transform precision.
constexpr int kMaxGather = 9;

// Physical fields of a forward transform launch formed as products on load:
// field f = a[f] * (b[f] + sh[f]) (b[f] null: a[f] as it is), each factor a
// physical field of nz planes.  The launch walks the planes z-major, so the
// factors of one z plane are read from HBM once and then from L2.
struct PhysProduct {
  const void* a[kMaxGather];
  const void* b[kMaxGather];
  double sh[kMaxGather];
  int nf;
};
template <typename T>
void dft_forward(const TransformDims& d, const FftPlan& px, const FftPlan& py,
                 const T* phys, double2* spec, int planes, void* work, cudaStream_t s,
                 const PhysProduct* prod = nullptr);
// whether dft_forward can form these products on load (power-of-two Nx, 16-byte aligned factors)
template <typename T>
bool dft_forward_products_ok(const TransformDims& d, const FftPlan& px, const PhysProduct& prod);
// Sources of a backward transform launch, one per field of nz planes: the
// spectral field as it is (deriv 0) or its x (1: i kx) or y (2: i ky)
// derivative, formed as the coefficients are loaded.  plane0 is the global
// plane index of the launch's first plane.
struct SpecGather {
  const double2* src[kMaxGather];
  int deriv[kMaxGather];
  const double* kx;
  const double* ky;
  int nf;       // fields; 0: plain contiguous source
  int plane0;
};
template <typename T>
void dft_backward(const TransformDims& d, const FftPlan& px, const FftPlan& py,
                  const double2* spec, T* phys, int planes, void* work, cudaStream_t s,
                  const SpecGather* gather = nullptr);
// Backward transforms of ncomp groups of three gradient fields (gathered
// spectral sources, grad.nf = 3 ncomp, grad.plane0 = 0), each group reduced on
// the x pass to out_c = (u+su) d_c/dx + (v+sv) d_c/dy + (w+sw) d_c/dz with the
// physical velocity unl (3 fields); power-of-two Nx, Ny only (see _ok).
template <typename T>
bool dft_backward_adv_ok(const TransformDims& d, const FftPlan& px, const FftPlan& py, const T* unl, const T* out);
template <typename T>
void dft_backward_adv(const TransformDims& d, const FftPlan& px, const FftPlan& py, const SpecGather& grad, int ncomp,
                      const T* unl, T* out, double su, double sv, double sw, void* work, cudaStream_t s);

// ---------------------------------------------------------------------------
// z-operator GEMM (gemm.cu):  out[r][m] = epi( sum_k A[r][k] in[k][m] )
// A: rows x K row-major FP64 with leading dimension lda (multiple of 2)
// in/out: batch of spectral components, stride comp_stride complex each.
// ---------------------------------------------------------------------------
enum EpiMode {
  EPI_STORE = 0,     // out = acc
  EPI_RSCALE = 1,    // out = acc * R(r,m)          (Helmholtz reciprocal)
  EPI_DIV = 2,       // out = s*(acc + i kx X0 + i ky X1)
  EPI_LAPRHS = 3,    // out = a*c2*H + a*U - (acc + dx2*U + dy2*U)
  EPI_GRAD = 4,      // out = acc; aux0 = i kx X; aux1 = i ky X (X = input)
  EPI_ADDTO = 5,     // out = acc + aux0 + aux1 (three-term sums)
};

struct EpiParams {
  int mode = EPI_STORE;
  int nz = 0;            // number of z rows (for boundary-row rules)
  int M = 0;
  // EPI_RSCALE
  const double* lam = nullptr;   // [nz]
  const double* k2 = nullptr;    // [M]  (-kx^2 - ky^2)
  double sigma = 0.0;
  int null_mode = 0;             // zero R(r,0) where |lam|<1e-11 (sigma == 0)
  // EPI_DIV / EPI_GRAD
  const double* kx = nullptr;    // [M]
  const double* ky = nullptr;    // [M]
  const double2* X0 = nullptr;
  const double2* X1 = nullptr;
  double s = 1.0;
  // EPI_LAPRHS
  const double2* H = nullptr;
  const double2* U = nullptr;
  const double* dx2 = nullptr;   // [M]
  const double* dy2 = nullptr;   // [M]
  double a = 0.0, c2 = 0.0;
  // EPI_GRAD
  double2* aux0 = nullptr;
  double2* aux1 = nullptr;
  // batch strides (complex elements) for the pointers above
  long long sX = 0, sH = 0, sU = 0, sAux = 0;
};

// FP64-accurate product from exact int8 tensor-core slices (islice.cu): the
// operator's slices and the data-slicing scratch of one component.
struct IsliceOp;
// Slices of the nrow x nz row-major operator A (S = 5), for products over
// components of M modes; op is built on the first call and refilled (same
// shape) on later ones.  Device memory through alloc (owned by the caller).
void islice_build(IsliceOp*& op, const std::vector<double>& A, int nrow, int nz, int S, int M,
                  const std::function<void*(size_t)>& alloc, int* err = nullptr);
void islice_destroy(IsliceOp* op);
// n <= 3 problems (distinct operators), one launch pair: out_i = epi_i(A_i in_i)
void islice_group(const IsliceOp* const* ops, const double2* const* ins, double2* const* outs,
                  const EpiParams* eps, int n, int M, cudaStream_t s, bool withhold_operator = false);
void islice_apply(const IsliceOp& op, const double2* in, long long in_stride, double2* out, long long out_stride,
                  int M, int batch, const EpiParams& ep, cudaStream_t s);
// the error flag of the product's bounded waits (synchronous read, clear)
int islice_error(const IsliceOp& op);
void islice_clear_error(const IsliceOp& op);

// A real nz x nz operator resident on the device: the dense copy and, when
// it is centro-symmetric (sgn +1) or centro-antisymmetric (sgn -1), the two
// folded halves used by the half-flop kernel.
struct ZOperator {
  int n = 0, lda = 0, rowsPad = 0;
  bool sym = false;
  int sgn = 1;
  // split solve halves (sym kernel): 0 = folded input and output of a
  // centro-(anti)symmetric operator; 1 = folded input, output rows 0..h the
  // even products and h+1..n-1 the odd ones; 2 = that split input, unfolded
  // output, plus x[n-1] += quirk * x[0]
  int split = 0;
  double quirk = 0.0;
  int rows = 0, mt = 0, tiles = 0;       // launch shape of the kernel used
  int mt_dense = 0, tiles_dense = 0;
  // row-tile preferences (most m-tiles of 8 rows per CTA) of the dense and
  // folded kernels; 0 = the built-in maximum
  int pref_dense = 0, pref_sym = 0;
  double* A = nullptr;
  double* Ae = nullptr;
  double* Ao = nullptr;
  // int8-slice form of a dense operator (mixed precision solves); used by
  // zgemm for the STORE and RSCALE epilogues when use_isl is set
  IsliceOp* isl = nullptr;
  bool use_isl = false;
};

// One problem of a grouped launch: batch components of `in` (stride in_stride
// complex) through op into `out`, with its own epilogue.
struct ZProblem {
  const ZOperator* op;
  const double2* in;
  long long in_stride;
  double2* out;
  long long out_stride;
  int batch;
  EpiParams ep;
};

void zgemm_init();
void row_tiling(int rows, int maxmt, int& mt, int& tiles);
void zop_build(ZOperator& op, const std::vector<double>& A, int n, bool allow_sym,
               const std::function<double*(size_t)>& alloc);
// halves of one step of a split Helmholtz solve (split = 1: Einvs, 2: Es)
void zop_build_split(ZOperator& op, const std::vector<double>& A, int n, int split, double quirk,
                     const std::function<double*(size_t)>& alloc);
// Re-tile an operator (built or not) for the row-tile preferences of the dense
// and folded kernels (0 = built-in maximum); results do not depend on the
// tiling, only the launch shape does.
void zop_set_tiling(ZOperator& op, int pref_dense, int pref_sym);
void zop_tiling_limits(int& max_dense, int& max_sym);
void zgemm(const ZOperator& op, const double2* in, long long in_stride, double2* out, long long out_stride, int M,
           int batch, const EpiParams& ep, cudaStream_t s);
// up to three problems whose operators share the kernel shape, in one launch
void zgemm_group(const ZProblem* probs, int nprob, int M, cudaStream_t s);

}  // namespace tg
