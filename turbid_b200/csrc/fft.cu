// Pruned plane transforms of RealCplxCube::DftForward / DftBackward
// (reference src/cube_real_cplx.cc:525-555, pruning of P3DFFT's
// build/ftran.F90:122-248 and build/btran.F90:137-243).
//
// Physical planes are x-fastest [plane][y][x]; spectral planes are the
// z-slab layout [plane][m], m = iy + Nyc*ix.  A transform is two kernels:
//   x pass: batched real FFT of two rows at a time packed as one complex FFT,
//           only kx < Nxh kept, written column-major [plane][kx][y];
//   y pass: complex FFT along y of each kept column, only the Nyc pruned
//           wavenumbers kept (kx-major), scaled by 1/(Nx*Ny).
// The backward transform runs the passes in reverse order; in FP32 its
// intermediate is row-major [plane][y][kx], so that each pass reads contiguous
// blocks (the strided side of the reorder is a write, which the L2 merges
// into full lines before they reach HBM).
// The 1-D FFTs are mixed-radix Stockham passes in shared memory with
// twiddles from a table computed once per length on the host.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include <cuda.h>

#include "fft_dev.cuh"

namespace tg {

// ---------------------------------------------------------------------------
// plan: factorisation + twiddle table
// ---------------------------------------------------------------------------
void fft_plan_create(FftPlan& p, int L) {
  p.L = L;
  p.npass = 0;
  int n = L;
  auto push = [&](int r) {
    if (p.npass >= kMaxPasses) throw Error{TG_ERR_SHAPE, "FftPlan > too many passes"};
    p.rad[p.npass++] = r;
  };
  while (n % 4 == 0) { push(4); n /= 4; }
  while (n % 2 == 0) { push(2); n /= 2; }
  const int primes[] = {3, 5, 7, 11, 13};
  for (int q : primes)
    while (n % q == 0) { push(q); n /= q; }
  if (n > 1) push(n);  // one direct DFT pass for the remaining factor
  std::vector<double2> t64(L);
  std::vector<float2> t32(L);
  for (int k = 0; k < L; ++k) {
    // angle -2 pi k / L evaluated in long double
    long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)L;
    long double c = cosl(a), s = sinl(a);
    t64[k] = make_double2((double)c, (double)s);
    t32[k] = make_float2((float)c, (float)s);
  }
  TG_CUDA(cudaMalloc(&p.tw64, sizeof(double2) * L));
  TG_CUDA(cudaMalloc(&p.tw32, sizeof(float2) * L));
  TG_CUDA(cudaMemcpy(p.tw64, t64.data(), sizeof(double2) * L, cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(p.tw32, t32.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
}

void fft_plan_destroy(FftPlan& p) {
  if (p.tw64) cudaFree(p.tw64);
  if (p.tw32) cudaFree(p.tw32);
  p.tw64 = nullptr;
  p.tw32 = nullptr;
}

struct PlanArgs {
  int L, npass;
  int rad[kMaxPasses];
};

static PlanArgs plan_args(const FftPlan& p) {
  PlanArgs a;
  a.L = p.L;
  a.npass = p.npass;
  for (int i = 0; i < kMaxPasses; ++i) a.rad[i] = p.rad[i];
  return a;
}

template <typename T, int DIR>
__device__ cplx<T>* fft_batch(cplx<T>* b0, cplx<T>* b1, int NB, const PlanArgs& pl,
                              const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  const int L = pl.L;
  C* in = b0;
  C* out = b1;
  int Ns = 1;
  for (int ps = 0; ps < pl.npass; ++ps) {
    const int R = pl.rad[ps];
    const int nb = L / R;
    const int twstep = L / (Ns * R);
    for (int idx = threadIdx.x; idx < NB * nb; idx += blockDim.x) {
      const int b = idx / nb;
      const int j = idx - b * nb;
      const C* src = in + b * L;
      C* dst = out + b * L;
      const int jm = j % Ns;
      const int base = (j - jm) * R + jm;
      if (R == 2) {
        C a0 = src[j];
        C a1 = cmul(src[j + nb], tw_get<T, DIR>(tw, jm * twstep));
        dst[base] = cadd(a0, a1);
        dst[base + Ns] = csub(a0, a1);
      } else if (R == 4) {
        C a0 = src[j];
        C a1 = cmul(src[j + nb], tw_get<T, DIR>(tw, jm * twstep));
        C a2 = cmul(src[j + 2 * nb], tw_get<T, DIR>(tw, 2 * jm * twstep));
        C a3 = cmul(src[j + 3 * nb], tw_get<T, DIR>(tw, 3 * jm * twstep));
        C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
        // DIR=-1: multiply t3 by -i ; DIR=+1: by +i
        C t3r = (DIR < 0) ? mkc<C>(t3.y, -t3.x) : mkc<C>(-t3.y, t3.x);
        dst[base] = cadd(t0, t2);
        dst[base + Ns] = cadd(t1, t3r);
        dst[base + 2 * Ns] = csub(t0, t2);
        dst[base + 3 * Ns] = csub(t1, t3r);
      } else if (R <= 16) {
        C v[16];
        for (int r = 0; r < R; ++r) v[r] = cmul(src[j + r * nb], tw_get<T, DIR>(tw, jm * r * twstep));
        const int ws = L / R;
        for (int k = 0; k < R; ++k) {
          C acc = v[0];
          for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], tw_get<T, DIR>(tw, ((r * k) % R) * ws)));
          dst[base + k * Ns] = acc;
        }
      } else {
        const int ws = L / R;
        for (int k = 0; k < R; ++k) {
          C acc = mkc<C>(0, 0);
          for (int r = 0; r < R; ++r) {
            C x = cmul(src[j + r * nb], tw_get<T, DIR>(tw, jm * r * twstep));
            acc = cadd(acc, cmul(x, tw_get<T, DIR>(tw, (int)(((long long)r * k) % R) * ws)));
          }
          dst[base + k * Ns] = acc;
        }
      }
    }
    __syncthreads();
    C* t = in;
    in = out;
    out = t;
    Ns *= R;
  }
  return in;
}

// Layout of the backward intermediate: [plane][y][kx] for FP32 (the x pass
// reads contiguous row blocks), [plane][kx][y] for FP64.
template <typename T> __host__ __device__ constexpr bool bwd_row_major() { return sizeof(T) == 4; }

// Source plane of a gathered backward launch and the derivative to form on load.
__device__ __forceinline__ const double2* gather_src(const SpecGather& g, int plane, int nz, int M, int& deriv) {
  const int gp = g.plane0 + plane, f = gp / nz, z = gp - f * nz;
  deriv = g.deriv[f];
  return g.src[f] + (size_t)z * M;
}
// coefficient m of the loaded plane, differentiated as (0 + i k) * v (the
// complex product of SpaceStepper::Gradient, src/stepper_space.cc:373-385)
__device__ __forceinline__ double2 gather_value(const SpecGather& g, int deriv, int m, double2 v) {
  if (deriv == 0) return v;
  const double k = deriv == 1 ? g.kx[m] : g.ky[m];
  return make_double2(0.0 * v.x - k * v.y, 0.0 * v.y + k * v.x);
}

// ---------------------------------------------------------------------------
// compile-time Stockham passes for power-of-two lengths: radix-16 passes
// while 16 divides the remaining length, then one radix-8/4/2 pass; the small
// DFTs are even/odd splits with constant twiddles, all indexing constant-folded.
// ---------------------------------------------------------------------------
template <typename T, int DIR, int L, int Ns>
__device__ __forceinline__ cplx<T>* ct_passes(cplx<T>* in, cplx<T>* out, int NB, const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  if constexpr (Ns >= L) {
    return in;
  } else {
    constexpr int rem = L / Ns;
    constexpr int R = rem >= 16 ? 16 : rem;
    constexpr int nb = L / R;
    constexpr int twstep = L / (Ns * R);
    for (int idx = threadIdx.x; idx < NB * nb; idx += blockDim.x) {
      const int b = idx / nb;
      const int j = idx - b * nb;
      const C* src = in + b * L;
      C* dst = out + b * L;
      const int jm = j % Ns;
      const int base = (j - jm) * R + jm;
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        v[r] = src[j + r * nb];
        if (Ns > 1 && r > 0) v[r] = cmul(v[r], tw_get<T, DIR>(tw, jm * r * twstep));
      }
      dft_ct<R, DIR>(v);
#pragma unroll
      for (int k = 0; k < R; ++k) dst[base + k * Ns] = v[k];
    }
    __syncthreads();
    return ct_passes<T, DIR, L, Ns * R>(out, in, NB, tw);
  }
}

// FFT of NB length-L transforms in shared memory; LC = L at compile time or 0
template <typename T, int DIR, int LC>
__device__ __forceinline__ cplx<T>* fft_any(cplx<T>* b0, cplx<T>* b1, int NB, const PlanArgs& pl,
                                            const cplx<T>* __restrict__ tw) {
  if constexpr (LC > 0)
    return ct_passes<T, DIR, LC, 1>(b0, b1, NB, tw);
  else
    return fft_batch<T, DIR>(b0, b1, NB, pl, tw);
}

// ---------------------------------------------------------------------------
// forward x pass: phys [plane][y][x] (T) -> work [plane][kx][y] (cplx<T>)
// ---------------------------------------------------------------------------
template <typename T, int LC>
__global__ void __launch_bounds__(256) fwd_x_kernel(TransformDims d, PlanArgs pl, const cplx<T>* __restrict__ tw,
                                                    const T* __restrict__ phys, cplx<T>* __restrict__ work, int NB) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + NB * (LC > 0 ? LC : pl.L);
  const int L = LC > 0 ? LC : pl.L;  // == nx
  const int plane = blockIdx.y;
  const int y0 = blockIdx.x * 2 * NB;
  const T* src = phys + (size_t)plane * d.ny * d.nx;
  for (int idx = threadIdx.x; idx < NB * L; idx += blockDim.x) {
    const int p = idx / L, x = idx - p * L;
    const int ya = y0 + 2 * p, yb = ya + 1;
    T re = ya < d.ny ? src[(size_t)ya * d.nx + x] : T(0);
    T im = yb < d.ny ? src[(size_t)yb * d.nx + x] : T(0);
    b0[idx] = mkc<C>(re, im);
  }
  __syncthreads();
  C* r = fft_any<T, -1, LC>(b0, b1, NB, pl, tw);
  const int rows = 2 * NB;
  C* dst = work + (size_t)plane * d.nxh * d.ny;
  for (int idx = threadIdx.x; idx < rows * d.nxh; idx += blockDim.x) {
    const int k = idx / rows, q = idx - k * rows;
    const int y = y0 + q;
    if (y >= d.ny) continue;
    const int p = q >> 1;
    C Z = r[p * L + k];
    C Zc = cconj(r[p * L + (k == 0 ? 0 : L - k)]);
    C X;
    if ((q & 1) == 0) {
      X = mkc<C>((Z.x + Zc.x) * T(0.5), (Z.y + Zc.y) * T(0.5));
    } else {
      C D = csub(Z, Zc);
      X = mkc<C>(D.y * T(0.5), -D.x * T(0.5));
    }
    dst[(size_t)k * d.ny + y] = X;
  }
}

// forward y pass: work [plane][kx][y] -> spec [plane][iy + nyc*kx] (double2)
template <typename T, int LC>
__global__ void __launch_bounds__(256) fwd_y_kernel(TransformDims d, PlanArgs pl, const cplx<T>* __restrict__ tw,
                                                    const cplx<T>* __restrict__ work, double2* __restrict__ spec,
                                                    int NB, double scale) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + NB * (LC > 0 ? LC : pl.L);
  const int L = LC > 0 ? LC : pl.L;  // == ny
  const int plane = blockIdx.y;
  const int k0 = blockIdx.x * NB;
  const C* src = work + (size_t)plane * d.nxh * d.ny;
  for (int idx = threadIdx.x; idx < NB * L; idx += blockDim.x) {
    const int c = idx / L, y = idx - c * L;
    const int k = k0 + c;
    b0[idx] = k < d.nxh ? src[(size_t)k * d.ny + y] : mkc<C>(0, 0);
  }
  __syncthreads();
  C* r = fft_any<T, -1, LC>(b0, b1, NB, pl, tw);
  double2* dst = spec + (size_t)plane * d.M;
  for (int idx = threadIdx.x; idx < NB * d.nyc; idx += blockDim.x) {
    const int c = idx / d.nyc, iy = idx - c * d.nyc;
    const int k = k0 + c;
    if (k >= d.nxh) continue;
    C v = r[c * L + d.yidx[iy]];
    dst[iy + (size_t)d.nyc * k] = make_double2((double)v.x * scale, (double)v.y * scale);
  }
}

// backward y pass: spec -> work (zero-filled pruned modes, unscaled)
template <typename T, int LC, bool GATHER>
__global__ void __launch_bounds__(256) bwd_y_kernel(TransformDims d, PlanArgs pl, const cplx<T>* __restrict__ tw,
                                                    const double2* __restrict__ spec, cplx<T>* __restrict__ work,
                                                    int NB, SpecGather gat) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + NB * (LC > 0 ? LC : pl.L);
  const int L = LC > 0 ? LC : pl.L;  // == ny
  const int plane = blockIdx.y;
  const int k0 = blockIdx.x * NB;
  for (int idx = threadIdx.x; idx < NB * L; idx += blockDim.x) b0[idx] = mkc<C>(0, 0);
  __syncthreads();
  int deriv = 0;
  const double2* src = GATHER ? gather_src(gat, plane, d.nz, d.M, deriv) : spec + (size_t)plane * d.M;
  for (int idx = threadIdx.x; idx < NB * d.nyc; idx += blockDim.x) {
    const int c = idx / d.nyc, iy = idx - c * d.nyc;
    const int k = k0 + c;
    if (k >= d.nxh) continue;
    const int m = iy + d.nyc * k;
    double2 v = GATHER ? gather_value(gat, deriv, m, src[m]) : src[m];
    b0[c * L + d.yidx[iy]] = mkc<C>((T)v.x, (T)v.y);
  }
  __syncthreads();
  C* r = fft_any<T, +1, LC>(b0, b1, NB, pl, tw);
  C* dst = work + (size_t)plane * d.nxh * d.ny;
  for (int idx = threadIdx.x; idx < NB * L; idx += blockDim.x) {
    if constexpr (bwd_row_major<T>()) {  // [y][kx]
      const int y = idx / NB, c = idx - y * NB;
      const int k = k0 + c;
      if (k < d.nxh) dst[(size_t)y * d.nxh + k] = r[c * L + y];
    } else {  // [kx][y]
      const int c = idx / L, y = idx - c * L;
      const int k = k0 + c;
      if (k < d.nxh) dst[(size_t)k * d.ny + y] = r[idx];
    }
  }
}

// backward x pass: work -> phys [plane][y][x]; two rows per
// complex FFT; the imaginary part of the kx = 0 coefficient is ignored (c2r).
template <typename T, int LC>
__global__ void __launch_bounds__(256) bwd_x_kernel(TransformDims d, PlanArgs pl, const cplx<T>* __restrict__ tw,
                                                    const cplx<T>* __restrict__ work, T* __restrict__ phys, int NB) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* b0 = reinterpret_cast<C*>(smem_raw);
  C* b1 = b0 + NB * (LC > 0 ? LC : pl.L);
  const int L = LC > 0 ? LC : pl.L;  // == nx
  const int plane = blockIdx.y;
  const int y0 = blockIdx.x * 2 * NB;
  for (int idx = threadIdx.x; idx < NB * L; idx += blockDim.x) b0[idx] = mkc<C>(0, 0);
  __syncthreads();
  const C* src = work + (size_t)plane * d.nxh * d.ny;
  for (int idx = threadIdx.x; idx < NB * d.nxh; idx += blockDim.x) {
    constexpr bool RM = bwd_row_major<T>();
    const int p = RM ? idx / d.nxh : idx % NB, k = RM ? idx - p * d.nxh : idx / NB;
    const int ya = y0 + 2 * p, yb = ya + 1;
    const size_t oa = RM ? (size_t)ya * d.nxh + k : (size_t)k * d.ny + ya;
    const size_t ob = RM ? (size_t)yb * d.nxh + k : (size_t)k * d.ny + yb;
    C h1 = ya < d.ny ? src[oa] : mkc<C>(0, 0);
    C h2 = yb < d.ny ? src[ob] : mkc<C>(0, 0);
    if (k == 0) {
      h1.y = T(0);
      h2.y = T(0);
    }
    // Z = X1 + i X2 with X[k] = h, X[L-k] = conj(h)
    b0[p * L + k] = mkc<C>(h1.x - h2.y, h1.y + h2.x);
    if (k > 0) b0[p * L + (L - k)] = mkc<C>(h1.x + h2.y, -h1.y + h2.x);
  }
  __syncthreads();
  C* r = fft_any<T, +1, LC>(b0, b1, NB, pl, tw);
  T* dst = phys + (size_t)plane * d.ny * d.nx;
  for (int idx = threadIdx.x; idx < NB * L; idx += blockDim.x) {
    const int p = idx / L, x = idx - p * L;
    const int ya = y0 + 2 * p, yb = ya + 1;
    C z = r[idx];
    if (ya < d.ny) dst[(size_t)ya * d.nx + x] = z.x;
    if (yb < d.ny) dst[(size_t)yb * d.nx + x] = z.y;
  }
}

// Per-precision access widths of the p2 kernels' staged paths (the lengths
// below 16 or 32 and the FP64 backward x pass; longer rows and columns form
// their first radix-16 butterfly from per-thread loads).  FP32: 16-byte
// vectors (four reals of a row, two complex values of a column) and the
// backward intermediate row-major [plane][y][kx], so that the backward x pass
// reads contiguous row blocks.  FP64: one real / one complex value per access
// and the backward intermediate [plane][kx][y] (measured faster for 16-byte
// complex values, whose accesses are already wide).
template <typename T> struct P2Vec;
template <> struct P2Vec<float> {
  using R = float4;   // VW reals of a row
  using CV = float4;  // VC complex values of a column
  static constexpr int VW = 4, VC = 2;
  static constexpr bool kBwdRowMajor = bwd_row_major<float>();
};
template <> struct P2Vec<double> {
  using R = double;
  using CV = double2;
  static constexpr int VW = 1, VC = 1;
  static constexpr bool kBwdRowMajor = bwd_row_major<double>();
};
__device__ __forceinline__ float vget(const float4& v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }
__device__ __forceinline__ double vget(const double& v, int) { return v; }
__device__ __forceinline__ void vset(float4& v, int j, float a) {
  if (j == 0) v.x = a; else if (j == 1) v.y = a; else if (j == 2) v.z = a; else v.w = a;
}
__device__ __forceinline__ void vset(double& v, int, double a) { v = a; }
__device__ __forceinline__ float2 cget(const float4& v, int j) { return j == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w); }
__device__ __forceinline__ double2 cget(const double2& v, int) { return v; }
__device__ __forceinline__ void cset(float4& v, int j, float2 a) {
  if (j == 0) { v.x = a.x; v.y = a.y; } else { v.z = a.x; v.w = a.y; }
}
__device__ __forceinline__ void cset(double2& v, int, double2 a) { v = a; }
template <typename V> __device__ __forceinline__ V vzero() { V v; memset(&v, 0, sizeof(V)); return v; }

// forward x pass, L = nx: NB row pairs per CTA, 2 rows packed per complex FFT
template <typename T, int L, int NB, bool PROD>
__global__ void __launch_bounds__(NB * L / 16) fx_p2_kernel(TransformDims d, const cplx<T>* __restrict__ tw,
                                                           const T* __restrict__ phys, cplx<T>* __restrict__ work,
                                                           PhysProduct prod) {
  using C = cplx<T>;
  using PV = P2Vec<T>;
  using R = typename PV::R;
  constexpr int VW = PV::VW, RS = P2<L>::RS, NT = NB * L / 16, rows = 2 * NB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  int plane = blockIdx.y;
  const int y0 = blockIdx.x * rows;
  const T* src;
  const T* srcb = nullptr;
  T shb = T(0);
  if constexpr (PROD) {  // planes z-major: z = blockIdx.y / nf, field f; output plane f*nz + z
    const int z = plane / prod.nf, f = plane - z * prod.nf;
    src = reinterpret_cast<const T*>(prod.a[f]) + (size_t)z * d.ny * L;
    if (prod.b[f]) srcb = reinterpret_cast<const T*>(prod.b[f]) + (size_t)z * d.ny * L;
    shb = (T)prod.sh[f];
    plane = f * d.nz + z;
  } else {
    src = phys + (size_t)plane * d.ny * L;
  }
  if constexpr (L >= 16) {
    {
      // the first radix-16 pass straight from the rows: thread (b, j) takes the
      // 16 values x = j + r * L/16 of row pair b (for each r the threads of a
      // row pair read 16 consecutive reals), so the tile is not staged in
      // shared memory before the pass; one butterfly per thread (NT = NB * L/16)
      constexpr int nb = L / 16;
      const int b = threadIdx.x / nb, j = threadIdx.x - b * nb;
      const int ya = y0 + 2 * b, yb = ya + 1;
      const bool oka = ya < d.ny, okb = yb < d.ny;
      const T* ra = src + (size_t)(oka ? ya : 0) * L + j;
      const T* rb = src + (size_t)(okb ? yb : 0) * L + j;
      T va[16], vb[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) {   // every load in flight before the first use
        va[r] = oka ? ra[r * nb] : T(0);
        vb[r] = okb ? rb[r * nb] : T(0);
      }
      if constexpr (PROD) {
        if (srcb) {  // a * (b + shift), the products of the reference's physical-space step
          const T* wa = srcb + (size_t)(oka ? ya : 0) * L + j;
          const T* wb = srcb + (size_t)(okb ? yb : 0) * L + j;
          T xa[16], xb[16];
#pragma unroll
          for (int r = 0; r < 16; ++r) {
            xa[r] = oka ? wa[r * nb] : T(0);
            xb[r] = okb ? wb[r * nb] : T(0);
          }
#pragma unroll
          for (int r = 0; r < 16; ++r) {
            va[r] = va[r] * (xa[r] + shb);
            vb[r] = vb[r] * (xb[r] + shb);
          }
        }
      }
      C v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = mkc<C>(va[r], vb[r]);
      dft_ct<16, -1>(v);
      C* row = buf + b * RS;
#pragma unroll
      for (int k = 0; k < 16; ++k) row[sp(16 * j + k)] = v[k];
    }
    __syncthreads();
    ip_passes<T, -1, L, NB, 16>(buf, tw);
  } else {  // L = 8: one radix-8 pass, two butterflies a thread
    {
      constexpr int IT = NB * L / (NT * VW);  // every load of the tile in flight before the first shared store
      R va[IT], vb[IT];
      R wa[PROD ? IT : 1], wb[PROD ? IT : 1];
#pragma unroll
      for (int i = 0; i < IT; ++i) {
        const int e = (threadIdx.x + i * NT) * VW;
        const int p = e / L, x = e % L;
        const int ya = y0 + 2 * p, yb = ya + 1;
        va[i] = ya < d.ny ? *reinterpret_cast<const R*>(src + (size_t)ya * L + x) : vzero<R>();
        vb[i] = yb < d.ny ? *reinterpret_cast<const R*>(src + (size_t)yb * L + x) : vzero<R>();
        if constexpr (PROD) {
          if (srcb) {
            wa[i] = ya < d.ny ? *reinterpret_cast<const R*>(srcb + (size_t)ya * L + x) : vzero<R>();
            wb[i] = yb < d.ny ? *reinterpret_cast<const R*>(srcb + (size_t)yb * L + x) : vzero<R>();
          }
        }
      }
      if constexpr (PROD) {
        if (srcb) {  // a * (b + shift), the products of the reference's physical-space step
#pragma unroll
          for (int i = 0; i < IT; ++i)
#pragma unroll
            for (int j = 0; j < VW; ++j) {
              vset(va[i], j, vget(va[i], j) * (vget(wa[i], j) + shb));
              vset(vb[i], j, vget(vb[i], j) * (vget(wb[i], j) + shb));
            }
        }
      }
#pragma unroll
      for (int i = 0; i < IT; ++i) {
        const int e = (threadIdx.x + i * NT) * VW;
        const int p = e / L, x = e % L;
#pragma unroll
        for (int j = 0; j < VW; ++j) buf[p * RS + sp(x + j)] = mkc<C>(vget(va[i], j), vget(vb[i], j));
      }
    }
    __syncthreads();
    ip_passes<T, -1, L, NB, 1>(buf, tw);
  }
  C* dst = work + (size_t)plane * d.nxh * d.ny;
  for (int idx = threadIdx.x; idx < rows * d.nxh; idx += NT) {
    const int k = idx / rows, q = idx % rows;
    const int y = y0 + q;
    if (y >= d.ny) continue;
    const C* row = buf + (q >> 1) * RS;
    const C Z = row[sp(k)];
    const C Zc = cconj(row[sp(k == 0 ? 0 : L - k)]);
    C X;
    if ((q & 1) == 0) {
      X = mkc<C>((Z.x + Zc.x) * T(0.5), (Z.y + Zc.y) * T(0.5));
    } else {
      const C D = csub(Z, Zc);
      X = mkc<C>(D.y * T(0.5), -D.x * T(0.5));
    }
    dst[(size_t)k * d.ny + y] = X;
  }
}

// forward y pass, L = ny: NB kx columns per CTA, pruned FP64 output scaled by 1/(Nx*Ny)
template <typename T, int L, int NB>
__global__ void __launch_bounds__(NB * L / 16) fy_p2_kernel(TransformDims d, const cplx<T>* __restrict__ tw,
                                                           const cplx<T>* __restrict__ work,
                                                           double2* __restrict__ spec, double scale) {
  using C = cplx<T>;
  using PV = P2Vec<T>;
  using CV = typename PV::CV;
  constexpr int VC = PV::VC, RS = P2<L>::RS, NT = NB * L / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int plane = blockIdx.y;
  const int k0 = blockIdx.x * NB;
  const C* src = work + (size_t)plane * d.nxh * L;
  constexpr int nyc = L / 3 * 2;   // d.nyc of a power-of-two Ny = L
  if constexpr (L >= 32) {
    // the first radix-16 pass straight from the columns (thread (c, j) takes
    // y = j + r * L/16 of column c) and the last one writing the kept modes
    // itself: the column is staged in shared memory only between the two
    constexpr int nb = L / 16;
    const int c = threadIdx.x / nb, j = threadIdx.x - c * nb;
    const bool okc = k0 + c < d.nxh;
    const C* col = src + (size_t)(okc ? k0 + c : 0) * L + j;
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = okc ? col[r * nb] : mkc<C>(0, 0);
    dft_ct<16, -1>(v);
    C* row = buf + c * RS;
#pragma unroll
    for (int k = 0; k < 16; ++k) row[sp(16 * j + k)] = v[k];
    __syncthreads();
    ip_passes<T, -1, L, NB, 16, NT, last_stride(L)>(buf, tw);
    double2* dst = spec + (size_t)plane * d.M;
    last_pass_out<T, -1, L, NB, NT>(buf, tw, [&](int cc, int y, int, C z) {
      const int k = k0 + cc;
      const bool lo = y < nyc / 2, hi = y >= L - nyc / 2;   // kept spectral rows
      if (k < d.nxh && (lo || hi)) {
        const int iy = lo ? y : y - (L - nyc);
        dst[iy + (size_t)nyc * k] = make_double2((double)z.x * scale, (double)z.y * scale);
      }
    });
    return;
  }
  {
    constexpr int IT = NB * L / (NT * VC);
    CV v[IT];
#pragma unroll
    for (int i = 0; i < IT; ++i) {
      const int e = (threadIdx.x + i * NT) * VC;
      const int c = e / L, y = e % L;
      v[i] = k0 + c < d.nxh ? *reinterpret_cast<const CV*>(src + (size_t)(k0 + c) * L + y) : vzero<CV>();
    }
#pragma unroll
    for (int i = 0; i < IT; ++i) {
      const int e = (threadIdx.x + i * NT) * VC;
      const int c = e / L, y = e % L;
#pragma unroll
      for (int j = 0; j < VC; ++j) buf[c * RS + sp(y + j)] = cget(v[i], j);
    }
  }
  __syncthreads();
  ip_passes<T, -1, L, NB, 1>(buf, tw);
  double2* dst = spec + (size_t)plane * d.M;
  for (int idx = threadIdx.x; idx < NB * nyc; idx += NT) {
    const int c = idx / nyc, iy = idx - c * nyc;
    const int k = k0 + c;
    if (k >= d.nxh) break;
    const C v = buf[c * RS + sp(y_of(iy, L, nyc))];
    dst[iy + (size_t)nyc * k] = make_double2((double)v.x * scale, (double)v.y * scale);
  }
}

// backward y pass: zero-filled pruned modes, unscaled
template <typename T, int L, int NB, bool GATHER>
__global__ void __launch_bounds__(NB * L / 16) by_p2_kernel(TransformDims d, const cplx<T>* __restrict__ tw,
                                                           const double2* __restrict__ spec,
                                                           cplx<T>* __restrict__ work, SpecGather gat) {
  using C = cplx<T>;
  constexpr int RS = P2<L>::RS, NT = NB * L / 16;
  constexpr bool RM = P2Vec<T>::kBwdRowMajor;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int plane = blockIdx.y;
  const int k0 = blockIdx.x * NB;
  constexpr int nyc = L / 3 * 2;   // d.nyc of a power-of-two Ny = L
  int deriv = 0;
  const double2* src = GATHER ? gather_src(gat, plane, d.nz, d.M, deriv) : spec + (size_t)plane * d.M;
  if constexpr (L >= 16 && !GATHER) {
    // the first radix-16 pass straight from the spectral columns: thread
    // (c, j) takes y = j + r * L/16 of column c (zero between the kept
    // bands), so the column is not staged in shared memory before the pass.
    // (The gathered form keeps the staged load: its derivative factors made
    // the per-thread loads slower than the one contiguous run.)
    constexpr int nb = L / 16;
    const int c = threadIdx.x / nb, j = threadIdx.x - c * nb;
    const int k = k0 + c;
    const bool okc = k < d.nxh;
    const double2* col = src + (size_t)(okc ? k : 0) * nyc;
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int y = j + r * nb;
      const bool lo = y < nyc / 2, hi = y >= L - nyc / 2;
      const int iy = lo ? y : y - (L - nyc);
      const bool ok = okc && (lo || hi);
      double2 w = ok ? col[iy] : make_double2(0.0, 0.0);
      v[r] = mkc<C>((T)w.x, (T)w.y);
    }
    dft_ct<16, +1>(v);
    C* row = buf + c * RS;
#pragma unroll
    for (int q = 0; q < 16; ++q) row[sp(16 * j + q)] = v[q];
    __syncthreads();
    ip_passes<T, +1, L, NB, 16>(buf, tw);
  } else {
    constexpr int gap = L - nyc;  // FFT indices [nyc/2, L - nyc/2) carry no spectral row
    for (int idx = threadIdx.x; idx < NB * gap; idx += NT) {
      const int c = idx / gap, y = nyc / 2 + (idx - c * gap);
      buf[c * RS + sp(y)] = mkc<C>(0, 0);
    }
    if constexpr (RM) {
      // the NB columns are one contiguous run of NB*nyc coefficients; every
      // load in flight before the first shared store
      constexpr int IT = (NB * (L / 3 * 2) + NT - 1) / NT;  // nyc = L/3*2
      const int run = min(NB, d.nxh - k0) * nyc;
      const double2* s0 = src + (size_t)k0 * nyc;
      double2 v[IT];
      double kf[GATHER ? IT : 1];   // wavenumber of a derivative, loaded with the coefficient
#pragma unroll
      for (int i = 0; i < IT; ++i) {
        const int idx = threadIdx.x + i * NT;
        v[i] = idx < run ? s0[idx] : make_double2(0.0, 0.0);
        if constexpr (GATHER) {
          const double* kt = deriv == 1 ? gat.kx : gat.ky;
          kf[i] = (deriv != 0 && idx < run) ? kt[k0 * nyc + idx] : 0.0;
        }
      }
#pragma unroll
      for (int i = 0; i < IT; ++i) {
        const int idx = threadIdx.x + i * NT;
        if (idx < NB * nyc) {
          const int c = idx / nyc, iy = idx - c * nyc;
          double2 w = v[i];
          if constexpr (GATHER) {
            if (deriv != 0) w = make_double2(0.0 * v[i].x - kf[i] * v[i].y, 0.0 * v[i].y + kf[i] * v[i].x);
          }
          buf[c * RS + sp(y_of(iy, L, nyc))] = mkc<C>((T)w.x, (T)w.y);
        }
      }
    } else {
#pragma unroll 4
      for (int idx = threadIdx.x; idx < NB * nyc; idx += NT) {
        const int c = idx / nyc, iy = idx - c * nyc;
        const int k = k0 + c;
        const int m = iy + nyc * k;
        double2 v = k < d.nxh ? (GATHER ? gather_value(gat, deriv, m, src[m]) : src[m]) : make_double2(0.0, 0.0);
        buf[c * RS + sp(y_of(iy, L, nyc))] = mkc<C>((T)v.x, (T)v.y);
      }
    }
    __syncthreads();
    ip_passes<T, +1, L, NB, 1>(buf, tw);
  }
  C* dst = work + (size_t)plane * d.nxh * L;
  if constexpr (RM) {
    // [plane][y][kx]: rows of NB kx values
#pragma unroll 4
    for (int idx = threadIdx.x; idx < NB * L; idx += NT) {
      const int y = idx / NB, c = idx % NB;
      if (k0 + c < d.nxh) dst[(size_t)y * d.nxh + k0 + c] = buf[c * RS + sp(y)];
    }
  } else {
    // [plane][kx][y]: NB contiguous columns
#pragma unroll 4
    for (int idx = threadIdx.x; idx < NB * L; idx += NT) {
      const int c = idx / L, y = idx % L;
      if (k0 + c < d.nxh) dst[(size_t)(k0 + c) * L + y] = buf[c * RS + sp(y)];
    }
  }
}

// backward x pass, L = nx: two rows per complex FFT; Im of the kx = 0 coefficient ignored (c2r).
// Backward x pass, first radix-16 pass straight from the row-major work
// plane (FP32 layout [plane][y][kx], L >= 16): thread (b, j) forms Z[x] =
// X1[x] + i X2[x] of row pair b at x = j + r * L/16 (X[L-k] = conj X[k]; zero
// between the kept bands; Im of kx = 0 ignored), transforms the 16 values and
// stores the pass's outputs in buf, so the packed rows are never staged in
// shared memory before the pass.  One butterfly per thread (NB * L/16
// threads); the caller synchronises and runs the passes of stride 16 on.
template <typename T, int L, int NB>
__device__ __forceinline__ void bx_first_pass(cplx<T>* buf, const TransformDims& d,
                                              const cplx<T>* __restrict__ work, int plane, int y0) {
  using C = cplx<T>;
  constexpr int RS = P2<L>::RS;
  constexpr int nb = L / 16, nxh = L / 3 * 2 / 2 + 1;
  const int b = threadIdx.x / nb, j = threadIdx.x - b * nb;
  const int ya = y0 + 2 * b, yb = ya + 1;
  const bool oka = ya < d.ny, okb = yb < d.ny;
  const C* src = work + (size_t)plane * nxh * d.ny;
  const C* r1 = src + (size_t)(oka ? ya : 0) * nxh;
  const C* r2 = src + (size_t)(okb ? yb : 0) * nxh;
  C v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int x = j + r * nb;
    const bool lo = x < nxh, hi = x > L - nxh;
    const int k = lo ? x : L - x;
    C a = (oka && (lo || hi)) ? r1[k] : mkc<C>(0, 0);
    C c = (okb && (lo || hi)) ? r2[k] : mkc<C>(0, 0);
    if (x == 0) a.y = c.y = T(0);
    v[r] = lo ? mkc<C>(a.x - c.y, a.y + c.x) : mkc<C>(a.x + c.y, -a.y + c.x);
  }
  dft_ct<16, +1>(v);
  C* row = buf + b * RS;
#pragma unroll
  for (int k = 0; k < 16; ++k) row[sp(16 * j + k)] = v[k];
}

// Backward x pass, loading half: the zero gap and the row pairs of one work
// plane combined into the packed two-row FFT input in buf (shared memory).
template <typename T, int L, int NB>
__device__ __forceinline__ void bx_fill(cplx<T>* buf, const TransformDims& d, const cplx<T>* __restrict__ work,
                                        int plane, int y0) {
  using C = cplx<T>;
  using PV = P2Vec<T>;
  constexpr int RS = P2<L>::RS, NT = NB * L / 16, rows = 2 * NB;
  constexpr int nxh = L / 3 * 2 / 2 + 1;   // d.nxh of a power-of-two Nx = L
  constexpr int gap = L - 2 * nxh + 1;  // FFT indices [nxh, L - nxh] are zero
  for (int idx = threadIdx.x; idx < NB * gap; idx += NT) {
    const int p = idx / gap, x = nxh + (idx - p * gap);
    buf[p * RS + sp(x)] = mkc<C>(0, 0);
  }
  if constexpr (PV::kBwdRowMajor) {
    // [plane][y][kx]: the 2*NB rows of the CTA are one contiguous block; each
    // thread loads one kx of a row pair (rows 2p, 2p+1) and forms Z[k], Z[L-k]
    const C* src = work + (size_t)plane * nxh * d.ny + (size_t)y0 * nxh;
    const int total = NB * nxh;
    constexpr int IT = (NB * (L / 3 + 1) + NT - 1) / NT;  // nxh <= L/3 + 1
    C h1[IT], h2[IT];
#pragma unroll
    for (int i = 0; i < IT; ++i) {  // every load in flight before the pairs are combined
      const int idx = threadIdx.x + i * NT;
      const int p = idx / nxh, k = idx - p * nxh;
      const int ya = y0 + 2 * p;
      h1[i] = (idx < total && ya < d.ny) ? src[(size_t)(2 * p) * nxh + k] : mkc<C>(0, 0);
      h2[i] = (idx < total && ya + 1 < d.ny) ? src[(size_t)(2 * p + 1) * nxh + k] : mkc<C>(0, 0);
    }
#pragma unroll
    for (int i = 0; i < IT; ++i) {
      const int idx = threadIdx.x + i * NT;
      if (idx < total) {
        const int p = idx / nxh, k = idx - p * nxh;
        C a = h1[i], b = h2[i];
        if (k == 0) a.y = b.y = T(0);
        C* row = buf + p * RS;
        row[sp(k)] = mkc<C>(a.x - b.y, a.y + b.x);                  // Z[k] = X1[k] + i X2[k]
        if (k > 0) row[sp(L - k)] = mkc<C>(a.x + b.y, -a.y + b.x);  // Z[L-k] = conj(X1[k]) + i conj(X2[k])
      }
    }
  } else {
    // [plane][kx][y]: each thread loads one coefficient (coalesced along y);
    // the row pair is combined across adjacent lanes
    const C* src = work + (size_t)plane * nxh * d.ny;
    const int total = rows * nxh;  // even; the pair (2p, 2p+1) sits in adjacent lanes
    constexpr int IT = (rows * (L / 3 + 1) + NT - 1) / NT;
    C hv[IT];
#pragma unroll
    for (int i = 0; i < IT; ++i) {
      const int idx = threadIdx.x + i * NT;
      const int k = idx / rows, q = idx % rows;
      hv[i] = (idx < total && y0 + q < d.ny) ? src[(size_t)k * d.ny + y0 + q] : mkc<C>(0, 0);
    }
#pragma unroll
    for (int i = 0; i < IT; ++i) {
      const int idx = threadIdx.x + i * NT;
      const bool ok = idx < total;
      const int k = idx / rows, q = idx % rows;
      C h = hv[i];
      if (k == 0) h.y = T(0);
      C o;
      o.x = __shfl_xor_sync(0xffffffffu, h.x, 1);
      o.y = __shfl_xor_sync(0xffffffffu, h.y, 1);
      if (ok) {
        C* row = buf + (q >> 1) * RS;
        if ((q & 1) == 0) {  // Z[k] = X1[k] + i X2[k], h1 = h, h2 = o
          row[sp(k)] = mkc<C>(h.x - o.y, h.y + o.x);
        } else if (k > 0) {  // Z[L-k] = conj(X1[k]) + i conj(X2[k]), h1 = o, h2 = h
          row[sp(L - k)] = mkc<C>(o.x + h.y, -o.y + h.x);
        }
      }
    }
  }
}

template <typename T, int L, int NB>
__global__ void __launch_bounds__(NB * L / 16) bx_p2_kernel(TransformDims d, const cplx<T>* __restrict__ tw,
                                                           const cplx<T>* __restrict__ work, T* __restrict__ phys) {
  using C = cplx<T>;
  using PV = P2Vec<T>;
  using R = typename PV::R;
  constexpr int VW = PV::VW, RS = P2<L>::RS, NT = NB * L / 16, rows = 2 * NB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int plane = blockIdx.y;
  const int y0 = blockIdx.x * rows;
  T* dst = phys + (size_t)plane * d.ny * L;
  if constexpr (L >= 32 && PV::kBwdRowMajor) {
    bx_first_pass<T, L, NB>(buf, d, work, plane, y0);
    __syncthreads();
    ip_passes<T, +1, L, NB, 16, NT, last_stride(L)>(buf, tw);
    last_pass_out<T, +1, L, NB, NT>(buf, tw, [&](int p, int x, int, C z) {
      const int ra = y0 + 2 * p, rb = ra + 1;
      if (ra < d.ny) dst[(size_t)ra * L + x] = z.x;
      if (rb < d.ny) dst[(size_t)rb * L + x] = z.y;
    });
    return;
  }
  bx_fill<T, L, NB>(buf, d, work, plane, y0);
  __syncthreads();
  if constexpr (L >= 16) {
    // the last pass writes the rows itself (threads of a row pair store
    // consecutive x), so its outputs are not staged in shared memory
    ip_passes<T, +1, L, NB, 1, NT, last_stride(L)>(buf, tw);
    last_pass_out<T, +1, L, NB, NT>(buf, tw, [&](int p, int x, int, C z) {
      const int ya = y0 + 2 * p, yb = ya + 1;
      if (ya < d.ny) dst[(size_t)ya * L + x] = z.x;
      if (yb < d.ny) dst[(size_t)yb * L + x] = z.y;
    });
  } else {
    ip_passes<T, +1, L, NB, 1>(buf, tw);
    constexpr int IS = NB * L / (NT * VW);
#pragma unroll 4
    for (int i = 0; i < IS; ++i) {
      const int e = (threadIdx.x + i * NT) * VW;
      const int p = e / L, x = e % L;
      const int ya = y0 + 2 * p, yb = ya + 1;
      R ra, rb;
#pragma unroll
      for (int j = 0; j < VW; ++j) {
        const C z = buf[p * RS + sp(x + j)];
        vset(ra, j, z.x);
        vset(rb, j, z.y);
      }
      if (ya < d.ny) *reinterpret_cast<R*>(dst + (size_t)ya * L + x) = ra;
      if (yb < d.ny) *reinterpret_cast<R*>(dst + (size_t)yb * L + x) = rb;
    }
  }
}

// Backward x pass of ncomp groups of three gradient fields (work planes
// (3c + j) * nz + z), each group reduced to the advection term
//   out_c = (u + su) d_c/dx + (v + sv) d_c/dy + (w + sw) d_c/dz
// of the advective nonlinear form (phase_carrier_flat.cc:786-797,
// phase_scalar_flat.cc:588-591), so the nine physical gradient fields are
// never written.  grid: (row blocks x ncomp, nz) with the component fastest:
// the ncomp CTAs of one row block run together, so the velocity rows they
// share come from DRAM once and from L2 after; unl: the physical velocity.
// FP32: registers capped for about 640 threads per SM (measured best).
template <typename T, int L, int NB>
__global__ void __launch_bounds__(NB * L / 16, sizeof(T) == 4 ? 640 / (NB * L / 16) : 1) bx_adv_p2_kernel(TransformDims d, const cplx<T>* __restrict__ tw,
                                                               const cplx<T>* __restrict__ work,
                                                               const T* __restrict__ unl, T* __restrict__ out,
                                                               size_t P, int ncomp, double su, double sv, double sw) {
  using C = cplx<T>;
  using PV = P2Vec<T>;
  using R = typename PV::R;
  constexpr int VW = PV::VW, RS = P2<L>::RS, NT = NB * L / 16, rows = 2 * NB;
  constexpr int IS = NB * L / (NT * VW);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int z = blockIdx.y, c = blockIdx.x % ncomp;
  const int y0 = (blockIdx.x / ncomp) * rows;
  const size_t zoff = (size_t)z * d.ny * L;
  R acca[IS], accb[IS];
#pragma unroll
  for (int i = 0; i < IS; ++i) acca[i] = accb[i] = vzero<R>();
#pragma unroll 1
  for (int j = 0; j < 3; ++j) {
    if (j > 0) __syncthreads();   // buf is refilled
    if constexpr (L >= 16 && PV::kBwdRowMajor) {
      bx_first_pass<T, L, NB>(buf, d, work, (3 * c + j) * d.nz + z, y0);
      __syncthreads();
      ip_passes<T, +1, L, NB, 16>(buf, tw);
    } else {
      bx_fill<T, L, NB>(buf, d, work, (3 * c + j) * d.nz + z, y0);
      __syncthreads();
      ip_passes<T, +1, L, NB, 1>(buf, tw);
    }
    const T* uj = unl + (size_t)j * P + zoff;
    const T sh = (T)(j == 0 ? su : j == 1 ? sv : sw);
#pragma unroll
    for (int i = 0; i < IS; ++i) {
      const int e = (threadIdx.x + i * NT) * VW;
      const int p = e / L, x = e % L;
      const int ya = y0 + 2 * p, yb = ya + 1;
      const R ua = ya < d.ny ? *reinterpret_cast<const R*>(uj + (size_t)ya * L + x) : vzero<R>();
      const R ub = yb < d.ny ? *reinterpret_cast<const R*>(uj + (size_t)yb * L + x) : vzero<R>();
#pragma unroll
      for (int q = 0; q < VW; ++q) {
        const C g = buf[p * RS + sp(x + q)];
        vset(acca[i], q, vget(acca[i], q) + (vget(ua, q) + sh) * g.x);
        vset(accb[i], q, vget(accb[i], q) + (vget(ub, q) + sh) * g.y);
      }
    }
  }
  T* dst = out + (size_t)c * P + zoff;
#pragma unroll
  for (int i = 0; i < IS; ++i) {
    const int e = (threadIdx.x + i * NT) * VW;
    const int p = e / L, x = e % L;
    const int ya = y0 + 2 * p, yb = ya + 1;
    if (ya < d.ny) *reinterpret_cast<R*>(dst + (size_t)ya * L + x) = acca[i];
    if (yb < d.ny) *reinterpret_cast<R*>(dst + (size_t)yb * L + x) = accb[i];
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static const size_t kFftSmemBudget = 64 * 1024;

static int pick_nb(int L, size_t csize) {
  const size_t budget = kFftSmemBudget;
  if (2 * (size_t)L * csize > budget)
    throw Error{TG_ERR_SHAPE, "RealCplxCube::DftForward > transform length too large for one CTA"};
  int nb = (int)(budget / (2 * (size_t)L * csize));
  if (nb > 16) nb = 16;
  if (nb < 1) nb = 1;
  return nb;
}

// lengths with a compile-time specialisation (powers of two); others use LC = 0
#define TG_FFT_LENGTHS(X) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)

#define TG_FFT_DISPATCH(L, CALL)          \
  switch (L) {                            \
    case 8: CALL(8); break;               \
    case 16: CALL(16); break;             \
    case 32: CALL(32); break;             \
    case 64: CALL(64); break;             \
    case 128: CALL(128); break;           \
    case 256: CALL(256); break;           \
    case 512: CALL(512); break;           \
    case 1024: CALL(1024); break;         \
    default: CALL(0); break;              \
  }

template <typename Kern>
static void set_smem(Kern k) {
  TG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFftSmemBudget));
}

template <typename T, int LC>
static void set_smem_all() {
  set_smem(fwd_x_kernel<T, LC>);
  set_smem(fwd_y_kernel<T, LC>);
  set_smem(bwd_y_kernel<T, LC, false>);
  set_smem(bwd_y_kernel<T, LC, true>);
  set_smem(bwd_x_kernel<T, LC>);
}

void fft_init() {
#define TG_INIT_L(L)          \
  set_smem_all<double, L>(); \
  set_smem_all<float, L>();
  TG_FFT_LENGTHS(TG_INIT_L)
#undef TG_INIT_L
  set_smem_all<double, 0>();
  set_smem_all<float, 0>();
}

static bool p2_length(int L) { return L >= 8 && L <= 1024 && (L & (L - 1)) == 0; }
static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

#define TG_P2_DISPATCH(L, CALL) \
  switch (L) {                  \
    case 8: CALL(8); break;     \
    case 16: CALL(16); break;   \
    case 32: CALL(32); break;   \
    case 64: CALL(64); break;   \
    case 128: CALL(128); break; \
    case 256: CALL(256); break; \
    case 512: CALL(512); break; \
    case 1024: CALL(1024); break; \
  }

// complex values per CTA of each power-of-two pass (measured at 256^2
// planes: FP32 x and y passes 2048, the backward x pass 1024 -- smaller CTAs
// keep more of them in flight per SM; FP64 2048 for all)
enum P2Kind { P2_FX, P2_FY, P2_BY, P2_BX };
template <typename T, int KIND> struct P2Elems {
  static constexpr int value = sizeof(T) == 8 ? 2048 : KIND == P2_BX ? 1024 : 2048;
};

template <typename T, int L, int KIND>
static size_t p2_smem() {
  return (size_t)(P2Elems<T, KIND>::value / L) * P2<L>::RS * sizeof(cplx<T>);
}

template <typename T>
bool dft_forward_products_ok(const TransformDims& d, const FftPlan& px, const PhysProduct& prod) {
  if (!p2_length(px.L) || d.nxh != px.L / 3 * 2 / 2 + 1 || prod.nf < 1 || prod.nf > kMaxGather) return false;
  for (int f = 0; f < prod.nf; ++f)
    if (!prod.a[f] || !aligned16(prod.a[f]) || (prod.b[f] && !aligned16(prod.b[f]))) return false;
  return true;
}

template <typename T>
void dft_forward(const TransformDims& d, const FftPlan& px, const FftPlan& py, const T* phys, double2* spec,
                 int planes, void* work, cudaStream_t s, const PhysProduct* prod) {
  using C = cplx<T>;
  C* w = reinterpret_cast<C*>(work);
  PhysProduct pp{};
  if (prod) {
    if (!dft_forward_products_ok<T>(d, px, *prod) || planes != prod->nf * d.nz)
      throw Error{TG_ERR_SHAPE, "RealCplxCube::DftForward > products on load need a power-of-two Nx"};
    pp = *prod;
  }
  {
    prof_begin(s, PC_FFT_FX, (double)planes * d.ny * (d.nx * sizeof(T) + d.nxh * sizeof(C)), 0);
    const C* tw = Tw<T>::get(px);
    if (prod || (p2_length(px.L) && aligned16(phys) && d.nxh == px.L / 3 * 2 / 2 + 1)) {
#define TG_CALL(LL)                                                                         \
  {                                                                                         \
    constexpr int NB = P2Elems<T, P2_FX>::value / LL;                                                \
    dim3 grid((d.ny + 2 * NB - 1) / (2 * NB), planes);                                      \
    if (prod)                                                                               \
      fx_p2_kernel<T, LL, NB, true><<<grid, NB * LL / 16, p2_smem<T, LL, P2_FX>(), s>>>(d, tw, phys, w, pp); \
    else                                                                                    \
      fx_p2_kernel<T, LL, NB, false><<<grid, NB * LL / 16, p2_smem<T, LL, P2_FX>(), s>>>(d, tw, phys, w, pp); \
  }
      TG_P2_DISPATCH(px.L, TG_CALL)
#undef TG_CALL
    } else {
      int nb = pick_nb(px.L, sizeof(C));
      size_t sm = 2 * (size_t)nb * px.L * sizeof(C);
      dim3 grid((d.ny + 2 * nb - 1) / (2 * nb), planes);
      const PlanArgs pa = plan_args(px);
      fwd_x_kernel<T, 0><<<grid, 256, sm, s>>>(d, pa, tw, phys, w, nb);
    }
    prof_end(s);
    TG_LAUNCH_CHECK("fwd_x_kernel");
  }
  {
    const double scale = 1.0 / ((double)d.nx * (double)d.ny);
    prof_begin(s, PC_FFT_FY, (double)planes * ((double)d.nxh * d.ny * sizeof(C) + (double)d.M * sizeof(double2)), 0);
    const C* tw = Tw<T>::get(py);
    if (p2_length(py.L) && d.nyc == py.L / 3 * 2) {
#define TG_CALL(LL)                                                                              \
  {                                                                                              \
    constexpr int NB = P2Elems<T, P2_FY>::value / LL;                                                     \
    dim3 grid((d.nxh + NB - 1) / NB, planes);                                                    \
    fy_p2_kernel<T, LL, NB><<<grid, NB * LL / 16, p2_smem<T, LL, P2_FY>(), s>>>(d, tw, w, spec, scale); \
  }
      TG_P2_DISPATCH(py.L, TG_CALL)
#undef TG_CALL
    } else {
      int nb = pick_nb(py.L, sizeof(C));
      size_t sm = 2 * (size_t)nb * py.L * sizeof(C);
      dim3 grid((d.nxh + nb - 1) / nb, planes);
      const PlanArgs pa = plan_args(py);
      fwd_y_kernel<T, 0><<<grid, 256, sm, s>>>(d, pa, tw, w, spec, nb, scale);
    }
    prof_end(s);
    TG_LAUNCH_CHECK("fwd_y_kernel");
  }
}

template <typename T>
void dft_backward(const TransformDims& d, const FftPlan& px, const FftPlan& py, const double2* spec, T* phys,
                  int planes, void* work, cudaStream_t s, const SpecGather* gather) {
  SpecGather gat{};
  if (gather) gat = *gather;
  using C = cplx<T>;
  C* w = reinterpret_cast<C*>(work);
  {
    prof_begin(s, PC_FFT_BY, (double)planes * ((double)d.nxh * d.ny * sizeof(C) + (double)d.M * sizeof(double2)), 0);
    const C* tw = Tw<T>::get(py);
    if (p2_length(py.L) && d.nyc == py.L / 3 * 2) {
#define TG_CALL(LL)                                                                       \
  {                                                                                       \
    constexpr int NB = P2Elems<T, P2_BY>::value / LL;                                              \
    dim3 grid((d.nxh + NB - 1) / NB, planes);                                             \
    if (gather)                                                                                  \
      by_p2_kernel<T, LL, NB, true><<<grid, NB * LL / 16, p2_smem<T, LL, P2_BY>(), s>>>(d, tw, spec, w, gat); \
    else                                                                                        \
      by_p2_kernel<T, LL, NB, false><<<grid, NB * LL / 16, p2_smem<T, LL, P2_BY>(), s>>>(d, tw, spec, w, gat); \
  }
      TG_P2_DISPATCH(py.L, TG_CALL)
#undef TG_CALL
    } else {
      int nb = pick_nb(py.L, sizeof(C));
      size_t sm = 2 * (size_t)nb * py.L * sizeof(C);
      dim3 grid((d.nxh + nb - 1) / nb, planes);
      const PlanArgs pa = plan_args(py);
      if (gather)
        bwd_y_kernel<T, 0, true><<<grid, 256, sm, s>>>(d, pa, tw, spec, w, nb, gat);
      else
        bwd_y_kernel<T, 0, false><<<grid, 256, sm, s>>>(d, pa, tw, spec, w, nb, gat);
    }
    prof_end(s);
    TG_LAUNCH_CHECK("bwd_y_kernel");
  }
  {
    prof_begin(s, PC_FFT_BX, (double)planes * d.ny * (d.nx * sizeof(T) + d.nxh * sizeof(C)), 0);
    const C* tw = Tw<T>::get(px);
    if (p2_length(px.L) && aligned16(phys) && d.nxh == px.L / 3 * 2 / 2 + 1) {
#define TG_CALL(LL)                                                                       \
  {                                                                                       \
    constexpr int NB = P2Elems<T, P2_BX>::value / LL;                                              \
    dim3 grid((d.ny + 2 * NB - 1) / (2 * NB), planes);                                    \
    bx_p2_kernel<T, LL, NB><<<grid, NB * LL / 16, p2_smem<T, LL, P2_BX>(), s>>>(d, tw, w, phys); \
  }
      TG_P2_DISPATCH(px.L, TG_CALL)
#undef TG_CALL
    } else {
      int nb = pick_nb(px.L, sizeof(C));
      size_t sm = 2 * (size_t)nb * px.L * sizeof(C);
      dim3 grid((d.ny + 2 * nb - 1) / (2 * nb), planes);
      const PlanArgs pa = plan_args(px);
      bwd_x_kernel<T, 0><<<grid, 256, sm, s>>>(d, pa, tw, w, phys, nb);
    }
    prof_end(s);
    TG_LAUNCH_CHECK("bwd_x_kernel");
  }
}

template void dft_forward<double>(const TransformDims&, const FftPlan&, const FftPlan&, const double*, double2*, int,
                                  void*, cudaStream_t, const PhysProduct*);
template void dft_forward<float>(const TransformDims&, const FftPlan&, const FftPlan&, const float*, double2*, int,
                                 void*, cudaStream_t, const PhysProduct*);
template bool dft_backward_adv_ok<double>(const TransformDims&, const FftPlan&, const FftPlan&, const double*,
                                          const double*);
template bool dft_backward_adv_ok<float>(const TransformDims&, const FftPlan&, const FftPlan&, const float*,
                                         const float*);
template void dft_backward_adv<double>(const TransformDims&, const FftPlan&, const FftPlan&, const SpecGather&, int,
                                       const double*, double*, double, double, double, void*, cudaStream_t);
template void dft_backward_adv<float>(const TransformDims&, const FftPlan&, const FftPlan&, const SpecGather&, int,
                                      const float*, float*, double, double, double, void*, cudaStream_t);
template bool dft_forward_products_ok<double>(const TransformDims&, const FftPlan&, const PhysProduct&);
template bool dft_forward_products_ok<float>(const TransformDims&, const FftPlan&, const PhysProduct&);
template <typename T>
bool dft_backward_adv_ok(const TransformDims& d, const FftPlan& px, const FftPlan& py, const T* unl, const T* out) {
  return p2_length(px.L) && p2_length(py.L) && d.nxh == px.L / 3 * 2 / 2 + 1 && d.nyc == py.L / 3 * 2 &&
         aligned16(unl) && aligned16(out) && ((size_t)d.nx * d.ny * d.nz * sizeof(T)) % 16 == 0;
}

template <typename T>
void dft_backward_adv(const TransformDims& d, const FftPlan& px, const FftPlan& py, const SpecGather& grad, int ncomp,
                      const T* unl, T* out, double su, double sv, double sw, void* work, cudaStream_t s) {
  using C = cplx<T>;
  if (ncomp < 1 || ncomp > 3 || grad.nf != 3 * ncomp || !dft_backward_adv_ok<T>(d, px, py, unl, out))
    throw Error{TG_ERR_SHAPE, "RealCplxCube::DftBackward > advection on the x pass needs power-of-two Nx, Ny"};
  C* w = reinterpret_cast<C*>(work);
  const int planes = grad.nf * d.nz;
  {  // y pass of the gradient fields, derivatives formed on load
    prof_begin(s, PC_FFT_BY, (double)planes * ((double)d.nxh * d.ny * sizeof(C) + (double)d.M * sizeof(double2)), 0);
    const C* tw = Tw<T>::get(py);
    SpecGather gat = grad;
#define TG_CALL(LL)                                                                                         \
  {                                                                                                         \
    constexpr int NB = P2Elems<T, P2_BY>::value / LL;                                                       \
    dim3 grid((d.nxh + NB - 1) / NB, planes);                                                               \
    by_p2_kernel<T, LL, NB, true><<<grid, NB * LL / 16, p2_smem<T, LL, P2_BY>(), s>>>(d, tw, nullptr, w, gat); \
  }
    TG_P2_DISPATCH(py.L, TG_CALL)
#undef TG_CALL
    prof_end(s);
    TG_LAUNCH_CHECK("by_p2_kernel");
  }
  {  // x pass and the advection sums
    const size_t P = (size_t)d.nx * d.ny * d.nz;
    // per component: three gradient intermediates in, one field out; the velocity once
    prof_begin(s, PC_ADV,
               (double)d.nz * d.ny * (ncomp * (3.0 * d.nxh * sizeof(C) + 1.0 * d.nx * sizeof(T)) + 3.0 * d.nx * sizeof(T)),
               0);
    const C* tw = Tw<T>::get(px);
#define TG_CALL(LL)                                                                                  \
  {                                                                                                  \
    constexpr int NB = P2Elems<T, P2_BX>::value / LL;                                                \
    dim3 grid((d.ny + 2 * NB - 1) / (2 * NB) * ncomp, d.nz);                                         \
    bx_adv_p2_kernel<T, LL, NB><<<grid, NB * LL / 16, p2_smem<T, LL, P2_BX>(), s>>>(d, tw, w, unl, out, P, ncomp, su, sv, sw); \
  }
    TG_P2_DISPATCH(px.L, TG_CALL)
#undef TG_CALL
    prof_end(s);
    TG_LAUNCH_CHECK("bx_adv_p2_kernel");
  }
}

template void dft_backward<double>(const TransformDims&, const FftPlan&, const FftPlan&, const double2*, double*, int,
                                   void*, cudaStream_t, const SpecGather*);
template void dft_backward<float>(const TransformDims&, const FftPlan&, const FftPlan&, const double2*, float*, int,
                                  void*, cudaStream_t, const SpecGather*);

}  // namespace tg

// ===========================================================================
// Allocation-free forward transform: tg_dft_forward_f64_noalloc.
//
// Same kernels, twiddles and pruning as tg_dft_forward_f64, but nothing is
// allocated: the x->y intermediate lives in a file-scope device array, and
// the twiddle tables / y-index maps of every supported length are written
// once per device into file-scope device arrays.  Host code must not use the
// arrays' names as device addresses (they are host-side stand-ins); their
// device addresses are taken with cudaGetSymbolAddress in the per-device
// set-up below.
// ===========================================================================
namespace tg {
namespace {
constexpr size_t kNoAllocScratch = size_t(1) << 20;   // double2 elements = 16 MiB
constexpr int kNoAllocMinL = 8, kNoAllocMaxL = 1024;  // power-of-two lengths
constexpr int kNoAllocTable = 2 * kNoAllocMaxL;       // sum of all supported lengths
__device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratch];
__device__ __align__(256) double2 g_noalloc_tw[kNoAllocTable];
__device__ __align__(256) int g_noalloc_yidx[kNoAllocTable];

struct NoAllocDevice {
  bool ready = false;
  unsigned long long ctx_id = 0;   // context the tables were written in (0: unknown)
  double2* scratch = nullptr;
  double2* tw = nullptr;
  int* yidx = nullptr;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// table offset of length L: 8 + 16 + ... + L/2 == L - 8
inline int noalloc_offset(int L) { return L - kNoAllocMinL; }

bool is_supported_pow2(int L) { return L >= kNoAllocMinL && L <= kNoAllocMaxL && (L & (L - 1)) == 0; }

// Unique id of the calling thread's current CUDA context (cuCtxGetId through
// the runtime's driver entry points, so the library does not link libcuda), or
// 0 when there is none yet or the driver does not offer the call.
unsigned long long current_context_id() {
  typedef CUresult (*GetCurrentFn)(CUcontext*);
  typedef CUresult (*GetIdFn)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(f);
    (void)cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Per-device set-up, run by the first call on each device (device current).
// The table copies are synchronous host->device copies, which a stream capture
// does not allow: the first call on a device must come before any capture.
// A reset of the device (cudaDeviceReset, or the primary context released and
// created again) wipes the device arrays and their addresses; the set-up is
// repeated when the current context is not the one it ran in.
NoAllocDevice& noalloc_setup() {
  int dev = 0;
  TG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) throw Error{TG_ERR_ARG, "tg_dft_forward_f64_noalloc > device index out of range"};
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (d.ready && d.ctx_id == current_context_id()) return d;
  d.ready = false;
  std::vector<double2> tw(kNoAllocTable, make_double2(0.0, 0.0));
  std::vector<int> ym(kNoAllocTable, 0);
  for (int L = kNoAllocMinL; L <= kNoAllocMaxL; L *= 2) {
    const int off = noalloc_offset(L);
    for (int k = 0; k < L; ++k) {  // same evaluation as fft_plan_create
      long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)L;
      tw[off + k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    const int nyc = L / 3 * 2, h = nyc / 2;
    for (int iy = 0; iy < nyc; ++iy) ym[off + iy] = iy < h ? iy : L - (nyc - iy);
  }
  TG_CUDA(cudaMemcpyToSymbol(g_noalloc_tw, tw.data(), sizeof(double2) * kNoAllocTable));
  TG_CUDA(cudaMemcpyToSymbol(g_noalloc_yidx, ym.data(), sizeof(int) * kNoAllocTable));
  TG_CUDA(cudaGetSymbolAddress((void**)&d.scratch, g_noalloc_scratch));
  TG_CUDA(cudaGetSymbolAddress((void**)&d.tw, g_noalloc_tw));
  TG_CUDA(cudaGetSymbolAddress((void**)&d.yidx, g_noalloc_yidx));
  set_smem_all<double, 0>();
#define TG_INIT_L(L) set_smem_all<double, L>();
  TG_FFT_LENGTHS(TG_INIT_L)
#undef TG_INIT_L
  d.ctx_id = current_context_id();   // the copies above made the context current
  d.ready = true;
  return d;
}

PlanArgs pow2_plan(int L) {
  PlanArgs a{};
  a.L = L;
  a.npass = 0;
  int n = L;
  while (n % 4 == 0) {
    a.rad[a.npass++] = 4;
    n /= 4;
  }
  while (n % 2 == 0) {
    a.rad[a.npass++] = 2;
    n /= 2;
  }
  return a;
}

void noalloc_forward(int nx, int ny, int nz, const double* phys, double* spec, int dim, cudaStream_t s) {
  if (!is_supported_pow2(nx) || !is_supported_pow2(ny))
    throw Error{TG_ERR_SHAPE, "tg_dft_forward_f64_noalloc > nx and ny must be powers of two in [8, 1024]"};
  if (nz < 1 || dim < 1) throw Error{TG_ERR_SHAPE, "tg_dft_forward_f64_noalloc > nz and dim must be positive"};
  if (!phys || !spec) throw Error{TG_ERR_ARG, "tg_dft_forward_f64_noalloc > null field pointer"};
  NoAllocDevice& dv = noalloc_setup();
  TransformDims d{};
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.nxh = nx / 3 * 2 / 2 + 1;
  d.nyc = ny / 3 * 2;
  d.M = d.nyc * d.nxh;
  d.yidx = dv.yidx + noalloc_offset(ny);
  const size_t plane_work = (size_t)d.nxh * ny;   // x->y intermediate per plane
  const int chunk = (int)(kNoAllocScratch / plane_work);
  if (chunk < 1) throw Error{TG_ERR_SHAPE, "tg_dft_forward_f64_noalloc > plane larger than the static scratch"};
  const PlanArgs pax = pow2_plan(nx), pay = pow2_plan(ny);
  const double2* twx = dv.tw + noalloc_offset(nx);
  const double2* twy = dv.tw + noalloc_offset(ny);
  const int nbx = pick_nb(nx, sizeof(double2)), nby = pick_nb(ny, sizeof(double2));
  const size_t smx = 2 * (size_t)nbx * nx * sizeof(double2), smy = 2 * (size_t)nby * ny * sizeof(double2);
  const double scale = 1.0 / ((double)nx * (double)ny);
  const int planes = dim * nz;
  for (int p0 = 0; p0 < planes; p0 += chunk) {
    const int np = std::min(chunk, planes - p0);
    const double* in = phys + (size_t)p0 * nx * ny;
    double2* out = reinterpret_cast<double2*>(spec) + (size_t)p0 * d.M;
    dim3 gx((ny + 2 * nbx - 1) / (2 * nbx), np), gy((d.nxh + nby - 1) / nby, np);
#define TG_CALL(LC) fwd_x_kernel<double, LC><<<gx, 256, smx, s>>>(d, pax, twx, in, dv.scratch, nbx)
    TG_FFT_DISPATCH(nx, TG_CALL)
#undef TG_CALL
    TG_LAUNCH_CHECK("fwd_x_kernel (noalloc)");
#define TG_CALL(LC) fwd_y_kernel<double, LC><<<gy, 256, smy, s>>>(d, pay, twy, dv.scratch, out, nby, scale)
    TG_FFT_DISPATCH(ny, TG_CALL)
#undef TG_CALL
    TG_LAUNCH_CHECK("fwd_y_kernel (noalloc)");
  }
}
}  // namespace

}  // namespace tg

extern "C" TG_API tg_status tg_dft_forward_f64_noalloc(int nx, int ny, int nz, const double* phys, double* spec,
                                                       int dim, void* stream) {
  try {
    tg::noalloc_forward(nx, ny, nz, phys, spec, dim, reinterpret_cast<cudaStream_t>(stream));
    return TG_OK;
  } catch (const tg::Error& e) {
    tg::set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    tg::set_error(e.what());
    return TG_ERR_CUDA;
  }
}
