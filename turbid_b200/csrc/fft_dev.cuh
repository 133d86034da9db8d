// Device building blocks of the transform kernels: twiddle access, the small
// DFTs of the compile-time passes, and the in-place radix-16 passes on padded
// shared rows.
#pragma once
#include "tg_common.cuh"

namespace tg {

// ---------------------------------------------------------------------------
// device FFT of NB transforms of length L held in shared memory
// DIR = -1: exp(-i...) (forward), DIR = +1: exp(+i...) (backward, unscaled)
// ---------------------------------------------------------------------------
template <typename T, int DIR>
__device__ __forceinline__ cplx<T> tw_get(const cplx<T>* tw, int idx) {
  cplx<T> w = tw[idx];
  if (DIR > 0) w.y = -w.y;
  return w;
}

template <typename C, int DIR>
__device__ __forceinline__ C rot(C a, double c, double s) {  // a * (c + i DIR s)
  using R = decltype(C::x);
  const R cr = (R)c, sr = (R)(DIR * s);
  return mkc<C>(a.x * cr - a.y * sr, a.x * sr + a.y * cr);
}

// cos(2 pi i / 16); sin(2 pi i / 16) = cos16(i - 4)
__host__ __device__ constexpr double cos16(int i) {
  i &= 15;
  if (i > 8) i = 16 - i;
  return i == 0 ? 1.0
       : i == 1 ? 0.92387953251128675613
       : i == 2 ? 0.70710678118654752440
       : i == 3 ? 0.38268343236508977173
       : i == 4 ? 0.0
       : i == 5 ? -0.38268343236508977173
       : i == 6 ? -0.70710678118654752440
       : i == 7 ? -0.92387953251128675613
       : -1.0;
}

template <int R, int DIR, typename C>
__device__ __forceinline__ void dft_ct(C* v) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else {
    constexpr int H = R / 2;
    C e[H], o[H];
#pragma unroll
    for (int m = 0; m < H; ++m) {
      e[m] = v[2 * m];
      o[m] = v[2 * m + 1];
    }
    dft_ct<H, DIR>(e);
    dft_ct<H, DIR>(o);
#pragma unroll
    for (int k = 0; k < H; ++k) {
      // W_R^k = cos(2 pi k/R) + i DIR sin(2 pi k/R) with DIR = -1 forward (R <= 16)
      const int i16 = k * (16 / R);
      C t;
      if (k == 0) {
        t = o[k];
      } else if (4 * k == R) {
        t = (DIR < 0) ? mkc<C>(o[k].y, -o[k].x) : mkc<C>(-o[k].y, o[k].x);
      } else {
        t = rot<C, DIR>(o[k], cos16(i16), cos16(i16 - 4));
      }
      v[k] = cadd(e[k], t);
      v[k + H] = csub(e[k], t);
    }
  }
}

template <typename T> struct Tw;
template <> struct Tw<double> {
  static __host__ const double2* get(const FftPlan& p) { return p.tw64; }
};
template <> struct Tw<float> {
  static __host__ const float2* get(const FftPlan& p) { return p.tw32; }
};

// ---------------------------------------------------------------------------
// Power-of-two lengths: in-place passes on one padded shared buffer.
//
// NB transforms of length L per CTA, NB*L/16 threads, every thread holding
// 16 complex values of a pass in registers (one radix-16 butterfly, or 16/R
// butterflies of a smaller final radix), so a pass reads all its inputs,
// synchronises, and writes its outputs in place.  Shared rows are padded with
// one spare slot per 16 values (index i -> i + i/16) and one more per row, so
// the stride-16 writes of the first pass and the column accesses of the
// x <-> y reorder hit distinct banks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sp(int i) { return i + (i >> 4); }

template <int L> struct P2 {
  static constexpr int RS = L + L / 16 + 1;  // padded row stride (complex values)
};

// the passes of strides Ns, Ns * 16, ... below NsEnd (all remaining ones by default)
template <typename T, int DIR, int L, int NB, int Ns, int NT = NB * L / 16, int NsEnd = L>
__device__ __forceinline__ void ip_passes(cplx<T>* buf, const cplx<T>* __restrict__ tw, int tid = threadIdx.x) {
  using C = cplx<T>;
  if constexpr (Ns < L && Ns < NsEnd) {
    constexpr int rem = L / Ns;
    constexpr int R = rem >= 16 ? 16 : rem;
    constexpr int nb = L / R;                    // butterflies per transform
    constexpr int groups = NB * nb;              // butterflies of the pass
    constexpr int GPT = (groups + NT - 1) / NT;  // butterflies per thread
    constexpr bool exact = groups % NT == 0;
    constexpr int RS = P2<L>::RS;
    constexpr int twstep = L / (Ns * R);
    C v[GPT][R];
#pragma unroll
    for (int t = 0; t < GPT; ++t) {
      const int g = tid + t * NT;
      if (exact || g < groups) {
        const int b = g / nb, j = g - b * nb;
        const C* src = buf + b * RS;
        const int jm = j % Ns;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          v[t][r] = src[sp(j + r * nb)];
          if (Ns > 1 && r > 0) v[t][r] = cmul(v[t][r], tw_get<T, DIR>(tw, jm * r * twstep));
        }
        dft_ct<R, DIR>(v[t]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < GPT; ++t) {
      const int g = tid + t * NT;
      if (exact || g < groups) {
        const int b = g / nb, j = g - b * nb;
        const int jm = j % Ns;
        const int base = (j - jm) * R + jm;
        C* dst = buf + b * RS;
#pragma unroll
        for (int k = 0; k < R; ++k) dst[sp(base + k * Ns)] = v[t][k];
      }
    }
    __syncthreads();
    ip_passes<T, DIR, L, NB, Ns * R, NT, NsEnd>(buf, tw, tid);
  }
}

// stride of the last pass of a length-L transform (passes of radix 16, the
// last one of radix L / stride)
__host__ __device__ constexpr int last_stride(int L) {
  int ns = 1;
  while (ns * 16 < L) ns *= 16;
  return ns;
}

// The last pass (stride Ns = last_stride(L)) reading the padded rows and
// handing each output, with its transform b, index x and slot i in the
// thread (0 .. NB*L/NT - 1, a compile-time constant once unrolled), to
// out(b, x, i, value) instead of writing it back: used where the pass's
// outputs leave for global memory.  Call after the earlier passes and a
// barrier.
template <typename T, int DIR, int L, int NB, int NT, typename Out>
__device__ __forceinline__ void last_pass_out(const cplx<T>* buf, const cplx<T>* __restrict__ tw, Out&& out,
                                              int tid = threadIdx.x) {
  using C = cplx<T>;
  constexpr int Ns = last_stride(L);
  constexpr int R = L / Ns;
  constexpr int nb = L / R;                    // = Ns
  constexpr int groups = NB * nb;
  constexpr int GPT = (groups + NT - 1) / NT;
  constexpr bool exact = groups % NT == 0;
  constexpr int RS = P2<L>::RS;
#pragma unroll
  for (int t = 0; t < GPT; ++t) {
    const int g = tid + t * NT;
    if (exact || g < groups) {
      const int b = g / nb, j = g - b * nb;   // j < Ns: the twiddle index and the output base
      const C* src = buf + b * RS;
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        v[r] = src[sp(j + r * nb)];
        if (Ns > 1 && r > 0) v[r] = cmul(v[r], tw_get<T, DIR>(tw, j * r));
      }
      dft_ct<R, DIR>(v);
#pragma unroll
      for (int k = 0; k < R; ++k) out(b, j + k * Ns, t * R + k, v[k]);
    }
  }
}

// spectral row iy -> FFT index along y (P3DFFT pruning, reference src/base.cc:228-237)
__device__ __forceinline__ int y_of(int iy, int ny, int nyc) { return iy < nyc / 2 ? iy : ny - (nyc - iy); }


}  // namespace tg
