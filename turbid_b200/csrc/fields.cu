// Elementwise stage kernels and reductions of the RK3 substep.
// Each kernel restates one block of the reference's Armadillo expressions
// (file:line cited per kernel), evaluated per element in the same order.
#include <type_traits>

#include "fields.cuh"

namespace tg {

namespace {
constexpr int kT = 256;
inline unsigned nblk(size_t n, int per = 1) {
  size_t b = (n + (size_t)kT * per - 1) / ((size_t)kT * per);
  if (b > 148u * 32u) b = 148u * 32u;   // grid-stride beyond ~32 CTAs per SM
  return (unsigned)(b ? b : 1);
}

__device__ __forceinline__ double2 mul_i(double k, double2 x) {  // (0, k) * x
  return make_double2(0.0 * x.x - k * x.y, 0.0 * x.y + k * x.x);
}
}  // namespace

// --- layout conversion: reference [c][m][z] <-> slab [c][z][m] ---------------
__global__ void k_ref_to_slab(const double2* __restrict__ ref, double2* __restrict__ slab, int M, int nz) {
  __shared__ double2 t[32][33];
  const int c = blockIdx.z;
  const double2* src = ref + (size_t)c * M * nz;
  double2* dst = slab + (size_t)c * M * nz;
  const int z0 = blockIdx.x * 32, m0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    int m = m0 + i, z = z0 + threadIdx.x;
    if (m < M && z < nz) t[i][threadIdx.x] = src[(size_t)m * nz + z];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    int z = z0 + i, m = m0 + threadIdx.x;
    if (m < M && z < nz) dst[(size_t)z * M + m] = t[threadIdx.x][i];
  }
}
__global__ void k_slab_to_ref(const double2* __restrict__ slab, double2* __restrict__ ref, int M, int nz) {
  __shared__ double2 t[32][33];
  const int c = blockIdx.z;
  const double2* src = slab + (size_t)c * M * nz;
  double2* dst = ref + (size_t)c * M * nz;
  const int z0 = blockIdx.x * 32, m0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    int z = z0 + i, m = m0 + threadIdx.x;
    if (m < M && z < nz) t[i][threadIdx.x] = src[(size_t)z * M + m];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    int m = m0 + i, z = z0 + threadIdx.x;
    if (m < M && z < nz) dst[(size_t)m * nz + z] = t[threadIdx.x][i];
  }
}
void ref_to_slab(const double2* ref, double2* slab, int M, int nz, int dim, cudaStream_t s) {
  dim3 g((nz + 31) / 32, (M + 31) / 32, dim), b(32, 8);
  k_ref_to_slab<<<g, b, 0, s>>>(ref, slab, M, nz);
  TG_LAUNCH_CHECK("k_ref_to_slab");
}
void slab_to_ref(const double2* slab, double2* ref, int M, int nz, int dim, cudaStream_t s) {
  dim3 g((nz + 31) / 32, (M + 31) / 32, dim), b(32, 8);
  k_slab_to_ref<<<g, b, 0, s>>>(slab, ref, M, nz);
  TG_LAUNCH_CHECK("k_slab_to_ref");
}

// --- physical products ---------------------------------------------------------
// divergence form products u_i u_j (phase_carrier_flat.cc:725-745): the six
// distinct ones uu, uv, uw, vv, vw, ww (u_i u_j == u_j u_i exactly).
template <typename T>
__global__ void k_products6(const T* __restrict__ unl, T* __restrict__ prd, size_t P) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x) {
    T u = unl[i], v = unl[P + i], w = unl[2 * P + i];
    prd[i] = u * u;
    prd[P + i] = u * v;
    prd[2 * P + i] = u * w;
    prd[3 * P + i] = v * v;
    prd[4 * P + i] = v * w;
    prd[5 * P + i] = w * w;
  }
}
template <typename T>
void products6(const T* unl, T* prd, size_t P, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 9.0 * sizeof(T) * (double)P, 0);
  k_products6<T><<<nblk(P), kT, 0, s>>>(unl, prd, P);
  prof_end(s);
  TG_LAUNCH_CHECK("k_products6");
}

// advective form out_i = u du_i/dx + v du_i/dy + w du_i/dz
// (phase_carrier_flat.cc:786-797; phase_scalar_flat.cc:588-591 with dim = 1).
// dup: ncomp x 3 physical gradient fields; sh: constant velocity shift (scalar
// phase settling velocity, phase_scalar_flat.cc:258-279).
template <typename T>
__global__ void k_adv(const T* __restrict__ unl, const T* __restrict__ dup, T* __restrict__ out, size_t P, int ncomp,
                      double su, double sv, double sw) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x) {
    T u = unl[i] + (T)su, v = unl[P + i] + (T)sv, w = unl[2 * P + i] + (T)sw;
    for (int c = 0; c < ncomp; ++c) {
      const T* d = dup + (size_t)c * 3 * P;
      out[(size_t)c * P + i] = u * d[i] + v * d[P + i] + w * d[2 * P + i];
    }
  }
}
template <typename T>
void adv_products(const T* unl, const T* dup, T* out, size_t P, int ncomp, double su, double sv, double sw,
                  cudaStream_t s) {
  prof_begin(s, PC_ELEM, (3.0 + 4.0 * ncomp) * sizeof(T) * (double)P, 0);
  k_adv<T><<<nblk(P), kT, 0, s>>>(unl, dup, out, P, ncomp, su, sv, sw);
  prof_end(s);
  TG_LAUNCH_CHECK("k_adv");
}

// phi * u_j (phase_scalar_flat.cc:563-569)
template <typename T>
__global__ void k_phi_products(const T* __restrict__ phip, const T* __restrict__ unl, T* __restrict__ out, size_t P,
                               double su, double sv, double sw) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x) {
    T p = phip[i];
    out[i] = p * (unl[i] + (T)su);
    out[P + i] = p * (unl[P + i] + (T)sv);
    out[2 * P + i] = p * (unl[2 * P + i] + (T)sw);
  }
}
template <typename T>
void phi_products(const T* phip, const T* unl, T* out, size_t P, double su, double sv, double sw, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 7.0 * sizeof(T) * (double)P, 0);
  k_phi_products<T><<<nblk(P), kT, 0, s>>>(phip, unl, out, P, su, sv, sw);
  prof_end(s);
  TG_LAUNCH_CHECK("k_phi_products");
}

// single product a * (b + shift) for the flux features (phase_scalar_flat.cc:500-518)
template <typename T>
__global__ void k_mul_shift(const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ out, size_t P,
                            double sh) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (b[i] + (T)sh) * a[i];
}
template <typename T>
void mul_shift(const T* a, const T* b, T* out, size_t P, double sh, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 3.0 * sizeof(T) * (double)P, 0);
  k_mul_shift<T><<<nblk(P), kT, 0, s>>>(a, b, out, P, sh);
  prof_end(s);
  TG_LAUNCH_CHECK("k_mul_shift");
}

// --- carrier H register (phase_carrier_flat.cc:293-296, 325-356, 503-504) -------
__global__ void k_h_update(double2* __restrict__ H, const double2* __restrict__ adv, const double2* __restrict__ phi,
                           size_t S, int M, double c1, double dt, double bcoef, double sinsl, double cossl, int sdir,
                           double dtf1, double dtf2, const double* __restrict__ dtf) {
  const size_t n = 3 * S;
  if (dtf) {  // forcing of this step from device memory (graph replay)
    dtf1 = dtf[0];
    dtf2 = dtf[1];
  }
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / S);
    const size_t e = i - (size_t)c * S;
    const int m = (int)(e % M);
    double2 h = H[i], a = adv[i];
    h = make_double2(c1 * h.x - dt * a.x, c1 * h.y - dt * a.y);
    if (phi) {
      double2 p = phi[e];
      if ((sdir == 1 && c == 0) || (sdir == 2 && c == 1)) {
        h.x = h.x + bcoef * p.x * sinsl;
        h.y = h.y + bcoef * p.y * sinsl;
      }
      if (c == 2) {
        h.x = h.x - bcoef * p.x * cossl;
        h.y = h.y - bcoef * p.y * cossl;
      }
    }
    if (m == 0) {
      if (c == 0) h.x += dtf1;
      if (c == 1) h.x += dtf2;
    }
    H[i] = h;
  }
}
void h_update(double2* H, const double2* adv, const double2* phi, size_t S, int M, double c1, double dt,
              double bcoef, double sinsl, double cossl, int sdir, double dtf1, double dtf2, const double* dtf,
              cudaStream_t s) {
  prof_begin(s, PC_ELEM, 144.0 * (double)S, 0);
  k_h_update<<<nblk(3 * S), kT, 0, s>>>(H, adv, phi, S, M, c1, dt, bcoef, sinsl, cossl, sdir, dtf1, dtf2, dtf);
  prof_end(s);
  TG_LAUNCH_CHECK("k_h_update");
}

// Buoyancy of the H update (phase_carrier_flat.cc:325-356), added after the
// right-hand side has been formed: component H_c gets sgn * bcoef * phi * trig
// (the H update's own expression), and the interior rows of the right-hand
// side the same term times a*c2, its coefficient of H in the Laplacian/rhs
// step (rows 0 and N-1 already hold the boundary values).  This lets the
// carrier's H update, Laplacian and u/v solves run before the scalar Correct
// that produces phi has finished.
__global__ void k_buoyancy(double2* __restrict__ H, double2* __restrict__ rhs, const double2* __restrict__ phi, int M,
                           int nz, double bcoef, double trig, int sgn, double ac2) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  const int z = blockIdx.y;
  const size_t e = (size_t)z * M + m;
  const double2 p = phi[e];
  double2 h = H[e];
  double tx, ty;
  if (sgn > 0) {
    h.x = h.x + bcoef * p.x * trig;
    h.y = h.y + bcoef * p.y * trig;
    tx = bcoef * p.x * trig;
    ty = bcoef * p.y * trig;
  } else {
    h.x = h.x - bcoef * p.x * trig;
    h.y = h.y - bcoef * p.y * trig;
    tx = -(bcoef * p.x * trig);
    ty = -(bcoef * p.y * trig);
  }
  H[e] = h;
  if (z != 0 && z != nz - 1) {
    double2 r = rhs[e];
    r.x += ac2 * tx;
    r.y += ac2 * ty;
    rhs[e] = r;
  }
}
void buoyancy(double2* H, double2* rhs, const double2* phi, int M, int nz, double bcoef, double trig, int sgn,
              double ac2, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 80.0 * (double)M * nz, 0);
  k_buoyancy<<<dim3((M + kT - 1) / kT, nz), kT, 0, s>>>(H, rhs, phi, M, nz, bcoef, trig, sgn, ac2);
  prof_end(s);
  TG_LAUNCH_CHECK("k_buoyancy");
}

// scalar register (phase_scalar_flat.cc:308-310)
__global__ void k_axpby(double2* __restrict__ y, const double2* __restrict__ x, size_t n, double a, double b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double2 v = y[i], w = x[i];
    y[i] = make_double2(a * v.x - b * w.x, a * v.y - b * w.y);
  }
}
void axmby(double2* y, const double2* x, size_t n, double a, double b, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 48.0 * (double)n, 0);
  k_axpby<<<nblk(n), kT, 0, s>>>(y, x, n, a, b);
  prof_end(s);
  TG_LAUNCH_CHECK("k_axpby");
}

// --- boundary rows ---------------------------------------------------------------
// FlatCarrierBoundary::Apply (boundary_carrier_flat.cc:230-242) + the mean-mode
// top values (phase_carrier_flat.cc:542-547).  hist: [8][3][M] rows
// 0 dp1m1top 1 dp1m1bot 2 dp1m2top 3 dp1m2bot 4 dp2m1top 5 dp2m1bot 6 dp2m2top 7 dp2m2bot
__global__ void k_boundary_apply(double2* __restrict__ rhs, const double2* __restrict__ hist, size_t S, int M, int nz,
                                 double fac, double r, int opentop, double tu, double tv, double tw) {
  const int n = 3 * M;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i / M, m = i - c * M;
    const double2* h = hist;
    const size_t R = (size_t)3 * M;
    double2 t1 = h[0 * R + i], t2 = h[2 * R + i], b1 = h[1 * R + i], b2 = h[3 * R + i];
    double2 top = make_double2(fac * ((1 + r) * t1.x + (0 - r) * t2.x), fac * ((1 + r) * t1.y + (0 - r) * t2.y));
    double2 bot = make_double2(fac * ((1 + r) * b1.x + (0 - r) * b2.x), fac * ((1 + r) * b1.y + (0 - r) * b2.y));
    if (opentop && c < 2) {
      double2 q1 = h[4 * R + i], q2 = h[6 * R + i];
      top = make_double2(fac * ((1 + r) * q1.x + (0 - r) * q2.x), fac * ((1 + r) * q1.y + (0 - r) * q2.y));
    }
    if (m == 0) top = make_double2(c == 0 ? tu : (c == 1 ? tv : tw), 0.0);
    rhs[(size_t)c * S + (size_t)(nz - 1) * M + m] = top;
    rhs[(size_t)c * S + m] = bot;
  }
}
void boundary_apply(double2* rhs, const double2* hist, size_t S, int M, int nz, double fac, double r, int opentop,
                    double tu, double tv, double tw, cudaStream_t s) {
  k_boundary_apply<<<nblk(3 * (size_t)M), kT, 0, s>>>(rhs, hist, S, M, nz, fac, r, opentop, tu, tv, tw);
  TG_LAUNCH_CHECK("k_boundary_apply");
}

// FlatCarrierBoundary::Update (boundary_carrier_flat.cc:131-170): history
// shift and new wall rows of grad p; with an open top the rows of grad(dp/dz)
// (phase_carrier_flat.cc:599-604) where only rows 0 and N-1 are needed.
// Rows 0 and N-1 of D1*f for columns [m0, m0+32) of one component: the z sum
// is split over the 8 thread rows of a (32 x 8) block (each a strided subset
// of z, loads coalesced along m) and reduced in shared memory.  Thread row 0
// returns the two sums of its column.
__device__ __forceinline__ void wall_rows_d1(const double2* __restrict__ f, int M, int nz, int m,
                                            const double* __restrict__ d1r0, const double* __restrict__ d1rn,
                                            double2& r0, double2& rn) {
  __shared__ double part[8][32][4];
  const int tx = threadIdx.x, ty = threadIdx.y;
  double a = 0, b = 0, c = 0, d = 0;
  if (m < M) {
#pragma unroll 4
    for (int k = ty; k < nz; k += 8) {
      const double2 v = f[(size_t)k * M + m];
      a += d1r0[k] * v.x;
      b += d1r0[k] * v.y;
      c += d1rn[k] * v.x;
      d += d1rn[k] * v.y;
    }
  }
  part[ty][tx][0] = a;
  part[ty][tx][1] = b;
  part[ty][tx][2] = c;
  part[ty][tx][3] = d;
  __syncthreads();
  if (ty == 0) {
    for (int j = 1; j < 8; ++j) {
      a += part[j][tx][0];
      b += part[j][tx][1];
      c += part[j][tx][2];
      d += part[j][tx][3];
    }
    r0 = make_double2(a, b);
    rn = make_double2(c, d);
  }
  __syncthreads();
}

// FlatCarrierBoundary::Update (boundary_carrier_flat.cc:131-170): shift the
// history rows, store the new pressure-gradient wall rows; with an open top
// also d(dp/dz)/dz at the walls (rows 0, N-1 of D1 applied to dp/dz).
// Block (32, 8): 32 columns, 8 rows of the z sum.
// grad p rows: x and y components i kx p, i ky p from p, z component dpz
__device__ __forceinline__ double2 grad_p_row(const double2* __restrict__ p, const double2* __restrict__ dpz,
                                              const double* __restrict__ kx, const double* __restrict__ ky, int c,
                                              size_t o, int m) {
  if (c == 2) return dpz[o];
  return mul_i(c == 0 ? kx[m] : ky[m], p[o]);
}

__global__ void k_boundary_update(double2* __restrict__ hist, const double2* __restrict__ p,
                                  const double2* __restrict__ dpz, int M, int nz, int opentop,
                                  const double* __restrict__ kx, const double* __restrict__ ky,
                                  const double* __restrict__ d1r0, const double* __restrict__ d1rn) {
  const size_t R = (size_t)3 * M;
  const int m = blockIdx.x * 32 + threadIdx.x;
  if (threadIdx.y < 3 && m < M) {
    const int c = threadIdx.y;
    const size_t i = (size_t)c * M + m;
    hist[2 * R + i] = hist[0 * R + i];
    hist[3 * R + i] = hist[1 * R + i];
    hist[6 * R + i] = hist[4 * R + i];
    hist[7 * R + i] = hist[5 * R + i];
    hist[1 * R + i] = grad_p_row(p, dpz, kx, ky, c, (size_t)m, m);
    hist[0 * R + i] = grad_p_row(p, dpz, kx, ky, c, (size_t)(nz - 1) * M + m, m);
  }
  if (opentop) {
    const double2* g = dpz;  // dp/dz
    double2 r0, rn;
    wall_rows_d1(g, M, nz, m, d1r0, d1rn, r0, rn);
    if (threadIdx.y == 0 && m < M) {
      const double2 g0 = g[m], gn = g[(size_t)(nz - 1) * M + m];
      hist[5 * R + 0 * M + m] = mul_i(kx[m], g0);
      hist[5 * R + 1 * M + m] = mul_i(ky[m], g0);
      hist[5 * R + 2 * M + m] = r0;
      hist[4 * R + 0 * M + m] = mul_i(kx[m], gn);
      hist[4 * R + 1 * M + m] = mul_i(ky[m], gn);
      hist[4 * R + 2 * M + m] = rn;
    }
  }
}
void boundary_update(double2* hist, const double2* p, const double2* dpz, int M, int nz, int opentop,
                     const double* kx, const double* ky, const double* d1r0, const double* d1rn, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 16.0 * (double)M * (opentop ? nz + 16 : 16), 0);
  k_boundary_update<<<(M + 31) / 32, dim3(32, 8), 0, s>>>(hist, p, dpz, M, nz, opentop, kx, ky, d1r0, d1rn);
  prof_end(s);
  TG_LAUNCH_CHECK("k_boundary_update");
}

// Wall rows of d(u_i)/dz only (rows 0 and N-1 of D1*u_i, i = 0..2): all the
// divergence-form step reads of the velocity gradient (bottom plane for the
// erosion flux, phase_scalar_flat.cc:349-353; mean-mode wall values for the
// features, phase_carrier_flat.cc:687-692).
__global__ void k_wall_dz(const double2* __restrict__ U, double2* __restrict__ DU, size_t S, int M, int nz,
                          const double* __restrict__ d1r0, const double* __restrict__ d1rn) {
  const int c = blockIdx.y;
  const int m = blockIdx.x * 32 + threadIdx.x;
  double2 r0, rn;
  wall_rows_d1(U + (size_t)c * S, M, nz, m, d1r0, d1rn, r0, rn);
  if (threadIdx.y == 0 && m < M) {
    double2* dz = DU + (size_t)(3 * c + 2) * S + m;
    dz[0] = r0;
    dz[(size_t)(nz - 1) * M] = rn;
  }
}
void wall_dz(const double2* U, double2* DU, size_t S, int M, int nz, const double* d1r0, const double* d1rn,
             cudaStream_t s) {
  prof_begin(s, PC_ELEM, 3.0 * 16.0 * (double)S, 0);
  k_wall_dz<<<dim3((M + 31) / 32, 3), dim3(32, 8), 0, s>>>(U, DU, S, M, nz, d1r0, d1rn);
  prof_end(s);
  TG_LAUNCH_CHECK("k_wall_dz");
}

// projection u = u* - 2 dt c3 grad p, mean w := 0 (phase_carrier_flat.cc:609-620)
__global__ void k_project(double2* __restrict__ U, const double2* __restrict__ SU, const double2* __restrict__ P,
                          const double2* __restrict__ DPZ, size_t S, int M, const double* __restrict__ kx,
                          const double* __restrict__ ky, double coef) {
  const size_t n = 3 * S;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / S);
    const size_t e = i - (size_t)c * S;
    const int m = (int)(e % M);
    double2 su = SU[i], dp = grad_p_row(P, DPZ, kx, ky, c, e, m);
    double2 u = make_double2(su.x - coef * dp.x, su.y - coef * dp.y);
    if (c == 2 && m == 0) u = make_double2(0.0, 0.0);
    U[i] = u;
  }
}
void project(double2* U, const double2* SU, const double2* P, const double2* DPZ, size_t S, int M, const double* kx,
             const double* ky, double coef, cudaStream_t s) {
  prof_begin(s, PC_ELEM, 112.0 * (double)S, 0);   // SU (3), p, dp/dz in; U (3) out
  k_project<<<nblk(3 * S), kT, 0, s>>>(U, SU, P, DPZ, S, M, kx, ky, coef);
  prof_end(s);
  TG_LAUNCH_CHECK("k_project");
}

// rows 0 and N-1 := 0 (boundary_scalar_flat.cc:150-151)
__global__ void k_zero_rows(double2* f, int M, int nz) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    f[m] = make_double2(0.0, 0.0);
    f[(size_t)(nz - 1) * M + m] = make_double2(0.0, 0.0);
  }
}
void zero_rows(double2* f, int M, int nz, cudaStream_t s) {
  k_zero_rows<<<nblk(M), kT, 0, s>>>(f, M, nz);
  TG_LAUNCH_CHECK("k_zero_rows");
}

// --- erosion / deposition bottom row (phase_scalar_flat.cc:340-384) ---------------
template <typename T>
__global__ void k_erosion_tau(const T* __restrict__ dudz, const T* __restrict__ dvdz, T* __restrict__ tau, size_t n,
                              double re, double tauc, double rate) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    T a = dudz[i], b = dvdz[i];
    T v = sqrt(a * a + b * b) / (T)re;
    tau[i] = (v < (T)tauc) ? T(0) : (T)rate * (v / (T)tauc - T(1));
  }
}
template <typename T>
void erosion_tau(const T* dudz, const T* dvdz, T* tau, size_t n, double re, double tauc, double rate,
                 cudaStream_t s) {
  k_erosion_tau<T><<<nblk(n), kT, 0, s>>>(dudz, dvdz, tau, n, re, tauc, rate);
  TG_LAUNCH_CHECK("k_erosion_tau");
}

__global__ void k_erosion_row(double2* __restrict__ rhs, const double2* __restrict__ ero, const double2* __restrict__ phi,
                              int M, double wsc, double conc, double resc, double* feat) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    double2 e = ero[m], p = phi[m];
    double2 r = make_double2(e.x - wsc * p.x * conc, e.y - wsc * p.y * conc);
    const double f = -1 * resc / conc * 10e6;
    rhs[m] = make_double2(r.x * f, r.y * f);
    if (m == 0) {
      feat[28] = e.x;
      feat[29] = wsc * p.x * conc;
    }
  }
}
void erosion_row(double2* rhs, const double2* ero, const double2* phi, int M, double wsc, double conc, double resc,
                 double* feat, cudaStream_t s) {
  k_erosion_row<<<nblk(M), kT, 0, s>>>(rhs, ero, phi, M, wsc, conc, resc, feat);
  TG_LAUNCH_CHECK("k_erosion_row");
}

// --- Bartnicki positivity filter (phase_scalar_flat.cc:419-478) -----------------
// One CTA per z plane, five sweeps in one launch.  Each sweep needs the sums
// of the positive and the negative values of the plane and their counts (the
// zero class sums to zero); the redistribution of sweep k and the sums for
// sweep k+1 share one pass over the plane, which stays in L2.  Passes run in
// batches of FB values per thread, all loads of a batch in flight together.
constexpr int kFilterThreads = 1024, kFilterBatch = 8;

__device__ __forceinline__ void filter_reduce(double (&a)[4], double (*red)[32], double* tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double x = a[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double x = 0;
    for (int w = 0; w < nw; ++w) x += red[threadIdx.x][w];
    tot[threadIdx.x] = x;
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ void filter_classify(T x, double& sp, int& cp, double& sn, int& cn) {
  const double d = (double)x;
  sp += d > 0 ? d : 0.0;
  cp += d > 0 ? 1 : 0;
  sn += d < 0 ? d : 0.0;
  cn += d < 0 ? 1 : 0;
}

// W values per access: 16-byte vectors where the plane is a whole number of
// them (W = 16 / sizeof(T)), one value otherwise; every thread keeps
// kFilterBatch values of a sweep in flight either way
template <typename T, int W>
struct alignas(sizeof(T) * W) FilterVec {
  T e[W];
};

template <typename T, int W>
__global__ void __launch_bounds__(kFilterThreads, 2) k_filter(T* __restrict__ phip, int plane_n) {
  using V = FilterVec<T, W>;
  constexpr int FB = kFilterBatch / W, STEP = FB * kFilterThreads;
  __shared__ double red[4][32];
  __shared__ double tot[4];
  V* p = reinterpret_cast<V*>(phip + (size_t)blockIdx.x * plane_n);
  const int nv = plane_n / W;
  double sp = 0, sn = 0;
  int cp = 0, cn = 0;
  for (int i0 = threadIdx.x; i0 < nv; i0 += STEP) {
    V x[FB];
#pragma unroll
    for (int b = 0; b < FB; ++b) {
      const int i = i0 + b * kFilterThreads;
      if (i < nv) x[b] = p[i];
      else
#pragma unroll
        for (int e = 0; e < W; ++e) x[b].e[e] = T(0);
    }
#pragma unroll
    for (int b = 0; b < FB; ++b)
#pragma unroll
      for (int e = 0; e < W; ++e) filter_classify(x[b].e[e], sp, cp, sn, cn);
  }
  for (int it = 0; it < 5; ++it) {
    double a[4] = {sp, (double)cp, sn, (double)cn};
    filter_reduce(a, red, tot);
    const bool kill = (tot[0] + tot[2]) < 0;
    const double add = tot[1] > 0 ? tot[2] / tot[1] : 0.0;
    sp = sn = 0;
    cp = cn = 0;
    for (int i0 = threadIdx.x; i0 < nv; i0 += STEP) {
      V x[FB];
#pragma unroll
      for (int b = 0; b < FB; ++b) {
        const int i = i0 + b * kFilterThreads;
        if (i < nv) x[b] = p[i];
        else
#pragma unroll
          for (int e = 0; e < W; ++e) x[b].e[e] = T(0);
      }
#pragma unroll
      for (int b = 0; b < FB; ++b) {
        const int i = i0 + b * kFilterThreads;
        V y;
#pragma unroll
        for (int e = 0; e < W; ++e) {
          const T v = x[b].e[e];
          y.e[e] = kill ? T(0) : ((v > 0) ? (T)((double)v + add) : T(0));
          filter_classify(y.e[e], sp, cp, sn, cn);   // sums for the next sweep
        }
        if (i < nv) p[i] = y;
      }
    }
    __syncthreads();   // the next sweep's reduction reuses red/tot
  }
}
template <typename T>
void positivity_filter(T* phip, int plane_n, int nz, cudaStream_t s) {
  prof_begin(s, PC_FILTER, 11.0 * sizeof(T) * (double)plane_n * nz, 0);   // 6 reads + 5 writes of the plane
  constexpr int W = 16 / sizeof(T);
  if (plane_n % W == 0 && reinterpret_cast<uintptr_t>(phip) % 16 == 0)
    k_filter<T, W><<<nz, kFilterThreads, 0, s>>>(phip, plane_n);
  else
    k_filter<T, 1><<<nz, kFilterThreads, 0, s>>>(phip, plane_n);
  prof_end(s);
  TG_LAUNCH_CHECK("k_filter");
}

// --- features ---------------------------------------------------------------------
// Stage-2 features of FlatCarrierPhase::Correct (phase_carrier_flat.cc:633-703).
// bits: 10 slots of non-negative doubles reduced with atomicMax on their bit
// patterns: 0-2 max|u_i|, 3-5 bottom plane, 6-8 top plane, 9 max CFL length.
// The maxima keep a NaN (fmax would drop it; a positive NaN's bit pattern is
// above +inf's, so atomicMax keeps it too): a non-finite velocity anywhere
// reaches the features, where the host's guard reports it.
__device__ __forceinline__ double max_keep_nan(double a, double b) { return (b > a || isnan(b)) ? b : a; }

template <typename T>
__global__ void k_feature_max(const T* __restrict__ unl, int nx, int ny, int nz, const double* __restrict__ glz,
                              double lmx, double lmy, unsigned long long* bits) {
  // blockIdx.y = z plane: the wall maxima and 1/glz need no per-element index division
  const size_t plane = (size_t)nx * ny, P = plane * nz;
  const int z = blockIdx.y;
  // the CFL length |u|/dx + |v|/dy + |w|/dz with the reciprocals taken once
  // (three FP64 divisions per point were most of this kernel's time; the
  // products differ from the quotients in the last bits only)
  const double ilx = 1.0 / lmx, ily = 1.0 / lmy, igl = 1.0 / glz[z];
  const T* pu = unl + (size_t)z * plane;
  double mu = 0, mv = 0, mw = 0, ml = 0;
  auto point = [&](T a, T b, T c) {
    const double u = fabs((double)a), v = fabs((double)b), w = fabs((double)c);
    mu = max_keep_nan(mu, u);
    mv = max_keep_nan(mv, v);
    mw = max_keep_nan(mw, w);
    ml = max_keep_nan(ml, u * ilx + v * ily + w * igl);
  };
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, step = (size_t)gridDim.x * blockDim.x;
  // 16-byte vectors of the three fields (the maxima do not depend on the
  // order), the plane's tail, if any, one value at a time
  constexpr int EV = 16 / sizeof(T);
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const size_t nvec = (plane % EV == 0 && P % EV == 0) ? plane / EV : 0;
  const V* pv = reinterpret_cast<const V*>(pu);
  for (size_t i = t0; i < nvec; i += step) {
    const V a = pv[i], b = pv[P / EV + i], c = pv[2 * P / EV + i];
    const T* ta = reinterpret_cast<const T*>(&a);
    const T* tb = reinterpret_cast<const T*>(&b);
    const T* tc = reinterpret_cast<const T*>(&c);
#pragma unroll
    for (int e = 0; e < EV; ++e) point(ta[e], tb[e], tc[e]);
  }
  for (size_t i = nvec * EV + t0; i < plane; i += step) point(pu[i], pu[P + i], pu[2 * P + i]);
  double mx[4] = {mu, mv, mw, ml};
#pragma unroll
  for (int k = 0; k < 4; ++k)
    for (int o = 16; o > 0; o >>= 1) mx[k] = max_keep_nan(mx[k], __shfl_down_sync(0xffffffffu, mx[k], o));
  // block maximum first: one atomic per block and value (the values are
  // non-negative, so their bit patterns order like the numbers)
  __shared__ double wm[32][4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 4; ++k) wm[warp][k] = mx[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w)
      for (int k = 0; k < 4; ++k) mx[k] = max_keep_nan(mx[k], wm[w][k]);
    for (int k = 0; k < 4; ++k)   // a NaN of either sign becomes the positive quiet NaN
      if (isnan(mx[k])) mx[k] = __longlong_as_double(0x7ff8000000000000LL);
    for (int k = 0; k < 3; ++k) {
      const unsigned long long b = (unsigned long long)__double_as_longlong(mx[k]);
      atomicMax(bits + k, b);
      if (z == 0) atomicMax(bits + 3 + k, b);
      if (z == nz - 1) atomicMax(bits + 6 + k, b);
    }
    atomicMax(bits + 9, (unsigned long long)__double_as_longlong(mx[3]));
  }
}
// flocal = feat[0..49], fglobal = feat[50..99]
__global__ void k_feature_final(double* feat, const unsigned long long* bits, const double2* __restrict__ du, size_t S,
                                int M, int nz) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < 9; ++k) feat[k] = __longlong_as_double((long long)bits[k]);
  feat[19] = __longlong_as_double((long long)bits[9]);
  for (int k = 0; k < 50; ++k) feat[50 + k] = feat[k];
  // du_i/dz of the mean mode at the walls (dudxyz[i] component 2)
  for (int i = 0; i < 3; ++i) {
    const double2* dz = du + (size_t)(3 * i + 2) * S;
    feat[50 + 10 + i] = dz[0].x;
    feat[50 + 13 + i] = dz[(size_t)(nz - 1) * M].x;
  }
}
template <typename T>
void features(const T* unl, int nx, int ny, int nz, const double* glz, double lmx, double lmy,
              unsigned long long* bits, double* feat, const double2* du, size_t S, int M, cudaStream_t s) {
  TG_CUDA(cudaMemsetAsync(bits, 0, 10 * sizeof(unsigned long long), s));
  size_t P = (size_t)nx * ny * nz;
  prof_begin(s, PC_FEAT, 3.0 * sizeof(T) * (double)P, 0);
  const size_t plane = (size_t)nx * ny;
  const unsigned bx = (unsigned)std::max<size_t>(1, std::min<size_t>((plane + 16 * kT - 1) / (16 * kT), 8));
  k_feature_max<T><<<dim3(bx, nz), kT, 0, s>>>(unl, nx, ny, nz, glz, lmx, lmy, bits);
  prof_end(s);
  TG_LAUNCH_CHECK("k_feature_max");
  k_feature_final<<<1, 32, 0, s>>>(feat, bits, du, S, M, nz);
  TG_LAUNCH_CHECK("k_feature_final");
}

// trapz(gridz, real(mean column) + shift)/2 into feat[slot] (arma::trapz, used at
// phase_carrier_flat.cc:509, phase_scalar_flat.cc:485-518)
__global__ void k_trapz_mean(const double2* __restrict__ f, int M, int nz, const double* __restrict__ gz, double shift,
                             double* feat, int slot) {
  // one warp: lane-strided intervals, then a shuffle sum
  double s = 0.0;
  for (int k = threadIdx.x; k < nz - 1; k += 32)
    s += (gz[k + 1] - gz[k]) * ((f[(size_t)k * M].x + shift) + (f[(size_t)(k + 1) * M].x + shift));
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) feat[slot] = s / 2 / 2;
}
void trapz_mean(const double2* f, int M, int nz, const double* gz, double shift, double* feat, int slot,
                cudaStream_t s) {
  prof_begin(s, PC_FEAT, 16.0 * (double)nz, 0);
  k_trapz_mean<<<1, 32, 0, s>>>(f, M, nz, gz, shift, feat, slot);
  prof_end(s);
  TG_LAUNCH_CHECK("k_trapz_mean");
}

__global__ void k_set_feat(double* feat, int slot, double v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) feat[slot] = v;
}
void set_feat(double* feat, int slot, double v, cudaStream_t s) {
  k_set_feat<<<1, 32, 0, s>>>(feat, slot, v);
  TG_LAUNCH_CHECK("k_set_feat");
}

// --- precision conversions for the mixed path --------------------------------------
template <typename A, typename B>
__global__ void k_convert(const A* __restrict__ a, B* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (B)a[i];
}

#define INST(T)                                                                                          \
  template void products6<T>(const T*, T*, size_t, cudaStream_t);                                      \
  template void adv_products<T>(const T*, const T*, T*, size_t, int, double, double, double, cudaStream_t); \
  template void phi_products<T>(const T*, const T*, T*, size_t, double, double, double, cudaStream_t);  \
  template void mul_shift<T>(const T*, const T*, T*, size_t, double, cudaStream_t);                     \
  template void erosion_tau<T>(const T*, const T*, T*, size_t, double, double, double, cudaStream_t);   \
  template void positivity_filter<T>(T*, int, int, cudaStream_t);                                       \
  template void features<T>(const T*, int, int, int, const double*, double, double, unsigned long long*, \
                            double*, const double2*, size_t, int, cudaStream_t);
INST(double)
INST(float)
#undef INST

}  // namespace tg

namespace tg {

// Swirling strength (FlatChannelPostprocessor::Execute,
// src/postprocessor_channel_flat.cc:209-230): lambda_ci = the largest
// |imaginary part| of the eigenvalues of A(i, j) = du_i/dx_j.  The eigenvalues
// of a real 3 x 3 matrix are the roots of lambda^3 - P lambda^2 + Q lambda - R
// (P trace, Q sum of the principal 2 x 2 minors, R determinant); with
// lambda = t + P/3 the depressed cubic t^3 + p t + q has a complex pair exactly
// when D = (q/2)^2 + (p/3)^3 > 0, and then (Cardano) the pair is
// -(u + v)/2 +- i sqrt(3)/2 (u - v) with u = cbrt(-q/2 + sqrt(D)), u v = -p/3.
__global__ void k_swirling(const double* __restrict__ g, size_t fstride, size_t n, double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double a[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = g[k * fstride + i];
    const double P = a[0] + a[4] + a[8];
    const double Q = (a[0] * a[4] - a[1] * a[3]) + (a[0] * a[8] - a[2] * a[6]) + (a[4] * a[8] - a[5] * a[7]);
    const double R = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
    const double p = Q - P * P / 3.0;
    const double q = -2.0 * P * P * P / 27.0 + P * Q / 3.0 - R;
    const double D = 0.25 * q * q + p * p * p / 27.0;
    double lci = 0.0;
    if (D > 0.0) {
      const double s = -0.5 * q;
      const double u = cbrt(s + copysign(sqrt(D), s));  // the root of larger magnitude
      const double v = u != 0.0 ? -p / (3.0 * u) : 0.0;
      lci = 0.86602540378443864676 * fabs(u - v);
    }
    out[i] = lci;
  }
}

void swirling(const double* grad9, size_t fstride, size_t n, double* out, cudaStream_t s) {
  k_swirling<<<nblk(n), kT, 0, s>>>(grad9, fstride, n, out);
  TG_LAUNCH_CHECK("k_swirling");
}

}  // namespace tg
