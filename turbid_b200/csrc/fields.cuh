// Launchers of the elementwise stage kernels and reductions (fields.cu).
#pragma once
#include "tg_common.cuh"

namespace tg {

void ref_to_slab(const double2* ref, double2* slab, int M, int nz, int dim, cudaStream_t s);
void slab_to_ref(const double2* slab, double2* ref, int M, int nz, int dim, cudaStream_t s);

template <typename T> void products6(const T* unl, T* prd, size_t P, cudaStream_t s);
template <typename T>
void adv_products(const T* unl, const T* dup, T* out, size_t P, int ncomp, double su, double sv, double sw,
                  cudaStream_t s);
template <typename T>
void phi_products(const T* phip, const T* unl, T* out, size_t P, double su, double sv, double sw, cudaStream_t s);
template <typename T> void mul_shift(const T* a, const T* b, T* out, size_t P, double sh, cudaStream_t s);

// dtf: when not null, the forcing pair (dt*f1, dt*f2) is read from device memory
void h_update(double2* H, const double2* adv, const double2* phi, size_t S, int M, double c1, double dt,
              double bcoef, double sinsl, double cossl, int sdir, double dtf1, double dtf2, const double* dtf,
              cudaStream_t s);
// H_c += sgn * bcoef * phi * trig; interior rows of rhs_c += a*c2 times that term
void buoyancy(double2* H, double2* rhs, const double2* phi, int M, int nz, double bcoef, double trig, int sgn,
              double ac2, cudaStream_t s);
void axmby(double2* y, const double2* x, size_t n, double a, double b, cudaStream_t s);
void boundary_apply(double2* rhs, const double2* hist, size_t S, int M, int nz, double fac, double r, int opentop,
                    double tu, double tv, double tw, cudaStream_t s);
// grad p enters as p (x and y components i kx p, i ky p) and dp/dz
void boundary_update(double2* hist, const double2* p, const double2* dpz, int M, int nz, int opentop,
                     const double* kx, const double* ky, const double* d1r0, const double* d1rn, cudaStream_t s);
void wall_dz(const double2* U, double2* DU, size_t S, int M, int nz, const double* d1r0, const double* d1rn,
             cudaStream_t s);
void project(double2* U, const double2* SU, const double2* P, const double2* DPZ, size_t S, int M, const double* kx,
             const double* ky, double coef, cudaStream_t s);
void zero_rows(double2* f, int M, int nz, cudaStream_t s);
template <typename T>
void erosion_tau(const T* dudz, const T* dvdz, T* tau, size_t n, double re, double tauc, double rate,
                 cudaStream_t s);
void erosion_row(double2* rhs, const double2* ero, const double2* phi, int M, double wsc, double conc, double resc,
                 double* feat, cudaStream_t s);
template <typename T> void positivity_filter(T* phip, int plane_n, int nz, cudaStream_t s);
template <typename T>
void features(const T* unl, int nx, int ny, int nz, const double* glz, double lmx, double lmy,
              unsigned long long* bits, double* feat, const double2* du, size_t S, int M, cudaStream_t s);
void trapz_mean(const double2* f, int M, int nz, const double* gz, double shift, double* feat, int slot,
                cudaStream_t s);
void set_feat(double* feat, int slot, double v, cudaStream_t s);
// swirling strength of n points; grad9 holds the nine gradient components
// du_i/dx_j (index 3 i + j), each fstride doubles apart
void swirling(const double* grad9, size_t fstride, size_t n, double* out, cudaStream_t s);

}  // namespace tg
