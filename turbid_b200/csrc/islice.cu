// FP64-accurate z-operator products from exact int8 tensor-core products
// (tcgen05.mma kind::i8, accumulators in tensor memory), for the dense
// Helmholtz solves of the mixed precision mode
// (reference: the E^-1 / E products of FlatCarrierPhase::Helmholtz and
// FlatScalarPhase::Helmholtz, src/phase_carrier_flat.cc:861-994,
// src/phase_scalar_flat.cc:635-667, through RealCplxCube::Multiply,
// src/cube_real_cplx.cc:461-471).
//
// Splitting (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of matrix
// multiplication", Numer. Algorithms 2012; integer slices as in Ootomo, Ozaki,
// Yokota, "DGEMM on integer matrix multiplication unit", 2024):
//   * the operator by rows and the data by columns, over the interior rows
//     k = 1 .. nz-2 only, into S slices of integers of magnitude <= 64, each
//     row / column scaled by a power of two 2^e with e from frexp of its
//     largest magnitude (|x| 2^-e <= 1): n = rint(x 2^-e 2^(6+7(S-1)))
//     (the only rounding), then n's signed base-128 digits in [-64, 63] from
//     the last slice up, the rest (in [-64, 64]) in slice 0;
//   * the slice pairs (p, q) with p + q < S multiplied exactly in int32, one
//     tensor-memory accumulator per diagonal d = p + q;
//   * the diagonals combined with weight 2^-(12+7d): exactly, as one int64
//     sum (below 2^53) converted to FP64, then the row and column scales;
//   * the two boundary rows of the data (z = 0 and z = nz-1; the scalar's
//     Robin rows carry values scaled by 1e7) as an FP64 rank-2 update:
//     out = (A[r][0] x0 + interior) + A[r][nz-1] x_{nz-1}.
//
// Layouts: one K-major tile per 128 data columns and slice (the MMA's A
// operand, M = 128 columns, K = 256 interior rows padded with zeros) and one
// K-major tile per BN operator rows and slice (the B operand, N = BN), both
// written in the canonical no-swizzle core-matrix order (8 rows x 16 bytes,
// K chunks 128 bytes apart, 8-row groups 2048 bytes apart) so that each tile
// is one contiguous bulk copy into shared memory.  The CTA keeps its 128
// columns' S data tiles in shared memory, walks the operator in chunks of BN
// rows (double-buffered bulk copies), and one thread issues the MMAs; after
// each chunk every thread reads its column's S accumulators from tensor memory
// (thread i = lane i = data column c0 + i) and stores the chunk's rows of its
// column, coalesced across the warp.  Every wait is bounded: a wait that gives
// up sets the error flag, the kernel drains what it issued (bounded too),
// frees its tensor memory and returns.
#include <cfloat>
#include <climits>
#include <cstdint>
#include <memory>
#include <vector>

#include "tg_common.cuh"

namespace tg {
namespace {

constexpr int KP = 256;                 // interior rows padded to 8 MMA K-steps of 32
constexpr int BM = 128;                 // data columns per CTA (MMA M, tensor-memory lanes)
constexpr int kGemmThreads = 512;        // 16 warps: 4 per lane quarter of the accumulators
constexpr int kTileX = BM * KP;         // bytes of one data tile
constexpr int kBadExp = INT_MIN;        // column exponent of a column holding NaN or inf
// A bounded wait polls at most kSpin times, each poll suspending the thread
// for at most kSuspendNs (a hint: it wakes as soon as the phase completes):
// about one second in all, far beyond any wait of a working product.
constexpr long long kSpin = 1ll << 20;
constexpr uint32_t kSuspendNs = 1000;

template <int S>
struct IslShape {
  static constexpr int BN = S <= 5 ? 96 : (S == 6 ? 80 : 64);   // S * BN accumulator columns <= 512
  static constexpr int kTileA = BN * KP;
  static constexpr int kRowsMax = 288;   // rows of the padded operator (nz <= 258 and BN = 96: 3 chunks)
  static constexpr size_t kSmem = 1024 + (size_t)S * kTileX + 2 * (size_t)kTileA + 4 * kRowsMax * sizeof(double);
  static_assert(kTileA % 2048 == 0, "half tiles must keep 1024-byte atom alignment");
  static_assert(S * BN <= 512, "one accumulator per slice diagonal must fit tensor memory");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "MMA N for M = 128");
};

// Byte offset of element (row, k) in a tile of `rows` rows, K-major with the
// 128-byte swizzle: the K range is cut into two 128-byte halves stored one
// after the other; within a half, 8-row atoms of 8 x 128 bytes lie 1024 bytes
// apart and the 16-byte chunk c of row r of an atom sits at chunk c ^ (r & 7)
// (so the tensor cores' and the slicer's accesses spread over all banks).
__host__ __device__ constexpr int ksw_off(int rows, int row, int k) {
  return (k >> 7) * (rows * 128) + (row >> 3) * 1024 + (row & 7) * 128 + ((((k & 127) >> 4) ^ (row & 7)) << 4) +
         (k & 15);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile of
// `rows` rows (1024-byte aligned), at the MMA K-step kk (32 bytes of K each)
__device__ __forceinline__ uint64_t smem_desc(uint32_t tile, int rows, int kk) {
  const uint32_t saddr = tile + (uint32_t)(kk >> 2) * (uint32_t)(rows * 128) + (uint32_t)(kk & 3) * 32u;
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);   // start address
  d |= (uint64_t)1 << 16;                   // leading byte offset (unused with the swizzle; 16 bytes)
  d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset: 8-row atoms
  d |= (uint64_t)1 << 46;                   // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                   // layout: 128-byte swizzle
  return d;                                 // base offset 0 (atoms 1024-byte aligned)
}

// instruction descriptor: s32 accumulator, signed 8-bit A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// true once the phase with the given parity has completed; false after kSpin polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kSpin; ++i) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity), "n"(kSuspendNs)
        : "memory");
    if (done) return true;
  }
  return false;
}
// global -> shared bulk copy (16-byte aligned, size a multiple of 16), completion on bar
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ double max_keep_nan(double a, double b) { return (b > a || isnan(b)) ? b : a; }

// 2^(6 + 7 (S - 1)): the grid of the last slice (slice 0 holds 6 bits and a
// sign, every further slice 7 bits and a sign)
template <int S>
constexpr double kGrid = (double)(1ll << (6 + 7 * (S - 1)));
// 64 (1 + 128 + ... + 128^(S-2)): makes the digits of slices 1 .. S-1 non-negative
template <int S>
constexpr long long kBias = (S <= 1) ? 0 : 64 * (((1ll << (7 * (S - 1))) - 1) / 127);

// ---------------------------------------------------------------------------
// Data slicing: a CTA of 16 warps slices 32 columns; warp q reads the 16
// interior rows of K chunk q (rows 16 q + 1 .. 16 q + 16) of its 32 columns
// (lane = column: 256 contiguous bytes per row), keeps them in registers, the
// column maxima meet in shared memory, and each warp writes the S slices of
// its K chunk into the column tile's image (16 bytes per column and slice).
// blockIdx.y selects the problem of a group.
// ---------------------------------------------------------------------------
constexpr int kMaxIsl = 3;
constexpr int kSliceCols = 32;
constexpr int kSliceThreads = kSliceCols * (KP / 16);   // 512

struct SliceArgs {
  const double* in[kMaxIsl];   // FP64 component, row-major [nz][ncol]
  int8_t* xs[kMaxIsl];         // data tiles [tile][S][kTileX]
  int* xe[kMaxIsl];            // column exponents [tile * 128 + i]
  int nz, ncol;
};

template <int S>
__global__ void __launch_bounds__(kSliceThreads) k_slice_data(const SliceArgs a) {
  __shared__ double part_max[KP / 16][kSliceCols];
  const int lane = threadIdx.x & 31, kc = threadIdx.x >> 5;   // column in the block, K chunk
  const int pb = blockIdx.y;
  const int c = blockIdx.x * kSliceCols + lane;
  const bool valid = c < a.ncol;
  // select the problem's pointers without indexing the parameter arrays
  // dynamically (that would copy them to local memory)
  const double* X = pb == 0 ? a.in[0] : (pb == 1 ? a.in[1] : a.in[2]);
  int8_t* xs = pb == 0 ? a.xs[0] : (pb == 1 ? a.xs[1] : a.xs[2]);
  int* xe = pb == 0 ? a.xe[0] : (pb == 1 ? a.xe[1] : a.xe[2]);
  double x[16];
  double mx = 0.0;
#pragma unroll
  for (int kk = 0; kk < 16; ++kk) {
    const int z = kc * 16 + kk + 1;
    x[kk] = (valid && z < a.nz - 1) ? X[(size_t)z * a.ncol + c] : 0.0;
    mx = max_keep_nan(mx, fabs(x[kk]));
  }
  part_max[kc][lane] = mx;
  __syncthreads();
  mx = 0.0;
#pragma unroll
  for (int q = 0; q < KP / 16; ++q) mx = max_keep_nan(mx, part_max[q][lane]);
  int e = 0;
  const bool bad = !(mx <= DBL_MAX);
  if (!bad && mx > 0.0) {
    int ee = 0;
    const double f = frexp(mx, &ee);
    e = f == 0.5 ? ee - 1 : ee;
  }
  const int tile = c / BM, t = c % BM;   // column tile and column within it
  if (valid && kc == 0) xe[c] = bad ? kBadExp : e;
  if (!valid && c >= (a.ncol + BM - 1) / BM * BM) return;   // beyond the last tile
  uint32_t w[S][4];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int j = 0; j < 4; ++j) w[p][j] = 0u;
  // 2^(6+7(S-1)-e) as one exact power-of-two factor when it is a normal
  // double (any column whose maximum is above 2^-980), else ldexp per value
  const int sh = 6 + 7 * (S - 1) - e;
  const bool fast = sh <= 1023;
  const double scale = fast ? ldexp(1.0, sh) : 0.0;
#pragma unroll
  for (int kk = 0; kk < 16; ++kk) {
    // the column value on the 2^-(6+7(S-1)) grid of its scale (the one
    // rounding), then its signed base-128 digits: with the bias
    // 64 (1 + 128 + ... + 128^(S-2)) the digits of slices 1 .. S-1 are the
    // plain base-128 digits of the low 7 (S-1) bits, less 64, and slice 0 is
    // the rest (the unique representation the digit-by-digit rule gives)
    const double xv = bad ? 0.0 : x[kk];
    const long long n = __double2ll_rn(fast ? xv * scale : ldexp(xv, -e) * kGrid<S>);
    const long long u = n + kBias<S>;
    const uint32_t lo = (uint32_t)u;
#pragma unroll
    for (int p = 1; p < S; ++p) {
      const uint32_t dg = ((lo >> (7 * (S - 1 - p))) & 127u) + 0xC0u;   // (digit - 64) as a byte
      w[p][kk >> 2] |= (dg & 0xffu) << (8 * (kk & 3));
    }
    w[0][kk >> 2] |= ((uint32_t)(int)(u >> (7 * (S - 1))) & 0xffu) << (8 * (kk & 3));
  }
  int8_t* dst = xs + (size_t)tile * S * kTileX;
#pragma unroll
  for (int p = 0; p < S; ++p)
    *reinterpret_cast<uint4*>(dst + (size_t)p * kTileX + ksw_off(BM, t, kc * 16)) =
        make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

struct IslProblem {
  const int8_t* xs;     // data tiles [tile][S][kTileX]
  const int* xe;        // column exponents [tile * 128 + i]
  const int8_t* as;     // operator chunk tiles [chunk][S][BN * KP]
  const double* a0;     // [rows_pad] A[r][0]
  const double* an;     // [rows_pad] A[r][nz-1]
  const double* asc;    // [rows_pad] 2^(row exponent)
  const double* in;     // FP64 input component (its boundary rows are read)
  double* out;
  EpiParams ep;         // EPI_STORE or EPI_RSCALE
};
struct IslArgs {
  IslProblem p[kMaxIsl];   // blockIdx.y selects the problem
  int nz, nrow, ncol, ntiles, nchunks;
  int* err;
  int withhold;            // failure-path check: the operator copies are never issued
};

// One CTA per 128 data columns, 16 warps.  Thread 0 issues the bulk copies
// and the MMAs; the operator is streamed in half tiles (BN rows x 128 bytes of
// K, one contiguous block of the swizzled tile) through four buffers, three
// copies ahead of the MMAs.  After each chunk of BN operator rows all warps
// read the accumulators: warp w reads tensor-memory lanes 32 (w % 4) .. +31
// (data columns) and every fourth 8-row group of the chunk starting at w / 4.
template <int S>
__global__ void __launch_bounds__(kGemmThreads, 1) k_islice_gemm(const IslArgs args) {
  using Sh = IslShape<S>;
  constexpr int BN = Sh::BN;
  constexpr int kHalf = Sh::kTileA / 2;               // bytes of one half tile
  constexpr int NBUF = 4;
  constexpr uint32_t idesc = idesc_i8(BM, BN);
  extern __shared__ __align__(16) uint8_t sm_raw[];
  // swizzle atoms need 1024-byte alignment: round the base up (1 KB reserved)
  uint8_t* sm = sm_raw + ((1024 - (smem_u32(sm_raw) & 1023)) & 1023);
  uint8_t* sx = sm;                                   // S data tiles
  uint8_t* sa = sm + (size_t)S * kTileX;              // four operator half tiles
  double* s_aux = reinterpret_cast<double*>(sa + NBUF * kHalf);   // a0, an, asc, lam: 4 x kRowsMax
  __shared__ __align__(8) uint64_t bars[2 + 2 * NBUF];  // data, accumulators, full[4], empty[4]
  __shared__ uint32_t tmem_slot;
  __shared__ int s_err;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x;
  const IslProblem& a = args.p[blockIdx.y];
  const uint32_t bar_x = smem_u32(&bars[0]), bar_acc = smem_u32(&bars[1]);
  auto bar_full = [&](int i) { return smem_u32(&bars[2 + i]); };
  auto bar_empty = [&](int i) { return smem_u32(&bars[2 + NBUF + i]); };
  const int total = args.nchunks * S * 2;   // (chunk, operator slice, K half) iterations

  if (tid == 0) {
    s_err = 0;
    for (int i = 0; i < 2 + 2 * NBUF; ++i) mbar_init(smem_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // per-row epilogue constants: boundary columns, row scale, eigenvalue
  const int rows_pad = args.nchunks * BN;
  for (int r = tid; r < rows_pad; r += kGemmThreads) {
    s_aux[r] = a.a0[r];
    s_aux[Sh::kRowsMax + r] = a.an[r];
    s_aux[2 * Sh::kRowsMax + r] = a.asc[r];
    s_aux[3 * Sh::kRowsMax + r] = (a.ep.mode == EPI_RSCALE && r < args.nz) ? a.ep.lam[r] : 0.0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;

  // operator loads issued (load i goes to buffer i % NBUF), so that an early
  // exit can drain them
  int issued = 0;
  auto issue_op_load = [&](int it) {
    if (args.withhold) return;   // failure-path check: the full-buffer wait will give up
    const int buf = it % NBUF;
    // iteration order = chunk-major, slice, K half: the half tiles lie in that order
    const int8_t* src = a.as + (size_t)it * kHalf;
    mbar_expect_tx(bar_full(buf), kHalf);
    bulk_g2s(smem_u32(sa + buf * kHalf), src, kHalf, bar_full(buf));
    issued = it + 1;
  };
  if (tid == 0) {
    mbar_expect_tx(bar_x, S * kTileX);
    for (int p = 0; p < S; ++p)
      bulk_g2s(smem_u32(sx + p * kTileX), a.xs + ((size_t)tile * S + p) * kTileX, kTileX, bar_x);
    for (int i = 0; i < NBUF - 1 && i < total; ++i) issue_op_load(i);
    if (!mbar_wait(bar_x, 0)) s_err = 1;
  }

  // per-thread column constants: this thread's lane quarter and column
  const int ncol = args.ncol, nz = args.nz;
  const int quarter = warp & 3, rgrp = warp >> 2;   // rows: 8-row groups rgrp, rgrp + 4, ...
  const int c = tile * BM + quarter * 32 + lane;
  const bool valid = c < ncol;
  const double xb = valid ? a.in[c] : 0.0;
  const double xt = valid ? a.in[(size_t)(nz - 1) * ncol + c] : 0.0;
  const int e = valid ? a.xe[tile * BM + quarter * 32 + lane] : 0;
  const bool bad = e == kBadExp;
  const double csc = bad ? 0.0 : ldexp(1.0, e);
  const int m = c >> 1;
  const bool rscale = a.ep.mode == EPI_RSCALE;
  const double k2m = (rscale && valid) ? a.ep.k2[m] : 0.0;
  double* out = a.out;

  int it = 0;
  for (int j = 0; j < args.nchunks; ++j) {
    if (tid == 0 && !s_err) {
      for (int p = 0; p < S && !s_err; ++p) {
        for (int h = 0; h < 2; ++h, ++it) {
          const int buf = it % NBUF;
          if (!mbar_wait(bar_full(buf), (it / NBUF) & 1)) {
            s_err = 1;
            ++it;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t sa_addr = smem_u32(sa + buf * kHalf);
          for (int q = 0; q < S - p; ++q) {
            const uint32_t dacc = tmem + (uint32_t)((p + q) * BN);
            const uint32_t sx_addr = smem_u32(sx + q * kTileX);
#pragma unroll
            for (int kl = 0; kl < 4; ++kl) {
              const uint64_t da = smem_desc(sx_addr, BM, 4 * h + kl);
              const uint64_t db = smem_desc(sa_addr, BN, kl);
              const uint32_t acc = (p == 0 && h == 0 && kl == 0) ? 0u : 1u;   // p = 0 opens every diagonal
              asm volatile(
                  "{\n\t.reg .pred pd;\n\t"
                  "setp.ne.b32 pd, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, pd;\n\t}" ::"r"(dacc),
                  "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              bar_empty(buf)));
          // refill the buffer of the previous iteration, NBUF - 1 iterations ahead
          const int next = it + NBUF - 1;
          if (next < total) {
            if (it >= 1 && !mbar_wait(bar_empty((it - 1) % NBUF), ((it - 1) / NBUF) & 1)) {
              s_err = 1;
              ++it;
              break;
            }
            issue_op_load(next);
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_acc));
    }
    // every thread: the chunk's accumulators are complete
    bool ok = mbar_wait(bar_acc, j & 1);
    ok = __all_sync(0xffffffffu, ok);   // warp-uniform: the tensor-memory loads below are .sync.aligned
    if (!ok) s_err = 1;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
      const int r0 = j * BN;
#pragma unroll 1
      for (int jg = rgrp * 8; jg < BN; jg += 32) {
        // the S diagonals' accumulators of 8 rows, all loads in flight before one wait
        uint32_t v[S][8];
#pragma unroll
        for (int d = 0; d < S; ++d) {
          const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(d * BN + jg);
          asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                       : "=r"(v[d][0]), "=r"(v[d][1]), "=r"(v[d][2]), "=r"(v[d][3]), "=r"(v[d][4]), "=r"(v[d][5]),
                         "=r"(v[d][6]), "=r"(v[d][7])
                       : "r"(taddr));
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // RSCALE: the reciprocal of a row pair is computed once per mode, the
        // even lane of a (re, im) lane pair taking the first row and the odd
        // lane the second, and exchanged
        double Rpair[8];
        if (rscale) {
#pragma unroll
          for (int i = 0; i < 8; i += 2) {
            const int rm = r0 + jg + i + (lane & 1);
            double R = 1.0;
            if (rm != 0 && rm < nz - 1) {
              const double lam = s_aux[3 * Sh::kRowsMax + rm];
              R = __drcp_rn((k2m + lam) + a.ep.sigma);   // correctly rounded 1 / x
              if (a.ep.null_mode && m == 0 && fabs(lam) < 10e-12) R = 0.0;
            }
            const double Ro = __shfl_xor_sync(0xffffffffu, R, 1);
            Rpair[i] = (lane & 1) ? Ro : R;
            Rpair[i + 1] = (lane & 1) ? R : Ro;
          }
        }
        if (valid) {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int r = r0 + jg + i;
            // sum_d D_d 2^-(12+7d) = 2^-(12+7(S-1)) sum_d D_d 2^(7(S-1-d)): an
            // integer below 2^53 in magnitude (|D_d| <= (d+1) 2^20), so the
            // int64 sum and its conversion to FP64 are exact
            long long isum = (int)v[0][i];
#pragma unroll
            for (int d = 1; d < S; ++d) isum = isum * 128 + (int)v[d][i];
            const double acc = __ll2double_rn(isum) * (1.0 / (double)(1ll << (12 + 7 * (S - 1))));
            if (r < args.nrow) {
              const double interior = __dmul_rn(__dmul_rn(acc, s_aux[2 * Sh::kRowsMax + r]), csc);
              double val = __dadd_rn(__dadd_rn(__dmul_rn(s_aux[r], xb), interior),
                                     __dmul_rn(s_aux[Sh::kRowsMax + r], xt));
              if (bad) val = __longlong_as_double(0x7ff8000000000000LL);
              if (rscale) val = __dmul_rn(val, Rpair[i]);
              out[(size_t)r * ncol + c] = val;
            }
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();   // accumulators read before the next chunk's MMAs overwrite them
    if (s_err) break;  // uniform: read after the barrier
  }
  // drain: every bulk copy issued must have landed before the shared memory is
  // released (the MMAs were awaited through the accumulator barrier)
  if (tid == 0 && s_err) {
    mbar_wait(bar_x, 0);
    for (int k = 0; k < NBUF && k < issued; ++k) {
      const int nk = (issued - 1 - k) / NBUF + 1;   // loads into buffer k
      mbar_wait(bar_full(k), (nk - 1) & 1);
    }
    atomicExch(args.err, 1);
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct IsliceOp {
  int S = 0, nz = 0, nrow = 0, nchunks = 0, BN = 0;
  int8_t* as = nullptr;   // operator chunk tiles
  double* aux = nullptr;  // a0, an, asc: 3 x rows_pad
  // slicing scratch for one component of M modes
  int8_t* xs = nullptr;
  int* xe = nullptr;
  int ntiles = 0, ncol = 0;
  int* err = nullptr;
};

namespace {
template <int S>
void islice_set_smem() {
  TG_CUDA(cudaFuncSetAttribute(k_islice_gemm<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)IslShape<S>::kSmem));
}
}  // namespace

// Slices of an nrow x nz operator (row-major FP64) for S slices, in the chunk
// tile order of the kernel; the same rule as the data slicing, per row over
// the interior columns.  Returns the row exponents' scales and the boundary
// columns in aux.
static void slice_operator_host(const std::vector<double>& A, int nrow, int nz, int S, int BN, int nchunks,
                                std::vector<int8_t>& tiles, std::vector<double>& aux) {
  const int rows_pad = nchunks * BN;
  tiles.assign((size_t)nchunks * S * BN * KP, 0);
  aux.assign((size_t)3 * rows_pad, 0.0);
  for (int r = 0; r < nrow; ++r) {
    double mx = 0.0;
    for (int k = 1; k < nz - 1; ++k) mx = std::max(mx, std::fabs(A[(size_t)r * nz + k]));
    int e = 0;
    if (mx > 0.0) {
      int ee = 0;
      const double f = std::frexp(mx, &ee);
      e = f == 0.5 ? ee - 1 : ee;
    }
    aux[r] = A[(size_t)r * nz];
    aux[rows_pad + r] = A[(size_t)r * nz + nz - 1];
    aux[2 * rows_pad + r] = std::ldexp(1.0, e);
    const int j = r / BN, rr = r % BN;
    const double grid = std::ldexp(1.0, 6 + 7 * (S - 1));
    for (int k = 0; k + 1 < nz - 1; ++k) {
      long long n = std::llrint(std::ldexp(A[(size_t)r * nz + k + 1], -e) * grid);   // ties to even
      for (int p = S - 1; p >= 1; --p) {
        const int dg = (int)(((n + 64) & 127) - 64);
        n = (n - dg) >> 7;
        tiles[((size_t)j * S + p) * BN * KP + ksw_off(BN, rr, k)] = (int8_t)dg;
      }
      tiles[((size_t)j * S + 0) * BN * KP + ksw_off(BN, rr, k)] = (int8_t)n;
    }
  }
}

void islice_build(IsliceOp*& op, const std::vector<double>& A, int nrow, int nz, int S, int M,
                  const std::function<void*(size_t)>& alloc, int* err) {
  if (S != 5) throw Error{TG_ERR_ARG, "islice > only 5 slices are built"};
  if (nz < 3 || nz - 2 > KP) throw Error{TG_ERR_SHAPE, "islice > nz - 2 must be at most 256"};
  if ((size_t)A.size() != (size_t)nrow * nz) throw Error{TG_ERR_SHAPE, "islice > operator size"};
  static bool smem_set = false;
  if (!smem_set) {
    islice_set_smem<5>();
    smem_set = true;
  }
  const int BN = IslShape<5>::BN, nchunks = (nrow + BN - 1) / BN;
  if (op && (op->nz != nz || op->nrow != nrow || op->ncol != 2 * M))
    throw Error{TG_ERR_SHAPE, "islice > rebuild with another shape"};
  std::vector<int8_t> tiles;
  std::vector<double> aux;
  slice_operator_host(A, nrow, nz, S, BN, nchunks, tiles, aux);
  if (!op) {
    std::unique_ptr<IsliceOp> o(new IsliceOp);
    o->S = S;
    o->nz = nz;
    o->nrow = nrow;
    o->BN = BN;
    o->nchunks = nchunks;
    o->ncol = 2 * M;
    o->ntiles = (o->ncol + BM - 1) / BM;
    o->as = static_cast<int8_t*>(alloc(tiles.size()));
    o->aux = static_cast<double*>(alloc(aux.size() * sizeof(double)));
    o->xs = static_cast<int8_t*>(alloc((size_t)o->ntiles * S * kTileX));
    o->xe = static_cast<int*>(alloc((size_t)o->ntiles * BM * sizeof(int)));
    if (err) {
      o->err = err;   // the caller's flag (shared by its products)
    } else {
      o->err = static_cast<int*>(alloc(sizeof(int)));
      TG_CUDA(cudaMemset(o->err, 0, sizeof(int)));
    }
    op = o.release();
  }
  TG_CUDA(cudaMemcpy(op->as, tiles.data(), tiles.size(), cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(op->aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice));
}

void islice_destroy(IsliceOp* op) { delete op; }   // device buffers belong to the allocator's owner

// Problems of one group: each batch component of each problem is one problem of
// the launch pair (slicing, then product), at most kMaxIsl per pair.
void islice_group(const IsliceOp* const* ops, const double2* const* ins, double2* const* outs,
                  const EpiParams* eps, int n, int M, cudaStream_t s, bool withhold_operator) {
  using Sh = IslShape<5>;
  if (n < 1 || n > kMaxIsl) throw Error{TG_ERR_ARG, "islice > bad group size"};
  const IsliceOp& op0 = *ops[0];
  SliceArgs sa{};
  IslArgs a{};
  for (int i = 0; i < n; ++i) {
    const IsliceOp& op = *ops[i];
    if (2 * M != op.ncol || op.nz != op0.nz || op.nrow != op0.nrow)
      throw Error{TG_ERR_SHAPE, "islice > operators of one group differ in shape"};
    if (eps[i].mode != EPI_STORE && eps[i].mode != EPI_RSCALE)
      throw Error{TG_ERR_ARG, "islice > unsupported epilogue"};
    if (reinterpret_cast<const void*>(ins[i]) == reinterpret_cast<const void*>(outs[i]))
      throw Error{TG_ERR_ARG, "islice > input and output must differ"};
    sa.in[i] = reinterpret_cast<const double*>(ins[i]);
    sa.xs[i] = op.xs;
    sa.xe[i] = op.xe;
    IslProblem& p = a.p[i];
    const int rows_pad = op.nchunks * op.BN;
    p.xs = op.xs;
    p.xe = op.xe;
    p.as = op.as;
    p.a0 = op.aux;
    p.an = op.aux + rows_pad;
    p.asc = op.aux + 2 * rows_pad;
    p.in = reinterpret_cast<const double*>(ins[i]);
    p.out = reinterpret_cast<double*>(outs[i]);
    p.ep = eps[i];
  }
  sa.nz = op0.nz;
  sa.ncol = op0.ncol;
  a.nz = op0.nz;
  a.nrow = op0.nrow;
  a.ncol = op0.ncol;
  a.ntiles = op0.ntiles;
  a.nchunks = op0.nchunks;
  a.err = op0.err;
  a.withhold = withhold_operator ? 1 : 0;
  const double by = n * (16.0 * M * op0.nz * 2 + (double)op0.ntiles * 5 * kTileX * 2);
  const double fl = n * 4.0 * op0.nz * op0.nz * (double)M;
  prof_begin(s, PC_ISLICE, by, fl, fl);
  k_slice_data<5><<<dim3(op0.ntiles * (BM / kSliceCols), n), kSliceThreads, 0, s>>>(sa);
  TG_LAUNCH_CHECK("k_slice_data");
  k_islice_gemm<5><<<dim3(op0.ntiles, n), kGemmThreads, Sh::kSmem, s>>>(a);
  prof_end(s);
  TG_LAUNCH_CHECK("k_islice_gemm");
}

// out = epi(A in) for `batch` components of M modes (strides in complex
// elements), in groups through the op's single slicing scratch: the
// components run one after another.
void islice_apply(const IsliceOp& op, const double2* in, long long in_stride, double2* out, long long out_stride,
                  int M, int batch, const EpiParams& ep, cudaStream_t s) {
  for (int b = 0; b < batch; ++b) {
    const IsliceOp* o = &op;
    const double2* i = in + (size_t)b * in_stride;
    double2* r = out + (size_t)b * out_stride;
    islice_group(&o, &i, &r, &ep, 1, M, s);
  }
}

// The error flag of the op's bounded waits (a synchronous read: call between steps).
int islice_error(const IsliceOp& op) {
  int v = 0;
  TG_CUDA(cudaMemcpy(&v, op.err, sizeof(int), cudaMemcpyDeviceToHost));
  return v;
}
void islice_clear_error(const IsliceOp& op) { TG_CUDA(cudaMemset(op.err, 0, sizeof(int))); }

}  // namespace tg
