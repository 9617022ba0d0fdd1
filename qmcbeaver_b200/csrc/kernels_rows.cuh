// kernels_rows.cuh -- batched orbital rows on the tcgen05 tensor cores.
//
// The orbital contraction of a single-electron move (QMCSlater::update_Ds
// -> Array2D::gemm, QMcBeaver/src/QMCSlater.cpp:856-862): the five rows
// chi, d/dx chi, d/dy chi, d/dz chi, lap chi of the moved electron's basis
// values times the spin's MO coefficients, D[r][o] = sum_k chi[r][k] C[o][k].
// Every walker of a step moves the same electron, so the rows of all walkers
// form one GEMM with a shared B operand: M = 5 x walkers, N = n orbitals,
// K = basis functions.
//
// FP64-equivalent rows from integer tensor-core products (the slice scheme
// of Ozaki, Ogita, Oishi, Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), in its integer form of
// Ootomo, Ozaki, Yokota, "DGEMM on integer matrix multiplication unit",
// IJHPCA 2024): every 32-function block of a row of chi and of an orbital of
// C is scaled by a power of two to |x| < 1 and cut into kSlices signed 7-bit
// digits,
//   x = scale * sum_s d_s 2^-(6 + 7 s),  |d_s| <= 64,
// the digit products of a block, sum_k a_i[r][k] b_j[k][o] over 32 k, are
// exact in int32 (|a b| <= 2^12), and the pairs with i + j = t share one TMEM
// accumulator (weight 2^-(12 + 7 t)).  The pairs with i + j < kSlices keep
// 56 bits of every product relative to the block's largest basis value and
// largest coefficient, and every block is rescaled and added in FP64: the
// rows carry the error of an FP64 dot product over the blocks' magnitudes.
// Per-row scales (one per row over all of K) are not enough: basis values of
// distant centres sit many orders below the row's largest, and their terms
// then lose the bits the Slater updates need (Slater matrices of random
// 50 x 50 orbitals reach condition numbers of 1e6, which amplify any
// FP32-class row error to 1e-1 Ha in the local energy).
//
//   k_rows_prep  one warp per walker: the move's proposal (the same draws as
//                the move kernel, which recomputes it), the basis values at
//                the proposed position, their per-row scales and int8 digits
//                in the tensor-core operand layout
//   k_rows_mma   one CTA per tile of 25 walkers (125 rows) and 32 orbitals:
//                int8 x int8 -> int32 tcgen05.mma (kind::i8, M = 128, N = 32,
//                K = 32 per instruction) over kSlices (kSlices + 1) / 2 digit
//                pairs per K step, operands staged in shared memory by
//                bulk copies (the TMA engine, 4 stages, one thread), two TMEM
//                accumulator buffers (one K step fills one while the eight
//                warps drain the other into FP64 registers); writes
//                rows[walker][5][n]
// The move kernel then reads the rows instead of evaluating the basis and
// contracting (MoveArgs::rows).
#pragma once

#include <cstring>

#include "kernels.cuh"

namespace qmcb {

constexpr int kSlices = 8;       // int8 digits per operand value
constexpr int kTileRows = 128;   // MMA M: TMEM lanes
constexpr int kTileWalkers = 25; // walkers per tile: rows 0 .. 124 used
constexpr int kNTile = 32;       // MMA N: orbitals per CTA
constexpr int kKStep = 32;       // int8 K of one MMA (bytes); also the block of K sharing a scale
constexpr int kABlock = kTileRows * kKStep;  // one digit plane of one K step of an A tile
constexpr int kBBlock = kNTile * kKStep;     // the same for B
constexpr int kRowsStages = 4;
constexpr int kRowsStageBytes = kSlices * (kABlock + kBBlock);
constexpr int kRowsSmem = kRowsStages * kRowsStageBytes + 1024;  // + barriers; > 113 KB: one CTA per SM
constexpr int kRowsThreads = 256;  // two warps per TMEM lane quarter, each draining half the columns
static_assert(kRowsStageBytes % 16 == 0 && kABlock % 16 == 0, "bulk copies move multiples of 16 bytes");
// two buffers of kSlices accumulators of kNTile int32 columns: the MMAs of
// one K step fill one buffer while the epilogue drains the other
constexpr uint32_t kRowsTmemCols = 512;
constexpr int kAccCols = kSlices * kNTile;  // columns of one buffer
static_assert(2 * kAccCols <= (int)kRowsTmemCols, "accumulators exceed the TMEM allocation");

// Byte offset of (row r, k) in one K-step block of the no-swizzle K-major
// operand layout: 8 x 16-byte core matrices, the two K halves 128 bytes
// apart (leading-dimension offset), 8-row groups 256 bytes apart (stride
// offset).
__host__ __device__ inline int rows_blk_off(int r, int k)
{
  return (r >> 3) * 256 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

// Digits of x (|x| < 1 after scaling): q = rint(x 2^(7 kSlices - 1)) is cut
// into balanced base-128 digits from the top, d_s = round(q_s / 2^w_s) with
// w_s = 7 (kSlices - 1 - s) and q_{s+1} = q_s - d_s 2^w_s, so that
// x = sum_s d_s 2^-(6 + 7 s) up to the rounding of q (2^-(7 kSlices - 1)),
// |d_s| <= 64.  q = hi 2^28 + lo with hi = rint(x 2^27) and lo =
// rint((x 2^27 - hi) 2^28) (the subtraction is exact), |hi|, |lo| <= 2^27:
// each half gives four digits in 32-bit integer arithmetic.
__host__ __device__ inline void rows_digits(double x, signed char *d)
{
  static_assert(kSlices == 8, "two halves of four digits");
  const double xs = x * 134217728.0;  // 2^27: exact
  const double h = rint(xs);
  const int half[2] = {(int)h, (int)rint((xs - h) * 268435456.0)};  // 2^28: exact
#pragma unroll
  for (int p = 0; p < 2; p++) {
    int q = half[p];
#pragma unroll
    for (int t = 0; t < 3; t++) {
      const int w = 21 - 7 * t;
      const int ds = (q + (1 << (w - 1))) >> w;  // arithmetic shift: floor
      d[4 * p + t] = (signed char)ds;
      q -= ds * (1 << w);
    }
    d[4 * p + 3] = (signed char)q;
  }
}

// Power-of-two scale 2^e with max |x| < 2^e (1 for an all-zero row).
__host__ __device__ inline double rows_scale(double amax)
{
  if (!(amax > 0.0)) return 1.0;
  int ex;
  frexp(amax, &ex);  // amax = f 2^ex, f in [0.5, 1)
  return ldexp(1.0, ex);
}

// ------------------------------------------------------------------------
// k_rows_prep: list entries [0, num) (d_num: device count); warp scratch:
// the staged positions and modified drift (2 x 3N, read by the proposal),
// then, in the same space, the exponential slots.  The basis rows stay in
// registers: lane l evaluates the four consecutive functions 4 l .. 4 l + 3
// of every 128 (the eight lanes of a 32-function K block are one shuffle
// group for its scale), so no [5][K] row array occupies shared memory.
__host__ __device__ inline int rows_prep_doubles(int N, int K, int nslot)
{
  (void)K;
  return max(2 * even(3 * N), even(nslot));
}

template <bool kMetropolis, bool kExtras>
__global__ void __launch_bounds__(128) k_rows_prep(DevSys S, Layout L, RunCfg cfg, const double *state,
                                                    const int *slots, int num, const int *d_num, const double *R_in,
                                                    MoveArgs mv, int ksteps, signed char *A, double *rscale)
{
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = lane_id();
  const int nw = d_num ? *d_num : num;
  const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (wi >= nw) return;
  const int N = S.N, K = S.K, e = mv.e;
  double *sm = smem + (size_t)warp * rows_prep_doubles(N, K, S.nslot);
  double *sR = sm, *smg = sm + even(3 * N), *ex = sm;
  const int slot = slots ? slots[wi] : wi;
  const double *blk = state + (size_t)slot * L.stride;
  for (int t = lane; t < 3 * N; t += 32) {
    sR[t] = blk[L.R + t];
    smg[t] = blk[L.mgrad + t];
  }
  __syncwarp();
  const double ro[3] = {sR[3 * e], sR[3 * e + 1], sR[3 * e + 2]};
  double rn[3], g_fwd, u_acc;
  propose_move<kMetropolis, kExtras>(S, cfg, slot, mv.step, e, N, sR, ro, smg, R_in, wi, rn, g_fwd, u_acc, mv.rin_moved);
  __syncwarp();  // the slots overwrite the staged arrays
  basis_slot_exps_warp(S, rn, ex);
  __syncwarp();
  // rows 5 wi .. 5 wi + 4 of the GEMM
  const int row0 = 5 * wi, tile = row0 / (5 * kTileWalkers), r0 = row0 - tile * 5 * kTileWalkers;
  const unsigned gmask = 0xFFu << (8 * (lane >> 3));
  for (int k0 = 4 * lane; k0 < ksteps * kKStep; k0 += 128) {
    double v[4][5];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (k0 + u < K) {
        basis_function_rows(S, rn, k0 + u, ex, v[u]);
      } else {
#pragma unroll
        for (int d = 0; d < 5; d++) v[u][d] = 0.0;
      }
    }
    const int kk = k0 / kKStep;
#pragma unroll
    for (int d = 0; d < 5; d++) {
      // the K block's scale of row d: the largest of the eight lanes' values
      double m = fmax(fmax(fabs(v[0][d]), fabs(v[1][d])), fmax(fabs(v[2][d]), fabs(v[3][d])));
      m = fmax(m, __shfl_xor_sync(gmask, m, 4));
      m = fmax(m, __shfl_xor_sync(gmask, m, 2));
      m = fmax(m, __shfl_xor_sync(gmask, m, 1));
      const double scale = rows_scale(m), inv = 1.0 / scale;  // exact: a power of two
      // a walker's five rows lie in one tile (25 walkers = 125 rows)
      const int r = r0 + d;
      if ((lane & 7) == 0) rscale[(size_t)(row0 + d) * ksteps + kk] = scale;
      // four consecutive k per lane: one 4-byte store per digit plane
      uint32_t w[kSlices];
#pragma unroll
      for (int s = 0; s < kSlices; s++) w[s] = 0u;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        signed char dg[kSlices];
        rows_digits(v[u][d] * inv, dg);
#pragma unroll
        for (int s = 0; s < kSlices; s++) w[s] |= (uint32_t)(unsigned char)dg[s] << (8 * u);
      }
      const size_t base = ((size_t)tile * ksteps + kk) * kSlices * kABlock + rows_blk_off(r, k0 % kKStep);
#pragma unroll
      for (int s = 0; s < kSlices; s++) *(uint32_t *)(A + base + (size_t)s * kABlock) = w[s];
    }
  }
}

// ------------------------------------------------------------------------
// tcgen05 helpers (PTX ISA 8.6+, sm_100a)
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major, no swizzle: start address,
// leading-dimension byte offset (the two 16-byte K halves), stride byte
// offset (8-row groups), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::i8: D s32, A and B signed 8-bit, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kNTile >> 3) << 17) |
                              ((uint32_t)(kTileRows >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescI8), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
               : "memory");
}

// Bounded wait on an mbarrier phase: false after ~0.5 s (2^30 cycles).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > (1ll << 30)) return false;
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *v)
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

// Bounded wait that also gives up once *abort is set (another thread of the
// CTA gave up first): false then, or after ~0.5 s (2^30 cycles).
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t mbar, uint32_t parity, const volatile int *abort)
{
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*abort || clock64() - t0 > (1ll << 30)) return false;
  }
}

// ------------------------------------------------------------------------
// k_rows_mma: one CTA per (tile, orbital tile), the orbital tiles of a tile
// adjacent in the 1-D grid (they read the same A blocks, once from HBM and
// then from L2), kRowsThreads threads.  A: [tile][kstep][slice] blocks of
// kABlock bytes; B: [orbital tile][kstep][slice] blocks of kBBlock bytes (the
// spin's MO coefficients, digits made at set-up); rscale [rows][ksteps]
// (one walker's scales contiguous for the prep kernel's stores), cscale
// [orbital tiles][ksteps][kNTile]: every
// 32-function block of K has its own power-of-two scale on both sides, so
// the digits keep 56 bits relative to the block's largest values and the
// rows carry the error of an FP64 dot product of 32-term blocks.  rows
// [nrows][n] FP64 with nrows = 5 x walkers.  err: set to 1 when a wait gave
// up (the rows are then not written).
//
// Per K step, thread 0 issues the kSlices (kSlices + 1) / 2 digit-pair MMAs
// into one of two TMEM buffers (the K step's parity) and commits them; the
// eight warps drain the other buffer meanwhile (warps w and w + 4 read TMEM
// lanes 32 (w mod 4) .. + 31, columns 16 (w / 4) .. + 15 of every
// accumulator): the eight int32 accumulators
// of a K step are below 2^20 in magnitude (32 products of digits <= 2^6 in
// magnitude, at most 8 pairs), so neighbouring accumulators combine exactly
// in int32 (a_t 2^7 + a_{t+1} < 2^28) and four exact FP64 conversions give
// the K step's scaled sum, which is added to the FP64 result in registers.
__global__ void __launch_bounds__(kRowsThreads, 1) k_rows_mma(const signed char *__restrict__ A,
                                                              const signed char *__restrict__ B,
                                                              const double *__restrict__ rscale,
                                                              const double *__restrict__ cscale, int n, int ntiles,
                                                              int ksteps, int num, const int *d_num,
                                                              double *__restrict__ rows, int *err)
{
  static_assert(kSlices == 8, "the drain combines accumulators in four pairs");
  extern __shared__ __align__(1024) unsigned char rsm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nw = d_num ? *d_num : num;
  const int tile = blockIdx.x / ntiles, ntile = blockIdx.x - tile * ntiles;
  if (tile * kTileWalkers >= nw) return;  // whole CTA: before any TMEM or barrier use
  unsigned char *stage0 = rsm;
  // full[s]: the stage's operands landed (bulk copies, transaction bytes);
  // empty[s]: the MMAs that read the stage completed (tcgen05.commit);
  // done[b]: the MMAs of TMEM buffer b completed (tcgen05.commit);
  // drained[b]: the kRowsThreads threads read buffer b (one arrival each)
  uint64_t *full = (uint64_t *)(rsm + kRowsStages * kRowsStageBytes);
  uint64_t *empty = full + kRowsStages;
  uint64_t *done = empty + kRowsStages;
  uint64_t *drained = done + 2;
  uint32_t *tslot = (uint32_t *)(drained + 2);
  volatile int *s_abort = (volatile int *)(tslot + 1);
  int *s_last = (int *)(tslot + 2);  // last committed K step (thread 0)
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(kRowsTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < kRowsStages; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(full + s)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(empty + s)));
    }
    for (int b = 0; b < 2; b++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(done + b)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(drained + b)), "r"(kRowsThreads));
    }
    *s_abort = 0;
    *s_last = -1;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  const signed char *Ag = A + (size_t)tile * ksteps * kSlices * kABlock;
  const signed char *Bg = B + (size_t)ntile * ksteps * kSlices * kBBlock;
  // one thread streams the K steps: the digit planes of a K step are
  // contiguous in global memory (kSlices x kABlock of A, kSlices x kBBlock of
  // B), so two bulk copies fill a stage; kRowsStages - 1 steps are in flight
  // while the tensor cores work on the current one
  auto load = [&](int kk) {
    const int st = kk % kRowsStages;
    const uint32_t fb = smem_u32(full + st), dst = smem_u32(stage0 + st * kRowsStageBytes);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"((uint32_t)kRowsStageBytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(Ag + (size_t)kk * kSlices * kABlock), "r"((uint32_t)(kSlices * kABlock)), "r"(fb)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     dst + kSlices * kABlock),
                 "l"(Bg + (size_t)kk * kSlices * kBBlock), "r"((uint32_t)(kSlices * kBBlock)), "r"(fb)
                 : "memory");
  };
  int loaded = 0;  // thread 0 only
  if (tid == 0)
    for (; loaded < kRowsStages && loaded < ksteps; loaded++) load(loaded);

  // the FP64 result of this thread's row (TMEM lane) and its half of the
  // CTA's orbitals
  const int quarter = warp & 3, half = warp >> 2;
  const int r = 32 * quarter + lane;
  const int row = tile * 5 * kTileWalkers + r;
  const bool live = r < 5 * kTileWalkers && row < 5 * nw;
  double out[16];
#pragma unroll
  for (int q = 0; q < 16; q++) out[q] = 0.0;
  const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(16 * half);

  // drain K step kk from buffer kk & 1; false when a wait gave up
  auto drain = [&](int kk) -> bool {
    const int b = kk & 1;
    // the scales first: their loads overlap the wait for the MMAs
    const double rs = live ? rscale[(size_t)row * ksteps + kk] : 0.0;
    const double *csp = cscale + ((size_t)ntile * ksteps + kk) * kNTile + 16 * half;
    double cs[16];
#pragma unroll
    for (int q = 0; q < 16; q++) cs[q] = csp[q];
    // warp-uniform: tcgen05.ld is .sync.aligned
    if (!__all_sync(0xFFFFFFFFu, mbar_wait_or_abort(smem_u32(done + b), (uint32_t)((kk >> 1) & 1), s_abort)))
      return false;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    double part[16];
#pragma unroll
    for (int q = 0; q < 16; q++) part[q] = 0.0;
    // two pairs of accumulators per wait: pair p holds weights
    // 2^-(12 + 14 p) (accumulator 2p) and 2^-(19 + 14 p) (accumulator
    // 2p + 1), so a_2p 2^7 + a_2p+1 (below 2^28) carries 2^-(19 + 14 p); it
    // becomes a double exactly as (2^52 + 2^31 + v) - (2^52 + 2^31), the
    // first term assembled from its bits (one FP64 add, no conversion)
#pragma unroll
    for (int pp = 0; pp < kSlices / 2; pp += 2) {
      uint32_t v[4][16];
#pragma unroll
      for (int u = 0; u < 4; u++) tmem_ld16(lane_base + (uint32_t)(b * kAccCols + (2 * pp + u) * kNTile), v[u]);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const double w = ldexp(1.0, -19 - 14 * (pp + u));
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const int c = (int)v[2 * u][q] * 128 + (int)v[2 * u + 1][q];
          const double x = __hiloint2double(0x43300000, c ^ (int)0x80000000) - 4503601774854144.0;
          part[q] = fma(x, w, part[q]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 16; q++) out[q] = fma(part[q], rs * cs[q], out[q]);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(drained + b)) : "memory");
    return true;
  };

  bool ok = true;
  for (int kk = 0; kk < ksteps && ok; kk++) {
    if (tid == 0 && !*s_abort) {
      const int st = kk % kRowsStages, b = kk & 1;
      bool w = mbar_wait_or_abort(smem_u32(full + st), (uint32_t)((kk / kRowsStages) & 1), s_abort);
      // the buffer's previous K step (kk - 2) has been read by every thread
      if (w && kk >= 2) w = mbar_wait_or_abort(smem_u32(drained + b), (uint32_t)(((kk - 2) >> 1) & 1), s_abort);
      if (w) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t a0 = smem_u32(stage0 + st * kRowsStageBytes), b0 = a0 + kSlices * kABlock;
#pragma unroll
        for (int i = 0; i < kSlices; i++) {
#pragma unroll
          for (int j = 0; j + i < kSlices; j++) {
            const uint64_t ad = umma_desc(a0 + i * kABlock, 128, 256);
            const uint64_t bd = umma_desc(b0 + j * kBBlock, 128, 256);
            // the first pair of accumulator t = i + j in this K step is (0, t)
            mma_i8(tmem + (uint32_t)(b * kAccCols + (i + j) * kNTile), ad, bd, i > 0 ? 1u : 0u);
          }
        }
        mma_commit(smem_u32(empty + st));
        mma_commit(smem_u32(done + b));
        *s_last = kk;
        // refill the stage the previous K step used, once its MMAs are done
        if (kk >= 1 && loaded < ksteps) {
          const int sp = (kk - 1) % kRowsStages;
          w = mbar_wait_or_abort(smem_u32(empty + sp), (uint32_t)(((kk - 1) / kRowsStages) & 1), s_abort);
          if (w) load(loaded++);
        }
      }
      if (!w) *s_abort = 1;
    }
    __syncwarp();
    if (kk >= 1) ok = drain(kk - 1);
    if (!ok) *s_abort = 1;
  }
  if (ok && ksteps > 0) ok = drain(ksteps - 1);
  if (!ok) *s_abort = 1;
  __syncthreads();
  const bool okall = !*s_abort;
  if (tid == 0) {
    // leave no copy or MMA in flight: the copies issued but not consumed
    // land (bounded waits), then the last commit's phase covers every MMA
    const int last = *s_last;
    for (int l = last + 1; l < loaded; l++)
      mbar_wait(smem_u32(full + l % kRowsStages), (uint32_t)((l / kRowsStages) & 1));
    if (last >= 0) mbar_wait(smem_u32(done + (last & 1)), (uint32_t)((last >> 1) & 1));
    if (!okall) atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kRowsTmemCols));
  if (okall && live) {
    const int o0 = ntile * kNTile + 16 * half;
#pragma unroll
    for (int q = 0; q < 16; q++)
      if (o0 + q < n) rows[(size_t)row * n + o0 + q] = out[q];
  }
}

// ------------------------------------------------------------------------
// BF16 tensor-core rows with FP32 accumulation (QMCB_PREC_BF16_TC,
// QMCB_PREC_BF16X3_TC): the same batched GEMM, rows[5 x walker][o] =
// sum_k chi[r][k] C[o][k], with BF16 operands and FP32 accumulation in TMEM
// over all of K.  QMCB_PREC_BF16_TC rounds each operand value to BF16 (8
// significant bits) once; QMCB_PREC_BF16X3_TC splits it as x = hi + lo
// (hi = x rounded to 8 bits, lo = x - hi rounded to 8 bits, so hi + lo
// keeps 16 bits) and accumulates the three products hi.hi + hi.lo + lo.hi
// (the split-precision compensated product; lo.lo, below 2^-16 of the
// product, is left out).  Floating-point operands need no block scales, so
// the accumulator is read once per tile, after the last K step.
//
//   k_rows_prep_bf   one warp per walker: proposal and basis values as
//                    k_rows_prep, written as kPlanes BF16 planes (hi, lo)
//                    in the K-major core-matrix layout, 16 functions (32
//                    bytes) per K step
//   k_rows_mma_bf    one CTA of 128 threads per tile of 25 walkers and 32
//                    orbitals: kPlanes == 1 one, kPlanes == 2 three
//                    tcgen05.mma kind::f16 (BF16 x BF16 -> FP32, M = 128,
//                    N = 32, K = 16) per K step into one 32-column TMEM
//                    accumulator, operands staged by bulk copies in
//                    kBfStages stages; writes rows[walker][5][n]
constexpr int kBfKStep = 16;  // BF16 K of one MMA (32 bytes per row)
constexpr int kBfStages = 6;
constexpr int kBfThreads = 128;  // one warp per TMEM lane quarter
constexpr uint32_t kBfTmemCols = 32;
__host__ __device__ inline int bf_stage_bytes(int planes) { return planes * (kABlock + kBBlock); }
__host__ __device__ inline int bf_smem_bytes(int planes) { return kBfStages * bf_stage_bytes(planes) + 256; }
// Instruction descriptor of kind::f16: D F32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kNTile >> 3) << 17) |
                                ((uint32_t)(kTileRows >> 4) << 24);

// x rounded to 8 significant bits (round to nearest by Veltkamp's split with
// the factor 2^45 + 1; ties are not necessarily even), flushed to zero below
// 2^-126 (BF16 normal range); the result is exactly a BF16 value.
__host__ __device__ inline double bf16_round(double x)
{
  // the product rounded on its own (never fused with the subtraction)
#ifdef __CUDA_ARCH__
  const double c = __dmul_rn(x, 35184372088833.0);  // 2^45 + 1
#else
  const double c = x * 35184372088833.0;
#endif
  const double h = c - (c - x);
  return fabs(h) < 1.1754943508222875e-38 ? 0.0 : h;
}

// Bits of a value that bf16_round produced (its FP32 form's upper half).
__host__ __device__ inline uint32_t bf16_bits(double v)
{
  const float f = (float)v;  // exact: 8 significant bits in FP32 range
#ifdef __CUDA_ARCH__
  return __float_as_uint(f) >> 16;
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u >> 16;
#endif
}

template <bool kMetropolis, bool kExtras, int kPlanes>
__global__ void __launch_bounds__(128) k_rows_prep_bf(DevSys S, Layout L, RunCfg cfg, const double *state,
                                                       const int *slots, int num, const int *d_num,
                                                       const double *R_in, MoveArgs mv, int ksteps,
                                                       unsigned char *A)
{
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = lane_id();
  const int nw = d_num ? *d_num : num;
  const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (wi >= nw) return;
  const int N = S.N, K = S.K, e = mv.e;
  double *sm = smem + (size_t)warp * rows_prep_doubles(N, K, S.nslot);
  double *sR = sm, *smg = sm + even(3 * N), *ex = sm;
  const int slot = slots ? slots[wi] : wi;
  const double *blk = state + (size_t)slot * L.stride;
  for (int t = lane; t < 3 * N; t += 32) {
    sR[t] = blk[L.R + t];
    smg[t] = blk[L.mgrad + t];
  }
  __syncwarp();
  const double ro[3] = {sR[3 * e], sR[3 * e + 1], sR[3 * e + 2]};
  double rn[3], g_fwd, u_acc;
  propose_move<kMetropolis, kExtras>(S, cfg, slot, mv.step, e, N, sR, ro, smg, R_in, wi, rn, g_fwd, u_acc, mv.rin_moved);
  __syncwarp();  // the slots overwrite the staged arrays
  basis_slot_exps_warp(S, rn, ex);
  __syncwarp();
  const int row0 = 5 * wi, tile = row0 / (5 * kTileWalkers), r0 = row0 - tile * 5 * kTileWalkers;
  for (int k0 = 4 * lane; k0 < ksteps * kBfKStep; k0 += 128) {
    double v[4][5];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (k0 + u < K) {
        basis_function_rows(S, rn, k0 + u, ex, v[u]);
      } else {
#pragma unroll
        for (int d = 0; d < 5; d++) v[u][d] = 0.0;
      }
    }
    // four consecutive functions: 8 bytes of a row in one 16-byte core-matrix row
    const int kk = k0 / kBfKStep, kb = 2 * (k0 % kBfKStep);
#pragma unroll
    for (int d = 0; d < 5; d++) {
      uint32_t hb[4], lb[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const double h = bf16_round(v[u][d]);
        hb[u] = bf16_bits(h);
        lb[u] = kPlanes > 1 ? bf16_bits(bf16_round(v[u][d] - h)) : 0u;
      }
      const size_t base = ((size_t)tile * ksteps + kk) * kPlanes * kABlock + rows_blk_off(r0 + d, kb);
      *(uint2 *)(A + base) = make_uint2(hb[0] | (hb[1] << 16), hb[2] | (hb[3] << 16));
      if (kPlanes > 1) *(uint2 *)(A + base + kABlock) = make_uint2(lb[0] | (lb[1] << 16), lb[2] | (lb[3] << 16));
    }
  }
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescBf16), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *v)
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// A: [tile][K step][plane] blocks of kABlock bytes (BF16, 16 functions per
// K step); B: [orbital tile][K step][2 planes] blocks of kBBlock bytes (hi,
// lo of the spin's MO coefficients, made at set-up; kPlanes == 1 reads the
// hi plane).  Thread 0 streams the stages (bulk copies, one mbarrier per
// stage) and issues the MMAs; the four warps read the accumulator once at
// the end.  err: set to 1 when a wait gave up (the rows are then not
// written).  Every wait is bounded; the kernel leaves no copy or MMA in
// flight and frees its TMEM on every path.
template <int kPlanes>
__global__ void __launch_bounds__(kBfThreads) k_rows_mma_bf(const unsigned char *__restrict__ A,
                                                           const unsigned char *__restrict__ B, int n, int ntiles,
                                                           int ksteps, int num, const int *d_num,
                                                           double *__restrict__ rows, int *err)
{
  extern __shared__ __align__(1024) unsigned char rsm[];
  constexpr int kStage = kPlanes * (kABlock + kBBlock);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nw = d_num ? *d_num : num;
  const int tile = blockIdx.x / ntiles, ntile = blockIdx.x - tile * ntiles;
  if (tile * kTileWalkers >= nw) return;  // whole CTA: before any TMEM or barrier use
  uint64_t *full = (uint64_t *)(rsm + kBfStages * kStage);
  uint64_t *empty = full + kBfStages;
  uint64_t *done = empty + kBfStages;
  uint32_t *tslot = (uint32_t *)(done + 1);
  volatile int *s_abort = (volatile int *)(tslot + 1);
  int *s_last = (int *)(tslot + 2);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(kBfTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < kBfStages; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(full + s)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(empty + s)));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(done)));
    *s_abort = 0;
    *s_last = -1;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  const unsigned char *Ag = A + (size_t)tile * ksteps * kPlanes * kABlock;
  const unsigned char *Bg = B + (size_t)ntile * ksteps * 2 * kBBlock;
  auto load = [&](int kk) {
    const int st = kk % kBfStages;
    const uint32_t fb = smem_u32(full + st), dst = smem_u32(rsm + st * kStage);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"((uint32_t)kStage)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(Ag + (size_t)kk * kPlanes * kABlock), "r"((uint32_t)(kPlanes * kABlock)), "r"(fb)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     dst + kPlanes * kABlock),
                 "l"(Bg + (size_t)kk * 2 * kBBlock), "r"((uint32_t)(kPlanes * kBBlock)), "r"(fb)
                 : "memory");
  };
  bool committed = false;  // thread 0: the final commit onto `done` was issued
  if (tid == 0) {
    int loaded = 0;
    for (; loaded < kBfStages && loaded < ksteps; loaded++) load(loaded);
    bool w = true;
    for (int kk = 0; kk < ksteps && w; kk++) {
      const int st = kk % kBfStages;
      w = mbar_wait(smem_u32(full + st), (uint32_t)((kk / kBfStages) & 1));
      if (!w) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a0 = smem_u32(rsm + st * kStage), b0 = a0 + kPlanes * kABlock;
      const uint64_t ah = umma_desc(a0, 128, 256), bh = umma_desc(b0, 128, 256);
      mma_bf16(tmem, ah, bh, kk > 0 ? 1u : 0u);
      if (kPlanes > 1) {
        const uint64_t al = umma_desc(a0 + kABlock, 128, 256), bl = umma_desc(b0 + kBBlock, 128, 256);
        mma_bf16(tmem, ah, bl, 1u);
        mma_bf16(tmem, al, bh, 1u);
      }
      mma_commit(smem_u32(empty + st));
      *s_last = kk;
      // refill the stage the previous K step used once its MMAs have read
      // it (this step's MMAs are queued meanwhile)
      if (kk >= 1 && loaded < ksteps) {
        const int sp = (kk - 1) % kBfStages;
        w = mbar_wait(smem_u32(empty + sp), (uint32_t)(((kk - 1) / kBfStages) & 1));
        if (w) load(loaded++);
      }
    }
    if (w) {
      mma_commit(smem_u32(done));
      committed = true;
    } else {
      *s_abort = 1;
      // leave no copy or MMA in flight: the copies issued but not consumed
      // land, then the last step's MMAs complete (bounded waits)
      const int last = *s_last;
      for (int l = last + 1; l < loaded; l++)
        mbar_wait(smem_u32(full + l % kBfStages), (uint32_t)((l / kBfStages) & 1));
      if (last >= 0) mbar_wait(smem_u32(empty + last % kBfStages), (uint32_t)((last / kBfStages) & 1));
    }
  }
  __syncwarp();
  __syncthreads();
  bool ok = !*s_abort;
  if (ok) ok = __all_sync(0xFFFFFFFFu, mbar_wait_or_abort(smem_u32(done), 0u, s_abort));
  if (!ok) *s_abort = 1;
  float acc[32];
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    uint32_t v[32];
    tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16), v);
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int q = 0; q < 32; q++) acc[q] = __uint_as_float(v[q]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  const bool okall = !*s_abort;
  if (tid == 0 && !okall) {
    // a warp gave up on `done`: the MMAs must still finish before the TMEM is freed
    if (committed) mbar_wait(smem_u32(done), 0u);
    atomicExch(err, 1);
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kBfTmemCols));
  const int r = 32 * warp + lane;
  const int row = tile * 5 * kTileWalkers + r;
  if (okall && r < 5 * kTileWalkers && row < 5 * nw) {
    const int o0 = ntile * kNTile;
#pragma unroll
    for (int q = 0; q < 32; q++)
      if (o0 + q < n) rows[(size_t)row * n + o0 + q] = (double)acc[q];
  }
}

}  // namespace qmcb
