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
// IJHPCA 2024): every row of chi and every orbital of C is scaled by a power
// of two to |x| < 1 and cut into kSlices signed 7-bit digits,
//   x = scale * sum_s d_s 2^-(6 + 7 s),  |d_s| <= 64,
// the digit products sum_k a_i[r][k] b_j[k][o] are exact in int32
// (|a b| <= 2^12, K <= 2^19 / kSlices), and the pairs with i + j = t share
// one TMEM accumulator (weight 2^-(12 + 7 t)).  The pairs with i + j < kSlices
// keep 56 bits of every product relative to the row's largest basis value
// and the orbital's largest coefficient: the rows carry FP64-level error in
// the normwise sense (an FP64 dot product's error is relative to the sum of
// its terms, which is smaller for elements far below their row's largest),
// so the per-move Slater updates downstream stay in the FP64 regime (Slater
// matrices of random 50 x 50 orbitals reach condition numbers of 1e6, which
// amplify any FP32-class row error to 1e-1 Ha in the local energy).
//
//   k_rows_prep  one warp per walker: the move's proposal (the same draws as
//                the move kernel, which recomputes it), the basis values at
//                the proposed position, their per-row scales and int8 digits
//                in the tensor-core operand layout
//   k_rows_mma   one CTA per tile of 25 walkers (125 rows) and 64 orbitals:
//                int8 x int8 -> int32 tcgen05.mma (kind::i8, M = 128, N = 64,
//                K = 32 per instruction) over kSlices (kSlices + 1) / 2 digit
//                pairs per K step, operands staged in shared memory by
//                bulk copies (the TMA engine, 3 stages, one thread), accumulators
//                in TMEM, FP64 recombination in the epilogue; writes
//                rows[walker][5][n]
// The move kernel then reads the rows instead of evaluating the basis and
// contracting (MoveArgs::rows).
#pragma once

#include "kernels.cuh"

namespace qmcb {

constexpr int kSlices = 8;       // int8 digits per operand value
constexpr int kTileRows = 128;   // MMA M: TMEM lanes
constexpr int kTileWalkers = 25; // walkers per tile: rows 0 .. 124 used
constexpr int kNTile = 64;       // MMA N: orbitals per CTA
constexpr int kKStep = 32;       // int8 K of one MMA (bytes)
constexpr int kABlock = kTileRows * kKStep;  // one digit plane of one K step of an A tile
constexpr int kBBlock = kNTile * kKStep;     // the same for B
constexpr int kRowsStages = 3;
constexpr int kRowsStageBytes = kSlices * (kABlock + kBBlock);
constexpr int kRowsSmem = kRowsStages * kRowsStageBytes + 1024;  // + barriers; > 113 KB: one CTA per SM
static_assert(kRowsStageBytes % 16 == 0 && kABlock % 16 == 0, "bulk copies move multiples of 16 bytes");
constexpr uint32_t kRowsTmemCols = 512;  // kSlices accumulators of kNTile int32 columns (all of TMEM)
static_assert(kSlices * kNTile <= (int)kRowsTmemCols, "accumulators exceed the TMEM allocation");

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
// |d_s| <= 64.  Integer arithmetic after the one conversion.
__host__ __device__ inline void rows_digits(double x, signed char *d)
{
  static_assert(7 * kSlices - 1 <= 62, "digits exceed a 64-bit fixed-point value");
  long long q = llrint(ldexp(x, 7 * kSlices - 1));
  for (int s = 0; s < kSlices; s++) {
    const int w = 7 * (kSlices - 1 - s);
    const long long ds = w > 0 ? (q + (1ll << (w - 1))) >> w : q;  // arithmetic shift: floor
    d[s] = (signed char)ds;
    q -= ds << w;
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
// then, in the same space, chi [5][K]; the exponential slots after both.
__host__ __device__ inline int rows_prep_doubles(int N, int K, int nslot)
{
  return max(2 * even(3 * N), even(5 * K)) + even(nslot);
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
  double *sR = sm, *smg = sm + even(3 * N), *chi = sm, *ex = sm + max(2 * even(3 * N), even(5 * K));
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
  __syncwarp();  // chi overwrites the staged arrays
  basis_slots_warp(S, rn, chi, K, ex);
  __syncwarp();
  // rows 5 wi .. 5 wi + 4 of the GEMM: tile, row in tile
  for (int d = 0; d < 5; d++) {
    const int row = 5 * wi + d, tile = row / (5 * kTileWalkers), r = row - tile * 5 * kTileWalkers;
    double m = 0.0;
    for (int k = lane; k < K; k += 32) m = fmax(m, fabs(chi[d * K + k]));
    const double scale = rows_scale(warp_max(m)), inv = 1.0 / scale;  // exact: a power of two
    if (lane == 0) rscale[row] = scale;
    // four consecutive k per lane: one 4-byte store per digit plane
    for (int k0 = 4 * lane; k0 < ksteps * kKStep; k0 += 128) {
      uint32_t w[kSlices];
#pragma unroll
      for (int s = 0; s < kSlices; s++) w[s] = 0u;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int k = k0 + u;
        signed char dg[kSlices];
        rows_digits(k < K ? chi[d * K + k] * inv : 0.0, dg);
#pragma unroll
        for (int s = 0; s < kSlices; s++) w[s] |= (uint32_t)(unsigned char)dg[s] << (8 * u);
      }
      const int kk = k0 / kKStep;
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

// ------------------------------------------------------------------------
// k_rows_mma: grid (tiles, orbital tiles), 128 threads.  A: [tile][kstep]
// [slice] blocks of kABlock bytes; B: [orbital tile][kstep][slice] blocks of
// kBBlock bytes (the spin's MO coefficients, digits made at set-up);
// rscale [rows], cscale [orbital tiles x kNTile]; rows [nrows][n] FP64 with
// nrows = 5 x walkers.  err: set to 1 when a wait gave up (the rows are then
// not written).
__global__ void __launch_bounds__(128, 1) k_rows_mma(const signed char *__restrict__ A,
                                                     const signed char *__restrict__ B,
                                                     const double *__restrict__ rscale,
                                                     const double *__restrict__ cscale, int n, int ksteps,
                                                     int num, const int *d_num, double *__restrict__ rows,
                                                     int *err)
{
  extern __shared__ __align__(1024) unsigned char rsm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nw = d_num ? *d_num : num;
  const int tile = blockIdx.x, ntile = blockIdx.y;
  if (tile * kTileWalkers >= nw) return;  // whole CTA: before any TMEM or barrier use
  unsigned char *stage0 = rsm;
  // full[s]: the stage's operands landed (bulk copies, transaction bytes);
  // empty[s]: the MMAs that read the stage completed (tcgen05.commit)
  uint64_t *full = (uint64_t *)(rsm + kRowsStages * kRowsStageBytes);
  uint64_t *empty = full + kRowsStages;
  uint32_t *tslot = (uint32_t *)(empty + kRowsStages);
  int *s_status = (int *)(tslot + 1);  // [0] ok, [1] last committed K step
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
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  const signed char *Ag = A + (size_t)tile * ksteps * kSlices * kABlock;
  const signed char *Bg = B + (size_t)ntile * ksteps * kSlices * kBBlock;
  if (tid == 0) {
    // one thread streams the K steps: the digit planes of a K step are
    // contiguous in global memory (kSlices x kABlock of A, kSlices x kBBlock
    // of B), so two bulk copies fill a stage; kRowsStages - 1 steps are in
    // flight while the tensor cores work on the current one
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
    int loaded = 0, committed = -1;
    bool ok = true;
    for (; loaded < kRowsStages && loaded < ksteps; loaded++) load(loaded);
    for (int kk = 0; kk < ksteps; kk++) {
      const int st = kk % kRowsStages;
      ok = mbar_wait(smem_u32(full + st), (uint32_t)((kk / kRowsStages) & 1));
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a0 = smem_u32(stage0 + st * kRowsStageBytes), b0 = a0 + kSlices * kABlock;
#pragma unroll
      for (int i = 0; i < kSlices; i++) {
#pragma unroll
        for (int j = 0; j + i < kSlices; j++) {
          const uint64_t ad = umma_desc(a0 + i * kABlock, 128, 256);
          const uint64_t bd = umma_desc(b0 + j * kBBlock, 128, 256);
          mma_i8(tmem + (uint32_t)((i + j) * kNTile), ad, bd, (kk > 0 || i > 0) ? 1u : 0u);
        }
      }
      mma_commit(smem_u32(empty + st));
      committed = kk;
      // refill the stage the previous K step used, once its MMAs are done
      if (kk >= 1 && loaded < ksteps) {
        const int sp = (kk - 1) % kRowsStages;
        ok = mbar_wait(smem_u32(empty + sp), (uint32_t)(((kk - 1) / kRowsStages) & 1));
        if (!ok) break;
        load(loaded++);
      }
    }
    if (!ok) {
      // a wait gave up: let the copies already issued land (bounded) before
      // the shared memory is left
      for (int l = committed + 1; l < loaded; l++) mbar_wait(smem_u32(full + l % kRowsStages), (uint32_t)((l / kRowsStages) & 1));
    }
    s_status[0] = ok ? 1 : 0;
    s_status[1] = committed;
  }
  __syncthreads();
  const bool ok = s_status[0] != 0;
  const int committed = s_status[1];
  // every MMA of this CTA is done once the last commit's phase completes
  // (waited for after a failed wait too, so that no MMA is in flight when
  // the TMEM is released)
  bool done = true;
  if (committed >= 0)
    done = mbar_wait(smem_u32(empty + committed % kRowsStages), (uint32_t)((committed / kRowsStages) & 1));
  const int okall = __syncthreads_and((ok && done && committed == ksteps - 1) ? 1 : 0);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (okall) {
    // epilogue: warp w holds rows 32 w .. 32 w + 31 (TMEM lanes)
    const int r = 32 * warp + lane;
    const int row = tile * 5 * kTileWalkers + r;
    const bool live = r < 5 * kTileWalkers && row < 5 * nw;
    const double rs = live ? rscale[row] : 0.0;
    for (int c = 0; c < kNTile / 16; c++) {
      double acc[16];
#pragma unroll
      for (int q = 0; q < 16; q++) acc[q] = 0.0;
      double w = 1.0 / 4096.0;  // 2^-(12 + 7 t)
#pragma unroll
      for (int t = 0; t < kSlices; t++) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(t * kNTile + 16 * c), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int q = 0; q < 16; q++) acc[q] = fma((double)(int)v[q], w, acc[q]);
        w *= 1.0 / 128.0;
      }
      if (live) {
        const int o0 = ntile * kNTile + 16 * c;
#pragma unroll
        for (int q = 0; q < 16; q++)
          if (o0 + q < n) rows[(size_t)row * n + o0 + q] = acc[q] * (rs * cscale[o0 + q]);
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kRowsTmemCols));
}

}  // namespace qmcb
