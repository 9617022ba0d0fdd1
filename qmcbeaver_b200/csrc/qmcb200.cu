// qmcb200.cu -- C ABI of the B200 Slater-Jastrow walker library.
//
// Host side of include/qmcb200.h: device tables for the molecular system,
// the per-walker state blocks, the live-walker list used by DMC branching,
// and the launch sequence of one Monte Carlo step.  Kernels are in
// kernels.cuh.  No CPU fallback: every entry point fails with QMCB_E_CUDA
// when no CUDA device is usable.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/qmcb200.h"
#include "cusp_fit.h"
#include "kernels.cuh"
#include "kernels_md.cuh"
#include "kernels_group.cuh"
#include "kernels_rows.cuh"

using namespace qmcb;

// Mixed precision: FP32 basis values, orbital rows and contraction; the
// inverse and its Sherman-Morrison update in MIXED_TI.
#ifndef MIXED_TI
#define MIXED_TI double
#endif

namespace {

const int kMaxWarpsPerBlock = 4;
const int kStagedInverseMax = 16;  // largest spin whose inverse the move kernel stages in shared memory

std::string g_create_error;

}  // namespace

struct qmcb_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  DevSys sys{};
  Layout lay{};
  int N = 0, K = 0, nmax = 0, max_walkers = 0;
  qmcb_run_params params{};
  // device buffers
  double4 *d_nuc = nullptr;
  int4 *d_bf = nullptr;
  double2 *d_prim = nullptr;
  double *d_ct[2] = {nullptr, nullptr};
  float *d_ctf[2] = {nullptr, nullptr};
  // batched orbital rows on the tensor cores (QMCB_PREC_INT8_SLICES), set up
  // on first use: the transposed MO coefficients [K][n_s] kept for the digit
  // tables, A digits of the step's basis rows, B digits per spin, row and
  // orbital scales, the rows [walker][5][n]
  std::vector<double> ct_host[2];
  signed char *d_rows_A = nullptr, *d_rows_B[2] = {nullptr, nullptr};
  double *d_rows_rs = nullptr, *d_rows_cs[2] = {nullptr, nullptr}, *d_rows_out = nullptr;
  int rows_ksteps = 0, wpb_rows = 1, wpb_prep = 1;
  // the BF16 forms (QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC): A planes of the
  // step's basis rows (room for two), hi / lo planes of the MO coefficients
  unsigned char *d_bf_A = nullptr, *d_bf_B[2] = {nullptr, nullptr};
  int bf_ksteps = 0;
  int rows_n = 0, rows_num = 0;  // the last tensor-core rows launch: orbitals per row, list capacity
  size_t smem_rows = 0, smem_prep = 0;
  Layout lay_rows{};  // move-kernel scratch without the basis rows
  double *d_pade = nullptr;
  int2 *d_pade_len = nullptr;
  double2 *d_pade_ab = nullptr;
  int *d_ctype = nullptr;
  double4 *d_cparam = nullptr;
  int4 *d_shell = nullptr;
  int2 *d_fn = nullptr;
  int2 *d_xsl = nullptr;
  int4 *d_fq = nullptr;
  double *d_pexp = nullptr, *d_pcoef = nullptr;
  int *d_en[2] = {nullptr, nullptr};
  int *d_docc[2] = {nullptr, nullptr};
  int *d_dswap[2] = {nullptr, nullptr};
  int *d_cns = nullptr;
  double *d_csexp = nullptr, *d_cscoef[2] = {nullptr, nullptr}, *d_cpar[2] = {nullptr, nullptr};
  double *d_crmax[2] = {nullptr, nullptr};
  int4 *d_tbi = nullptr;
  double *d_tbL = nullptr, *d_tbc = nullptr;
  int *d_tbp = nullptr;
  double *d_ci = nullptr;
  bool md = false;  // several determinants: the k_*_md kernels
  bool extras = false;  // cusp replacement or three-body terms: the k_move<..., true> instantiation
  bool ginv = false;    // large spins: inverses in HBM, double-buffered (k_move<..., kGInv = true>)
  double *d_state = nullptr;
  int *d_live = nullptr, *d_live_tmp = nullptr, *d_free = nullptr, *d_ctl = nullptr;
  int2 *d_copies = nullptr;
  double *d_stats = nullptr;
  double *d_dump = nullptr;  // configuration records of one step (qmcb_run_step_configs), on first use
  EnergyCtl *d_ectl = nullptr;
  // staging for the host-pointer evaluate
  int *d_slots = nullptr;
  double *d_R = nullptr, *d_out = nullptr;
  unsigned char *d_status = nullptr;
  int n_live_host = 0;
  double target_weight = 0.0;
  size_t smem_move = 0, smem_full = 0, smem_refresh = 0;
  int wpb_move = 1, wpb_full = 1, wpb_refresh = 1;  // warps (walkers) per CTA of k_move / k_full / the refresh
  bool evaluated_once = false;
  int state_prec = -1;  // precision the stored walker state was written in
  // asynchronous step batches (qmcb_run_steps_async)
  // up to two batches in flight, each with its own pinned statistics copy
  double *h_stats = nullptr;  // pinned, [2][ST_COUNT]
  int *h_ctl = nullptr;       // pinned, [2][4]
  cudaEvent_t done_ev[2] = {nullptr, nullptr};
  int n_flight = 0;           // batches enqueued and not yet collected
  EnergyCtl *h_ectl = nullptr;  // pinned [4]: E_T / E_est uploads of qmcb_set_params
  cudaEvent_t ectl_ev[4] = {nullptr, nullptr, nullptr, nullptr};  // each slot's copy done
  int ectl_next = 0;
  int head = 0;               // slot of the oldest of them
  // kernel timing (qmcb_set_profiling)
  bool prof = false;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_kind;
  size_t prof_used = 0;
  double prof_ms[QMCB_KERNEL_COUNT] = {0};
  double prof_n[QMCB_KERNEL_COUNT] = {0};
  // slot allocator of the evaluate entry points (qmcb_alloc_slot / qmcb_free_slot)
  std::mutex slot_mu;
  std::vector<char> slot_used;
  std::vector<int> slot_free;
  std::string err;
};

// Event pair around one launch when profiling is on.
struct ProfScope {
  qmcb_handle *h;
  size_t idx;
  ProfScope(qmcb_handle *hh, int kind, cudaStream_t st, bool on = true) : h(hh), idx((size_t)-1)
  {
    if (!h->prof || !on) return;
    if (h->prof_used + 2 > h->prof_ev.size()) {
      size_t grow = std::max<size_t>(256, h->prof_ev.size());
      for (size_t i = 0; i < grow; i++) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        h->prof_ev.push_back(e);
      }
    }
    idx = h->prof_used;
    h->prof_used += 2;
    h->prof_kind.push_back(kind);
    cudaEventRecord(h->prof_ev[idx], st);
  }
  void end(cudaStream_t st)
  {
    if (idx != (size_t)-1) cudaEventRecord(h->prof_ev[idx + 1], st);
  }
};

// Folds the recorded event pairs into the totals (stream must be idle).
static void prof_collect(qmcb_handle *h)
{
  for (size_t i = 0; i + 1 < h->prof_used && i / 2 < h->prof_kind.size(); i += 2) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->prof_ev[i], h->prof_ev[i + 1]) == cudaSuccess) {
      int k = h->prof_kind[i / 2];
      h->prof_ms[k] += ms;
      h->prof_n[k] += 1.0;
    }
  }
  h->prof_used = 0;
  h->prof_kind.clear();
}

static int fail(qmcb_handle *h, int code, const std::string &msg)
{
  if (h)
    h->err = msg;
  else
    g_create_error = msg;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(h, QMCB_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));   \
  } while (0)

static RunCfg make_cfg(const qmcb_run_params &p)
{
  RunCfg c{};
  c.run_type = p.run_type;
  c.sampling = p.sampling;
  c.qf_mod = p.qf_modification;
  c.emod = p.energy_modification;
  c.reweighting = p.reweighting;
  c.old_walker_acceptance = p.old_walker_acceptance;
  c.qf_a = p.qf_equal_a;
  c.dt = p.dt;
  c.dt_eff = p.dt_effective;
  c.branching_threshold = p.branching_threshold;
  c.fusion_threshold = p.fusion_threshold;
  c.seed = p.seed;
  c.limit_branching = p.limit_branching;
  c.ecut = p.energy_cutoff;
  c.exact_gf = p.exact_single_electron_gf;
  c.dyn_dt = p.dynamic_time_step;
  c.deletion = p.walker_deletion;
  c.equil_steps = p.equilibration_steps;
  c.e_orig = p.energy_original != 0.0 ? p.energy_original : (p.energy_estimated != 0.0 ? p.energy_estimated : -1.0);
  c.rel_cutoff = p.rel_cutoff > 0 ? p.rel_cutoff : 1e300;
  return c;
}

static void default_params(qmcb_run_params *p)
{
  std::memset(p, 0, sizeof(*p));
  p->run_type = QMCB_VMC;
  p->sampling = QMCB_NO_IMPORTANCE_SAMPLING;
  p->qf_modification = QMCB_QF_NONE;
  p->qf_equal_a = 0.5;
  p->dt = 0.09;
  p->dt_effective = 0.09;
  p->energy_modification = QMCB_EMOD_NONE;
  p->reweighting = QMCB_RW_UMRIGAR93_PROBABILITY_WEIGHTED;
  p->branching_threshold = 2.0;
  p->fusion_threshold = 0.45;
  p->old_walker_acceptance = 50;
  p->refresh_interval = 0;
  p->precision = QMCB_PREC_FP64;
  p->seed = 12345;
  p->population_control = 1.0;
  p->target_walkers = 0;
  p->reweight_start_step = 100;
  p->energy_original = 0.0;
  p->rel_cutoff = 100.0;
  p->limit_branching = 1;
  p->energy_cutoff = QMCB_ECUT_NONE;
}

template <typename T>
static cudaError_t upload(T **d, const std::vector<T> &v)
{
  cudaError_t e = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(v.size(), 1));
  if (e != cudaSuccess) return e;
  if (!v.empty()) e = cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
  return e;
}

// ---------------------------------------------------------------------------
// Allocation-free branching pass over a caller's weight list.
//
// The working weights and the index lists live in these file-scope device
// arrays instead of memory the library would allocate; every GPU that loads
// the library holds them (768 KB) until the process exits.  All calls share
// them, so calls that overlap on the GPU race.
static __device__ __align__(256) double g_noalloc_weight[QMCB_NOALLOC_MAX_WALKERS];
static __device__ __align__(256) int g_noalloc_index[QMCB_NOALLOC_MAX_WALKERS];

// Same decisions as k_branch (nonunit-weight branching, fusion pairs in list
// order, random stream of a pair keyed by its first member's list index, the
// split test on the weight before fusion), on plain arrays: survivors keep
// their order, split copies are appended.  w_out / parent_out need room for
// 2 n entries.
__global__ void __launch_bounds__(1024) k_branch_list(const double *w_in, int n, double thr_split, double thr_fuse,
                                                      uint64_t seed, int step, double *w_work, int *idx,
                                                      double *w_out, int *parent_out, int *n_out)
{
  __shared__ int s_warp[32];
  __shared__ int s_tot;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // every working element read below is written here first in this call
  for (int i = tid; i < n; i += 1024) w_work[i] = w_in[i];
  __syncthreads();
  auto block_scan = [&](int flag, int &excl, int &total) {
    unsigned b = __ballot_sync(QMCB_FULL_MASK, flag);
    int pre = __popc(b & ((1u << lane) - 1));
    if (lane == 31) s_warp[wid] = pre + flag;
    __syncthreads();
    if (wid == 0) {
      int v = s_warp[lane], x = v;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(QMCB_FULL_MASK, x, o);
        if (lane >= o) x += y;
      }
      s_warp[lane] = x - v;
      if (lane == 31) s_tot = x;
    }
    __syncthreads();
    excl = s_warp[wid] + pre;
    total = s_tot;
    __syncthreads();
  };
  // fusion candidates in list order
  int nc = 0;
  for (int c0 = 0; c0 < n; c0 += 1024) {
    int i = c0 + tid;
    double w = i < n ? w_work[i] : 0.0;
    int is_c = (i < n && w <= thr_split && w >= 0.01 && w < thr_fuse) ? 1 : 0;
    int ex, tot;
    block_scan(is_c, ex, tot);
    if (is_c) idx[nc + ex] = i;
    nc += tot;
  }
  __syncthreads();
  for (int m = tid; 2 * m + 1 < nc; m += 1024) {
    int ia = idx[2 * m], ib = idx[2 * m + 1];
    double w1 = w_work[ia], w2 = w_work[ib], w3 = w1 + w2;
    double u[4];
    rng_uniform4(seed, (uint32_t)ia, (uint32_t)step, 7u, u);
    if (u[0] < w1 / w3) {
      w_work[ia] = w3;
      w_work[ib] = -1.0;
    } else {
      w_work[ib] = w3;
      w_work[ia] = -1.0;
    }
  }
  __syncthreads();
  // survivors in order
  int nk = 0;
  for (int c0 = 0; c0 < n; c0 += 1024) {
    int i = c0 + tid;
    int keep = (i < n && w_work[i] >= 0.01) ? 1 : 0;
    int ex, tot;
    block_scan(keep, ex, tot);
    if (keep) idx[nk + ex] = i;
    nk += tot;
  }
  __syncthreads();
  // splits appended after the survivors
  int ns = 0;
  for (int c0 = 0; c0 < nk; c0 += 1024) {
    int j = c0 + tid;
    int src = j < nk ? idx[j] : -1;
    double w = src >= 0 ? w_work[src] : 0.0;
    // w_in holds the weight before fusion: a fused survivor does not split
    int sp = (src >= 0 && w_in[src] > thr_split) ? 1 : 0;
    int ex, tot;
    block_scan(sp, ex, tot);
    if (src >= 0) {
      double wk = sp ? 0.5 * w : w;
      w_out[j] = wk;
      parent_out[j] = src;
      if (sp) {
        w_out[nk + ns + ex] = wk;
        parent_out[nk + ns + ex] = src;
      }
    }
    ns += tot;
  }
  if (tid == 0) *n_out = nk + ns;
}

namespace {
// The order in which determinant c's columns are swapped in from determinant
// c-1 so that no intermediate matrix holds one orbital twice
// (QMCWavefunction::makeCoefficients, QMcBeaver/src/QMCWavefunction.cpp:924-976).
// occ: [ndet][n] increasing active rows.  Returns [ndet][n] columns, -1 ends.
// (Increasing column lists never block for good; the scan stops after n
// passes regardless.)
std::vector<int> determinant_swaps(const int *occ, int ndet, int n)
{
  std::vector<int> iu(occ, occ + (size_t)ndet * n), sw((size_t)ndet * std::max(n, 1), -1);
  for (int c = 1; c < ndet; c++) {
    int k = 0, pass = 0;
    bool blocked;
    do {
      blocked = false;
      for (int o = 0; o < n; o++) {
        if (iu[(size_t)c * n + o] == iu[(size_t)(c - 1) * n + o]) continue;
        bool good = true;
        for (int o2 = 0; o2 < n; o2++)
          if (o != o2 && iu[(size_t)c * n + o] == iu[(size_t)(c - 1) * n + o2]) {
            blocked = true;
            good = false;
            break;
          }
        if (good) {
          iu[(size_t)(c - 1) * n + o] = iu[(size_t)c * n + o];
          sw[(size_t)c * n + k++] = o;
        }
      }
    } while (blocked && ++pass <= n);
  }
  return sw;
}

std::mutex g_noalloc_mu;
void *g_noalloc_w_addr[64];
void *g_noalloc_i_addr[64];
}  // namespace

// One launch of the single-determinant move kernel in the walker state's
// precision, with the cusp / three-body code only when the system has them.
template <bool kMetropolis, typename TS, typename TI, bool kExtras>
static void launch_move_g(qmcb_handle *h, const dim3 &g, const dim3 &b, size_t sm, cudaStream_t st, const RunCfg &cfg,
                          const int *slots, int num, const int *d_num, const double *R_in, const MoveArgs &mv,
                          const EvalOut &o)
{
  // with rows from the tensor cores the scratch has no basis rows
  const Layout &L = mv.rows ? h->lay_rows : h->lay;
  if (h->ginv)
    k_move<kMetropolis, TS, TI, kExtras, true><<<g, b, sm, st>>>(h->sys, L, cfg, h->d_state, slots, num, d_num,
                                                                 R_in, mv, h->d_ectl, h->d_stats, o);
  else
    k_move<kMetropolis, TS, TI, kExtras, false><<<g, b, sm, st>>>(h->sys, L, cfg, h->d_state, slots, num, d_num,
                                                                  R_in, mv, h->d_ectl, h->d_stats, o);
}

// Walker state written under QMCB_PREC_FP64 serves the tensor-core rows modes too.
static int state_kind(int prec) { return prec == QMCB_PREC_MIXED ? QMCB_PREC_MIXED : QMCB_PREC_FP64; }

// The modes whose orbital rows come from a batched tensor-core contraction.
static bool rows_mode(int prec)
{
  return prec == QMCB_PREC_INT8_SLICES || prec == QMCB_PREC_BF16_TC || prec == QMCB_PREC_BF16X3_TC;
}

// The batched orbital rows of one single-electron step (the tensor-core
// rows modes) into h->d_rows_out: proposal + basis operand planes, then the
// contraction; prof: record the two kernels' times (not under stream capture).
template <bool kMetropolis>
static void launch_rows(qmcb_handle *h, int cap, cudaStream_t st, const RunCfg &cfg, const int *slots, int num,
                        const int *d_num, const double *R_in, const MoveArgs &mv, bool extras, bool prof)
{
  const int prec = h->params.precision;
  const int sp = mv.e < h->sys.na ? 0 : 1, n = sp ? h->sys.nb : h->sys.na;
  const int pb = (cap + h->wpb_prep - 1) / h->wpb_prep;
  const unsigned th = 32 * h->wpb_prep;
  const int ntiles = (n + kNTile - 1) / kNTile;
  const unsigned g = (unsigned)((cap + kTileWalkers - 1) / kTileWalkers) * (unsigned)ntiles;
  if (prec == QMCB_PREC_BF16_TC || prec == QMCB_PREC_BF16X3_TC) {
    const bool x3 = prec == QMCB_PREC_BF16X3_TC;
    {
      ProfScope ps(h, QMCB_KERNEL_ROWS_PREP, st, prof);
      if (extras && x3)
        k_rows_prep_bf<kMetropolis, true, 2><<<pb, th, h->smem_prep, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num,
                                                                            d_num, R_in, mv, h->bf_ksteps, h->d_bf_A);
      else if (extras)
        k_rows_prep_bf<kMetropolis, true, 1><<<pb, th, h->smem_prep, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num,
                                                                            d_num, R_in, mv, h->bf_ksteps, h->d_bf_A);
      else if (x3)
        k_rows_prep_bf<kMetropolis, false, 2><<<pb, th, h->smem_prep, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num,
                                                                             d_num, R_in, mv, h->bf_ksteps, h->d_bf_A);
      else
        k_rows_prep_bf<kMetropolis, false, 1><<<pb, th, h->smem_prep, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num,
                                                                             d_num, R_in, mv, h->bf_ksteps, h->d_bf_A);
      ps.end(st);
    }
    ProfScope ps(h, QMCB_KERNEL_ROWS_MMA, st, prof);
    if (x3)
      k_rows_mma_bf<2><<<g, kBfThreads, bf_smem_bytes(2), st>>>(h->d_bf_A, h->d_bf_B[sp], n, ntiles, h->bf_ksteps, num,
                                                                d_num, h->d_rows_out, h->d_ctl + 3);
    else
      k_rows_mma_bf<1><<<g, kBfThreads, bf_smem_bytes(1), st>>>(h->d_bf_A, h->d_bf_B[sp], n, ntiles, h->bf_ksteps, num,
                                                                d_num, h->d_rows_out, h->d_ctl + 3);
    ps.end(st);
  } else {
    {
      ProfScope ps(h, QMCB_KERNEL_ROWS_PREP, st, prof);
      if (extras)
        k_rows_prep<kMetropolis, true><<<pb, th, h->smem_prep, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num, d_num,
                                                                      R_in, mv, h->rows_ksteps, h->d_rows_A, h->d_rows_rs);
      else
        k_rows_prep<kMetropolis, false><<<pb, th, h->smem_prep, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num, d_num,
                                                                       R_in, mv, h->rows_ksteps, h->d_rows_A, h->d_rows_rs);
      ps.end(st);
    }
    // the orbital tiles of a tile adjacent in the grid (A read once from HBM)
    ProfScope ps(h, QMCB_KERNEL_ROWS_MMA, st, prof);
    k_rows_mma<<<g, kRowsThreads, kRowsSmem, st>>>(h->d_rows_A, h->d_rows_B[sp], h->d_rows_rs, h->d_rows_cs[sp], n,
                                                   ntiles, h->rows_ksteps, num, d_num, h->d_rows_out, h->d_ctl + 3);
    ps.end(st);
  }
  h->rows_n = n;
  h->rows_num = cap;
}

// One single-electron move of list entries [0, num) (d_num: device count,
// grids sized for `cap` entries).  Under QMCB_PREC_INT8_SLICES three
// launches: proposal + basis digits, the tensor-core contraction, the move
// kernel on the rows; else the move kernel alone.
template <bool kMetropolis>
static void launch_move(qmcb_handle *h, int cap, cudaStream_t st, const RunCfg &cfg, const int *slots, int num,
                        const int *d_num, const double *R_in, MoveArgs mv, EvalOut o)
{
  // the Umrigar93 move is compiled only into the extras instantiation
  const bool extras = h->extras || (kMetropolis && cfg.sampling == QMCB_UMRIGAR93_IMPORTANCE_SAMPLING);
  if (rows_mode(h->params.precision)) {
    launch_rows<kMetropolis>(h, cap, st, cfg, slots, num, d_num, R_in, mv, extras, true);
    mv.rows = h->d_rows_out;
    const dim3 g((cap + h->wpb_rows - 1) / h->wpb_rows), b(32 * h->wpb_rows);
    ProfScope ps(h, QMCB_KERNEL_MOVE, st);
    if (extras)
      launch_move_g<kMetropolis, double, double, true>(h, g, b, h->smem_rows, st, cfg, slots, num, d_num, R_in, mv, o);
    else
      launch_move_g<kMetropolis, double, double, false>(h, g, b, h->smem_rows, st, cfg, slots, num, d_num, R_in, mv, o);
    ps.end(st);
    return;
  }
  const dim3 g((cap + h->wpb_move - 1) / h->wpb_move), b(32 * h->wpb_move);
  const size_t sm = h->smem_move;
  ProfScope ps(h, QMCB_KERNEL_MOVE, st);
  if (h->params.precision == QMCB_PREC_MIXED) {
    if (extras)
      launch_move_g<kMetropolis, float, MIXED_TI, true>(h, g, b, sm, st, cfg, slots, num, d_num, R_in, mv, o);
    else
      launch_move_g<kMetropolis, float, MIXED_TI, false>(h, g, b, sm, st, cfg, slots, num, d_num, R_in, mv, o);
  } else {
    if (extras)
      launch_move_g<kMetropolis, double, double, true>(h, g, b, sm, st, cfg, slots, num, d_num, R_in, mv, o);
    else
      launch_move_g<kMetropolis, double, double, false>(h, g, b, sm, st, cfg, slots, num, d_num, R_in, mv, o);
  }
  ps.end(st);
}

// The dynamic shared-memory limit of every move-kernel instantiation.
template <bool kMetropolis, typename TS, typename TI>
static cudaError_t move_smem_limits(int bytes)
{
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_move<kMetropolis, TS, TI, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_move<kMetropolis, TS, TI, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_move<kMetropolis, TS, TI, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_move<kMetropolis, TS, TI, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

// ---------------------------------------------------------------------------
// Batched orbital rows on the tensor cores (QMCB_PREC_INT8_SLICES,
// kernels_rows.cuh).


template <bool kMetropolis>
static cudaError_t rows_prep_limits(int bytes)
{
  cudaError_t e = cudaFuncSetAttribute(k_rows_prep<kMetropolis, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rows_prep<kMetropolis, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

// Warps per CTA (1 .. kMaxWarpsPerBlock) that keep the most warps of a kernel
// resident per SM when each warp needs `per_warp` bytes of shared memory
// (large scratches pack better in small CTAs).
static int best_warps_per_block(const qmcb_handle *h, size_t per_warp)
{
  int max_optin = 0, smem_sm = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->device);
  int wpb = 1, best = 0;
  for (int w = 1; w <= kMaxWarpsPerBlock && (size_t)w * per_warp <= (size_t)max_optin; w++) {
    const int resident = w * (int)(smem_sm / (w * per_warp + 1024));  // 1 KB reserved per CTA
    if (resident >= best) {
      best = resident;
      wpb = w;
    }
  }
  return wpb;
}

#define CKR(call)                                                                                    \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return fail(h, e_ == cudaErrorMemoryAllocation ? QMCB_E_NOMEM : QMCB_E_CUDA,                   \
                  std::string("tensor-core rows set-up: " #call ": ") + cudaGetErrorString(e_));     \
  } while (0)

template <bool kMetropolis>
static cudaError_t rows_prep_bf_limits(int bytes)
{
  cudaError_t e = cudaFuncSetAttribute(k_rows_prep_bf<kMetropolis, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rows_prep_bf<kMetropolis, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rows_prep_bf<kMetropolis, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rows_prep_bf<kMetropolis, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

// What every tensor-core rows mode shares, once per handle: the rows
// buffer, the move kernel's smaller scratch layout (no basis rows), the
// prep kernels' CTA shapes and shared-memory limits.
static int rows_common_setup(qmcb_handle *h)
{
  if (h->d_rows_out) return QMCB_OK;
  const int K = h->K, N = h->N;
  // the move kernel without the basis rows: region A holds only the slice
  // sums and the new drifts (and the three-body partner gradients)
  Layout L = h->lay;
  const int ra = even(std::max(kPart + 6 * N, h->sys.ntb > 0 ? 3 * N * h->sys.M : 0));
  L.mv_stride += ra - L.mv_region_a;
  L.mv_region_a = ra;
  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  const size_t per_move = sizeof(double) * (size_t)L.mv_stride;
  const size_t per_prep = sizeof(double) * (size_t)rows_prep_doubles(N, K, h->sys.nslot);
  if (per_move > (size_t)max_optin || per_prep > (size_t)max_optin || kRowsSmem > max_optin ||
      bf_smem_bytes(2) > max_optin)
    return fail(h, QMCB_E_LIMIT, "tensor-core rows: system too large for the per-walker shared-memory scratch");
  CKR(cudaMalloc(&h->d_rows_out, sizeof(double) * (size_t)h->max_walkers * 5 * h->nmax));
  // a wait inside a contraction kernel that gave up sets ctl[3], which
  // returns with every batch's live count
  CKR(cudaMemsetAsync(h->d_ctl + 3, 0, sizeof(int), h->stream));
  h->lay_rows = L;
  h->wpb_rows = best_warps_per_block(h, per_move);
  h->smem_rows = per_move * h->wpb_rows;
  h->wpb_prep = best_warps_per_block(h, per_prep);
  h->smem_prep = per_prep * h->wpb_prep;
  CKR(rows_prep_limits<true>(max_optin));
  CKR(rows_prep_limits<false>(max_optin));
  CKR(rows_prep_bf_limits<true>(max_optin));
  CKR(rows_prep_bf_limits<false>(max_optin));
  CKR(cudaFuncSetAttribute(k_rows_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowsSmem));
  CKR(cudaFuncSetAttribute(k_rows_mma_bf<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bf_smem_bytes(1)));
  CKR(cudaFuncSetAttribute(k_rows_mma_bf<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bf_smem_bytes(2)));
  return QMCB_OK;
}

// QMCB_PREC_INT8_SLICES: digit tables of the MO coefficients and the
// operand buffers; once per handle, on the first use of the mode.
static int rows_setup(qmcb_handle *h)
{
  const int rc = rows_common_setup(h);
  if (rc) return rc;
  if (h->d_rows_A) return QMCB_OK;
  const int K = h->K;
  const int ks = (K + kKStep - 1) / kKStep;
  const size_t tiles = (size_t)(h->max_walkers + kTileWalkers - 1) / kTileWalkers;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? h->sys.nb : h->sys.na;
    const int nt = std::max((n + kNTile - 1) / kNTile, 1);
    std::vector<signed char> B((size_t)nt * ks * kSlices * kBBlock, 0);
    // one scale per (orbital, K step): cs[(orbital tile x ks + K step) x kNTile + orbital in tile]
    std::vector<double> cs((size_t)nt * ks * kNTile, 1.0);
    const std::vector<double> &ct = h->ct_host[sp];
    for (int o = 0; o < n; o++) {
      for (int kk = 0; kk < ks; kk++) {
        const int k1 = std::min(K, (kk + 1) * kKStep);
        double amax = 0.0;
        for (int k = kk * kKStep; k < k1; k++) amax = std::max(amax, std::fabs(ct[(size_t)k * n + o]));
        const double scale = rows_scale(amax), inv = 1.0 / scale;
        cs[((size_t)(o / kNTile) * ks + kk) * kNTile + o % kNTile] = scale;
        for (int k = kk * kKStep; k < k1; k++) {
          signed char dg[kSlices];
          rows_digits(ct[(size_t)k * n + o] * inv, dg);
          for (int q = 0; q < kSlices; q++)
            B[(((size_t)(o / kNTile) * ks + kk) * kSlices + q) * kBBlock + rows_blk_off(o % kNTile, k % kKStep)] = dg[q];
        }
      }
    }
    CKR(cudaMalloc(&h->d_rows_B[sp], B.size()));
    CKR(cudaMemcpy(h->d_rows_B[sp], B.data(), B.size(), cudaMemcpyHostToDevice));
    CKR(cudaMalloc(&h->d_rows_cs[sp], sizeof(double) * cs.size()));
    CKR(cudaMemcpy(h->d_rows_cs[sp], cs.data(), sizeof(double) * cs.size(), cudaMemcpyHostToDevice));
  }
  const size_t abytes = tiles * ks * kSlices * kABlock;
  CKR(cudaMalloc(&h->d_rows_A, abytes));
  // on the handle's stream (non-blocking: a legacy-stream memset would not
  // be ordered with its work)
  CKR(cudaMemsetAsync(h->d_rows_A, 0, abytes, h->stream));  // rows 125 .. 127 of every tile stay zero
  CKR(cudaMalloc(&h->d_rows_rs, sizeof(double) * tiles * kTileRows * ks));  // [row][K step], 128 rows a tile
  h->rows_ksteps = ks;
  return QMCB_OK;
}

// QMCB_PREC_BF16_TC / QMCB_PREC_BF16X3_TC: hi and lo BF16 planes of the MO
// coefficients ([orbital tile][K step][plane] blocks) and the A buffer
// (room for two planes); once per handle, on the first use of either mode.
static int rows_bf_setup(qmcb_handle *h)
{
  const int rc = rows_common_setup(h);
  if (rc) return rc;
  if (h->d_bf_A) return QMCB_OK;
  const int K = h->K;
  const int ks = (K + kBfKStep - 1) / kBfKStep;
  const size_t tiles = (size_t)(h->max_walkers + kTileWalkers - 1) / kTileWalkers;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? h->sys.nb : h->sys.na;
    const int nt = std::max((n + kNTile - 1) / kNTile, 1);
    std::vector<unsigned char> B((size_t)nt * ks * 2 * kBBlock, 0);
    const std::vector<double> &ct = h->ct_host[sp];
    for (int o = 0; o < n; o++)
      for (int k = 0; k < K; k++) {
        const double c = ct[(size_t)k * n + o], hi = bf16_round(c), lo = bf16_round(c - hi);
        const size_t blk = ((size_t)(o / kNTile) * ks + k / kBfKStep) * 2;
        const int off = rows_blk_off(o % kNTile, 2 * (k % kBfKStep));
        const uint32_t hb = bf16_bits(hi), lb = bf16_bits(lo);
        B[blk * kBBlock + off] = (unsigned char)(hb & 0xff);
        B[blk * kBBlock + off + 1] = (unsigned char)(hb >> 8);
        B[(blk + 1) * kBBlock + off] = (unsigned char)(lb & 0xff);
        B[(blk + 1) * kBBlock + off + 1] = (unsigned char)(lb >> 8);
      }
    CKR(cudaMalloc(&h->d_bf_B[sp], B.size()));
    CKR(cudaMemcpy(h->d_bf_B[sp], B.data(), B.size(), cudaMemcpyHostToDevice));
  }
  const size_t abytes = tiles * ks * 2 * kABlock;
  CKR(cudaMalloc(&h->d_bf_A, abytes));
  CKR(cudaMemsetAsync(h->d_bf_A, 0, abytes, h->stream));  // rows 125 .. 127 of every tile stay zero
  h->bf_ksteps = ks;
  return QMCB_OK;
}
#undef CKR

extern "C" {

const char *qmcb_version(void) { return "qmcb200 0.1 (sm_100a, FP64 parity path)"; }

const char *qmcb_last_error(const qmcb_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int qmcb_fit_cusps(const qmcb_system_desc *d, int beta, double *out)
{
  if (!d || !out || d->n_nuclei <= 0 || d->n_basis <= 0) return fail(nullptr, QMCB_E_ARG, "qmcb_fit_cusps: bad argument");
  const int rows = d->n_det > 1 ? (beta ? d->n_act_beta : d->n_act_alpha) : (beta ? d->n_beta : d->n_alpha);
  const double *mo = beta ? d->mo_beta : d->mo_alpha;
  if (rows <= 0) return QMCB_OK;
  char err[256];
  if (qmcb_cusp_fit(d->n_nuclei, d->nuc_xyz, d->nuc_charge, d->n_basis, d->bf_atom, d->bf_powers, d->bf_nprim,
                    d->bf_prim_offset, d->prim_exponent, d->prim_coeff, rows, mo, out, err))
    return fail(nullptr, QMCB_E_ARG, std::string("qmcb_fit_cusps: ") + err);
  return QMCB_OK;
}

int qmcb_create(const qmcb_system_desc *d, int max_walkers, qmcb_handle **out)
{
  qmcb_handle *h = nullptr;
  if (!d || !out || max_walkers <= 0) return fail(nullptr, QMCB_E_ARG, "qmcb_create: null argument or max_walkers <= 0");
  *out = nullptr;
  const int M = d->n_nuclei, na = d->n_alpha, nb = d->n_beta, K = d->n_basis;
  if (M <= 0 || na < 0 || nb < 0 || na + nb <= 0 || K <= 0 || d->n_pade < 0)
    return fail(nullptr, QMCB_E_ARG, "qmcb_create: bad sizes");
  if (na > 256 || nb > 256 || K > 4096 || M > 1024)
    return fail(nullptr, QMCB_E_LIMIT, "qmcb_create: n_alpha/n_beta <= 256, n_basis <= 4096, n_nuclei <= 1024");
  // several determinants: active rows and increasing column lists
  const bool md = d->n_det > 1;
  const int nact[2] = {md ? d->n_act_alpha : na, md ? d->n_act_beta : nb};
  if (md) {
    if (!d->ci_coeff || (na > 0 && !d->det_occ_alpha) || (nb > 0 && !d->det_occ_beta) || nact[0] < na ||
        nact[1] < nb || nact[0] > 1024 || nact[1] > 1024 || d->n_det > 4096)
      return fail(nullptr, QMCB_E_ARG, "qmcb_create: bad determinant tables");
    for (int sp = 0; sp < 2; sp++) {
      const int n = sp ? nb : na;
      const int *occ = sp ? d->det_occ_beta : d->det_occ_alpha;
      for (int c = 0; c < d->n_det; c++)
        for (int o = 0; o < n; o++) {
          const int v = occ[c * n + o];
          if (v < 0 || v >= nact[sp] || (o > 0 && v <= occ[c * n + o - 1]))
            return fail(nullptr, QMCB_E_ARG, "qmcb_create: determinant columns must be increasing active rows");
        }
    }
    for (int c = 0; c < d->n_det; c++)
      if (!std::isfinite(d->ci_coeff[c])) return fail(nullptr, QMCB_E_ARG, "qmcb_create: CI coefficient not finite");
  }
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || ndev == 0)
    return fail(nullptr, QMCB_E_CUDA, std::string("qmcb_create: no CUDA device: ") + cudaGetErrorString(ce));

  h = new (std::nothrow) qmcb_handle();
  if (!h) return fail(nullptr, QMCB_E_NOMEM, "qmcb_create: out of host memory");
  cudaGetDevice(&h->device);
  h->N = na + nb;
  h->K = K;
  h->nmax = std::max(na, nb);
  h->max_walkers = max_walkers;
  default_params(&h->params);

  // ---- system tables
  std::vector<double4> nuc(M);
  for (int a = 0; a < M; a++)
    nuc[a] = make_double4(d->nuc_xyz[3 * a], d->nuc_xyz[3 * a + 1], d->nuc_xyz[3 * a + 2], d->nuc_charge[a]);
  std::vector<int4> bf(K);
  for (int k = 0; k < K; k++) {
    int a = d->bf_powers[3 * k], b = d->bf_powers[3 * k + 1], c = d->bf_powers[3 * k + 2];
    if (d->bf_atom[k] < 0 || d->bf_atom[k] >= M || a < 0 || b < 0 || c < 0 || a > 15 || b > 15 || c > 15 ||
        d->bf_nprim[k] <= 0 || d->bf_prim_offset[k] < 0 ||
        d->bf_prim_offset[k] + d->bf_nprim[k] > d->n_prim_total) {
      delete h;
      return fail(nullptr, QMCB_E_ARG, "qmcb_create: bad basis function table");
    }
    bf[k] = make_int4(d->bf_atom[k], a | (b << 8) | (c << 16), d->bf_nprim[k], d->bf_prim_offset[k]);
  }
  std::vector<double2> prim(d->n_prim_total);
  for (int i = 0; i < d->n_prim_total; i++) prim[i] = make_double2(d->prim_exponent[i], d->prim_coeff[i]);
  // shells: runs of consecutive functions on one centre with the same angular
  // momentum and identical exponent lists (their exps are shared)
  std::vector<double> pexp(d->prim_exponent, d->prim_exponent + d->n_prim_total);
  std::vector<double> pcoef(d->prim_coeff, d->prim_coeff + d->n_prim_total);
  std::vector<int2> fn(K);
  std::vector<int4> shells;
  for (int k = 0; k < K;) {
    const int atom = d->bf_atom[k], np = d->bf_nprim[k], off = d->bf_prim_offset[k];
    const int L = d->bf_powers[3 * k] + d->bf_powers[3 * k + 1] + d->bf_powers[3 * k + 2];
    const int maxmem = (L + 1) * (L + 2) / 2;
    int m = 1;
    while (k + m < K && m < maxmem && m < 255 && np <= kShellPrim) {
      const int k2 = k + m;
      const int L2 = d->bf_powers[3 * k2] + d->bf_powers[3 * k2 + 1] + d->bf_powers[3 * k2 + 2];
      if (d->bf_atom[k2] != atom || d->bf_nprim[k2] != np || L2 != L) break;
      bool same = true;
      for (int i = 0; i < np; i++)
        if (d->prim_exponent[d->bf_prim_offset[k2] + i] != d->prim_exponent[off + i]) same = false;
      if (!same) break;
      m++;
    }
    shells.push_back(make_int4(atom, k, m | (L << 8) | (np << 16), off));
    k += m;
  }
  for (int k = 0; k < K; k++) {
    int a = d->bf_powers[3 * k], b = d->bf_powers[3 * k + 1], c = d->bf_powers[3 * k + 2];
    fn[k] = make_int2(a | (b << 8) | (c << 16), d->bf_prim_offset[k]);
  }
  // lanes of a warp take consecutive shells: order them by angular momentum
  // and size so neighbouring lanes run the same member loop
  std::stable_sort(shells.begin(), shells.end(), [](const int4 &x, const int4 &y) {
    return (x.z & 0xffff) < (y.z & 0xffff);
  });
  // exponential slots of the move kernel's basis pass: one per (shell,
  // primitive) in shell order; every function points at its shell's slots
  std::vector<int2> xsl;
  std::vector<int4> fq(K);
  for (const int4 &sh : shells) {
    const int nmem = sh.z & 0xff, L = (sh.z >> 8) & 0xff, np = sh.z >> 16;
    const int q0 = (int)xsl.size();
    for (int i = 0; i < np; i++) xsl.push_back(make_int2(sh.x, sh.w + i));
    for (int m = 0; m < nmem; m++) fq[sh.y + m] = make_int4(sh.x, q0, np, L);
  }
  std::vector<double> ct[2];
  for (int sp = 0; sp < 2; sp++) {
    int n = nact[sp];
    const double *mo = sp ? d->mo_beta : d->mo_alpha;
    ct[sp].assign((size_t)K * std::max(n, 1), 0.0);
    for (int o = 0; o < n; o++)
      for (int k = 0; k < K; k++) ct[sp][(size_t)k * n + o] = mo[(size_t)o * K + k];
  }
  std::vector<int> docc[2], dswap[2];
  std::vector<double> ci(md ? d->n_det : 1, 1.0);
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? nb : na;
    const int *occ = sp ? d->det_occ_beta : d->det_occ_alpha;
    docc[sp].assign((size_t)std::max(md ? d->n_det * n : 0, 1), 0);
    if (md)
      for (int t = 0; t < d->n_det * n; t++) docc[sp][t] = occ[t];
    dswap[sp] = md ? determinant_swaps(docc[sp].data(), d->n_det, n) : std::vector<int>(1, -1);
  }
  if (md)
    for (int c = 0; c < d->n_det; c++) ci[c] = d->ci_coeff[c];
  // three-body Jastrow tables
  const int ntb = d->n_tb > 0 ? d->n_tb : 0;
  std::vector<int4> tbi(std::max(ntb, 1), make_int4(0, 0, 0, 0));
  std::vector<double> tbL(std::max(ntb, 1), 0.0), tbc(1, 0.0);
  std::vector<int> tbp((size_t)3 * M, -1);
  if (ntb > 0) {
    if (!d->tb_nen || !d->tb_nee || !d->tb_C || !d->tb_cutoff || !d->tb_offset || !d->tb_coeff || !d->tb_pair) {
      delete h;
      return fail(nullptr, QMCB_E_ARG, "qmcb_create: incomplete three-body tables");
    }
    size_t ncoef = 0;
    for (int f = 0; f < ntb; f++) {
      const int nen = d->tb_nen[f], nee = d->tb_nee[f];
      if (nen < 1 || nee < 1 || nen > kTbMax || nee > kTbMax || d->tb_C[f] < 0 || d->tb_C[f] > 16 || d->tb_offset[f] < 0) {
        delete h;
        return fail(nullptr, QMCB_E_ARG, "qmcb_create: three-body sizes out of range (NeN, Nee <= 8, C <= 16)");
      }
      tbi[f] = make_int4(nen, nee, d->tb_C[f], d->tb_offset[f]);
      tbL[f] = d->tb_cutoff[f];
      ncoef = std::max(ncoef, (size_t)d->tb_offset[f] + (size_t)nen * nen * nee);
    }
    tbc.assign(d->tb_coeff, d->tb_coeff + ncoef);
    for (int t = 0; t < 3 * M; t++) {
      tbp[t] = d->tb_pair[t];
      if (tbp[t] >= ntb) {
        delete h;
        return fail(nullptr, QMCB_E_ARG, "qmcb_create: three-body function index out of range");
      }
    }
  }
  // electron-nucleus cusp replacement tables
  std::vector<int> cns(M, 0);
  int nsmax = 1;
  for (int k = 0; k < K; k++)
    if (d->bf_powers[3 * k] + d->bf_powers[3 * k + 1] + d->bf_powers[3 * k + 2] == 0) cns[d->bf_atom[k]] += d->bf_nprim[k];
  for (int a = 0; a < M; a++) nsmax = std::max(nsmax, cns[a]);
  std::vector<double> csexp((size_t)M * nsmax, 0.0), cscoef[2], cpar[2], crmax[2];
  for (int sp = 0; sp < 2; sp++) {
    const int a_ = std::max(nact[sp], 1);
    cscoef[sp].assign((size_t)M * a_ * nsmax, 0.0);
    cpar[sp].assign((size_t)M * a_ * QMCB_CUSP_REC, 0.0);
    crmax[sp].assign(M, 0.0);
  }
  if (d->replace_cusps) {
    std::vector<int> fill(M, 0);
    for (int k = 0; k < K; k++) {
      const int at = d->bf_atom[k];
      if (d->bf_powers[3 * k] + d->bf_powers[3 * k + 1] + d->bf_powers[3 * k + 2] != 0) continue;
      for (int l = 0; l < d->bf_nprim[k]; l++) csexp[(size_t)at * nsmax + fill[at]++] = d->prim_exponent[d->bf_prim_offset[k] + l];
    }
    for (int sp = 0; sp < 2; sp++) {
      const int a_ = nact[sp];
      if (a_ == 0) continue;
      const double *mo = sp ? d->mo_beta : d->mo_alpha;
      const double *given = sp ? d->cusp_beta : d->cusp_alpha;
      if (given) {
        std::copy(given, given + (size_t)M * a_ * QMCB_CUSP_REC, cpar[sp].begin());
      } else {
        std::vector<double> xyz(3 * M), Zd(M);
        for (int at = 0; at < M; at++) {
          for (int x = 0; x < 3; x++) xyz[3 * at + x] = d->nuc_xyz[3 * at + x];
          Zd[at] = d->nuc_charge[at];
        }
        char err[256];
        if (qmcb_cusp_fit(M, xyz.data(), Zd.data(), K, d->bf_atom, d->bf_powers, d->bf_nprim, d->bf_prim_offset,
                          d->prim_exponent, d->prim_coeff, a_, mo, cpar[sp].data(), err)) {
          delete h;
          return fail(nullptr, QMCB_E_ARG, std::string("qmcb_create: ") + err);
        }
      }
      // s-part coefficients of every (nucleus, orbital): primitive coefficient x orbital coefficient
      for (int at = 0; at < M; at++) {
        for (int o = 0; o < a_; o++) {
          int cnt = 0;
          for (int k = 0; k < K; k++) {
            if (d->bf_atom[k] != at || d->bf_powers[3 * k] + d->bf_powers[3 * k + 1] + d->bf_powers[3 * k + 2] != 0)
              continue;
            for (int l = 0; l < d->bf_nprim[k]; l++)
              cscoef[sp][((size_t)at * a_ + o) * nsmax + cnt++] =
                  d->prim_coeff[d->bf_prim_offset[k] + l] * mo[(size_t)o * K + k];
          }
          crmax[sp][at] = std::max(crmax[sp][at], cpar[sp][((size_t)at * a_ + o) * QMCB_CUSP_REC]);
        }
      }
    }
  }
  std::vector<double> pade((size_t)std::max(d->n_pade, 1) * 2 * kPadeMax, 0.0);
  std::vector<int2> plen(std::max(d->n_pade, 1), make_int2(1, 1));
  for (int f = 0; f < d->n_pade; f++) {
    int ln = d->pade_nnum[f], ld = d->pade_nden[f];
    if (ln < 1 || ln > kPadeMax || ld < 1 || ld > kPadeMax) {
      delete h;
      return fail(nullptr, QMCB_E_ARG, "qmcb_create: Pade polynomial length out of range");
    }
    for (int i = 0; i < kPadeMax; i++) {
      pade[(size_t)f * 2 * kPadeMax + i] = d->pade_num[f * kPadeMax + i];
      pade[(size_t)f * 2 * kPadeMax + kPadeMax + i] = d->pade_den[f * kPadeMax + i];
    }
    plen[f] = make_int2(ln, ld);
  }
  std::vector<int> ctype(std::max(d->n_pade, 1), 0);
  std::vector<double4> cparam(std::max(d->n_pade, 1), make_double4(0.0, 0.0, 0.0, 0.0));
  for (int f = 0; f < d->n_pade; f++) {
    ctype[f] = d->corr_type ? d->corr_type[f] : QMCB_CORR_PADE;
    if (ctype[f] != QMCB_CORR_PADE && ctype[f] != QMCB_CORR_CAMBRIDGE2) {
      delete h;
      return fail(nullptr, QMCB_E_ARG, "qmcb_create: unknown correlation function type");
    }
    if (ctype[f] == QMCB_CORR_CAMBRIDGE2) {
      if (!d->corr_param) {
        delete h;
        return fail(nullptr, QMCB_E_ARG, "qmcb_create: Cambridge2 function without corr_param");
      }
      const double *cp = d->corr_param + 4 * f;
      if (cp[1] < 1.0 || cp[1] > 16.0) {
        delete h;
        return fail(nullptr, QMCB_E_ARG, "qmcb_create: Cambridge2 exponent C out of range");
      }
      cparam[f] = make_double4(cp[0], cp[1], cp[2], cp[3]);
    }
  }
  // every function of the form a r / (1 + b r) takes the closed-form path
  std::vector<double2> pade_ab(std::max(d->n_pade, 1), make_double2(0.0, 0.0));
  bool pade_simple = d->n_pade > 0;
  for (int f = 0; f < d->n_pade; f++) {
    const double *nu = d->pade_num + f * kPadeMax, *de = d->pade_den + f * kPadeMax;
    if (ctype[f] == QMCB_CORR_PADE && d->pade_nnum[f] == 2 && d->pade_nden[f] == 2 && nu[0] == 0.0 && de[0] == 1.0)
      pade_ab[f] = make_double2(nu[1], de[1]);
    else
      pade_simple = false;
  }
  for (int i = 0; i < 3; i++)
    if (d->ee_pade[i] >= d->n_pade) {
      delete h;
      return fail(nullptr, QMCB_E_ARG, "qmcb_create: ee_pade index out of range");
    }
  std::vector<int> en[2];
  for (int sp = 0; sp < 2; sp++) {
    const int *src = sp ? d->en_pade_dn : d->en_pade_up;
    en[sp].assign(M, -1);
    for (int a = 0; a < M; a++) {
      en[sp][a] = src ? src[a] : -1;
      if (en[sp][a] >= d->n_pade) {
        delete h;
        return fail(nullptr, QMCB_E_ARG, "qmcb_create: en_pade index out of range");
      }
    }
  }
  double Pnn = 0.0;
  for (int i = 0; i < M; i++)
    for (int j = i + 1; j < M; j++) {
      double dx = nuc[i].x - nuc[j].x, dy = nuc[i].y - nuc[j].y, dz = nuc[i].z - nuc[j].z;
      Pnn += (nuc[i].w * nuc[j].w) / std::sqrt(dx * dx + dy * dy + dz * dz);
    }

#define CKC(call)                                                                           \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      std::string m_ = std::string("qmcb_create: " #call ": ") + cudaGetErrorString(e_);    \
      qmcb_destroy(h);                                                                      \
      return fail(nullptr, e_ == cudaErrorMemoryAllocation ? QMCB_E_NOMEM : QMCB_E_CUDA, m_); \
    }                                                                                       \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  CKC(upload(&h->d_nuc, nuc));
  CKC(upload(&h->d_bf, bf));
  CKC(upload(&h->d_prim, prim));
  CKC(upload(&h->d_shell, shells));
  CKC(upload(&h->d_fn, fn));
  CKC(upload(&h->d_xsl, xsl));
  CKC(upload(&h->d_fq, fq));
  CKC(upload(&h->d_pexp, pexp));
  CKC(upload(&h->d_pcoef, pcoef));
  CKC(upload(&h->d_ct[0], ct[0]));
  CKC(upload(&h->d_ct[1], ct[1]));
  h->ct_host[0] = ct[0];
  h->ct_host[1] = ct[1];
  for (int sp = 0; sp < 2; sp++) {
    std::vector<float> cf(ct[sp].begin(), ct[sp].end());
    CKC(upload(&h->d_ctf[sp], cf));
  }
  CKC(upload(&h->d_pade, pade));
  CKC(upload(&h->d_pade_len, plen));
  CKC(upload(&h->d_pade_ab, pade_ab));
  CKC(upload(&h->d_ctype, ctype));
  CKC(upload(&h->d_cparam, cparam));
  CKC(upload(&h->d_en[0], en[0]));
  CKC(upload(&h->d_en[1], en[1]));
  CKC(upload(&h->d_docc[0], docc[0]));
  CKC(upload(&h->d_docc[1], docc[1]));
  CKC(upload(&h->d_dswap[0], dswap[0]));
  CKC(upload(&h->d_dswap[1], dswap[1]));
  CKC(upload(&h->d_ci, ci));
  CKC(upload(&h->d_tbi, tbi));
  CKC(upload(&h->d_tbL, tbL));
  CKC(upload(&h->d_tbc, tbc));
  CKC(upload(&h->d_tbp, tbp));
  CKC(upload(&h->d_cns, cns));
  CKC(upload(&h->d_csexp, csexp));
  for (int sp = 0; sp < 2; sp++) {
    CKC(upload(&h->d_cscoef[sp], cscoef[sp]));
    CKC(upload(&h->d_cpar[sp], cpar[sp]));
    CKC(upload(&h->d_crmax[sp], crmax[sp]));
  }
  h->md = md;

  DevSys &S = h->sys;
  S.M = M;
  S.na = na;
  S.nb = nb;
  S.N = h->N;
  S.K = K;
  S.npade = d->n_pade;
  for (int i = 0; i < 3; i++) S.ee[i] = d->ee_pade[i];
  S.Pnn = Pnn;
  S.nuc = h->d_nuc;
  S.bf = h->d_bf;
  S.prim = h->d_prim;
  S.nshell = (int)shells.size();
  S.shell = h->d_shell;
  S.fn = h->d_fn;
  S.nslot = (int)xsl.size();
  S.xsl = h->d_xsl;
  S.fq = h->d_fq;
  S.pexp = h->d_pexp;
  S.pcoef = h->d_pcoef;
  S.ct[0] = h->d_ct[0];
  S.ct[1] = h->d_ct[1];
  S.ctf[0] = h->d_ctf[0];
  S.ctf[1] = h->d_ctf[1];
  S.pade = h->d_pade;
  S.pade_len = h->d_pade_len;
  S.pade_ab = h->d_pade_ab;
  S.pade_simple = pade_simple ? 1 : 0;
  S.ctype = h->d_ctype;
  S.cparam = h->d_cparam;
  S.en[0] = h->d_en[0];
  S.en[1] = h->d_en[1];
  S.ndet = md ? d->n_det : 1;
  S.nact[0] = nact[0];
  S.nact[1] = nact[1];
  S.docc[0] = h->d_docc[0];
  S.docc[1] = h->d_docc[1];
  S.dswap[0] = h->d_dswap[0];
  S.dswap[1] = h->d_dswap[1];
  S.ntb = ntb;
  S.tbi = h->d_tbi;
  S.tbL = h->d_tbL;
  S.tbc = h->d_tbc;
  S.tbp = h->d_tbp;
  S.cusp = d->replace_cusps ? 1 : 0;
  h->extras = S.cusp || S.ntb > 0;
  S.nsmax = nsmax;
  S.cns = h->d_cns;
  S.csexp = h->d_csexp;
  for (int sp = 0; sp < 2; sp++) {
    S.cscoef[sp] = h->d_cscoef[sp];
    S.cpar[sp] = h->d_cpar[sp];
    S.crmax[sp] = h->d_crmax[sp];
  }
  S.ci = h->d_ci;

  // ---- per-walker block layout (offsets in doubles, arrays 32-byte aligned)
  Layout &L = h->lay;
  // spins above kStagedInverseMax electrons keep their inverse in HBM: a
  // staged n x n copy would cost the move kernel most of its occupancy
  int staged_max = kStagedInverseMax;
  if (const char *ev = getenv("QMCB_STAGED_INVERSE_MAX")) staged_max = atoi(ev);
  const bool ginv = !md && h->nmax > staged_max;
  h->ginv = ginv;
  L.invsz[0] = L.invsz[1] = 0;
  int off = 0;
  auto take = [&](int count) {
    int o = off;
    off += (count + 3) & ~3;
    return o;
  };
  L.R = take(3 * h->N);
  for (int sp = 0; sp < 2; sp++) {
    int n = sp ? nb : na, a = nact[sp];
    L.Dv[sp] = take(n * a);
    L.DgT[sp] = take(3 * a * n);
    L.DlT[sp] = take(a * n);
    if (md) {
      // two copies of [inverses | grad ratios | (ln|det|, sign, lap, singular)]
      L.mdsz[sp] = (S.ndet * n * n + S.ndet * 3 * n + S.ndet * 4 + 3) & ~3;
      L.Inv[sp] = take(2 * L.mdsz[sp]);
    } else if (ginv) {
      // two copies: the move reads one and writes the other
      L.mdsz[sp] = 0;
      L.invsz[sp] = (n * n + 3) & ~3;
      L.Inv[sp] = take(2 * L.invsz[sp]);
    } else {
      L.mdsz[sp] = 0;
      L.Inv[sp] = take(n * n);
    }
  }
  // the move kernel stages gradD .. sc in one copy; grad (an evaluate
  // output only) sits after them
  L.gradD = take(3 * h->N);
  L.Ux = take(3 * h->N);
  L.mgrad = take(3 * h->N);
  L.sc = take(kScalars);
  L.grad = take(3 * h->N);
  L.stride = (off + 31) & ~31;  // 256-byte aligned blocks
  // move-kernel scratch: staged copies read whole padded ranges of the block
  // (all inside the block: arrays start on 32-byte boundaries, the block is
  // padded to 256 bytes)
  L.mv_dn = even(5 * h->nmax);
  L.mv_valc = even(h->nmax);
  // the basis pass keeps its exponential slots after the five chi rows,
  // reaching into the Dn / valc space
  L.mv_region_a = std::max(move_region_a(h->N, K), even(5 * K + (int)xsl.size() - L.mv_dn - L.mv_valc));
  // three-body partner gradients (3 N M doubles) use region A before the basis
  if (S.ntb > 0) L.mv_region_a = std::max(L.mv_region_a, even(3 * h->N * S.M));
  L.mv_r = even(3 * h->N);
  L.mv_tail = even(L.sc + kScalars - L.gradD);
  for (int sp = 0; sp < 2; sp++) {
    int n = sp ? nb : na;
    L.mv_spin[sp] = ginv ? 0 : even(n * n);
  }
  L.mv_stride = L.mv_region_a + L.mv_dn + L.mv_valc + L.mv_r + L.mv_tail + std::max(L.mv_spin[0], L.mv_spin[1]) + 2;
  if (!md && (L.R + L.mv_r > L.stride || L.gradD + L.mv_tail > L.stride || L.Inv[0] + L.mv_spin[0] > L.stride ||
              L.Inv[1] + L.mv_spin[1] > L.stride)) {
    qmcb_destroy(h);
    return fail(nullptr, QMCB_E_ARG, "qmcb_create: internal layout error (staged ranges exceed the walker block)");
  }

  size_t bytes = (size_t)max_walkers * L.stride * sizeof(double);
  CKC(cudaMalloc(&h->d_state, bytes));
  CKC(cudaMemset(h->d_state, 0, bytes));
  CKC(cudaMalloc(&h->d_live, sizeof(int) * max_walkers));
  CKC(cudaMalloc(&h->d_live_tmp, sizeof(int) * max_walkers));
  CKC(cudaMalloc(&h->d_free, sizeof(int) * max_walkers));
  CKC(cudaMalloc(&h->d_ctl, sizeof(int) * 4));
  CKC(cudaMemset(h->d_ctl, 0, sizeof(int) * 4));
  CKC(cudaMalloc(&h->d_copies, sizeof(int2) * max_walkers));
  CKC(cudaMalloc(&h->d_stats, sizeof(double) * ST_COUNT));
  CKC(cudaMemset(h->d_stats, 0, sizeof(double) * ST_COUNT));
  CKC(cudaMalloc(&h->d_ectl, sizeof(EnergyCtl)));
  CKC(cudaMalloc(&h->d_slots, sizeof(int) * max_walkers));
  CKC(cudaMalloc(&h->d_R, sizeof(double) * (size_t)max_walkers * 3 * h->N));
  CKC(cudaMalloc(&h->d_out, sizeof(double) * (size_t)max_walkers * (6 * h->N + 8)));
  CKC(cudaMalloc(&h->d_status, max_walkers));
  CKC(cudaMallocHost(&h->h_stats, sizeof(double) * 2 * ST_COUNT));
  CKC(cudaMallocHost(&h->h_ctl, sizeof(int) * 2 * 4));
  CKC(cudaMallocHost(&h->h_ectl, sizeof(EnergyCtl) * 4));
  for (int k = 0; k < 4; k++) CKC(cudaEventCreateWithFlags(&h->ectl_ev[k], cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&h->done_ev[0], cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&h->done_ev[1], cudaEventDisableTiming));

  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  const int amax = std::max(nact[0], nact[1]);
  const size_t per_move =
      sizeof(double) * (size_t)(md ? move_md_scratch_doubles(h->N, K, h->nmax, amax, S.ndet, L.sc + kScalars - L.gradD, S.nslot,
                                                           S.ntb > 0 ? 3 * h->N * S.M : 0)
                                   : L.mv_stride);
  const size_t per_full =
      sizeof(double) * (size_t)(md ? full_md_scratch_doubles(h->N, K, h->nmax, amax, S.ndet)
                                   : full_scratch_doubles(h->N, K, h->nmax));
  if (per_move > (size_t)max_optin || per_full > (size_t)max_optin) {
    qmcb_destroy(h);
    return fail(nullptr, QMCB_E_LIMIT, "qmcb_create: system too large for the per-walker shared-memory scratch");
  }
  h->wpb_move = (int)std::min<size_t>(kMaxWarpsPerBlock, max_optin / per_move);
  h->wpb_full = (int)std::min<size_t>(kMaxWarpsPerBlock, max_optin / per_full);
  h->smem_move = per_move * h->wpb_move;
  h->smem_full = per_full * h->wpb_full;
  const size_t per_refresh = sizeof(double) * (size_t)refresh_scratch_doubles(h->N, h->nmax);
  h->wpb_refresh = best_warps_per_block(h, per_refresh);
  h->smem_refresh = per_refresh * h->wpb_refresh;
  // the dynamic shared-memory limit is a per-kernel, process-wide attribute:
  // raise it to the device maximum once, so handles of different systems
  // (each launching with its own size) never undercut one another
  CKC((move_smem_limits<true, double, double>(max_optin)));
  CKC((move_smem_limits<false, double, double>(max_optin)));
  CKC((move_smem_limits<true, float, MIXED_TI>(max_optin)));
  CKC((move_smem_limits<false, float, MIXED_TI>(max_optin)));
  CKC(cudaFuncSetAttribute(k_full<double, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  CKC(cudaFuncSetAttribute(k_full<float, MIXED_TI, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  CKC(cudaFuncSetAttribute(k_full<double, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  CKC(cudaFuncSetAttribute(k_full<float, MIXED_TI, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  CKC(cudaFuncSetAttribute(k_full_md, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  CKC(cudaFuncSetAttribute(k_move_md<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  CKC(cudaFuncSetAttribute(k_move_md<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_optin));
  // the memsets above ran on the legacy default stream, which does not order
  // against the handle's non-blocking stream: finish them before any work is
  // queued there (a late memset of the control words would zero the live count)
  CKC(cudaStreamSynchronize(0));
#undef CKC
  *out = h;
  return QMCB_OK;
}

int qmcb_destroy(qmcb_handle *h)
{
  if (!h) return QMCB_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  void *ptrs[] = {h->d_tbi, h->d_tbL, h->d_tbc, h->d_tbp, h->d_cns, h->d_csexp, h->d_cscoef[0], h->d_cscoef[1], h->d_cpar[0], h->d_cpar[1], h->d_crmax[0],
                  h->d_crmax[1], h->d_docc[0], h->d_docc[1], h->d_dswap[0], h->d_dswap[1], h->d_ci, h->d_ctype, h->d_cparam, h->d_ctf[0], h->d_ctf[1], h->d_pade_ab, h->d_shell, h->d_fn, h->d_xsl, h->d_fq, h->d_pexp, h->d_pcoef, h->d_nuc,   h->d_bf,   h->d_prim,     h->d_ct[0], h->d_ct[1], h->d_pade,   h->d_pade_len,
                  h->d_en[0], h->d_en[1], h->d_state,   h->d_live,  h->d_live_tmp, h->d_free, h->d_ctl,
                  h->d_copies, h->d_stats, h->d_dump, h->d_ectl,   h->d_slots, h->d_R,     h->d_out,    h->d_status,
                  h->d_rows_A, h->d_rows_B[0], h->d_rows_B[1], h->d_rows_rs, h->d_rows_cs[0], h->d_rows_cs[1],
                  h->d_rows_out, h->d_bf_A, h->d_bf_B[0], h->d_bf_B[1]};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : h->done_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->ectl_ev)
    if (e) cudaEventDestroy(e);
  if (h->h_ectl) cudaFreeHost(h->h_ectl);
  if (h->h_stats) cudaFreeHost(h->h_stats);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return QMCB_OK;
}

int qmcb_set_params(qmcb_handle *h, const qmcb_run_params *p)
{
  if (!h || !p) return fail(h, QMCB_E_ARG, "qmcb_set_params: null argument");
  if (!(p->dt > 0)) return fail(h, QMCB_E_ARG, "qmcb_set_params: dt must be positive");
  if (p->qf_modification == QMCB_QF_UMRIGAR93_EQUAL && (p->qf_equal_a > 1 || p->qf_equal_a <= 0))
    return fail(h, QMCB_E_ARG, "qmcb_set_params: umrigar93_equalelectrons_parameter must be in (0, 1]");
  if (p->run_type < 0 || p->run_type > 1 || p->sampling < 0 || p->sampling > 2 || p->qf_modification < 0 ||
      p->qf_modification > 2 || p->energy_modification < 0 || p->energy_modification > 2 || p->reweighting < 0 ||
      p->reweighting > 2 || p->energy_cutoff < 0 || p->energy_cutoff > 2 || p->exact_single_electron_gf < 0 ||
      p->exact_single_electron_gf > 1 || p->dynamic_time_step < 0 || p->dynamic_time_step > 1 ||
      p->walker_deletion < 0 || p->walker_deletion > 1)
    return fail(h, QMCB_E_ARG, "qmcb_set_params: unknown method selector");
  if (p->precision < QMCB_PREC_FP64 || p->precision > QMCB_PREC_BF16X3_TC)
    return fail(h, QMCB_E_ARG, "qmcb_set_params: unknown precision");
  if (h->md && p->precision != QMCB_PREC_FP64)
    return fail(h, QMCB_E_ARG, "qmcb_set_params: several determinants run in FP64 only");
  if (p->precision == QMCB_PREC_INT8_SLICES) {
    const int rc = rows_setup(h);
    if (rc) return rc;
  }
  if (p->precision == QMCB_PREC_BF16_TC || p->precision == QMCB_PREC_BF16X3_TC) {
    const int rc = rows_bf_setup(h);
    if (rc) return rc;
  }
  h->params = *p;
  if (h->n_live_host > 0) {
    // the host's E_T / E_est feed the next steps (QMCManager::updateTrialEnergy)
    // from a pinned slot (a ring of four, so that slots still being read by
    // copies in flight are not rewritten), asynchronous to the host
    const int k = h->ectl_next;
    h->ectl_next = (k + 1) & 3;
    CK(cudaEventSynchronize(h->ectl_ev[k]));  // this slot's previous copy has left it
    EnergyCtl &ec = h->h_ectl[k];
    ec = EnergyCtl{};
    ec.e_trial = p->energy_trial;
    ec.e_est = p->energy_estimated;
    ec.target_weight = p->target_walkers > 0 ? p->target_walkers : h->target_weight;
    ec.pop_control = p->population_control;
    ec.dt_eff = p->dt_effective;
    CK(cudaMemcpyAsync(h->d_ectl, &ec, sizeof(ec), cudaMemcpyHostToDevice, h->stream));
    CK(cudaEventRecord(h->ectl_ev[k], h->stream));
  }
  return QMCB_OK;
}

int qmcb_get_params(const qmcb_handle *h, qmcb_run_params *p)
{
  if (!h || !p) return QMCB_E_ARG;
  *p = h->params;
  return QMCB_OK;
}

int qmcb_num_electrons(const qmcb_handle *h) { return h ? h->N : -1; }
int qmcb_max_walkers(const qmcb_handle *h) { return h ? h->max_walkers : -1; }
void *qmcb_stream(qmcb_handle *h) { return h ? (void *)h->stream : nullptr; }

int qmcb_get_rows(qmcb_handle *h, int num, int *n, double *rows)
{
  if (!h || !n) return QMCB_E_ARG;
  if (h->rows_n == 0) return fail(h, QMCB_E_STATE, "qmcb_get_rows: no single-electron move in a tensor-core rows mode yet");
  *n = h->rows_n;
  if (num < 0 || num > h->rows_num || (num > 0 && !rows)) return fail(h, QMCB_E_ARG, "qmcb_get_rows: bad argument");
  if (num == 0) return QMCB_OK;
  CK(cudaMemcpyAsync(rows, h->d_rows_out, sizeof(double) * 5 * (size_t)h->rows_n * num, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return QMCB_OK;
}

int qmcb_synchronize(qmcb_handle *h)
{
  if (!h) return QMCB_E_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return QMCB_OK;
}

// One launch of the single-determinant full-evaluation / refresh kernel.
static void launch_full(qmcb_handle *h, int cap, cudaStream_t st, const RunCfg &cfg, const int *slots, int num,
                        const int *d_num, const double *R_in, int do_basis, EvalOut o)
{
  // list entries [0, num) (d_num: device count), grid sized for `cap`;
  // the refresh (do_basis = 0) runs with its smaller per-warp scratch
  const int wpb = do_basis ? h->wpb_full : h->wpb_refresh;
  const dim3 g((cap + wpb - 1) / wpb), b(32 * wpb);
  const size_t sm = do_basis ? h->smem_full : h->smem_refresh;
  if (h->params.precision == QMCB_PREC_MIXED) {
    if (h->extras)
      k_full<float, MIXED_TI, true><<<g, b, sm, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num, d_num, R_in, do_basis, o);
    else
      k_full<float, MIXED_TI, false><<<g, b, sm, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num, d_num, R_in, do_basis,
                                                       o);
  } else {
    if (h->extras)
      k_full<double, double, true><<<g, b, sm, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num, d_num, R_in, do_basis, o);
    else
      k_full<double, double, false><<<g, b, sm, st>>>(h->sys, h->lay, cfg, h->d_state, slots, num, d_num, R_in, do_basis,
                                                      o);
  }
}

// Device address of a host array that kernels can store into directly:
// page-locked memory mapped into the device's address space (every
// cudaMallocHost / cudaHostAlloc allocation under unified addressing, and
// cudaHostRegister'd ranges that are mapped); null for pageable memory.
static void *mapped_device_ptr(void *p)
{
  if (!p) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // not a pointer the runtime knows: pageable
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

// Destinations of the evaluate outputs.  The per-electron arrays (grad,
// mod_grad) go straight into the caller's array when that array is
// page-locked and mapped: the kernel's stores of a walker's 3N values cross
// the bus while it runs.  The per-walker values (psi, sign, lap, E_L,
// potentials, status) always go to the handle's device buffer first; after
// the kernel, one k_put_outputs launch moves the ones whose host arrays are
// mapped in full packets, and one copy each brings back the rest (pageable
// arrays).  Outputs not selected are not written at all.
struct EvalDst {
  void *host[8], *dev[8], *kernel[8];
  size_t bytes[8];
  bool mapped[8];
};

static EvalOut eval_destinations(qmcb_handle *h, int num, unsigned mask, double *log_abs_psi, double *sign,
                                 double *grad, double *mod_grad, double *lap, double *e_local, double *pe,
                                 unsigned char *status, EvalDst &d)
{
  const size_t N = h->N;
  double *o_lp = h->d_out, *o_sg = o_lp + num, *o_lap = o_sg + num, *o_el = o_lap + num, *o_pe = o_el + num;
  double *o_g = o_pe + 3 * (size_t)num, *o_mg = o_g + 3 * N * num;
  const unsigned bit[8] = {QMCB_OUT_PSI, QMCB_OUT_PSI, QMCB_OUT_GRAD, QMCB_OUT_MOD_GRAD,
                           QMCB_OUT_LAP, QMCB_OUT_E_LOCAL, QMCB_OUT_PE, QMCB_OUT_STATUS};
  void *host[8] = {log_abs_psi, sign, grad, mod_grad, lap, e_local, pe, status};
  void *dev[8] = {o_lp, o_sg, o_g, o_mg, o_lap, o_el, o_pe, h->d_status};
  const size_t bytes[8] = {sizeof(double) * num, sizeof(double) * num, sizeof(double) * 3 * N * num,
                           sizeof(double) * 3 * N * num, sizeof(double) * num, sizeof(double) * num,
                           sizeof(double) * 3 * num, (size_t)num};
  for (int i = 0; i < 8; i++) {
    d.host[i] = host[i];
    d.dev[i] = dev[i];
    d.bytes[i] = bytes[i];
    d.kernel[i] = nullptr;
    d.mapped[i] = false;
    if ((mask & bit[i]) && host[i]) {
      void *m = mapped_device_ptr(host[i]);
      d.mapped[i] = m != nullptr;
      if (m) d.host[i] = m;
      const bool per_electron = i == 2 || i == 3;
      d.kernel[i] = (m && per_electron) ? m : dev[i];
    }
  }
  return EvalOut{(double *)d.kernel[0], (double *)d.kernel[1], (double *)d.kernel[2], (double *)d.kernel[3],
                 (double *)d.kernel[4], (double *)d.kernel[5], (double *)d.kernel[6], (unsigned char *)d.kernel[7]};
}

// After the kernel (enqueued on st): the mapped per-walker outputs by one
// k_put_outputs launch, the pageable ones by one copy each.
static cudaError_t eval_deliver(const EvalDst &d, cudaStream_t st)
{
  PutList P{};
  int nput = 0;
  size_t most = 0;
  for (int i = 0; i < 8; i++) {
    if (!d.kernel[i] || d.kernel[i] != d.dev[i]) continue;  // not selected, or stored by the kernel
    if (d.mapped[i]) {
      P.src[nput] = d.dev[i];
      P.dst[nput] = d.host[i];
      P.bytes[nput] = d.bytes[i];
      most = std::max(most, d.bytes[i]);
      nput++;
    } else {
      const cudaError_t e = cudaMemcpyAsync(d.host[i], d.dev[i], d.bytes[i], cudaMemcpyDeviceToHost, st);
      if (e != cudaSuccess) return e;
    }
  }
  if (nput > 0) {
    const int blocks = (int)std::min<size_t>((most / 8 + 255) / 256, 64);
    k_put_outputs<<<dim3(std::max(blocks, 1), nput), 256, 0, st>>>(P);
    return cudaGetLastError();
  }
  return cudaSuccess;
}

static int launch_eval(qmcb_handle *h, int which_e, const int *d_slots, int num, const double *d_R, EvalOut o,
                       cudaStream_t st, int rin_moved = 0)
{
  RunCfg cfg = make_cfg(h->params);
  const bool mixed = h->params.precision == QMCB_PREC_MIXED;
  if (h->md) {
    if (mixed) return fail(h, QMCB_E_ARG, "evaluate: several determinants run in FP64 (precision QMCB_PREC_FP64)");
    if (which_e < 0) {
      int blocks = (num + h->wpb_full - 1) / h->wpb_full;
      k_full_md<<<blocks, 32 * h->wpb_full, h->smem_full, st>>>(h->sys, h->lay, cfg, h->d_state, d_slots, num,
                                                                 nullptr, d_R, 1, o);
    } else {
      MoveArgs mv{which_e, 0, 0, 0};
      mv.rin_moved = rin_moved;
      int blocks = (num + h->wpb_move - 1) / h->wpb_move;
      k_move_md<false><<<blocks, 32 * h->wpb_move, h->smem_move, st>>>(h->sys, h->lay, cfg, h->d_state, d_slots,
                                                                        num, nullptr, d_R, mv, h->d_ectl,
                                                                        h->d_stats, o);
    }
    CK(cudaGetLastError());
    if (which_e < 0) h->state_prec = h->params.precision;
    return QMCB_OK;
  }
  if (which_e < 0) {
    launch_full(h, num, st, cfg, d_slots, num, nullptr, d_R, 1, o);
  } else {
    if (h->state_prec != state_kind(h->params.precision))
      return fail(h, QMCB_E_STATE, "evaluate: walker state was written in another precision; evaluate all electrons first");
    MoveArgs mv{which_e, 0, 0, 0};
    mv.rin_moved = rin_moved;
    launch_move<false>(h, num, st, cfg, d_slots, num, nullptr, d_R, mv, o);
  }
  CK(cudaGetLastError());
  if (which_e < 0) h->state_prec = state_kind(h->params.precision);
  return QMCB_OK;
}

int qmcb_evaluate_device(qmcb_handle *h, int which_e, const int *d_slots, int num, const double *d_R,
                         double *d_log_abs_psi, double *d_sign, double *d_grad, double *d_mod_grad, double *d_lap,
                         double *d_e_local, double *d_pe, unsigned char *d_status, void *stream)
{
  if (!h) return QMCB_E_ARG;
  if (num < 0 || num > h->max_walkers || which_e < -1 || which_e >= h->N || !d_R || (num > 0 && !d_slots))
    return fail(h, QMCB_E_ARG, "qmcb_evaluate_device: bad argument");
  if (which_e >= 0 && !h->evaluated_once)
    return fail(h, QMCB_E_STATE, "qmcb_evaluate_device: one-electron update before any full evaluation");
  if (num == 0) return QMCB_OK;
  EvalOut o{d_log_abs_psi, d_sign, d_grad, d_mod_grad, d_lap, d_e_local, d_pe, d_status};
  int rc = launch_eval(h, which_e, d_slots, num, d_R, o, stream ? (cudaStream_t)stream : h->stream);
  if (rc == QMCB_OK && which_e < 0) h->evaluated_once = true;
  return rc;
}

int qmcb_evaluate(qmcb_handle *h, int which_e, const int *slots, int num, const double *R, double *log_abs_psi,
                  double *sign, double *grad, double *mod_grad, double *lap, double *e_local, double *pe,
                  unsigned char *status)
{
  if (!h) return QMCB_E_ARG;
  if (num < 0 || num > h->max_walkers || which_e < -1 || which_e >= h->N || !R || !slots)
    return fail(h, QMCB_E_ARG, "qmcb_evaluate: bad argument");
  for (int i = 0; i < num; i++)
    if (slots[i] < 0 || slots[i] >= h->max_walkers) return fail(h, QMCB_E_ARG, "qmcb_evaluate: slot out of range");
  if (which_e >= 0 && !h->evaluated_once)
    return fail(h, QMCB_E_STATE, "qmcb_evaluate: one-electron update before any full evaluation");
  if (num == 0) return QMCB_OK;
  const int N = h->N;
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(h->d_slots, slots, sizeof(int) * num, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_R, R, sizeof(double) * (size_t)num * 3 * N, cudaMemcpyHostToDevice, st));
  // every non-NULL output is returned
  EvalDst dst;
  const EvalOut o = eval_destinations(h, num, QMCB_OUT_ALL, log_abs_psi, sign, grad, mod_grad, lap, e_local, pe,
                                      status, dst);
  int rc = launch_eval(h, which_e, h->d_slots, num, h->d_R, o, st);
  if (rc) return rc;
  if (which_e < 0) h->evaluated_once = true;
  CK(eval_deliver(dst, st));
  int rows_err = 0;
  if (rows_mode(h->params.precision) && which_e >= 0)
    CK(cudaMemcpyAsync(&rows_err, h->d_ctl + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (rows_err) return fail(h, QMCB_E_CUDA, "qmcb_evaluate: the tensor-core contraction gave up waiting (rows not written)");
  return QMCB_OK;
}

int qmcb_evaluate_moved(qmcb_handle *h, int which_e, const int *slots, int num, const double *r_moved,
                        unsigned out_mask, double *log_abs_psi, double *sign, double *grad, double *mod_grad,
                        double *lap, double *e_local, double *pe, unsigned char *status)
{
  if (!h) return QMCB_E_ARG;
  if (num < 0 || num > h->max_walkers || which_e < 0 || which_e >= h->N || !r_moved || !slots)
    return fail(h, QMCB_E_ARG, "qmcb_evaluate_moved: bad argument");
  for (int i = 0; i < num; i++)
    if (slots[i] < 0 || slots[i] >= h->max_walkers) return fail(h, QMCB_E_ARG, "qmcb_evaluate_moved: slot out of range");
  if (!h->evaluated_once)
    return fail(h, QMCB_E_STATE, "qmcb_evaluate_moved: one-electron update before any full evaluation");
  if (((out_mask & QMCB_OUT_PSI) && (!log_abs_psi || !sign)) || ((out_mask & QMCB_OUT_GRAD) && !grad) ||
      ((out_mask & QMCB_OUT_MOD_GRAD) && !mod_grad) || ((out_mask & QMCB_OUT_LAP) && !lap) ||
      ((out_mask & QMCB_OUT_E_LOCAL) && !e_local) || ((out_mask & QMCB_OUT_PE) && !pe) ||
      ((out_mask & QMCB_OUT_STATUS) && !status))
    return fail(h, QMCB_E_ARG, "qmcb_evaluate_moved: an output selected in out_mask is NULL");
  if (num == 0) return QMCB_OK;
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(h->d_slots, slots, sizeof(int) * num, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_R, r_moved, sizeof(double) * 3 * (size_t)num, cudaMemcpyHostToDevice, st));
  EvalDst dst;
  const EvalOut o = eval_destinations(h, num, out_mask, log_abs_psi, sign, grad, mod_grad, lap, e_local, pe,
                                      status, dst);
  int rc = launch_eval(h, which_e, h->d_slots, num, h->d_R, o, st, 1);
  if (rc) return rc;
  CK(eval_deliver(dst, st));
  int rows_err = 0;
  if (rows_mode(h->params.precision))
    CK(cudaMemcpyAsync(&rows_err, h->d_ctl + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (rows_err) return fail(h, QMCB_E_CUDA, "qmcb_evaluate_moved: the tensor-core contraction gave up waiting");
  return QMCB_OK;
}

int qmcb_alloc_slot(qmcb_handle *h, int *slot)
{
  if (!h || !slot) return QMCB_E_ARG;
  std::lock_guard<std::mutex> lock(h->slot_mu);
  if (h->slot_used.empty()) {
    h->slot_used.assign(h->max_walkers, 0);
    h->slot_free.clear();
    for (int s = h->max_walkers - 1; s >= 0; s--) h->slot_free.push_back(s);
  }
  if (h->slot_free.empty()) return fail(h, QMCB_E_LIMIT, "qmcb_alloc_slot: all max_walkers slots are in use");
  *slot = h->slot_free.back();
  h->slot_free.pop_back();
  h->slot_used[*slot] = 1;
  return QMCB_OK;
}

int qmcb_free_slot(qmcb_handle *h, int slot)
{
  if (!h) return QMCB_E_ARG;
  std::lock_guard<std::mutex> lock(h->slot_mu);
  if (slot < 0 || slot >= h->max_walkers || h->slot_used.empty() || !h->slot_used[slot])
    return fail(h, QMCB_E_ARG, "qmcb_free_slot: slot was not handed out by qmcb_alloc_slot");
  h->slot_used[slot] = 0;
  h->slot_free.push_back(slot);
  return QMCB_OK;
}

int qmcb_init_walkers(qmcb_handle *h, int n, const double *R)
{
  if (!h) return QMCB_E_ARG;
  if (n <= 0 || n > h->max_walkers || !R) return fail(h, QMCB_E_ARG, "qmcb_init_walkers: bad argument");
  cudaStream_t st = h->stream;
  std::vector<int> live(h->max_walkers), fr(h->max_walkers);
  for (int i = 0; i < n; i++) live[i] = i;
  // free stack: popped from the top, so store the highest slots first
  int nf = h->max_walkers - n;
  for (int i = 0; i < nf; i++) fr[i] = h->max_walkers - 1 - i;
  CK(cudaMemcpyAsync(h->d_live, live.data(), sizeof(int) * h->max_walkers, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_free, fr.data(), sizeof(int) * h->max_walkers, cudaMemcpyHostToDevice, st));
  int ctl[4] = {n, nf, 0, 0};
  CK(cudaMemcpyAsync(h->d_ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_R, R, sizeof(double) * (size_t)n * 3 * h->N, cudaMemcpyHostToDevice, st));
  EvalOut o{};
  int rc = launch_eval(h, -1, h->d_live, n, h->d_R, o, st);
  if (rc) return rc;
  h->evaluated_once = true;
  EnergyCtl ec{};
  ec.e_trial = h->params.energy_trial;
  ec.e_est = h->params.energy_estimated;
  ec.target_weight = h->params.target_walkers > 0 ? h->params.target_walkers : n;
  ec.pop_control = h->params.population_control;
  ec.dt_eff = h->params.dt_effective;
  h->target_weight = ec.target_weight;
  CK(cudaMemcpyAsync(h->d_ectl, &ec, sizeof(ec), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(h->d_stats, 0, sizeof(double) * ST_COUNT, st));
  CK(cudaStreamSynchronize(st));
  h->n_live_host = n;
  return QMCB_OK;
}

// Enqueues n_steps Monte Carlo steps and the copy of the step statistics
// into the handle's pinned buffer, then records the completion event.
// dump: device buffer for the configuration records of every step's move
// (each step overwrites it; null: none).
static int enqueue_steps(qmcb_handle *h, int first_step, int n_steps, double *dump = nullptr)
{
  if (n_steps < 0 || first_step < 0) return fail(h, QMCB_E_ARG, "qmcb_run_steps: bad step range");
  if (!h->evaluated_once) return fail(h, QMCB_E_STATE, "qmcb_run_steps: call qmcb_init_walkers first");
  if (h->state_prec != state_kind(h->params.precision))
    return fail(h, QMCB_E_STATE, "qmcb_run_steps: walker state was written in another precision; call qmcb_init_walkers");
  if (h->n_flight >= 2) return fail(h, QMCB_E_STATE, "qmcb_run_steps_async: two batches of steps are already in flight on this handle");
  if (h->n_live_host <= 0) return fail(h, QMCB_E_STATE, "qmcb_run_steps: no live walkers (population died out)");
  cudaStream_t st = h->stream;
  RunCfg cfg = make_cfg(h->params);
  // per-call sums; the running E_est sums persist across calls
  CK(cudaMemsetAsync(h->d_stats, 0, sizeof(double) * ST_RUN_SUM_W, st));
  const int blocks = (h->max_walkers + h->wpb_move - 1) / h->wpb_move;
  const int blocks_full = (h->max_walkers + h->wpb_full - 1) / h->wpb_full;
  const bool dmc = h->params.run_type == QMCB_DMC;
  for (int s = 0; s < n_steps; s++) {
    int step = first_step + s;
    MoveArgs mv;
    mv.e = step % h->N;
    mv.step = step;
    mv.do_reweight = mv.e == 0;
    mv.reweight_on = step >= h->params.reweight_start_step;
    mv.dump = dump;
    EvalOut o{};
    if (h->md) {
      ProfScope ps(h, QMCB_KERNEL_MOVE, st);
      k_move_md<true><<<blocks, 32 * h->wpb_move, h->smem_move, st>>>(h->sys, h->lay, cfg, h->d_state, h->d_live, 0,
                                                                       h->d_ctl, nullptr, mv, h->d_ectl, h->d_stats, o);
      ps.end(st);
    } else {
      launch_move<true>(h, h->max_walkers, st, cfg, h->d_live, 0, h->d_ctl, nullptr, mv, o);
    }
    if (dmc && mv.e == 0) {
      {
        ProfScope ps(h, QMCB_KERNEL_BRANCH, st);
        k_branch<<<1, 1024, 0, st>>>(h->d_state, h->lay, h->d_live, h->d_live_tmp, h->d_free, h->d_ctl,
                                     h->d_copies, h->params.branching_threshold, h->params.fusion_threshold,
                                     h->params.seed, step, h->d_stats, cfg.e_orig, cfg.limit_branching);
        ps.end(st);
      }
      {
        ProfScope ps(h, QMCB_KERNEL_COPY, st);
        k_copy<<<592, 256, 0, st>>>(h->d_state, h->lay, h->d_copies, h->d_ctl);
        ps.end(st);
      }
      {
        ProfScope ps(h, QMCB_KERNEL_ENERGY, st);
        k_energy<<<1, 32, 0, st>>>(h->d_ectl, h->d_stats, 1, cfg.dyn_dt, cfg.dt);
        ps.end(st);
      }
    }
    if (h->params.refresh_interval > 0 && (step + 1) % h->params.refresh_interval == 0) {
      EvalOut o2{};
      ProfScope ps(h, QMCB_KERNEL_REFRESH, st);
      if (h->md)
        k_full_md<<<blocks_full, 32 * h->wpb_full, h->smem_full, st>>>(h->sys, h->lay, cfg, h->d_state, h->d_live, 0,
                                                                        h->d_ctl, nullptr, 0, o2);
      else
        launch_full(h, h->max_walkers, st, cfg, h->d_live, 0, h->d_ctl, nullptr, 0, o2);
      ps.end(st);
    }
  }
  CK(cudaGetLastError());
  const int slot = (h->head + h->n_flight) & 1;
  CK(cudaMemcpyAsync(h->h_stats + slot * ST_COUNT, h->d_stats, sizeof(double) * ST_COUNT, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h->h_ctl + slot * 4, h->d_ctl, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(h->done_ev[slot], st));
  h->n_flight++;
  return QMCB_OK;
}

// Waits for the batch in flight and converts the pinned statistics.
static int finish_steps(qmcb_handle *h, qmcb_step_stats *stats)
{
  if (h->n_flight == 0) return fail(h, QMCB_E_STATE, "qmcb_steps_collect: no batch in flight");
  const int slot = h->head;
  CK(cudaEventSynchronize(h->done_ev[slot]));
  h->head ^= 1;
  h->n_flight--;
  if (h->prof) prof_collect(h);
  const double *sv = h->h_stats + slot * ST_COUNT;
  const int *cv = h->h_ctl + slot * 4;
  h->n_live_host = cv[0];
  if (cv[3]) return fail(h, QMCB_E_CUDA, "qmcb_run_steps: the tensor-core contraction gave up waiting (rows not written)");
  if (stats) {
    stats->sum_weight = sv[ST_SUM_W];
    stats->sum_weight_energy = sv[ST_SUM_WE];
    stats->sum_weight_energy2 = sv[ST_SUM_WE2];
    stats->sum_accept = sv[ST_SUM_ACC];
    stats->n_moves = sv[ST_MOVES];
    stats->final_weight = sv[ST_FINAL_W];
    stats->n_walkers = cv[0];
    stats->n_singular = (int)sv[ST_SINGULAR];
  }
  return QMCB_OK;
}

int qmcb_run_steps(qmcb_handle *h, int first_step, int n_steps, qmcb_step_stats *stats)
{
  if (!h) return QMCB_E_ARG;
  if (h->n_flight) return fail(h, QMCB_E_STATE, "qmcb_run_steps: collect the batches in flight first");
  int rc = enqueue_steps(h, first_step, n_steps);
  if (rc) return rc;
  return finish_steps(h, stats);
}

int qmcb_run_step_configs(qmcb_handle *h, int step, double *records, int capacity, int *n_records,
                          qmcb_step_stats *stats)
{
  if (!h || !records || !n_records) return QMCB_E_ARG;
  const int n = h->n_live_host;
  if (capacity < n) return fail(h, QMCB_E_ARG, "qmcb_run_step_configs: capacity below the live walker count");
  const size_t rec = (size_t)QMCB_CONFIG_RECORD(h->N);
  if (!h->d_dump) CK(cudaMalloc(&h->d_dump, sizeof(double) * 2 * rec * (size_t)h->max_walkers));
  if (h->n_flight) return fail(h, QMCB_E_STATE, "qmcb_run_step_configs: collect the batches in flight first");
  int rc = enqueue_steps(h, step, 1, h->d_dump);
  if (rc) return rc;
  // the walkers that moved are the n live before the step, in list order
  CK(cudaMemcpyAsync(records, h->d_dump, sizeof(double) * 2 * rec * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
  rc = finish_steps(h, stats);
  if (rc) return rc;
  *n_records = 2 * n;
  return QMCB_OK;
}

int qmcb_run_steps_async(qmcb_handle *h, int first_step, int n_steps)
{
  if (!h) return QMCB_E_ARG;
  return enqueue_steps(h, first_step, n_steps);
}

int qmcb_steps_done(qmcb_handle *h)
{
  if (!h) return -QMCB_E_ARG;
  if (h->n_flight == 0) return 1;
  cudaError_t e = cudaEventQuery(h->done_ev[h->head]);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  fail(h, QMCB_E_CUDA, std::string("qmcb_steps_done: ") + cudaGetErrorString(e));
  return -QMCB_E_CUDA;
}

int qmcb_steps_collect(qmcb_handle *h, qmcb_step_stats *stats)
{
  if (!h) return QMCB_E_ARG;
  return finish_steps(h, stats);
}

size_t qmcb_state_bytes(const qmcb_handle *h)
{
  if (!h) return 0;
  size_t b = (size_t)h->max_walkers * h->lay.stride * sizeof(double);
  // the tensor-core rows modes' buffers, once a mode has set them up
  const size_t tiles = (size_t)(h->max_walkers + kTileWalkers - 1) / kTileWalkers;
  if (h->d_rows_out) b += sizeof(double) * (size_t)h->max_walkers * 5 * h->nmax;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? h->sys.nb : h->sys.na;
    const size_t nt = (size_t)std::max((n + kNTile - 1) / kNTile, 1);
    if (h->d_rows_A) b += nt * h->rows_ksteps * (kSlices * kBBlock + kNTile * sizeof(double));
    if (h->d_bf_A) b += nt * h->bf_ksteps * 2 * kBBlock;
  }
  if (h->d_rows_A) b += tiles * h->rows_ksteps * (kSlices * kABlock + kTileRows * sizeof(double));
  if (h->d_bf_A) b += tiles * h->bf_ksteps * 2 * kABlock;
  return b;
}

int qmcb_num_walkers(const qmcb_handle *h) { return h ? h->n_live_host : -1; }

int qmcb_get_walkers(qmcb_handle *h, int n, double *R, double *weight, double *e_local, double *log_abs_psi,
                     double *sign)
{
  if (!h) return QMCB_E_ARG;
  if (n < 0 || n > h->n_live_host) return fail(h, QMCB_E_ARG, "qmcb_get_walkers: n beyond live walkers");
  if (n == 0) return QMCB_OK;
  cudaStream_t st = h->stream;
  const int N = h->N, rec = 3 * N + 4;
  k_gather<<<(n + 3) / 4, 128, 0, st>>>(h->d_state, h->lay, N, h->d_live, n, h->d_out);
  CK(cudaGetLastError());
  std::vector<double> buf((size_t)n * rec);
  CK(cudaMemcpyAsync(buf.data(), h->d_out, sizeof(double) * buf.size(), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int i = 0; i < n; i++) {
    const double *o = buf.data() + (size_t)i * rec;
    if (R) std::memcpy(R + (size_t)i * 3 * N, o, sizeof(double) * 3 * N);
    if (weight) weight[i] = o[3 * N];
    if (e_local) e_local[i] = o[3 * N + 1];
    if (log_abs_psi) log_abs_psi[i] = o[3 * N + 2];
    if (sign) sign[i] = o[3 * N + 3];
  }
  return QMCB_OK;
}

int qmcb_set_walker_weights(qmcb_handle *h, int n, const double *w)
{
  if (!h) return QMCB_E_ARG;
  if (n < 0 || n > h->n_live_host || (n > 0 && !w)) return fail(h, QMCB_E_ARG, "qmcb_set_walker_weights: bad n");
  if (n == 0) return QMCB_OK;
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(h->d_out, w, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  k_set_weights<<<(n + 255) / 256, 256, 0, st>>>(h->d_state, h->lay, h->d_live, n, h->d_out);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return QMCB_OK;
}

int qmcb_branch(qmcb_handle *h, int step, int *n_live)
{
  if (!h) return QMCB_E_ARG;
  if (!h->evaluated_once || h->n_live_host <= 0) return fail(h, QMCB_E_STATE, "qmcb_branch: no live walkers");
  cudaStream_t st = h->stream;
  RunCfg cfg = make_cfg(h->params);
  k_branch<<<1, 1024, 0, st>>>(h->d_state, h->lay, h->d_live, h->d_live_tmp, h->d_free, h->d_ctl, h->d_copies,
                               h->params.branching_threshold, h->params.fusion_threshold, h->params.seed, step,
                               h->d_stats, cfg.e_orig, cfg.limit_branching);
  k_copy<<<592, 256, 0, st>>>(h->d_state, h->lay, h->d_copies, h->d_ctl);
  CK(cudaGetLastError());
  int ctl[4];
  CK(cudaMemcpyAsync(ctl, h->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  h->n_live_host = ctl[0];
  if (n_live) *n_live = ctl[0];
  return QMCB_OK;
}

int qmcb_set_profiling(qmcb_handle *h, int enable)
{
  if (!h) return QMCB_E_ARG;
  h->prof = enable != 0;
  return QMCB_OK;
}

int qmcb_get_kernel_stats(qmcb_handle *h, double *out, int reset)
{
  if (!h || !out) return QMCB_E_ARG;
  for (int k = 0; k < QMCB_KERNEL_COUNT; k++) {
    out[2 * k] = h->prof_ms[k];
    out[2 * k + 1] = h->prof_n[k];
    if (reset) h->prof_ms[k] = h->prof_n[k] = 0.0;
  }
  return QMCB_OK;
}

int qmcb_copy_slot(qmcb_handle *h, int src, int dst)
{
  if (!h) return QMCB_E_ARG;
  if (src < 0 || dst < 0 || src >= h->max_walkers || dst >= h->max_walkers)
    return fail(h, QMCB_E_ARG, "qmcb_copy_slot: slot out of range");
  if (src == dst) return QMCB_OK;
  size_t b = sizeof(double) * h->lay.stride;
  CK(cudaMemcpyAsync(h->d_state + (size_t)dst * h->lay.stride, h->d_state + (size_t)src * h->lay.stride, b,
                     cudaMemcpyDeviceToDevice, h->stream));
  return QMCB_OK;
}

int qmcb_branch_weights_noalloc(const double *d_weight_in, int n, double branching_threshold,
                                double fusion_threshold, uint64_t seed, int step, double *d_weight_out,
                                int *d_parent_out, int *d_n_out, void *stream)
{
  if (n < 0 || (n > 0 && (!d_weight_in || !d_weight_out || !d_parent_out)) || !d_n_out)
    return fail(nullptr, QMCB_E_ARG, "qmcb_branch_weights_noalloc: null buffer or negative n");
  if (n > QMCB_NOALLOC_MAX_WALKERS)
    return fail(nullptr, QMCB_E_LIMIT,
                "qmcb_branch_weights_noalloc: n exceeds QMCB_NOALLOC_MAX_WALKERS (65536)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64)
    return fail(nullptr, QMCB_E_CUDA, std::string("qmcb_branch_weights_noalloc: no CUDA device: ") +
                                          cudaGetErrorString(e));
  void *pw = nullptr, *pi = nullptr;
  {
    // once per device, with that device current: the device addresses of
    // the static scratch arrays (their host-side names are not device addresses)
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_w_addr[dev] || !g_noalloc_i_addr[dev]) {
      e = cudaGetSymbolAddress(&pw, g_noalloc_weight);
      if (e != cudaSuccess)
        return fail(nullptr, QMCB_E_CUDA, std::string("qmcb_branch_weights_noalloc: cudaGetSymbolAddress: ") +
                                              cudaGetErrorString(e));
      e = cudaGetSymbolAddress(&pi, g_noalloc_index);
      if (e != cudaSuccess)
        return fail(nullptr, QMCB_E_CUDA, std::string("qmcb_branch_weights_noalloc: cudaGetSymbolAddress: ") +
                                              cudaGetErrorString(e));
      g_noalloc_w_addr[dev] = pw;
      g_noalloc_i_addr[dev] = pi;
    }
    pw = g_noalloc_w_addr[dev];
    pi = g_noalloc_i_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  k_branch_list<<<1, 1024, 0, st>>>(d_weight_in, n, branching_threshold, fusion_threshold, seed, step, (double *)pw,
                                    (int *)pi, d_weight_out, d_parent_out, d_n_out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(nullptr, QMCB_E_CUDA, std::string("qmcb_branch_weights_noalloc: launch: ") + cudaGetErrorString(e));
  return QMCB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Groups: the walkers of many handles (systems of different sizes) stepped
// by one persistent launch per bucket of similar shared-memory need
// (kernels_group.cuh).  No counterpart in the reference, which runs one
// molecule per process.

struct qmcb_group {
  int device = 0;
  int n_sm = 0, max_optin = 0;  // max_optin: dynamic shared memory a group block may use
  cudaStream_t stream = nullptr;
  std::vector<qmcb_handle *> mem;  // in launch order (extras flag, then per-warp scratch)
  std::vector<int> user;           // mem[i] is the caller's member user[i]
  GroupMember *d_gm = nullptr;
  std::vector<GroupMember> h_gm;
  int *d_counter = nullptr;  // one per bucket
  int cbase = -1;            // first slot of the member table in c_gm (-1: table in global memory)
  struct Bucket {
    int first, count, stride, wpb, grid;
    bool extras, ginv, md;
  };
  std::vector<std::vector<Bucket>> cands;  // launch configurations the tuner tries
  std::vector<double> cost;                // ms per walker-move of each (< 0: not yet timed)
  int chosen = -1;                         // the tuned configuration
  int last = -1;                           // configuration of the last batch
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t fork_ev = nullptr;
  std::vector<cudaStream_t> side;  // one stream per bucket
  std::vector<cudaEvent_t> side_ev;
  // members on tensor-core rows: a step's rows kernels run on the member's
  // own stream, forked from its bucket's stream (step_ev[bucket]) and joined
  // back before the bucket's move kernel (rows_ev[member])
  std::vector<cudaEvent_t> step_ev, rows_ev;
  cudaGraphExec_t gexec = nullptr;  // the last batch's launch sequence
  int g_steps = -1, g_config = -1;
  std::string err;
};

static int gfail(qmcb_group *g, int code, const std::string &msg)
{
  if (g)
    g->err = msg;
  else
    g_create_error = msg;
  return code;
}

#define GK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return gfail(g, QMCB_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));  \
  } while (0)

static bool member_extras(const qmcb_handle *h)
{
  return h->extras || h->params.sampling == QMCB_UMRIGAR93_IMPORTANCE_SAMPLING;
}

// Persistent grid of one bucket: as many blocks as fit on every SM at once.
// The group move kernel for a bucket's flags; cbase >= 0: the group's
// member table sits in c_gm from cbase on.
static const void *group_move_fn(bool extras, bool ginv, bool cst, bool md)
{
  const void *fns[10] = {
      (const void *)k_move_group<false, false, false, false>, (const void *)k_move_group<true, false, false, false>,
      (const void *)k_move_group<false, true, false, false>,  (const void *)k_move_group<true, true, false, false>,
      (const void *)k_move_group<false, false, true, false>,  (const void *)k_move_group<true, false, true, false>,
      (const void *)k_move_group<false, true, true, false>,   (const void *)k_move_group<true, true, true, false>,
      (const void *)k_move_group<true, false, false, true>,   (const void *)k_move_group<true, false, true, true>};
  if (md) return fns[8 + (cst ? 1 : 0)];
  return fns[(extras ? 1 : 0) + (ginv ? 2 : 0) + (cst ? 4 : 0)];
}

// Doubles of shared memory one warp of the member's move kernel uses.
static int member_stride(const qmcb_handle *h) { return (int)(h->smem_move / sizeof(double) / h->wpb_move); }

static cudaError_t launch_group_move_any(const qmcb_group::Bucket &B, cudaStream_t st, const GroupMember *gm, int t,
                                         int *counter, int cbase)
{
  const size_t smem = sizeof(double) * (size_t)B.stride * B.wpb;
  int nm = B.count, stride = B.stride;
  void *args[] = {(void *)&gm, (void *)&nm, (void *)&t, (void *)&stride, (void *)&counter, (void *)&cbase};
  return cudaLaunchKernel(group_move_fn(B.extras, B.ginv, cbase >= 0, B.md), dim3(B.grid), dim3(32 * B.wpb), args,
                          smem, st);
}

// Slots of c_gm per device, handed out to groups at create.
static std::mutex g_const_mu;
static std::vector<std::vector<char>> g_const_used;

static int const_reserve(int device, int n)
{
  std::lock_guard<std::mutex> lock(g_const_mu);
  if ((int)g_const_used.size() <= device) g_const_used.resize(device + 1);
  auto &u = g_const_used[device];
  if (u.empty()) u.assign(kConstMembers, 0);
  for (int b = 0; b + n <= kConstMembers; b++) {
    bool free = true;
    for (int i = b; i < b + n && free; i++) free = !u[i];
    if (free) {
      for (int i = b; i < b + n; i++) u[i] = 1;
      return b;
    }
  }
  return -1;
}

static void const_release(int device, int base, int n)
{
  if (base < 0) return;
  std::lock_guard<std::mutex> lock(g_const_mu);
  auto &u = g_const_used[device];
  for (int i = base; i < base + n; i++) u[i] = 0;
}

static int bucket_grid(qmcb_group *g, bool extras, bool ginv, bool md, int stride, int wpb, int *grid)
{
  int per_sm = 0;
  const size_t smem = sizeof(double) * (size_t)stride * wpb;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, group_move_fn(extras, ginv, g->cbase >= 0, md),
                                                                32 * wpb, smem);
  if (e != cudaSuccess) return gfail(g, QMCB_E_CUDA, std::string("qmcb_group: occupancy: ") + cudaGetErrorString(e));
  if (per_sm < 1) return gfail(g, QMCB_E_LIMIT, "qmcb_group: a member's scratch does not fit one block");
  *grid = per_sm * g->n_sm;
  return QMCB_OK;
}

// The configurations the tuner tries: members in runs of equal extras flag,
// each run one bucket or cut into size classes whose per-warp scratch stays
// within a factor 2, 1.4 or 1.15 of the class's smallest; 4 or 2 warps per block
// (fewer where one block could not hold them).
static int build_candidates(qmcb_group *g)
{
  const int n = (int)g->mem.size();
  std::vector<std::vector<int>> splits;
  for (double ratio : {0.0, 2.0, 1.4, 1.15}) {
    std::vector<int> c;
    int lo = 0;
    for (int i = 1; i < n; i++) {
      const bool run_end = member_extras(g->mem[i]) != member_extras(g->mem[i - 1]) ||
                           g->mem[i]->ginv != g->mem[i - 1]->ginv || g->mem[i]->md != g->mem[i - 1]->md;
      const bool class_end = ratio > 0 && member_stride(g->mem[i]) > ratio * member_stride(g->mem[lo]);
      if (run_end || class_end) {
        c.push_back(i);
        lo = i;
      }
    }
    if (std::find(splits.begin(), splits.end(), c) == splits.end()) splits.push_back(c);
  }
  g->cands.clear();
  for (const auto &c : splits)
    for (int wpb : {4, 2}) {
      std::vector<qmcb_group::Bucket> bs;
      int lo = 0;
      for (size_t j = 0; j <= c.size(); j++) {
        const int hi = j < c.size() ? c[j] : n;
        if (hi <= lo) continue;
        qmcb_group::Bucket b{};
        b.first = lo;
        b.count = hi - lo;
        b.extras = member_extras(g->mem[lo]);
        b.ginv = g->mem[lo]->ginv;
        b.md = g->mem[lo]->md;
        b.stride = 0;
        long long walkers = 0;
        for (int i = lo; i < hi; i++) {
          b.stride = std::max(b.stride, member_stride(g->mem[i]));
          walkers += g->mem[i]->max_walkers;
        }
        b.wpb = std::max(1, std::min<int>(wpb, g->max_optin / (int)(sizeof(double) * b.stride)));
        int rc = bucket_grid(g, b.extras, b.ginv, b.md, b.stride, b.wpb, &b.grid);
        if (rc) return rc;
        // no more warps than the bucket has walkers, so that concurrent
        // buckets leave each other room on the SMs
        b.grid = (int)std::min<long long>(b.grid, (walkers + b.wpb - 1) / b.wpb);
        bs.push_back(b);
        lo = hi;
      }
      g->cands.push_back(bs);
    }
  g->cost.assign(g->cands.size(), -1.0);
  g->chosen = g->cands.size() == 1 ? 0 : -1;
  size_t nb = 0;
  for (const auto &bs : g->cands) nb = std::max(nb, bs.size());
  while (g->side.size() < nb) {
    cudaStream_t s2 = nullptr;
    cudaEvent_t e2 = nullptr;
    GK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    g->side.push_back(s2);
    GK(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
    g->side_ev.push_back(e2);
  }
  return QMCB_OK;
}

// The launches of n_steps steps in configuration c (graph capturable when
// no member refreshes).  Buckets are independent (a member's step depends
// only on its own previous step), so each runs all its steps on a stream of
// its own, forked from and joined back into the group stream.
static int group_enqueue(qmcb_group *g, int c, int n_steps, const int *first_steps, bool refresh)
{
  cudaStream_t st = g->stream;
  const auto &bs = g->cands[c];
  GK(cudaEventRecord(g->fork_ev, st));
  for (size_t b = 0; b < bs.size(); b++) {
    const auto &B = bs[b];
    cudaStream_t sb = g->side[b];
    GK(cudaStreamWaitEvent(sb, g->fork_ev, 0));
    bool dmc = false;
    for (int i = B.first; i < B.first + B.count; i++) dmc |= g->mem[i]->params.run_type == QMCB_DMC;
    const GroupMember *gm = g->d_gm + B.first;
    for (int t = 0; t < n_steps; t++) {
      // members on tensor-core rows: their step's rows first (one prep and
      // one contraction launch per member), each member's on its own stream
      // so that the members' small kernels overlap, joined back into the
      // bucket's stream before its move kernel
      bool forked = false;
      for (int i = B.first; i < B.first + B.count; i++) {
        qmcb_handle *h = g->mem[i];
        if (!rows_mode(h->params.precision)) continue;
        if (!forked) {
          GK(cudaEventRecord(g->step_ev[b], sb));
          forked = true;
        }
        GK(cudaStreamWaitEvent(h->stream, g->step_ev[b], 0));
        MoveArgs mv;
        mv.step = first_steps[g->user[i]] + t;
        mv.e = mv.step % h->N;
        mv.do_reweight = mv.e == 0;
        mv.reweight_on = mv.step >= h->params.reweight_start_step;
        mv.dump = nullptr;
        launch_rows<true>(h, h->max_walkers, h->stream, make_cfg(h->params), h->d_live, 0, h->d_ctl, nullptr, mv,
                          member_extras(h), false);
        GK(cudaEventRecord(g->rows_ev[i], h->stream));
        GK(cudaStreamWaitEvent(sb, g->rows_ev[i], 0));
      }
      GK(cudaMemsetAsync(g->d_counter + b, 0, sizeof(int), sb));
      GK(launch_group_move_any(B, sb, gm, t, g->d_counter + b, g->cbase >= 0 ? g->cbase + B.first : -1));
      if (dmc) {
        k_branch_group<<<B.count, 1024, 0, sb>>>(gm, t);
        k_copy_group<<<dim3(64, B.count), 256, 0, sb>>>(gm, t);
        k_energy_group<<<(B.count + 127) / 128, 128, 0, sb>>>(gm, B.count, t);
      }
      if (refresh) {
        for (int i = B.first; i < B.first + B.count; i++) {
          qmcb_handle *h = g->mem[i];
          const int step = first_steps[g->user[i]] + t;
          if (h->params.refresh_interval > 0 && (step + 1) % h->params.refresh_interval == 0) {
            EvalOut o2{};
            const int blocks_full = (h->max_walkers + h->wpb_full - 1) / h->wpb_full;
            if (h->md)
              k_full_md<<<blocks_full, 32 * h->wpb_full, h->smem_full, sb>>>(h->sys, h->lay, make_cfg(h->params),
                                                                              h->d_state, h->d_live, 0, h->d_ctl,
                                                                              nullptr, 0, o2);
            else
              launch_full(h, h->max_walkers, sb, make_cfg(h->params), h->d_live, 0, h->d_ctl, nullptr, 0, o2);
          }
        }
      }
    }
    GK(cudaEventRecord(g->side_ev[b], sb));
    GK(cudaStreamWaitEvent(st, g->side_ev[b], 0));
  }
  GK(cudaGetLastError());
  return QMCB_OK;
}

extern "C" {

int qmcb_group_create(qmcb_handle *const *members, int n, qmcb_group **out)
{
  if (!members || !out || n <= 0) return gfail(nullptr, QMCB_E_ARG, "qmcb_group_create: bad argument");
  if (n > kGroupMax) return gfail(nullptr, QMCB_E_LIMIT, "qmcb_group_create: more than 512 members");
  *out = nullptr;
  for (int i = 0; i < n; i++) {
    const qmcb_handle *h = members[i];
    if (!h) return gfail(nullptr, QMCB_E_ARG, "qmcb_group_create: null member");
    if (h->device != members[0]->device)
      return gfail(nullptr, QMCB_E_ARG, "qmcb_group_create: members on different devices");
    for (int j = 0; j < i; j++)
      if (members[j] == h) return gfail(nullptr, QMCB_E_ARG, "qmcb_group_create: a handle appears twice");
  }
  qmcb_group *g = new qmcb_group();
  g->device = members[0]->device;
  cudaSetDevice(g->device);
  cudaDeviceGetAttribute(&g->n_sm, cudaDevAttrMultiProcessorCount, g->device);
  cudaDeviceGetAttribute(&g->max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, g->device);
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
    if (members[a]->md != members[b]->md) return !members[a]->md;
    const bool ea = member_extras(members[a]), eb = member_extras(members[b]);
    if (ea != eb) return !ea;
    if (members[a]->ginv != members[b]->ginv) return !members[a]->ginv;
    return member_stride(members[a]) < member_stride(members[b]);
  });
  for (int i : idx) {
    g->mem.push_back(members[i]);
    g->user.push_back(i);
  }
  int rc = QMCB_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_gm, sizeof(GroupMember) * n);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_counter, sizeof(int) * (n + 1));
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev1);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork_ev, cudaEventDisableTiming);
  // the group kernels hold the member prefix sums in static shared memory:
  // the dynamic part may use the rest of the opt-in maximum
  g->cbase = const_reserve(g->device, n);
  const void *fns[10];
  for (int k = 0; k < 8; k++) fns[k] = group_move_fn(k & 1, k & 2, k & 4, false);
  fns[8] = group_move_fn(true, false, false, true);
  fns[9] = group_move_fn(true, false, true, true);
  size_t stat = 0;
  for (const void *fn : fns) {
    cudaFuncAttributes fa{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
    stat = std::max(stat, fa.sharedSizeBytes);
  }
  if (e == cudaSuccess) g->max_optin -= (int)stat;
  for (const void *fn : fns)
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, g->max_optin);
  if (e != cudaSuccess) rc = gfail(nullptr, QMCB_E_CUDA, std::string("qmcb_group_create: ") + cudaGetErrorString(e));
  if (!rc) {
    rc = build_candidates(g);
    if (rc) g_create_error = g->err;
  }
  if (rc) {
    qmcb_group_destroy(g);
    return rc;
  }
  *out = g;
  return QMCB_OK;
}

int qmcb_group_destroy(qmcb_group *g)
{
  if (!g) return QMCB_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  const_release(g->device, g->cbase, (int)g->mem.size());
  if (g->gexec) cudaGraphExecDestroy(g->gexec);
  if (g->d_gm) cudaFree(g->d_gm);
  if (g->d_counter) cudaFree(g->d_counter);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (g->fork_ev) cudaEventDestroy(g->fork_ev);
  for (cudaEvent_t e : g->side_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : g->step_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : g->rows_ev) cudaEventDestroy(e);
  for (cudaStream_t s2 : g->side) {
    cudaStreamSynchronize(s2);
    cudaStreamDestroy(s2);
  }
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return QMCB_OK;
}

const char *qmcb_group_last_error(const qmcb_group *g) { return g ? g->err.c_str() : g_create_error.c_str(); }

int qmcb_group_run_steps(qmcb_group *g, const int *first_steps, int n_steps, qmcb_step_stats *stats)
{
  if (!g || !first_steps || n_steps < 0) return gfail(g, QMCB_E_ARG, "qmcb_group_run_steps: bad argument");
  const int nm = (int)g->mem.size();
  bool refresh = false, rows_members = false;
  for (int i = 0; i < nm; i++) {
    qmcb_handle *h = g->mem[i];
    const std::string who = "qmcb_group_run_steps: member " + std::to_string(g->user[i]);
    if (first_steps[g->user[i]] < 0) return gfail(g, QMCB_E_ARG, who + ": negative first step");
    if (!h->evaluated_once) return gfail(g, QMCB_E_STATE, who + ": call qmcb_init_walkers first");
    if (h->n_flight) return gfail(g, QMCB_E_STATE, who + ": a batch of steps is in flight on its handle");
    if ((h->params.precision != QMCB_PREC_FP64 && !rows_mode(h->params.precision)) || h->state_prec != QMCB_PREC_FP64)
      return gfail(g, QMCB_E_ARG, who + ": groups step FP64 walkers (FP64 or tensor-core orbital rows) only");
    if (h->md && h->params.precision != QMCB_PREC_FP64)
      return gfail(g, QMCB_E_ARG, who + ": several determinants run in FP64 only");
    refresh |= h->params.refresh_interval > 0;
    // the rows kernels take the step number as an argument: no graph replay
    rows_members |= rows_mode(h->params.precision);
  }
  cudaSetDevice(g->device);
  // members' tables, parameters and step numbers
  g->h_gm.assign(nm, GroupMember{});
  for (int i = 0; i < nm; i++) {
    qmcb_handle *h = g->mem[i];
    GroupMember &G = g->h_gm[i];
    const bool rows = rows_mode(h->params.precision);
    G.S = h->sys;
    G.L = rows ? h->lay_rows : h->lay;  // the move kernel on rows needs no basis scratch
    G.rows = rows ? h->d_rows_out : nullptr;
    G.cfg = make_cfg(h->params);
    G.state = h->d_state;
    G.live = h->d_live;
    G.live_tmp = h->d_live_tmp;
    G.free_stack = h->d_free;
    G.ctl = h->d_ctl;
    G.copies = h->d_copies;
    G.ectl = h->d_ectl;
    G.stats = h->d_stats;
    G.step0 = first_steps[g->user[i]];
    G.reweight_start = h->params.reweight_start_step;
    G.dmc = h->params.run_type == QMCB_DMC;
    G.limit_branching = h->params.limit_branching;
    G.thr_split = h->params.branching_threshold;
    G.thr_fuse = h->params.fusion_threshold;
  }
  cudaStream_t st = g->stream;
  if (rows_members && g->rows_ev.empty()) {
    size_t nb = 0;
    for (const auto &cand : g->cands) nb = std::max(nb, cand.size());
    g->step_ev.assign(nb, nullptr);
    g->rows_ev.assign(nm, nullptr);
    for (auto &e : g->step_ev) GK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : g->rows_ev) GK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  // the members' own streams finish first (their last evaluate or copy)
  for (auto *h : g->mem) GK(cudaStreamSynchronize(h->stream));
  GK(cudaMemcpyAsync(g->d_gm, g->h_gm.data(), sizeof(GroupMember) * nm, cudaMemcpyHostToDevice, st));
  if (g->cbase >= 0)
    GK(cudaMemcpyToSymbolAsync(c_gm, g->h_gm.data(), sizeof(GroupMember) * nm, sizeof(GroupMember) * g->cbase,
                               cudaMemcpyHostToDevice, st));
  for (auto *h : g->mem) GK(cudaMemsetAsync(h->d_stats, 0, sizeof(double) * ST_RUN_SUM_W, st));
  // configuration: the tuned one, else the next one not yet timed
  int c = g->chosen;
  if (c < 0)
    for (size_t k = 0; k < g->cost.size(); k++)
      if (g->cost[k] < 0) {
        c = (int)k;
        break;
      }
  GK(cudaEventRecord(g->ev0, st));
  if (!refresh && !rows_members && n_steps > 0) {
    if (!(g->gexec && g->g_steps == n_steps && g->g_config == c)) {
      if (g->gexec) {
        cudaGraphExecDestroy(g->gexec);
        g->gexec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      GK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int rc = group_enqueue(g, c, n_steps, first_steps, false);
      cudaError_t ec = cudaStreamEndCapture(st, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ec != cudaSuccess) return gfail(g, QMCB_E_CUDA, std::string("qmcb_group_run_steps: capture: ") + cudaGetErrorString(ec));
      ec = cudaGraphInstantiate(&g->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ec != cudaSuccess) {
        g->gexec = nullptr;
        return gfail(g, QMCB_E_CUDA, std::string("qmcb_group_run_steps: instantiate: ") + cudaGetErrorString(ec));
      }
      g->g_steps = n_steps;
      g->g_config = c;
    }
    GK(cudaGraphLaunch(g->gexec, st));
  } else {
    int rc = group_enqueue(g, c, n_steps, first_steps, refresh);
    if (rc) return rc;
  }
  GK(cudaEventRecord(g->ev1, st));
  for (auto *h : g->mem) {
    GK(cudaMemcpyAsync(h->h_stats, h->d_stats, sizeof(double) * ST_COUNT, cudaMemcpyDeviceToHost, st));
    GK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  }
  GK(cudaStreamSynchronize(st));
  g->last = c;
  for (int i = 0; i < nm; i++)
    if (g->mem[i]->h_ctl[3])
      return gfail(g, QMCB_E_CUDA, "qmcb_group_run_steps: member " + std::to_string(g->user[i]) +
                                       ": the tensor-core contraction gave up waiting (rows not written)");
  double moves = 0.0;
  for (int i = 0; i < nm; i++) {
    qmcb_handle *h = g->mem[i];
    const double *sv = h->h_stats;
    h->n_live_host = h->h_ctl[0];
    moves += sv[ST_MOVES];
    if (stats) {
      qmcb_step_stats &s = stats[g->user[i]];
      s.sum_weight = sv[ST_SUM_W];
      s.sum_weight_energy = sv[ST_SUM_WE];
      s.sum_weight_energy2 = sv[ST_SUM_WE2];
      s.sum_accept = sv[ST_SUM_ACC];
      s.n_moves = sv[ST_MOVES];
      s.final_weight = sv[ST_FINAL_W];
      s.n_walkers = h->h_ctl[0];
      s.n_singular = (int)sv[ST_SINGULAR];
    }
  }
  if (g->chosen < 0 && moves > 0) {
    float ms = 0.0f;
    GK(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    g->cost[c] = ms / moves;
    bool done = true;
    for (double v : g->cost) done &= v >= 0;
    if (done) g->chosen = (int)(std::min_element(g->cost.begin(), g->cost.end()) - g->cost.begin());
  }
  return QMCB_OK;
}

int qmcb_group_config(const qmcb_group *g, int *n_configs, int *chosen, int *last, int *n_buckets, int *wpb)
{
  if (!g) return QMCB_E_ARG;
  if (n_configs) *n_configs = (int)g->cands.size();
  if (chosen) *chosen = g->chosen;
  if (last) *last = g->last;
  const int c = g->last >= 0 ? g->last : (g->chosen >= 0 ? g->chosen : 0);
  if (n_buckets) *n_buckets = (int)g->cands[c].size();
  if (wpb) *wpb = g->cands[c].empty() ? 0 : g->cands[c][0].wpb;
  return QMCB_OK;
}

int qmcb_group_set_config(qmcb_group *g, int config)
{
  if (!g) return QMCB_E_ARG;
  if (config < -1 || config >= (int)g->cands.size()) return gfail(g, QMCB_E_ARG, "qmcb_group_set_config: no such configuration");
  if (config == -1) {
    g->cost.assign(g->cands.size(), -1.0);
    g->chosen = -1;
  } else {
    g->chosen = config;
  }
  return QMCB_OK;
}

}  // extern "C"
