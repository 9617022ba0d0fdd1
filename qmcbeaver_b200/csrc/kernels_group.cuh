// kernels_group.cuh -- the single-electron step of many systems in one launch.
//
// Walkers of systems of different sizes (each system a qmcb_handle with its
// own tables, walker blocks and live list) are processed by one persistent
// kernel: every warp takes the next walker of the flattened list
// (member, walker) from an atomic counter and runs move_walker with that
// member's tables, so small and large systems share the SMs without a
// launch per system.  The members of one launch share the per-warp shared
// memory slice (the largest member's); the host groups members of similar
// slice size into separate launches (buckets) and picks the bucketing and
// the warps per block by timing.  DMC members branch in group launches too
// (one block per member, doing nothing on steps that do not move electron 0),
// so a batch of steps is a fixed launch sequence that is captured once as a
// CUDA graph and replayed.
#pragma once

namespace qmcb {

constexpr int kGroupMax = 512;  // members of one group

struct GroupMember {
  DevSys S;
  Layout L;
  RunCfg cfg;
  double *state;
  int *live, *live_tmp, *free_stack, *ctl;
  int2 *copies;
  EnergyCtl *ectl;
  double *stats;
  int step0;           // the member's step number at step offset 0
  int reweight_start;  // reweight_start_step
  int dmc;
  int limit_branching;
  double thr_split, thr_fuse;
  const double *rows;  // tensor-core rows modes: the step's orbital rows (null: FP64 basis and contraction)
};

// Member tables of groups that fit (kConst launches): read through the
// constant cache with warp-uniform indices; groups that do not fit read
// their table from global memory.
constexpr int kConstMembers = 84;
__constant__ GroupMember c_gm[kConstMembers];

__device__ __forceinline__ int group_step(const GroupMember &G, int t) { return G.step0 + t; }

// Largest m with prefix[m] <= i (members without live walkers have equal
// prefixes and are skipped).
__device__ __forceinline__ int group_find(const int *prefix, int nm, int i)
{
  int lo = 0, hi = nm - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// One Metropolis / DMC step (step offset t) of every live walker of the
// members gm[0..nm) (kConst: c_gm[cbase .. cbase + nm)); stride: doubles of
// shared memory per warp (at least every member's L.mv_stride); *counter is
// zero at launch.
// kMD: the members have several determinants (md_move_walker).
template <bool kExtras, bool kGInv, bool kConst, bool kMD>
__global__ void __launch_bounds__(128, (kMD || kGInv) ? 3 : 5) k_move_group(const GroupMember *__restrict__ gm, int nm, int t,
                                                              int stride, int *counter, int cbase)
{
  extern __shared__ double smem[];
  __shared__ int prefix[kGroupMax + 1];
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int m = 0; m < nm; m++) {
      prefix[m] = acc;
      acc += kConst ? *c_gm[cbase + m].ctl : *gm[m].ctl;
    }
    prefix[nm] = acc;
  }
  __syncthreads();
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  double *sm = smem + (size_t)warp * stride;
  const int total = prefix[nm];
  // the first walker of every warp by its place in the grid, the rest from
  // the counter; the next index is claimed when a walker starts, so the
  // atomic's round trip overlaps the move
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  int i = blockIdx.x * (blockDim.x >> 5) + warp;
  for (;; ) {
    if (i >= total) break;
    int nx = 0;
    if (lane == 0) nx = nwarps + atomicAdd(counter, 1);
    const int m = group_find(prefix, nm, i);
    const GroupMember &G = kConst ? c_gm[cbase + m] : gm[m];
    MoveArgs mv;
    mv.step = group_step(G, t);
    mv.e = mv.step % G.S.N;
    mv.do_reweight = mv.e == 0;
    mv.reweight_on = mv.step >= G.reweight_start;
    mv.dump = nullptr;
    mv.rows = G.rows;
    if constexpr (kMD)
      md_move_walker<true>(G.S, G.L, G.cfg, G.state, G.live, i - prefix[m], sm, nullptr, mv, G.ectl, G.stats,
                           EvalOut{});
    else
      move_walker<true, double, double, kExtras, kGInv>(G.S, G.L, G.cfg, G.state, G.live, i - prefix[m], sm, nullptr,
                                                        mv, G.ectl, G.stats, EvalOut{});
    __syncwarp();
    i = __shfl_sync(QMCB_FULL_MASK, nx, 0);
  }
}

// Branching of the DMC members whose step t moved electron 0: block m for
// member m (QMCRun::nonunitWeightBranching, as k_branch).
__global__ void __launch_bounds__(1024) k_branch_group(const GroupMember *__restrict__ gm, int t)
{
  const GroupMember &G = gm[blockIdx.x];
  if (!G.dmc || group_step(G, t) % G.S.N != 0) return;
  branch_block(G.state, G.L, G.live, G.live_tmp, G.free_stack, G.ctl, G.copies, G.thr_split, G.thr_fuse, G.cfg.seed,
               group_step(G, t), G.stats, G.cfg.e_orig, G.limit_branching);
}

// Walker copies of those branchings: blockIdx.y = member.
__global__ void k_copy_group(const GroupMember *__restrict__ gm, int t)
{
  const GroupMember &G = gm[blockIdx.y];
  if (!G.dmc || group_step(G, t) % G.S.N != 0) return;
  copy_blocks(G.state, G.L, G.copies, G.ctl, blockIdx.x, gridDim.x);
}

// Trial energies of those members: thread m for member m.
__global__ void k_energy_group(const GroupMember *__restrict__ gm, int nm, int t)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  const GroupMember &G = gm[m];
  if (!G.dmc || group_step(G, t) % G.S.N != 0) return;
  update_energy(G.ectl, G.stats, 1, G.cfg.dyn_dt, G.cfg.dt);
}

}  // namespace qmcb
