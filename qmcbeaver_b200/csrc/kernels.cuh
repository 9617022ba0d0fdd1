// kernels.cuh -- the walker-path kernels (sm_100a, FP64 parity arithmetic).
//
// One warp owns one walker for the duration of a kernel; several warps (one
// walker each) share a CTA.  Per-warp scratch lives in dynamic shared
// memory; per-walker state lives in HBM as one contiguous block per slot.
//
//   k_full      full evaluation (whichE = -1) or LU refresh of stored Slater
//               values; QMCSCFJastrow::evaluate with all electrons
//   k_move      one single-electron move of every walker: proposal (or the
//               caller's position), basis + orbital rows, Sherman-Morrison
//               inverse update, ratio sums, incremental Jastrow and
//               potential, psi quantities, Metropolis test, DMC reweight and
//               observables, commit on accept
//   k_branch    nonunit-weight branching of the live list (single CTA)
//   k_copy      state copies for split walkers
//   k_energy    E_est / E_T update after a branching step
#pragma once

#include "device_common.cuh"

namespace qmcb {

// Output pointers of the evaluate entry points (device memory, may be null).
struct EvalOut {
  double *log_abs_psi, *sign, *grad, *mgrad, *lap, *e_local, *pe;
  unsigned char *status;
};

// Device accumulators of one qmcb_run_steps call.
enum StatIdx {
  ST_SUM_W = 0,
  ST_SUM_WE,
  ST_SUM_WE2,
  ST_SUM_ACC,
  ST_MOVES,
  ST_FINAL_W,
  ST_SINGULAR,
  ST_RUN_SUM_W,   // running sums for E_est (kept across calls)
  ST_RUN_SUM_WE,
  ST_RUN_COUNT,   // samples in the running sums
  ST_RUN_SUM_WPD2,  // running sums of w p dR^2 and w dR^2 for the effective time step
  ST_RUN_SUM_WD2,
  ST_COUNT
};

// E_T, E_est, population target (device copies so device-side updates are
// seen by the following launches without a host round trip).
struct EnergyCtl {
  double e_trial, e_est, target_weight, pop_control;
  double dt_eff;  // effective time step of the reweighting (RunCfg::dyn_dt)
};

// Shared-memory doubles needed by one warp.
constexpr int kPart = 160;  // 5 quantities x 32 lanes of slice partial sums
// rows of the HBM-kept inverse per load batch of its update (eight orbitals'
// 48 loads in flight per lane; 168 registers, no spills)
constexpr int kGInvBatch = 8;

// Loads and stores of the HBM-kept inverse with an L2 eviction policy (FP64
// elements; other element types plain).
template <typename T>
__device__ __forceinline__ T ginv_ld(const T *p, uint64_t pol)
{
  if constexpr (sizeof(T) == 8) return ld_l2hint((const double *)p, pol);
  else return *p;
}
template <typename T>
__device__ __forceinline__ void ginv_st(T *p, T v, uint64_t pol)
{
  if constexpr (sizeof(T) == 8) st_l2hint((double *)p, v, pol);
  else *p = v;
}
// Move-kernel scratch per warp (sizes in Layout::mv_*, set by the host):
// region A holds the basis values chi[5][K]; once the contraction has
// consumed them it is reused for the slice partial sums and the new drift /
// modified drift; then the new rows, the Sherman-Morrison factors, and the
// staged copies of the walker's positions, per-electron arrays and the moved
// spin's derivative rows and inverse.
__host__ __device__ inline int even(int x) { return (x + 1) & ~1; }
__host__ __device__ inline int move_region_a(int N, int K) { return even(max(5 * K, kPart + 6 * N)); }
// k_full: chi [5][K + 1], new rows [5][nmax], the matrix inverted in place
// [nmax][nmax], pivot scales, pivot rows, saved pivot column [nmax] each,
// positions [3N].
__host__ __device__ inline int full_scratch_doubles(int N, int K, int nmax)
{
  return even(5 * (K + 1) + 5 * nmax + nmax * nmax + 3 * nmax + 3 * N + kPart + 8);
}
// The refresh of stored Slater values (k_full with do_basis = 0) needs no
// basis rows and no new-row space: a smaller per-warp scratch, more warps per SM.
__host__ __device__ inline int refresh_scratch_doubles(int N, int nmax)
{
  return even(nmax * nmax + 3 * nmax + 3 * N + kPart + 8);
}

// ------------------------------------------------------------------------
// Modified quantum force, QMCSCFJastrow::calculate_Modified_Grad_PsiRatio
// (QMcBeaver/src/QMCSCFJastrow.cpp:329-472).  gr, mg, R: [N][3] (shared).
// Returns |mg| / |gr|; sets *bad when the reference flags the walker singular.
__device__ inline double qf_modify_warp(const DevSys &S, const RunCfg &cfg, const double *R, const double *gr,
                                        double *mg, bool *bad)
{
  const int lane = lane_id(), N = S.N;
  if (cfg.qf_mod == 1) {
    double part = 0.0;
    for (int t = lane; t < 3 * N; t += 32) part += gr[t] * gr[t];
    double magsq = warp_sum(part);
    double a = cfg.qf_a;
    double factor = (-1.0 + sqrt(1.0 + 2 * a * magsq * cfg.dt)) / (a * magsq * cfg.dt);
    for (int t = lane; t < 3 * N; t += 32) mg[t] = gr[t] * factor;
  } else if (cfg.qf_mod == 2) {
    for (int i = lane; i < N; i += 32) {
      // closest nucleus (QMCMolecule::findClosestNucleusIndex): smallest
      // distance, first index on ties -- compared on squared distances
      int cn = 0;
      double cd = 1e300;
      for (int A = 0; A < S.M; A++) {
        double4 P = S.nuc[A];
        double dx = R[3 * i] - P.x, dy = R[3 * i + 1] - P.y, dz = R[3 * i + 2] - P.z;
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < cd) {
          cd = d2;
          cn = A;
        }
      }
      double4 P = S.nuc[cn];
      double nv[3] = {R[3 * i] - P.x, R[3 * i + 1] - P.y, R[3 * i + 2] - P.z};
      double d2 = nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
      double il = rsqrt(d2);
      double ev[3] = {gr[3 * i], gr[3 * i + 1], gr[3 * i + 2]};
      double ev2 = ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2];
      double sc = fabs(ev2) < 1e-10 ? 0.0 : rsqrt(ev2);
      double dotp = 0.0;
      for (int x = 0; x < 3; x++) dotp += (nv[x] * il) * (ev[x] * sc);
      double temp = P.w * P.w * d2;
      double a = 0.5 * (1.0 + dotp) + temp / (10.0 * (4.0 + temp));
      double factor = fabs(ev2) < 1e-10 ? 1.0 : (-1.0 + sqrt(1.0 + 2.0 * a * ev2 * cfg.dt)) / (a * ev2 * cfg.dt);
      for (int x = 0; x < 3; x++) mg[3 * i + x] = gr[3 * i + x] * factor;
    }
  } else {
    for (int t = lane; t < 3 * N; t += 32) mg[t] = gr[t];
  }
  __syncwarp();
  double pm = 0.0, pu = 0.0;
  for (int t = lane; t < 3 * N; t += 32) {
    pm += mg[t] * mg[t];
    pu += gr[t] * gr[t];
  }
  double lm = sqrt(warp_sum(pm)), lu = sqrt(warp_sum(pu));
  double ratio = lm / lu;
  if (isnan(lm) || isnan(lu) || isnan(ratio) || lu == 0.0) *bad = true;
  return ratio;
}

// ------------------------------------------------------------------------
// Warp LU with the reference's implicitly scaled partial pivoting
// (Array2D::ludcmp, QMcBeaver/include/Array2D.h:1204-1340) and the inverse
// by forward / back substitution of the identity (lubksb :1352-1421).
// A: [n][n] row-major (destroyed), X: [n][n] receives A^-1 in X[o][e],
// vv / piv scratch of n doubles.  Returns false when singular.
__device__ inline bool lu_inverse_warp(double *A, double *X, double *vv, double *piv, int n, double &logdet,
                                       double &sign)
{
  const int lane = lane_id();
  bool sing = false;
  for (int i = lane; i < n; i += 32) {
    double big = 0.0;
    for (int j = 0; j < n; j++) big = fmax(big, fabs(A[i * n + j]));
    if (big == 0.0) sing = true;
    vv[i] = big == 0.0 ? 0.0 : 1.0 / big;
  }
  sing = __any_sync(QMCB_FULL_MASK, sing);
  __syncwarp();
  if (sing) {
    logdet = -INFINITY;
    sign = 0.0;
    return false;
  }
  double sg = 1.0, ld = 0.0;
  for (int j = 0; j < n; j++) {
    double best = -1.0;
    int bi = -1;
    for (int i = j + lane; i < n; i += 32) {
      double v = vv[i] * fabs(A[i * n + j]);
      if (v >= best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(QMCB_FULL_MASK, best, o);
      int oi = __shfl_xor_sync(QMCB_FULL_MASK, bi, o);
      if (ob > best || (ob == best && oi > bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (bi != j) {
      for (int k = lane; k < n; k += 32) {
        double t = A[bi * n + k];
        A[bi * n + k] = A[j * n + k];
        A[j * n + k] = t;
      }
      __syncwarp();
      if (lane == 0) vv[bi] = vv[j];
      sg = -sg;
    }
    if (lane == 0) piv[j] = (double)bi;
    __syncwarp();
    double p = A[j * n + j];
    if (p == 0.0) {
      sing = true;
      break;
    }
    double dum = 1.0 / p;
    ld += log(fabs(p));
    if (p < 0) sg = -sg;
    for (int i = j + 1 + lane; i < n; i += 32) A[i * n + j] *= dum;
    __syncwarp();
    // trailing update, element t = (i, c) of the (n-j-1)^2 block on lane
    // t mod 32; the position advances by 32 elements without a division
    const int m = n - j - 1;
    if (m > 0) {
      const int q32 = 32 / m, r32 = 32 - q32 * m;
      int i = lane / m, c = lane - i * m;
      for (int t = lane; t < m * m; t += 32) {
        A[(j + 1 + i) * n + j + 1 + c] -= A[(j + 1 + i) * n + j] * A[j * n + j + 1 + c];
        c += r32;
        i += q32;
        if (c >= m) {
          c -= m;
          i++;
        }
      }
    }
    __syncwarp();
  }
  if (sing) {
    logdet = -INFINITY;
    sign = 0.0;
    return false;
  }
  logdet = ld;
  sign = sg;
  // inverse: column jc of X solves A x = e_jc
  for (int jc = lane; jc < n; jc += 32) {
    for (int i = 0; i < n; i++) X[i * n + jc] = (i == jc) ? 1.0 : 0.0;
    for (int i = 0; i < n; i++) {
      int ip = (int)piv[i];
      double s = X[ip * n + jc];
      X[ip * n + jc] = X[i * n + jc];
      for (int k = 0; k < i; k++) s -= A[i * n + k] * X[k * n + jc];
      X[i * n + jc] = s;
    }
    for (int i = n - 1; i >= 0; i--) {
      double s = X[i * n + jc];
      for (int k = i + 1; k < n; k++) s -= A[i * n + k] * X[k * n + jc];
      X[i * n + jc] = s / A[i * n + i];
    }
  }
  __syncwarp();
  return true;
}

// Warp Gauss-Jordan inverse in place, with the pivot rule of the
// reference's LU (implicitly scaled partial pivoting, Array2D::ludcmp,
// QMcBeaver/include/Array2D.h:1204-1340): the rows below the diagonal of
// column j hold the same Schur complement in both eliminations, so the
// pivots, ln|det| and the sign are the LU's.  Every step updates all rows
// (lanes own columns, rows streamed with independent FMAs) instead of the
// LU's two triangular solves per column, whose FMAs form one dependent
// chain per lane; one n x n array instead of two.  A: [n][n] row-major,
// receives A^-1 in A[o][e] (the layout of lu_inverse_warp's X); vv, piv,
// col: n doubles of scratch each.  Returns false when singular.
__device__ inline bool gj_inverse_warp(double *A, double *vv, double *piv, double *col, int n, double &logdet,
                                       double &sign)
{
  const int lane = lane_id();
  bool sing = false;
  for (int i = lane; i < n; i += 32) {
    double big = 0.0;
    for (int j = 0; j < n; j++) big = fmax(big, fabs(A[i * n + j]));
    if (big == 0.0) sing = true;
    vv[i] = big == 0.0 ? 0.0 : 1.0 / big;
  }
  sing = __any_sync(QMCB_FULL_MASK, sing);
  __syncwarp();
  if (sing) {
    logdet = -INFINITY;
    sign = 0.0;
    return false;
  }
  double sg = 1.0, ld = 0.0;
  for (int j = 0; j < n; j++) {
    double best = -1.0;
    int bi = -1;
    for (int i = j + lane; i < n; i += 32) {
      double v = vv[i] * fabs(A[i * n + j]);
      if (v >= best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(QMCB_FULL_MASK, best, o);
      int oi = __shfl_xor_sync(QMCB_FULL_MASK, bi, o);
      if (ob > best || (ob == best && oi > bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (bi != j) {
      for (int k = lane; k < n; k += 32) {
        double t = A[bi * n + k];
        A[bi * n + k] = A[j * n + k];
        A[j * n + k] = t;
      }
      if (lane == 0) vv[bi] = vv[j];
      sg = -sg;
    }
    if (lane == 0) piv[j] = (double)bi;
    __syncwarp();
    const double p = A[j * n + j];
    if (p == 0.0) {
      sing = true;
      break;
    }
    ld += log(fabs(p));
    if (p < 0) sg = -sg;
    // column j is saved and replaced by the identity's column j, whose
    // image under the step's row operations is column j of the inverse
    for (int i = lane; i < n; i += 32) {
      col[i] = A[i * n + j];
      A[i * n + j] = i == j ? 1.0 : 0.0;
    }
    __syncwarp();
    const double pinv = 1.0 / p;
    for (int k = lane; k < n; k += 32) A[j * n + k] *= pinv;
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
      const double rj = A[j * n + k];
      int i = 0;
      for (; i + 4 <= n; i += 4) {
        double c[4], a[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          c[u] = col[i + u];
          a[u] = A[(i + u) * n + k];
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (i + u != j) A[(i + u) * n + k] = fma(-c[u], rj, a[u]);
      }
      for (; i < n; i++)
        if (i != j) A[i * n + k] = fma(-col[i], rj, A[i * n + k]);
    }
    __syncwarp();
  }
  if (sing) {
    logdet = -INFINITY;
    sign = 0.0;
    return false;
  }
  logdet = ld;
  sign = sg;
  // the row interchanges, undone as column interchanges, last first
  for (int j = n - 1; j >= 0; j--) {
    const int bi = (int)piv[j];
    if (bi != j)
      for (int i = lane; i < n; i += 32) {
        const double t = A[i * n + j];
        A[i * n + j] = A[i * n + bi];
        A[i * n + bi] = t;
      }
  }
  __syncwarp();
  return true;
}

// ------------------------------------------------------------------------
// Jastrow and potential from scratch for all electrons (updateAll order of
// pairs is irrelevant here: totals are summed fresh, not incrementally).
// Writes Ux[N][3] to `ux`, returns U, U_xx, V_ee, V_en through refs.
template <bool kTB>
__device__ inline void jastrow_pe_full_warp(const DevSys &S, const double *R, double *ux, double &U, double &Uxx,
                                            double &Vee, double &Ven)
{
  const int lane = lane_id(), N = S.N;
  double pu = 0, pxx = 0, pee = 0, pen = 0;
  for (int i = lane; i < N; i += 32) {
    double xi = R[3 * i], yi = R[3 * i + 1], zi = R[3 * i + 2];
    double gx = 0, gy = 0, gz = 0;
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      double dx = xi - R[3 * j], dy = yi - R[3 * j + 1], dz = zi - R[3 * j + 2];
      // 1 / r from one reciprocal square root (ulp-level differences from
      // sqrt and divisions, far inside the parity bound)
      const double r2 = dx * dx + dy * dy + dz * dz, ir = rsqrt(r2), r = r2 * ir;
      if (j < i) pee += ir;
      int f = ee_func(S, i, j);
      if (f < 0) continue;
      double u, du, d2u;
      pade_eval(S, f, r, u, du, d2u);
      gx += du * (dx * ir);
      gy += du * (dy * ir);
      gz += du * (dz * ir);
      if (j < i) {
        pu += u;
        pxx += 2.0 * (2.0 * ir * du + d2u);
      }
    }
    int sp = i < S.na ? 0 : 1;
    for (int A = 0; A < S.M; A++) {
      double4 P = S.nuc[A];
      double dx = xi - P.x, dy = yi - P.y, dz = zi - P.z;
      const double r2 = dx * dx + dy * dy + dz * dz, ir = rsqrt(r2), r = r2 * ir;
      pen -= P.w * ir;
      int f = S.en[sp][A];
      if (f < 0) continue;
      double u, du, d2u;
      pade_eval(S, f, r, u, du, d2u);
      gx += du * (dx * ir);
      gy += du * (dy * ir);
      gz += du * (dz * ir);
      pu += u;
      pxx += 2.0 * ir * du + d2u;
    }
    ux[3 * i] = gx;
    ux[3 * i + 1] = gy;
    ux[3 * i + 2] = gz;
  }
  if (kTB && S.ntb > 0) {
    double acc[2] = {0.0, 0.0};
    tb_full_lane(S, R, ux, acc);
    pu += acc[0];
    pxx += acc[1];
  }
  U = warp_sum(pu);
  Uxx = warp_sum(pxx);
  Vee = warp_sum(pee);
  Ven = warp_sum(pen);
}

// Psi quantities (QMCSCFJastrow::calculate_Psi_quantities / update_SCF,
// QMcBeaver/src/QMCSCFJastrow.cpp:196-327): gr = gD + Ux and
// lap = Dxx + U_xx + sum(2 Ux.gD + Ux.Ux).
__device__ inline double psi_lap_warp(int N, const double *gD, const double *Ux, double *gr, double Dxx, double Uxx)
{
  const int lane = lane_id();
  double part = 0.0;
  for (int i = lane; i < N; i += 32) {
    for (int d = 0; d < 3; d++) {
      double dx = gD[3 * i + d], u = Ux[3 * i + d];
      gr[3 * i + d] = dx + u;
      part += u * dx * 2.0;
      part += u * u;
    }
  }
  return Dxx + Uxx + warp_sum(part);
}

// ------------------------------------------------------------------------
// Full evaluation (do_basis = true: QMCSCFJastrow::evaluate with whichE = -1)
// or refresh from the stored Slater values (do_basis = false).
// R_in: [num][N][3] positions to store first (null: use the stored ones).
template <typename TS, typename TI, bool kExtras>
__global__ void __launch_bounds__(128) k_full(DevSys S, Layout L, RunCfg cfg, double *state, const int *slots,
                                              int num, const int *d_num, const double *R_in, int do_basis,
                                              EvalOut out)
{
  extern __shared__ double smem[];
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  const int nw = d_num ? *d_num : num;
  const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (wi >= nw) return;
  const int N = S.N, K = S.K, nmax = max(S.na, S.nb);
  const int slot = slots ? slots[wi] : wi;
  double *blk = state + (size_t)slot * L.stride;
  double *sm = smem + (size_t)warp * (do_basis ? full_scratch_doubles(N, K, nmax) : refresh_scratch_doubles(N, nmax));
  const int ldc = K + 1;
  double *chi = sm;
  double *Dn = chi + 5 * ldc;
  double *A = do_basis ? Dn + 5 * nmax : sm;  // the refresh has no basis rows
  double *X = A;                              // inverted in place
  double *vv = A + nmax * nmax;
  double *piv = vv + nmax;
  double *col = piv + nmax;
  double *Rs = col + nmax;
  double *R = blk + L.R;
  double *sc = blk + L.sc;

  if (R_in) {
    for (int t = lane; t < 3 * N; t += 32) R[t] = R_in[(size_t)wi * 3 * N + t];
  }
  for (int t = lane; t < 3 * N; t += 32) Rs[t] = R[t];
  __syncwarp();

  bool bad = false;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? S.nb : S.na, base = sp ? S.na : 0;
    if (n == 0) {
      sc[SC_LAPR_A + sp] = 0.0;
      sc[SC_LOGDET_A + sp] = 0.0;
      sc[SC_SIGN_A + sp] = 1.0;
      continue;
    }
    // stored Slater rows in the state precision TS; the basis, LU and ratio
    // sums here always run in FP64 (this is the refresh of the mixed path)
    TS *Dv = (TS *)(blk + L.Dv[sp]), *DgT = (TS *)(blk + L.DgT[sp]), *DlT = (TS *)(blk + L.DlT[sp]);
    if (do_basis) {
      for (int e = 0; e < n; e++) {
        double r[3] = {Rs[3 * (base + e)], Rs[3 * (base + e) + 1], Rs[3 * (base + e) + 2]};
        basis_shells_warp(S, r, chi, ldc);
        __syncwarp();
        contract_dmma_warp(chi, ldc, S.ct[sp], n, K, Dn);
        __syncwarp();
        if (kExtras && S.cusp) {
          cusp_replace_warp(S, sp, r, Dn, n, n);
          __syncwarp();
        }
        for (int o = lane; o < n; o += 32) {
          Dv[e * n + o] = (TS)Dn[o];
          DgT[(0 * n + o) * n + e] = (TS)Dn[n + o];
          DgT[(1 * n + o) * n + e] = (TS)Dn[2 * n + o];
          DgT[(2 * n + o) * n + e] = (TS)Dn[3 * n + o];
          DlT[o * n + e] = (TS)Dn[4 * n + o];
        }
        __syncwarp();
      }
    }
    for (int t = lane; t < n * n; t += 32) A[t] = (double)Dv[t];
    __syncwarp();
    double logdet, sign;
    bool ok = gj_inverse_warp(A, vv, piv, col, n, logdet, sign);
    if (!ok) bad = true;
    TI *Inv = (TI *)(blk + L.Inv[sp]);
    for (int t = lane; t < n * n; t += 32) Inv[t] = (TI)X[t];
    // ratio sums (QMcBeaver/src/QMCSlater.cpp:741-762)
    double lp = 0.0;
    for (int e = lane; e < n; e += 32) {
      double gx = 0, gy = 0, gz = 0;
      for (int o = 0; o < n; o++) {
        double iv = X[o * n + e];
        lp += (double)DlT[o * n + e] * iv;
        gx += (double)DgT[(0 * n + o) * n + e] * iv;
        gy += (double)DgT[(1 * n + o) * n + e] * iv;
        gz += (double)DgT[(2 * n + o) * n + e] * iv;
      }
      blk[L.gradD + 3 * (base + e)] = gx;
      blk[L.gradD + 3 * (base + e) + 1] = gy;
      blk[L.gradD + 3 * (base + e) + 2] = gz;
    }
    lp = warp_sum(lp);
    if (lane == 0) {
      sc[SC_LAPR_A + sp] = lp;
      sc[SC_LOGDET_A + sp] = logdet;
      sc[SC_SIGN_A + sp] = sign;
      sc[SC_INVCUR_A + sp] = 0.0;  // the inverse was written to its first copy
    }
    __syncwarp();
  }

  double U, Uxx, Vee, Ven;
  double *ux = blk + L.Ux;
  jastrow_pe_full_warp<kExtras>(S, Rs, ux, U, Uxx, Vee, Ven);
  __syncwarp();
  double *gD = blk + L.gradD, *gr = blk + L.grad, *mg = blk + L.mgrad;
  double Dxx = 0.0;
  if (S.na > 0) Dxx += sc[SC_LAPR_A];
  if (S.nb > 0) Dxx += sc[SC_LAPR_B];
  double lap = psi_lap_warp(N, gD, ux, gr, Dxx, Uxx);
  __syncwarp();
  double modratio = qf_modify_warp(S, cfg, Rs, gr, mg, &bad);
  double PE = S.Pnn + Vee + Ven;
  double EL = -0.5 * lap + PE;
  unsigned st = bad ? 1u : 0u;
  if (isnan(EL) || isnan(lap)) st |= 2u;
  if (lane == 0) {
    sc[SC_U] = U;
    sc[SC_UXX] = Uxx;
    sc[SC_VEE] = Vee;
    sc[SC_VEN] = Ven;
    sc[SC_PE] = PE;
    sc[SC_EL] = EL;
    sc[SC_LAP] = lap;
    sc[SC_MODRATIO] = modratio;
    sc[SC_STATUS] = (double)st;
    if (R_in) {
      sc[SC_WEIGHT] = 1.0;
      sc[SC_AGE] = 0.0;
      sc[SC_AGE_MOVED] = 0.0;
      sc[SC_DW] = 1.0;
    }
    if (out.log_abs_psi) out.log_abs_psi[wi] = sc[SC_LOGDET_A] + sc[SC_LOGDET_B] + U;
    if (out.sign) out.sign[wi] = sc[SC_SIGN_A] * sc[SC_SIGN_B];
    if (out.lap) out.lap[wi] = lap;
    if (out.e_local) out.e_local[wi] = EL;
    if (out.pe) {
      out.pe[3 * wi] = PE;
      out.pe[3 * wi + 1] = Ven;
      out.pe[3 * wi + 2] = Vee;
    }
    if (out.status) out.status[wi] = (unsigned char)st;
  }
  __syncwarp();
  if (out.grad)
    for (int t = lane; t < 3 * N; t += 32) out.grad[(size_t)wi * 3 * N + t] = gr[t];
  if (out.mgrad)
    for (int t = lane; t < 3 * N; t += 32) out.mgrad[(size_t)wi * 3 * N + t] = mg[t];
}

struct MoveArgs {
  int e;             // moved electron
  int step;          // global step number (random stream position)
  int do_reweight;   // this step reweights / collects observables (whichE == 0)
  int reweight_on;   // step >= reweight_start_step
  double *dump;      // configuration records of this step (null: none), see dump_configs
  // orbital rows of the moved electron at the proposed position, [list
  // index][5][n] (null: the move kernel evaluates the basis and contracts)
  const double *rows = nullptr;
  // evaluate entry points: R_in holds only the moved electron's position per
  // walker ([num][3]) instead of all positions ([num][N][3])
  int rin_moved = 0;
};

// Configuration records of one Metropolis step (print_configs:
// QMCWalker::processPropagation -> QMCWalkerData::writeConfigs ->
// QMCConfigIO::writeCorrelatedSamplingConfiguration, QMcBeaver/src/QMCWalker.cpp:
// 238-250, QMcBeaver/src/QMCWalkerData.cpp:216-224): the trial walker with
// weight p, then the original walker with weight 1 - p.  A record is
// R[3N], lap(D)/D, grad(D)/D [3N], ln J, potential energy, weight (6N + 4
// doubles); walker wi writes records 2 wi and 2 wi + 1.  sR holds the trial
// positions, gD_new / gD_old the Slater gradient ratios of all electrons.
__device__ __forceinline__ void dump_configs(double *dump, int wi, int N, int e, const double *sR,
                                             const double ro[3], double Dxx_new, const double *gD_new,
                                             double U_new, double PE_new, double Dxx_old, const double *gD_old,
                                             double U_old, double PE_old, double p)
{
  const int lane = lane_id();
  const int rec = 6 * N + 4;
  double *t = dump + (size_t)wi * 2 * rec, *o = t + rec;
  for (int k = lane; k < 3 * N; k += 32) {
    const double x = sR[k];
    t[k] = x;
    o[k] = (k / 3 == e) ? ro[k - 3 * e] : x;
    t[3 * N + 1 + k] = gD_new[k];
    o[3 * N + 1 + k] = gD_old[k];
  }
  if (lane == 0) {
    t[3 * N] = Dxx_new;
    o[3 * N] = Dxx_old;
    t[6 * N + 1] = U_new;
    o[6 * N + 1] = U_old;
    t[6 * N + 2] = PE_new;
    o[6 * N + 2] = PE_old;
    t[6 * N + 3] = p;
    o[6 * N + 3] = 1.0 - p;
  }
}

// ------------------------------------------------------------------------
// Pieces of the single-electron move shared by the one- and the
// several-determinant move kernels.

// ---- umrigar93_importance_sampling (QMCWalker::moveElectronsUmrigar93ImportanceSampling
//      and calculateReverseGreensFunctionUmrigar93ImportanceSampling,
//      QMcBeaver/src/QMCWalker.cpp:400-586, 783-926; C. J. Umrigar, M. P.
//      Nightingale, K. J. Runge, J. Chem. Phys. 99, 2865 (1993)).  Each
//      electron moves either by the drift-diffusion Gaussian, its drift split
//      into components along and across the direction from the nearest
//      nucleus, or by a hydrogen-like exponential centred on that nucleus.
struct UmrigarFrame {
  double A[3], c[3];   // nearest nucleus, centre of the drifted Gaussian
  double zeta, pg, ps; // exponential's exponent, Gaussian / exponential move probabilities
};

__device__ inline void umrigar_frame(const DevSys &S, const RunCfg &cfg, const double x[3], const double v[3],
                                     UmrigarFrame &F)
{
  int nn = 0;
  double best = 1e300;
  for (int A = 0; A < S.M; A++) {
    const double4 P = S.nuc[A];
    const double dx = x[0] - P.x, dy = x[1] - P.y, dz = x[2] - P.z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 < best) {
      best = d2;
      nn = A;
    }
  }
  const double4 P = S.nuc[nn];
  F.A[0] = P.x;
  F.A[1] = P.y;
  F.A[2] = P.z;
  const double tau = cfg.dt;
  const double d = sqrt(best);
  double zu[3], rad[3], zc = 0.0, rc = 0.0;
  for (int k = 0; k < 3; k++) {
    zu[k] = (x[k] - F.A[k]) / d;
    zc += zu[k] * v[k];
  }
  for (int k = 0; k < 3; k++) {
    rad[k] = v[k] - zc * zu[k];
    rc += rad[k] * rad[k];
  }
  rc = sqrt(rc);
  if (rc > 1e-15)
    for (int k = 0; k < 3; k++) rad[k] /= rc;
  const double zC = fmax(d + zc * tau, 0.0);
  const double rC = 2.0 * rc * tau * zC / (d + zC);
  F.zeta = sqrt(P.w * P.w + 1.0 / tau);
  F.ps = fmin(fmax(0.5 * erfc((d + zc * tau) / sqrt(2.0 * tau)), 0.0), 1.0);
  F.pg = 1.0 - F.ps;
  for (int k = 0; k < 3; k++) F.c[k] = F.A[k] + rC * rad[k] + zC * zu[k];
}

// ln of the one-electron transition density of the frame at y:
// pg (2 pi tau)^-3/2 exp(-|y - c|^2 / 2 tau) + ps / pi zeta^3 exp(-2 zeta |y - A|)
__device__ inline double umrigar_log_gf(const UmrigarFrame &F, const RunCfg &cfg, const double y[3])
{
  double d1 = 0.0, d2 = 0.0;
  for (int k = 0; k < 3; k++) {
    d1 += (y[k] - F.c[k]) * (y[k] - F.c[k]);
    d2 += (y[k] - F.A[k]) * (y[k] - F.A[k]);
  }
  const double tau = cfg.dt;
  const double lg = F.pg > 0.0 ? log(F.pg) - 1.5 * log(6.283185307179586 * tau) - d1 / (2.0 * tau) : -INFINITY;
  const double ls = F.ps > 0.0 ? log(F.ps / 3.141592653589793) + 3.0 * log(F.zeta) - 2.0 * F.zeta * sqrt(d2)
                               : -INFINITY;
  const double m = fmax(lg, ls);
  if (m == -INFINITY) return -INFINITY;
  return m + log(exp(lg - m) + exp(ls - m));
}

// Proposal of electron e and ln G(R -> R') over all electrons (the
// unmoved ones contribute their stay-in-place density; cfg.exact_gf: the
// moved electron only).
__device__ __noinline__ void umrigar_propose(const DevSys &S, const RunCfg &cfg, int slot, int step, int e, int N,
                                             const double *R, const double *mgo, double *rn, double *log_fwd,
                                             double *u_acc)
{
  const int lane = threadIdx.x & 31;
  // lanes 0-3 draw two uniforms each from their own Philox counters
  double u[8];
  {
    const U4 c = philox4x32(U4{(uint32_t)slot, (uint32_t)step, (uint32_t)(8 + (lane & 3)), 0x0A7E5A21u}, cfg.seed);
    const double ua = u01(c.x, c.y), ub = u01(c.z, c.w);
    for (int k = 0; k < 4; k++) {
      u[2 * k] = __shfl_sync(QMCB_FULL_MASK, ua, k);
      u[2 * k + 1] = __shfl_sync(QMCB_FULL_MASK, ub, k);
    }
  }
  UmrigarFrame F;
  umrigar_frame(S, cfg, R + 3 * e, mgo + 3 * e, F);
  if (u[0] < F.pg) {
    // Gaussian around the drifted centre (Box-Muller from u[1..4])
    const double r1 = sqrt(-2.0 * log(u[1])), r2 = sqrt(-2.0 * log(u[3]));
    const double g[3] = {r1 * cos(6.283185307179586 * u[2]), r1 * sin(6.283185307179586 * u[2]),
                         r2 * cos(6.283185307179586 * u[4])};
    const double sg = sqrt(cfg.dt);
    for (int k = 0; k < 3; k++) rn[k] = F.c[k] + sg * g[k];
  } else {
    // hydrogen-like: r from r^2 exp(-2 zeta r) (a Gamma(3) variate over 2 zeta;
    // Random::randomDistribution1 draws the same law by rejection), uniform direction
    const double r = -log(u[1] * u[2] * u[3]) / (2.0 * F.zeta);
    const double phi = 6.283185307179586 * u[4], theta = acos(1.0 - 2.0 * u[5]);
    rn[0] = F.A[0] + r * sin(theta) * cos(phi);
    rn[1] = F.A[1] + r * sin(theta) * sin(phi);
    rn[2] = F.A[2] + r * cos(theta);
  }
  *u_acc = u[6];
  double part = 0.0;
  for (int i = lane; i < N; i += 32) {
    UmrigarFrame Fi;
    if (i == e) {
      part += umrigar_log_gf(F, cfg, rn);
    } else if (!cfg.exact_gf) {
      umrigar_frame(S, cfg, R + 3 * i, mgo + 3 * i, Fi);
      part += umrigar_log_gf(Fi, cfg, R + 3 * i);
    }
  }
  *log_fwd = warp_sum(part);
}

// ln G(R' -> R): frames of the new positions R' with the new drift, density
// at the old positions (the moved electron's old position is ro).
__device__ __noinline__ double umrigar_log_reverse(const DevSys &S, const RunCfg &cfg, int e, int N, const double *Rn,
                                                   const double *mg, const double *ro)
{
  double part = 0.0;
  for (int i = threadIdx.x & 31; i < N; i += 32) {
    if (cfg.exact_gf && i != e) continue;
    UmrigarFrame F;
    umrigar_frame(S, cfg, Rn + 3 * i, mg + 3 * i, F);
    part += umrigar_log_gf(F, cfg, i == e ? ro : Rn + 3 * i);
  }
  return warp_sum(part);
}

// New position of electron e: the walker's own Philox stream and the drift
// (QMCWalker::moveElectronsNoImportanceSampling / moveElectronsImportanceSampling /
// moveElectronsUmrigar93ImportanceSampling, QMcBeaver/src/QMCWalker.cpp:313-586),
// or the caller's position.  g_fwd: the exponent sum of G(R -> R') (drift
// diffusion) or ln G(R -> R') (Umrigar93); u_acc the acceptance uniform.
// kUmr: the Umrigar93 move is compiled in (the launcher picks such an
// instantiation whenever the run uses it).
template <bool kMetropolis, bool kUmr>
__device__ __forceinline__ void propose_move(const DevSys &S, const RunCfg &cfg, int slot, int step, int e, int N,
                                             const double *R, const double ro[3], const double *mgo,
                                             const double *R_in, int wi, double rn[3], double &g_fwd, double &u_acc,
                                             int rin_moved)
{
  const int lane = lane_id();
  g_fwd = 0.0;
  u_acc = 0.5;
  if (kMetropolis && kUmr && cfg.sampling == 2) {
    umrigar_propose(S, cfg, slot, step, e, N, R, mgo, rn, &g_fwd, &u_acc);
  } else if (kMetropolis) {
    // lanes 0-2 draw the three Gaussian displacements, lane 3 the acceptance
    // uniform, each from its own Philox counter; one round trip for the warp
    double zr, z[3];
    {
      const U4 c = philox4x32(U4{(uint32_t)slot, (uint32_t)step, (uint32_t)(lane & 3), 0x51ED2701u}, cfg.seed);
      // Box-Muller in single precision: the proposal only needs a Gaussian
      // sample, not a particular one (the random streams differ from the
      // reference's ran1 in any case)
      const float u1 = ((float)(c.x >> 8) + 0.5f) * (1.0f / 16777216.0f);
      const float u2 = (float)(c.y >> 8) * (1.0f / 16777216.0f);
      const float rad = sqrtf(-2.0f * __logf(u1));
      float sn, cs;
      __sincosf(6.2831853f * u2, &sn, &cs);
      zr = (lane & 3) == 3 ? u01(c.z, c.w) : (double)(rad * cs);
    }
    z[0] = __shfl_sync(QMCB_FULL_MASK, zr, 0);
    z[1] = __shfl_sync(QMCB_FULL_MASK, zr, 1);
    z[2] = __shfl_sync(QMCB_FULL_MASK, zr, 2);
    u_acc = __shfl_sync(QMCB_FULL_MASK, zr, 3);
    const double sigma = sqrt(cfg.dt);
    for (int d = 0; d < 3; d++) {
      const double drift = sigma * z[d];
      double disp = drift;
      if (cfg.sampling == 1) disp += cfg.dt * mgo[3 * e + d];
      rn[d] = ro[d] + disp;
      g_fwd += drift * drift;
    }
    if (cfg.sampling == 1 && !cfg.exact_gf) {
      // G(R -> R') includes the drift of the electrons that do not move
      // (QMcBeaver/src/QMCWalker.cpp:383-388)
      double prt = 0.0;
      for (int t = lane; t < 3 * N; t += 32) {
        if (t / 3 == e) continue;
        const double dd = cfg.dt * mgo[t];
        prt += dd * dd;
      }
      g_fwd += warp_sum(prt);
    }
  } else {
    // the caller's position of electron e: R_in[wi][N][3], or R_in[wi][3]
    // when the caller sends the moved electron only
    for (int d = 0; d < 3; d++) rn[d] = rin_moved ? R_in[(size_t)wi * 3 + d] : R_in[(size_t)wi * 3 * N + 3 * e + d];
  }
}

// Incremental Jastrow + potential of moving electron e from ro to rn
// (QMCJastrowElectronElectron::updateOne, QMCJastrowElectronNuclear::evaluate,
// QMCPotential_Energy::evaluate); lane j updates its own U_x[j] in place,
// U_x[e] and the staged position of e are written last.  kTB: the system
// may have three-body terms (a separate instantiation keeps them out of the
// register allocation of the plain move); tbs: 3 N M doubles of shared
// scratch for them.
template <bool kTB>
__device__ __forceinline__ void jastrow_pe_move_warp(const DevSys &S, double *sR, double *Ux, int e, int sp,
                                                     const double ro[3], const double rn[3], double &dU,
                                                     double &dUxx, double &dVee, double &dVen, double *tbs)
{
  const int lane = lane_id(), N = S.N;
  double ge[3] = {0, 0, 0};
  dU = dUxx = dVee = dVen = 0.0;
  const double uxe[3] = {Ux[3 * e], Ux[3 * e + 1], Ux[3 * e + 2]};
  __syncwarp();
  for (int j = lane; j < N; j += 32) {
    if (j == e) continue;
    const double Rj[3] = {sR[3 * j], sR[3 * j + 1], sR[3 * j + 2]};
    const double dxo = ro[0] - Rj[0], dyo = ro[1] - Rj[1], dzo = ro[2] - Rj[2];
    const double dxn = rn[0] - Rj[0], dyn = rn[1] - Rj[1], dzn = rn[2] - Rj[2];
    // 1 / r from one reciprocal square root, r = r^2 / r (ulp-level
    // differences from sqrt and a division, far inside the parity bound)
    const double r2o = dxo * dxo + dyo * dyo + dzo * dzo, r2n = dxn * dxn + dyn * dyn + dzn * dzn;
    const double io = rsqrt(r2o), in_ = rsqrt(r2n);
    const double r_o = r2o * io, r_n = r2n * in_;
    dVee += in_ - io;
    const int f = ee_func(S, e, j);
    if (f >= 0) {
      double uo, duo, d2uo, un, dun, d2un;
      pade_eval(S, f, r_o, uo, duo, d2uo);
      pade_eval(S, f, r_n, un, dun, d2un);
      dU += un - uo;
      dUxx += 2.0 * (2.0 * in_ * dun + d2un) - 2.0 * (2.0 * io * duo + d2uo);
      const double sn = dun * in_, so = duo * io;
      const double vx = sn * dxn - so * dxo, vy = sn * dyn - so * dyo, vz = sn * dzn - so * dzo;
      ge[0] += vx;
      ge[1] += vy;
      ge[2] += vz;
      Ux[3 * j] -= vx;
      Ux[3 * j + 1] -= vy;
      Ux[3 * j + 2] -= vz;
    }
  }
  for (int A = lane; A < S.M; A += 32) {
    const double4 P = S.nuc[A];
    const double dxo = ro[0] - P.x, dyo = ro[1] - P.y, dzo = ro[2] - P.z;
    const double dxn = rn[0] - P.x, dyn = rn[1] - P.y, dzn = rn[2] - P.z;
    // 1 / r from one reciprocal square root, r = r^2 / r (ulp-level
    // differences from sqrt and a division, far inside the parity bound)
    const double r2o = dxo * dxo + dyo * dyo + dzo * dzo, r2n = dxn * dxn + dyn * dyn + dzn * dzn;
    const double io = rsqrt(r2o), in_ = rsqrt(r2n);
    const double r_o = r2o * io, r_n = r2n * in_;
    dVen -= P.w * (in_ - io);
    const int f = S.en[sp][A];
    if (f >= 0) {
      double uo, duo, d2uo, un, dun, d2un;
      pade_eval(S, f, r_o, uo, duo, d2uo);
      pade_eval(S, f, r_n, un, dun, d2un);
      dU += un - uo;
      dUxx += (2.0 * in_ * dun + d2un) - (2.0 * io * duo + d2uo);
      const double sn = dun * in_, so = duo * io;
      ge[0] += sn * dxn - so * dxo;
      ge[1] += sn * dyn - so * dyo;
      ge[2] += sn * dzn - so * dzo;
    }
  }
  if (kTB && S.ntb > 0) {
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    tb_move_lane(S, sR, Ux, e, ro, rn, acc, tbs);
    dU += acc[0];
    dUxx += acc[1];
    ge[0] += acc[2];
    ge[1] += acc[3];
    ge[2] += acc[4];
  }
  dU = warp_sum(dU);
  dUxx = warp_sum(dUxx);
  dVee = warp_sum(dVee);
  dVen = warp_sum(dVen);
  for (int d = 0; d < 3; d++) ge[d] = warp_sum(ge[d]);
  __syncwarp();
  if (lane == 0)
    for (int d = 0; d < 3; d++) {
      Ux[3 * e + d] = uxe[d] + ge[d];
      sR[3 * e + d] = rn[d];
    }
}

// Acceptance (QMCWalker::calculateMoveAcceptanceProbability,
// QMcBeaver/src/QMCWalker.cpp:1578-1654), DMC reweight (reweight_walker,
// :1060-1185) and observables (:2096-2123, 2306-2387) of one proposed move.
// log_ratio = ln|psi'/psi|, negative = the ratio changed sign.  Writes the
// walker's weight, age and the per-call sums; returns the acceptance.
template <bool kUmr>
__device__ __forceinline__ bool metropolis_reweight(const DevSys &S, const RunCfg &cfg, const MoveArgs &mv,
                                                    const EnergyCtl *ectl, double *stats, double *sc,
                                                    const double *sc0, int N, int e, const double *Rn,
                                                    const double ro[3], const double rn[3], const double *mg,
                                                    double g_fwd, double u_acc, double log_ratio, bool negative,
                                                    bool bad, double EL, double modratio, double &p_acc)
{
  const int lane = lane_id();
  // G(R' -> R): only electron e moved, the others contribute (dt v'_i)^2
  double log_g = 0.0;
  if (kUmr && cfg.sampling == 2) {
    log_g = umrigar_log_reverse(S, cfg, e, N, Rn, mg, ro) - g_fwd;
  } else if (cfg.sampling == 1) {
    double pr = 0.0;
    for (int t = lane; t < 3 * N; t += 32) {
      if (cfg.exact_gf && t / 3 != e) continue;
      const double tt = (t / 3 == e) ? (ro[t - 3 * e] - rn[t - 3 * e] - cfg.dt * mg[t]) : (cfg.dt * mg[t]);
      pr += tt * tt;
    }
    const double g_rev = warp_sum(pr);
    log_g = -(g_rev - g_fwd) / (2.0 * cfg.dt);
  }
  double p = exp(2.0 * log_ratio + log_g);
  const double age = sc0[SC_AGE];
  const double over = age - cfg.old_walker_acceptance;
  if (!isnan(p)) {
    if (over > 500)
      p = 1.0;
    else if (over > 0)
      p *= pow(1.1, over);
  } else {
    p = 0.0;
  }
  if (bad) p = 0.0;
  if (cfg.run_type == 1 && negative) p = 0.0;
  if (p > 1.0) p = 1.0;
  p_acc = p;
  const bool accept = p > u_acc;
  const double new_age = accept ? 0.0 : age + 1.0;
  double w = sc0[SC_WEIGHT];
  if (mv.do_reweight) {
    if (cfg.run_type == 1 && mv.reweight_on) {
      const double ET = ectl->e_trial, Eest = ectl->e_est;
      const double mo = sc0[SC_MODRATIO];
      double Eo = sc0[SC_EL];
      double Et = bad ? Eo : EL;
      if (cfg.ecut == 1) {
        Et *= bad ? mo : modratio;
        Eo *= mo;
      } else if (cfg.ecut == 2) {
        // DePasquale, Rothstein, Vrbik (1988) cutoff |E_L - E_orig| <= 2 / sqrt(dt)
        const double cut = 2.0 / sqrt(cfg.dt);
        Et = fmin(fmax(Et, cfg.e_orig - cut), cfg.e_orig + cut);
        Eo = fmin(fmax(Eo, cfg.e_orig - cut), cfg.e_orig + cut);
      }
      double St, So;
      if (cfg.emod == 0) {
        St = ET - Et;
        So = ET - Eo;
      } else if (cfg.emod == 2) {
        St = (ET - Et) * (bad ? mo : modratio);
        So = (ET - Eo) * mo;
      } else {
        St = (ET - Eest) + (Eest - Et) * (bad ? mo : modratio);
        So = (ET - Eest) + (Eest - Eo) * mo;
      }
      double rw;
      if (cfg.reweighting == 0)
        rw = 0.5 * (St + So);
      else if (cfg.reweighting == 1)
        rw = accept ? 0.5 * (St + So) : So;
      else
        rw = p * 0.5 * (So + St) + (1.0 - p) * So;
      const double dW = exp(rw * (cfg.dyn_dt ? ectl->dt_eff : cfg.dt_eff));
      if (new_age - cfg.old_walker_acceptance > 0)
        w *= 0.9;
      else
        w *= dW;
      if (lane == 0) sc[SC_DW] = dW;
      if (cfg.deletion) {
        // QMCWalker::reweight_walker's deletions (QMcBeaver/src/QMCWalker.cpp:1196-1365),
        // on the accepted configuration's local energy
        const double rel = fabs(((accept ? EL : sc0[SC_EL]) - cfg.e_orig) / cfg.e_orig);
        bool del;
        if (mv.step - cfg.equil_steps < -100)
          del = w > 2.0 * cfg.branching_threshold || w < 0.1 || dW > 1.5 || dW < 0.5 || isnan(dW) ||
                (rel > cfg.rel_cutoff && mv.step > 5) || new_age >= 30.0;
        else
          del = pow(dW, new_age + 1.0) > 15.0 || isnan(dW) || w > 50.0 || rel > cfg.rel_cutoff;
        if (del) w = 0.0;
      }
      // a non-finite weight (NaN energy or exp overflow) removes the walker
      // at the next branching instead of poisoning the ensemble sums
      if (!isfinite(w)) w = 0.0;
    }
    const double Eobs = p * (bad ? 0.0 : EL) + (1.0 - p) * sc0[SC_EL];
    // rel_cutoff filter of QMCWalker::calculateObservables (QMcBeaver/src/QMCWalker.cpp:2336-2351)
    const bool in_avg = fabs((Eobs - cfg.e_orig) / cfg.e_orig) < cfg.rel_cutoff;
    if (lane == 0 && w > 0.0 && in_avg) {
      atomicAdd(&stats[ST_SUM_W], w);
      atomicAdd(&stats[ST_SUM_WE], w * Eobs);
      atomicAdd(&stats[ST_SUM_WE2], w * Eobs * Eobs);
      atomicAdd(&stats[ST_RUN_SUM_W], w);
      atomicAdd(&stats[ST_RUN_SUM_WE], w * Eobs);
      atomicAdd(&stats[ST_RUN_COUNT], 1.0);
      if (cfg.dyn_dt) {
        // distance the moved electron was proposed to go, as
        // QMCWalker::calculateObservables samples it (QMcBeaver/src/QMCWalker.cpp:2176-2178, 2376-2383)
        const double d2 = (rn[0] - ro[0]) * (rn[0] - ro[0]) + (rn[1] - ro[1]) * (rn[1] - ro[1]) +
                          (rn[2] - ro[2]) * (rn[2] - ro[2]);
        atomicAdd(&stats[ST_RUN_SUM_WPD2], w * p * d2);
        atomicAdd(&stats[ST_RUN_SUM_WD2], w * d2);
      }
    }
  }
  if (lane == 0) {
    atomicAdd(&stats[ST_SUM_ACC], p);
    atomicAdd(&stats[ST_MOVES], 1.0);
    if (bad) atomicAdd(&stats[ST_SINGULAR], 1.0);
    sc[SC_WEIGHT] = w;
    sc[SC_AGE] = new_age;
    if (accept) sc[SC_AGE_MOVED] = age;
  }
  return accept;
}

// Outputs of one evaluate call for walker wi.
__device__ __forceinline__ void write_eval_out(const EvalOut &out, int wi, int N, double log_abs_psi, double sign,
                                               double lap, double EL, double PE, double Ven, double Vee, bool bad,
                                               const double *gr, const double *mg)
{
  const int lane = lane_id();
  if (lane == 0) {
    unsigned st = bad ? 1u : 0u;
    if (isnan(EL) || isnan(lap)) st |= 2u;
    if (out.log_abs_psi) out.log_abs_psi[wi] = log_abs_psi;
    if (out.sign) out.sign[wi] = sign;
    if (out.lap) out.lap[wi] = lap;
    if (out.e_local) out.e_local[wi] = EL;
    if (out.pe) {
      out.pe[3 * wi] = PE;
      out.pe[3 * wi + 1] = Ven;
      out.pe[3 * wi + 2] = Vee;
    }
    if (out.status) out.status[wi] = (unsigned char)st;
  }
  if (out.grad)
    for (int t = lane; t < 3 * N; t += 32) out.grad[(size_t)wi * 3 * N + t] = gr[t];
  if (out.mgrad)
    for (int t = lane; t < 3 * N; t += 32) out.mgrad[(size_t)wi * 3 * N + t] = mg[t];
}

// ------------------------------------------------------------------------
// One single-electron move of electron e for every walker in the list.
// kMetropolis = false: the caller's positions R_in[wi] are taken and the
// new state is committed unconditionally (QMCFunctions::evaluate with
// whichE = e).  kMetropolis = true: proposal from the walker's own random
// stream, acceptance test, DMC reweight when do_reweight, commit on accept
// (QMCWalker::initializePropagation / processPropagation,
// QMcBeaver/src/QMCWalker.cpp:179-282).

// kExtras: cusp replacement, three-body terms and the Umrigar93 move compiled
// in (the plain instantiation, used when the run needs none of them, carries
// none of their code).
//
// move_walker is the work of one warp on walker wi of the list (sm: the
// warp's L.mv_stride doubles of shared memory); k_move runs it for one
// system, k_move_group for the walkers of many systems in one launch.
//
// kGInv: the moved spin's inverse stays in HBM (large spins, whose inverse
// would crowd shared memory): the update reads the current copy and writes
// the other one, and acceptance flips which copy is current.
template <bool kMetropolis, typename TS, typename TI, bool kExtras, bool kGInv>
__device__ __forceinline__ void move_walker(const DevSys &S, const Layout &L, const RunCfg &cfg, double *state,
                                            const int *slots, int wi, double *sm, const double *R_in,
                                            const MoveArgs &mv, const EnergyCtl *ectl, double *stats,
                                            const EvalOut &out)
{
  const int lane = lane_id();
  const int N = S.N, K = S.K;
  const int e = mv.e;
  const int sp = e < S.na ? 0 : 1;
  const int n = sp ? S.nb : S.na, base = sp ? S.na : 0, el = e - base;
  const int slot = slots ? slots[wi] : wi;
  double *blk = state + (size_t)slot * L.stride;

  // ---- scratch of this warp (offsets in doubles, all even: 16-byte aligned)
  const int ldc = K;
  TS *chi = (TS *)sm;                  // region A: basis values ...
  TS *cpart = (TS *)sm;                // ... then contraction slice sums
  double *part = sm;                   // ... then ratio-sum slice sums
  double *gr = sm + kPart;             // ... and the new drift / modified drift
  double *mg = gr + 3 * N;
  TS *Dn = (TS *)(sm + L.mv_region_a); // new Slater / derivative rows [5][n]
  TI *valc = (TI *)(sm + L.mv_region_a + L.mv_dn);  // Sherman-Morrison factors [n]
  double *sR = sm + L.mv_region_a + L.mv_dn + L.mv_valc;  // positions (electron e updated in place)
  double *sT = sR + L.mv_r;            // gradD, Ux, grad, mgrad, scalars (prefetched copy)
  double *sS = sT + L.mv_tail;         // inverse of the moved spin (prefetched copy)
  double *gD = sT;                     // grad(D)/D, updated in place for the moved spin
  double *Ux = sT + (L.Ux - L.gradD);  // grad ln J, updated in place
  const double *mgo = sT + (L.mgrad - L.gradD);
  const double *sc0 = sT + (L.sc - L.gradD);
  const TS *DgT = (const TS *)(blk + L.DgT[sp]);  // read once per move by the ratio sums
  const TS *DlT = (const TS *)(blk + L.DlT[sp]);
  double *sc = blk + L.sc;
  const int inv_d = even((n * n * (int)sizeof(TI) + 7) / 8);
  // L2 policies of the HBM-kept inverse (kGInv): kept between its two reads
  const uint64_t keep = kGInv ? l2_evict_last_policy() : 0, drop = kGInv ? l2_evict_first_policy() : 0;

  // ---- stage the walker's state: positions and the per-electron arrays
  //      first, the moved spin's inverse as a second group that lands while
  //      the basis and orbital rows are computed
  warp_copy_async(sR, blk + L.R, L.mv_r);
  warp_copy_async(sT, blk + L.gradD, L.mv_tail);
  cp_async_commit();
  if (!kGInv) warp_copy_async(sS, blk + L.Inv[sp], inv_d);
  cp_async_commit();
  cp_async_wait<1>();
  __syncwarp();
  // the inverse the update reads (InvO) and the one it leaves (Inv): the
  // staged copy updated in place, or the spin's two copies in HBM
  const int icur = kGInv ? (int)sc0[SC_INVCUR_A + sp] : 0;
  const TI *InvO = kGInv ? (const TI *)(blk + L.Inv[sp] + icur * L.invsz[sp]) : (const TI *)sS;
  TI *Inv = kGInv ? (TI *)(blk + L.Inv[sp] + (1 - icur) * L.invsz[sp]) : (TI *)sS;

  const double ro[3] = {sR[3 * e], sR[3 * e + 1], sR[3 * e + 2]};
  double rn[3], g_fwd, u_acc;
  propose_move<kMetropolis, kExtras>(S, cfg, slot, mv.step, e, N, sR, ro, mgo, R_in, wi, rn, g_fwd, u_acc,
                                     mv.rin_moved);

  // ---- incremental Jastrow + potential
  double dU, dUxx, dVee, dVen;
  // (three-body partner gradients use region A, free until the basis)
  jastrow_pe_move_warp<kExtras>(S, sR, Ux, e, sp, ro, rn, dU, dUxx, dVee, dVen, sm);

  // ---- basis at the new position and the new Slater / derivative rows
  if (mv.rows) {
    // computed for the whole step by the batched tensor-core contraction
    const double *src = mv.rows + (size_t)wi * 5 * n;
    for (int t = lane; t < 5 * n; t += 32) Dn[t] = (TS)src[t];
    __syncwarp();
  } else if constexpr (sizeof(TS) == 8) {
    // the exponential slots follow the five chi rows (into the Dn / valc
    // space, unused until the contraction)
    basis_slots_warp(S, rn, (double *)chi, ldc, sm + 5 * ldc);
    __syncwarp();
    contract_dmma_warp((const double *)chi, ldc, S.ct[sp], n, K, (double *)Dn);
  } else {
    // FP32 chi rows take half of region A; the slots follow them
    basis_slots_warp_f(S, rn, (float *)chi, ldc, (float *)chi + 5 * ldc);
    __syncwarp();
    contract_slices_warp_f((const float *)chi, ldc, S.ctf[sp], n, K, (float *)Dn, (float *)cpart);
  }
  if constexpr (kExtras) {
    if (S.cusp) {
      __syncwarp();
      cusp_replace_warp(S, sp, rn, Dn, n, n);
    }
  }
  cp_async_wait<0>();
  __syncwarp();

  // ---- Sherman-Morrison row replacement (Array2D::inverseUpdateOneRow,
  //      QMcBeaver/include/Array2D.h:1567-1610), in place on the staged inverse
  // determinant ratio accumulated in FP64; the inverse update itself runs
  // in the state precision TS
  double rpart = 0.0;
  for (int o = lane; o < n; o += 32) rpart = fma((double)Dn[o], (double)InvO[o * n + el], rpart);
  const double ratio = warp_sum(rpart);
  bool bad = !(ratio != 0.0) || !isfinite(ratio);
  const double q = 1.0 / ratio;
  for (int c = lane; c < n; c += 32) {
    if (c == el) continue;
    TI val = (TI)0;
    if (kGInv) {
      // HBM / L2 operands: eight loads in flight before their FMAs
      int l = 0;
      for (; l + 8 <= n; l += 8) {
        TI v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = ginv_ld(&InvO[(l + u) * n + c], keep);
#pragma unroll
        for (int u = 0; u < 8; u++) val = fma((TI)Dn[l + u], v[u], val);
      }
      for (; l < n; l++) val = fma((TI)Dn[l], ginv_ld(&InvO[l * n + c], keep), val);
    } else {
      for (int l = 0; l < n; l++) val = fma((TI)Dn[l], Inv[l * n + c], val);
    }
    valc[c] = (TI)(val * q);
  }
  __syncwarp();
  double lp = 0.0;
  if (kGInv) {
    // the same element formulas as the in-place update, old copy -> new
    // copy, fused with the ratio sums of the moved spin
    // (QMcBeaver/src/QMCSlater.cpp:741-762): lane = electron column c, the
    // new inverse elements feed the sums as they are made (never read back)
    // and the walker's derivative rows stream from HBM alongside, kGInvBatch
    // orbitals' loads in flight at a time, evict-first
    constexpr int kB = kGInvBatch;
    for (int c = lane; c < n; c += 32) {
      const TI vc = c == el ? (TI)0 : valc[c];
      double gx = 0, gy = 0, gz = 0, ll = 0;
      int r = 0;
      for (; r + kB <= n; r += kB) {
        TI ie[kB], x[kB];
        TS g0[kB], g1[kB], g2[kB], gl[kB];
#pragma unroll
        for (int u = 0; u < kB; u++) {
          ie[u] = ginv_ld(&InvO[(r + u) * n + el], drop);
          x[u] = ginv_ld(&InvO[(r + u) * n + c], drop);
          if (c == el) {
            g0[u] = Dn[n + r + u];
            g1[u] = Dn[2 * n + r + u];
            g2[u] = Dn[3 * n + r + u];
            gl[u] = Dn[4 * n + r + u];
          } else {
            g0[u] = __ldcs(&DgT[(0 * n + r + u) * n + c]);
            g1[u] = __ldcs(&DgT[(1 * n + r + u) * n + c]);
            g2[u] = __ldcs(&DgT[(2 * n + r + u) * n + c]);
            gl[u] = __ldcs(&DlT[(r + u) * n + c]);
          }
        }
#pragma unroll
        for (int u = 0; u < kB; u++) {
          const TI nv = c == el ? (TI)(ie[u] * q) : x[u] - vc * ie[u];
          ginv_st(&Inv[(r + u) * n + c], nv, drop);
          const double iv = (double)nv;
          gx = fma((double)g0[u], iv, gx);
          gy = fma((double)g1[u], iv, gy);
          gz = fma((double)g2[u], iv, gz);
          ll = fma((double)gl[u], iv, ll);
        }
      }
      for (; r < n; r++) {
        const TI ie = ginv_ld(&InvO[r * n + el], drop);
        const TI nv = c == el ? (TI)(ie * q) : ginv_ld(&InvO[r * n + c], drop) - vc * ie;
        ginv_st(&Inv[r * n + c], nv, drop);
        const double iv = (double)nv;
        if (c == el) {
          gx = fma((double)Dn[n + r], iv, gx);
          gy = fma((double)Dn[2 * n + r], iv, gy);
          gz = fma((double)Dn[3 * n + r], iv, gz);
          ll = fma((double)Dn[4 * n + r], iv, ll);
        } else {
          gx = fma((double)__ldcs(&DgT[(0 * n + r) * n + c]), iv, gx);
          gy = fma((double)__ldcs(&DgT[(1 * n + r) * n + c]), iv, gy);
          gz = fma((double)__ldcs(&DgT[(2 * n + r) * n + c]), iv, gz);
          ll = fma((double)__ldcs(&DlT[r * n + c]), iv, ll);
        }
      }
      lp += ll;
      gD[3 * (base + c)] = gx;
      gD[3 * (base + c) + 1] = gy;
      gD[3 * (base + c) + 2] = gz;
    }
  } else if (n <= 32) {
    const int rpp = 32 / n, r0 = lane / n, c = lane - r0 * n;
    if (r0 < rpp && c != el) {
      const TI vc = valc[c];
      for (int r = r0; r < n; r += rpp) Inv[r * n + c] -= vc * Inv[r * n + el];
    }
  } else {
    for (int c = lane; c < n; c += 32) {
      if (c == el) continue;
      const TI vc = valc[c];
      for (int r = 0; r < n; r++) Inv[r * n + c] -= vc * Inv[r * n + el];
    }
  }
  __syncwarp();
  if (!kGInv)
    for (int r = lane; r < n; r += 32) Inv[r * n + el] = (TI)(Inv[r * n + el] * q);
  __syncwarp();

  // ---- ratio sums of the moved spin (QMcBeaver/src/QMCSlater.cpp:741-762)
  //      lanes = (orbital slice, electron) for n <= 16 (the inverse in HBM:
  //      fused with its update above)
  if (!kGInv) {
    const int S2 = n <= 32 ? 32 / n : 1;
    const int s2 = n <= 32 ? lane / n : 0;
    const int oa = n <= 32 ? (n * s2) / S2 : 0, ob = n <= 32 ? (n * (s2 + 1)) / S2 : n;
    for (int e2 = (n <= 32 ? lane - s2 * n : lane); e2 < n && s2 < S2; e2 += (n <= 32 ? n : 32)) {
      double gx = 0, gy = 0, gz = 0, ll = 0;
      if (e2 == el) {
        for (int o = oa; o < ob; o++) {
          const double iv = (double)Inv[o * n + el];
          gx = fma((double)Dn[n + o], iv, gx);
          gy = fma((double)Dn[2 * n + o], iv, gy);
          gz = fma((double)Dn[3 * n + o], iv, gz);
          ll = fma((double)Dn[4 * n + o], iv, ll);
        }
      } else {
        // the walker's rows stream from HBM once per move: load four
        // orbitals' worth before using them, evict-first so the system
        // tables keep the L1
        int o = oa;
        for (; o + 4 <= ob; o += 4) {
          TS g0[4], g1[4], g2[4], gl[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            g0[u] = __ldcs(&DgT[(0 * n + o + u) * n + e2]);
            g1[u] = __ldcs(&DgT[(1 * n + o + u) * n + e2]);
            g2[u] = __ldcs(&DgT[(2 * n + o + u) * n + e2]);
            gl[u] = __ldcs(&DlT[(o + u) * n + e2]);
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const double iv = (double)Inv[(o + u) * n + e2];
            gx = fma((double)g0[u], iv, gx);
            gy = fma((double)g1[u], iv, gy);
            gz = fma((double)g2[u], iv, gz);
            ll = fma((double)gl[u], iv, ll);
          }
        }
        for (; o < ob; o++) {
          const double iv = (double)Inv[o * n + e2];
          gx = fma((double)__ldcs(&DgT[(0 * n + o) * n + e2]), iv, gx);
          gy = fma((double)__ldcs(&DgT[(1 * n + o) * n + e2]), iv, gy);
          gz = fma((double)__ldcs(&DgT[(2 * n + o) * n + e2]), iv, gz);
          ll = fma((double)__ldcs(&DlT[o * n + e2]), iv, ll);
        }
      }
      lp += ll;
      if (S2 == 1) {
        gD[3 * (base + e2)] = gx;
        gD[3 * (base + e2) + 1] = gy;
        gD[3 * (base + e2) + 2] = gz;
      } else {
        part[(s2 * 3 + 0) * n + e2] = gx;
        part[(s2 * 3 + 1) * n + e2] = gy;
        part[(s2 * 3 + 2) * n + e2] = gz;
      }
    }
    if (S2 > 1) {
      __syncwarp();
      for (int e2 = lane; e2 < n; e2 += 32) {
        double gx = 0, gy = 0, gz = 0;
        for (int ss = 0; ss < S2; ss++) {
          gx += part[(ss * 3 + 0) * n + e2];
          gy += part[(ss * 3 + 1) * n + e2];
          gz += part[(ss * 3 + 2) * n + e2];
        }
        gD[3 * (base + e2)] = gx;
        gD[3 * (base + e2) + 1] = gy;
        gD[3 * (base + e2) + 2] = gz;
      }
    }
  }
  const double lapR = warp_sum(lp);
  __syncwarp();

  // ---- psi quantities, quantum force, local energy
  const double U_new = sc0[SC_U] + dU, Uxx_new = sc0[SC_UXX] + dUxx;
  const double lapA = sp == 0 ? lapR : sc0[SC_LAPR_A];
  const double lapB = sp == 1 ? lapR : sc0[SC_LAPR_B];
  double Dxx = 0.0;
  if (S.na > 0) Dxx += lapA;
  if (S.nb > 0) Dxx += lapB;
  const double lap = psi_lap_warp(N, gD, Ux, gr, Dxx, Uxx_new);
  __syncwarp();
  const double modratio = qf_modify_warp(S, cfg, sR, gr, mg, &bad);
  const double Vee = sc0[SC_VEE] + dVee, Ven = sc0[SC_VEN] + dVen;
  const double PE = S.Pnn + Vee + Ven;
  const double EL = -0.5 * lap + PE;
  if (isnan(EL)) bad = true;
  const double logdet_new = sc0[SC_LOGDET_A + sp] + log(fabs(ratio));
  const double sign_new = sc0[SC_SIGN_A + sp] * (ratio < 0 ? -1.0 : 1.0);

  bool accept = true;
  if (kMetropolis) {
    double p_acc;
    accept = metropolis_reweight<kExtras>(S, cfg, mv, ectl, stats, sc, sc0, N, e, sR, ro, rn, mg, g_fwd, u_acc,
                                          log(fabs(ratio)) + dU, ratio < 0, bad, EL, modratio, p_acc);
    if (mv.dump) {
      const double Dxx_old = (S.na > 0 ? sc0[SC_LAPR_A] : 0.0) + (S.nb > 0 ? sc0[SC_LAPR_B] : 0.0);
      dump_configs(mv.dump, wi, N, e, sR, ro, Dxx, gD, U_new, PE, Dxx_old, blk + L.gradD, sc0[SC_U],
                   sc0[SC_PE], p_acc);
    }
  }
  __syncwarp();

  if (accept) {
    double *Rw = blk + L.R;
    if (lane < 3) Rw[3 * e + lane] = rn[lane];
    if (!kGInv) {
      // the staged inverse goes back by one bulk (TMA) store of its 16-byte
      // part, issued after every lane's shared-memory writes are fenced for
      // the async proxy; its last odd element by plain store.  Both ends are
      // 16-byte aligned (per-warp scratch offsets and walker-block arrays).
      TI *InvW = (TI *)(blk + L.Inv[sp]);
      const int bytes = n * n * (int)sizeof(TI), bulk = bytes & ~15;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0 && bulk > 0) {
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(InvW),
                     "r"((unsigned)__cvta_generic_to_shared(Inv)), "r"(bulk)
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
      }
      for (int t = bulk / (int)sizeof(TI) + lane; t < n * n; t += 32) InvW[t] = Inv[t];
    } else if (lane == 0) {
      sc[SC_INVCUR_A + sp] = (double)(1 - icur);
    }
    TS *Dv = (TS *)(blk + L.Dv[sp]), *DgW = (TS *)(blk + L.DgT[sp]), *DlW = (TS *)(blk + L.DlT[sp]);
    for (int o = lane; o < n; o += 32) {
      Dv[el * n + o] = Dn[o];
      DgW[(0 * n + o) * n + el] = Dn[n + o];
      DgW[(1 * n + o) * n + el] = Dn[2 * n + o];
      DgW[(2 * n + o) * n + el] = Dn[3 * n + o];
      DlW[o * n + el] = Dn[4 * n + o];
    }
    for (int t = lane; t < 3 * n; t += 32) blk[L.gradD + 3 * base + t] = gD[3 * base + t];
    for (int t = lane; t < 3 * N; t += 32) {
      blk[L.Ux + t] = Ux[t];
      blk[L.mgrad + t] = mg[t];
      // gradPsiRatio itself is an evaluate output; the chain needs only the
      // modified drift (its length ratio is kept as a scalar)
      if (!kMetropolis) blk[L.grad + t] = gr[t];
    }
    if (lane == 0) {
      sc[SC_U] = U_new;
      sc[SC_UXX] = Uxx_new;
      sc[SC_LAPR_A + sp] = lapR;
      sc[SC_LOGDET_A + sp] = logdet_new;
      sc[SC_SIGN_A + sp] = sign_new;
      sc[SC_VEE] = Vee;
      sc[SC_VEN] = Ven;
      sc[SC_PE] = PE;
      sc[SC_EL] = EL;
      sc[SC_LAP] = lap;
      sc[SC_MODRATIO] = modratio;
      sc[SC_STATUS] = bad ? 1.0 : 0.0;
    }
  }
  if (!kGInv && accept) {
    // the bulk store must have read the staged inverse before this warp's
    // scratch is left (or reused for the next walker).  .read waits for the
    // shared-memory source only, not for the global writes: correct because
    // every launch of k_move / k_move_group moves each walker at most once,
    // so the kernel boundary orders these writes before the next read of the
    // inverse.  A kernel that re-reads a walker's inverse within one launch
    // must wait with cp.async.bulk.wait_group 0 (full completion) instead.
    if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
    __syncwarp();
  }
  if (!kMetropolis) {
    const double la = sp == 0 ? logdet_new : sc0[SC_LOGDET_A];
    const double lb = sp == 1 ? logdet_new : sc0[SC_LOGDET_B];
    const double sa = sp == 0 ? sign_new : sc0[SC_SIGN_A];
    const double sb = sp == 1 ? sign_new : sc0[SC_SIGN_B];
    write_eval_out(out, wi, N, la + lb + U_new, sa * sb, lap, EL, PE, Ven, Vee, bad, gr, mg);
  }
}

template <bool kMetropolis, typename TS, typename TI, bool kExtras, bool kGInv>
__global__ void __launch_bounds__(128, kGInv ? 3 : 5) k_move(DevSys S, Layout L, RunCfg cfg, double *state, const int *slots,
                                              int num, const int *d_num, const double *R_in, MoveArgs mv,
                                              const EnergyCtl *ectl, double *stats, EvalOut out)
{
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5;
  const int nw = d_num ? *d_num : num;
  const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (wi >= nw) return;
  move_walker<kMetropolis, TS, TI, kExtras, kGInv>(S, L, cfg, state, slots, wi, smem + (size_t)warp * L.mv_stride,
                                                   R_in, mv, ectl, stats, out);
}

// ------------------------------------------------------------------------
// Nonunit-weight branching (QMCRun::nonunitWeightBranching,
// QMcBeaver/src/QMCRun.cpp:740-814) on the live slot list, one CTA of
// 1024 threads.  Walkers above the branching threshold split in two with
// half the weight each (the copy is appended to the list), walkers below
// 0.01 die, walkers below the fusion threshold are paired in list order and
// one of each pair survives with the sum of the weights (probability
// w1 / (w1 + w2) for the first; the uniform draw of a pair is keyed by
// (seed, position of its first member in the live list, step)).  The split
// test uses the weight before fusion, so a fused survivor does not split in
// the same pass.  Dead slots go on the free stack; copies
// take slots from it and are written to the copy list for k_copy.
// ctl: [0] n_live, [1] n_free, [2] n_copies.
// QMCWalker::branchRecommended (limit_branching): no split for a walker that
// has not moved for more than 4 steps, whose weight grows too fast
// (dW^(age+1) > 5), that is heavy (> 100) and still growing (> 1.5), or whose
// local energy is more than 100x off the input energy.
__device__ __forceinline__ bool branch_recommended(const double *sc, double e_orig, int limit)
{
  if (!limit) return true;
  const double age = sc[SC_AGE], W = sc[SC_WEIGHT], dW = sc[SC_DW];
  const double growth = pow(dW, age + 1.0);
  bool ok = true;
  if (age > 4.0) ok = false;
  if (growth > 5.0)
    ok = false;
  else if (W > 100.0 && growth > 1.5)
    ok = false;
  if (fabs((sc[SC_EL] - e_orig) / e_orig) > 100.0) ok = false;
  return ok;
}

__device__ __forceinline__ void branch_block(double *state, const Layout &L, int *live, int *live_tmp,
                                             int *free_stack, int *ctl, int2 *copies, double thr_split,
                                             double thr_fuse, uint64_t seed, int step, double *stats, double e_orig,
                                             int limit_branching)
{
  __shared__ int s_warp[32];
  __shared__ int s_base[4];
  __shared__ double s_wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int n = ctl[0];
  int nfree = ctl[1];
  // pass 1: pair fusion candidates in list order and decide
  int cand_base = 0;
  for (int c0 = 0; c0 < n; c0 += 1024) {
    int i = c0 + tid;
    int slot = i < n ? live[i] : -1;
    double w = slot >= 0 ? state[(size_t)slot * L.stride + L.sc + SC_WEIGHT] : 0.0;
    int is_c = (slot >= 0 && w <= thr_split && w >= 0.01 && w < thr_fuse) ? 1 : 0;
    // block exclusive scan of is_c
    unsigned b = __ballot_sync(QMCB_FULL_MASK, is_c);
    int wpre = __popc(b & ((1u << lane) - 1));
    if (lane == 31) s_warp[wid] = wpre + is_c;
    __syncthreads();
    if (wid == 0) {
      int v = s_warp[lane], x = v;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(QMCB_FULL_MASK, x, o);
        if (lane >= o) x += y;
      }
      s_warp[lane] = x - v;
      if (lane == 31) s_base[0] = x;
    }
    __syncthreads();
    int rank = cand_base + s_warp[wid] + wpre;  // global candidate rank
    int total = s_base[0];
    // candidate ranks are global over the whole list, so pairs (0,1), (2,3)
    // ... may straddle chunk boundaries.
    if (is_c) live_tmp[rank] = i;
    __syncthreads();
    cand_base += total;
  }
  __syncthreads();
  // decide pairs: candidate 2m and 2m+1
  for (int m = tid; 2 * m + 1 < cand_base; m += 1024) {
    int ia = live_tmp[2 * m], ib = live_tmp[2 * m + 1];
    int sa = live[ia], sb = live[ib];
    double *wa = &state[(size_t)sa * L.stride + L.sc + SC_WEIGHT];
    double *wb = &state[(size_t)sb * L.stride + L.sc + SC_WEIGHT];
    double w1 = *wa, w2 = *wb, w3 = w1 + w2;
    double u[4];
    rng_uniform4(seed, (uint32_t)ia, (uint32_t)step, 7u, u);
    if (u[0] < w1 / w3) {
      *wa = w3;
      *wb = -1.0;  // marked dead
      wa[SC_FUSED - SC_WEIGHT] = 1.0;
    } else {
      *wb = w3;
      *wa = -1.0;
      wb[SC_FUSED - SC_WEIGHT] = 1.0;
    }
  }
  __syncthreads();
  // pass 2: survivors keep list order; dead slots to the free stack; splits append copies
  int out_base = 0, split_base = 0;
  // first count survivors + kills to know where split copies go and how many slots free
  for (int c0 = 0; c0 < n; c0 += 1024) {
    int i = c0 + tid;
    int slot = i < n ? live[i] : -1;
    double w = slot >= 0 ? state[(size_t)slot * L.stride + L.sc + SC_WEIGHT] : 0.0;
    int dead = (slot >= 0 && w < 0.01) ? 1 : 0;
    int keep = (slot >= 0 && !dead) ? 1 : 0;
    unsigned bk = __ballot_sync(QMCB_FULL_MASK, keep), bd = __ballot_sync(QMCB_FULL_MASK, dead);
    int pk = __popc(bk & ((1u << lane) - 1)), pd = __popc(bd & ((1u << lane) - 1));
    if (lane == 31) s_warp[wid] = ((pk + keep) << 16) | (pd + dead);
    __syncthreads();
    if (wid == 0) {
      int v = s_warp[lane];
      int vk = v >> 16, vd = v & 0xffff, xk = vk, xd = vd;
      for (int o = 1; o < 32; o <<= 1) {
        int yk = __shfl_up_sync(QMCB_FULL_MASK, xk, o), yd = __shfl_up_sync(QMCB_FULL_MASK, xd, o);
        if (lane >= o) {
          xk += yk;
          xd += yd;
        }
      }
      s_warp[lane] = ((xk - vk) << 16) | (xd - vd);
      if (lane == 31) {
        s_base[1] = xk;
        s_base[2] = xd;
      }
    }
    __syncthreads();
    int ok = s_warp[wid] >> 16, od = s_warp[wid] & 0xffff;
    if (keep) live_tmp[out_base + ok + pk] = slot;
    if (dead) free_stack[nfree + od + pd] = slot;
    int tk = s_base[1], td = s_base[2];
    __syncthreads();
    out_base += tk;
    nfree += td;
  }
  __syncthreads();
  // splits among survivors (in new list order), appended at the end
  int n_keep = out_base;
  double wsum_part = 0.0;
  for (int c0 = 0; c0 < n_keep; c0 += 1024) {
    int i = c0 + tid;
    int slot = i < n_keep ? live_tmp[i] : -1;
    double *wp = slot >= 0 ? &state[(size_t)slot * L.stride + L.sc + SC_WEIGHT] : nullptr;
    double w = wp ? *wp : 0.0;
    // the split test reads the weight before fusion, as the reference's single
    // pass does: the survivor of a fused pair (weight below the fusion
    // threshold before) never splits in the same pass
    const bool fused = wp && wp[SC_FUSED - SC_WEIGHT] != 0.0;
    if (fused) wp[SC_FUSED - SC_WEIGHT] = 0.0;
    int sp = (slot >= 0 && !fused && w > thr_split &&
              branch_recommended(state + (size_t)slot * L.stride + L.sc, e_orig, limit_branching)) ? 1 : 0;
    unsigned bs = __ballot_sync(QMCB_FULL_MASK, sp);
    int ps = __popc(bs & ((1u << lane) - 1));
    if (lane == 31) s_warp[wid] = ps + sp;
    __syncthreads();
    if (wid == 0) {
      int v = s_warp[lane], x = v;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(QMCB_FULL_MASK, x, o);
        if (lane >= o) x += y;
      }
      s_warp[lane] = x - v;
      if (lane == 31) s_base[3] = x;
    }
    __syncthreads();
    int r = split_base + s_warp[wid] + ps;
    if (sp) {
      if (r < nfree) {
        int dst = free_stack[nfree - 1 - r];
        *wp = w * 0.5;
        copies[r] = make_int2(slot, dst);
        live_tmp[n_keep + r] = dst;
        wsum_part += w;  // both halves
      } else {
        wsum_part += w;  // no free slot: keep the walker whole
      }
    } else if (slot >= 0) {
      wsum_part += w;
    }
    int ts = s_base[3];
    __syncthreads();
    split_base += ts;
  }
  int n_split = min(split_base, nfree);
  __syncthreads();
  for (int i = tid; i < n_keep + n_split; i += 1024) live[i] = live_tmp[i];
  double ws = warp_sum(wsum_part);
  if (lane == 0) s_wsum[wid] = ws;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int k = 0; k < 32; k++) t += s_wsum[k];
    stats[ST_FINAL_W] = t;
    ctl[0] = n_keep + n_split;
    ctl[1] = nfree - n_split;
    ctl[2] = n_split;
  }
}

__global__ void __launch_bounds__(1024) k_branch(double *state, Layout L, int *live, int *live_tmp, int *free_stack,
                                                 int *ctl, int2 *copies, double thr_split, double thr_fuse,
                                                 uint64_t seed, int step, double *stats, double e_orig,
                                                 int limit_branching)
{
  branch_block(state, L, live, live_tmp, free_stack, ctl, copies, thr_split, thr_fuse, seed, step, stats, e_orig,
               limit_branching);
}

// Copies whole walker blocks for the splits recorded by k_branch; the copy
// keeps the halved weight already written to the source.
__device__ __forceinline__ void copy_blocks(double *state, const Layout &L, const int2 *copies, const int *ctl,
                                            int first, int stride)
{
  const int nc = ctl[2];
  for (int c = first; c < nc; c += stride) {
    int2 p = copies[c];
    const double *src = state + (size_t)p.x * L.stride;
    double *dst = state + (size_t)p.y * L.stride;
    for (int t = threadIdx.x; t < L.stride; t += blockDim.x) dst[t] = src[t];
  }
}

__global__ void k_copy(double *state, Layout L, const int2 *copies, const int *ctl)
{
  copy_blocks(state, L, copies, ctl, blockIdx.x, gridDim.x);
}

// E_est from the running weighted energy average and
// E_T = E_est - c ln(W / W0) (QMCManager::updateEstimatedEnergy /
// updateTrialEnergy, QMcBeaver/src/QMCManager.cpp:2247-2310).
// dyn_dt: also the effective time step dt <w p dR^2> / <w dR^2>
// (QMCDerivativeProperties::getEffectiveTimeStep, QMcBeaver/src/QMCDerivativeProperties.cpp:25-42).
__device__ __forceinline__ void update_energy(EnergyCtl *ectl, const double *stats, int min_samples_ok, int dyn_dt,
                                              double dt)
{
  if (dyn_dt && stats[ST_RUN_SUM_WD2] > 1e-20) ectl->dt_eff = dt * stats[ST_RUN_SUM_WPD2] / stats[ST_RUN_SUM_WD2];
  double sw = stats[ST_RUN_SUM_W];
  // E_est follows the running average once it holds 100 samples
  // (QMCManager::updateEstimatedEnergy, QMcBeaver/src/QMCManager.cpp:2247-2261)
  if (min_samples_ok && sw > 0.0 && stats[ST_RUN_COUNT] >= 100.0) ectl->e_est = stats[ST_RUN_SUM_WE] / sw;
  double ratio = stats[ST_FINAL_W] / ectl->target_weight;
  double lr = ratio > 1e-250 ? log(ratio) : 0.0;
  ectl->e_trial = ectl->e_est - ectl->pop_control * lr;
}

__global__ void k_energy(EnergyCtl *ectl, const double *stats, int min_samples_ok, int dyn_dt, double dt)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  update_energy(ectl, stats, min_samples_ok, dyn_dt, dt);
}

// Packs R, weight, E_L, log|psi|, sign of the first n live walkers into
// out[n][3N + 4] for one device-to-host copy.
__global__ void k_gather(const double *state, Layout L, int N, const int *live, int n, double *out)
{
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = lane_id();
  if (w >= n) return;
  const double *blk = state + (size_t)live[w] * L.stride;
  double *o = out + (size_t)w * (3 * N + 4);
  for (int t = lane; t < 3 * N; t += 32) o[t] = blk[L.R + t];
  if (lane == 0) {
    const double *sc = blk + L.sc;
    o[3 * N] = sc[SC_WEIGHT];
    o[3 * N + 1] = sc[SC_EL];
    o[3 * N + 2] = sc[SC_LOGDET_A] + sc[SC_LOGDET_B] + sc[SC_U];
    o[3 * N + 3] = sc[SC_SIGN_A] * sc[SC_SIGN_B];
  }
}

// Sets the weights of the first n live walkers.
__global__ void k_set_weights(double *state, Layout L, const int *live, int n, const double *w)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    state[(size_t)live[i] * L.stride + L.sc + SC_WEIGHT] = w[i];
}

// Per-walker evaluate outputs moved from the device buffer into mapped
// page-locked host arrays with consecutive threads on consecutive elements,
// so the stores cross the bus as full packets (the evaluate kernels store a
// walker's scalars from one lane, one 8-byte packet each).  Segment
// blockIdx.y: bytes[y] bytes from src[y] to dst[y]; whole 8-byte words when
// both ends and the length allow it, bytes otherwise.
struct PutList {
  const void *src[8];
  void *dst[8];
  size_t bytes[8];
};

__global__ void k_put_outputs(PutList P)
{
  const int y = blockIdx.y;
  const size_t n = P.bytes[y];
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, di = (size_t)gridDim.x * blockDim.x;
  if (((uintptr_t)P.src[y] | (uintptr_t)P.dst[y] | n) % 8 == 0) {
    const unsigned long long *s = (const unsigned long long *)P.src[y];
    unsigned long long *d = (unsigned long long *)P.dst[y];
    for (size_t i = i0; i < n / 8; i += di) d[i] = s[i];
  } else {
    const unsigned char *s = (const unsigned char *)P.src[y];
    unsigned char *d = (unsigned char *)P.dst[y];
    for (size_t i = i0; i < n; i += di) d[i] = s[i];
  }
}

}  // namespace qmcb
