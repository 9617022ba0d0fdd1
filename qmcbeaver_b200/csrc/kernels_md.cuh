// kernels_md.cuh -- the walker-path kernels for several determinants,
// psi_D = sum_c ci[c] det_alpha(c) det_beta(c) (FP64 only).
//
// Same execution model as kernels.cuh: one warp per walker.  Each spin keeps
// the orbital rows of its ACTIVE orbitals (every orbital some determinant
// occupies) once, and per determinant its own inverse, gradient ratios and
// (ln|det|, sign, laplacian ratio, singular).  That determinant block is
// double-buffered: a proposed move writes the updated block of the moved
// spin into the idle copy and an accepted move flips the spin's copy index
// (SC_MDCUR_A/B), so a rejection costs no copy back.
//
//   k_full_md   full evaluation or refresh from the stored rows
//   k_move_md   one single-electron move: a Sherman-Morrison row update of
//               every determinant, the determinant-weighted ratio sums, then
//               the same Jastrow / energy / acceptance steps as k_move
//
// As in the reference, a full evaluation factors the first determinant and
// reaches each further one by column swaps from the previous one
// (QMcBeaver/src/QMCSlater.cpp:666-712), falling back to an LU when a swap
// ratio is zero.
#pragma once

#include "kernels.cuh"

namespace qmcb {

// Per-warp scratch (doubles) of k_full_md and k_move_md.
__host__ __device__ inline int full_md_scratch_doubles(int N, int K, int nmax, int amax, int ndet)
{
  return even(5 * (K + 1)) + even(5 * amax) + 2 * nmax * nmax + 2 * even(nmax) + even(3 * N) + even(ndet) + 8;
}
// chi rows of the move kernel; the basis pass's exponential slots follow
// them into the gr .. valc space (written only after the contraction)
// tbneed: doubles of three-body scratch (3 N M, or 0), also taken from the
// chi .. valc space before the basis
__host__ __device__ inline int move_md_chi_doubles(int N, int K, int nmax, int amax, int ndet, int nslot,
                                                   int tbneed)
{
  const int rest = 2 * even(3 * N) + even(5 * amax) + 2 * even(ndet) + even(nmax);
  // after the contraction the chi rows hold every determinant's
  // Sherman-Morrison factors, laplacian partial sums and 1 / ratio
  return even(max(max(max(5 * K, 5 * K + nslot - rest), tbneed - rest), 2 * ndet * nmax + ndet));
}
__host__ __device__ inline int move_md_scratch_doubles(int N, int K, int nmax, int amax, int ndet, int tail, int nslot,
                                                       int tbneed)
{
  return move_md_chi_doubles(N, K, nmax, amax, ndet, nslot, tbneed) + 2 * even(3 * N) + even(5 * amax) +
         2 * even(ndet) + even(nmax) + even(3 * N) + even(tail) + 2;
}

// One copy of spin sp's determinant block.
struct MdBlock {
  double *inv;   // [ndet][n][n]
  double *g;     // [ndet][n][3]
  double *dsc;   // [ndet][4] ln|det|, sign, lap ratio, singular
};
__device__ __forceinline__ MdBlock md_block(const DevSys &S, const Layout &L, double *blk, int sp, int copy)
{
  const int n = sp ? S.nb : S.na;
  MdBlock b;
  b.inv = blk + L.Inv[sp] + (size_t)copy * L.mdsz[sp];
  b.g = b.inv + (size_t)S.ndet * n * n;
  b.dsc = b.g + (size_t)S.ndet * 3 * n;
  return b;
}

// Column `col` of the matrix whose inverse is X (X[o][e], n x n, shared)
// becomes column `col` of A (A[e][o]): Array2D::inverseUpdateOneColumn
// (QMcBeaver/include/Array2D.h:1628-1671).  v: scratch of n.  Returns the
// determinant ratio.
__device__ inline double inverse_update_col_warp(double *X, const double *A, double *v, int n, int col)
{
  const int lane = lane_id();
  double p = 0.0;
  for (int c = lane; c < n; c += 32) p += A[c * n + col] * X[col * n + c];
  const double ratio = warp_sum(p);
  const double q = 1.0 / ratio;
  for (int r = lane; r < n; r += 32) {
    double val = 0.0;
    if (r != col)
      for (int l = 0; l < n; l++) val += A[l * n + col] * X[r * n + l];
    v[r] = val * q;
  }
  __syncwarp();
  for (int t = lane; t < n * n; t += 32) {
    const int r = t / n, c = t - r * n;
    if (r != col) X[t] -= v[r] * X[col * n + c];
  }
  __syncwarp();
  for (int c = lane; c < n; c += 32) X[col * n + c] *= q;
  __syncwarp();
  return ratio;
}

// Relative determinant weights termPR[c] = ci[c] det_a(c) det_b(c) / psi_D
// (QMCSCFJastrow::update_SCF, QMcBeaver/src/QMCSCFJastrow.cpp:284-305),
// scaled by the largest |det_a det_b| so that nothing under- or overflows.
// dA / dB: the (ln|det|, sign, lap, singular) rows of each spin (null for a
// spin without electrons).  Writes tpr[ndet] (shared), returns ln|psi_D|,
// its sign and whether some determinant is singular.
__device__ inline void md_weights(const DevSys &S, const double *dA, const double *dB, double *tpr, double &logD,
                                  double &sgnD, bool &sing)
{
  const int lane = lane_id(), nd = S.ndet;
  double lmax = -INFINITY;
  bool sg = false;
  for (int c = lane; c < nd; c += 32) {
    const double l = (dA ? dA[4 * c] : 0.0) + (dB ? dB[4 * c] : 0.0);
    if (S.ci[c] != 0.0) lmax = fmax(lmax, l);
    if ((dA && dA[4 * c + 3] != 0.0) || (dB && dB[4 * c + 3] != 0.0)) sg = true;
  }
  lmax = warp_max(lmax);
  sing = __any_sync(QMCB_FULL_MASK, sg);
  double part = 0.0;
  for (int c = lane; c < nd; c += 32) {
    const double l = (dA ? dA[4 * c] : 0.0) + (dB ? dB[4 * c] : 0.0);
    const double s = (dA ? dA[4 * c + 1] : 1.0) * (dB ? dB[4 * c + 1] : 1.0);
    const double t = S.ci[c] * s * exp(l - lmax);
    tpr[c] = t;
    part += t;
  }
  const double D = warp_sum(part);
  __syncwarp();
  const double iD = 1.0 / D;
  for (int c = lane; c < nd; c += 32) tpr[c] *= iD;
  __syncwarp();
  logD = lmax + log(fabs(D));
  sgnD = D < 0 ? -1.0 : 1.0;
  if (!(D != 0.0) || !isfinite(logD)) sing = true;
}

// grad(D)/D of every electron and lap(D)/D from the per-determinant ratios
// and the weights: D_x = sum_c termPR_c rDc_x(c), D_xx = sum_c termPR_c
// (lapA_c + lapB_c) (QMcBeaver/src/QMCSCFJastrow.cpp:307-327).
__device__ inline double md_combine(const DevSys &S, const MdBlock *blkA, const MdBlock *blkB, const double *tpr,
                                    double *gD)
{
  const int lane = lane_id(), nd = S.ndet, N = S.N;
  double lp = 0.0;
  for (int c = lane; c < nd; c += 32) {
    double l = 0.0;
    if (S.na > 0) l += blkA->dsc[4 * c + 2];
    if (S.nb > 0) l += blkB->dsc[4 * c + 2];
    lp += tpr[c] * l;
  }
  for (int i = lane; i < N; i += 32) {
    const bool a = i < S.na;
    const int n = a ? S.na : S.nb, el = a ? i : i - S.na;
    const double *g = a ? blkA->g : blkB->g;
    double gx = 0, gy = 0, gz = 0;
    for (int c = 0; c < nd; c++) {
      const double t = tpr[c];
      const double *gc = g + ((size_t)c * n + el) * 3;
      gx += t * gc[0];
      gy += t * gc[1];
      gz += t * gc[2];
    }
    gD[3 * i] = gx;
    gD[3 * i + 1] = gy;
    gD[3 * i + 2] = gz;
  }
  return warp_sum(lp);
}

// ------------------------------------------------------------------------
// Full evaluation (do_basis = true) or refresh from the stored rows.
__global__ void __launch_bounds__(128) k_full_md(DevSys S, Layout L, RunCfg cfg, double *state, const int *slots,
                                                 int num, const int *d_num, const double *R_in, int do_basis,
                                                 EvalOut out)
{
  extern __shared__ double smem[];
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  const int nw = d_num ? *d_num : num;
  const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (wi >= nw) return;
  const int N = S.N, K = S.K, nmax = max(S.na, S.nb), amax = max(S.nact[0], S.nact[1]), nd = S.ndet;
  const int slot = slots ? slots[wi] : wi;
  double *blk = state + (size_t)slot * L.stride;
  double *sm = smem + (size_t)warp * full_md_scratch_doubles(N, K, nmax, amax, nd);
  const int ldc = K + 1;
  double *chi = sm;
  double *Dn = chi + even(5 * ldc);
  double *A = Dn + even(5 * amax);
  double *X = A + nmax * nmax;
  double *vv = X + nmax * nmax;
  double *piv = vv + even(nmax);
  double *Rs = piv + even(nmax);
  double *tpr = Rs + even(3 * N);
  double *R = blk + L.R;
  double *sc = blk + L.sc;

  if (R_in) {
    for (int t = lane; t < 3 * N; t += 32) R[t] = R_in[(size_t)wi * 3 * N + t];
    if (lane < 2) sc[SC_MDCUR_A + lane] = 0.0;
  }
  for (int t = lane; t < 3 * N; t += 32) Rs[t] = R[t];
  __syncwarp();

  MdBlock mb[2];
  for (int sp = 0; sp < 2; sp++) mb[sp] = md_block(S, L, blk, sp, sc[SC_MDCUR_A + sp] != 0.0 ? 1 : 0);
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? S.nb : S.na, a = S.nact[sp], base = sp ? S.na : 0;
    if (n == 0) continue;
    double *Dv = blk + L.Dv[sp], *DgT = blk + L.DgT[sp], *DlT = blk + L.DlT[sp];
    if (do_basis) {
      for (int e = 0; e < n; e++) {
        const double r[3] = {Rs[3 * (base + e)], Rs[3 * (base + e) + 1], Rs[3 * (base + e) + 2]};
        basis_shells_warp(S, r, chi, ldc);
        __syncwarp();
        contract_dmma_warp(chi, ldc, S.ct[sp], a, K, Dn);
        __syncwarp();
        if (S.cusp) {
          cusp_replace_warp(S, sp, r, Dn, a, a);
          __syncwarp();
        }
        for (int o = lane; o < a; o += 32) {
          Dv[e * a + o] = Dn[o];
          DgT[(0 * a + o) * n + e] = Dn[a + o];
          DgT[(1 * a + o) * n + e] = Dn[2 * a + o];
          DgT[(2 * a + o) * n + e] = Dn[3 * a + o];
          DlT[o * n + e] = Dn[4 * a + o];
        }
        __syncwarp();
      }
    }
    double logdet = 0.0, sign = 1.0;
    bool ok = true;
    for (int c = 0; c < nd; c++) {
      const int *occ = S.docc[sp] + (size_t)c * n;
      // QMCWavefunction::getDataForCI: the columns of determinant c
      for (int t = lane; t < n * n; t += 32) A[t] = Dv[(t / n) * a + occ[t % n]];
      __syncwarp();
      bool lu = c == 0;
      if (c > 0 && ok) {
        // swap in the columns that differ from determinant c-1
        const int *sw = S.dswap[sp] + (size_t)c * n;
        for (int k = 0; k < n && sw[k] >= 0; k++) {
          const double r = inverse_update_col_warp(X, A, vv, n, sw[k]);
          if (!(r != 0.0) || !isfinite(r)) {
            lu = true;
            break;
          }
          logdet += log(fabs(r));
          if (r < 0) sign = -sign;
        }
      } else if (c > 0) {
        lu = true;
      }
      if (lu) {
        for (int t = lane; t < n * n; t += 32) A[t] = Dv[(t / n) * a + occ[t % n]];
        __syncwarp();
        ok = lu_inverse_warp(A, X, vv, piv, n, logdet, sign);
      }
      double *Inv = mb[sp].inv + (size_t)c * n * n;
      for (int t = lane; t < n * n; t += 32) Inv[t] = X[t];
      // ratio sums of determinant c (QMcBeaver/src/QMCSlater.cpp:741-762)
      double lp = 0.0;
      for (int e = lane; e < n; e += 32) {
        double gx = 0, gy = 0, gz = 0;
        for (int o = 0; o < n; o++) {
          const int orb = occ[o];
          const double iv = X[o * n + e];
          lp += DlT[orb * n + e] * iv;
          gx += DgT[(0 * a + orb) * n + e] * iv;
          gy += DgT[(1 * a + orb) * n + e] * iv;
          gz += DgT[(2 * a + orb) * n + e] * iv;
        }
        double *g = mb[sp].g + ((size_t)c * n + e) * 3;
        g[0] = gx;
        g[1] = gy;
        g[2] = gz;
      }
      lp = warp_sum(lp);
      if (lane == 0) {
        double *d = mb[sp].dsc + 4 * c;
        d[0] = ok ? logdet : 0.0;
        d[1] = ok ? sign : 1.0;
        d[2] = ok ? lp : 0.0;
        d[3] = ok ? 0.0 : 1.0;
      }
      __syncwarp();
    }
  }

  double logD, sgnD;
  bool bad;
  md_weights(S, S.na > 0 ? mb[0].dsc : nullptr, S.nb > 0 ? mb[1].dsc : nullptr, tpr, logD, sgnD, bad);
  double *gD = blk + L.gradD, *gr = blk + L.grad, *mg = blk + L.mgrad, *ux = blk + L.Ux;
  const double Dxx = md_combine(S, &mb[0], &mb[1], tpr, gD);
  double U, Uxx, Vee, Ven;
  jastrow_pe_full_warp<true>(S, Rs, ux, U, Uxx, Vee, Ven);
  __syncwarp();
  const double lap = psi_lap_warp(N, gD, ux, gr, Dxx, Uxx);
  __syncwarp();
  const double modratio = qf_modify_warp(S, cfg, Rs, gr, mg, &bad);
  const double PE = S.Pnn + Vee + Ven;
  const double EL = -0.5 * lap + PE;
  if (lane == 0) {
    sc[SC_U] = U;
    sc[SC_UXX] = Uxx;
    sc[SC_VEE] = Vee;
    sc[SC_VEN] = Ven;
    sc[SC_PE] = PE;
    sc[SC_EL] = EL;
    sc[SC_LAP] = lap;
    sc[SC_MODRATIO] = modratio;
    sc[SC_LOGDET_A] = logD;
    sc[SC_LOGDET_B] = 0.0;
    sc[SC_SIGN_A] = sgnD;
    sc[SC_SIGN_B] = 1.0;
    sc[SC_LAPR_A] = Dxx;
    sc[SC_LAPR_B] = 0.0;
    unsigned st = bad ? 1u : 0u;
    if (isnan(EL) || isnan(lap)) st |= 2u;
    sc[SC_STATUS] = (double)st;
    if (R_in) {
      sc[SC_WEIGHT] = 1.0;
      sc[SC_AGE] = 0.0;
      sc[SC_AGE_MOVED] = 0.0;
      sc[SC_DW] = 1.0;
    }
  }
  __syncwarp();
  write_eval_out(out, wi, N, logD + U, sgnD, lap, EL, PE, Ven, Vee, bad, gr, mg);
}

// ------------------------------------------------------------------------
// One single-electron move of every walker in the list (see k_move).
// md_move_walker: the work of one warp on walker wi (sm: its
// move_md_scratch_doubles of shared memory); k_move_md runs it for one
// system, k_move_group for the walkers of many.
template <bool kMetropolis>
__device__ __forceinline__ void md_move_walker(const DevSys &S, const Layout &L, const RunCfg &cfg, double *state,
                                               const int *slots, int wi, double *sm, const double *R_in,
                                               const MoveArgs &mv, const EnergyCtl *ectl, double *stats,
                                               const EvalOut &out)
{
  const int lane = lane_id();
  const int N = S.N, K = S.K, nd = S.ndet;
  const int nmax = max(S.na, S.nb), amax = max(S.nact[0], S.nact[1]);
  const int e = mv.e;
  const int sp = e < S.na ? 0 : 1, osp = 1 - sp;
  const int n = sp ? S.nb : S.na, a = S.nact[sp], base = sp ? S.na : 0, el = e - base;
  const int slot = slots ? slots[wi] : wi;
  double *blk = state + (size_t)slot * L.stride;
  const int tail = L.sc + kScalars - L.gradD;

  const int tbneed = S.ntb > 0 ? 3 * N * S.M : 0;
  double *chi = sm;
  double *gr = chi + move_md_chi_doubles(N, K, nmax, amax, nd, S.nslot, tbneed);
  double *mg = gr + even(3 * N);
  double *Dn = mg + even(3 * N);       // new rows of the active orbitals [5][a]
  double *rat = Dn + even(5 * amax);   // per-determinant ratios
  double *tpr = rat + even(nd);        // determinant weights
  double *valc = tpr + even(nd);       // Sherman-Morrison factors [n]
  double *sR = valc + even(nmax);
  double *sT = sR + even(3 * N);       // gradD, Ux, grad, mgrad, scalars
  double *gD = sT;
  double *Ux = sT + (L.Ux - L.gradD);
  const double *mgo = sT + (L.mgrad - L.gradD);
  const double *sc0 = sT + (L.sc - L.gradD);
  double *sc = blk + L.sc;
  const double *DgT = blk + L.DgT[sp], *DlT = blk + L.DlT[sp];

  for (int t = lane; t < 3 * N; t += 32) sR[t] = blk[L.R + t];
  for (int t = lane; t < tail; t += 32) sT[t] = blk[L.gradD + t];
  __syncwarp();

  const double ro[3] = {sR[3 * e], sR[3 * e + 1], sR[3 * e + 2]};
  double rn[3], g_fwd, u_acc;
  propose_move<kMetropolis, true>(S, cfg, slot, mv.step, e, N, sR, ro, mgo, R_in, wi, rn, g_fwd, u_acc, mv.rin_moved);
  double dU, dUxx, dVee, dVen;
  jastrow_pe_move_warp<true>(S, sR, Ux, e, sp, ro, rn, dU, dUxx, dVee, dVen, chi);

  basis_slots_warp(S, rn, chi, K, chi + 5 * K);
  __syncwarp();
  contract_dmma_warp(chi, K, S.ct[sp], a, K, Dn);
  __syncwarp();
  if (S.cusp) {
    cusp_replace_warp(S, sp, rn, Dn, a, a);
    __syncwarp();
  }

  const int cur = sc0[SC_MDCUR_A + sp] != 0.0 ? 1 : 0;
  const MdBlock src = md_block(S, L, blk, sp, cur), dst = md_block(S, L, blk, sp, 1 - cur);
  const MdBlock oth = md_block(S, L, blk, osp, sc0[SC_MDCUR_A + osp] != 0.0 ? 1 : 0);
  const int no = osp ? S.nb : S.na;

  // ---- weights before the move and every determinant's ratio
  double logD0, sgnD0;
  bool bad;
  md_weights(S, sp == 0 ? src.dsc : (no > 0 ? oth.dsc : nullptr), sp == 1 ? src.dsc : (no > 0 ? oth.dsc : nullptr),
             tpr, logD0, sgnD0, bad);
  // lane c takes determinant c's row ratio
  bool zero_ratio = false;
  for (int c = lane; c < nd; c += 32) {
    const int *occ = S.docc[sp] + (size_t)c * n;
    const double *Inv = src.inv + (size_t)c * n * n;
    double r = 0.0;
    for (int o = 0; o < n; o++) r = fma(Dn[occ[o]], Inv[o * n + el], r);
    rat[c] = r;
    if (!(r != 0.0) || !isfinite(r)) zero_ratio = true;
  }
  zero_ratio = __any_sync(QMCB_FULL_MASK, zero_ratio);
  __syncwarp();
  double rpart = 0.0;
  for (int c = lane; c < nd; c += 32) rpart += tpr[c] * rat[c];
  const double RD = warp_sum(rpart);
  if (zero_ratio || !(RD != 0.0) || !isfinite(RD)) bad = true;
  const double iRD = 1.0 / RD;

  // ---- Sherman-Morrison row update of every determinant into the idle
  //      copy (Array2D::inverseUpdateOneRow, QMcBeaver/include/Array2D.h:1567-1610)
  //      and its ratio sums with the new inverse; the lanes share out the
  //      determinants' columns, elements and electrons (the chi rows, free
  //      after the contraction, hold the factors and partial sums)
  double *vall = chi;                    // [nd][n] factors
  double *lpp = chi + nd * n;            // [nd][n] laplacian partial sums
  double *qd = chi + 2 * nd * n;         // [nd] 1 / ratio
  for (int c = lane; c < nd; c += 32) qd[c] = 1.0 / rat[c];
  __syncwarp();
  for (int t = lane; t < nd * n; t += 32) {
    const int c = t / n, col = t - c * n;
    const int *occ = S.docc[sp] + (size_t)c * n;
    const double *Iv = src.inv + (size_t)c * n * n;
    double v = 0.0;
    if (col != el)
      for (int l = 0; l < n; l++) v = fma(Dn[occ[l]], Iv[l * n + col], v);
    vall[t] = v * qd[c];
  }
  __syncwarp();
  for (int u = lane; u < nd * n * n; u += 32) {
    const int c = u / (n * n), t = u - c * n * n, r = t / n, col = t - r * n;
    const double *Iv = src.inv + (size_t)c * n * n;
    dst.inv[u] = col == el ? Iv[r * n + el] * qd[c] : Iv[t] - vall[c * n + col] * Iv[r * n + el];
  }
  __syncwarp();
  for (int t = lane; t < nd * n; t += 32) {
    const int c = t / n, e2 = t - c * n;
    const int *occ = S.docc[sp] + (size_t)c * n;
    const double *Iw = dst.inv + (size_t)c * n * n;
    double gx = 0, gy = 0, gz = 0, lp = 0;
    for (int o = 0; o < n; o++) {
      const int orb = occ[o];
      const double iv = Iw[o * n + e2];
      if (e2 == el) {
        gx = fma(Dn[a + orb], iv, gx);
        gy = fma(Dn[2 * a + orb], iv, gy);
        gz = fma(Dn[3 * a + orb], iv, gz);
        lp = fma(Dn[4 * a + orb], iv, lp);
      } else {
        gx = fma(DgT[(0 * a + orb) * n + e2], iv, gx);
        gy = fma(DgT[(1 * a + orb) * n + e2], iv, gy);
        gz = fma(DgT[(2 * a + orb) * n + e2], iv, gz);
        lp = fma(DlT[orb * n + e2], iv, lp);
      }
    }
    double *g = dst.g + ((size_t)c * n + e2) * 3;
    g[0] = gx;
    g[1] = gy;
    g[2] = gz;
    lpp[t] = lp;
  }
  __syncwarp();
  for (int c = lane; c < nd; c += 32) {
    double lp = 0.0;
    for (int e2 = 0; e2 < n; e2++) lp += lpp[c * n + e2];
    const double *d0 = src.dsc + 4 * c;
    double *d = dst.dsc + 4 * c;
    d[0] = d0[0] + log(fabs(rat[c]));
    d[1] = d0[1] * (rat[c] < 0 ? -1.0 : 1.0);
    d[2] = lp;
    d[3] = (!(rat[c] != 0.0) || !isfinite(rat[c])) ? 1.0 : d0[3];
  }
  __syncwarp();

  // ---- new weights termPR'_c = termPR_c ratio_c / R_D and the combined ratios
  for (int c = lane; c < nd; c += 32) tpr[c] *= rat[c] * iRD;
  __syncwarp();
  const double Dxx = sp == 0 ? md_combine(S, &dst, &oth, tpr, gD) : md_combine(S, &oth, &dst, tpr, gD);
  __syncwarp();

  const double U_new = sc0[SC_U] + dU, Uxx_new = sc0[SC_UXX] + dUxx;
  const double lap = psi_lap_warp(N, gD, Ux, gr, Dxx, Uxx_new);
  __syncwarp();
  const double modratio = qf_modify_warp(S, cfg, sR, gr, mg, &bad);
  const double Vee = sc0[SC_VEE] + dVee, Ven = sc0[SC_VEN] + dVen;
  const double PE = S.Pnn + Vee + Ven;
  const double EL = -0.5 * lap + PE;
  if (isnan(EL)) bad = true;
  const double logD_new = logD0 + log(fabs(RD));
  const double sgnD_new = sgnD0 * (RD < 0 ? -1.0 : 1.0);

  bool accept = true;
  if (kMetropolis) {
    double p_acc;
    accept = metropolis_reweight<true>(S, cfg, mv, ectl, stats, sc, sc0, N, e, sR, ro, rn, mg, g_fwd, u_acc,
                                 log(fabs(RD)) + dU, RD < 0, bad, EL, modratio, p_acc);
    if (mv.dump)
      dump_configs(mv.dump, wi, N, e, sR, ro, Dxx, gD, U_new, PE, sc0[SC_LAPR_A], blk + L.gradD, sc0[SC_U],
                   sc0[SC_PE], p_acc);
  }
  __syncwarp();

  if (accept) {
    double *Rw = blk + L.R;
    if (lane < 3) Rw[3 * e + lane] = rn[lane];
    double *Dv = blk + L.Dv[sp], *DgW = blk + L.DgT[sp], *DlW = blk + L.DlT[sp];
    for (int o = lane; o < a; o += 32) {
      Dv[el * a + o] = Dn[o];
      DgW[(0 * a + o) * n + el] = Dn[a + o];
      DgW[(1 * a + o) * n + el] = Dn[2 * a + o];
      DgW[(2 * a + o) * n + el] = Dn[3 * a + o];
      DlW[o * n + el] = Dn[4 * a + o];
    }
    for (int t = lane; t < 3 * N; t += 32) {
      blk[L.gradD + t] = gD[t];
      blk[L.Ux + t] = Ux[t];
      blk[L.mgrad + t] = mg[t];
      if (!kMetropolis) blk[L.grad + t] = gr[t];
    }
    if (lane == 0) {
      sc[SC_MDCUR_A + sp] = (double)(1 - cur);
      sc[SC_U] = U_new;
      sc[SC_UXX] = Uxx_new;
      sc[SC_LAPR_A] = Dxx;
      sc[SC_LOGDET_A] = logD_new;
      sc[SC_SIGN_A] = sgnD_new;
      sc[SC_VEE] = Vee;
      sc[SC_VEN] = Ven;
      sc[SC_PE] = PE;
      sc[SC_EL] = EL;
      sc[SC_LAP] = lap;
      sc[SC_MODRATIO] = modratio;
      sc[SC_STATUS] = bad ? 1.0 : 0.0;
    }
  }
  if (!kMetropolis) write_eval_out(out, wi, N, logD_new + U_new, sgnD_new, lap, EL, PE, Ven, Vee, bad, gr, mg);
}

template <bool kMetropolis>
__global__ void __launch_bounds__(128, 3) k_move_md(DevSys S, Layout L, RunCfg cfg, double *state, const int *slots,
                                                 int num, const int *d_num, const double *R_in, MoveArgs mv,
                                                 const EnergyCtl *ectl, double *stats, EvalOut out)
{
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5;
  const int nw = d_num ? *d_num : num;
  const int wi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (wi >= nw) return;
  const int nmax = max(S.na, S.nb), amax = max(S.nact[0], S.nact[1]);
  const int tail = L.sc + kScalars - L.gradD, tbneed = S.ntb > 0 ? 3 * S.N * S.M : 0;
  double *sm = smem + (size_t)warp * move_md_scratch_doubles(S.N, S.K, nmax, amax, S.ndet, tail, S.nslot, tbneed);
  md_move_walker<kMetropolis>(S, L, cfg, state, slots, wi, sm, R_in, mv, ectl, stats, out);
}

}  // namespace qmcb
