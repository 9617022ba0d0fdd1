/*
 * qmc_oracle.c -- CPU restatement of QMcBeaver's Slater-Jastrow walker
 * evaluation.  TEST INFRASTRUCTURE ONLY (the checker for the CUDA path).
 *
 * Each routine follows the reference function named beside it, with the
 * same loop orders and operation order, including the long double
 * accumulators of the LU decomposition, so that it reproduces the reference
 * to the last bits on the same inputs.  Pinned by tests/test_oracle.py
 * against the reference built from its own sources (oracle/_ref) and the
 * committed golden vectors.
 */
#include "qmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct orc_system {
  int M, na, nb, N, K;
  double *nuc_xyz, *nuc_z;
  int *bf_atom, *bf_pow, *bf_nprim, *bf_off;
  double *pexp, *pcoef;
  int *atom_first, *atom_nbf, *atom_lmax; /* per atom function ranges */
  double *mo_a, *mo_b;                    /* [nact][K] orbital rows of each spin */
  int ndet, nact[2];
  int *occ[2];                            /* [ndet][n] active row of each column */
  int *swaps[2];                          /* [ndet][n] columns replaced from det ci-1, -1 ends */
  double *ci;                             /* [ndet] */
  int cusp, nsmax;                        /* electron-nucleus cusp replacement */
  int *cns;                               /* [M] s primitives per nucleus */
  double *csexp;                          /* [M][nsmax] */
  double *cscoef[2];                      /* [M][nact][nsmax] */
  double *cpar[2];                        /* [M][nact][8] rc, sgn0, C, alpha_0..4 */
  int ntb;                                /* three-body functions */
  int *tb_nen, *tb_nee, *tb_C, *tb_off, *tb_pair;
  double *tb_cut, *tb_coef;
  int npade;
  double *pnum, *pden;
  int *pnn, *pnd;
  int *ctype;
  double *cparam;
  int ee[3];
  int *en_up, *en_dn;
  double Pnn;
  int qf_mod;
  double qf_a, dt;
};

struct orc_walker {
  const orc_system *s;
  double *inv[2];     /* [ndet][n][n] inv[o*n+e] per determinant (Dc_invA(ci) / Dc_invB(ci)) */
  double *Dx[2][3];   /* [n][nact] derivative rows, row = electron (D_xA) */
  double *Dxx[2];     /* [n][nact] (D_xxA) */
  double *Dv[2];      /* [n][nact] orbital values (Dw) */
  double *det[2];     /* [ndet] DcA(ci), DcB(ci) */
  double *rDx[2];     /* [ndet][n][3] grad ratios (rDc_xA(ci)) */
  double *rDxx[2];    /* [ndet] rDc_xxA(ci) */
  int *sing[2];       /* [ndet] */
  double *rij, *rij_uvec, *riA, *riA_uvec;
  double *Uij, *Uij_x, *Uij_xx, *UiA, *UiA_x, *UiA_xx;
  double U, U_xx;
  double *U_x;
  double D_xx;
  double *D_x, *grad, *mgrad;
  double E_L, KE, PE, neE, eeE, lap;
  int singular;
  double logpsi, sign;
  double kappa;       /* condition number of the determinant-weighted laplacian sum */
  double *tU, *tUxx, *tUx1, *tUx2;  /* three-body pair caches UijA, UijA_xx, UijA_x1, UijA_x2 [N][N](x3) */
};

static double *dup_d(const double *p, size_t n)
{
  double *q = (double *)malloc(sizeof(double) * (n ? n : 1));
  if (n) memcpy(q, p, sizeof(double) * n);
  return q;
}
static int *dup_i(const int *p, size_t n)
{
  int *q = (int *)malloc(sizeof(int) * (n ? n : 1));
  if (n) memcpy(q, p, sizeof(int) * n);
  return q;
}

/* The order in which determinant ci's columns are swapped in from
 * determinant ci-1 so that no intermediate matrix holds one orbital twice
 * (QMCWavefunction::makeCoefficients, QMcBeaver/src/QMCWavefunction.cpp:924-976).
 * idx: [ndet][n] active rows; swaps: [ndet][n] receives the columns, -1 ends.
 * (The reference loops until no blocked swap is left; sorted occupation
 * lists never block for good, the loop here stops after n passes.) */
static void make_swaps(const int *idx, int ndet, int n, int *swaps)
{
  int *iu = dup_i(idx, (size_t)ndet * n);
  for (int t = 0; t < ndet * n; t++) swaps[t] = -1;
  for (int ci = 1; ci < ndet; ci++) {
    int swap = 0, bad, pass = 0;
    do {
      bad = 0;
      for (int o = 0; o < n; o++) {
        if (iu[ci * n + o] == iu[(ci - 1) * n + o]) continue;
        int good = 1;
        for (int o2 = 0; o2 < n; o2++)
          if (o != o2 && iu[ci * n + o] == iu[(ci - 1) * n + o2]) {
            bad = 1;
            good = 0;
            break;
          }
        if (good) {
          iu[(ci - 1) * n + o] = iu[ci * n + o];
          swaps[ci * n + swap] = o;
          swap++;
        }
      }
    } while (bad && ++pass <= n);
  }
  free(iu);
}

orc_system *orc_system_new(const qmcb_system_desc *d, int qf_mod, double qf_a, double dt)
{
  orc_system *s = (orc_system *)calloc(1, sizeof(orc_system));
  s->M = d->n_nuclei;
  s->na = d->n_alpha;
  s->nb = d->n_beta;
  s->N = s->na + s->nb;
  s->K = d->n_basis;
  s->nuc_xyz = dup_d(d->nuc_xyz, 3 * s->M);
  s->nuc_z = dup_d(d->nuc_charge, s->M);
  s->bf_atom = dup_i(d->bf_atom, s->K);
  s->bf_pow = dup_i(d->bf_powers, 3 * s->K);
  s->bf_nprim = dup_i(d->bf_nprim, s->K);
  s->bf_off = dup_i(d->bf_prim_offset, s->K);
  s->pexp = dup_d(d->prim_exponent, d->n_prim_total);
  s->pcoef = dup_d(d->prim_coeff, d->n_prim_total);
  s->ndet = d->n_det > 1 ? d->n_det : 1;
  s->nact[0] = d->n_det > 1 ? d->n_act_alpha : s->na;
  s->nact[1] = d->n_det > 1 ? d->n_act_beta : s->nb;
  s->mo_a = dup_d(d->mo_alpha, (size_t)s->nact[0] * s->K);
  s->mo_b = dup_d(d->mo_beta, (size_t)s->nact[1] * s->K);
  s->ci = (double *)malloc(sizeof(double) * s->ndet);
  for (int c = 0; c < s->ndet; c++) s->ci[c] = d->n_det > 1 ? d->ci_coeff[c] : 1.0;
  for (int sp = 0; sp < 2; sp++) {
    int n = sp ? s->nb : s->na;
    const int *src = sp ? d->det_occ_beta : d->det_occ_alpha;
    s->occ[sp] = (int *)malloc(sizeof(int) * (size_t)s->ndet * (n ? n : 1));
    s->swaps[sp] = (int *)malloc(sizeof(int) * (size_t)s->ndet * (n ? n : 1));
    for (int c = 0; c < s->ndet; c++)
      for (int o = 0; o < n; o++) s->occ[sp][c * n + o] = d->n_det > 1 ? src[c * n + o] : o;
    make_swaps(s->occ[sp], s->ndet, n, s->swaps[sp]);
  }
  /* three-body Jastrow tables */
  s->ntb = d->n_tb;
  {
    int nt = s->ntb > 0 ? s->ntb : 1, ncoef = 0;
    s->tb_nen = (int *)calloc(nt, sizeof(int));
    s->tb_nee = (int *)calloc(nt, sizeof(int));
    s->tb_C = (int *)calloc(nt, sizeof(int));
    s->tb_off = (int *)calloc(nt, sizeof(int));
    s->tb_cut = (double *)calloc(nt, sizeof(double));
    s->tb_pair = (int *)malloc(sizeof(int) * 3 * s->M);
    for (int t = 0; t < 3 * s->M; t++) s->tb_pair[t] = s->ntb > 0 ? d->tb_pair[t] : -1;
    for (int f = 0; f < s->ntb; f++) {
      s->tb_nen[f] = d->tb_nen[f];
      s->tb_nee[f] = d->tb_nee[f];
      s->tb_C[f] = d->tb_C[f];
      s->tb_off[f] = d->tb_offset[f];
      s->tb_cut[f] = d->tb_cutoff[f];
      int e = d->tb_offset[f] + d->tb_nen[f] * d->tb_nen[f] * d->tb_nee[f];
      if (e > ncoef) ncoef = e;
    }
    s->tb_coef = dup_d(s->ntb > 0 ? d->tb_coeff : NULL, ncoef);
  }
  /* cusp replacement: the fitted records come with the descriptor; the s
   * parts (sTypeCoeffs, QMcBeaver/src/QMCElectronNucleusCusp.cpp:83-102) are
   * built here from the basis and the orbital rows */
  s->cusp = d->replace_cusps != 0;
  s->cns = (int *)calloc(s->M, sizeof(int));
  for (int k = 0; k < s->K; k++)
    if (s->bf_pow[3 * k] + s->bf_pow[3 * k + 1] + s->bf_pow[3 * k + 2] == 0) s->cns[s->bf_atom[k]] += s->bf_nprim[k];
  s->nsmax = 1;
  for (int a = 0; a < s->M; a++)
    if (s->cns[a] > s->nsmax) s->nsmax = s->cns[a];
  s->csexp = (double *)calloc((size_t)s->M * s->nsmax, sizeof(double));
  for (int a = 0; a < s->M; a++) {
    int cnt = 0;
    for (int k = 0; k < s->K; k++) {
      if (s->bf_atom[k] != a) continue;
      if (s->bf_pow[3 * k] + s->bf_pow[3 * k + 1] + s->bf_pow[3 * k + 2] != 0) continue;
      for (int l = 0; l < s->bf_nprim[k]; l++) s->csexp[(size_t)a * s->nsmax + cnt++] = s->pexp[s->bf_off[k] + l];
    }
  }
  for (int sp = 0; sp < 2; sp++) {
    int a_ = s->nact[sp] ? s->nact[sp] : 1;
    const double *mo = sp ? s->mo_b : s->mo_a;
    const double *given = sp ? d->cusp_beta : d->cusp_alpha;
    s->cpar[sp] = (double *)calloc((size_t)s->M * a_ * 8, sizeof(double));
    s->cscoef[sp] = (double *)calloc((size_t)s->M * a_ * s->nsmax, sizeof(double));
    if (!s->cusp || s->nact[sp] == 0) continue;
    if (given) memcpy(s->cpar[sp], given, sizeof(double) * (size_t)s->M * s->nact[sp] * 8);
    for (int a = 0; a < s->M; a++)
      for (int o = 0; o < s->nact[sp]; o++) {
        int cnt = 0;
        for (int k = 0; k < s->K; k++) {
          if (s->bf_atom[k] != a || s->bf_pow[3 * k] + s->bf_pow[3 * k + 1] + s->bf_pow[3 * k + 2] != 0) continue;
          for (int l = 0; l < s->bf_nprim[k]; l++)
            s->cscoef[sp][((size_t)a * s->nact[sp] + o) * s->nsmax + cnt++] = s->pcoef[s->bf_off[k] + l] * mo[(size_t)o * s->K + k];
        }
      }
  }
  s->npade = d->n_pade;
  s->pnum = dup_d(d->pade_num, (size_t)s->npade * QMCB_PADE_MAX);
  s->pden = dup_d(d->pade_den, (size_t)s->npade * QMCB_PADE_MAX);
  s->pnn = dup_i(d->pade_nnum, s->npade);
  s->pnd = dup_i(d->pade_nden, s->npade);
  s->ctype = (int *)calloc(s->npade ? s->npade : 1, sizeof(int));
  s->cparam = (double *)calloc(4 * (s->npade ? s->npade : 1), sizeof(double));
  for (int f = 0; f < s->npade; f++) {
    s->ctype[f] = d->corr_type ? d->corr_type[f] : QMCB_CORR_PADE;
    if (d->corr_param)
      for (int i = 0; i < 4; i++) s->cparam[4 * f + i] = d->corr_param[4 * f + i];
  }
  for (int i = 0; i < 3; i++) s->ee[i] = d->ee_pade[i];
  s->en_up = dup_i(d->en_pade_up, s->M);
  s->en_dn = dup_i(d->en_pade_dn, s->M);
  s->atom_first = (int *)calloc(s->M, sizeof(int));
  s->atom_nbf = (int *)calloc(s->M, sizeof(int));
  s->atom_lmax = (int *)calloc(s->M, sizeof(int));
  for (int a = 0; a < s->M; a++) s->atom_first[a] = -1;
  for (int k = 0; k < s->K; k++) {
    int a = s->bf_atom[k];
    if (s->atom_first[a] < 0) s->atom_first[a] = k;
    s->atom_nbf[a]++;
    int l = s->bf_pow[3 * k] + s->bf_pow[3 * k + 1] + s->bf_pow[3 * k + 2];
    if (l > s->atom_lmax[a]) s->atom_lmax[a] = l;
  }
  /* calc_P_nn, QMcBeaver/src/QMCPotential_Energy.cpp:285-307 */
  s->Pnn = 0.0;
  for (int i = 0; i < s->M; i++)
    for (int j = i + 1; j < s->M; j++) {
      const double *a = s->nuc_xyz + 3 * i, *b = s->nuc_xyz + 3 * j;
      double r = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) +
                      (a[2] - b[2]) * (a[2] - b[2]));
      s->Pnn += (s->nuc_z[i] * s->nuc_z[j]) / r;
    }
  s->qf_mod = qf_mod;
  s->qf_a = qf_a;
  s->dt = dt;
  return s;
}

void orc_system_free(orc_system *s)
{
  if (!s) return;
  free(s->nuc_xyz); free(s->nuc_z); free(s->bf_atom); free(s->bf_pow); free(s->bf_nprim);
  free(s->bf_off); free(s->pexp); free(s->pcoef); free(s->mo_a); free(s->mo_b); free(s->pnum);
  free(s->pden); free(s->pnn); free(s->pnd); free(s->ctype); free(s->cparam); free(s->en_up); free(s->en_dn);
  free(s->atom_first); free(s->atom_nbf); free(s->atom_lmax);
  free(s->ci);
  free(s->cns);
  free(s->csexp);
  free(s->tb_nen); free(s->tb_nee); free(s->tb_C); free(s->tb_off); free(s->tb_cut); free(s->tb_pair); free(s->tb_coef);
  for (int sp = 0; sp < 2; sp++) { free(s->occ[sp]); free(s->swaps[sp]); free(s->cpar[sp]); free(s->cscoef[sp]); }
  free(s);
}

int orc_num_electrons(const orc_system *s) { return s->N; }

/* ------------------------------------------------------------ walker state */
static void walker_alloc(orc_walker *w, const orc_system *s)
{
  int N = s->N, M = s->M, nd = s->ndet;
  w->s = s;
  for (int sp = 0; sp < 2; sp++) {
    int n = sp ? s->nb : s->na, a = s->nact[sp];
    size_t nn = (size_t)(n ? n * n : 1), na_ = (size_t)(n && a ? n * a : 1);
    w->inv[sp] = (double *)calloc(nn * nd, sizeof(double));
    for (int d = 0; d < 3; d++) w->Dx[sp][d] = (double *)calloc(na_, sizeof(double));
    w->Dxx[sp] = (double *)calloc(na_, sizeof(double));
    w->Dv[sp] = (double *)calloc(na_, sizeof(double));
    w->det[sp] = (double *)calloc(nd, sizeof(double));
    w->rDx[sp] = (double *)calloc((size_t)nd * N * 3, sizeof(double));
    w->rDxx[sp] = (double *)calloc(nd, sizeof(double));
    w->sing[sp] = (int *)calloc(nd, sizeof(int));
    for (int c = 0; c < nd; c++) w->det[sp][c] = 1.0;
  }
  w->rij = (double *)calloc((size_t)N * N, sizeof(double));
  w->rij_uvec = (double *)calloc((size_t)N * N * 3, sizeof(double));
  w->riA = (double *)calloc((size_t)N * M + 1, sizeof(double));
  w->riA_uvec = (double *)calloc((size_t)N * M * 3 + 1, sizeof(double));
  w->Uij = (double *)calloc((size_t)N * N, sizeof(double));
  w->Uij_x = (double *)calloc((size_t)N * N * 3, sizeof(double));
  w->Uij_xx = (double *)calloc((size_t)N * N, sizeof(double));
  w->UiA = (double *)calloc((size_t)N * M + 1, sizeof(double));
  w->UiA_x = (double *)calloc((size_t)N * M * 3 + 1, sizeof(double));
  w->UiA_xx = (double *)calloc((size_t)N * M + 1, sizeof(double));
  w->U_x = (double *)calloc((size_t)N * 3, sizeof(double));
  w->D_x = (double *)calloc((size_t)N * 3, sizeof(double));
  w->grad = (double *)calloc((size_t)N * 3, sizeof(double));
  w->mgrad = (double *)calloc((size_t)N * 3, sizeof(double));
  w->tU = (double *)calloc((size_t)N * N, sizeof(double));
  w->tUxx = (double *)calloc((size_t)N * N, sizeof(double));
  w->tUx1 = (double *)calloc((size_t)N * N * 3, sizeof(double));
  w->tUx2 = (double *)calloc((size_t)N * N * 3, sizeof(double));
}

orc_walker *orc_walker_new(const orc_system *s)
{
  orc_walker *w = (orc_walker *)calloc(1, sizeof(orc_walker));
  walker_alloc(w, s);
  return w;
}

void orc_walker_free(orc_walker *w)
{
  if (!w) return;
  for (int sp = 0; sp < 2; sp++) {
    free(w->inv[sp]);
    for (int d = 0; d < 3; d++) free(w->Dx[sp][d]);
    free(w->Dxx[sp]);
    free(w->Dv[sp]);
    free(w->det[sp]);
    free(w->rDx[sp]);
    free(w->rDxx[sp]);
    free(w->sing[sp]);
  }
  free(w->rij); free(w->rij_uvec); free(w->riA); free(w->riA_uvec); free(w->Uij); free(w->Uij_x);
  free(w->Uij_xx); free(w->UiA); free(w->UiA_x); free(w->UiA_xx); free(w->U_x); free(w->D_x);
  free(w->grad); free(w->mgrad);
  free(w->tU); free(w->tUxx); free(w->tUx1); free(w->tUx2);
  free(w);
}

void orc_walker_copy(orc_walker *dst, const orc_walker *src)
{
  const orc_system *s = src->s;
  int N = s->N, M = s->M, nd = s->ndet;
  for (int sp = 0; sp < 2; sp++) {
    int n = sp ? s->nb : s->na, a = s->nact[sp];
    size_t nn = (size_t)(n ? n * n : 1), na_ = (size_t)(n && a ? n * a : 1);
    memcpy(dst->inv[sp], src->inv[sp], nn * nd * sizeof(double));
    for (int d = 0; d < 3; d++) memcpy(dst->Dx[sp][d], src->Dx[sp][d], na_ * sizeof(double));
    memcpy(dst->Dxx[sp], src->Dxx[sp], na_ * sizeof(double));
    memcpy(dst->Dv[sp], src->Dv[sp], na_ * sizeof(double));
    memcpy(dst->det[sp], src->det[sp], nd * sizeof(double));
    memcpy(dst->rDx[sp], src->rDx[sp], (size_t)nd * N * 3 * sizeof(double));
    memcpy(dst->rDxx[sp], src->rDxx[sp], nd * sizeof(double));
    memcpy(dst->sing[sp], src->sing[sp], nd * sizeof(int));
  }
  memcpy(dst->rij, src->rij, (size_t)N * N * sizeof(double));
  memcpy(dst->rij_uvec, src->rij_uvec, (size_t)N * N * 3 * sizeof(double));
  memcpy(dst->riA, src->riA, ((size_t)N * M + 1) * sizeof(double));
  memcpy(dst->riA_uvec, src->riA_uvec, ((size_t)N * M * 3 + 1) * sizeof(double));
  memcpy(dst->Uij, src->Uij, (size_t)N * N * sizeof(double));
  memcpy(dst->Uij_x, src->Uij_x, (size_t)N * N * 3 * sizeof(double));
  memcpy(dst->Uij_xx, src->Uij_xx, (size_t)N * N * sizeof(double));
  memcpy(dst->UiA, src->UiA, ((size_t)N * M + 1) * sizeof(double));
  memcpy(dst->UiA_x, src->UiA_x, ((size_t)N * M * 3 + 1) * sizeof(double));
  memcpy(dst->UiA_xx, src->UiA_xx, ((size_t)N * M + 1) * sizeof(double));
  memcpy(dst->U_x, src->U_x, (size_t)N * 3 * sizeof(double));
  memcpy(dst->D_x, src->D_x, (size_t)N * 3 * sizeof(double));
  memcpy(dst->grad, src->grad, (size_t)N * 3 * sizeof(double));
  memcpy(dst->mgrad, src->mgrad, (size_t)N * 3 * sizeof(double));
  memcpy(dst->tU, src->tU, (size_t)N * N * sizeof(double));
  memcpy(dst->tUxx, src->tUxx, (size_t)N * N * sizeof(double));
  memcpy(dst->tUx1, src->tUx1, (size_t)N * N * 3 * sizeof(double));
  memcpy(dst->tUx2, src->tUx2, (size_t)N * N * 3 * sizeof(double));
  dst->U = src->U; dst->U_xx = src->U_xx; dst->D_xx = src->D_xx;
  dst->E_L = src->E_L; dst->KE = src->KE; dst->PE = src->PE; dst->neE = src->neE; dst->eeE = src->eeE;
  dst->lap = src->lap; dst->singular = src->singular; dst->logpsi = src->logpsi; dst->sign = src->sign;
}

orc_walker *orc_walker_clone(const orc_walker *w)
{
  orc_walker *c = orc_walker_new(w->s);
  orc_walker_copy(c, w);
  return c;
}

/* ------------------------------------------------------- distances (a8) */
/* QMCWalkerData::updateDistances, QMcBeaver/src/QMCWalkerData.cpp:302-344 */
static double dist(const double *a, const double *b)
{
  return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
}

static void update_distances(const orc_system *s, orc_walker *w, const double *R, int whichE)
{
  int N = s->N, M = s->M;
  if (whichE == -1) {
    for (int i = 0; i < N; i++) {
      for (int j = 0; j < i; j++) {
        double r = dist(R + 3 * i, R + 3 * j);
        w->rij[i * N + j] = r;
        for (int x = 0; x < 3; x++) w->rij_uvec[(i * N + j) * 3 + x] = (R[3 * i + x] - R[3 * j + x]) / r;
      }
      for (int j = 0; j < M; j++) {
        double r = dist(R + 3 * i, s->nuc_xyz + 3 * j);
        w->riA[i * M + j] = r;
        for (int x = 0; x < 3; x++) w->riA_uvec[(i * M + j) * 3 + x] = (R[3 * i + x] - s->nuc_xyz[3 * j + x]) / r;
      }
    }
  } else {
    for (int j = 0; j < N; j++) {
      if (j == whichE) continue;
      double r = dist(R + 3 * j, R + 3 * whichE);
      int e1 = whichE > j ? whichE : j;
      int e2 = whichE < j ? whichE : j;
      w->rij[e1 * N + e2] = r;
      for (int x = 0; x < 3; x++) w->rij_uvec[(e1 * N + e2) * 3 + x] = (R[3 * e1 + x] - R[3 * e2 + x]) / r;
    }
    for (int j = 0; j < M; j++) {
      w->riA[whichE * M + j] = dist(R + 3 * whichE, s->nuc_xyz + 3 * j);
      for (int x = 0; x < 3; x++)
        w->riA_uvec[(whichE * M + j) * 3 + x] = (R[3 * whichE + x] - s->nuc_xyz[3 * j + x]) / w->riA[whichE * M + j];
    }
  }
}

/* ------------------------------------------------------------ basis (a2) */
/* QMCBasisFunction::evaluateBasisFunctions, QMcBeaver/src/QMCBasisFunction.cpp:287-403,
 * including the exponent cache keyed on the previous primitive (:310,372-379). */
static void basis_eval(const orc_system *s, const double *R, int start, int stop, double *chi /* [nUP][5][K] */)
{
  int K = s->K;
  double temp1 = 0, temp2 = 0, temp3x = 0, temp3y = 0, temp3z = 0;
  int el = 0;
  for (int idx = start; idx <= stop; idx++) {
    int bf = 0;
    double p0 = 0.0;
    for (int atom = 0; atom < s->M; atom++) {
      double Xc[3];
      for (int x = 0; x < 3; x++) Xc[x] = R[3 * idx + x] - s->nuc_xyz[3 * atom + x];
      const int numl = s->atom_lmax[atom] + 1;
      const int numn = numl > 3 ? numl : 3;
      double xyz_abc[3][16][3];
      for (int x = 0; x < 3; x++) {
        xyz_abc[x][0][0] = 1.0;
        xyz_abc[x][1][0] = Xc[x];
        for (int abc = 2; abc < numn; abc++) xyz_abc[x][abc][0] = xyz_abc[x][1][0] * xyz_abc[x][abc - 1][0];
        xyz_abc[x][0][1] = 0.0;
        xyz_abc[x][0][2] = 0.0;
        for (int abc = 1; abc < numn; abc++) {
          xyz_abc[x][abc][1] = abc / xyz_abc[x][1][0];
          xyz_abc[x][abc][2] = abc * (abc - 1.0) / xyz_abc[x][2][0];
        }
      }
      double r_sq = xyz_abc[0][2][0] + xyz_abc[1][2][0] + xyz_abc[2][2][0];
      int nbf = s->atom_nbf[atom];
      int f0 = s->atom_first[atom];
      for (int j = 0; j < nbf; j++) {
        int k = f0 + j;
        int a = s->bf_pow[3 * k], b = s->bf_pow[3 * k + 1], c = s->bf_pow[3 * k + 2];
        double xyzA0 = xyz_abc[0][a][0] * xyz_abc[1][b][0] * xyz_abc[2][c][0];
        double xyzA1 = 4.0 * (a + b + c) + 6.0;
        double x_val = 0, x_grx = 0, x_gry = 0, x_grz = 0, x_lap = 0;
        int np = s->bf_nprim[k];
        const double *ex = s->pexp + s->bf_off[k];
        const double *co = s->pcoef + s->bf_off[k];
        for (int i = 0; i < np; i++) {
          if (fabs(p0 - ex[i]) > 1e-10) {
            p0 = ex[i];
            temp1 = exp(-p0 * r_sq);
            temp2 = 4.0 * r_sq * p0 * p0;
            temp3x = -2.0 * p0 * xyz_abc[0][1][0];
            temp3y = -2.0 * p0 * xyz_abc[1][1][0];
            temp3z = -2.0 * p0 * xyz_abc[2][1][0];
          }
          double exp_term = temp1 * co[i] * xyzA0;
          x_val += exp_term;
          x_grx += exp_term * (xyz_abc[0][a][1] + temp3x);
          x_gry += exp_term * (xyz_abc[1][b][1] + temp3y);
          x_grz += exp_term * (xyz_abc[2][c][1] + temp3z);
          x_lap += exp_term * (xyz_abc[0][a][2] + xyz_abc[1][b][2] + xyz_abc[2][c][2] - p0 * xyzA1 + temp2);
        }
        double *o = chi + (size_t)el * 5 * K;
        o[0 * K + bf] = x_val;
        o[1 * K + bf] = x_grx;
        o[2 * K + bf] = x_gry;
        o[3 * K + bf] = x_grz;
        o[4 * K + bf] = x_lap;
        bf++;
      }
    }
    el++;
  }
}

void orc_basis_at(const orc_system *s, const double *r, double *out)
{
  /* evaluate a single position as electron 0 */
  double *R = (double *)malloc(sizeof(double) * 3);
  R[0] = r[0]; R[1] = r[1]; R[2] = r[2];
  basis_eval(s, R, 0, 0, out);
  free(R);
}

/* ----------------------------------------------------- contraction (a3) */
/* Array2D::gemm with rhsIsTransposed (QMcBeaver/include/Array2D.h:473-485):
 * D[e][o] = sum_k chi[e][k] * C[o][k], k ascending. */
static void contract(const orc_system *s, const double *chi, int nUP, const double *C, int n, double *D /* [5][nUP][n] */)
{
  int K = s->K;
  for (int q = 0; q < 5; q++)
    for (int e = 0; e < nUP; e++)
      for (int o = 0; o < n; o++) {
        const double *A = chi + ((size_t)e * 5 + q) * K;
        const double *B = C + (size_t)o * K;
        double cij = 0;
        for (int k = 0; k < K; k++) cij += A[k] * B[k];
        D[((size_t)q * nUP + e) * n + o] = cij;
      }
}

/* ---------------------------------------------------------- LU (a4) */
/* Array2D::ludcmp (QMcBeaver/include/Array2D.h:1204-1340), Crout with implicit
 * row scaling and long double accumulators. a is n x n row-major, destroyed. */
static void ludcmp(double *a, int n, int *indx, double *d, int *calcOK)
{
  int imax = -1;
  long double big, dum, temp, sum;
  double *vv = (double *)malloc(sizeof(double) * (n ? n : 1));
  *calcOK = 1;
  *d = 1.0;
  for (int i = 0; i < n; i++) {
    big = 0.0L;
    for (int j = 0; j < n; j++)
      if ((temp = (double)fabs(a[i * n + j])) > big) big = temp;
    if (big == 0.0L) {
      *calcOK = 0;
      free(vv);
      return;
    }
    vv[i] = (double)(1.0L / big);
  }
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < j; i++) {
      sum = -1.0 * a[i * n + j];
      for (int k = 0; k < i; k++) sum += a[i * n + k] * a[k * n + j];
      a[i * n + j] = (double)(-1.0 * sum);
    }
    big = 0.0L;
    for (int i = j; i < n; i++) {
      sum = -1.0 * a[i * n + j];
      for (int k = 0; k < j; k++) sum += a[i * n + k] * a[k * n + j];
      a[i * n + j] = (double)(-1.0 * sum);
      if ((dum = vv[i] * (double)(fabs((double)sum))) >= big) {
        big = dum;
        imax = i;
      }
    }
    if (j != imax) {
      for (int k = 0; k < n; k++) {
        dum = a[imax * n + k];
        a[imax * n + k] = a[j * n + k];
        a[j * n + k] = (double)dum;
      }
      *d = -(*d);
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (a[j * n + j] == 0.0) a[j * n + j] = 1e-300;
    if (j != n) {
      dum = 1.0L / (a[j * n + j]);
      for (int i = j + 1; i < n; i++) a[i * n + j] *= (double)dum;
    }
  }
  free(vv);
}

/* Array2D::lubksb (QMcBeaver/include/Array2D.h:1352-1421) */
static void lubksb(const double *a, int n, const int *indx, double *b)
{
  int ii = -1, ip;
  long double sum;
  for (int i = 0; i < n; i++) {
    ip = indx[i];
    sum = -1.0 * b[ip];
    b[ip] = b[i];
    if (ii >= 0) {
      for (int j = ii; j <= i - 1; j++) sum += a[i * n + j] * b[j];
    } else if (sum) {
      ii = i;
    }
    b[i] = (double)(-1.0 * sum);
  }
  for (int i = n - 1; i >= 0; i--) {
    sum = -1.0 * b[i];
    for (int j = i + 1; j < n; j++) sum += a[i * n + j] * b[j];
    b[i] = (double)(-1.0 * sum / a[i * n + i]);
  }
}

/* Array2D::determinant_and_inverse, NR branch (QMcBeaver/include/Array2D.h:1521-1548).
 * inv[i*n+j] = (A^-1)(i,j). */
static void det_and_inverse(double *a, int n, double *inv, double *det, int *calcOK)
{
  double d;
  int *indx = (int *)malloc(sizeof(int) * (n ? n : 1));
  double *col = (double *)malloc(sizeof(double) * (n ? n : 1));
  ludcmp(a, n, indx, &d, calcOK);
  if (*calcOK) {
    for (int j = 0; j < n; j++) {
      for (int i = 0; i < n; i++) col[i] = 0.0;
      col[j] = 1.0;
      lubksb(a, n, indx, col);
      for (int i = 0; i < n; i++) inv[i * n + j] = col[i];
    }
  }
  for (int i = 0; i < n; i++) d *= a[i * n + i];
  *det = d;
  free(indx);
  free(col);
}

/* Array2D::inverseUpdateOneRow (QMcBeaver/include/Array2D.h:1567-1610): inv is
 * n x n, row = replaced electron, v = the new Slater row. Returns det ratio. */
static double inverse_update_row(double *inv, int n, int row, const double *v)
{
  double detRatio = 0;
  for (int r = 0; r < n; r++) detRatio += v[r] * inv[r * n + row];
  double q = 1.0 / detRatio;
  for (int c = 0; c < n; c++) {
    if (c == row) continue;
    double val = 0.0;
    for (int l = 0; l < n; l++) val += v[l] * inv[l * n + c];
    val *= q;
    for (int r = 0; r < n; r++) inv[r * n + c] -= val * inv[r * n + row];
  }
  for (int r = 0; r < n; r++) inv[r * n + row] *= q;
  return detRatio;
}

/* Array2D::inverseUpdateOneColumn (QMcBeaver/include/Array2D.h:1628-1671): the
 * column `col` of the matrix becomes column `col` of newD (n x n, row-major
 * [e][o]); inv[o*n+e]. Returns the determinant ratio. */
static double inverse_update_col(double *inv, int n, int col, const double *newD)
{
  double detRatio = 0;
  for (int c = 0; c < n; c++) detRatio += newD[c * n + col] * inv[col * n + c];
  double q = 1.0 / detRatio;
  for (int r = 0; r < n; r++) {
    if (r == col) continue;
    double val = 0.0;
    for (int l = 0; l < n; l++) val += newD[l * n + col] * inv[r * n + l];
    val *= q;
    for (int c = 0; c < n; c++) inv[r * n + c] -= val * inv[col * n + c];
  }
  for (int c = 0; c < n; c++) inv[col * n + c] *= q;
  return detRatio;
}

static void poly_all(const double *c, int len, double x, double *f, double *df, double *d2f);

/* QMCElectronNucleusCusp::replaceCusps (QMcBeaver/src/QMCElectronNucleusCusp.cpp:574-638)
 * with QMCElectronNucleusCuspParameters::replaceOrbitalValues,
 * evaluateOriginalOrbital and evaluateReplacementOrbital
 * (QMcBeaver/src/QMCElectronNucleusCuspParameters.cpp:107-285).
 * D: [5][nUP][a] rows of electrons start..stop. */
static void replace_cusps(const orc_system *s, int sp, const double *R, int start, int stop, double *D, int nUP, int a)
{
  for (int i = 0; i < s->M; i++) {
    const double *nuc = s->nuc_xyz + 3 * i;
    int counter = 0;
    for (int j = start; j <= stop; j++) {
      double xrel = R[3 * j] - nuc[0], yrel = R[3 * j + 1] - nuc[1], zrel = R[3 * j + 2] - nuc[2];
      double rrel = sqrt(xrel * xrel + yrel * yrel + zrel * zrel);
      for (int k = 0; k < a; k++) {
        const double *par = s->cpar[sp] + ((size_t)i * a + k) * 8;
        if (!(rrel < par[0])) continue;
        double v = 0.0, gx = 0.0, gy = 0.0, gz = 0.0, l = 0.0;
        /* evaluateOriginalOrbital */
        const double *co = s->cscoef[sp] + ((size_t)i * a + k) * s->nsmax;
        const double *ex = s->csexp + (size_t)i * s->nsmax;
        double r_sq = rrel * rrel, ov = 0.0, ogx = 0.0, ogy = 0.0, ogz = 0.0, ol = 0.0;
        for (int q = 0; q < s->cns[i]; q++) {
          double p0 = ex[q], p1 = co[q];
          double term = p1 * exp(-p0 * r_sq);
          ov += term;
          double temp = -2 * p0 * term;
          ogx += xrel * temp;
          ogy += yrel * temp;
          ogz += zrel * temp;
          ol += 2 * p0 * (2 * p0 * r_sq - 3) * term;
        }
        v -= ov;
        gx -= ogx;
        gy -= ogy;
        gz -= ogz;
        l -= ol;
        /* evaluateReplacementOrbital */
        double f, df, d2f;
        poly_all(par + 3, 5, rrel, &f, &df, &d2f);
        double e = par[1] * exp(f);
        double tg = (e * df) / rrel;
        v += par[2] + e;
        gx += tg * xrel;
        gy += tg * yrel;
        gz += tg * zrel;
        l += e * (d2f + df * (2.0 / rrel + df));
        D[((size_t)0 * nUP + counter) * a + k] += v;
        D[((size_t)1 * nUP + counter) * a + k] += gx;
        D[((size_t)2 * nUP + counter) * a + k] += gy;
        D[((size_t)3 * nUP + counter) * a + k] += gz;
        D[((size_t)4 * nUP + counter) * a + k] += l;
      }
      counter++;
    }
  }
}

/* ---------------------------------------------------- Slater spin (a2-a4) */
/* QMCSlater::evaluate (QMcBeaver/src/QMCSlater.cpp:828-884) followed by
 * update_Ds (:390-541) and calculate_DerivativeRatios (:648-764) for one spin,
 * every determinant: the first one by LU (all electrons) or a row update
 * (one electron), the others by column swaps from the previous determinant
 * (all electrons) or their own row update (one electron). */
static void slater_spin(const orc_system *s, orc_walker *w, int sp, const double *R, int whichE)
{
  int n = sp ? s->nb : s->na;
  int Start = sp ? s->na : 0;
  int Stop = Start + n - 1;
  if (n == 0) return;
  if (whichE != -1 && (whichE < Start || whichE > Stop)) return;
  int start = whichE == -1 ? Start : whichE;
  int stop = whichE == -1 ? Stop : whichE;
  int nUP = stop - start + 1;
  int K = s->K, a = s->nact[sp], nd = s->ndet;
  const double *C = sp ? s->mo_b : s->mo_a;
  double *chi = (double *)malloc(sizeof(double) * (size_t)nUP * 5 * K);
  double *D = (double *)malloc(sizeof(double) * (size_t)5 * nUP * a);
  double *ciDet = (double *)malloc(sizeof(double) * (size_t)nUP * n);
  basis_eval(s, R, start, stop, chi);
  contract(s, chi, nUP, C, a, D);
  if (s->cusp) replace_cusps(s, sp, R, start, stop, D, nUP, a);
  /* splice new rows into D_x / D_xx (QMcBeaver/src/QMCSlater.cpp:465-491) */
  int iEl = whichE == -1 ? 0 : whichE - Start;
  for (int e = 0; e < nUP; e++)
    for (int o = 0; o < a; o++) {
      w->Dv[sp][(iEl + e) * a + o] = D[(size_t)e * a + o];
      for (int d = 0; d < 3; d++) w->Dx[sp][d][(iEl + e) * a + o] = D[((size_t)(1 + d) * nUP + e) * a + o];
      w->Dxx[sp][(iEl + e) * a + o] = D[((size_t)4 * nUP + e) * a + o];
    }
  for (int ci = 0; ci < nd; ci++) {
    const int *occ = s->occ[sp] + ci * n;
    double *inv = w->inv[sp] + (size_t)ci * n * n;
    /* QMCWavefunction::getDataForCI: the columns of determinant ci */
    for (int e = 0; e < nUP; e++)
      for (int o = 0; o < n; o++) ciDet[e * n + o] = D[(size_t)e * a + occ[o]];
    int calcOK = 1;
    if (whichE == -1) {
      if (ci == 0) {
        det_and_inverse(ciDet, n, inv, &w->det[sp][0], &calcOK);
      } else {
        memcpy(inv, inv - (size_t)n * n, sizeof(double) * n * n);
        w->det[sp][ci] = w->det[sp][ci - 1];
        for (int o = 0; o < n; o++) {
          int so = s->swaps[sp][ci * n + o];
          if (so < 0) break;
          double ratio = inverse_update_col(inv, n, so, ciDet);
          w->det[sp][ci] *= ratio;
          if (ratio == 0) break;
        }
        if (w->det[sp][ci] == 0) {
          calcOK = 0;
          det_and_inverse(ciDet, n, inv, &w->det[sp][ci], &calcOK);
        }
      }
    } else {
      double ratio = inverse_update_row(inv, n, whichE - Start, ciDet);
      if (ratio != 0.0)
        w->det[sp][ci] *= ratio;
      else
        calcOK = 0;
    }
    w->sing[sp][ci] = !calcOK;
    if (calcOK) {
      double lap_PR = 0.0;
      double *g = w->rDx[sp] + (size_t)ci * s->N * 3;
      for (int e = 0; e < n; e++) g[3 * e] = g[3 * e + 1] = g[3 * e + 2] = 0.0;
      for (int o = 0; o < n; o++) {
        int orb = occ[o];
        for (int e = 0; e < n; e++) {
          double inv_v = inv[o * n + e];
          lap_PR += w->Dxx[sp][e * a + orb] * inv_v;
          g[3 * e + 0] += w->Dx[sp][0][e * a + orb] * inv_v;
          g[3 * e + 1] += w->Dx[sp][1][e * a + orb] * inv_v;
          g[3 * e + 2] += w->Dx[sp][2][e * a + orb] * inv_v;
        }
      }
      w->rDxx[sp][ci] = lap_PR;
    }
  }
  free(chi);
  free(D);
  free(ciDet);
}

/* ------------------------------------------------------------ Jastrow (a6) */
/* FixedCuspPadeCorrelationFunction::evaluate (QMcBeaver/src/FixedCuspPadeCorrelationFunction.cpp:89-111)
 * with Polynomial::evaluateAll (QMcBeaver/src/Polynomial.cpp:127-148). */
static void poly_all(const double *c, int len, double x, double *f, double *df, double *d2f)
{
  int n = len - 1;
  *f = c[n];
  *df = 0.0;
  *d2f = 0.0;
  for (int i = n - 1; i >= 0; i--) {
    *d2f = *d2f * x + *df;
    *df = *df * x + *f;
    *f = *f * x + c[i];
  }
  *d2f *= 2;
}

static void pade(const orc_system *s, int idx, double r, double *u, double *du, double *d2u)
{
  if (s->ctype[idx] == QMCB_CORR_CAMBRIDGE2) {
    /* Cambridge2CorrelationFunction::evaluate (QMcBeaver/src/Cambridge2CorrelationFunction.cpp) */
    const double *cp = s->cparam + 4 * idx;
    double fL = cp[0];
    int C = (int)cp[1];
    *u = *du = *d2u = 0.0;
    if (cp[2] == 0.0) return;
    double d = fL * r - 1.0;
    if (d > 0.0) return;
    double a, ap, app;
    poly_all(s->pnum + idx * QMCB_PADE_MAX, s->pnn[idx], fL * r, &a, &ap, &app);
    double P = a, dP_r = fL * ap, dP_rr = fL * fL * app;
    double dpc = pow(d, C);
    double dpc_r = C * fL * dpc / d;
    double dpc_rr = (C - 1.0) * fL * dpc_r / d;
    *u = dpc * P;
    *du = dpc_r * P + dpc * dP_r;
    *d2u = dpc_rr * P + dpc_r * dP_r * 2.0 + dpc * dP_rr;
    return;
  }
  double a, ap, app, b, bp, bpp;
  poly_all(s->pnum + idx * QMCB_PADE_MAX, s->pnn[idx], r, &a, &ap, &app);
  poly_all(s->pden + idx * QMCB_PADE_MAX, s->pnd[idx], r, &b, &bp, &bpp);
  double aDIVb = a / b;
  double bpDIVb = bp / b;
  double apDIVb = ap / b;
  *u = aDIVb;
  *du = apDIVb - bpDIVb * aDIVb;
  *d2u = (app - bpp * aDIVb) / b - 2 * bpDIVb * (*du);
}

/* QMCJastrowElectronElectron::collectForPair (QMcBeaver/src/QMCJastrowElectronElectron.cpp:221-268) */
static void collect_pair(const orc_system *s, orc_walker *w, int E1, int E2, int f)
{
  int N = s->N;
  double r = w->rij[E1 * N + E2];
  double u, du, d2u;
  pade(s, f, r, &u, &du, &d2u);
  double Uij = u, Uij_x = du, Uij_xx = 2.0 * (2.0 / r * Uij_x + d2u);
  w->U -= w->Uij[E1 * N + E2];
  w->U += Uij;
  w->Uij[E1 * N + E2] = Uij;
  for (int i = 0; i < 3; i++) {
    double temp = w->Uij_x[(E1 * N + E2) * 3 + i];
    w->U_x[E1 * 3 + i] -= temp;
    w->U_x[E2 * 3 + i] += temp;
    temp = Uij_x * w->rij_uvec[(E1 * N + E2) * 3 + i];
    w->Uij_x[(E1 * N + E2) * 3 + i] = temp;
    w->U_x[E1 * 3 + i] += temp;
    w->U_x[E2 * 3 + i] -= temp;
  }
  w->U_xx -= w->Uij_xx[E1 * N + E2];
  w->U_xx += Uij_xx;
  w->Uij_xx[E1 * N + E2] = Uij_xx;
}

/* QMCJastrowElectronElectron::updateOne / updateAll (:68-219) */
static void jastrow_ee(const orc_system *s, orc_walker *w, int whichE)
{
  int na = s->na, nb = s->nb, N = s->N;
  int fA = (na > 0 && nb > 0) ? s->ee[0] : -1;
  int fUU = na > 1 ? s->ee[1] : -1;
  int fDD = nb > 1 ? s->ee[2] : -1;
  if (whichE != -1) {
    int E = whichE;
    int isAlpha = E < na;
    if (fA >= 0) {
      if (isAlpha)
        for (int EB = na; EB < N; EB++) collect_pair(s, w, EB, E, fA);
      else
        for (int EA = 0; EA < na; EA++) collect_pair(s, w, E, EA, fA);
    }
    if (fUU >= 0 && isAlpha) {
      for (int EA = 0; EA < E; EA++) collect_pair(s, w, E, EA, fUU);
      for (int EA = E + 1; EA < na; EA++) collect_pair(s, w, EA, E, fUU);
    }
    if (fDD >= 0 && !isAlpha) {
      for (int EB = na; EB < E; EB++) collect_pair(s, w, E, EB, fDD);
      for (int EB = E + 1; EB < N; EB++) collect_pair(s, w, EB, E, fDD);
    }
  } else {
    if (fA >= 0)
      for (int E1 = 0; E1 < na; E1++)
        for (int E2 = na; E2 < N; E2++) collect_pair(s, w, E2, E1, fA);
    if (fUU >= 0)
      for (int E1 = 0; E1 < na; E1++)
        for (int E2 = 0; E2 < E1; E2++) collect_pair(s, w, E1, E2, fUU);
    if (fDD >= 0)
      for (int E1 = na; E1 < N; E1++)
        for (int E2 = na; E2 < E1; E2++) collect_pair(s, w, E1, E2, fDD);
  }
}

/* QMCJastrowElectronNuclear::evaluate (QMcBeaver/src/QMCJastrowElectronNuclear.cpp:54-187) */
static void jastrow_en(const orc_system *s, orc_walker *w, int whichE)
{
  int M = s->M, N = s->N, na = s->na;
  for (int nuc = 0; nuc < M; nuc++) {
    for (int e = 0; e < N; e++) {
      if (whichE != e && whichE != -1) continue;
      int f = e < na ? s->en_up[nuc] : s->en_dn[nuc];
      if (f < 0) continue;
      double r = w->riA[e * M + nuc];
      double u, du, d2u;
      pade(s, f, r, &u, &du, &d2u);
      double UiA = u, UiA_x = du, UiA_xx = 2.0 / r * UiA_x + d2u;
      w->U -= w->UiA[e * M + nuc];
      w->U += UiA;
      w->UiA[e * M + nuc] = UiA;
      w->U_xx -= w->UiA_xx[e * M + nuc];
      w->U_xx += UiA_xx;
      w->UiA_xx[e * M + nuc] = UiA_xx;
      for (int i = 0; i < 3; i++) {
        double temp = w->UiA_x[(e * M + nuc) * 3 + i];
        w->U_x[e * 3 + i] -= temp;
        temp = UiA_x * w->riA_uvec[(e * M + nuc) * 3 + i];
        w->UiA_x[(e * M + nuc) * 3 + i] = temp;
        w->U_x[e * 3 + i] += temp;
      }
    }
  }
}

/* ------------------------------------------------------- three-body (a6) */
/* CambridgeThreeBodyCorrelationFunction::setElectron / evaluate / getLapPoly
 * (QMcBeaver/src/CambridgeThreeBodyCorrelationFunction.cpp:150-470) for the
 * pair (E1 first, E2 second) around nucleus `nuc` with function f.  Returns 0
 * when either electron is outside the cutoff. */
static int tb_pair_eval(const orc_system *s, const orc_walker *w, int f, int E1, int E2, int nuc, double *U,
                        double *lapv, double g1[3], double g2[3])
{
  int N = s->N, M = s->M;
  int Nen = s->tb_nen[f], Nee = s->tb_nee[f], C = s->tb_C[f];
  double L = s->tb_cut[f];
  if (fabs(L) < 1e-10) L = 1.0e10;
  const double *coeffs = s->tb_coef + s->tb_off[f];
  double d1pow[16], d1pow1[16], d1pow2[16], d2pow[16], d2pow1[16], d2pow2[16], r12pow[16], r12pow1[16], r12pow2[16];
  /* setElectron(true, E1) */
  double r1 = w->riA[E1 * M + nuc] * L, d1 = r1 - 1.0;
  if (d1 > 0.0) return 0;
  const double *r1v = w->riA_uvec + ((size_t)E1 * M + nuc) * 3;
  double pre1 = pow(d1, C), d1pre1 = pre1 * C / d1, d2pre1 = (C - 1.0) * d1pre1 / d1;
  d1pow[0] = 1.0; d1pow1[0] = 0.0; d1pow2[0] = 0.0; d1pow2[1] = 0.0;
  for (int i = 1; i < Nen; i++) {
    d1pow[i] = d1pow[i - 1] * r1;
    d1pow1[i] = d1pow[i - 1] * i;
    if (i < 2) continue;
    d1pow2[i] = d1pow[i - 2] * i * (i - 1);
  }
  /* setElectron(false, E2) */
  double r2 = w->riA[E2 * M + nuc] * L, d2 = r2 - 1.0;
  if (d2 > 0.0) return 0;
  const double *r2v = w->riA_uvec + ((size_t)E2 * M + nuc) * 3;
  double pre2 = pow(d2, C), d1pre2 = pre2 * C / d2, d2pre2 = (C - 1.0) * d1pre2 / d2;
  d2pow[0] = 1.0; d2pow1[0] = 0.0; d2pow2[0] = 0.0; d2pow2[1] = 0.0;
  for (int i = 1; i < Nen; i++) {
    d2pow[i] = d2pow[i - 1] * r2;
    d2pow1[i] = d2pow[i - 1] * i;
    if (i < 2) continue;
    d2pow2[i] = d2pow[i - 2] * i * (i - 1);
  }
  /* evaluate(rij_uvec(E1, E2), rij(E1, E2)) */
  double r12 = w->rij[E1 * N + E2] * L;
  const double *r12v = w->rij_uvec + ((size_t)E1 * N + E2) * 3;
  r12pow[0] = 1.0; r12pow1[0] = 0.0; r12pow2[0] = 0.0; r12pow2[1] = 0.0;
  for (int i = 1; i < Nee; i++) {
    r12pow[i] = r12pow[i - 1] * r12;
    r12pow1[i] = r12pow[i - 1] * i;
    if (i < 2) continue;
    r12pow2[i] = r12pow[i - 2] * i * (i - 1);
  }
  double P = 0, Pl = 0, Pl2 = 0, Pln = 0, Pm = 0, Pm2 = 0, Pmn = 0, Pn = 0, Pn2 = 0;
  int ai = 0;
  for (int l = 0; l < Nen; l++)
    for (int m = 0; m < Nen; m++) {
      double lm = d1pow[l] * d2pow[m], dlm = d1pow1[l] * d2pow[m], ldm = d1pow[l] * d2pow1[m];
      double d2lm = d1pow2[l] * d2pow[m], ld2m = d1pow[l] * d2pow2[m];
      for (int n = 0; n < Nee; n++) {
        double coeff = coeffs[ai];
        ai++;
        if (fabs(coeff) < 1e-30) continue;
        double term = lm * r12pow[n];
        double _l = dlm * r12pow[n], _m = ldm * r12pow[n], _n = lm * r12pow1[n];
        double ln = dlm * r12pow1[n], mn = ldm * r12pow1[n];
        double l2 = d2lm * r12pow[n], m2 = ld2m * r12pow[n], n2 = lm * r12pow2[n];
        P += coeff * term;
        Pl += coeff * _l;
        Pm += coeff * _m;
        Pn += coeff * _n;
        Pln += coeff * ln;
        Pmn += coeff * mn;
        Pl2 += coeff * l2;
        Pm2 += coeff * m2;
        Pn2 += coeff * n2;
      }
    }
  *U = pre1 * pre2 * P;
  double dU_dr12 = pre1 * pre2 * Pn;
  double dU_dr1 = (d1pre1 * P + pre1 * Pl) * pre2;
  double dU_dr2 = (d1pre2 * P + pre2 * Pm) * pre1;
  for (int i = 0; i < 3; i++) {
    g1[i] = L * (dU_dr1 * r1v[i] + dU_dr12 * r12v[i]);
    g2[i] = L * (dU_dr2 * r2v[i] - dU_dr12 * r12v[i]);
  }
  /* getLapPoly */
  double lap = 2.0 * (2.0 * dU_dr12 / r12 + dU_dr1 / r1 + dU_dr2 / r2);
  double d2U_d2r1 = pre2 * (d2pre1 * P + 2.0 * d1pre1 * Pl + pre1 * Pl2);
  double d2U_d2r2 = pre1 * (d2pre2 * P + 2.0 * d1pre2 * Pm + pre2 * Pm2);
  double d2U_d2r12 = pre1 * pre2 * Pn2;
  lap += 2.0 * d2U_d2r12 + d2U_d2r1 + d2U_d2r2;
  double d2U_dr1r12 = 2.0 * pre2 * (d1pre1 * Pn + pre1 * Pln);
  double d2U_dr2r12 = 2.0 * pre1 * (d1pre2 * Pn + pre2 * Pmn);
  for (int i = 0; i < 3; i++) lap += r12v[i] * (r1v[i] * d2U_dr1r12 - r2v[i] * d2U_dr2r12);
  *lapv = lap * L * L;
  return 1;
}

/* QMCThreeBodyJastrow::collectForPair (QMcBeaver/src/QMCThreeBodyJastrow.cpp:403-441) */
static void tb_collect(const orc_system *s, orc_walker *w, int f, int E1, int E2, int nuc)
{
  if (f < 0) return;
  int N = s->N;
  double U, lap, g1[3], g2[3];
  if (!tb_pair_eval(s, w, f, E1, E2, nuc, &U, &lap, g1, g2)) return;
  w->tU[E1 * N + E2] += U;
  w->tUxx[E1 * N + E2] += lap;
  for (int i = 0; i < 3; i++) {
    w->tUx1[(E1 * N + E2) * 3 + i] += g1[i];
    w->tUx2[(E1 * N + E2) * 3 + i] += g2[i];
  }
}

/* QMCThreeBodyJastrow::updateAll / updateOne (QMcBeaver/src/QMCThreeBodyJastrow.cpp:43-178,320-401) */
static void jastrow_3b(const orc_system *s, orc_walker *w, int whichE)
{
  if (s->ntb <= 0) return;
  int N = s->N, na = s->na, nb = s->nb, M = s->M;
  if (whichE == -1) {
    for (int E1 = 0; E1 < N; E1++)
      for (int E2 = 0; E2 < E1; E2++) {
        w->U -= w->tU[E1 * N + E2];
        w->U_xx -= w->tUxx[E1 * N + E2];
        for (int x = 0; x < 3; x++) {
          w->U_x[E1 * 3 + x] -= w->tUx1[(E1 * N + E2) * 3 + x];
          w->U_x[E2 * 3 + x] -= w->tUx2[(E1 * N + E2) * 3 + x];
        }
      }
    memset(w->tU, 0, sizeof(double) * N * N);
    memset(w->tUxx, 0, sizeof(double) * N * N);
    memset(w->tUx1, 0, sizeof(double) * N * N * 3);
    memset(w->tUx2, 0, sizeof(double) * N * N * 3);
    for (int nuc = 0; nuc < M; nuc++) {
      int fud = s->tb_pair[3 * nuc], fuu = s->tb_pair[3 * nuc + 1], fdd = s->tb_pair[3 * nuc + 2];
      if (na > 0 && nb > 0)
        for (int E2 = na; E2 < na + nb; E2++)
          for (int E1 = 0; E1 < na; E1++) tb_collect(s, w, fud, E2, E1, nuc);
      if (na > 1)
        for (int E1 = 1; E1 < na; E1++)
          for (int E2 = 0; E2 < E1; E2++) tb_collect(s, w, fuu, E1, E2, nuc);
      if (nb > 1)
        for (int E1 = na + 1; E1 < N; E1++)
          for (int E2 = na; E2 < E1; E2++) tb_collect(s, w, fdd, E1, E2, nuc);
    }
    for (int E1 = 0; E1 < N; E1++)
      for (int E2 = 0; E2 < E1; E2++) {
        w->U += w->tU[E1 * N + E2];
        w->U_xx += w->tUxx[E1 * N + E2];
        for (int x = 0; x < 3; x++) {
          w->U_x[E1 * 3 + x] += w->tUx1[(E1 * N + E2) * 3 + x];
          w->U_x[E2 * 3 + x] += w->tUx2[(E1 * N + E2) * 3 + x];
        }
      }
    return;
  }
  int E = whichE, isAlpha = E < na;
  for (int E2 = 0; E2 < N; E2++) {
    if (E == E2) continue;
    int EH = E > E2 ? E : E2, EL = E < E2 ? E : E2;
    w->U -= w->tU[EH * N + EL];
    w->tU[EH * N + EL] = 0.0;
    w->U_xx -= w->tUxx[EH * N + EL];
    w->tUxx[EH * N + EL] = 0.0;
    for (int x = 0; x < 3; x++) {
      w->U_x[EH * 3 + x] -= w->tUx1[(EH * N + EL) * 3 + x];
      w->tUx1[(EH * N + EL) * 3 + x] = 0.0;
      w->U_x[EL * 3 + x] -= w->tUx2[(EH * N + EL) * 3 + x];
      w->tUx2[(EH * N + EL) * 3 + x] = 0.0;
    }
  }
  for (int nuc = 0; nuc < M; nuc++) {
    int fud = s->tb_pair[3 * nuc], fuu = s->tb_pair[3 * nuc + 1], fdd = s->tb_pair[3 * nuc + 2];
    if (na > 0 && nb > 0) {
      if (isAlpha)
        for (int EB = na; EB < N; EB++) tb_collect(s, w, fud, EB, E, nuc);
      else
        for (int EA = 0; EA < na; EA++) tb_collect(s, w, fud, E, EA, nuc);
    }
    if (na > 1 && isAlpha) {
      for (int EA = 0; EA < E; EA++) tb_collect(s, w, fuu, E, EA, nuc);
      for (int EA = E + 1; EA < na; EA++) tb_collect(s, w, fuu, EA, E, nuc);
    }
    if (nb > 1 && !isAlpha) {
      for (int EB = na; EB < E; EB++) tb_collect(s, w, fdd, E, EB, nuc);
      for (int EB = E + 1; EB < N; EB++) tb_collect(s, w, fdd, EB, E, nuc);
    }
  }
  for (int E2 = 0; E2 < N; E2++) {
    if (E == E2) continue;
    int EH = E > E2 ? E : E2, EL = E < E2 ? E : E2;
    w->U += w->tU[EH * N + EL];
    w->U_xx += w->tUxx[EH * N + EL];
    for (int x = 0; x < 3; x++) {
      w->U_x[EH * 3 + x] += w->tUx1[(EH * N + EL) * 3 + x];
      w->U_x[EL * 3 + x] += w->tUx2[(EH * N + EL) * 3 + x];
    }
  }
}

/* -------------------------------------------------------- potential (a7) */
/* QMCPotential_Energy::evaluate / calc_P_en / calc_P_ee (QMcBeaver/src/QMCPotential_Energy.cpp:242-333) */
static void potential(const orc_system *s, orc_walker *w)
{
  int M = s->M, N = s->N;
  double Pen = 0.0;
  for (int nuc = 0; nuc < M; nuc++) {
    double Zeff = s->nuc_z[nuc];
    for (int el = 0; el < N; el++) Pen -= Zeff / w->riA[el * M + nuc];
  }
  double Pee = 0.0;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < i; j++) Pee += (-1.0 * -1.0) / w->rij[i * N + j];
  w->PE = s->Pnn + Pee + Pen;
  w->neE = Pen;
  w->eeE = Pee;
}

/* ------------------------------------------------------- psi quantities (a5) */
/* QMCSCFJastrow::calculate_Psi_quantities / update_SCF / calculate_Modified_Grad_PsiRatio
 * (QMcBeaver/src/QMCSCFJastrow.cpp:196-472) and calculate_E_Local (QMcBeaver/include/QMCSCFJastrow.h:311-314). */
static void psi_quantities(const orc_system *s, orc_walker *w, const double *R)
{
  int N = s->N, na = s->na, nb = s->nb, M = s->M;
  int nd = s->ndet, any_sing = 0;
  for (int ci = 0; ci < nd; ci++) any_sing |= w->sing[0][ci] | w->sing[1][ci];
  /* update_SCF: D = sum_ci c_ci detA(ci) detB(ci), termPR(ci) = term / D.
   * The reference keeps D in its extended-exponent QMCDouble, which is plain
   * double arithmetic while the magnitudes stay within 1e+-100 (each factor)
   * and 1e+-200 (products); outside that range the terms here are scaled by
   * the largest |detA detB| instead (log_D = lmax + log|Dtot|). */
  double Dtot = 1.0, lmax = 0.0;
  if (any_sing) {
    w->singular = 1;
  } else {
    double *termPR = (double *)malloc(sizeof(double) * nd);
    int plain = 1; /* magnitudes where QMCDouble keeps everything in its plain mantissa */
    for (int ci = 0; ci < nd; ci++) {
      double a = fabs(w->det[0][ci]), b = fabs(w->det[1][ci]), t = a * b;
      if (a > 1e100 || a < 1e-100 || b > 1e100 || b < 1e-100 || t > 1e200 || t < 1e-200) plain = 0;
    }
    if (nd == 1) {
      termPR[0] = 1.0;
    } else if (plain) {
      Dtot = 0.0;
      for (int ci = 0; ci < nd; ci++) {
        termPR[ci] = s->ci[ci] * w->det[0][ci] * w->det[1][ci];
        Dtot += termPR[ci];
      }
      if (Dtot != 0.0)
        for (int ci = 0; ci < nd; ci++) termPR[ci] /= Dtot;
      lmax = 0.0;
    } else {
      lmax = -INFINITY;
      for (int ci = 0; ci < nd; ci++) {
        double l = log(fabs(w->det[0][ci])) + log(fabs(w->det[1][ci]));
        if (s->ci[ci] != 0.0 && l > lmax) lmax = l;
      }
      Dtot = 0.0;
      for (int ci = 0; ci < nd; ci++) {
        double sg = (w->det[0][ci] < 0) != (w->det[1][ci] < 0) ? -1.0 : 1.0;
        termPR[ci] = s->ci[ci] * sg * exp(log(fabs(w->det[0][ci])) + log(fabs(w->det[1][ci])) - lmax);
        Dtot += termPR[ci];
      }
      if (Dtot != 0.0)
        for (int ci = 0; ci < nd; ci++) termPR[ci] /= Dtot;
    }
    w->D_xx = 0.0;
    for (int i = 0; i < 3 * N; i++) w->D_x[i] = 0.0;
    /* determinant-mixing amplification of rounding in the laplacian:
     * [sum_c |t_c lap_c| + 2 sum_i |U_x,i| . sum_c |t_c g_c,i|] over the same
     * sums without the absolute values inside (1 for one determinant) */
    double abs_l = 0.0, sum_l = 0.0, abs_g = 0.0, sum_g = 0.0;
    for (int ci = 0; ci < nd; ci++) {
      double l = (na > 0 ? w->rDxx[0][ci] : 0.0) + (nb > 0 ? w->rDxx[1][ci] : 0.0);
      abs_l += fabs(termPR[ci] * l);
      sum_l += termPR[ci] * l;
    }
    for (int i = 0; i < N; i++) {
      int sp_i = i < na ? 0 : 1, e = i < na ? i : i - na;
      for (int k = 0; k < 3; k++) {
        double a = 0.0, b = 0.0;
        for (int ci = 0; ci < nd; ci++) {
          double g = w->rDx[sp_i][((size_t)ci * N + e) * 3 + k];
          a += fabs(termPR[ci] * g);
          b += termPR[ci] * g;
        }
        abs_g += fabs(w->U_x[3 * i + k]) * a;
        sum_g += fabs(w->U_x[3 * i + k] * b);
      }
    }
    for (int ci = 0; ci < nd; ci++) {
      if (na > 0) w->D_xx += termPR[ci] * w->rDxx[0][ci];
      if (nb > 0) w->D_xx += termPR[ci] * w->rDxx[1][ci];
      const double *ga = w->rDx[0] + (size_t)ci * N * 3, *gb = w->rDx[1] + (size_t)ci * N * 3;
      for (int e = 0; e < na; e++)
        for (int k = 0; k < 3; k++) w->D_x[e * 3 + k] += termPR[ci] * ga[e * 3 + k];
      for (int e = 0; e < nb; e++)
        for (int k = 0; k < 3; k++) w->D_x[(e + na) * 3 + k] += termPR[ci] * gb[e * 3 + k];
    }
    free(termPR);
    {
      double den = fabs(sum_l) + 2.0 * sum_g;
      w->kappa = (abs_l + 2.0 * abs_g) / (den > 1.0 ? den : 1.0);
    }
    double L = w->D_xx + w->U_xx;
    for (int i = 0; i < N; i++)
      for (int j = 0; j < 3; j++) {
        w->grad[i * 3 + j] = w->D_x[i * 3 + j] + w->U_x[i * 3 + j];
        L += w->U_x[i * 3 + j] * w->D_x[i * 3 + j] * 2.0;
        L += w->U_x[i * 3 + j] * w->U_x[i * 3 + j];
      }
    w->lap = L;
  }
  /* modified quantum force */
  if (s->qf_mod == QMCB_QF_NONE) {
    for (int i = 0; i < 3 * N; i++) w->mgrad[i] = w->grad[i];
  } else if (s->qf_mod == QMCB_QF_UMRIGAR93_EQUAL) {
    double a = s->qf_a;
    double magsq = 0.0;
    for (int i = 0; i < 3 * N; i++) magsq += w->grad[i] * w->grad[i];
    double factor = (-1.0 + sqrt(1.0 + 2 * a * magsq * s->dt)) / (a * magsq * s->dt);
    for (int i = 0; i < 3 * N; i++) w->mgrad[i] = w->grad[i] * factor;
  } else {
    for (int i = 0; i < N; i++) {
      /* QMCMolecule::findClosestNucleusIndex: smallest riA, first on ties */
      int cn = 0;
      for (int j = 1; j < M; j++)
        if (w->riA[i * M + j] < w->riA[i * M + cn]) cn = j;
      double Zc = s->nuc_z[cn];
      double nv[3], ev[3], d2 = 0.0, temp;
      for (int x = 0; x < 3; x++) {
        temp = R[3 * i + x] - s->nuc_xyz[3 * cn + x];
        nv[x] = temp;
        d2 += temp * temp;
      }
      double inv_len = 1.0 / sqrt(d2);
      for (int x = 0; x < 3; x++) nv[x] *= inv_len;
      for (int x = 0; x < 3; x++) ev[x] = w->grad[3 * i + x];
      double ev2 = ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2];
      if (fabs(ev2) < 1e-10) {
        for (int x = 0; x < 3; x++) ev[x] *= 0.0;
      } else {
        double sc = 1.0 / sqrt(ev2);
        for (int x = 0; x < 3; x++) ev[x] *= sc;
      }
      temp = Zc * Zc * d2;
      double dotp = 0;
      for (int x = 0; x < 3; x++) dotp += nv[x] * ev[x];
      double a = 0.5 * (1.0 + dotp) + temp / (10.0 * (4.0 + temp));
      double factor;
      if (fabs(ev2) < 1e-10)
        factor = 1.0;
      else
        factor = (-1.0 + sqrt(1.0 + 2.0 * a * ev2 * s->dt)) / (a * ev2 * s->dt);
      for (int x = 0; x < 3; x++) w->mgrad[3 * i + x] = w->grad[3 * i + x] * factor;
    }
  }
  double lm = 0.0, lu = 0.0;
  for (int i = 0; i < 3 * N; i++) {
    lm += w->mgrad[i] * w->mgrad[i];
    lu += w->grad[i] * w->grad[i];
  }
  lm = sqrt(lm);
  lu = sqrt(lu);
  if (isnan(lm) || isnan(lu) || isnan(lm / lu) || lu == 0) w->singular = 1;
  w->KE = -0.5 * w->lap;
  w->E_L = -0.5 * w->lap + w->PE;
  if (nd == 1) {
    w->logpsi = log(fabs(w->det[0][0])) + log(fabs(w->det[1][0])) + w->U;
    w->sign = (w->det[0][0] * w->det[1][0] < 0) ? -1.0 : 1.0;
  } else {
    w->logpsi = lmax + log(fabs(Dtot)) + w->U;
    w->sign = Dtot < 0 ? -1.0 : 1.0;
  }
}

/* --------------------------------------------------------- evaluate (a1) */
int orc_evaluate(const orc_system *s, orc_walker **walkers, const double *R, int num, int whichE)
{
  int N = s->N;
  for (int wi = 0; wi < num; wi++) {
    orc_walker *w = walkers[wi];
    const double *Rw = R + (size_t)wi * N * 3;
    w->singular = 0;
    update_distances(s, w, Rw, whichE);
    /* QMCJastrow::evaluate: e-n then e-e (QMcBeaver/src/QMCJastrow.cpp:134-151) */
    jastrow_en(s, w, whichE);
    jastrow_ee(s, w, whichE);
    jastrow_3b(s, w, whichE);
    slater_spin(s, w, 0, Rw, whichE);
    slater_spin(s, w, 1, Rw, whichE);
    potential(s, w);
    psi_quantities(s, w, Rw);
  }
  return 0;
}

void orc_walker_get(const orc_walker *w, double *sc, double *grad, double *mgrad)
{
  int N = w->s->N;
  sc[0] = w->E_L;
  sc[1] = w->KE;
  sc[2] = w->PE;
  sc[3] = w->neE;
  sc[4] = w->eeE;
  sc[5] = w->U;
  sc[6] = w->U_xx;
  sc[7] = w->D_xx;
  sc[8] = w->s->na > 0 ? w->det[0][0] : 1.0;
  sc[9] = w->s->nb > 0 ? w->det[1][0] : 1.0;
  sc[10] = w->singular ? 1.0 : 0.0;
  sc[11] = w->logpsi;
  sc[12] = w->sign;
  sc[13] = w->sign * exp(w->logpsi);
  for (int i = 0; i < 3 * N; i++) {
    if (grad) grad[i] = w->grad[i];
    if (mgrad) mgrad[i] = w->mgrad[i];
  }
}

/* grad(D)/D of every electron, the Slater part without the Jastrow
   (QMCWalkerData::D_x, written to configuration files) */
void orc_walker_slater_grad(const orc_walker *w, double *out)
{
  for (int i = 0; i < 3 * w->s->N; i++) out[i] = w->D_x[i];
}

/* the inverse of determinant 0 (Dc_invA(0) / Dc_invB(0)) */
void orc_walker_inverse(const orc_walker *w, int beta, double *out)
{
  int n = beta ? w->s->nb : w->s->na;
  memcpy(out, w->inv[beta ? 1 : 0], sizeof(double) * n * n);
}

/* how much more the determinant-weighted sums of the laplacian amplify
 * rounding than a single determinant would (1 for one determinant) */
double orc_walker_kappa(const orc_walker *w) { return w->kappa; }

/* the inverse of determinant ci */
void orc_walker_inverse_det(const orc_walker *w, int beta, int ci, double *out)
{
  int n = beta ? w->s->nb : w->s->na;
  memcpy(out, w->inv[beta ? 1 : 0] + (size_t)ci * n * n, sizeof(double) * n * n);
}
