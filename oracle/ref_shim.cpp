// ref_shim.cpp -- C entry points into the reference QMcBeaver CPU code.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's own sources (read-only tree, see oracle/Makefile) into
// oracle/_ref/libqmcref.so.  It is used by tests/golden/make_golden.py to
// produce golden vectors and by tests that pin the C restatement
// (oracle/qmc_oracle.c) to the reference.  Nothing in the product links it.
//
// It drives the reference exactly the way QMCWalker / QMCRun do:
//   * QMCWalkerData::initialize(3,-1,-1)        QMcBeaver/src/QMCWalkerData.cpp:56
//   * QMCWalkerData::updateDistances(R)         QMcBeaver/src/QMCWalkerData.cpp:302
//   * QMCSCFJastrow::evaluate(wd[], R[], num)   QMcBeaver/src/QMCSCFJastrow.cpp:91
// with whichE = -1 for a full (LU) evaluation and whichE = e for a single
// electron update (Sherman-Morrison path, requires one_e_per_iter 1 in the
// input file, QMcBeaver/src/QMCSlater.cpp:700-711).

// Standard headers first; then the reference's own headers with their
// private members opened, so that the cusp-replacement records the
// reference fitted can be read back for comparison (ref_cusp_params).
#include <cmath>
#include <iostream>
#include <list>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#define private public
#define protected public
#include "QMCInput.h"
#include "QMCSCFJastrow.h"
#include "QMCWalkerData.h"
#include "Array1D.h"
#include "Array2D.h"
#include <cmath>
#include <vector>

// The reference defines these globals next to main() in QMcBeaver.cpp,
// which is left out of the library; they are defined here instead.
QMCInput globalInput;
int argc = 0;
char **argv = 0;

static QMCSCFJastrow *g_qmf = 0;
static int g_nel = 0;

// The evaluator ref_walker.cpp drives walkers with.
QMCSCFJastrow *ref_shim_functions(void) { return g_qmf; }

extern "C" {

int ref_init(const char *ckmf)
{
  globalInput.read(std::string(ckmf));
  g_nel = globalInput.WF.getNumberElectrons();
  g_qmf = new QMCSCFJastrow();
  g_qmf->initialize(&globalInput, 0);
  return g_nel;
}

int ref_num_electrons(void) { return g_nel; }
int ref_num_alpha(void) { return globalInput.WF.getNumberElectrons(true); }
int ref_num_basis(void) { return globalInput.WF.getNumberBasisFunctions(); }

void *ref_walker_new(void)
{
  QMCWalkerData *wd = new QMCWalkerData();
  wd->initialize(3, -1, -1);
  return wd;
}

void ref_walker_free(void *w) { delete (QMCWalkerData *)w; }

void *ref_walker_clone(void *w)
{
  QMCWalkerData *src = (QMCWalkerData *)w;
  QMCWalkerData *dst = new QMCWalkerData();
  dst->initialize(3, -1, -1);
  *dst = *src;
  return dst;
}

// Evaluates `num` walkers at positions R[num][N][3] with a uniform whichE,
// as QMCRun::propagateWalkers does (QMcBeaver/src/QMCRun.cpp:43-55).
int ref_evaluate(void **walkers, const double *R, int num, int whichE)
{
  std::vector<Array2D<double> > Rs(num);
  Array1D<Array2D<double> *> rp(num);
  Array1D<QMCWalkerData *> wp(num);
  for (int w = 0; w < num; w++) {
    Rs[w].allocate(g_nel, 3);
    for (int e = 0; e < g_nel; e++)
      for (int d = 0; d < 3; d++) Rs[w](e, d) = R[(w * g_nel + e) * 3 + d];
    QMCWalkerData *wd = (QMCWalkerData *)walkers[w];
    wd->whichE = whichE;
    wd->singular = false;
    wd->updateDistances(Rs[w]);
    rp(w) = &Rs[w];
    wp(w) = wd;
  }
  g_qmf->evaluate(wp, rp, num);
  return 0;
}

// scalars: [0] E_L, [1] kinetic, [2] potential, [3] e-n potential,
// [4] e-e potential, [5] ln Jastrow U, [6] lap(lnJ) U_xx, [7] lap(D)/D D_xx,
// [8] alpha determinant, [9] beta determinant, [10] singular flag,
// [11] ln|psi| (= ln|detA detB| + U), [12] sign(psi), [13] (double)psi
// grad[N][3]: gradPsiRatio; mgrad[N][3]: modifiedGradPsiRatio
void ref_walker_get(void *w, double *scalars, double *grad, double *mgrad)
{
  QMCWalkerData *wd = (QMCWalkerData *)w;
  scalars[0] = wd->localEnergy;
  scalars[1] = wd->kineticEnergy;
  scalars[2] = wd->potentialEnergy;
  scalars[3] = wd->neEnergy;
  scalars[4] = wd->eeEnergy;
  scalars[5] = wd->U;
  scalars[6] = wd->U_xx;
  scalars[7] = wd->D_xx;
  double da = wd->DcA.dim1() > 0 ? wd->DcA(0) : 1.0;
  double db = wd->DcB.dim1() > 0 ? wd->DcB(0) : 1.0;
  scalars[8] = da;
  scalars[9] = db;
  scalars[10] = wd->singular ? 1.0 : 0.0;
  scalars[11] = std::log(std::fabs(da)) + std::log(std::fabs(db)) + wd->U;
  scalars[12] = (da * db < 0) ? -1.0 : 1.0;
  const int ndet = globalInput.WF.getNumberDeterminants();
  if (ndet > 1) {
    // psi_D = sum_ci c_ci DcA(ci) DcB(ci) (QMCSCFJastrow::update_SCF)
    double D = 0.0;
    for (int ci = 0; ci < ndet; ci++) {
      double a = wd->DcA.dim1() > ci ? wd->DcA(ci) : 1.0;
      double b = wd->DcB.dim1() > ci ? wd->DcB(ci) : 1.0;
      D += globalInput.WF.CI_coeffs(ci) * a * b;
    }
    scalars[11] = std::log(std::fabs(D)) + wd->U;
    scalars[12] = D < 0 ? -1.0 : 1.0;
  }
  scalars[13] = (double)wd->psi;
  for (int e = 0; e < g_nel; e++)
    for (int d = 0; d < 3; d++) {
      if (grad) grad[e * 3 + d] = wd->gradPsiRatio(e, d);
      if (mgrad) mgrad[e * 3 + d] = wd->modifiedGradPsiRatio(e, d);
    }
}

// The alpha / beta inverse Slater matrices as stored by the reference
// (Dc_invA(0)(o,e), QMcBeaver/src/QMCWalkerData.cpp:69-76).
void ref_walker_inverse(void *w, int beta, double *out)
{
  QMCWalkerData *wd = (QMCWalkerData *)w;
  Array2D<double> &inv = beta ? wd->Dc_invB(0) : wd->Dc_invA(0);
  for (int i = 0; i < inv.dim1(); i++)
    for (int j = 0; j < inv.dim2(); j++) out[i * inv.dim2() + j] = inv(i, j);
}

// The reference's fitted cusp replacement of (nucleus, orbital) for one
// spin: rc, sgn0, C, alpha_0..alpha_4 (QMCElectronNucleusCuspParameters);
// zeros where no replacement was fitted.
void ref_cusp_params(int beta, int atom, int orbital, double *out)
{
  for (int i = 0; i < 8; i++) out[i] = 0.0;
  QMCSlater &S = beta ? g_qmf->Beta : g_qmf->Alpha;
  QMCElectronNucleusCuspParameters &P = S.ElectronNucleusCusp.ORParams(atom, orbital);
  out[0] = P.rc;
  if (P.rc <= 0.0) return;
  out[1] = P.sgn0;
  out[2] = P.C;
  Array1D<double> c = P.alpha.getCoefficients();
  for (int i = 0; i < 5 && i < c.dim1(); i++) out[3 + i] = c(i);
}

// The reference's three-body coefficients for nucleus type j (in its
// NucleiTypes order) and pair kind (0 up-down, 1 up-up, 2 down-down):
// out = [NeN, Nee, C, cutoff, used, coefficients...]; returns the count
// written (0 when the kind has no function).
int ref_three_body(int kind, int j, double *out, int cap)
{
  QMCJastrowParameters &JP = globalInput.JP;
  Array1D<QMCThreeBodyCorrelationFunctionParameters> &A =
      kind == 0 ? JP.EupEdnNuclear : (kind == 1 ? JP.EupEupNuclear : JP.EdnEdnNuclear);
  if (j >= A.dim1()) return 0;
  QMCThreeBodyCorrelationFunctionParameters &P = A(j);
  if (!P.isUsed()) return 0;
  int T = P.Parameters.dim1();
  if (5 + T > cap) return -1;
  out[0] = P.NeN;
  out[1] = P.Nee;
  out[2] = P.C;
  out[3] = P.cutoff;
  out[4] = 1.0;
  for (int i = 0; i < T; i++) out[5 + i] = P.Parameters(i);
  return 5 + T;
}

} // extern "C"
