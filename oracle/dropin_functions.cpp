// dropin_functions.cpp -- QMcBeaver's QMCFunctions implemented by
// libqmcb200: the drop-in a QMcBeaver maintainer would add, compiled here
// against the reference's own headers and linked with its objects into
// oracle/_ref/QMcBeaver_b200.x (oracle/Makefile, target `dropin`).
//
// INTEGRATION BUILD.  Nothing in the product links this file; it shows the
// library running inside the unmodified reference driver (QMCRun,
// QMCWalker, their random numbers and statistics) and is run by
// tests/test_dropin_gpu.py.
//
//   * QMCB200Functions derives from QMCSCFJastrow so that QMCRun's own
//     set-up (QMCRun::initializeFunction static_casts the object and calls
//     initialize, QMcBeaver/src/QMCRun.cpp:143-159) keeps working; it
//     overrides both QMCFunctions::evaluate forms
//     (QMcBeaver/include/QMCFunctions.h:67-70) with qmcb_evaluate.
//   * QMCFunctionsFactory::functionsFactory is replaced by the version
//     below (the reference's QMCFunctionsFactory.o is left out of the
//     link): with QMCB_DROPIN set in the environment it returns the library
//     for "restricted" / "unrestricted" inputs, otherwise what the
//     reference returns (QMcBeaver/src/QMCFunctionsFactory.cpp:20-37).
//   * The system description is read from what QMCInput holds: nuclei
//     (Molecule), basis functions (BF, one coefficient table per atom),
//     the occupied orbital rows (WF), Pade / FixedCuspPade two-body
//     functions (JP).  Cusp replacement is fitted by the library (its fit
//     is bit-identical to the reference's).  Several determinants,
//     three-body terms and other correlation-function forms are refused.
//   * Every call here is an all-electron evaluation (which_e = -1) of the
//     configurations the reference hands over.
//     The reference passes one shared trial-walker QMCWalkerData to
//     evaluate for every walker (QMCWalker::initializePropagation copies the
//     walker into a static child, QMcBeaver/src/QMCWalker.cpp:179-198), so
//     a QMCWalkerData address does not identify a walker; single-electron
//     inputs (one_e_per_iter 1) are therefore evaluated here by a full
//     evaluation of the moved configuration in a scratch slot.
//
// Private members of the reference classes are opened to read the tables
// the reference keeps there (a maintainer would add accessors instead).
#include <execinfo.h>
#include <signal.h>
#include <unistd.h>

#include <cmath>
#include <cstdlib>
#include <iostream>
#include <list>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#define private public
#define protected public
#include "FixedCuspPadeCorrelationFunction.h"
#include "PadeCorrelationFunction.h"
#include "QMCFunctionsFactory.h"
#include "QMCHarmonicOscillator.h"
#include "QMCInput.h"
#include "QMCSCFJastrow.h"
#undef private
#undef protected

#include "qmcb200.h"

namespace {

[[noreturn]] void die(const std::string &msg)
{
  std::cerr << "QMCB200Functions: " << msg << std::endl;
  std::exit(1);
}

// P(r) / Q(r) coefficients of a Pade-family correlation function; false
// for the zero function, a fatal error for forms the library lacks.
bool pade_tables(QMCCorrelationFunctionParameters *cp, std::vector<double> &num, std::vector<double> &den)
{
  if (!cp) return false;
  QMCCorrelationFunction *f = cp->getCorrelationFunction();
  if (cp->CorrelationFunctionType == "None" || !f) return false;
  Array1D<double> *pn = nullptr, *pd = nullptr;
  if (auto *p = dynamic_cast<PadeCorrelationFunction *>(f)) {
    pn = &p->Numerator.coefficients;
    pd = &p->Denominator.coefficients;
  } else if (auto *q = dynamic_cast<FixedCuspPadeCorrelationFunction *>(f)) {
    pn = &q->Numerator.coefficients;
    pd = &q->Denominator.coefficients;
  } else {
    die("correlation function type " + cp->CorrelationFunctionType + " is not evaluated by the library");
  }
  if (pn->dim1() > QMCB_PADE_MAX || pd->dim1() > QMCB_PADE_MAX) die("Pade polynomial longer than QMCB_PADE_MAX");
  num.assign(QMCB_PADE_MAX, 0.0);
  den.assign(QMCB_PADE_MAX, 0.0);
  for (int i = 0; i < pn->dim1(); i++) num[i] = (*pn)(i);
  for (int i = 0; i < pd->dim1(); i++) den[i] = (*pd)(i);
  return true;
}

// A fatal signal prints the call stack (module + offset per frame, for
// addr2line) before the default action ends the process.
void fatal_signal(int sig)
{
  const char msg[] = "QMCB200Functions: fatal signal, call stack:\n";
  (void)!write(2, msg, sizeof(msg) - 1);
  void *frames[64];
  backtrace_symbols_fd(frames, backtrace(frames, 64), 2);
  signal(sig, SIG_DFL);
  raise(sig);
}

}  // namespace

// Handles of every QMCB200Functions created (released at exit).
static std::vector<qmcb_handle *> &live_handles()
{
  static std::vector<qmcb_handle *> v;
  return v;
}

class QMCB200Functions : public QMCSCFJastrow {
 public:
  explicit QMCB200Functions(QMCInput *in) : in_(in)
  {
    signal(SIGBUS, fatal_signal);
    signal(SIGSEGV, fatal_signal);
    build_desc();
    // one scratch slot per walker of a pass, twice for the reference's
    // second evaluation of a rejected move
    const int cap = 2 * (int)std::max<long>(1, in->flags.walkers_per_pass);
    if (qmcb_create(&desc_, cap, &h_) != QMCB_OK) die(qmcb_last_error(nullptr));
    qmcb_run_params p;
    qmcb_get_params(h_, &p);
    p.dt = in->flags.dt;
    p.qf_modification = in->flags.QF_modification_type == "umrigar93_equalelectrons"     ? QMCB_QF_UMRIGAR93_EQUAL
                        : in->flags.QF_modification_type == "umrigar93_unequalelectrons" ? QMCB_QF_UMRIGAR93_UNEQUAL
                                                                                          : QMCB_QF_NONE;
    p.qf_equal_a = in->flags.umrigar93_equalelectrons_parameter;
    if (qmcb_set_params(h_, &p) != QMCB_OK) die(qmcb_last_error(h_));
    live_handles().push_back(h_);
    static bool registered = false;
    if (!registered) {
      std::atexit([] {
        for (qmcb_handle *x : live_handles()) qmcb_destroy(x);
        live_handles().clear();
      });
      registered = true;
    }
    std::clog << "QMCB200Functions: evaluate through " << qmcb_version() << std::endl;
  }
  // The handle lives until the process ends and is released by an exit
  // handler registered after the library's first CUDA call, so that it runs
  // before the CUDA runtime's own exit handler (handlers run in reverse
  // order); the reference deletes its QMCFunctions from destructors whose
  // order against the runtime's shutdown is not fixed.
  ~QMCB200Functions()
  {
    // QMCSlater::ciDet is set only for several determinants at allocation
    // (QMcBeaver/src/QMCSlater.cpp:113-116) and otherwise pointed at a
    // Slater matrix by QMCSlater's own evaluation (:669), which this class
    // never runs; its destructor deletes it when nonzero (:299-300), so the
    // uninitialised pointer is cleared here, before ~QMCSCFJastrow runs.
    if (in_->WF.getNumberDeterminants() == 1) {
      Alpha.ciDet = nullptr;
      Beta.ciDet = nullptr;
    }
  }

  void evaluate(Array1D<QMCWalkerData *> &wd, Array1D<Array2D<double> *> &X, int num)
  {
    const int N = N_;
    std::vector<int> slots(num);
    std::vector<double> R((size_t)num * N * 3);
    for (int w = 0; w < num; w++) {
      slots[w] = w;
      for (int e = 0; e < N; e++)
        for (int d = 0; d < 3; d++) R[((size_t)w * N + e) * 3 + d] = X(w)->get(e, d);
    }
    std::vector<double> lp(num), sg(num), g((size_t)num * N * 3), mg((size_t)num * N * 3), lap(num), el(num),
        pe(3 * num);
    std::vector<unsigned char> st(num);
    // all-electron evaluation of every configuration handed over (see the
    // file comment on single-electron inputs)
    if (qmcb_evaluate(h_, -1, slots.data(), num, R.data(), lp.data(), sg.data(), g.data(), mg.data(), lap.data(),
                      el.data(), pe.data(), st.data()) != QMCB_OK)
      die(qmcb_last_error(h_));
    for (int w = 0; w < num; w++) {
      QMCWalkerData *d = wd(w);
      d->psi = QMCDouble(sg[w], 1.0, 0.0, lp[w]);
      d->localEnergy = el[w];
      d->kineticEnergy = -0.5 * lap[w];
      d->potentialEnergy = pe[3 * w];
      d->neEnergy = pe[3 * w + 1];
      d->eeEnergy = pe[3 * w + 2];
      for (int e = 0; e < N; e++)
        for (int k = 0; k < 3; k++) {
          d->gradPsiRatio(e, k) = g[((size_t)w * N + e) * 3 + k];
          d->modifiedGradPsiRatio(e, k) = mg[((size_t)w * N + e) * 3 + k];
        }
      d->singular |= (st[w] & (QMCB_ST_SINGULAR | QMCB_ST_NAN)) != 0;
      d->x2 = d->y2 = d->z2 = 0.0;
      for (int e = 0; e < N; e++) {
        d->x2 += X(w)->get(e, 0) * X(w)->get(e, 0);
        d->y2 += X(w)->get(e, 1) * X(w)->get(e, 1);
        d->z2 += X(w)->get(e, 2) * X(w)->get(e, 2);
      }
    }
  }

  void evaluate(Array2D<double> &X, QMCWalkerData &data)
  {
    Array1D<QMCWalkerData *> a(1);
    a(0) = &data;
    Array1D<Array2D<double> *> x(1);
    x(0) = &X;
    evaluate(a, x, 1);
  }

 private:
  QMCInput *in_;
  qmcb_handle *h_ = nullptr;
  qmcb_system_desc desc_{};
  int N_ = 0;
  // tables the descriptor points into
  std::vector<double> nuc_xyz_, nuc_z_, pexp_, pcoef_, mo_a_, mo_b_, pnum_, pden_;
  std::vector<int> bf_atom_, bf_pow_, bf_np_, bf_off_, nnum_, nden_, en_up_, en_dn_;

  int add_pade(QMCCorrelationFunctionParameters *cp)
  {
    std::vector<double> n, d;
    if (!pade_tables(cp, n, d)) return -1;
    pnum_.insert(pnum_.end(), n.begin(), n.end());
    pden_.insert(pden_.end(), d.begin(), d.end());
    nnum_.push_back(QMCB_PADE_MAX);
    nden_.push_back(QMCB_PADE_MAX);
    return (int)nnum_.size() - 1;
  }

  void build_desc()
  {
    QMCInput &I = *in_;
    if (I.WF.getNumberDeterminants() != 1) die("several determinants are not evaluated by this drop-in");
    if (I.flags.use_three_body_jastrow && I.JP.getNumberNEupEdnParameters() + I.JP.getNumberNEupEupParameters() +
                                                  I.JP.getNumberNEdnEdnParameters() > 0)
      die("three-body Jastrow terms are not evaluated by this drop-in");
    const int M = I.Molecule.getNumberAtoms();
    for (int a = 0; a < M; a++) {
      for (int x = 0; x < 3; x++) nuc_xyz_.push_back(I.Molecule.Atom_Positions(a, x));
      nuc_z_.push_back(I.Molecule.Z(a));
    }
    // basis: one coefficient table per atom, functions in file order
    // (QMCBasisFunction's BFLookupTable, QMcBeaver/src/QMCBasisFunction.cpp:177-201)
    for (int a = 0; a < M; a++) {
      QMCBasisFunctionCoefficients *c = I.BF.getBFCoeffs(a);
      for (int f = 0; f < c->getNumberBasisFunctions(); f++) {
        bf_atom_.push_back(a);
        for (int x = 0; x < 3; x++) bf_pow_.push_back(c->xyz_powers(f, x));
        bf_np_.push_back(c->N_Gauss(f));
        bf_off_.push_back((int)pexp_.size());
        for (int g = 0; g < c->N_Gauss(f); g++) {
          pexp_.push_back(c->Coeffs(f, g, 0));
          pcoef_.push_back(c->Coeffs(f, g, 1));
        }
      }
    }
    const int K = (int)bf_atom_.size();
    const int na = I.WF.getNumberElectrons(true), nb = I.WF.getNumberElectrons(false);
    N_ = na + nb;
    // occupied orbital rows (QMCWavefunction::getCoeff: the active rows of
    // the one determinant, QMcBeaver/src/QMCWavefunction.cpp:843-905)
    for (int sp = 0; sp < 2; sp++) {
      Array2D<qmcfloat> *C = I.WF.getCoeff(sp == 0);
      std::vector<double> &mo = sp == 0 ? mo_a_ : mo_b_;
      const int n = sp == 0 ? na : nb;
      if (n > 0 && (C->dim1() != n || C->dim2() != K)) die("orbital table shape does not match the occupation");
      for (int o = 0; o < n; o++)
        for (int k = 0; k < K; k++) mo.push_back((*C)(o, k));
    }
    // two-body functions
    int ee[3] = {-1, -1, -1};
    if (na > 0 && nb > 0) ee[0] = add_pade(I.JP.getElectronUpElectronDownParameters());
    if (na > 1) ee[1] = add_pade(I.JP.getElectronUpElectronUpParameters());
    if (nb > 1) ee[2] = add_pade(I.JP.getElectronDownElectronDownParameters());
    Array1D<std::string> *types = I.JP.getNucleiTypes();
    Array1D<QMCCorrelationFunctionParameters> *up = na > 0 ? I.JP.getElectronUpNuclearParameters() : nullptr;
    Array1D<QMCCorrelationFunctionParameters> *dn = nb > 0 ? I.JP.getElectronDownNuclearParameters() : nullptr;
    std::map<int, int> f_up, f_dn;
    for (int t = 0; types && t < types->dim1(); t++) {
      f_up[t] = up ? add_pade(&(*up)(t)) : -1;
      f_dn[t] = dn ? add_pade(&(*dn)(t)) : -1;
    }
    for (int a = 0; a < M; a++) {
      int t = -1;
      for (int i = 0; types && i < types->dim1(); i++)
        if (I.Molecule.Atom_Labels(a) == (*types)(i)) {
          t = i;
          break;
        }
      en_up_.push_back(t >= 0 ? f_up[t] : -1);
      en_dn_.push_back(t >= 0 ? f_dn[t] : -1);
    }
    qmcb_system_desc &d = desc_;
    d.n_nuclei = M;
    d.nuc_xyz = nuc_xyz_.data();
    d.nuc_charge = nuc_z_.data();
    d.n_alpha = na;
    d.n_beta = nb;
    d.n_basis = K;
    d.bf_atom = bf_atom_.data();
    d.bf_powers = bf_pow_.data();
    d.bf_nprim = bf_np_.data();
    d.bf_prim_offset = bf_off_.data();
    d.n_prim_total = (int)pexp_.size();
    d.prim_exponent = pexp_.data();
    d.prim_coeff = pcoef_.data();
    d.mo_alpha = mo_a_.data();
    d.mo_beta = mo_b_.data();
    d.n_pade = (int)nnum_.size();
    d.pade_num = pnum_.data();
    d.pade_den = pden_.data();
    d.pade_nnum = nnum_.data();
    d.pade_nden = nden_.data();
    d.corr_type = nullptr;
    d.corr_param = nullptr;
    for (int k = 0; k < 3; k++) d.ee_pade[k] = ee[k];
    d.en_pade_up = en_up_.data();
    d.en_pade_dn = en_dn_.data();
    d.n_det = 1;
    d.replace_cusps = I.flags.replace_electron_nucleus_cusps ? 1 : 0;
    d.cusp_alpha = nullptr;
    d.cusp_beta = nullptr;
    d.n_tb = 0;
  }
};

QMCFunctions *QMCFunctionsFactory::functionsFactory(QMCInput *input, string &Type)
{
  if (Type == "restricted" || Type == "unrestricted") {
    if (std::getenv("QMCB_DROPIN")) return new QMCB200Functions(input);
    return new QMCSCFJastrow();
  }
  if (Type == "harmonicoscillator") return new QMCHarmonicOscillator(input);
  std::cerr << "ERROR: Unknown wavefunction type (" << Type << ") being assigned in QMCFunctionsFactory!" << std::endl;
  std::exit(0);
}
