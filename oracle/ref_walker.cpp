// ref_walker.cpp -- one move of the reference QMcBeaver's own QMCWalker.
//
// TEST INFRASTRUCTURE ONLY.  Compiled with the reference's sources (read-only
// tree, see oracle/Makefile) into oracle/_ref/libqmcref.so next to
// ref_shim.cpp, in a translation unit of its own so that the reference's
// headers are read exactly as its own sources read them.  The two private
// members it needs (the forward Green's function a move records and the
// reverse Green's function of the trial walker) are reached through member
// pointers named in explicit template instantiations, where access checking
// does not apply; so are the four fields of a QMCDouble, k a^b exp(c).
#include <cmath>
#include "QMCInput.h"
#include "QMCSCFJastrow.h"
#include "QMCWalker.h"
#include "Random.h"

extern QMCInput globalInput;
QMCSCFJastrow *ref_shim_functions(void);

namespace {
template <typename Tag, typename Tag::type M> struct Expose {
  friend typename Tag::type member(Tag) { return M; }
};
struct ForwardGF {
  typedef QMCDouble QMCWalker::*type;
  friend type member(ForwardGF);
};
struct ReverseGF {
  typedef QMCDouble (QMCWalker::*type)();
  friend type member(ReverseGF);
};
struct QK { typedef double QMCDouble::*type; friend type member(QK); };
struct QA { typedef double QMCDouble::*type; friend type member(QA); };
struct QB { typedef double QMCDouble::*type; friend type member(QB); };
struct QC { typedef double QMCDouble::*type; friend type member(QC); };

// ln of a QMCDouble k a^b exp(c) without forming its value (which
// under- or overflows for many-electron Green's functions).
double log_of(const QMCDouble &q)
{
  const double k = q.*member(QK()), a = q.*member(QA()), b = q.*member(QB()), c = q.*member(QC());
  return log(k) + (b != 0.0 ? b * log(a) : 0.0) + c;
}
}  // namespace
template struct Expose<QK, &QMCDouble::k>;
template struct Expose<QA, &QMCDouble::a>;
template struct Expose<QB, &QMCDouble::b>;
template struct Expose<QC, &QMCDouble::c>;
template struct Expose<ForwardGF, &QMCWalker::forwardGreensFunction>;
template struct Expose<ReverseGF, &QMCWalker::calculateReverseGreensFunction>;

extern "C" {

// One move from positions R0[N][3] (QMCWalker::initializePropagation ->
// moveElectrons, the trial walker's evaluation, calculateReverseGreensFunction;
// QMcBeaver/src/QMCWalker.cpp:179-198, 283-310, 400-586, 783-926) with the
// sampling_method of the input file and the reference's random stream
// seeded by `seed`.  Rnew[N][3]: the proposed positions; gf[0] =
// ln G(R -> R'), gf[1] = ln G(R' -> R), gf[2] = G(R' -> R) / G(R -> R') as
// QMCDouble divides; mg[2][N][3]: modifiedGradPsiRatio of the original and
// the trial walker.  Returns the electron moved (-1: all).
int ref_walker_move(const double *R0, int iteration, long seed, double *Rnew, double *gf, double *mg)
{
  QMCSCFJastrow *qmf = ref_shim_functions();
  const int N = globalInput.WF.getNumberElectrons();
  ran.initialize(seed, 0);
  QMCWalker w;
  w.initialize(&globalInput);
  Array2D<double> R(N, 3);
  for (int e = 0; e < N; e++)
    for (int d = 0; d < 3; d++) R(e, d) = R0[3 * e + d];
  w.setR(R);
  QMCWalkerData *wd = w.getWalkerData();
  wd->updateDistances(*w.getR());
  qmf->evaluate(*w.getR(), *wd);
  for (int e = 0; e < N; e++)
    for (int d = 0; d < 3; d++) mg[3 * e + d] = wd->modifiedGradPsiRatio(e, d);
  QMCWalkerData *data = 0;
  Array2D<double> *rc = 0;
  w.initializePropagation(data, rc, iteration);
  qmf->evaluate(*rc, *data);
  QMCDouble fwd = w.*member(ForwardGF());
  QMCDouble rev = (w.*member(ReverseGF()))();
  for (int e = 0; e < N; e++)
    for (int d = 0; d < 3; d++) {
      Rnew[3 * e + d] = (*rc)(e, d);
      mg[3 * (N + e) + d] = data->modifiedGradPsiRatio(e, d);
    }
  gf[0] = log_of(fwd);
  gf[1] = log_of(rev);
  gf[2] = (double)(rev / fwd);
  return data->whichE;
}

}  // extern "C"
