/*
 * qmc_oracle.h -- CPU restatement of QMcBeaver's Slater-Jastrow walker
 * evaluation (TEST INFRASTRUCTURE: used only by tests/, the smoke check and
 * the CPU baseline of bench.py as the checker; never by the product path).
 *
 * The entry points mirror oracle/ref_shim.cpp (the reference itself, linked
 * from its sources) so the two can be compared call for call:
 *   orc_evaluate(walkers[], R, num, whichE)  ==  QMCSCFJastrow::evaluate
 *     (QMcBeaver/src/QMCSCFJastrow.cpp:91-181) after
 *     QMCWalkerData::updateDistances (QMcBeaver/src/QMCWalkerData.cpp:302-344)
 * Pinned against the reference build (oracle/_ref) and the golden vectors
 * under tests/golden/.
 */
#ifndef QMC_ORACLE_H
#define QMC_ORACLE_H

#include "../include/qmcb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system orc_system;
typedef struct orc_walker orc_walker;

/* qf_mod / qf_a / dt feed calculate_Modified_Grad_PsiRatio. */
orc_system *orc_system_new(const qmcb_system_desc *d, int qf_mod, double qf_a, double dt);
void orc_system_free(orc_system *s);
int orc_num_electrons(const orc_system *s);

orc_walker *orc_walker_new(const orc_system *s);
orc_walker *orc_walker_clone(const orc_walker *w);
void orc_walker_copy(orc_walker *dst, const orc_walker *src);
void orc_walker_free(orc_walker *w);

/* R: [num][N][3]; whichE = -1 (all electrons) or the moved electron. */
int orc_evaluate(const orc_system *s, orc_walker **walkers, const double *R, int num, int whichE);

/* Same layout as ref_walker_get (oracle/ref_shim.cpp). */
void orc_walker_get(const orc_walker *w, double *scalars, double *grad, double *mgrad);
void orc_walker_slater_grad(const orc_walker *w, double *out);
void orc_walker_inverse(const orc_walker *w, int beta, double *out);
void orc_walker_inverse_det(const orc_walker *w, int beta, int ci, double *out);
double orc_walker_kappa(const orc_walker *w);

/* Basis values for one electron position (5 x K: val, gx, gy, gz, lap),
 * exposed for unit tests of the basis kernel. */
void orc_basis_at(const orc_system *s, const double *r, double *out);

#ifdef __cplusplus
}
#endif
#endif
