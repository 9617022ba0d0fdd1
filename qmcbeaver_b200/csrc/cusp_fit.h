/*
 * cusp_fit.h -- the electron-nucleus cusp replacement fit of QMcBeaver
 * (replace_electron_nucleus_cusps = 1), host code in plain C99.
 *
 * Near every nucleus the s-type part of each orbital is replaced by
 *   phi~(r) = C + sgn0 exp(alpha(r)),  alpha a quartic,  for r < rc,
 * fitted so that value, first and second derivative match the original at
 * rc, the cusp condition holds at the nucleus, and the local energy of the
 * replacement stays closest to an ideal curve (Ma, Towler, Drummond, Needs,
 * J. Chem. Phys. 122, 224322 (2005)).  This file restates, with the same
 * operation order, QMCElectronNucleusCusp::fitReplacementOrbitals /
 * determineRc / fitOrbitalParameters (QMcBeaver/src/QMCElectronNucleusCusp.cpp:
 * 46-572), QMCElectronNucleusCuspParameters::fitReplacementOrbital /
 * calculateSigmaSq / findMaxDeviation / calculateLocalEnergy
 * (QMcBeaver/src/QMCElectronNucleusCuspParameters.cpp:287-587), and the
 * Laguerre root finder it uses (Polynomial::zroots / laguer,
 * QMcBeaver/src/Polynomial.cpp:253-430, with the Complex arithmetic of
 * QMcBeaver/src/Complex.cpp).  Loops the reference runs until a condition
 * holds are bounded here; exceeding a bound is reported as an error.
 */
#ifndef QMCB_CUSP_FIT_H
#define QMCB_CUSP_FIT_H

#ifdef __cplusplus
extern "C" {
#endif

/* One fitted record: rc, sgn0, C, alpha_0..alpha_4 (rc = 0: no replacement). */
#define QMCB_CUSP_REC 8

/*
 * Fits the replacement of every (nucleus, orbital) pair.
 *   M, xyz[M][3], Z[M]            nuclei (Z integral, as the reference's int Z)
 *   K, bf_atom[K], bf_pow[K][3], bf_nprim[K], bf_off[K], pexp[], pcoef[]
 *                                 the basis (functions grouped by atom, file order)
 *   n_orb, mo[n_orb][K]           orbital rows of the spin (the Slater columns)
 *   out[M][n_orb][QMCB_CUSP_REC]
 * Returns 0, or -1 with a message in err[256] when a search does not end.
 */
int qmcb_cusp_fit(int M, const double *xyz, const double *Z, int K, const int *bf_atom, const int *bf_pow,
                  const int *bf_nprim, const int *bf_off, const double *pexp, const double *pcoef, int n_orb,
                  const double *mo, double *out, char *err);

#ifdef __cplusplus
}
#endif
#endif
