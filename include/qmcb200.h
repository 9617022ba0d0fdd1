/*
 * qmcb200.h -- C ABI of the B200 Slater-Jastrow walker-evaluation library
 * (libqmcb200.so).
 *
 * The library replaces QMcBeaver's wavefunction-evaluation hot path:
 *   QMCFunctions::evaluate(Array1D<QMCWalkerData*>&, Array1D<Array2D<double>*>&, int)
 *     (QMcBeaver/include/QMCFunctions.h:67-70), implemented by
 *   QMCSCFJastrow::evaluate (QMcBeaver/src/QMCSCFJastrow.cpp:91-181)
 * and the single-electron Metropolis / DMC step around it
 *   QMCRun::propagateWalkers + QMCWalker::{initialize,process}Propagation
 *     (QMcBeaver/src/QMCRun.cpp:28-87, QMcBeaver/src/QMCWalker.cpp:179-282).
 *
 * Conventions
 *   - Plain C types only; every function returns 0 on success and a positive
 *     QMCB_E_* code on failure; qmcb_last_error() gives the message.
 *   - Electrons are ordered alpha [0, n_alpha) then beta
 *     (QMcBeaver/src/QMCSCFJastrow.cpp:68-76); positions are [N][3] doubles.
 *   - Per-walker state (inverse Slater matrices, Slater rows and derivative
 *     rows, Jastrow gradients, energies) lives in device memory, addressed by
 *     a walker slot in [0, max_walkers).  This is the state QMCWalkerData
 *     carries in the reference (QMcBeaver/src/QMCWalkerData.cpp:56-161).
 *   - One handle = one CUDA stream; a handle is not thread safe.
 */
#ifndef QMCB200_H
#define QMCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QMCB_PADE_MAX 16

/* two-body correlation function forms (QMcBeaver/src/QMCCorrelationFunctionFactory.cpp) */
#define QMCB_CORR_PADE 0        /* P(r)/Q(r): Pade and FixedCuspPade */
#define QMCB_CORR_CAMBRIDGE2 1  /* (fL r - 1)^C alpha(fL r) for fL r < 1, else 0 */

/* error codes */
#define QMCB_OK 0
#define QMCB_E_ARG 1      /* bad argument / size */
#define QMCB_E_CUDA 2     /* CUDA runtime error */
#define QMCB_E_NOMEM 3    /* device allocation failed */
#define QMCB_E_STATE 4    /* call order (e.g. evaluate one electron before a full evaluation) */
#define QMCB_E_LIMIT 5    /* size beyond a compiled limit */

/* per-walker status bits written by evaluate / steps */
#define QMCB_ST_SINGULAR 1 /* Slater matrix singular or psi ratio 0 (wd->singular) */
#define QMCB_ST_NAN 2      /* NaN in gradient / energy */

/* run types, samplers, quantum-force modifications (QMcBeaver/src/QMCFlags.cpp) */
#define QMCB_VMC 0
#define QMCB_DMC 1
#define QMCB_NO_IMPORTANCE_SAMPLING 0
#define QMCB_IMPORTANCE_SAMPLING 1
/* umrigar93_importance_sampling: the drift-diffusion move near a nucleus mixed
   with a hydrogen-like move (QMCWalker::moveElectronsUmrigar93ImportanceSampling,
   QMcBeaver/src/QMCWalker.cpp:400-586) */
#define QMCB_UMRIGAR93_IMPORTANCE_SAMPLING 2
#define QMCB_QF_NONE 0
#define QMCB_QF_UMRIGAR93_EQUAL 1
#define QMCB_QF_UMRIGAR93_UNEQUAL 2
#define QMCB_EMOD_NONE 0
#define QMCB_EMOD_UMRIGAR93 1
#define QMCB_EMOD_MODIFIED_UMRIGAR93 2
#define QMCB_RW_SIMPLE_SYMMETRIC 0
#define QMCB_RW_SIMPLE_ASYMMETRIC 1
#define QMCB_RW_UMRIGAR93_PROBABILITY_WEIGHTED 2

/* arithmetic of the orbital contraction and Slater updates */
#define QMCB_PREC_FP64 0  /* plain FP64 everywhere (parity path) */
#define QMCB_PREC_MIXED 1 /* FP32 orbital rows / SM update, FP64 refresh and accumulators */
/* FP64 walker state and updates; each single-electron move's orbital rows
 * (QMCSlater::update_Ds -> Array2D::gemm, QMcBeaver/src/QMCSlater.cpp:856-862)
 * come from one batched tensor-core contraction over all walkers of the step:
 * basis values and MO coefficients scaled per 32-function block and cut
 * into 8 int8 digit planes, int8 x int8 products accumulated exactly in int32
 * (tcgen05 kind::i8), every block recombined in FP64.  56 bits of every
 * product are kept relative to its block's largest basis value and largest
 * coefficient, so results match QMCB_PREC_FP64 to ~1e-15 relative on
 * well-conditioned walkers (parity bound of this mode: 1e-9).  One
 * determinant per system; the full evaluation and the LU refresh run in
 * FP64. */
#define QMCB_PREC_INT8_SLICES 2
/* FP64 walker state and updates; each move's orbital rows from the same
 * batched contraction with BF16 operands and FP32 accumulation in the tensor
 * memory (tcgen05 kind::f16, M = 128, N = 32, K = 16 per instruction):
 *   QMCB_PREC_BF16_TC    basis values and MO coefficients rounded to BF16
 *                        (8 significant bits), one product per pair;
 *   QMCB_PREC_BF16X3_TC  the split-precision variant: each value split as
 *                        hi + lo (two BF16 values, 16 significant bits) and
 *                        the products hi.hi + hi.lo + lo.hi accumulated in
 *                        FP32 (compensated products, FP32-class rows).
 * The reference's own reduced-precision option keeps float orbitals with a
 * double inverse (qmcfloat, QMcBeaver/include/Array2D.h:79-84,
 * QMcBeaver/src/QMCSlater.cpp:526-532).  These rows carry FP32-class or
 * BF16-class errors that the Slater matrices' conditioning amplifies in the
 * local energy; one determinant per system, FP64 full evaluation and LU
 * refresh. */
#define QMCB_PREC_BF16_TC 3
#define QMCB_PREC_BF16X3_TC 4

/*
 * Molecular system: what QMCInput reads from the .ckmf &geometry, &basis,
 * &wavefunction and &Jastrow sections: one or several determinants of
 * restricted or unrestricted orbitals, Pade / Cambridge2 two-body Jastrows.
 */
typedef struct qmcb_system_desc {
  int n_nuclei;                 /* M */
  const double *nuc_xyz;        /* [M][3] bohr */
  const double *nuc_charge;     /* [M] Z (Zeff) */
  int n_alpha, n_beta;          /* electrons per spin */
  int n_basis;                  /* K contracted Cartesian Gaussians */
  const int *bf_atom;           /* [K] centre of function k */
  const int *bf_powers;         /* [K][3] Cartesian powers a, b, c */
  const int *bf_nprim;          /* [K] primitives of function k */
  const int *bf_prim_offset;    /* [K] first primitive of function k */
  int n_prim_total;
  const double *prim_exponent;  /* [n_prim_total] */
  const double *prim_coeff;     /* [n_prim_total] raw contraction coefficients */
  const double *mo_alpha;       /* [n_alpha][K] occupied orbital rows (AlphaCoeffs) */
  const double *mo_beta;        /* [n_beta][K] (BetaCoeffs) */
  int n_pade;                   /* two-body correlation functions */
  const double *pade_num;       /* [n_pade][QMCB_PADE_MAX] Pade: P coefficients, P[0] = 0;
                                   Cambridge2: polynomial alpha coefficients */
  const double *pade_den;       /* [n_pade][QMCB_PADE_MAX] Pade: Q coefficients, Q[0] = 1 */
  const int *pade_nnum;         /* [n_pade] used length of the first table */
  const int *pade_nden;         /* [n_pade] used length of Q */
  const int *corr_type;         /* [n_pade] QMCB_CORR_* (NULL: all Pade) */
  const double *corr_param;     /* [n_pade][4] Cambridge2: fL, C, active (1/0), unused */
  int ee_pade[3];               /* up-down, up-up, down-down function (-1 = none) */
  const int *en_pade_up;        /* [M] up electron - nucleus function (-1 = none) */
  const int *en_pade_dn;        /* [M] down electron - nucleus function */
  /* Several determinants, psi_D = sum_c ci_coeff[c] det_alpha(c) det_beta(c)
     (QMCWavefunction with Ndeterminants > 1, QMcBeaver/src/QMCWavefunction.cpp:
     311-472, 873-977; QMCSCFJastrow::update_SCF, QMcBeaver/src/QMCSCFJastrow.cpp:
     284-327).  n_det <= 1: one determinant of all the mo_alpha / mo_beta rows
     and the fields below are ignored.  n_det > 1: mo_alpha / mo_beta hold the
     n_act_alpha / n_act_beta active orbital rows of each spin and every
     determinant lists the rows of its columns in increasing order. */
  int n_det;
  int n_act_alpha, n_act_beta;
  const int *det_occ_alpha;     /* [n_det][n_alpha] */
  const int *det_occ_beta;      /* [n_det][n_beta] */
  const double *ci_coeff;       /* [n_det] */
  /* Electron-nucleus cusp replacement (replace_electron_nucleus_cusps,
     QMCElectronNucleusCusp, QMcBeaver/src/QMCSlater.cpp:85-93,856-872): near
     each nucleus the s-type part of every orbital row is replaced by
     C + sgn0 exp(alpha(r)).  replace_cusps = 1 turns it on; cusp_alpha /
     cusp_beta may hold the fitted records of qmcb_fit_cusps
     ([M][rows of mo_alpha / mo_beta][QMCB_CUSP_REC]); NULL = fit in
     qmcb_create. */
  int replace_cusps;
  const double *cusp_alpha;
  const double *cusp_beta;
  /* Three-body electron-electron-nucleus Jastrow (QMCThreeBodyJastrow with
     CambridgeThreeBodyCorrelationFunction, QMcBeaver/src/QMCThreeBodyJastrow.cpp,
     QMcBeaver/src/CambridgeThreeBodyCorrelationFunction.cpp): n_tb functions,
     each U = (L r1 - 1)^C (L r2 - 1)^C sum_lmn c_lmn (L r1)^l (L r2)^m (L r12)^n
     for L r1, L r2 < 1; the coefficients after the input's dependency matrix. */
  int n_tb;
  const int *tb_nen;            /* [n_tb] NeN (powers of r1, r2: 0 .. NeN-1) */
  const int *tb_nee;            /* [n_tb] Nee (powers of r12) */
  const int *tb_C;              /* [n_tb] cutoff exponent C */
  const double *tb_cutoff;      /* [n_tb] L */
  const int *tb_offset;         /* [n_tb] first coefficient in tb_coeff */
  const double *tb_coeff;       /* c_lmn at offset + l*NeN*Nee + m*Nee + n */
  const int *tb_pair;           /* [M][3] function of up-down, up-up, down-down pairs (-1 none) */
} qmcb_system_desc;

/* One fitted cusp-replacement record: rc, sgn0, C, alpha_0 .. alpha_4
   (rc = 0: the orbital keeps its own s part at this nucleus). */
#define QMCB_CUSP_REC 8

/* Sampling / DMC parameters (the QMCFlags fields the path reads). */
typedef struct qmcb_run_params {
  int run_type;              /* QMCB_VMC | QMCB_DMC (run_type) */
  int sampling;              /* sampling_method */
  int qf_modification;       /* QF_modification_type */
  double qf_equal_a;         /* umrigar93_equalelectrons_parameter */
  double dt;                 /* dt */
  double dt_effective;       /* dt_effective (reweighting exponent) */
  int energy_modification;   /* energy_modification_type */
  int reweighting;           /* walker_reweighting_method */
  double energy_trial;       /* E_T */
  double energy_estimated;   /* E_est */
  double branching_threshold;
  double fusion_threshold;
  int old_walker_acceptance; /* old_walker_acceptance_parameter */
  int refresh_interval;      /* steps between full LU refreshes, 0 = never */
  int precision;             /* QMCB_PREC_* */
  uint64_t seed;             /* Philox key for device random numbers */
  double population_control; /* population_control_parameter (E_T feedback) */
  int target_walkers;        /* W0 of updateTrialEnergy; 0 = walkers at init */
  int reweight_start_step;   /* steps below this keep dW = 1 (QMCWalker.cpp:1071) */
  double energy_original;    /* energy_estimated_original (input energy); 0 = energy_estimated */
  double rel_cutoff;         /* observables with |E - E_orig| / |E_orig| >= rel_cutoff are left out */
  int limit_branching;       /* QMCWalker::branchRecommended rules on splits (QMCWalker.cpp) */
  int energy_cutoff;         /* QMCB_ECUT_*: local energy used in the reweighting exponent */
  /* 0 (the reference): the Green's functions of a single-electron
   * importance-sampled move multiply in every unmoved electron's term
   * (QMcBeaver/src/QMCWalker.cpp:383-388, 756-780, 540-583); their drifts
   * differ before and after the move, so the acceptance ratio is not the
   * proposal's and VMC samples a distribution slightly off |psi|^2 (h2o:
   * 10 mHa high).  1: the moved electron's density only -- the exact
   * Metropolis-Hastings ratio of a single-electron proposal.  No counterpart
   * in the reference; all-electron moves are unaffected by the choice. */
  int exact_single_electron_gf;
  /* 1 (the reference): DMC reweights with the running effective time step
   * dt <w p dR^2> / <w dR^2> over the moves sampled so far
   * (QMCManager::updateEffectiveTimeStep, QMcBeaver/src/QMCManager.cpp:2312-2331,
   * updated here with the trial energy); 0: dt_effective as given. */
  int dynamic_time_step;
  /* 1: after each DMC reweight a walker is deleted (weight 0, removed at the
   * next branching) by the reference's rules (QMCWalker::reweight_walker,
   * QMcBeaver/src/QMCWalker.cpp:1196-1365), with iteration = step -
   * equilibration_steps: while iteration < -100 (equilibrating) when its
   * weight exceeds twice the branching threshold or falls below 0.1, dW is
   * outside [0.5, 1.5] or NaN, |E_L - E_orig| / |E_orig| > rel_cutoff (after
   * step 5) or its age reaches 30; afterwards when dW^(age+1) > 15 or dW is
   * NaN, its weight exceeds 50, or |E_L - E_orig| / |E_orig| > rel_cutoff.
   * E_L is the accepted configuration's.  0: no deletion. */
  int walker_deletion;
  int equilibration_steps;   /* equilibration_steps: steps before iteration 0 */
} qmcb_run_params;

/* Energy cutoffs in the reweighting exponent.  The reference defines them
 * (QMCWalkerData::getModifiedLocalEnergy, QMcBeaver/src/QMCWalkerData.cpp:163-205)
 * but never calls that function, so its energy_cutoff_type changes nothing:
 * QMCB_ECUT_NONE is the reference's behaviour, the other two are an opt-in
 * stabiliser for poor trial functions (they bias the DMC energy). */
#define QMCB_ECUT_NONE 0
#define QMCB_ECUT_UMRIGAR93 1    /* E_L * |modified drift| / |drift| */
#define QMCB_ECUT_BDJM_PUSH88 2  /* E_L clamped to E_orig +- 2 / sqrt(dt) */

/* Ensemble sums over one call of qmcb_run_steps (for E_est / E_T and error bars). */
typedef struct qmcb_step_stats {
  double sum_weight;         /* sum over walker-steps of weight */
  double sum_weight_energy;  /* sum of weight * E_L (observable, p/q weighted) */
  double sum_weight_energy2; /* sum of weight * E_L^2 */
  double sum_accept;         /* sum of acceptance probabilities */
  double n_moves;            /* walker-moves performed */
  double final_weight;       /* total weight after the last step */
  int n_walkers;             /* walkers alive after the last step */
  int n_singular;            /* rejected singular / NaN proposals */
} qmcb_step_stats;

typedef struct qmcb_handle qmcb_handle;

/* Library version string. */
const char *qmcb_version(void);

/* Fits the electron-nucleus cusp replacement of every (nucleus, orbital
   row) of one spin (beta = 0: mo_alpha rows, 1: mo_beta rows) into
   out[n_nuclei][rows][QMCB_CUSP_REC], as QMCElectronNucleusCusp::
   fitReplacementOrbitals does (QMcBeaver/src/QMCElectronNucleusCusp.cpp:
   46-172).  Host only, needs no device.  Errors: qmcb_last_error(NULL). */
int qmcb_fit_cusps(const qmcb_system_desc *desc, int beta, double *out);

/* Message of the last failure on this handle (or of the last failed create
 * or handle-free call when h is NULL). */
const char *qmcb_last_error(const qmcb_handle *h);

/* Builds device tables for the system and allocates state for max_walkers
 * slots on the current CUDA device.  Replaces QMCSCFJastrow::initialize
 * (QMcBeaver/src/QMCSCFJastrow.cpp:61-89) + QMCWalkerData::initialize
 * (QMcBeaver/src/QMCWalkerData.cpp:56-161). */
int qmcb_create(const qmcb_system_desc *sys, int max_walkers, qmcb_handle **out);
int qmcb_destroy(qmcb_handle *h);
int qmcb_set_params(qmcb_handle *h, const qmcb_run_params *p);
int qmcb_get_params(const qmcb_handle *h, qmcb_run_params *p);
int qmcb_num_electrons(const qmcb_handle *h);
int qmcb_max_walkers(const qmcb_handle *h);

/*
 * QMCFunctions::evaluate(walkerData[], xData[], num) for the walkers in
 * slots[0..num), all with the same which_e (QMcBeaver/src/QMCSCFJastrow.cpp:91-181):
 *   which_e = -1: full evaluation (LU inverse, all Slater rows, all Jastrow
 *                 pairs), as for walker initialisation / all-electron moves;
 *   which_e = e : electron e moved; Sherman-Morrison row update of that
 *                 spin's inverse (QMcBeaver/include/Array2D.h:1567-1610) and
 *                 incremental Jastrow update (QMcBeaver/src/QMCJastrowElectronElectron.cpp:68-147).
 * The state of each slot is updated unconditionally, as the reference does.
 * R: host [num][N][3].  Outputs (host, any may be NULL):
 *   log_abs_psi[num], sign[num]            psi = sign * exp(log_abs_psi)
 *   grad[num][N][3]                        gradPsiRatio
 *   mod_grad[num][N][3]                    modifiedGradPsiRatio
 *   lap[num]                               lap(psi)/psi
 *   e_local[num]                           localEnergy
 *   pe[num][3]                             potentialEnergy, neEnergy, eeEnergy
 *   status[num]                            QMCB_ST_* bits (wd->singular)
 * Outputs in mapped page-locked memory are stored by the kernel directly;
 * pageable ones come back by one copy each.  Returns when they are in place.
 */
int qmcb_evaluate(qmcb_handle *h, int which_e, const int *slots, int num, const double *R,
                  double *log_abs_psi, double *sign, double *grad, double *mod_grad, double *lap,
                  double *e_local, double *pe, unsigned char *status);

/*
 * Single-electron form of qmcb_evaluate for drivers that keep the positions
 * on the host (QMCWalker moves one electron, QMcBeaver/src/QMCWalker.cpp:
 * 313-398, then QMCRun::propagateWalkers calls QMCFunctions::evaluate,
 * QMcBeaver/src/QMCRun.cpp:43-55): the other electrons' positions are already
 * in the walker state, so only r_moved[num][3], the new position of
 * electron which_e, crosses the bus, and only the outputs selected in
 * out_mask (QMCB_OUT_*) come back (their pointers must be non-NULL; the
 * others may be NULL).  Same numbers as qmcb_evaluate.  Host buffers may be
 * pageable (outputs then come back by one copy each after the kernel);
 * outputs in page-locked memory mapped into the device's address space
 * (cudaMallocHost / cudaHostAlloc, or cudaHostRegister with
 * cudaHostRegisterMapped) are stored by the kernel directly, so their
 * transfer overlaps the evaluation.  Returns when every output is in place.
 */
#define QMCB_OUT_PSI 1        /* log_abs_psi[num], sign[num] */
#define QMCB_OUT_GRAD 2       /* grad[num][N][3] */
#define QMCB_OUT_MOD_GRAD 4   /* mod_grad[num][N][3] */
#define QMCB_OUT_LAP 8        /* lap[num] */
#define QMCB_OUT_E_LOCAL 16   /* e_local[num] */
#define QMCB_OUT_PE 32        /* pe[num][3] */
#define QMCB_OUT_STATUS 64    /* status[num] */
#define QMCB_OUT_ALL 127
int qmcb_evaluate_moved(qmcb_handle *h, int which_e, const int *slots, int num, const double *r_moved,
                        unsigned out_mask, double *log_abs_psi, double *sign, double *grad, double *mod_grad,
                        double *lap, double *e_local, double *pe, unsigned char *status);

/* Walker slots for drivers that own their walkers one by one through the
 * evaluate entry points (the reference keeps a std::list<QMCWalker>, adds
 * copies and erases walkers in QMCRun::nonunitWeightBranching,
 * QMcBeaver/src/QMCRun.cpp:740-814): qmcb_alloc_slot hands out a free slot,
 * qmcb_free_slot returns one (QMCB_E_ARG if it was not handed out).  The
 * walker list of qmcb_init_walkers / qmcb_run_steps is separate and is not
 * touched.  Thread safe. */
int qmcb_alloc_slot(qmcb_handle *h, int *slot);
int qmcb_free_slot(qmcb_handle *h, int slot);

/* Same as qmcb_evaluate with every pointer in device memory and no
 * host synchronisation; stream NULL = the handle's stream. */
int qmcb_evaluate_device(qmcb_handle *h, int which_e, const int *d_slots, int num, const double *d_R,
                         double *d_log_abs_psi, double *d_sign, double *d_grad, double *d_mod_grad,
                         double *d_lap, double *d_e_local, double *d_pe, unsigned char *d_status,
                         void *stream);

/* Uploads positions of walkers [0, n) from host R[n][N][3] into slots 0..n-1
 * and runs the full evaluation on them (QMCWalker::initializeWalkerPosition,
 * QMcBeaver/src/QMCWalker.cpp:2006-2034). Sets weight 1, age 0. */
int qmcb_init_walkers(qmcb_handle *h, int n, const double *R);

/*
 * n_steps single-electron Metropolis steps (VMC) or DMC steps on the live
 * walkers (QMCRun::step, QMcBeaver/src/QMCRun.cpp:1179-1236): step s moves
 * electron (first_step + s) % N of every walker (QMcBeaver/src/QMCWalker.cpp:186-190),
 * accepts or rejects, reweights when that electron is 0 (DMC), and branches
 * after such steps (nonunit weight branching, QMcBeaver/src/QMCRun.cpp:740-814).
 * Full LU refresh every refresh_interval steps.  Stats are accumulated.
 */
int qmcb_run_steps(qmcb_handle *h, int first_step, int n_steps, qmcb_step_stats *stats);

/*
 * One step, as qmcb_run_steps(h, step, 1, stats), that also returns the
 * configuration records the reference writes with print_configs 1
 * (QMCWalker::processPropagation -> QMCWalkerData::writeConfigs,
 * QMcBeaver/src/QMCWalker.cpp:238-250, QMcBeaver/src/QMCWalkerData.cpp:216-224;
 * the binary record of QMCConfigIO::writeCorrelatedSamplingConfiguration,
 * QMcBeaver/src/QMCConfigIO.cpp:271-384, less its leading int electron count):
 * for every walker live before the step, in list order, the trial walker
 * with weight p (the acceptance probability) and then the original walker
 * with weight 1 - p.  Each record is QMCB_CONFIG_RECORD(N) doubles:
 * R[N][3], lap(D)/D, grad(D)/D [N][3], ln J, potential energy, weight.
 * records holds capacity walkers (2 * capacity records); *n_records is set.
 */
#define QMCB_CONFIG_RECORD(N) (6 * (N) + 4)
int qmcb_run_step_configs(qmcb_handle *h, int step, double *records, int capacity, int *n_records,
                          qmcb_step_stats *stats);

/* Asynchronous form for drivers that keep several handles busy at once
 * (one stream per handle; kernels of different handles overlap on the GPU)
 * or that prepare a batch while the previous one runs:
 * qmcb_run_steps_async enqueues the steps and returns; qmcb_steps_done
 * returns 1 when the oldest batch in flight finished (0 while running,
 * negative on error); qmcb_steps_collect waits for it and returns its
 * statistics.  At most two batches in flight per handle, collected in the
 * order they were enqueued; qmcb_run_steps needs none in flight. */
int qmcb_run_steps_async(qmcb_handle *h, int first_step, int n_steps);
int qmcb_steps_done(qmcb_handle *h);
int qmcb_steps_collect(qmcb_handle *h, qmcb_step_stats *stats);

/*
 * Groups: many handles (systems of different sizes, each with its own
 * walkers) stepped together.  No counterpart in the reference, which runs
 * one molecule per process; it serves many small jobs on one GPU.  Each step
 * is one persistent kernel per bucket of members with similar per-walker
 * shared-memory needs, in which every warp takes the next walker of any
 * member, then (DMC members) one branching launch for all members.  The
 * first calls of qmcb_group_run_steps time the candidate launch
 * configurations (bucketing, warps per block) on the real steps and keep the
 * fastest; results do not depend on the configuration.  Batches without
 * refresh are captured as one CUDA graph and replayed while the batch length
 * and configuration stay the same.
 * Members: FP64 handles (one or several determinants) on one device, each initialised
 * (qmcb_init_walkers), none in flight; the caller does not use a member's
 * handle for steps while the group steps it.  At most 512 members.
 * qmcb_group_run_steps advances member i by n_steps steps from
 * first_steps[i] (the same steps as qmcb_run_steps(member, first_steps[i],
 * n_steps)); stats[i] receives member i's statistics (stats may be NULL).
 */
typedef struct qmcb_group qmcb_group;
int qmcb_group_create(qmcb_handle *const *members, int n, qmcb_group **out);
int qmcb_group_destroy(qmcb_group *g);
const char *qmcb_group_last_error(const qmcb_group *g);
int qmcb_group_run_steps(qmcb_group *g, const int *first_steps, int n_steps, qmcb_step_stats *stats);
/* Candidate configurations, the tuned one (-1 while tuning), the one the
 * last batch ran, and that one's bucket count and warps per block. */
int qmcb_group_config(const qmcb_group *g, int *n_configs, int *chosen, int *last, int *n_buckets, int *wpb);
/* Fix the configuration (0 .. n_configs - 1), or -1 to time them again. */
int qmcb_group_set_config(qmcb_group *g, int config);

/* Layout choice at qmcb_create: spins of more than 16 electrons keep their
 * inverse in device memory (two copies per walker and spin) instead of
 * staging it in the move kernel's shared memory; the environment variable
 * QMCB_STAGED_INVERSE_MAX, read by qmcb_create, moves that threshold.  Both
 * layouts compute the same numbers. */

/* Device bytes of the walker state of a handle (admission control), plus the
 * operand and row buffers of the tensor-core rows modes once one of them
 * has been set up on the handle. */
size_t qmcb_state_bytes(const qmcb_handle *h);

/* Live walker count and per-walker read back (host buffers, any may be NULL). */
int qmcb_num_walkers(const qmcb_handle *h);
int qmcb_get_walkers(qmcb_handle *h, int n, double *R, double *weight, double *e_local,
                     double *log_abs_psi, double *sign);

/* Copies the full device state of walker slot src into dst (branching,
 * QMcBeaver/src/QMCRun.cpp:758). */
int qmcb_copy_slot(qmcb_handle *h, int src, int dst);

/* Overwrites the weights of the first n live walkers (host w[n]); for
 * drivers that manage the population themselves (QMCWalker::setWeight). */
int qmcb_set_walker_weights(qmcb_handle *h, int n, const double *w);

/* One nonunit-weight branching pass over the live walkers
 * (QMCRun::branchWalkers / nonunitWeightBranching,
 * QMcBeaver/src/QMCRun.cpp:89-127,740-814); `step` selects the random
 * stream of the fusion draws, the draw of a fused pair is keyed by the live-list
 * position of its first member, and a split is decided on the weight before
 * fusion (a fused survivor does not split in the same pass, as in the
 * reference's single loop).  Returns the new live count in *n_live. */
int qmcb_branch(qmcb_handle *h, int step, int *n_live);

/* Kernel timing: when enabled, qmcb_run_steps records CUDA events around
 * every launch on the handle's stream and accumulates per-kernel totals.
 * out[2*k] = total ms, out[2*k+1] = launches for k = QMCB_KERNEL_*. */
#define QMCB_KERNEL_MOVE 0
#define QMCB_KERNEL_BRANCH 1
#define QMCB_KERNEL_COPY 2
#define QMCB_KERNEL_ENERGY 3
#define QMCB_KERNEL_REFRESH 4
#define QMCB_KERNEL_ROWS_PREP 5 /* tensor-core rows modes: proposal, basis values and their operand planes */
#define QMCB_KERNEL_ROWS_MMA 6  /* tensor-core rows modes: the tensor-core contraction */
#define QMCB_KERNEL_COUNT 7
int qmcb_set_profiling(qmcb_handle *h, int enable);
int qmcb_get_kernel_stats(qmcb_handle *h, double *out, int reset);

/* Blocks until the handle's stream is idle. */
int qmcb_synchronize(qmcb_handle *h);

/* The CUDA stream of the handle (cudaStream_t as void*). */
void *qmcb_stream(qmcb_handle *h);

/* Diagnostic, no counterpart in the reference: the orbital rows the last
 * single-electron move of a tensor-core rows mode (QMCB_PREC_INT8_SLICES,
 * QMCB_PREC_BF16_TC, QMCB_PREC_BF16X3_TC) used, rows[num][5][*n] in the
 * order of that move's walker list (value, d/dx, d/dy, d/dz, Laplacian rows
 * of the moved electron at its proposed position times the spin's MO
 * coefficients; *n = orbitals of the moved spin).  QMCB_E_STATE before any
 * such move. */
int qmcb_get_rows(qmcb_handle *h, int num, int *n, double *rows);

/*
 * Allocation-free branching pass (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory at call time: drivers that
 * hand every byte of HBM to their own memory pool up front (a serving process
 * with a pre-reserved arena), or that must not trigger the device-wide
 * synchronisation cudaMalloc / cudaFree imply in the middle of an
 * asynchronous step sequence.  It needs no handle and calls no allocator: its
 * scratch is a static device array inside the library.
 *
 * Same decisions as qmcb_branch on a plain list of n walker weights (split
 * above branching_threshold, die below 0.01, fuse pairs below
 * fusion_threshold in list order, the draw of a pair keyed by (seed, list
 * position of its first member, step), the split test on the weight before
 * fusion), without the branch-recommendation rules.  qmcb_branch keys its
 * draws by live-list position as well, so the two agree for any list order.
 * Outputs: d_weight_out / d_parent_out (room for 2n entries each) receive the
 * new list -- survivors in order, split copies appended -- with each entry's
 * source index; *d_n_out the new count.  All pointers are device memory;
 * launched on `stream` (NULL = legacy default stream), not synchronised.
 * Limits: n <= QMCB_NOALLOC_MAX_WALKERS, else QMCB_E_LIMIT.  Every call shares
 * the one static scratch array, so calls that overlap on the GPU race; keep
 * them on one stream.  The first call on a device looks up the array's
 * device address; make that call before any stream capture.
 */
#define QMCB_NOALLOC_MAX_WALKERS 65536
int qmcb_branch_weights_noalloc(const double *d_weight_in, int n, double branching_threshold,
                                double fusion_threshold, uint64_t seed, int step, double *d_weight_out,
                                int *d_parent_out, int *d_n_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* QMCB200_H */
