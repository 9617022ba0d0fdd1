// device_common.cuh -- device-side building blocks of the walker path.
//
// Layout conventions (HBM):
//   * per-walker state is one contiguous block of `stride` doubles per slot
//     (walker-major), so one warp reads a walker's arrays with unit stride;
//   * Slater values Dv[e][o] are stored electron-major (rows = electrons, as
//     the reference's Slater matrix), the derivative matrices transposed,
//     DgT[d][o][e] and DlT[o][e], so the per-move ratio sums read them with
//     consecutive lanes on consecutive electrons;
//   * inverse Inv[o][e] = (D^-1)(o,e), the reference's Dc_inv layout
//     (QMcBeaver/src/QMCWalkerData.cpp:69-76).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define QMCB_FULL_MASK 0xffffffffu

namespace qmcb {

constexpr int kPadeMax = 16;

// Scalars kept per walker (offsets inside the SC block of a walker).
enum Sc {
  SC_U = 0,        // ln Jastrow
  SC_UXX,          // lap ln J
  SC_LAPR_A,       // lap(D_a)/D_a  (rDc_xxA)
  SC_LAPR_B,
  SC_LOGDET_A,     // ln |det D_a|
  SC_LOGDET_B,
  SC_SIGN_A,       // sign det D_a
  SC_SIGN_B,
  SC_VEN,          // e-n potential
  SC_VEE,          // e-e potential
  SC_PE,           // total potential (incl. V_nn)
  SC_EL,           // local energy
  SC_LAP,          // lap(psi)/psi
  SC_WEIGHT,       // DMC weight
  SC_AGE,          // steps since the last accepted move
  SC_STATUS,       // QMCB_ST_* bits
  SC_MODRATIO,     // |modified grad| / |grad|
  SC_AGE_MOVED,    // age when the walker last moved
  SC_DW,           // weight factor of the last reweight
  SC_MDCUR_A,      // several determinants: current copy (0/1) of the spin's determinant block
  SC_MDCUR_B,
  SC_INVCUR_A,     // inverse kept in HBM (large spins): current copy (0/1) of the spin's inverse
  SC_INVCUR_B,
  SC_FUSED,        // branching pass: 1 on the survivor of a fused pair until the pass's split test
  SC_COUNT
};
constexpr int kScalars = 24;  // padded

constexpr int kShellPrim = 6;  // primitives kept in registers per shell
constexpr int kFnPrim = 3;      // primitives per function in the fixed-count loop of basis_function_rows
constexpr int kTbMax = 8;      // largest NeN / Nee of a three-body function

struct DevSys {
  int M, na, nb, N, K, npade, nshell;
  int ndet;              // determinants (1: the one-determinant kernels)
  int nact[2];           // active orbital rows per spin (= na, nb for one determinant)
  const int *docc[2];    // [ndet][n] active row of each determinant column
  const int *dswap[2];   // [ndet][n] columns swapped in from determinant c-1 (-1 ends)
  const double *ci;      // [ndet] CI coefficients
  // electron-nucleus cusp replacement (cusp = 0: off)
  int cusp, nsmax;
  const int *cns;        // [M] s-type primitives on each nucleus
  const double *csexp;   // [M][nsmax] their exponents
  const double *cscoef[2];  // [M][nact][nsmax] primitive coefficient x orbital coefficient
  const double *cpar[2];    // [M][nact][8] rc, sgn0, C, alpha_0..alpha_4
  const double *crmax[2];   // [M] largest rc of the spin's orbitals at the nucleus
  // three-body (e-e-n) Jastrow (ntb = 0: none)
  int ntb;
  const int4 *tbi;       // [ntb] NeN, Nee, C, coefficient offset
  const double *tbL;     // [ntb] L (inverse cutoff)
  const double *tbc;     // coefficients
  const int *tbp;        // [M][3] function of up-down, up-up, down-down pairs
  int ee[3];
  double Pnn;
  const double4 *nuc;    // [M] x, y, z, Z
  const int4 *bf;        // [K] atom, a | b<<8 | c<<16, nprim, prim offset
  const double2 *prim;   // [P] exponent, coefficient
  const int4 *shell;     // [nshell] atom, first function, nmem | L<<8 | nprim<<16, exponent offset
  const int2 *fn;        // [K] a | b<<8 | c<<16, coefficient offset
  int nslot;             // exponential slots: one per (shell, primitive), shells in order
  const int2 *xsl;       // [nslot] atom, exponent index of the slot
  const int4 *fq;        // [K] atom, first slot of the function's shell, nprim, L
  const double *pexp;    // [P] exponents
  const double *pcoef;   // [P] coefficients
  const double *ct[2];   // [K][n_s] MO coefficients, transposed
  const float *ctf[2];   // the same in FP32 (mixed-precision path)
  const double *pade;    // [npade][2][kPadeMax] numerator, denominator
  const int2 *pade_len;  // [npade] numerator length, denominator length
  const int *en[2];      // [M] e-n function per spin
  const double2 *pade_ab; // [npade] (a, b) when every function is a r / (1 + b r)
  int pade_simple;
  const int *ctype;       // [npade] QMCB_CORR_*
  const double4 *cparam;  // [npade] Cambridge2: fL, C, active
};

// Offsets (in doubles) of each array in a walker block.
struct Layout {
  int stride;
  int R;         // [N][3]
  int Dv[2];     // [n][a]  electron-major Slater values (a = active orbitals, = n
                 //         for one determinant)
  int DgT[2];    // [3][a][n] orbital-major gradients
  int DlT[2];    // [a][n]    orbital-major laplacians
  int Inv[2];    // [n][n]    Inv[o][e]; several determinants: two copies of
                 // [ndet][n][n] inverses | [ndet][n][3] grad ratios | [ndet][4]
                 // (ln|det|, sign, lap ratio, singular), mdsz doubles each
  int gradD;     // [N][3] grad(D)/D per electron (rDc_x of its spin)
  int Ux;        // [N][3] grad ln J
  int grad;      // [N][3] gradPsiRatio
  int mgrad;     // [N][3] modifiedGradPsiRatio
  int sc;        // [kScalars]
  int mdsz[2];   // several determinants: doubles in one copy of the determinant block
  int invsz[2];  // inverse kept in HBM: offset of its second copy (0: one copy, staged in shared memory)
  // move-kernel scratch (doubles, even counts): region A, rows, factors,
  // staged positions, staged per-electron tail, staged spin block, stride
  int mv_region_a, mv_dn, mv_valc, mv_r, mv_tail, mv_spin[2], mv_stride;
};

struct RunCfg {
  int run_type, sampling, qf_mod, emod, reweighting, old_walker_acceptance, limit_branching, ecut;
  int exact_gf;  // single-electron moves: Green's functions of the moved electron only
  int dyn_dt;    // reweight with the running effective time step (EnergyCtl::dt_eff)
  int deletion;  // the reference's walker deletion rules after a reweight
  int equil_steps;  // step of iteration 0 (deletion rules: equilibrating while step - equil_steps < -100)
  double qf_a, dt, dt_eff;
  double branching_threshold, fusion_threshold;
  double e_orig, rel_cutoff;
  uint64_t seed;
};

// ------------------------------------------------------------------ warp
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(QMCB_FULL_MASK, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(QMCB_FULL_MASK, v, o));
  return v;
}

// ------------------------------------------------------------------ async copy
// 16-byte global -> shared copies that complete in the background
// (cp.async, LDGSTS); the warp waits on its commit groups before reading.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int Pending>
__device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;\n" ::"n"(Pending) : "memory");
}
// `count` doubles (even; both addresses 16-byte aligned), lanes stride by 2.
__device__ __forceinline__ void warp_copy_async(double *dst, const double *src, int count)
{
  for (int c = 2 * lane_id(); c < count; c += 64) cp_async16(dst + c, src + c);
}

// ------------------------------------------------------------------ RNG
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), written from the
// published round function: two 32x32->64 multiplies per round with the
// Weyl key schedule.
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1)
{
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  U4 r;
  r.x = hi1 ^ c.y ^ k0;
  r.y = lo1;
  r.z = hi0 ^ c.w ^ k1;
  r.w = lo0;
  return r;
}

__device__ __forceinline__ U4 philox4x32(U4 c, uint64_t key)
{
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
  for (int i = 0; i < 10; i++) {
    c = philox_round(c, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// uniform double in (0, 1] from 53 random bits
__device__ __forceinline__ double u01(uint32_t a, uint32_t b)
{
  uint64_t v = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return ((double)v + 1.0) * (1.0 / 9007199254740992.0);
}

// Four uniforms for (walker identity, step, purpose).
__device__ __forceinline__ void rng_uniform4(uint64_t seed, uint32_t walker, uint32_t step, uint32_t purpose,
                                             double u[4])
{
  U4 c{walker, step, purpose, 0x51ED2701u};
  U4 r1 = philox4x32(c, seed);
  c.w = 0x51ED2702u;
  U4 r2 = philox4x32(c, seed);
  u[0] = u01(r1.x, r1.y);
  u[1] = u01(r1.z, r1.w);
  u[2] = u01(r2.x, r2.y);
  u[3] = u01(r2.z, r2.w);
}

// ------------------------------------------------------------------ Pade
// u = P(r)/Q(r) with u', u'' in the operation order of
// FixedCuspPadeCorrelationFunction::evaluate (QMcBeaver/src/FixedCuspPadeCorrelationFunction.cpp:89-111)
// and Polynomial::evaluateAll (QMcBeaver/src/Polynomial.cpp:127-148).
__device__ __forceinline__ void poly_all(const double *c, int len, double x, double &f, double &df, double &d2f)
{
  int n = len - 1;
  f = c[n];
  df = 0.0;
  d2f = 0.0;
  for (int i = n - 1; i >= 0; i--) {
    d2f = d2f * x + df;
    df = df * x + f;
    f = f * x + c[i];
  }
  d2f *= 2.0;
}

// Electron-nucleus cusp replacement of one electron's orbital rows
// D[q * ld + k] (q = value, d/dx, d/dy, d/dz, laplacian; k < a orbitals):
// within rc of nucleus i the s-type part of orbital k from that nucleus is
// replaced by C + sgn0 exp(alpha(r)) (QMCElectronNucleusCusp::replaceCusps,
// QMcBeaver/src/QMCElectronNucleusCusp.cpp:574-638, and
// QMCElectronNucleusCuspParameters::replaceOrbitalValues /
// evaluateOriginalOrbital / evaluateReplacementOrbital,
// QMcBeaver/src/QMCElectronNucleusCuspParameters.cpp:107-285).
template <typename T>
__device__ inline void cusp_replace_warp(const DevSys &S, int sp, const double r[3], T *D, int ld, int a)
{
  const int lane = threadIdx.x & 31;
  for (int i = 0; i < S.M; i++) {
    const double4 P = S.nuc[i];
    const double x = r[0] - P.x, y = r[1] - P.y, z = r[2] - P.z;
    const double rr = sqrt(x * x + y * y + z * z);
    if (!(rr < S.crmax[sp][i])) continue;
    const int ns = S.cns[i];
    const double r_sq = rr * rr;
    for (int k = lane; k < a; k += 32) {
      const double *par = S.cpar[sp] + ((size_t)i * a + k) * 8;
      if (!(rr < par[0])) continue;
      const double *co = S.cscoef[sp] + ((size_t)i * a + k) * S.nsmax;
      const double *ex = S.csexp + (size_t)i * S.nsmax;
      double ov = 0.0, ogx = 0.0, ogy = 0.0, ogz = 0.0, ol = 0.0;
      for (int l = 0; l < ns; l++) {
        const double p0 = ex[l], p1 = co[l];
        const double t = p1 * exp(-p0 * r_sq);
        ov += t;
        const double tmp = -2 * p0 * t;
        ogx += x * tmp;
        ogy += y * tmp;
        ogz += z * tmp;
        ol += 2 * p0 * (2 * p0 * r_sq - 3) * t;
      }
      double f, df, d2f;
      poly_all(par + 3, 5, rr, f, df, d2f);
      const double e = par[1] * exp(f);
      const double tg = (e * df) / rr;
      const double rl = e * (d2f + df * (2.0 / rr + df));
      D[k] = (T)((double)D[k] + ((0.0 - ov) + (par[2] + e)));
      D[ld + k] = (T)((double)D[ld + k] + ((0.0 - ogx) + tg * x));
      D[2 * ld + k] = (T)((double)D[2 * ld + k] + ((0.0 - ogy) + tg * y));
      D[3 * ld + k] = (T)((double)D[3 * ld + k] + ((0.0 - ogz) + tg * z));
      D[4 * ld + k] = (T)((double)D[4 * ld + k] + ((0.0 - ol) + rl));
    }
  }
}

__device__ __forceinline__ void pade_eval(const DevSys &S, int f, double r, double &u, double &du, double &d2u)
{
  if (S.pade_simple) {
    // u = a r / (1 + b r): u' = a q^2, u'' = -2 a b q^3 with q = 1 / (1 + b r)
    // (the FixedCuspPade form of the workloads; same values as the general
    // quotient-rule evaluation below up to rounding)
    const double2 ab = __ldg(&S.pade_ab[f]);
    const double q = 1.0 / fma(ab.y, r, 1.0);
    const double aq = ab.x * q;
    u = aq * r;
    du = aq * q;
    d2u = -2.0 * ab.y * du * q;
    return;
  }
  const double *P = S.pade + (size_t)f * 2 * kPadeMax;
  int2 L = S.pade_len[f];
  if (S.ctype[f] == 1) {
    // Cambridge2 (Cambridge2CorrelationFunction::evaluate,
    // QMcBeaver/src/Cambridge2CorrelationFunction.cpp): u = d^C alpha(fL r),
    // d = fL r - 1, zero for d > 0 or an inactive function
    const double4 cp = S.cparam[f];
    u = du = d2u = 0.0;
    const double fL = cp.x;
    const int C = (int)cp.y;
    const double d = fL * r - 1.0;
    if (cp.z == 0.0 || d > 0.0) return;
    double a, ap, app;
    poly_all(P, L.x, fL * r, a, ap, app);
    const double dP_r = fL * ap, dP_rr = fL * fL * app;
    double dpc = 1.0;
    for (int i = 0; i < C; i++) dpc *= d;
    const double dpc_r = C * fL * dpc / d;
    const double dpc_rr = (C - 1.0) * fL * dpc_r / d;
    u = dpc * a;
    du = dpc_r * a + dpc * dP_r;
    d2u = dpc_rr * a + dpc_r * dP_r * 2.0 + dpc * dP_rr;
    return;
  }
  double a, ap, app, b, bp, bpp;
  poly_all(P, L.x, r, a, ap, app);
  poly_all(P + kPadeMax, L.y, r, b, bp, bpp);
  const double ib = 1.0 / b;
  double aDIVb = a * ib, bpDIVb = bp * ib, apDIVb = ap * ib;
  u = aDIVb;
  du = apDIVb - bpDIVb * aDIVb;
  d2u = (app - bpp * aDIVb) * ib - 2.0 * bpDIVb * du;
}

// ------------------------------------------------------------ three-body
// The coefficient sums of one three-body term for fixed sizes (the
// common NeN = Nee = 4), unrolled; the same operations in the same order
// as the general loop in tb_term.
template <int NEN, int NEE>
__device__ __forceinline__ void tb_poly(const double *__restrict__ c, const double *x1, const double *x2,
                                        const double *x12, double &P, double &Pl, double &Pm, double &Pn,
                                        double &Pll, double &Pmm, double &Pnn, double &Pln, double &Pmn)
{
#pragma unroll
  for (int l = 0; l < NEN; l++) {
    const double xl = x1[l], xl1 = l > 0 ? l * x1[l - 1] : 0.0, xl2 = l > 1 ? l * (l - 1.0) * x1[l - 2] : 0.0;
#pragma unroll
    for (int m = 0; m < NEN; m++) {
      const double xm = x2[m], xm1 = m > 0 ? m * x2[m - 1] : 0.0, xm2 = m > 1 ? m * (m - 1.0) * x2[m - 2] : 0.0;
      const double lm = xl * xm, dlm = xl1 * xm, ldm = xl * xm1;
      double s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
      for (int n = 0; n < NEE; n++) {
        const double cc = __ldg(&c[(l * NEN + m) * NEE + n]);
        s0 = fma(cc, x12[n], s0);
        if (n > 0) s1 = fma(cc * n, x12[n - 1], s1);
        if (n > 1) s2 = fma(cc * (n * (n - 1.0)), x12[n - 2], s2);
      }
      P = fma(lm, s0, P);
      Pl = fma(dlm, s0, Pl);
      Pm = fma(ldm, s0, Pm);
      Pn = fma(lm, s1, Pn);
      Pln = fma(dlm, s1, Pln);
      Pmn = fma(ldm, s1, Pmn);
      Pll = fma(xl2 * xm, s0, Pll);
      Pmm = fma(xl * xm2, s0, Pmm);
      Pnn = fma(lm, s2, Pnn);
    }
  }
}

// One Cambridge three-body term (CambridgeThreeBodyCorrelationFunction::
// setElectron / evaluate / getLapPoly, QMcBeaver/src/CambridgeThreeBodyCorrelationFunction.cpp:
// 150-470) of the electron pair (first, second) around one nucleus: d1, d2 the
// electrons' offsets from the nucleus, d12 = first - second.  Returns false
// (and zeros) outside the cutoff.  g1 / g2: gradients on the two electrons,
// lap: the sum of both laplacians.
__device__ inline bool tb_term(const DevSys &S, int f, const double d1[3], const double d2[3], const double d12[3],
                               double &U, double &lap, double g1[3], double g2[3])
{
  const int4 info = S.tbi[f];
  const int Nen = info.x, Nee = info.y, C = info.z;
  double L = S.tbL[f];
  if (fabs(L) < 1e-10) L = 1.0e10;
  const double a1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
  const double a2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
  const double r1 = a1 * L, r2 = a2 * L, e1 = r1 - 1.0, e2 = r2 - 1.0;
  U = lap = 0.0;
  g1[0] = g1[1] = g1[2] = g2[0] = g2[1] = g2[2] = 0.0;
  if (e1 > 0.0 || e2 > 0.0) return false;
  const double a12 = sqrt(d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2]);
  const double r12 = a12 * L;
  double p1 = 1.0, p2 = 1.0;
  for (int i = 0; i < C; i++) {
    p1 *= e1;
    p2 *= e2;
  }
  const double dp1 = p1 * C / e1, ddp1 = (C - 1.0) * dp1 / e1;
  const double dp2 = p2 * C / e2, ddp2 = (C - 1.0) * dp2 / e2;
  double x1[kTbMax], x2[kTbMax], x12[kTbMax];
  x1[0] = x2[0] = x12[0] = 1.0;
  for (int i = 1; i < Nen; i++) {
    x1[i] = x1[i - 1] * r1;
    x2[i] = x2[i - 1] * r2;
  }
  for (int i = 1; i < Nee; i++) x12[i] = x12[i - 1] * r12;
  // polynomial sums: value, d/dr1, d/dr2, d/dr12 and the second derivatives
  double P = 0, Pl = 0, Pm = 0, Pn = 0, Pll = 0, Pmm = 0, Pnn = 0, Pln = 0, Pmn = 0;
  const double *c = S.tbc + info.w;
  if (Nen == 4 && Nee == 4)
    tb_poly<4, 4>(c, x1, x2, x12, P, Pl, Pm, Pn, Pll, Pmm, Pnn, Pln, Pmn);
  else
  for (int l = 0; l < Nen; l++) {
    const double xl = x1[l], xl1 = l > 0 ? l * x1[l - 1] : 0.0, xl2 = l > 1 ? l * (l - 1.0) * x1[l - 2] : 0.0;
    for (int m = 0; m < Nen; m++) {
      const double xm = x2[m], xm1 = m > 0 ? m * x2[m - 1] : 0.0, xm2 = m > 1 ? m * (m - 1.0) * x2[m - 2] : 0.0;
      const double lm = xl * xm, dlm = xl1 * xm, ldm = xl * xm1;
      double s0 = 0, s1 = 0, s2 = 0;  // sum c x12^n, sum c n x12^(n-1), sum c n(n-1) x12^(n-2)
      for (int n = 0; n < Nee; n++) {
        const double cc = __ldg(&c[(l * Nen + m) * Nee + n]);
        s0 = fma(cc, x12[n], s0);
        if (n > 0) s1 = fma(cc * n, x12[n - 1], s1);
        if (n > 1) s2 = fma(cc * (n * (n - 1.0)), x12[n - 2], s2);
      }
      P = fma(lm, s0, P);
      Pl = fma(dlm, s0, Pl);
      Pm = fma(ldm, s0, Pm);
      Pn = fma(lm, s1, Pn);
      Pln = fma(dlm, s1, Pln);
      Pmn = fma(ldm, s1, Pmn);
      Pll = fma(xl2 * xm, s0, Pll);
      Pmm = fma(xl * xm2, s0, Pmm);
      Pnn = fma(lm, s2, Pnn);
    }
  }
  U = p1 * p2 * P;
  const double dU12 = p1 * p2 * Pn;
  const double dU1 = (dp1 * P + p1 * Pl) * p2;
  const double dU2 = (dp2 * P + p2 * Pm) * p1;
  const double i1 = 1.0 / a1, i2 = 1.0 / a2, i12 = 1.0 / a12;
  double dot = 0.0;
  for (int k = 0; k < 3; k++) {
    const double u1 = d1[k] * i1, u2 = d2[k] * i2, u12 = d12[k] * i12;
    g1[k] = L * (dU1 * u1 + dU12 * u12);
    g2[k] = L * (dU2 * u2 - dU12 * u12);
    dot += u12 * (u1 * (2.0 * p2 * (dp1 * Pn + p1 * Pln)) - u2 * (2.0 * p1 * (dp2 * Pn + p2 * Pmn)));
  }
  double lp = 2.0 * (2.0 * dU12 / r12 + dU1 / r1 + dU2 / r2);
  lp += 2.0 * (p1 * p2 * Pnn) + p2 * (ddp1 * P + 2.0 * dp1 * Pl + p1 * Pll) + p1 * (ddp2 * P + 2.0 * dp2 * Pm + p2 * Pmm);
  lap = (lp + dot) * L * L;
  return true;
}

// Three-body function of the pair (i, j) around nucleus A (-1: none).
__device__ __forceinline__ int tb_func(const DevSys &S, int A, int i, int j)
{
  const bool ai = i < S.na, aj = j < S.na;
  return S.tbp[3 * A + (ai != aj ? 0 : (ai ? 1 : 2))];
}

// Three-body changes when electron e moves from ro to rn
// (QMCThreeBodyJastrow::updateOne, QMcBeaver/src/QMCThreeBodyJastrow.cpp:43-178):
// the lanes share out the (partner j, nucleus A) pairs, each adding U, the
// laplacian and the gradient on e to its partial sums and leaving the
// gradient change on j in pg[(j M + A)][3] (shared scratch, 3 N M doubles);
// then U_x[j] takes those changes in nucleus order, as a loop over the
// nuclei of one partner would.
__device__ __noinline__ void tb_move_lane(const DevSys &S, const double *R, double *Ux, int e, const double *ro,
                                          const double *rn, double *acc, double *pg)
{
  const int N = S.N, M = S.M, lane = threadIdx.x & 31;
  for (int q = lane; q < N * M; q += 32) {
    const int j = q / M, A = q - j * M;
    double gj[3] = {0.0, 0.0, 0.0};
    const int f = j == e ? -1 : tb_func(S, A, e, j);
    if (f >= 0) {
      const double *rj = R + 3 * j;
      const bool e_first = e > j;
      const double4 P = S.nuc[A];
      const double dj[3] = {rj[0] - P.x, rj[1] - P.y, rj[2] - P.z};
      double Uo, Lo, go1[3], go2[3], Un, Ln, gn1[3], gn2[3];
      {
        const double de[3] = {ro[0] - P.x, ro[1] - P.y, ro[2] - P.z};
        const double d12[3] = {e_first ? ro[0] - rj[0] : rj[0] - ro[0], e_first ? ro[1] - rj[1] : rj[1] - ro[1],
                               e_first ? ro[2] - rj[2] : rj[2] - ro[2]};
        tb_term(S, f, e_first ? de : dj, e_first ? dj : de, d12, Uo, Lo, go1, go2);
      }
      {
        const double de[3] = {rn[0] - P.x, rn[1] - P.y, rn[2] - P.z};
        const double d12[3] = {e_first ? rn[0] - rj[0] : rj[0] - rn[0], e_first ? rn[1] - rj[1] : rj[1] - rn[1],
                               e_first ? rn[2] - rj[2] : rj[2] - rn[2]};
        tb_term(S, f, e_first ? de : dj, e_first ? dj : de, d12, Un, Ln, gn1, gn2);
      }
      acc[0] += Un - Uo;
      acc[1] += Ln - Lo;
      for (int k = 0; k < 3; k++) {
        acc[2 + k] += e_first ? gn1[k] - go1[k] : gn2[k] - go2[k];
        gj[k] = e_first ? gn2[k] - go2[k] : gn1[k] - go1[k];
      }
    }
    for (int k = 0; k < 3; k++) pg[3 * q + k] = gj[k];
  }
  __syncwarp();
  for (int j = lane; j < N; j += 32) {
    if (j == e) continue;
    for (int A = 0; A < M; A++)
      for (int k = 0; k < 3; k++) Ux[3 * j + k] += pg[3 * (j * M + A) + k];
  }
  __syncwarp();
}

// Three-body U, laplacian and gradients of all electrons from scratch
// (QMCThreeBodyJastrow::updateAll, QMcBeaver/src/QMCThreeBodyJastrow.cpp:320-401):
// lane i sums the gradient on its electron over every partner; U and the
// laplacian count each pair once (on its higher electron).
__device__ __noinline__ void tb_full_lane(const DevSys &S, const double *R, double *ux, double *acc)
{
  const int N = S.N;
  for (int i = threadIdx.x & 31; i < N; i += 32) {
    const double *ri = R + 3 * i;
    double g[3] = {0, 0, 0};
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      const double *rj = R + 3 * j;
      const bool i_first = i > j;
      for (int A = 0; A < S.M; A++) {
        const int f = tb_func(S, A, i, j);
        if (f < 0) continue;
        const double4 P = S.nuc[A];
        const double di[3] = {ri[0] - P.x, ri[1] - P.y, ri[2] - P.z};
        const double dj[3] = {rj[0] - P.x, rj[1] - P.y, rj[2] - P.z};
        const double d12[3] = {i_first ? ri[0] - rj[0] : rj[0] - ri[0], i_first ? ri[1] - rj[1] : rj[1] - ri[1],
                               i_first ? ri[2] - rj[2] : rj[2] - ri[2]};
        double U, Lp, g1[3], g2[3];
        if (!tb_term(S, f, i_first ? di : dj, i_first ? dj : di, d12, U, Lp, g1, g2)) continue;
        for (int k = 0; k < 3; k++) g[k] += i_first ? g1[k] : g2[k];
        if (i_first) {
          acc[0] += U;
          acc[1] += Lp;
        }
      }
    }
    for (int k = 0; k < 3; k++) ux[3 * i + k] += g[k];
  }
}

// e-e correlation function index for electrons i, j
__device__ __forceinline__ int ee_func(const DevSys &S, int i, int j)
{
  bool ai = i < S.na, aj = j < S.na;
  if (ai != aj) return S.ee[0];
  return ai ? S.ee[1] : S.ee[2];
}

// ------------------------------------------------------------------ basis
// L2 eviction policies and FP64 loads / stores that carry one: the HBM-kept
// inverse of a large spin is read twice per move (Sherman-Morrison factors,
// then the update), so its first read asks L2 to keep the lines and the
// second read, the streamed derivative rows and the new inverse's stores ask
// L2 to drop theirs first.
__device__ __forceinline__ uint64_t l2_evict_last_policy()
{
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ double ld_l2hint(const double *p, uint64_t pol)
{
  double v;
  asm("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ void st_l2hint(double *p, double v, uint64_t pol)
{
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}

// Contracted Cartesian Gaussian k with value, gradient and Laplacian, the
// formulas of QMCBasisFunction::evaluateBasisFunctions
// (QMcBeaver/src/QMCBasisFunction.cpp:287-403):
//   f = sum_i c_i x^a y^b z^c exp(-alpha_i r^2)
//   df/dx = f_i (a/x - 2 alpha_i x) ...
//   lap f = f_i (a(a-1)/x^2 + b(b-1)/y^2 + c(c-1)/z^2 - alpha_i (4L+6) + 4 alpha_i^2 r^2)
__device__ __forceinline__ double ipow(double x, int a)
{
  double r = 1.0;
  for (int i = 0; i < a; i++) r *= x;
  return r;
}

// x^a, x^(a-1), x^(a-2) (1 for negative powers) with the products of ipow
// in its order (x, x*x, (x*x)*x, ...), picked by selects for a <= 4 so that
// the lanes of a warp run one instruction stream whatever their functions'
// powers; larger powers take the loop.
__device__ __forceinline__ void ipow3(double x, int a, double &pa, double &pa1, double &pa2)
{
  if (a > 4) {
    pa = ipow(x, a);
    pa1 = ipow(x, a - 1);
    pa2 = ipow(x, a - 2);
    return;
  }
  const double p2 = x * x, p3 = p2 * x, p4 = p3 * x;
  pa = a == 0 ? 1.0 : a == 1 ? x : a == 2 ? p2 : a == 3 ? p3 : p4;
  pa1 = a <= 1 ? 1.0 : a == 2 ? x : a == 3 ? p2 : p3;
  pa2 = a <= 2 ? 1.0 : a == 3 ? x : p2;
}

__device__ __forceinline__ float ipowf(float x, int a)
{
  float r = 1.0f;
  for (int i = 0; i < a; i++) r *= x;
  return r;
}

// Basis functions of all shells at position r (lanes over shells).  A shell
// is a run of functions on one centre sharing their exponents; exp(-a r^2)
// is evaluated once per primitive and shell.  With P = x^a y^b z^c and
// E_m = sum_i c_i a_i^m exp(-a_i r^2) (m = 0, 1, 2) the reference's formulas
// (QMcBeaver/src/QMCBasisFunction.cpp:370-391) become
//   f = E0 P,  df/dx = E0 dP/dx - 2 x P E1,
//   lap f = E0 lap P + P sum_i c_i e_i (4 r^2 a_i^2 - (4L + 6) a_i),
// polynomial derivatives instead of the reference's a/x and a(a-1)/x^2
// factors (same values, no division by a coordinate).
__device__ __forceinline__ void shell_members(const DevSys &S, int4 sh, double x, double y, double z, double r2,
                                              const double *ex, const double *al, double *chi, int ldc)
{
  const int nmem = sh.z & 0xff, L = (sh.z >> 8) & 0xff, np = sh.z >> 16;
  const double Lf = 4.0 * L + 6.0;
  for (int m = 0; m < nmem; m++) {
    const int k = sh.y + m;
    const int2 f = __ldg(&S.fn[k]);
    const int a = f.x & 0xff, b = (f.x >> 8) & 0xff, c = (f.x >> 16) & 0xff;
    const double *co = S.pcoef + f.y;
    // E0 = sum c e, E1 = sum c a e, El = sum c e (4 r^2 a^2 - (4L+6) a): the
    // Laplacian factor is combined per primitive, as the reference does, so
    // its cancellation happens before the sum
    double E0 = 0.0, E1 = 0.0, El = 0.0;
    const double r2x4 = 4.0 * r2;
    if (np <= kShellPrim) {
#pragma unroll
      for (int i = 0; i < kShellPrim; i++) {
        if (i < np) {
          const double e = __ldg(&co[i]) * ex[i];
          E0 += e;
          E1 = fma(e, al[i], E1);
          El = fma(e, al[i] * fma(r2x4, al[i], -Lf), El);
        }
      }
    } else {
      for (int i = 0; i < np; i++) {
        const double ai = __ldg(&S.pexp[sh.w + i]);
        const double e = __ldg(&co[i]) * exp(-ai * r2);
        E0 += e;
        E1 = fma(e, ai, E1);
        El = fma(e, ai * fma(r2x4, ai, -Lf), El);
      }
    }
    const double xa = ipow(x, a), yb = ipow(y, b), zc = ipow(z, c);
    const double P = xa * yb * zc;
    const double Px = a ? a * ipow(x, a - 1) * yb * zc : 0.0;
    const double Py = b ? b * xa * ipow(y, b - 1) * zc : 0.0;
    const double Pz = c ? c * xa * yb * ipow(z, c - 1) : 0.0;
    double Pl = 0.0;
    if (a > 1) Pl += a * (a - 1.0) * ipow(x, a - 2) * yb * zc;
    if (b > 1) Pl += b * (b - 1.0) * xa * ipow(y, b - 2) * zc;
    if (c > 1) Pl += c * (c - 1.0) * xa * yb * ipow(z, c - 2);
    const double PE1 = P * E1;
    chi[0 * ldc + k] = E0 * P;
    chi[1 * ldc + k] = fma(E0, Px, -2.0 * x * PE1);
    chi[2 * ldc + k] = fma(E0, Py, -2.0 * y * PE1);
    chi[3 * ldc + k] = fma(E0, Pz, -2.0 * z * PE1);
    chi[4 * ldc + k] = fma(E0, Pl, P * El);
  }
}

__device__ __forceinline__ void basis_shells_warp(const DevSys &S, const double r[3], double *chi, int ldc)
{
  for (int si = lane_id(); si < S.nshell; si += 32) {
    const int4 sh = __ldg(&S.shell[si]);
    const double4 A = S.nuc[sh.x];
    const double x = r[0] - A.x, y = r[1] - A.y, z = r[2] - A.z;
    const double r2 = x * x + y * y + z * z;
    const int np = sh.z >> 16;
    double ex[kShellPrim], al[kShellPrim];
#pragma unroll
    for (int i = 0; i < kShellPrim; i++) {
      al[i] = 0.0;
      ex[i] = 0.0;
      if (i < np && np <= kShellPrim) {
        al[i] = __ldg(&S.pexp[sh.w + i]);
        ex[i] = exp(-al[i] * r2);
      }
    }
    shell_members(S, sh, x, y, z, r2, ex, al, chi, ldc);
  }
}

// The same basis values in two balanced passes for the single-electron
// move: lanes over the (shell, primitive) slots evaluate exp(-a r^2) into
// ex[nslot] (shared), then lanes over the functions combine their shell's
// exponentials with their own coefficients (E0, E1, El as in shell_members).
// Both passes spread the work evenly over the lanes, where one lane per
// shell leaves the lanes of s shells idle while d shells run six members.
// The exponential slots exp(-a |r - A|^2) of every (nucleus, primitive
// exponent) pair at r, lanes over slots.
__device__ __forceinline__ void basis_slot_exps_warp(const DevSys &S, const double r[3], double *ex)
{
  for (int q = lane_id(); q < S.nslot; q += 32) {
    const int2 t = __ldg(&S.xsl[q]);
    const double4 A = S.nuc[t.x];
    const double x = r[0] - A.x, y = r[1] - A.y, z = r[2] - A.z;
    ex[q] = exp(-__ldg(&S.pexp[t.y]) * (x * x + y * y + z * z));
  }
}

// Basis function k at r from the slot exponentials: value, gradient,
// Laplacian into v[0..4].
__device__ __forceinline__ void basis_function_rows(const DevSys &S, const double r[3], int k, const double *ex,
                                                    double v[5])
{
  const int4 fq = __ldg(&S.fq[k]);
  const int2 f = __ldg(&S.fn[k]);
  const double4 A = S.nuc[fq.x];
  const double x = r[0] - A.x, y = r[1] - A.y, z = r[2] - A.z;
  const double r2 = x * x + y * y + z * z;
  const int a = f.x & 0xff, b = (f.x >> 8) & 0xff, c = (f.x >> 16) & 0xff;
  const double Lf = 4.0 * fq.w + 6.0, r2x4 = 4.0 * r2;
  double E0 = 0.0, E1 = 0.0, El = 0.0;
  if (fq.z <= kFnPrim) {
    // fixed trip count (predicated): no data-dependent loop branch, the
    // loads of all primitives in flight together
#pragma unroll
    for (int i = 0; i < kFnPrim; i++) {
      if (i < fq.z) {
        const double al = __ldg(&S.pexp[f.y + i]);
        const double e = __ldg(&S.pcoef[f.y + i]) * ex[fq.y + i];
        E0 += e;
        E1 = fma(e, al, E1);
        El = fma(e, al * fma(r2x4, al, -Lf), El);
      }
    }
  } else {
    for (int i = 0; i < fq.z; i++) {
      const double al = __ldg(&S.pexp[f.y + i]);
      const double e = __ldg(&S.pcoef[f.y + i]) * ex[fq.y + i];
      E0 += e;
      E1 = fma(e, al, E1);
      El = fma(e, al * fma(r2x4, al, -Lf), El);
    }
  }
  double xa, xa1, xa2, yb, yb1, yb2, zc, zc1, zc2;
  ipow3(x, a, xa, xa1, xa2);
  ipow3(y, b, yb, yb1, yb2);
  ipow3(z, c, zc, zc1, zc2);
  const double P = xa * yb * zc;
  const double Px = a ? a * xa1 * yb * zc : 0.0;
  const double Py = b ? b * xa * yb1 * zc : 0.0;
  const double Pz = c ? c * xa * yb * zc1 : 0.0;
  double Pl = 0.0;
  if (a > 1) Pl += a * (a - 1.0) * xa2 * yb * zc;
  if (b > 1) Pl += b * (b - 1.0) * xa * yb2 * zc;
  if (c > 1) Pl += c * (c - 1.0) * xa * yb * zc2;
  const double PE1 = P * E1;
  v[0] = E0 * P;
  v[1] = fma(E0, Px, -2.0 * x * PE1);
  v[2] = fma(E0, Py, -2.0 * y * PE1);
  v[3] = fma(E0, Pz, -2.0 * z * PE1);
  v[4] = fma(E0, Pl, P * El);
}

__device__ __forceinline__ void basis_slots_warp(const DevSys &S, const double r[3], double *chi, int ldc,
                                                 double *ex)
{
  basis_slot_exps_warp(S, r, ex);
  __syncwarp();
  for (int k = lane_id(); k < S.K; k += 32) {
    double v[5];
    basis_function_rows(S, r, k, ex, v);
#pragma unroll
    for (int d = 0; d < 5; d++) chi[d * ldc + k] = v[d];
  }
}

// FP32 form of basis_slots_warp for the mixed-precision move: the slots'
// exp(-a r^2) formed as in basis_shells_warp_f (argument in FP64, split
// into a power of two and a fraction), the functions' sums in FP32.
__device__ __forceinline__ void basis_slots_warp_f(const DevSys &S, const double r[3], float *chi, int ldc,
                                                   float *ex)
{
  const int lane = lane_id();
  for (int q = lane; q < S.nslot; q += 32) {
    const int2 t = __ldg(&S.xsl[q]);
    const double4 A = S.nuc[t.x];
    const double x = r[0] - A.x, y = r[1] - A.y, z = r[2] - A.z;
    const double a = -__ldg(&S.pexp[t.y]) * (x * x + y * y + z * z) * 1.4426950408889634;  // log2(e)
    const double fl = floor(a);
    ex[q] = fl < -150.0 ? 0.0f : ldexpf(exp2f((float)(a - fl)), (int)fl);
  }
  __syncwarp();
  for (int k = lane; k < S.K; k += 32) {
    const int4 fq = __ldg(&S.fq[k]);
    const int2 f = __ldg(&S.fn[k]);
    const double4 A = S.nuc[fq.x];
    const float x = (float)(r[0] - A.x), y = (float)(r[1] - A.y), z = (float)(r[2] - A.z);
    const float r2 = x * x + y * y + z * z;
    const int a = f.x & 0xff, b = (f.x >> 8) & 0xff, c = (f.x >> 16) & 0xff;
    const float Lf = 4.0f * fq.w + 6.0f, r2x4 = 4.0f * r2;
    float E0 = 0.0f, E1 = 0.0f, El = 0.0f;
    for (int i = 0; i < fq.z; i++) {
      const float al = (float)__ldg(&S.pexp[f.y + i]);
      const float e = (float)__ldg(&S.pcoef[f.y + i]) * ex[fq.y + i];
      E0 += e;
      E1 = fmaf(e, al, E1);
      El = fmaf(e, al * fmaf(r2x4, al, -Lf), El);
    }
    const float xa = ipowf(x, a), yb = ipowf(y, b), zc = ipowf(z, c);
    const float P = xa * yb * zc;
    const float Px = a ? a * ipowf(x, a - 1) * yb * zc : 0.0f;
    const float Py = b ? b * xa * ipowf(y, b - 1) * zc : 0.0f;
    const float Pz = c ? c * xa * yb * ipowf(z, c - 1) : 0.0f;
    float Pl = 0.0f;
    if (a > 1) Pl += a * (a - 1.0f) * ipowf(x, a - 2) * yb * zc;
    if (b > 1) Pl += b * (b - 1.0f) * xa * ipowf(y, b - 2) * zc;
    if (c > 1) Pl += c * (c - 1.0f) * xa * yb * ipowf(z, c - 2);
    const float PE1 = P * E1;
    chi[0 * ldc + k] = E0 * P;
    chi[1 * ldc + k] = fmaf(E0, Px, -2.0f * x * PE1);
    chi[2 * ldc + k] = fmaf(E0, Py, -2.0f * y * PE1);
    chi[3 * ldc + k] = fmaf(E0, Pz, -2.0f * z * PE1);
    chi[4 * ldc + k] = fmaf(E0, Pl, P * El);
  }
}

// FP64 tensor-core tile D(8x8) += A(8x4) B(4x8), mma.sync m8n8k4 (row.col).
// Fragments: a = A[lane/4][lane%4], b = B[lane%4][lane/4],
// d0,d1 = D[lane/4][2(lane%4)], D[lane/4][2(lane%4)+1].
__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// D[q][o] = sum_k chi[q][k] Ct[k][o] on the FP64 tensor pipe: rows q = the
// five basis quantities (padded to 8), columns = orbitals in tiles of 8,
// k in steps of 4; two column tiles in flight for latency hiding.
__device__ __forceinline__ void contract_dmma_warp(const double *chi, int ldc, const double *__restrict__ Ct, int n,
                                                   int K, double *D)
{
  const int lane = lane_id(), r = lane >> 2, c4 = lane & 3;
  const int ntiles = (n + 7) >> 3;
  constexpr int U = 4;  // k-steps whose operands are loaded before their mma
  for (int t0 = 0; t0 < ntiles; t0 += 2) {
    const bool two = t0 + 1 < ntiles;
    const int o0 = t0 * 8 + r, o1 = o0 + 8;
    const bool in0 = o0 < n, in1 = two && o1 < n;
    double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
    for (int k0 = 0; k0 < K; k0 += 4 * U) {
      double a[U], b0[U], b1[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int k = k0 + 4 * u + c4;
        const bool kin = k < K;
        a[u] = (r < 5 && kin) ? chi[r * ldc + k] : 0.0;
        b0[u] = (kin && in0) ? __ldg(&Ct[k * n + o0]) : 0.0;
        b1[u] = (kin && in1) ? __ldg(&Ct[k * n + o1]) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        dmma_m8n8k4(d00, d01, a[u], b0[u]);
        if (two) dmma_m8n8k4(d10, d11, a[u], b1[u]);
      }
    }
    if (r < 5) {
      const int oc = t0 * 8 + 2 * c4;
      if (oc < n) D[r * n + oc] = d00;
      if (oc + 1 < n) D[r * n + oc + 1] = d01;
      if (two) {
        if (oc + 8 < n) D[r * n + oc + 8] = d10;
        if (oc + 9 < n) D[r * n + oc + 9] = d11;
      }
    }
  }
}

// ------------------------------------------------------------------ FP32
// Single-precision basis for the mixed-precision path: the same shell
// formulas as basis_shells_warp with exp on the special-function unit.
__device__ __forceinline__ void basis_shells_warp_f(const DevSys &S, const double r[3], float *chi, int ldc)
{
  for (int si = lane_id(); si < S.nshell; si += 32) {
    const int4 sh = __ldg(&S.shell[si]);
    const double4 A = S.nuc[sh.x];
    const float x = (float)(r[0] - A.x), y = (float)(r[1] - A.y), z = (float)(r[2] - A.z);
    const float r2 = x * x + y * y + z * z;
    const int nmem = sh.z & 0xff, L = (sh.z >> 8) & 0xff, np = sh.z >> 16;
    const float Lf = 4.0f * L + 6.0f, r2x4 = 4.0f * r2;
    // exp(-a r^2) with the exponent formed in FP64 and split into an
    // integer power of two and a fraction in [0, 1): FP32 rounding of a large
    // argument a r^2 would otherwise cost |a r^2| * 6e-8 relative accuracy
    const double r2d = (r[0] - A.x) * (r[0] - A.x) + (r[1] - A.y) * (r[1] - A.y) + (r[2] - A.z) * (r[2] - A.z);
    float ex[kShellPrim], al[kShellPrim];
#pragma unroll
    for (int i = 0; i < kShellPrim; i++) {
      al[i] = 0.0f;
      ex[i] = 0.0f;
      if (i < np && np <= kShellPrim) {
        const double ad = __ldg(&S.pexp[sh.w + i]);
        al[i] = (float)ad;
        const double t = -ad * r2d * 1.4426950408889634;  // log2(e)
        const double fl = floor(t);
        ex[i] = fl < -150.0 ? 0.0f : ldexpf(exp2f((float)(t - fl)), (int)fl);
      }
    }
    for (int m = 0; m < nmem; m++) {
      const int k = sh.y + m;
      const int2 f = __ldg(&S.fn[k]);
      const int a = f.x & 0xff, b = (f.x >> 8) & 0xff, c = (f.x >> 16) & 0xff;
      const double *co = S.pcoef + f.y;
      float E0 = 0.0f, E1 = 0.0f, El = 0.0f;
      if (np <= kShellPrim) {
#pragma unroll
        for (int i = 0; i < kShellPrim; i++) {
          if (i < np) {
            const float e = (float)__ldg(&co[i]) * ex[i];
            E0 += e;
            E1 = fmaf(e, al[i], E1);
            El = fmaf(e, al[i] * fmaf(r2x4, al[i], -Lf), El);
          }
        }
      } else {
        for (int i = 0; i < np; i++) {
          const float ai = (float)__ldg(&S.pexp[sh.w + i]);
          const float e = (float)__ldg(&co[i]) * __expf(-ai * r2);
          E0 += e;
          E1 = fmaf(e, ai, E1);
          El = fmaf(e, ai * fmaf(r2x4, ai, -Lf), El);
        }
      }
      const float xa = ipowf(x, a), yb = ipowf(y, b), zc = ipowf(z, c);
      const float P = xa * yb * zc;
      const float Px = a ? a * ipowf(x, a - 1) * yb * zc : 0.0f;
      const float Py = b ? b * xa * ipowf(y, b - 1) * zc : 0.0f;
      const float Pz = c ? c * xa * yb * ipowf(z, c - 1) : 0.0f;
      float Pl = 0.0f;
      if (a > 1) Pl += a * (a - 1.0f) * ipowf(x, a - 2) * yb * zc;
      if (b > 1) Pl += b * (b - 1.0f) * xa * ipowf(y, b - 2) * zc;
      if (c > 1) Pl += c * (c - 1.0f) * xa * yb * ipowf(z, c - 2);
      const float PE1 = P * E1;
      chi[0 * ldc + k] = E0 * P;
      chi[1 * ldc + k] = fmaf(E0, Px, -2.0f * x * PE1);
      chi[2 * ldc + k] = fmaf(E0, Py, -2.0f * y * PE1);
      chi[3 * ldc + k] = fmaf(E0, Pz, -2.0f * z * PE1);
      chi[4 * ldc + k] = fmaf(E0, Pl, P * El);
    }
  }
}

// D[q][o] = sum_k chi[q][k] Ct[k][o] in FP32 with lanes split into K-slices
// of n orbitals (n <= 32), five independent accumulators per lane; the
// slices' partial sums meet in `part` (5 * 32 floats).
__device__ __forceinline__ void contract_slices_warp_f(const float *chi, int ldc, const float *__restrict__ Ct, int n,
                                                       int K, float *D, float *part)
{
  // FP32 operands, FP64 accumulation: each product of two FP32 values is
  // exact in FP64, so the sum carries no cancellation loss
  const int lane = lane_id();
  double *dpart = (double *)part;
  if (n <= 32) {
    const int S = 32 / n, s = lane / n, o = lane - s * n;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (s < S) {
      const int k0 = (K * s) / S, k1 = (K * (s + 1)) / S;
      int k = k0;
      for (; k + 4 <= k1; k += 4) {
        float cf[4];
#pragma unroll
        for (int u = 0; u < 4; u++) cf[u] = __ldg(&Ct[(k + u) * n + o]);
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int q = 0; q < 5; q++) acc[q] = fma((double)chi[q * ldc + k + u], (double)cf[u], acc[q]);
      }
      for (; k < k1; k++) {
        const double cf = (double)__ldg(&Ct[k * n + o]);
#pragma unroll
        for (int q = 0; q < 5; q++) acc[q] = fma((double)chi[q * ldc + k], cf, acc[q]);
      }
    }
    __syncwarp();  // part may alias chi
    if (S == 1) {
      if (s < S)
#pragma unroll
        for (int q = 0; q < 5; q++) D[q * n + o] = (float)acc[q];
    } else {
      if (s < S)
#pragma unroll
        for (int q = 0; q < 5; q++) dpart[(s * 5 + q) * n + o] = acc[q];
      __syncwarp();
      if (lane < n) {
#pragma unroll
        for (int q = 0; q < 5; q++) {
          double t = 0.0;
          for (int ss = 0; ss < S; ss++) t += dpart[(ss * 5 + q) * n + lane];
          D[q * n + lane] = (float)t;
        }
      }
    }
  } else {
    for (int o = lane; o < n; o += 32) {
      double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < K; k++) {
        const double cf = (double)__ldg(&Ct[k * n + o]);
#pragma unroll
        for (int q = 0; q < 5; q++) acc[q] = fma((double)chi[q * ldc + k], cf, acc[q]);
      }
#pragma unroll
      for (int q = 0; q < 5; q++) D[q * n + o] = (float)acc[q];
    }
  }
}

}  // namespace qmcb
