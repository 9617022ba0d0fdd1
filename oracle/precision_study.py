"""How much local-energy error the orbital contraction's arithmetic costs
(test infrastructure: a numpy restatement on the CPU, not the product).

For a workload's walkers at their initial positions, the Slater part of the
local energy -1/2 sum_e lap(D)/D is computed from orbital rows (values,
gradients, Laplacians) contracted in FP64 and in reduced-precision forms:
FP64 rows stored as FP32, FP32 operands and accumulation, TF32, BF16,
3xTF32 and 3xBF16 split products with FP32 accumulation, and the int8
digit-plane scheme with exact integer sums (Ozaki et al. 2012; Ootomo,
Ozaki, Yokota 2024) with 3-8 digit planes, scaled per row / orbital over
all of K or per 32-wide block of K (ozakiblk).  The inverse is FP64 in every
case.  Printed per mode: the per-walker error of the Laplacian term and of
the gradient ratios against FP64 (median, p90, max), and the Slater
matrices' condition numbers.

    python oracle/precision_study.py mixed_20nuc_100e 16
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from qmcbeaver_b200.system import make_system  # noqa: E402


def basis_eval(s, r):
    """chi, grad chi (3), lap chi for positions r[P,3] -> arrays [P,K]."""
    atom, pw, nprim, off, ex, co = s.flat_basis()
    K = len(atom)
    P = r.shape[0]
    nuc = np.asarray(s.coords, np.float64)
    chi = np.zeros((P, K)); gx = np.zeros((P, K)); gy = np.zeros((P, K)); gz = np.zeros((P, K)); lap = np.zeros((P, K))
    for k in range(K):
        d = r - nuc[atom[k]]
        x, y, z = d[:, 0], d[:, 1], d[:, 2]
        r2 = x * x + y * y + z * z
        a, b, c = pw[k]
        for p in range(off[k], off[k] + nprim[k]):
            al, cf = ex[p], co[p]
            e = cf * np.exp(-al * r2)
            def f(t, m):
                return t ** m if m > 0 else np.ones_like(t)
            def d1(t, m):
                return (m * f(t, m - 1) if m > 0 else 0.0) - 2 * al * f(t, m + 1)
            def d2(t, m):
                return (m * (m - 1) * f(t, m - 2) if m > 1 else 0.0) - 2 * al * (2 * m + 1) * f(t, m) + 4 * al * al * f(t, m + 2)
            fx, fy, fz = f(x, a), f(y, b), f(z, c)
            chi[:, k] += e * fx * fy * fz
            gx[:, k] += e * d1(x, a) * fy * fz
            gy[:, k] += e * fx * d1(y, b) * fz
            gz[:, k] += e * fx * fy * d1(z, c)
            lap[:, k] += e * (d2(x, a) * fy * fz + fx * d2(y, b) * fz + fx * fy * d2(z, c))
    return [chi, gx, gy, gz, lap]


def round_tf32(x):
    x = np.asarray(x, np.float32)
    i = x.view(np.uint32).astype(np.uint64)
    i = ((i + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return i.view(np.float32)


def round_bf16(x):
    x = np.asarray(x, np.float32)
    i = x.view(np.uint32).astype(np.uint64)
    i = ((i + 0x7FFF + ((i >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return i.view(np.float32)


def contract(rows, C, mode):
    # rows [5][P,K], C [n,K] -> [5][P,n]
    out = []
    for X in rows:
        if mode == "fp64":
            out.append(X @ C.T)
        elif mode == "fp32":
            out.append((X.astype(np.float32) @ C.T.astype(np.float32)).astype(np.float64))
        elif mode == "bf16":
            out.append((round_bf16(X) @ round_bf16(C.T)).astype(np.float64))
        elif mode == "tf32":
            out.append((round_tf32(X) @ round_tf32(C.T)).astype(np.float64))
        elif mode == "3xtf32":
            Xh = round_tf32(X); Xl = round_tf32(X.astype(np.float32) - Xh)
            Ch = round_tf32(C.T); Cl = round_tf32(C.T.astype(np.float32) - Ch)
            acc = (Xh @ Ch) + (Xh @ Cl) + (Xl @ Ch)  # fp32 accumulation
            out.append(acc.astype(np.float64))
        elif mode == "3xbf16":
            X32 = X.astype(np.float32); C32 = C.T.astype(np.float32)
            Xs = [round_bf16(X32)]; Xs.append(round_bf16(X32 - Xs[0])); Xs.append(round_bf16(X32 - Xs[0] - Xs[1]))
            Cs = [round_bf16(C32)]; Cs.append(round_bf16(C32 - Cs[0])); Cs.append(round_bf16(C32 - Cs[0] - Cs[1]))
            acc = np.zeros((X.shape[0], C.shape[0]), np.float32)
            for i in range(3):
                for j in range(3 - i):
                    acc += Xs[i] @ Cs[j]
            out.append(acc.astype(np.float64))
        elif mode.startswith("fp64x32"):
            # fp64 chi, fp64 C, but output rounded to fp32 (storage)
            out.append((X @ C.T).astype(np.float32).astype(np.float64))
        elif mode.startswith("ozakiblk"):
            S = int(mode[8:])
            out.append(ozaki_blocked(X, C.T, S))
        elif mode.startswith("ozaki"):
            S = int(mode[5:])
            out.append(ozaki(X, C.T, S))
    return out


def ozaki(A, B, S):
    """int8 slices with per-row / per-column power-of-two scales, exact int
    products, FP64 combination of the slice pairs with i + j < S."""
    def split(M, axis):
        # power-of-two scale per row (A) / column (B), then digits of 7 bits:
        # d_s = rint(rem 2^(6 + 7 s)), |d_s| <= 64
        amax = np.max(np.abs(M), axis=axis, keepdims=True)
        amax[amax == 0] = 1.0
        sc = 2.0 ** np.ceil(np.log2(amax))
        rem = M / sc
        sl = []
        for s in range(S):
            d = np.rint(rem * 2.0 ** (6 + 7 * s))
            sl.append(d)
            rem = rem - d / 2.0 ** (6 + 7 * s)
        return sl, sc
    As, sa = split(A, 1)
    Bs, sb = split(B, 0)
    acc = np.zeros((A.shape[0], B.shape[1]))
    for i in range(S):
        for j in range(S - i):
            P = (As[i] @ Bs[j])  # exact in float64 for these sizes (|.| < 2^53)
            acc += P / 2.0 ** (12 + 7 * (i + j))
    return acc * sa * sb


def ozaki_blocked(A, B, S, block=32):
    """The same digits with one scale per 32-wide block of K on both sides
    (the layout of the tensor-core kernel): every block's pairs recombined
    and rescaled in FP64, the blocks summed in FP64."""
    K = A.shape[1]
    acc = np.zeros((A.shape[0], B.shape[1]))
    for k0 in range(0, K, block):
        acc += ozaki(A[:, k0:k0 + block], B[k0:k0 + block, :], S)
    return acc


def slater_lap(s, R, mode):
    N = s.n_electrons
    na = s.n_alpha
    out = []
    for sp, (lo, hi, C) in enumerate(((0, na, s.mo_alpha()), (na, N, s.mo_beta()))):
        pts = R[:, lo:hi, :].reshape(-1, 3)
        rows = basis_eval(s, pts)
        Dv, Dx, Dy, Dz, Dl = contract(rows, C, mode)
        W = R.shape[0]
        n = hi - lo
        res = []
        for w in range(W):
            D = Dv[w * n:(w + 1) * n]
            Inv = np.linalg.inv(D)  # Inv[o,e]
            lapR = np.einsum("eo,oe->e", Dl[w * n:(w + 1) * n], Inv)
            g = np.stack([np.einsum("eo,oe->e", X[w * n:(w + 1) * n], Inv) for X in (Dx, Dy, Dz)], 1)
            res.append((lapR.sum(), g, np.linalg.cond(D)))
        out.append(res)
    return out


def main():
    wl = sys.argv[1] if len(sys.argv) > 1 else "mixed_20nuc_100e"
    W = int(sys.argv[2]) if len(sys.argv) > 2 else 24
    s = make_system(wl, seed=1)
    R = s.initial_positions(W, seed=5)
    base = slater_lap(s, R, "fp64")
    for mode in (sys.argv[3].split(",") if len(sys.argv) > 3 else ["fp64x32", "fp32", "3xtf32", "ozaki5", "ozaki6", "ozaki7", "ozaki8",
                                                                   "ozakiblk7", "ozakiblk8"]):
        res = slater_lap(s, R, mode)
        errs, gerr = [], []
        for sp in range(2):
            for w in range(W):
                errs.append(abs(res[sp][w][0] - base[sp][w][0]))
                gerr.append(np.max(np.abs(res[sp][w][1] - base[sp][w][1])))
        el = 0.5 * np.array(errs)  # per spin lap error contribution to E_L
        print(f"{wl} {mode:8s} E_L(lap part) err p50 {np.median(el):.2e} p90 {np.percentile(el, 90):.2e} "
              f"max {el.max():.2e}   grad err p50 {np.median(gerr):.2e} max {np.max(gerr):.2e}")
    conds = [base[sp][w][2] for sp in range(2) for w in range(W)]
    print("cond median %.2e max %.2e" % (np.median(conds), np.max(conds)))
    lapmag = [abs(base[sp][w][0]) for sp in range(2) for w in range(W)]
    print("|lapR| median %.2e max %.2e" % (np.median(lapmag), np.max(lapmag)))


if __name__ == "__main__":
    main()
