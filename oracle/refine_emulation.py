"""Conditioning of 1 - A G and the contraction of mixed-precision refinement,
emulated in numpy on small cases (test infrastructure, not the product).

For each channel with deuteron states and each on-shell energy of a run:
  - kappa_2(1 - A G) from the oracle's A and resolvent on the run's own host
    state space (tictac_b200.Run: grids, V, SWP states);
  - a right-looking blocked LU (32 columns, partial pivoting) in complex64
    whose trailing updates use the tensor-core products of the library:
    "tf32" (operands rounded to 10 mantissa bits, FP32 sums) or "bf16x3"
    (x = hi + lo in bf16, hi*hi + hi*lo + lo*hi, FP32 sums);
  - FP64 iterative refinement of the on-shell columns with that factor,
    reporting the first contraction rho1 = |d2| / |d1| and the number of steps
    until the correction is below 1e-15 of the solution.

    python oracle/refine_emulation.py <golden case> [lec offsets|-] [channels] [N]

e.g. `python oracle/refine_emulation.py lo_j1_J3_n8 0,-0.0004 0,2` (a deeper
deuteron) or `python oracle/refine_emulation.py mt_swave_n16 - 0 24` (N = 24).
"""
import os
import sys

import numpy as np
import scipy.linalg as sl

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "tic-tac_b200", "python"))

import harness as oracle  # noqa: E402


def _round_bits(x, drop):
    """Round float32 values to (23 - drop) mantissa bits, ties away from zero."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + (1 << (drop - 1))) & (0xFFFFFFFF ^ ((1 << drop) - 1))
    return u.astype(np.uint32).view(np.float32)


def tf32(x):
    return _round_bits(x, 13)


def bf16(x):
    return _round_bits(x, 16)


def real_product(X, Y, mode):
    if mode == "tf32":
        return (tf32(X) @ tf32(Y)).astype(np.float32)
    xh, yh = bf16(X), bf16(Y)
    xl, yl = bf16(X - xh), bf16(Y - yh)
    return (xh @ yh + xh @ yl + xl @ yh).astype(np.float32)


def lu_emulated(M, mode, nb=32):
    F = M.astype(np.complex64).copy()
    n = F.shape[0]
    piv = np.arange(n)
    for k0 in range(0, n, nb):
        k1 = min(n, k0 + nb)
        for k in range(k0, k1):
            p = k + int(np.argmax(np.abs(F[k:, k])))
            if p != k:
                F[[k, p]] = F[[p, k]]
                piv[[k, p]] = piv[[p, k]]
            F[k + 1:, k] /= F[k, k]
            F[k + 1:, k + 1:k1] -= np.outer(F[k + 1:, k], F[k, k + 1:k1])
        if k1 < n:
            L11 = np.tril(F[k0:k1, k0:k1], -1) + np.eye(k1 - k0, dtype=np.complex64)
            F[k0:k1, k1:] = np.linalg.solve(L11, F[k0:k1, k1:]).astype(np.complex64)
            L21, U12 = F[k1:, k0:k1], F[k0:k1, k1:]
            re = real_product(L21.real, U12.real, mode) - real_product(L21.imag, U12.imag, mode)
            im = real_product(L21.real, U12.imag, mode) + real_product(L21.imag, U12.real, mode)
            F[k1:, k1:] -= (re + 1j * im).astype(np.complex64)
    return F, piv


def lu_solve(F, piv, b):
    L = np.tril(F, -1).astype(np.complex128) + np.eye(F.shape[0])
    y = sl.solve_triangular(L, b[piv].astype(np.complex128), lower=True, unit_diagonal=True)
    return sl.solve_triangular(np.triu(F).astype(np.complex128), y, lower=False)


def refine(M, b, F, piv, max_steps=20):
    x = lu_solve(F, piv, b)
    changes = []
    for _ in range(max_steps):
        d = lu_solve(F, piv, b - M @ x)
        changes.append(np.max(np.abs(d)) / np.max(np.abs(x)))
        x = x + d
        if changes[-1] < 1e-15:
            break
    rho1 = changes[1] / changes[0] if len(changes) > 1 else 0.0
    return rho1, len(changes)


def main(argv):
    import tictac_b200 as tt
    from conftest import load_case
    case = argv[1] if len(argv) > 1 else "lo_j1_J3_n8"
    g, m = load_case(case)
    opts = dict(m["opts"])
    if len(argv) > 2 and argv[2] != "-":
        opts["lec_offsets"] = argv[2]
    if len(argv) > 4:
        opts["Np_WP"] = opts["Nq_WP"] = int(argv[4])
    run = tt.Run(**opts)
    Np = Nq = int(opts["Np_WP"])
    T, E, q = run.energies()
    Eb = run.E_bound
    chans = [int(x) for x in argv[3].split(",")] if len(argv) > 3 else range(run.num_channels)
    print(f"{case} {opts.get('lec_offsets', '')} N={Np} E_bound={Eb:.4f}")
    for c in chans:
        pw = run.host_array(0, c).reshape(-1, 9)
        deut = oracle.deuterons(pw)
        if not deut:
            continue
        lay = oracle.layout(pw, Np, run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                            run.host_array(7), run.host_array(8), m["tensor_force"], m["iso"])
        r, cc, v = oracle.p123(pw, run.host_array(1), run.host_array(2), m["Nphi"], m["Nx"])
        A = oracle.build_A(lay, pw.shape[0], Nq, Np, r, cc, v)
        n = A.shape[0]
        for j, e in enumerate(E):
            G = oracle.resolvent(lay, pw.shape[0], Nq, Np, run.host_array(2), e + Eb)
            M = np.eye(n) - A * G[None, :]
            b = A[:, [d * Nq * Np + q[j] * Np for d in deut]].astype(np.complex128)
            row = [f"chn {c} n {n} E_com {e:.2f} kappa {np.linalg.cond(M):.2e}"]
            for mode in ("tf32", "bf16x3"):
                rho1, steps = refine(M, b, *lu_emulated(M, mode))
                row.append(f"{mode} rho1 {rho1:.1e} steps {steps}")
            print(" | ".join(row), flush=True)


if __name__ == "__main__":
    main(sys.argv)
