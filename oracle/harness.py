"""Python side of the CPU oracle (test infrastructure only).

Loads oracle/_build/liboracle.so (the plain-C restatement in oracle/*.c) and
restates in numpy the 2N block bookkeeping the reference keeps in its C^T /
V C pointer tables (CPP/solve_faddeev.cpp:1588-1927) and resolvent
(CPP/make_resolvent.cpp:109-156), so that the oracle chain
P123 -> A -> dense LU solve -> U runs independently of the product library.
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this.
"""
import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_int64

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} missing: run `make -C oracle lib`")
        _lib = ctypes.CDLL(LIB)
    return _lib


def _p(a, t):
    return a.ctypes.data_as(POINTER(t))


def p123(pw, p_WP, q_WP, Nphi, Nx):
    """Row-major COO (row, col, val) of P123 for one channel."""
    L = lib()
    pw = np.ascontiguousarray(pw, dtype=np.int32).reshape(-1, 9)
    p = np.ascontiguousarray(p_WP, dtype=np.float64)
    q = np.ascontiguousarray(q_WP, dtype=np.float64)
    nnz = c_int64()
    r = POINTER(ctypes.c_int32)()
    c = POINTER(ctypes.c_int32)()
    v = POINTER(c_double)()
    L.to_p123(len(p) - 1, len(q) - 1, _p(p, c_double), _p(q, c_double), Nphi, Nx, pw.shape[0],
              _p(pw, ctypes.c_int32), ctypes.byref(nnz), ctypes.byref(r), ctypes.byref(c), ctypes.byref(v))
    m = nnz.value
    out = (np.ctypeslib.as_array(r, shape=(max(m, 1),))[:m].copy(),
           np.ctypeslib.as_array(c, shape=(max(m, 1),))[:m].copy(),
           np.ctypeslib.as_array(v, shape=(max(m, 1),))[:m].copy())
    for ptr in (r, c, v):
        L.to_free(ctypes.cast(ptr, ctypes.c_void_p))
    return out


def unique_2N_idx(L, S, J, T, coupled, tensor_force, iso):
    """make_pw_symm_states.cpp:4-60"""
    s1S0 = (S == 0 and J == 0 and L == 0 and T == 1)
    if tensor_force:
        if coupled:
            idx = J - 1
            if not s1S0 and iso:
                idx += 1
            if s1S0 and iso:
                idx = 0
            return idx
        idx = 2 * J + S
        return idx - 1 if iso else idx
    if coupled:
        return 0 if iso else -1
    idx = J * (4 * (J > 1) + 2) + (S == 1) + (S == 1 and J != 0) * (J - L + 1)
    return idx - 1 if iso else idx


def layout(pw, Np, V_unco, V_coup, C_unco, C_coup, e_unco, e_coup, tensor_force=True, iso=True):
    """2N block structure of a channel: per alpha block/part/e-offset, coupling lists, C and VC blocks."""
    pw = np.asarray(pw).reshape(-1, 9)
    Na = pw.shape[0]
    blocks, blk, part, e_off = {}, [], [], []
    Cs, VCs, offs, dims = [], [], [], []
    off = 0
    for a in range(Na):
        L, S, J, T = (int(x) for x in pw[a, :4])
        tT = int(pw[a, 7])
        via_L = tensor_force and L != J and J != 0
        via_T = (S == 0 and J == 0 and L == 0) and iso
        coupled = via_L or via_T
        chn = unique_2N_idx(L, S, J, T, coupled, tensor_force, iso)
        prt = (0 if L < J else 1) if via_L else ((0 if tT == 1 else 1) if via_T else 0)
        key = (coupled, chn)
        if key not in blocks:
            d = 2 * Np if coupled else Np
            src_C = C_coup if coupled else C_unco
            src_V = V_coup if coupled else V_unco
            Cm = np.asarray(src_C[chn * d * d:(chn + 1) * d * d]).reshape(d, d)
            Vm = np.asarray(src_V[chn * d * d:(chn + 1) * d * d]).reshape(d, d)
            blocks[key] = len(dims)
            dims.append(d)
            offs.append(off)
            off += d * d
            Cs.append(Cm.reshape(-1))
            VCs.append((Vm @ Cm).reshape(-1))
        blk.append(blocks[key])
        part.append(prt)
        e_off.append(len(e_unco) + chn * 2 * (Np + 1) + prt * (Np + 1) if coupled else chn * (Np + 1))
    cpl_off, cpl = [0], []
    for r in range(Na):
        for c in range(Na):
            chk_L = (tensor_force and abs(int(pw[r, 0]) - int(pw[c, 0])) <= 2) or pw[r, 0] == pw[c, 0]
            if (pw[r, 3] == pw[c, 3] and pw[r, 2] == pw[c, 2] and pw[r, 1] == pw[c, 1] and chk_L
                    and pw[r, 4] == pw[c, 4] and pw[r, 5] == pw[c, 5]):
                cpl.append(c)
        cpl_off.append(len(cpl))
    i32 = lambda x: np.ascontiguousarray(x, dtype=np.int32)
    return dict(blk=i32(blk), part=i32(part), e_off=i32(e_off), cpl_off=i32(cpl_off), cpl=i32(cpl),
                blk_off=np.ascontiguousarray(offs, dtype=np.int64), blk_dim=i32(dims),
                C=np.ascontiguousarray(np.concatenate(Cs)), VC=np.ascontiguousarray(np.concatenate(VCs)),
                e_swp=np.ascontiguousarray(np.concatenate([e_unco, e_coup]), dtype=np.float64))


def resolvent(lay, Na, Nq, Np, q_WP, E):
    G = np.zeros(Na * Nq * Np, dtype=np.complex128)
    q = np.ascontiguousarray(q_WP, dtype=np.float64)
    lib().to_resolvent(Na, Nq, Np, _p(lay["e_off"], ctypes.c_int32), _p(lay["e_swp"], c_double), _p(q, c_double),
                       c_double(E), G.ctypes.data_as(POINTER(c_double)))
    return G


def build_A(lay, Na, Nq, Np, row, col, val):
    """Dense A from row-major COO P123 (converted to the reference's CSC)."""
    n = Na * Nq * Np
    order = np.lexsort((row, col))
    r = np.ascontiguousarray(row[order], dtype=np.int32)
    v = np.ascontiguousarray(val[order], dtype=np.float64)
    colptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(colptr, np.asarray(col, dtype=np.int64) + 1, 1)
    colptr = np.cumsum(colptr)
    A = np.zeros((n, n))
    lib().to_build_A(Na, Nq, Np, _p(colptr, c_int64), _p(r, ctypes.c_int32), _p(v, c_double),
                     _p(lay["blk"], ctypes.c_int32), _p(lay["part"], ctypes.c_int32), _p(lay["cpl_off"], ctypes.c_int32),
                     _p(lay["cpl"], ctypes.c_int32), _p(lay["blk_off"], c_int64), _p(lay["blk_dim"], ctypes.c_int32),
                     _p(lay["C"], c_double), _p(lay["VC"], c_double), A.ctypes.data_as(POINTER(c_double)))
    return A


def dense_solve(A, G, q_idx, deut, Nq, Np):
    n = A.shape[0]
    G = np.ascontiguousarray(np.asarray(G, dtype=np.complex128).reshape(-1))
    nE = len(q_idx)
    qi = np.ascontiguousarray(q_idx, dtype=np.int32)
    di = np.ascontiguousarray(deut, dtype=np.int32)
    U = np.zeros(nE * len(di) * len(di), dtype=np.complex128)
    st = lib().to_dense_solve(n, np.ascontiguousarray(A).ctypes.data_as(POINTER(c_double)), nE,
                              G.ctypes.data_as(POINTER(c_double)), _p(qi, ctypes.c_int32), len(di),
                              _p(di, ctypes.c_int32), Nq, Np, U.ctypes.data_as(POINTER(c_double)))
    if st:
        raise RuntimeError(f"oracle LU: zero pivot at column {st}")
    return U


def deuterons(pw):
    pw = np.asarray(pw).reshape(-1, 9)
    return [a for a in range(pw.shape[0]) if tuple(int(x) for x in pw[a, :4]) == (0, 1, 1, 0)]


# ---------------------------------------------------------------------------
# Pade-resummed Neumann series of the reference's default production solver
# (pade_method_solve, CPP/solve_faddeev.cpp:440-1444; pade_approximant,
# :271-296; determinant, CPP/General_functions/matrix_routines.cpp:82-101),
# restated in numpy.  Row r = d_row*nE + j of the on-shell rows; a_n for
# element (d_row, d_col, j) = (A (G_j A)^n)[row(d_row, j), col(d_col, j)].

NM_MAX = 14


def pade_approximant(a, N, M, z=1.0):
    """[N/M] Pade approximant at z from the series coefficients a[0..N+M]."""
    P = np.zeros((M + 1, M + 1), dtype=np.complex128)
    Q = np.zeros((M + 1, M + 1), dtype=np.complex128)
    for r in range(M):
        for c in range(M + 1):
            P[r, c] = Q[r, c] = a[N - M + 1 + r + c]
    for c in range(M + 1):
        Q[M, c] = z ** (M - c)
        P[M, c] = sum(a[j - (M - c)] * z ** j for j in range(M - c, N + 1))
    return np.linalg.det(P) / np.linalg.det(Q)


def pade_solve(A, G, q_idx, deut, Nq, Np):
    n = A.shape[0]
    G = np.asarray(G, dtype=np.complex128).reshape(len(q_idx), n)
    nE, nd = len(q_idx), len(deut)
    rows = [deut[d] * Nq * Np + q_idx[j] * Np for d in range(nd) for j in range(nE)]
    R = A[rows, :].astype(np.complex128)  # n = 0 rows
    nel = nd * nd * nE
    a = np.zeros((nel, 2 * NM_MAX + 1), dtype=np.complex128)
    pa = np.zeros((nel, NM_MAX + 1), dtype=np.complex128)
    conv = np.zeros(nel, dtype=bool)
    best = np.zeros(nel, dtype=int)

    def el(dr, dc, j):
        return dr * nd * nE + dc * nE + j

    def extract(nterm):
        for dr in range(nd):
            for dc in range(nd):
                for j in range(nE):
                    e = el(dr, dc, j)
                    if not conv[e]:
                        a[e, nterm] = R[dr * nE + j, deut[dc] * Nq * Np + q_idx[j] * Np]

    extract(0)
    for NM in range(NM_MAX + 1):
        if conv.all():
            break
        for nterm in (2 * NM - 1, 2 * NM):
            if nterm <= 0:
                continue
            for dr in range(nd):
                for j in range(nE):
                    R[dr * nE + j] = (R[dr * nE + j] * G[j]) @ A
            extract(nterm)
        for e in range(nel):
            if conv[e]:
                continue
            pa[e, NM] = pade_approximant(a[e], NM, NM)
            idx_best, min_diff = 0, 1.0
            for prev in range(NM):
                d = abs(pa[e, prev] - pa[e, prev - 1])  # index -1 reads the last slot, as in the reference
                if min_diff > d > 1e-15:
                    idx_best, min_diff = prev, d
            d = abs(pa[e, NM] - pa[e, NM - 1])
            if min_diff > d > 1e-15:
                idx_best, min_diff = NM, d
            if NM == NM_MAX or NM - idx_best > 4 or min_diff < 1e-6 * abs(pa[e, idx_best]) or min_diff < 1e-7:
                conv[e] = True
                best[e] = idx_best
    return np.array([pa[e, best[e]] for e in range(nel)])


# ---------------------------------------------------------------------------
# Breakup amplitudes (include_breakup_channels=true).  The reference locates,
# per on-shell energy, the (alpha, q, p) wave-packet cells whose energy range
# holds E_com, plus three neighbours chosen by the quadrant of the cell that
# E_com falls in (find_on_shell_bins, CPP/run_organizer.cpp:134-339), and
# reads their amplitudes off the same on-shell rows of A (G A)^n as the
# elastic ones, each Pade-resummed with the elastic criteria
# (CPP/solve_faddeev.cpp:867-890, 1176-1205, 1299-1407).

M_P, M_N = 938.272, 939.565


def mu1_free():
    """kinetic_conversion.cpp:16-19"""
    M12 = M_P + M_N
    return M_N * M12 / (M_N + M12)


def breakup_cells(Na, Np, Nq, q_WP, e_swp, e_off, E_com, E_bound):
    """start[nE+1] and cells[num][3] = (alpha, q, p) in the reference's order.
    Neighbour bins may lie outside 0..N-1 at the grid's edge, as there."""
    start, cells = [0], []
    mu = mu1_free()
    for E in E_com:
        if E + E_bound < 0:
            start.append(len(cells))
            continue
        found = False
        for a in range(Na):
            e = e_swp[e_off[a]:e_off[a] + Np + 1]
            for qi in range(Nq):
                Eql = 0.5 * (q_WP[qi] * q_WP[qi]) / mu
                Equ = 0.5 * (q_WP[qi + 1] * q_WP[qi + 1]) / mu
                for pi in range(Np):
                    Epl, Epu = e[pi], e[pi + 1]
                    Ecl, Ecu = Epl + Eql, Epu + Equ
                    if not (Ecl <= E <= Ecu and Epl >= 0 and Epu >= 0):
                        continue
                    found = True
                    cells.append((a, qi, pi))
                    Ep, Eq = 0.5 * (Epu + Epl), 0.5 * (Equ + Eql)
                    if Eq + Ep <= E <= Ecu:
                        pr, qr = (pi, pi + 1), (qi, qi + 1)
                    elif Eq + Epl <= E <= Ep + Equ:
                        pr, qr = (pi - 1, pi), (qi, qi + 1)
                    elif Ecl <= E <= Eq + Ep:
                        pr, qr = (pi - 1, pi), (qi - 1, qi)
                    elif Eql + Ep <= E <= Epu + Eq:
                        pr, qr = (pi, pi + 1), (qi - 1, qi)
                    else:
                        continue
                    for p2 in range(pr[0], pr[1] + 1):
                        for q2 in range(qr[0], qr[1] + 1):
                            if p2 != pi or q2 != qi:
                                cells.append((a, q2, p2))
        if not found:
            raise ValueError(f"on-shell energy {E} outside the WP state space")
        start.append(len(cells))
    return np.array(start, dtype=np.int32), np.array(cells, dtype=np.int32).reshape(-1, 3)


def pade_solve_breakup(A, G, q_idx, deut, Nq, Np, start, cells):
    """pade_solve plus the breakup amplitudes U_BU[d * num + b] of the cells
    (NaN for a cell outside the grid).  Also returns whether the reference's
    loop test (solve_faddeev.cpp:921: stop when elastic + breakup elements
    converged equal the number of elastic elements) would stop it with
    elements still open, where the reference then reads an unset index."""
    n = A.shape[0]
    Na = n // (Nq * Np)
    G = np.asarray(G, dtype=np.complex128).reshape(len(q_idx), n)
    nE, nd, nb = len(q_idx), len(deut), len(cells)
    rows = [deut[d] * Nq * Np + q_idx[j] * Np for d in range(nd) for j in range(nE)]
    R = A[rows, :].astype(np.complex128)
    e_of = np.zeros(nb, dtype=int)
    for j in range(nE):
        e_of[start[j]:start[j + 1]] = j
    inside = [(0 <= c[0] < Na and 0 <= c[1] < Nq and 0 <= c[2] < Np) for c in cells]
    # element list: elastic (d', d, j) first, then breakup (d, b) over in-grid cells
    pick = [(dr * nE + j, deut[dc] * Nq * Np + q_idx[j] * Np) for dr in range(nd) for dc in range(nd)
            for j in range(nE)]
    nel_el = len(pick)
    bu_el = []
    for d in range(nd):
        for b in range(nb):
            if inside[b]:
                a, q, p = (int(x) for x in cells[b])
                bu_el.append(d * nb + b)
                pick.append((d * nE + e_of[b], a * Nq * Np + q * Np + p))
    nel = len(pick)
    a = np.zeros((nel, 2 * NM_MAX + 1), dtype=np.complex128)
    pa = np.zeros((nel, NM_MAX + 1), dtype=np.complex128)
    conv = np.zeros(nel, dtype=bool)
    best = np.zeros(nel, dtype=int)
    early_stop = False

    def extract(nterm):
        for e in range(nel):
            if not conv[e]:
                a[e, nterm] = R[pick[e][0], pick[e][1]]

    extract(0)
    for NM in range(NM_MAX + 1):
        if conv.all():
            break
        if conv.sum() == nel_el and nb:
            early_stop = True
        for nterm in (2 * NM - 1, 2 * NM):
            if nterm <= 0:
                continue
            for dr in range(nd):
                for j in range(nE):
                    R[dr * nE + j] = (R[dr * nE + j] * G[j]) @ A
            extract(nterm)
        for e in range(nel):
            if conv[e]:
                continue
            pa[e, NM] = pade_approximant(a[e], NM, NM)
            idx_best, min_diff = 0, 1.0
            for prev in range(NM):
                d = abs(pa[e, prev] - pa[e, prev - 1])
                if min_diff > d > 1e-15:
                    idx_best, min_diff = prev, d
            d = abs(pa[e, NM] - pa[e, NM - 1])
            if min_diff > d > 1e-15:
                idx_best, min_diff = NM, d
            if NM == NM_MAX or NM - idx_best > 4 or min_diff < 1e-6 * abs(pa[e, idx_best]) or min_diff < 1e-7:
                conv[e] = True
                best[e] = idx_best
    U = np.array([pa[e, best[e]] for e in range(nel_el)])
    U_BU = np.full(nd * nb, np.nan + 1j * np.nan)
    for k, slot in enumerate(bu_el):
        e = nel_el + k
        U_BU[slot] = pa[e, best[e]]
    return U, U_BU, early_stop
