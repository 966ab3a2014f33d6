"""Breakup channels (include_breakup_channels=true): the on-shell cells, their
Pade amplitudes and the breakup table against the reference's own outputs
(tests/golden/<case>_breakup.npz, written by make_golden.py --breakup from the
compiled reference).

The CPU tests pin the oracle (oracle/harness.py) and the library's host side
(cell search, table writer); the GPU tests run the Pade solve with breakup
elements through the C-ABI."""
import os

import numpy as np
import pytest

import harness as oracle
import tictac_b200 as tt
from conftest import GOLDEN, load_case, rel

BREAKUP_CASES = ["mt_swave_n16", "lo_j1_J3_n8"]


def breakup_fixture(case):
    return np.load(os.path.join(GOLDEN, f"{case}_breakup.npz"))


def oracle_cells(g, m, c):
    pw = g[f"pw_c{c}"]
    lay = oracle.layout(pw, m["Np"], g["V_unco"], g["V_coup"], g["C_unco"], g["C_coup"], g["e_unco"], g["e_coup"],
                        m["tensor_force"], m["iso"])
    st, cells = oracle.breakup_cells(pw.shape[0], m["Np"], m["Nq"], g["q_WP"], lay["e_swp"], lay["e_off"], g["E_com"],
                                     float(g["E_bound"]))
    return lay, st, cells


def inside(cells, Na, Nq, Np):
    return (cells[:, 0] >= 0) & (cells[:, 0] < Na) & (cells[:, 1] >= 0) & (cells[:, 1] < Nq) & (cells[:, 2] >= 0) & \
        (cells[:, 2] < Np)


def in_grid_mask(cells, nd, Na, Nq, Np):
    """U_BU[d * num + b] entries whose cell lies inside the grid."""
    return np.tile(inside(cells, Na, Nq, Np), nd)


@pytest.mark.parametrize("case", BREAKUP_CASES)
def test_oracle_breakup_cells_match_reference(case):
    g, m = load_case(case)
    f = breakup_fixture(case)
    for c in map(int, f["channels"]):
        _, st, cells = oracle_cells(g, m, c)
        assert np.array_equal(st, f[f"bu_start_c{c}"])
        assert np.array_equal(cells, f[f"bu_cells_c{c}"])


@pytest.mark.parametrize("case", BREAKUP_CASES)
def test_oracle_breakup_amplitudes_match_reference(case):
    # the Pade amplitudes of the in-grid cells at the method's accuracy (its
    # stopping rule is 1e-6 relative), as for the elastic Pade elements
    g, m = load_case(case)
    f = breakup_fixture(case)
    Np, Nq = m["Np"], m["Nq"]
    for c in map(int, f["channels"]):
        pw = g[f"pw_c{c}"]
        lay, st, cells = oracle_cells(g, m, c)
        A = oracle.build_A(lay, pw.shape[0], Nq, Np, g[f"p123_row_c{c}"], g[f"p123_col_c{c}"], g[f"p123_val_c{c}"])
        deut = oracle.deuterons(pw)
        with np.errstate(invalid="ignore", divide="ignore"):
            U, U_BU, early = oracle.pade_solve_breakup(A, g[f"G_c{c}"], g["q_idx"], deut, Nq, Np, st, cells)
        assert not early
        ok = in_grid_mask(cells, len(deut), pw.shape[0], Nq, Np)
        assert np.all(np.isnan(U_BU[~ok])) and np.all(np.isfinite(U_BU[ok]))
        assert rel(U_BU[ok], f[f"U_BU_c{c}"][ok]) <= 1e-5
        assert rel(U, f[f"U_pade_c{c}"]) <= 1e-5


def test_reference_early_stop_of_excluded_channel():
    # channel 3 of lo_j1_J3_n8 is not in the fixture: the reference's loop test
    # (elastic + breakup converged == elastic count) stops it with elastic
    # elements open; the oracle's restatement of that test says so
    g, m = load_case("lo_j1_J3_n8")
    assert 3 not in breakup_fixture("lo_j1_J3_n8")["channels"]
    pw = g["pw_c3"]
    lay, st, cells = oracle_cells(g, m, 3)
    A = oracle.build_A(lay, pw.shape[0], m["Nq"], m["Np"], g["p123_row_c3"], g["p123_col_c3"], g["p123_val_c3"])
    with np.errstate(invalid="ignore", divide="ignore"):
        _, _, early = oracle.pade_solve_breakup(A, g["G_c3"], g["q_idx"], oracle.deuterons(pw), m["Nq"], m["Np"], st,
                                                cells)
    assert early


@pytest.mark.parametrize("case", BREAKUP_CASES)
def test_run_breakup_cells_match_reference(case):
    # the library's host cell search (tt_run_breakup_cells), bit for bit
    g, m = load_case(case)
    f = breakup_fixture(case)
    run = tt.Run(**m["opts"], include_breakup_channels="true")
    for c in map(int, f["channels"]):
        st, cells = run.breakup_cells(c)
        assert np.array_equal(st, f[f"bu_start_c{c}"])
        assert np.array_equal(cells, f[f"bu_cells_c{c}"])
    run.close()


def test_breakup_cells_below_threshold_and_option_parsing():
    # an energy below the breakup threshold (E_com + E_bound < 0) owns no cells
    g, m = load_case("mt_swave_n16")
    opts = dict(m["opts"], lab_energies="1.5")
    run = tt.Run(**opts)
    T, E, q = run.energies()
    Eb = run.E_bound
    st, cells = run.breakup_cells(0)
    assert len(st) == len(T) + 1 and st[0] == 0
    for j in range(len(T)):
        if E[j] + Eb < 0:
            assert st[j + 1] == st[j]
        else:
            assert st[j + 1] > st[j]
    run.close()
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(**m["opts"], include_breakup_channels="yes")
    assert e.value.code == tt.TT_ERR_BADARG


def table_tokens(text):
    """(header lines, data lines as token lists) of a breakup table."""
    head, rows = [], []
    for line in text.split("\n"):
        if line.startswith("#") or not line.strip():
            head.append(line)
        else:
            rows.append(line.split())
    return head, rows


@pytest.mark.parametrize("case", BREAKUP_CASES)
def test_breakup_table_matches_reference(case, tmp_path):
    # tt_run_write_U_BU_table given the reference's U_BU: the header and every
    # U token identical, the kinematic columns within rounding of the SWP
    # energies (this library's eigensolver and the reference's LAPACK differ in
    # the last bits); nan only in the boundary columns of cells outside the grid
    g, m = load_case(case)
    f = breakup_fixture(case)
    run = tt.Run(**m["opts"], include_breakup_channels="true")
    tables = [int(c) for c in f["channels"] if f"table_c{c}" in f]
    assert tables
    for c in tables:
        path = tmp_path / f"U_BU_c{c}.txt"
        run.write_U_BU_table(c, f[f"U_BU_c{c}"], path)
        ours = path.read_text()
        h1, r1 = table_tokens(ours)
        h2, r2 = table_tokens(str(f[f"table_c{c}"]))
        assert h1 == h2
        assert len(r1) == len(r2)
        worst, nan_tokens = 0.0, 0
        for a, b in zip(r1, r2):
            assert len(a) == len(b)
            for x, y in zip(a, b):
                if "nan" in x:
                    nan_tokens += 1
                elif x.endswith("j"):
                    assert x == y
                else:
                    worst = max(worst, abs(float(x) - float(y)) / max(abs(float(y)), 1e-300))
        assert worst <= 1e-12
        cells = f[f"bu_cells_c{c}"]
        Na = g[f"pw_c{c}"].shape[0]
        assert nan_tokens <= 2 * int(np.sum(~inside(cells, Na, m["Nq"], m["Np"]))) * len(oracle.deuterons(g[f"pw_c{c}"]))
    run.close()


def test_breakup_dropin_rejects_dense_precisions():
    # the reference computes breakup amplitudes on its Pade path only
    g, m = load_case("mt_swave_n16")
    lib = tt.load()
    pwt = g["pw_c0"]
    rp = tt.run_params(precision=tt.PRECISION_MIXED)
    st = np.zeros(len(g["q_idx"]) + 1, dtype=np.int32)
    bu = tt.tt_bu_indexing(0, st.ctypes.data_as(tt.POINTER(tt.c_int)), st.ctypes.data_as(tt.POINTER(tt.c_int)))
    U = np.zeros(4, dtype=np.complex128)
    G = np.ascontiguousarray(g["G_c0"])
    colptr = np.zeros(pwt.shape[0] * m["Np"] * m["Nq"] + 1, dtype=np.uint64)
    qi = np.ascontiguousarray(g["q_idx"], dtype=np.int32)
    di = np.array([1], dtype=np.int32)
    os_ = tt.tt_os_indexing(len(qi), qi.ctypes.data_as(tt.POINTER(tt.c_int)), di.ctypes.data_as(tt.POINTER(tt.c_int)), 1)
    swp = tt.SWP(m["Np"], m["Nq"], len(g["e_unco"]) // (m["Np"] + 1), 0, float(g["E_bound"]), g["e_unco"], g["e_coup"],
                 g["C_unco"], g["C_coup"], g["q_WP"])
    V = np.ascontiguousarray(g["V_unco"])
    pw = tt.PW(pwt)
    rc = lib.tt_solve_faddeev_equations_breakup(
        U.ctypes.data_as(tt.c_void_p), U.ctypes.data_as(tt.c_void_p), tt.byref(bu), G.ctypes.data_as(tt.c_void_p),
        V.ctypes.data_as(tt.c_void_p), st.ctypes.data_as(tt.c_void_p), colptr.ctypes.data_as(tt.c_void_p),
        tt.c_size_t(0), V.ctypes.data_as(tt.c_void_p), V.ctypes.data_as(tt.c_void_p), tt.byref(swp.s), tt.byref(os_),
        tt.byref(pw.s), tt.byref(rp), None)
    assert rc == tt.TT_ERR_UNSUPPORTED


def swp_signs(g, m, c, run):
    """s[alpha, p] = +-1: the sign of the run's SWP eigenvector of state
    (alpha, p) relative to the reference's.  The reference keeps the signs its
    LAPACK eigensolver returns; this library makes each eigenvector's largest
    component positive.  An elastic U element carries the deuteron state's
    sign twice, a breakup element the deuteron's and the cell's."""
    pw = g[f"pw_c{c}"]
    Na, Np = pw.shape[0], m["Np"]
    ref = oracle.layout(pw, Np, g["V_unco"], g["V_coup"], g["C_unco"], g["C_coup"], g["e_unco"], g["e_coup"],
                        m["tensor_force"], m["iso"])
    ours = oracle.layout(pw, Np, run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                         run.host_array(7), run.host_array(8), m["tensor_force"], m["iso"])
    s = np.ones((Na, Np))
    for a in range(Na):
        b = ref["blk"][a]
        d, off = int(ref["blk_dim"][b]), int(ref["blk_off"][b])
        Cr = ref["C"][off:off + d * d].reshape(d, d)
        Co = ours["C"][off:off + d * d].reshape(d, d)
        for p in range(Np):
            col = int(ref["part"][a]) * Np + p
            s[a, p] = 1.0 if Cr[:, col] @ Co[:, col] >= 0 else -1.0
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("case", BREAKUP_CASES)
def test_gpu_breakup_run_matches_reference(case):
    # tt_run_solve_breakup: the Pade solve on the device with the breakup
    # elements, against the reference's amplitudes at the method's accuracy,
    # in the reference's SWP eigenvector signs
    g, m = load_case(case)
    f = breakup_fixture(case)
    run = tt.Run(**m["opts"], include_breakup_channels="true")
    for c in map(int, f["channels"]):
        st, cells = run.breakup_cells(c)
        info = run.channel_info(c)
        U, U_BU, rep = run.solve_breakup(c)
        nd, nb = info["n_deuteron"], len(cells)
        ok = in_grid_mask(cells, nd, info["Nalpha"], m["Nq"], m["Np"])
        assert np.all(np.isnan(U_BU[~ok])) and np.all(np.isfinite(U_BU[ok]))
        s = swp_signs(g, m, c, run)
        deut = oracle.deuterons(g[f"pw_c{c}"])
        sign = np.ones(nd * nb)
        for d in range(nd):
            for b in range(nb):
                if ok[d * nb + b]:
                    sign[d * nb + b] = s[deut[d], 0] * s[cells[b, 0], cells[b, 2]]
        assert rel((sign * U_BU)[ok], f[f"U_BU_c{c}"][ok]) <= 1e-5, (c, rep)
        assert rel(U, f[f"U_pade_c{c}"]) <= 1e-5, (c, rep)
    run.close()


@pytest.mark.gpu
def test_gpu_breakup_dropin_matches_reference():
    # tt_solve_faddeev_equations_breakup with the reference's own P123, G, V,
    # SWP states and breakup indexing
    case = "lo_j1_J3_n8"
    g, m = load_case(case)
    f = breakup_fixture(case)
    Np, Nq = m["Np"], m["Nq"]
    swp = tt.SWP(Np, Nq, len(g["e_unco"]) // (Np + 1), len(g["e_coup"]) // (2 * (Np + 1)), float(g["E_bound"]),
                 g["e_unco"], g["e_coup"], g["C_unco"], g["C_coup"], g["q_WP"])
    for c in map(int, f["channels"]):
        pwt = g[f"pw_c{c}"]
        n = pwt.shape[0] * Np * Nq
        row, col, val = g[f"p123_row_c{c}"], g[f"p123_col_c{c}"], g[f"p123_val_c{c}"]
        order = np.lexsort((row, col))
        colptr = np.zeros(n + 1, dtype=np.uint64)
        np.add.at(colptr, np.asarray(col, dtype=np.int64) + 1, 1)
        cells = f[f"bu_cells_c{c}"]
        deut = oracle.deuterons(pwt)
        U, U_BU, rep = tt.solve_faddeev_breakup(g[f"G_c{c}"], val[order], row[order], np.cumsum(colptr), g["V_unco"],
                                                g["V_coup"], swp, g["q_idx"], deut, tt.PW(pwt), f[f"bu_start_c{c}"],
                                                cells, tensor_force=int(m["tensor_force"]),
                                                isospin_breaking_1S0=int(m["iso"]))
        ok = in_grid_mask(cells, len(deut), pwt.shape[0], Nq, Np)
        assert np.all(np.isnan(U_BU[~ok]))
        assert rel(U_BU[ok], f[f"U_BU_c{c}"][ok]) <= 1e-5, (c, rep)
        assert rel(U, f[f"U_pade_c{c}"]) <= 1e-5, (c, rep)
