"""The CPU oracle (oracle/*.c) against the reference's own outputs
(tests/golden/*.npz, produced by the reference's CPP/ code: make_golden.py)."""
import numpy as np
import pytest

import harness as oracle
import os

from conftest import CASES, GOLDEN, load_case, rel, rel_elem


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    g, m = load_case(case)
    Np, Nq = m["Np"], m["Nq"]
    for c in range(int(g["n_chn"])):
        pw = g[f"pw_c{c}"]
        Na = pw.shape[0]
        r, cc, v = oracle.p123(pw, g["p_WP"], g["q_WP"], m["Nphi"], m["Nx"])
        rr, rc, rv = g[f"p123_row_c{c}"], g[f"p123_col_c{c}"], g[f"p123_val_c{c}"]
        # nonzero pattern bit-exact, in the reference's row-major order
        assert np.array_equal(r, rr) and np.array_equal(cc, rc)
        assert rel(v, rv) <= 1e-13
        lay = oracle.layout(pw, Np, g["V_unco"], g["V_coup"], g["C_unco"], g["C_coup"], g["e_unco"], g["e_coup"],
                            m["tensor_force"], m["iso"])
        E = g["E_com"] + float(g["E_bound"])
        G = np.stack([oracle.resolvent(lay, Na, Nq, Np, g["q_WP"], e) for e in E])
        assert rel(G.reshape(-1), g[f"G_c{c}"]) <= 1e-12
        A = oracle.build_A(lay, Na, Nq, Np, rr, rc, rv)
        U = oracle.dense_solve(A, G, g["q_idx"], oracle.deuterons(pw), Nq, Np)
        assert rel_elem(U, g[f"U_c{c}"]) <= 1e-10


def test_oracle_empty_channel_edge():
    # a channel without deuteron states has no elastic U elements
    g, m = load_case("lo_j1_J3_n8")
    pw = g["pw_c0"]
    A = np.eye(pw.shape[0] * m["Np"] * m["Nq"])
    G = np.zeros((1, A.shape[0]), dtype=np.complex128)
    U = oracle.dense_solve(A, G, g["q_idx"][:1], [], m["Nq"], m["Np"])
    assert U.size == 0


@pytest.mark.parametrize("case", ["mt_swave_n16", "lo_j1_J3_n8"])
def test_oracle_pade_matches_reference_pade(case):
    # the reference's default production path (Pade-resummed Neumann series);
    # high-order Pade ratios amplify 1e-15 differences in the coefficients to
    # about 1e-7, so the method is compared at its own accuracy
    g, m = load_case(case)
    p = np.load(os.path.join(GOLDEN, f"{case}_pade.npz"))
    for c in range(int(g["n_chn"])):
        pw = g[f"pw_c{c}"]
        lay = oracle.layout(pw, m["Np"], g["V_unco"], g["V_coup"], g["C_unco"], g["C_coup"], g["e_unco"], g["e_coup"],
                            m["tensor_force"], m["iso"])
        A = oracle.build_A(lay, pw.shape[0], m["Nq"], m["Np"], g[f"p123_row_c{c}"], g[f"p123_col_c{c}"],
                           g[f"p123_val_c{c}"])
        U = oracle.pade_solve(A, g[f"G_c{c}"], g["q_idx"], oracle.deuterons(pw), m["Nq"], m["Np"])
        assert rel(U, p[f"U_pade_c{c}"]) <= 1e-5
        assert rel(U, g[f"U_c{c}"]) <= 1e-5
