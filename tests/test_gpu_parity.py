"""GPU path (through the C-ABI) against the reference's golden outputs and the CPU oracle."""
import numpy as np
import pytest

import harness as oracle
import tictac_b200 as tt
from conftest import CASES, GOLDEN, load_case, rel, rel_elem

pytestmark = pytest.mark.gpu

PRECISIONS = [tt.PRECISION_FP64, tt.PRECISION_MIXED, tt.PRECISION_MIXED_SIMT]


def swp_of(g, m):
    Np, Nq = m["Np"], m["Nq"]
    return tt.SWP(Np, Nq, len(g["e_unco"]) // (Np + 1), len(g["e_coup"]) // (2 * (Np + 1)), float(g["E_bound"]),
                  g["e_unco"], g["e_coup"], g["C_unco"], g["C_coup"], g["q_WP"])


def csc_of(n, row, col, val):
    order = np.lexsort((row, col))
    colptr = np.zeros(n + 1, dtype=np.uint64)
    np.add.at(colptr, np.asarray(col, dtype=np.int64) + 1, 1)
    return val[order], row[order], np.cumsum(colptr).astype(np.uint64)


@pytest.mark.parametrize("case", CASES)
def test_p123_pattern_bit_exact_and_values(case):
    g, m = load_case(case)
    for c in range(int(g["n_chn"])):
        pw = tt.PW(g[f"pw_c{c}"])
        r, cc, v = tt.fill_P123_arrays(pw, g["p_WP"], g["q_WP"], Nphi=m["Nphi"], Nx=m["Nx"])
        assert np.array_equal(r, g[f"p123_row_c{c}"]) and np.array_equal(cc, g[f"p123_col_c{c}"])
        assert rel(v, g[f"p123_val_c{c}"]) <= 1e-13


@pytest.mark.parametrize("case", CASES)
def test_resolvent_matches_reference(case):
    g, m = load_case(case)
    swp = swp_of(g, m)
    E = g["E_com"] + float(g["E_bound"])
    for c in range(int(g["n_chn"])):
        pw = tt.PW(g[f"pw_c{c}"])
        G = np.stack([tt.resolvent(e, swp, pw, tensor_force=int(m["tensor_force"]), isospin_breaking_1S0=int(m["iso"]))
                      for e in E])
        assert rel(G.reshape(-1), g[f"G_c{c}"]) <= 1e-11


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision", PRECISIONS)
def test_solve_dropin_matches_reference(case, precision):
    g, m = load_case(case)
    swp = swp_of(g, m)
    for c in range(int(g["n_chn"])):
        pwt = g[f"pw_c{c}"]
        n = pwt.shape[0] * m["Np"] * m["Nq"]
        v, r, cp = csc_of(n, g[f"p123_row_c{c}"], g[f"p123_col_c{c}"], g[f"p123_val_c{c}"])
        U, rep = tt.solve_faddeev(g[f"G_c{c}"], v, r, cp, g["V_unco"], g["V_coup"], swp, g["q_idx"],
                                  oracle.deuterons(pwt), tt.PW(pwt), precision=precision,
                                  tensor_force=int(m["tensor_force"]), isospin_breaking_1S0=int(m["iso"]))
        assert rel_elem(U, g[f"U_c{c}"]) <= 1e-10, (c, rep)


@pytest.mark.parametrize("case", CASES)
def test_run_handle_end_to_end(case):
    g, m = load_case(case)
    run = tt.Run(**m["opts"])
    for c in range(run.num_channels):
        for prec in (tt.PRECISION_FP64, tt.PRECISION_MIXED):
            U, rep = run.solve(c, prec)
            assert rel_elem(U, g[f"U_c{c}"]) <= 1e-10
    run.close()


@pytest.mark.parametrize("case", ["mt_swave_n16", "lo_j1_J3_n8"])
def test_A_matches_oracle(case):
    g, m = load_case(case)
    run = tt.Run(**m["opts"])
    for c in range(run.num_channels):
        pw = run.host_array(0, c).reshape(-1, 9)
        lay = oracle.layout(pw, m["Np"], run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                            run.host_array(7), run.host_array(8), m["tensor_force"], m["iso"])
        run.build_A(c)
        A = run.A(c)
        A_o = oracle.build_A(lay, pw.shape[0], m["Nq"], m["Np"], g[f"p123_row_c{c}"], g[f"p123_col_c{c}"],
                             g[f"p123_val_c{c}"])
        assert rel(A, A_o) <= 1e-12
    run.close()


def test_larger_case_against_oracle():
    # j <= 2, J <= 3/2, N = 8 with tensor force and isospin breaking: beyond the fixtures
    opts = dict(potential_model="LO_internal", J_2N_max=2, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=20, Nx=20,
                lab_energies="7,40")
    run = tt.Run(**opts)
    Np = Nq = 8
    T, E_com, q_idx = run.energies()
    for c in [0, run.num_channels - 1]:
        pw = run.host_array(0, c).reshape(-1, 9)
        nnz = run.build_P123(c)
        rowptr, col, val = run.P123_csr(c, nnz)
        r_o, c_o, v_o = oracle.p123(pw, run.host_array(1), run.host_array(2), 20, 20)
        rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int32), np.diff(rowptr))
        assert np.array_equal(rows, r_o) and np.array_equal(col, c_o)
        assert rel(val, v_o) <= 1e-13
        lay = oracle.layout(pw, Np, run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                            run.host_array(7), run.host_array(8))
        G_o = np.stack([oracle.resolvent(lay, pw.shape[0], Nq, Np, run.host_array(2), e + run.E_bound) for e in E_com])
        A_o = oracle.build_A(lay, pw.shape[0], Nq, Np, r_o, c_o, v_o)
        U_o = oracle.dense_solve(A_o, G_o, q_idx, oracle.deuterons(pw), Nq, Np)
        for prec in PRECISIONS:
            U, rep = run.solve(c, prec)
            assert rel_elem(U, U_o) <= 1e-10, (prec, rep)
    run.close()


@pytest.mark.parametrize("Np,Nq", [(9, 7), (11, 3)])
def test_ragged_block_sizes_against_oracle(Np, Nq):
    # n = Nalpha * Np * Nq (363 .. 945) is no multiple of the 32/64/128-row
    # blocks of the factorisation and the substitutions: partial blocks everywhere
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=Np, Nq_WP=Nq, Nphi=16, Nx=16,
                lab_energies="12")
    run = tt.Run(**opts)
    T, E_com, q_idx = run.energies()
    for c in range(run.num_channels):
        pw = run.host_array(0, c).reshape(-1, 9)
        nnz = run.build_P123(c)
        rowptr, col, val = run.P123_csr(c, nnz)
        lay = oracle.layout(pw, Np, run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                            run.host_array(7), run.host_array(8))
        rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int32), np.diff(rowptr))
        G_o = np.stack([oracle.resolvent(lay, pw.shape[0], Nq, Np, run.host_array(2), e + run.E_bound) for e in E_com])
        A_o = oracle.build_A(lay, pw.shape[0], Nq, Np, rows, col, val)
        run.build_A(c)  # odd Np: chunks of 7 (63 columns) or 5 (55) q' values, unaligned rows
        assert rel(run.A(c), A_o) <= 1e-12, c
        U_o = oracle.dense_solve(A_o, G_o, q_idx, oracle.deuterons(pw), Nq, Np)
        for prec in PRECISIONS:
            U, rep = run.solve(c, prec)
            assert rel_elem(U, U_o) <= 1e-10, (c, prec, rep)
    run.close()


@pytest.mark.parametrize("case", ["mt_swave_n16", "lo_j1_J3_n8"])
def test_pade_path_matches_reference_pade(case):
    # TT_PRECISION_PADE against the reference's own Pade output and its dense
    # solve, at the method's accuracy (its stopping rule is 1e-6 relative)
    g, m = load_case(case)
    p = np.load(f"{GOLDEN}/{case}_pade.npz")
    run = tt.Run(**m["opts"])
    for c in range(run.num_channels):
        U, rep = run.solve(c, tt.PRECISION_PADE)
        assert rel(U, p[f"U_pade_c{c}"]) <= 1e-5, (c, rep)
        assert rel(U, g[f"U_c{c}"]) <= 1e-5, (c, rep)
        assert 1 <= rep["refine_iters"] <= 14
    run.close()


def test_full_size_channel_mixed_agrees_with_fp64():
    # largest channel of the j<=3, J<=7/2 basis at N=16 (n = 16128): size-independent check
    # that refinement recovers the FP64 solution
    run = tt.Run(potential_model="LO_internal", J_2N_max=3, two_J_3N_max=7, Np_WP=16, Nq_WP=16, lab_energies="10")
    c = max(range(run.num_channels), key=lambda k: run.channel_info(k)["n"])
    U64, _ = run.solve(c, tt.PRECISION_FP64)
    Um, rep = run.solve(c, tt.PRECISION_MIXED)
    assert rep["final_correction"] <= 1e-12 and rep["refine_iters"] >= 1
    assert rel_elem(Um, U64) <= 1e-10
    run.close()


def test_refinement_nonconvergence_is_reported():
    g, m = load_case("mt_swave_n16")
    pwt = g["pw_c0"]
    n = pwt.shape[0] * m["Np"] * m["Nq"]
    v, r, cp = csc_of(n, g["p123_row_c0"], g["p123_col_c0"], g["p123_val_c0"])
    with pytest.raises(tt.TicTacError) as e:
        tt.solve_faddeev(g["G_c0"], v, r, cp, g["V_unco"], g["V_coup"], swp_of(g, m), g["q_idx"], [1], tt.PW(pwt),
                         precision=tt.PRECISION_MIXED, tensor_force=0, isospin_breaking_1S0=0, refine_max_iter=1,
                         refine_tol=1e-300)
    assert e.value.code == tt.TT_ERR_NOCONVERGE


def test_hbm_admission_reports_nomem_without_fault():
    # n = 2 * 316 * 316 = 199712: A alone would need 319 GB
    Np = Nq = 316
    pw = np.array([[0, 0, 0, 1, 0, 1, 1, 1, 1], [0, 1, 1, 0, 0, 1, 1, 1, 1]], dtype=np.int32)
    n = 2 * Np * Nq
    qwp = np.linspace(0, 1000, Nq + 1)
    # tensor force off, no isospin breaking: 6 uncoupled 2N slots for j <= 1 (CPP/main.cpp:283-288)
    swp = tt.SWP(Np, Nq, 6, 0, -2.0, np.linspace(-2, 100, (Np + 1) * 6), None, np.tile(np.eye(Np).ravel(), 6),
                 None, qwp)
    G = np.zeros(n, dtype=np.complex128)
    with pytest.raises(tt.TicTacError) as e:
        tt.solve_faddeev(G, np.zeros(0), np.zeros(0, dtype=np.int32), np.zeros(n + 1, dtype=np.uint64),
                         np.zeros(Np * Np * 6), None, swp, [0], [1], tt.PW(pw), tensor_force=0, isospin_breaking_1S0=0)
    assert e.value.code == tt.TT_ERR_NOMEM
    # the device stays usable afterwards
    g, m = load_case("mt_swave_n16")
    run = tt.Run(**m["opts"])
    U, _ = run.solve(0, tt.PRECISION_FP64)
    assert rel_elem(U, g["U_c0"]) <= 1e-10


def test_no_deuteron_states_gives_empty_U():
    g, m = load_case("mt_swave_n16")
    pwt = g["pw_c0"]
    n = pwt.shape[0] * m["Np"] * m["Nq"]
    v, r, cp = csc_of(n, g["p123_row_c0"], g["p123_col_c0"], g["p123_val_c0"])
    U, rep = tt.solve_faddeev(g["G_c0"], v, r, cp, g["V_unco"], g["V_coup"], swp_of(g, m), g["q_idx"], [],
                              tt.PW(pwt), tensor_force=0, isospin_breaking_1S0=0)
    assert U.size == 0


def test_kernel_launch_counter_advances():
    g, m = load_case("mt_swave_n16")
    before = tt.kernel_launches()
    run = tt.Run(**m["opts"])
    run.solve(0, tt.PRECISION_MIXED)
    assert tt.kernel_launches() > before


def _large_fixture_tools():
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import pattern_hash, value_checksums, vector_checksums
    return pattern_hash, value_checksums, vector_checksums


@pytest.mark.parametrize("product", ["bf16x3", "tf32", "bf16x3_n128"])
def test_bench_basis_n12_against_reference(product):
    # The bench workload's basis (j <= 3, J <= 7/2, both parities) at Np = Nq = 12: eight channels,
    # n = 3,888 .. 9,072, so 8 - 18 panels of 512 columns with the K = 512 tensor-core trailing updates,
    # interchanges across panels and the two on-shell energies factored together.  Against the reference's
    # own dense solve (zgetrf + zgetrs, nrhs = n): P123 pattern (hash) and values (checksums), G
    # (checksums) and every on-shell U element, in FP64, in mixed precision with each tensor-core product
    # and (once) on CUDA cores.
    pattern_hash, value_checksums, vector_checksums = _large_fixture_tools()
    g = np.load(f"{GOLDEN}/lo_j3_J7_n12.npz")
    opts = dict(o.split("=", 1) for o in g["opts"])
    run = tt.Run(**opts, tc_product=product)
    assert run.num_channels == int(g["n_chn"])
    T, E_com, q_idx = run.energies()
    assert np.array_equal(q_idx, g["q_idx"])
    precisions = [tt.PRECISION_MIXED] + ([tt.PRECISION_FP64, tt.PRECISION_MIXED_SIMT] if product == "bf16x3" else [])
    for c in range(run.num_channels):
        n = run.channel_info(c)["n"]
        assert n == int(g[f"n_c{c}"])
        if product == "bf16x3":
            nnz = run.build_P123(c)
            assert nnz == int(g[f"nnz_c{c}"])
            rowptr, col, val = run.P123_csr(c, nnz)
            rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rowptr))
            assert pattern_hash(rows, col, n) == int(g[f"p123_hash_c{c}"])
            assert rel(value_checksums(rows, col, val, n), g[f"p123_sums_c{c}"]) <= 1e-12
            run.build_resolvent(c)
            assert rel(vector_checksums(run.G(c).reshape(-1)), g[f"G_sums_c{c}"]) <= 1e-11
        for prec in precisions:
            U, rep = run.solve(c, prec)
            err = rel_elem(U, g[f"U_c{c}"])
            assert err <= 1e-10, (c, n, prec, err, rep)
        run.release(c)
    run.close()


@pytest.mark.parametrize("batch", [2, 3, 4])
def test_energy_batched_factorisation_matches_one_at_a_time(batch):
    # Five on-shell bins (T_lab = 5, 30, 100 MeV) at n = 1,100 (ragged against every block size): the
    # complex64 matrices factored in groups of 2+2+1, 3+2 and 4+1 energies (the batched sub-panel kernel
    # splits its grid into one group of CTAs per matrix, with a remainder group of fewer matrices) give
    # the U of the one-at-a-time factorisation bit for bit (same arithmetic per row, same pivots), and U
    # matches the oracle per element.
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=1, Np_WP=10, Nq_WP=10, Nphi=16, Nx=16,
                lab_energies="5,30,100")
    base = tt.Run(**opts, energy_batch=1)
    run = tt.Run(**opts, energy_batch=batch)
    T, E_com, q_idx = run.energies()
    assert len(T) == 5
    Np = Nq = 10
    for c in range(run.num_channels):
        U1, _ = base.solve(c, tt.PRECISION_MIXED)
        Ub, rep = run.solve(c, tt.PRECISION_MIXED)
        assert np.array_equal(U1, Ub), (c, batch, rel_elem(Ub, U1))
        pw = run.host_array(0, c).reshape(-1, 9)
        nnz = run.build_P123(c)
        rowptr, col, val = run.P123_csr(c, nnz)
        rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int32), np.diff(rowptr))
        lay = oracle.layout(pw, Np, run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                            run.host_array(7), run.host_array(8))
        G_o = np.stack([oracle.resolvent(lay, pw.shape[0], Nq, Np, run.host_array(2), e + run.E_bound) for e in E_com])
        A_o = oracle.build_A(lay, pw.shape[0], Nq, Np, rows, col, val)
        U_o = oracle.dense_solve(A_o, G_o, q_idx, oracle.deuterons(pw), Nq, Np)
        assert rel_elem(Ub, U_o) <= 1e-10, (c, batch, rep)
    base.close()
    run.close()


def test_tf32_refinement_falls_back_to_bf16x3():
    # with at most three refinement steps the TF32 factors (about 2^-11 per
    # product, four steps to 1e-12) do not refine in time; each such energy
    # group is factored again with BF16x3 (two steps), and U still matches the
    # reference in every element
    g, m = load_case("lo_j1_J3_n8")
    run = tt.Run(**m["opts"], tc_product="tf32", refine_max_iter=3)
    fallbacks = 0
    for c in range(run.num_channels):
        U, rep = run.solve(c, tt.PRECISION_MIXED)
        assert rel_elem(U, g[f"U_c{c}"]) <= 1e-10, (c, rep)
        fallbacks += rep["product_fallbacks"]
    assert fallbacks >= 1
    run.close()


@pytest.mark.parametrize("product", ["tf32", "bf16x3"])
def test_panel_widths_agree(product):
    # n = 1,100 factored with outer panels of 32, 96, 256 and 512 columns
    # (ragged last panel for each) and unit-lower inverses of 32 to 512 rows:
    # the refined U agrees per element with the FP64 solve whatever the choice
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=1, Np_WP=10, Nq_WP=10, Nphi=16, Nx=16,
                lab_energies="5,30")
    run = tt.Run(**opts, tc_product=product)
    for c in range(run.num_channels):
        U64, _ = run.solve(c, tt.PRECISION_FP64)
        # panel widths, and the largest unit-lower block solved by its explicit inverse
        # and the updates on single CTAs or on CTA pairs (256-row tiles)
        # and panels in mid-panels of 64 or 128 columns
        for w, ib, pairs, mid in ((32, 0, 0, 0), (96, 0, 0, 0), (256, 0, 0, 0), (512, 0, 0, 0), (512, 32, 0, 0),
                                  (512, 128, 0, 0), (512, 0, 1, 0), (256, 128, 1, 0), (512, 0, 0, 128),
                                  (512, 0, 1, 128), (384, 0, 0, 64), (512, 32, 0, 96)):
            run.set_solve_option("panel_width", w)
            run.set_solve_option("inverse_block", ib)
            run.set_solve_option("cta_pairs", "true" if pairs else "false")
            run.set_solve_option("mid_panel", mid)
            U, rep = run.solve(c, tt.PRECISION_MIXED)
            assert rel_elem(U, U64) <= 1e-10, (c, w, ib, pairs, mid, rep)
        for k, v in (("panel_width", 0), ("inverse_block", 0), ("cta_pairs", "false"), ("mid_panel", 0)):
            run.set_solve_option(k, v)
    run.close()
