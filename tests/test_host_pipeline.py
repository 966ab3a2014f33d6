"""Host state-space setup behind the C-ABI (no GPU needed) against the reference."""
import numpy as np
import pytest

import tictac_b200 as tt
from conftest import CASES, load_case, rel


@pytest.mark.parametrize("case", CASES)
def test_state_space_matches_reference(case):
    g, m = load_case(case)
    run = tt.Run(**m["opts"])
    assert run.num_channels == int(g["n_chn"])
    for c in range(run.num_channels):
        assert np.array_equal(run.host_array(0, c).reshape(-1, 9), g[f"pw_c{c}"])
    # WP boundaries and potential matrices are bit-identical
    assert np.array_equal(run.host_array(1), g["p_WP"])
    assert np.array_equal(run.host_array(2), g["q_WP"])
    assert np.array_equal(run.host_array(3), g["V_unco"])
    assert np.array_equal(run.host_array(4), g["V_coup"])
    # SWP energies from a different symmetric eigensolver: FP64 rounding level
    scale = max(np.max(np.abs(g["e_unco"])), 1.0)
    assert np.max(np.abs(run.host_array(7) - g["e_unco"])) <= 1e-12 * scale
    if g["e_coup"].size:
        assert np.max(np.abs(run.host_array(8) - g["e_coup"])) <= 1e-12 * max(np.max(np.abs(g["e_coup"])), 1.0)
    assert abs(run.E_bound - float(g["E_bound"])) <= 1e-12 * abs(float(g["E_bound"]))
    T, E, q = run.energies()
    assert np.array_equal(q, g["q_idx"])
    assert rel(T, g["T_lab"]) <= 1e-12 and rel(E, g["E_com"]) <= 1e-12


def test_bad_option_and_model_errors():
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(not_a_key="3")
    assert e.value.code == tt.TT_ERR_BADARG
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(two_J_3N_max=2)
    assert e.value.code == tt.TT_ERR_BADARG
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(tensor_force="maybe")
    assert e.value.code == tt.TT_ERR_BADARG
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(potential_model="Idaho_N3LO", J_2N_max=1, Np_WP=8, Nq_WP=8, lab_energies="10")
    assert "Fortran" in str(e.value)
    # an energy beyond every pair of q-bin midpoints selects no on-shell bin
    # (run_organizer.cpp:57-85): no energies, not an error
    run = tt.Run(potential_model="malfliet_tjon", J_2N_max=1, Np_WP=8, Nq_WP=8, lab_energies="1e9")
    assert len(run.energies()[0]) == 0


def test_u_table_format(tmp_path):
    g, m = load_case("mt_swave_n16")
    run = tt.Run(**m["opts"])
    U = g["U_c0"]
    p = str(tmp_path / "U.txt")
    run.write_U_table(0, U, p)
    txt = open(p).read().splitlines()
    labels = [l for l in txt if l.strip().startswith("U")]
    rows = [l for l in txt if l.strip() and not l.startswith("#") and not l.strip().startswith("U")]
    assert len(labels) == 1 and len(rows) == len(g["q_idx"])  # disk_io_routines.cpp:820-908 layout
    for j, line in enumerate(rows):
        f = line.split()
        assert int(f[2]) == int(g["q_idx"][j])
        assert abs(complex(f[3]) - U[j]) <= 1e-15 * abs(U[j])


def test_energy_batch_option_range():
    opts = dict(potential_model="malfliet_tjon", J_2N_max=1, two_J_3N_max=1, Np_WP=8, Nq_WP=8, lab_energies="10")
    for v in (1, 2, 4):
        tt.Run(energy_batch=v, **opts).close()
    for v in (0, 5):
        with pytest.raises(tt.TicTacError, match="energy_batch"):
            tt.Run(energy_batch=v, **opts)


def test_solve_options_on_a_run():
    opts = dict(potential_model="malfliet_tjon", J_2N_max=1, two_J_3N_max=1, Np_WP=8, Nq_WP=8, lab_energies="10")
    for v in (0, 32, 256, 384, 512):
        tt.Run(panel_width=v, **opts).close()
    for v in (16, 600, -32):
        with pytest.raises(tt.TicTacError, match="panel_width"):
            tt.Run(panel_width=v, **opts)
    run = tt.Run(**opts)
    for k, v in (("panel_width", 384), ("tc_product", "bf16x3"), ("panel_order", "recursive"), ("energy_batch", 2),
                 ("refine_tol", 1e-11), ("refine_max_iter", 30), ("inverse_block", 256), ("cta_pairs", "true"),
                 ("mid_panel", 128)):
        run.set_solve_option(k, v)
    with pytest.raises(tt.TicTacError, match="panel_width"):
        run.set_solve_option("panel_width", 48)
    with pytest.raises(tt.TicTacError, match="inverse_block"):
        run.set_solve_option("inverse_block", 1024)
    # state-space options are fixed once the run is built
    with pytest.raises(tt.TicTacError, match="not a solve option"):
        run.set_solve_option("Np_WP", 10)
    run.close()


def test_panel_table_rows_and_header():
    from tictac_b200 import autotune
    timings = {"tf32": {9072: {256: 3.0, 512: 2.0}, 20000: {256: 9.0, 512: 8.0}, 56700: {256: 50.0, 512: 51.0}},
               "bf16x3": {9072: {256: 4.0, 512: 5.0}}}
    rows = autotune.table_rows(timings)
    assert rows == [(2, (20000 + 56700) // 2, 512), (2, 1 << 30, 256), (3, 1 << 30, 256)]
    h = autotune.render_header(rows, "test")
    assert "{2, 38350, 512}," in h and "{2, 1 << 30, 256}," in h and "{1, 1 << 30, 512}," in h
    # the committed header has the same shape as the rendered one
    src = open(autotune.HEADER).read()
    assert "kPanelWidthTable" in src and "struct PanelWidthRow" in src


def write_custom_grids(g, tmp_path):
    paths = {}
    for key in ("p", "q"):
        p = tmp_path / f"{key}_grid.dat"
        p.write_text(str(g[f"{key}_grid_text"]))
        paths[f"{key}_grid_filename"] = str(p)
    return paths


def test_custom_grids_match_reference(tmp_path):
    # p_grid_type=custom: boundaries read from files (CPP/make_wp_states.cpp:46-75,
    # disk_io_routines.cpp:977-994); the fixture was made by the reference with
    # the same files.  The host stages reproduce the reference's grids and V bit
    # for bit, and the oracle chain (P123 -> A -> LU) on them its U
    import harness as oracle
    from conftest import load_case as _load, rel_elem
    g, m = _load("mt_swave_custom_n8")
    run = tt.Run(**m["opts"], **write_custom_grids(g, tmp_path))
    assert np.array_equal(run.host_array(1), g["p_WP"])
    assert np.array_equal(run.host_array(2), g["q_WP"])
    assert np.array_equal(run.host_array(3), g["V_unco"])
    assert np.max(np.abs(run.host_array(7) - g["e_unco"])) <= 1e-12 * max(np.max(np.abs(g["e_unco"])), 1.0)
    T, E, q = run.energies()
    assert np.array_equal(q, g["q_idx"]) and rel(T, g["T_lab"]) <= 1e-12 and rel(E, g["E_com"]) <= 1e-12
    pw = run.host_array(0, 0).reshape(-1, 9)
    assert np.array_equal(pw, g["pw_c0"])
    r, c, v = oracle.p123(pw, run.host_array(1), run.host_array(2), m["Nphi"], m["Nx"])
    assert np.array_equal(r, g["p123_row_c0"]) and np.array_equal(c, g["p123_col_c0"])
    assert rel(v, g["p123_val_c0"]) <= 1e-13
    lay = oracle.layout(pw, m["Np"], run.host_array(3), run.host_array(4), run.host_array(5), run.host_array(6),
                        run.host_array(7), run.host_array(8), tensor_force=False, iso=False)
    Na = pw.shape[0]
    G = np.stack([oracle.resolvent(lay, Na, m["Nq"], m["Np"], run.host_array(2), e + run.E_bound) for e in E])
    A = oracle.build_A(lay, Na, m["Nq"], m["Np"], r, c, v)
    U = oracle.dense_solve(A, G, q, oracle.deuterons(pw), m["Nq"], m["Np"])
    assert rel_elem(U, g["U_c0"]) <= 1e-10
    run.close()


def test_custom_grid_errors(tmp_path):
    g, m = load_case("mt_swave_custom_n8")
    paths = write_custom_grids(g, tmp_path)
    base = {k: v for k, v in m["opts"].items() if k not in ("p_grid_type", "q_grid_type")}
    # the q grid is read from its file only when the p grid type is "custom",
    # as in the reference (make_wp_states.cpp:69)
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(**base, **paths, p_grid_type="chebyshev", q_grid_type="custom")
    assert "q-momentum gridtype" in str(e.value)
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(**base, **paths, p_grid_type="linear")
    assert "p-momentum gridtype" in str(e.value)
    short = tmp_path / "short.dat"
    short.write_text("0.0\n1.0\n")
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(**base, p_grid_type="custom", q_grid_type="custom", p_grid_filename=str(short),
               q_grid_filename=paths["q_grid_filename"])
    assert "mismatch with number of wave-packets" in str(e.value)
    bad = tmp_path / "bad.dat"
    bad.write_text("0.0\nx\n" + "1.0\n" * 7)
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(**base, p_grid_type="custom", q_grid_type="custom", p_grid_filename=str(bad),
               q_grid_filename=paths["q_grid_filename"])
    assert "Unknown format" in str(e.value)


def test_input_list_file(tmp_path):
    # an argument ending in .txt is an input list of key=value lines, applied in
    # order with the other options (CPP/set_run_parameters.cpp:247-279, 641-644)
    g, m = load_case("mt_j2_J1_n8")
    lst = tmp_path / "run.txt"
    lines = ["# options of the mt_j2_J1_n8 case", "no delimiter on this line", "Nphi = "]
    lines += [f"{k}= {v}" for k, v in m["opts"].items()]
    lst.write_text("\n".join(lines) + "\n")
    a = tt.Run(str(lst))
    b = tt.Run(**m["opts"])
    for which in (1, 2, 3, 7):
        assert np.array_equal(a.host_array(which), b.host_array(which))
    assert np.array_equal(a.energies()[2], b.energies()[2])
    # a later keyword option overrides the list
    c = tt.Run(str(lst), lab_energies="30")
    assert len(c.energies()[0]) >= 1 and not np.array_equal(c.energies()[0], a.energies()[0])
    with pytest.raises(tt.TicTacError) as e:
        tt.Run(str(tmp_path / "missing.txt"))
    assert e.value.code == tt.TT_ERR_BADARG
    for r in (a, b, c):
        r.close()


@pytest.mark.parametrize("case", ["mt_swave_n16", "lo_j1_J3_n8"])
def test_u_table_matches_reference_table(case, tmp_path):
    # tt_run_write_U_table against the reference's own table of the same U
    # (store_U_matrix_elements_txt, disk_io_routines.cpp:759-913; fixture from
    # make_golden.py --tables): header lines and U columns identical, T_lab and
    # E_com within the host set-up's rounding
    import os
    from conftest import GOLDEN
    g, m = load_case(case)
    t = np.load(os.path.join(GOLDEN, f"{case}_tables.npz"))
    run = tt.Run(**m["opts"])
    for c in range(run.num_channels):
        p = str(tmp_path / f"U_c{c}.txt")
        run.write_U_table(c, t[f"U_c{c}"], p)
        ours = open(p).read().split("\n")
        ref = str(t[f"table_c{c}"]).split("\n")
        assert len(ours) == len(ref)
        for a, b in zip(ours, ref):
            if a.startswith("#") or not a.strip() or a.strip().startswith("U"):
                assert a == b
                continue
            ta, tb = a.split(), b.split()
            assert len(ta) == len(tb) and len(a) == len(b)
            for x, y in zip(ta, tb):
                if x.endswith("j") or "." not in x:
                    assert x == y
                else:
                    assert abs(float(x) - float(y)) <= 1e-13 * abs(float(y))
    run.close()


def test_parallel_run_needs_channel_index():
    # set_run_parameters.cpp:666-668
    opts = dict(potential_model="malfliet_tjon", J_2N_max=1, two_J_3N_max=1, Np_WP=8, Nq_WP=8, lab_energies="10")
    with pytest.raises(tt.TicTacError, match="channel index"):
        tt.Run(parallel_run="true", **opts)
    tt.Run(parallel_run="true", channel_idx=0, **opts).close()
    # main.cpp:162-164
    with pytest.raises(tt.TicTacError, match="nothing to do"):
        tt.Run(solve_faddeev="false", calculate_and_store_P123="false", **opts)
