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
