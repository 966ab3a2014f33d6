"""tt_calculate_resolvent_array_in_SWP_basis_noalloc (static device scratch,
no device allocation) against the allocating tt_calculate_resolvent_array_in_SWP_basis.

The file name sorts last so that the GPU test also runs after every other test
in the same process (the scratch lookup must work on a device that other
entry points have already used)."""
import numpy as np
import pytest

import tictac_b200 as tt
from conftest import load_case, rel

# Same kernel, same arithmetic on the same tables: the results agree to
# rounding; the bound leaves room only for the order of device operations.
TOL = 1e-14


def swp_of(g, m):
    Np, Nq = m["Np"], m["Nq"]
    return tt.SWP(Np, Nq, len(g["e_unco"]) // (Np + 1), len(g["e_coup"]) // (2 * (Np + 1)), float(g["E_bound"]),
                  g["e_unco"], g["e_coup"], g["C_unco"], g["C_coup"], g["q_WP"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["mt_swave_n16", "lo_j1_J3_n8"])
def test_noalloc_resolvent_matches_allocating_entry_point(case):
    import torch

    g, m = load_case(case)
    swp = swp_of(g, m)
    kw = dict(tensor_force=int(m["tensor_force"]), isospin_breaking_1S0=int(m["iso"]))
    E0 = g["E_com"] + float(g["E_bound"])
    # two consecutive calls on one stream, the second with other energies
    calls = [E0, np.concatenate([E0[::-1] + 0.75, [E0[0] - 3.0]])]
    stream = torch.cuda.current_stream()
    for c in range(int(g["n_chn"])):
        pw = tt.PW(g[f"pw_c{c}"])
        n = pw.Nalpha * m["Np"] * m["Nq"]
        outs = []
        for E in calls:
            G_dev = torch.full((len(E) * n,), float("nan"), dtype=torch.complex128, device="cuda")
            stream.synchronize()
            tt.resolvent_noalloc(G_dev.data_ptr(), E, swp, pw, stream=stream.cuda_stream, **kw)
            outs.append((E, G_dev))
        stream.synchronize()
        for E, G_dev in outs:
            G = G_dev.cpu().numpy().reshape(len(E), n)
            for j, e in enumerate(E):
                ref = tt.resolvent(float(e), swp, pw, **kw)
                assert np.all(np.isfinite(G[j]))
                assert rel(G[j], ref) <= TOL, (case, c, j)


def test_noalloc_resolvent_rejects_tables_beyond_scratch():
    # 40000 energies alone need 320000 bytes of scratch (limit 262144): the call
    # returns before any device work, so the dummy device address is never used
    g, m = load_case("mt_swave_n16")
    swp = swp_of(g, m)
    E = np.linspace(-2.0, 30.0, 40000)
    with pytest.raises(tt.TicTacError) as e:
        tt.resolvent_noalloc(0x100, E, swp, tt.PW(g["pw_c0"]), tensor_force=0, isospin_breaking_1S0=0)
    assert e.value.code == tt.TT_ERR_UNSUPPORTED
    assert "static scratch holds 262144" in str(e.value)
