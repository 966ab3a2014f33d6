"""Adjoint dU/dtheta (tt_solve_faddeev_adjoint, tt_run_solve_adjoint) against
central finite differences, and the potential's LEC derivatives.

Two derivatives are checked.  The drop-in adjoint differentiates
solve_faddeev_equations with respect to its potential arguments: the
scattering wave-packet basis (C, e_SWP) and the resolvent G are inputs of that
function and stay fixed, as in the finite differences of the drop-in solve.
The run handle's adjoint (adjoint_basis=total, the default) is the physical
derivative: the SWP eigenstates, bin energies and deuteron energy move with the
potential, and with them the resolvent; it is checked against differences of
whole runs with shifted low-energy constants."""
import numpy as np
import pytest

import harness as oracle
import tictac_b200 as tt
from conftest import load_case, rel, rel_elem

# central differences with h = 1e-5 of the potential scale: truncation ~ h^2,
# rounding ~ 1e-16 / h; the adjoint of the refined mixed solve is refined in FP64
FD_TOL = 1e-6


def swp_of(g, m):
    Np, Nq = m["Np"], m["Nq"]
    return tt.SWP(Np, Nq, len(g["e_unco"]) // (Np + 1), len(g["e_coup"]) // (2 * (Np + 1)), float(g["E_bound"]),
                  g["e_unco"], g["e_coup"], g["C_unco"], g["C_coup"], g["q_WP"])


def csc_of(n, row, col, val):
    order = np.lexsort((row, col))
    colptr = np.zeros(n + 1, dtype=np.uint64)
    np.add.at(colptr, np.asarray(col, dtype=np.int64) + 1, 1)
    return val[order], row[order], np.cumsum(colptr).astype(np.uint64)


def symmetric_blocks(rng, V, dim):
    """Seeded perturbations shaped like V ([count][dim][dim]), symmetric per block,
    scaled to the size of V."""
    count = V.size // (dim * dim)
    X = rng.standard_normal((count, dim, dim))
    X = 0.5 * (X + X.transpose(0, 2, 1))
    return (X * np.max(np.abs(V))).reshape(-1)


def test_lec_derivative_is_linear_and_matches_run_difference():
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=1, Np_WP=8, Nq_WP=8, lab_energies="10")
    run = tt.Run(**opts)
    lecs = run.lecs()
    assert lecs.shape == (2,)
    for k in range(2):
        dVu, dVc = run.lec_derivative(k)
        off = [0.0, 0.0]
        off[k] = 1e-3 * abs(lecs[k])
        r2 = tt.Run(lec_offsets=",".join(repr(float(o)) for o in off), **opts)
        assert np.allclose(r2.lecs(), lecs + np.array(off), rtol=0, atol=1e-12 * abs(lecs[k]))
        fd_u = (r2.host_array(3) - run.host_array(3)) / off[k]
        fd_c = (r2.host_array(4) - run.host_array(4)) / off[k]
        scale = max(np.max(np.abs(fd_u)), np.max(np.abs(fd_c)))
        assert scale > 0
        assert np.max(np.abs(dVu - fd_u)) <= 1e-6 * scale
        assert np.max(np.abs(dVc - fd_c)) <= 1e-6 * scale
        r2.close()
    # the 3S1 constant moves the coupled 3S1-3D1 block; with isospin breaking the
    # 1S0 wave is a coupled (T3 = 1/2, 3/2) block as well
    assert np.max(np.abs(run.lec_derivative(1)[1])) > 0.0
    assert np.max(np.abs(run.lec_derivative(0)[1])) > 0.0
    run.close()


def test_lec_offsets_rejected_for_model_without_constants():
    with pytest.raises(tt.TicTacError):
        tt.Run(potential_model="malfliet_tjon", J_2N_max=1, two_J_3N_max=1, Np_WP=8, Nq_WP=8, lec_offsets="0.1")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [tt.PRECISION_FP64, tt.PRECISION_MIXED])
def test_adjoint_dropin_matches_finite_differences(precision):
    g, m = load_case("lo_j1_J3_n8")
    swp = swp_of(g, m)
    Np = m["Np"]
    rng = np.random.default_rng(7)
    dVu = np.stack([symmetric_blocks(rng, g["V_unco"], Np) for _ in range(2)])
    dVc = np.stack([symmetric_blocks(rng, g["V_coup"], 2 * Np) for _ in range(2)])
    kw = dict(tensor_force=int(m["tensor_force"]), isospin_breaking_1S0=int(m["iso"]))
    h = 1e-5
    for c in [0, int(g["n_chn"]) - 1]:
        pwt = g[f"pw_c{c}"]
        n = pwt.shape[0] * Np * m["Nq"]
        v, r, cp = csc_of(n, g[f"p123_row_c{c}"], g[f"p123_col_c{c}"], g[f"p123_val_c{c}"])
        args = (g[f"G_c{c}"], v, r, cp)
        tail = (swp, g["q_idx"], oracle.deuterons(pwt), tt.PW(pwt))
        U, dU, rep = tt.solve_faddeev_adjoint(*args, g["V_unco"], g["V_coup"], *tail, dVu, dVc, precision=precision,
                                              **kw)
        assert rel_elem(U, g[f"U_c{c}"]) <= 1e-10
        if precision == tt.PRECISION_MIXED:
            assert rep["adjoint_refine_iters"] >= 1
        for k in range(2):
            Up, _ = tt.solve_faddeev(*args, g["V_unco"] + h * dVu[k], g["V_coup"] + h * dVc[k], *tail,
                                     precision=tt.PRECISION_FP64, **kw)
            Um, _ = tt.solve_faddeev(*args, g["V_unco"] - h * dVu[k], g["V_coup"] - h * dVc[k], *tail,
                                     precision=tt.PRECISION_FP64, **kw)
            fd = (Up - Um) / (2 * h)
            assert np.max(np.abs(fd)) > 0
            assert rel(dU[k], fd) <= FD_TOL, (c, k, rel(dU[k], fd))


@pytest.mark.gpu
def test_adjoint_run_handle_lec_gradients():
    # dU/dC_1S0 and dU/dC_3S1 of every channel, FP64 and mixed, against central
    # differences of the drop-in FP64 solve with V +- h dV/dC
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=20, Nx=20,
                lab_energies="12")
    run = tt.Run(**opts, adjoint_basis="fixed")
    Np = Nq = 8
    T, E_com, q_idx = run.energies()
    dV = [run.lec_derivative(k) for k in range(2)]
    dVu = np.stack([d[0] for d in dV])
    dVc = np.stack([d[1] for d in dV])
    Vu, Vc = run.host_array(3), run.host_array(4)
    e_unco, e_coup = run.host_array(7), run.host_array(8)
    swp = tt.SWP(Np, Nq, len(e_unco) // (Np + 1), len(e_coup) // (2 * (Np + 1)), run.E_bound, e_unco, e_coup,
                 run.host_array(5), run.host_array(6), run.host_array(2))
    for c in range(run.num_channels):
        pwt = run.host_array(0, c).reshape(-1, 9)
        nnz = run.build_P123(c)
        rowptr, col, val = run.P123_csr(c, nnz)
        n = len(rowptr) - 1
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rowptr))
        v, r, cp = csc_of(n, rows, col, val)
        run.build_resolvent(c)
        G = run.G(c).reshape(-1)
        deut = oracle.deuterons(pwt)
        U64, _ = run.solve(c, tt.PRECISION_FP64)
        for prec in (tt.PRECISION_FP64, tt.PRECISION_MIXED):
            U, dU, rep = run.solve_adjoint(c, dVu, dVc, prec)
            assert rel_elem(U, U64) <= 1e-10
            for k in range(2):
                h = 1e-5 * abs(run.lecs()[k])
                Up, _ = tt.solve_faddeev(G, v, r, cp, Vu + h * dVu[k], Vc + h * dVc[k], swp, q_idx, deut, tt.PW(pwt),
                                         precision=tt.PRECISION_FP64)
                Um, _ = tt.solve_faddeev(G, v, r, cp, Vu - h * dVu[k], Vc - h * dVc[k], swp, q_idx, deut, tt.PW(pwt),
                                         precision=tt.PRECISION_FP64)
                fd = (Up - Um) / (2 * h)
                assert rel(dU[k], fd) <= FD_TOL, (c, prec, k, rel(dU[k], fd))
    run.close()


@pytest.mark.gpu
def test_torch_autograd_wrapper():
    import torch

    from tictac_b200.autograd import u_of_theta

    g, m = load_case("lo_j1_J3_n8")
    Np = m["Np"]
    c = 0
    pwt = g[f"pw_c{c}"]
    n = pwt.shape[0] * Np * m["Nq"]
    v, r, cp = csc_of(n, g[f"p123_row_c{c}"], g[f"p123_col_c{c}"], g[f"p123_val_c{c}"])
    rng = np.random.default_rng(3)
    dVu = np.stack([symmetric_blocks(rng, g["V_unco"], Np) for _ in range(3)])
    dVc = np.stack([symmetric_blocks(rng, g["V_coup"], 2 * Np) for _ in range(3)])
    problem = dict(G=g[f"G_c{c}"], P_val=v, P_row=r, P_colptr=cp, V_unco=g["V_unco"], V_coup=g["V_coup"],
                   swp=swp_of(g, m), q_idx=g["q_idx"], deut=oracle.deuterons(pwt), pw=tt.PW(pwt), dV_unco=dVu,
                   dV_coup=dVc, precision=tt.PRECISION_FP64,
                   rp=dict(tensor_force=int(m["tensor_force"]), isospin_breaking_1S0=int(m["iso"])))
    theta = torch.zeros(3, dtype=torch.float64, requires_grad=True)
    loss = (u_of_theta(theta, problem).abs() ** 2).sum()
    loss.backward()
    # d/dtheta sum |U|^2 = 2 Re(sum conj(U) dU/dtheta), dU from the same adjoint
    U, dU, _ = tt.solve_faddeev_adjoint(problem["G"], v, r, cp, g["V_unco"], g["V_coup"], problem["swp"],
                                        g["q_idx"], problem["deut"], problem["pw"], dVu, dVc,
                                        precision=tt.PRECISION_FP64, **problem["rp"])
    ref = 2 * np.real(np.conj(U)[None, :] * dU).sum(axis=1)
    assert np.allclose(theta.grad.numpy(), ref, rtol=1e-12, atol=0)
    # and against a central difference of the loss
    h = 1e-5
    for k in range(3):
        e = torch.zeros(3, dtype=torch.float64)
        e[k] = h
        fd = ((u_of_theta(e, problem).abs() ** 2).sum() - (u_of_theta(-e, problem).abs() ** 2).sum()) / (2 * h)
        assert abs(fd.item() - theta.grad[k].item()) <= 1e-6 * abs(theta.grad[k].item())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [tt.PRECISION_FP64, tt.PRECISION_MIXED])
def test_adjoint_total_derivative_matches_full_runs(precision):
    # dU/dC_1S0 and dU/dC_3S1 with the chain rule through the SWP eigenstates,
    # bin energies, deuteron energy and resolvent, against central differences
    # of whole FP64 runs with the constants shifted by +- 1e-4 of their value
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=20, Nx=20,
                lab_energies="12")
    run = tt.Run(**opts)
    lecs = run.lecs()
    dV = [run.lec_derivative(k) for k in range(2)]
    dVu = np.stack([d[0] for d in dV])
    dVc = np.stack([d[1] for d in dV])
    shifted = []
    for k in range(2):
        h = 1e-5 * abs(lecs[k])
        pair = []
        for sgn in (1.0, -1.0):
            off = [0.0, 0.0]
            off[k] = sgn * h
            pair.append(tt.Run(lec_offsets=",".join(repr(float(o)) for o in off), **opts))
        shifted.append((h, pair))
    fixed = tt.Run(**opts, adjoint_basis="fixed")
    miss = []
    for c in range(run.num_channels):
        U, dU, rep = run.solve_adjoint(c, dVu, dVc, precision)
        _, dU_fixed, _ = fixed.solve_adjoint(c, dVu, dVc, tt.PRECISION_FP64)
        for k, (h, (rp, rm)) in enumerate(shifted):
            Up, _ = rp.solve(c, tt.PRECISION_FP64)
            Um, _ = rm.solve(c, tt.PRECISION_FP64)
            fd = (Up - Um) / (2 * h)
            assert np.max(np.abs(fd)) > 0
            assert rel(dU[k], fd) <= FD_TOL, (c, k, rel(dU[k], fd))
            miss.append(rel(dU_fixed[k], fd))
    # the basis held fixed misses the chain rule by far more than the tolerance
    assert max(miss) > 100 * FD_TOL, miss
    for _, pair in shifted:
        for r in pair:
            r.close()
    fixed.close()
    run.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [tt.PRECISION_FP64, tt.PRECISION_MIXED])
def test_forward_backward_pair_autograd(precision):
    # the run handle's forward (factors kept) and backward (cotangent) through
    # torch.autograd, against central differences of the loss over whole runs
    import torch

    from tictac_b200.autograd import u_of_lecs

    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=20, Nx=20,
                lab_energies="12")
    c = 2
    theta = torch.zeros(2, dtype=torch.float64, requires_grad=True)
    loss = (u_of_lecs(theta, opts, c, precision).abs() ** 2).sum()
    loss.backward()
    run = tt.Run(**opts)
    lecs = run.lecs()
    run.close()
    for k in range(2):
        h = 1e-5 * abs(lecs[k])
        e = torch.zeros(2, dtype=torch.float64)
        e[k] = h
        lp = (u_of_lecs(e, opts, c, tt.PRECISION_FP64).abs() ** 2).sum().item()
        lm = (u_of_lecs(-e, opts, c, tt.PRECISION_FP64).abs() ** 2).sum().item()
        fd = (lp - lm) / (2 * h)
        assert abs(fd - theta.grad[k].item()) <= FD_TOL * max(abs(fd), 1e-300), (k, fd, theta.grad[k].item())


@pytest.mark.gpu
def test_backward_without_kept_factors_factors_again():
    # five on-shell energies with energy_batch=2: the forward solve cannot keep
    # every energy's factor, so backward factors again; same result as the
    # one-call adjoint
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=1, Np_WP=10, Nq_WP=10, Nphi=16, Nx=16,
                lab_energies="5,30,100", energy_batch=2)
    run = tt.Run(**opts)
    assert len(run.energies()[0]) == 5
    dV = [run.lec_derivative(k) for k in range(2)]
    dVu = np.stack([d[0] for d in dV])
    dVc = np.stack([d[1] for d in dV])
    U, dU, _ = run.solve_adjoint(0, dVu, dVc, tt.PRECISION_MIXED)
    Uf, _ = run.adjoint_forward(0, tt.PRECISION_MIXED)
    assert rel_elem(Uf, U) <= 1e-10
    Ubar = np.conj(Uf)
    g, _ = run.adjoint_backward(0, dVu, dVc, Ubar)
    ref = np.real(np.conj(Ubar)[None, :] * dU).sum(axis=1)
    assert np.allclose(g, ref, rtol=1e-8, atol=0)
    run.close()


def test_swp_derivative_matches_run_differences():
    # the SWP basis derivative (eigenvectors, bin boundaries, deuteron energy)
    # against central differences of runs with a shifted contact constant;
    # host only
    opts = dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=20, Nx=20,
                lab_energies="12")
    run = tt.Run(**opts)
    lecs = run.lecs()
    for k in range(2):
        dVu, dVc = run.lec_derivative(k)
        dCu, dCc, deu, dec, dEb = run.swp_derivative(dVu, dVc)
        h = 1e-5 * abs(lecs[k])
        rs = []
        for sgn in (1.0, -1.0):
            off = [0.0, 0.0]
            off[k] = sgn * h
            rs.append(tt.Run(lec_offsets=",".join(repr(float(o)) for o in off), **opts))
        for which, d in ((5, dCu), (6, dCc), (7, deu), (8, dec)):
            fd = (rs[0].host_array(which) - rs[1].host_array(which)) / (2 * h)
            if np.max(np.abs(fd)) > 0:
                assert rel(d, fd) <= 1e-6, (k, which, rel(d, fd))
            else:
                assert np.max(np.abs(d)) == 0.0
        fdEb = (rs[0].E_bound - rs[1].E_bound) / (2 * h)
        assert abs(dEb - fdEb) <= 1e-6 * max(abs(fdEb), 1e-300) or fdEb == dEb == 0.0
        # the on-shell energies E_j = E_com,j + E_bound: E_com,j is the bin's
        # mid-point energy with the n-d reduced mass mu1(E_bound), so
        # dE_j = dEb (1 - E_com,j dln mu1/dEb), Md = Mn + Mp + E_bound
        Mn, Mp = 939.565, 938.272
        Md = Mn + Mp + run.E_bound
        dlnmu1 = 1.0 / Md - 1.0 / (Mn + Md)
        E_com = run.energies()[1]
        dE = dEb * (1.0 - E_com * dlnmu1)
        fdE = ((rs[0].energies()[1] + rs[0].E_bound) - (rs[1].energies()[1] + rs[1].E_bound)) / (2 * h)
        assert np.max(np.abs(dE - fdE)) <= 1e-6 * max(np.max(np.abs(fdE)), 1e-300) or np.all(fdE == 0.0), (k, dE, fdE)
        for r in rs:
            r.close()
    run.close()
