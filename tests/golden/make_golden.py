"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs oracle/_ref/tictac_ref (the reference's own CPP/ sources compiled
against the shims in oracle/ref/shim, see oracle/Makefile) on small
configurations and packs every stage it dumps (partial-wave tables, WP
boundaries, V, C, SWP energies, P123 in the reference's row-major COO order,
resolvents, on-shell U) into one .npz per case.

    make -C oracle ref && python tests/golden/make_golden.py [--pade]

(--pade regenerates only the Pade fixtures <case>_pade.npz.)

Test infrastructure only; the product never reads these files.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.normpath(os.path.join(HERE, "..", ".."))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "tictac_ref")

CASES = {
    # config 1 of the benchmark set: Malfliet-Tjon, s-waves, one channel 1/2+, N=16, T_lab = 13 MeV
    "mt_swave_n16": dict(potential_model="malfliet_tjon", swave_only="true", isospin_breaking_1S0="false",
                         tensor_force="false", J_2N_max=1, two_J_3N_max=1, Np_WP=16, Nq_WP=16, lab_energies="13"),
    # chiral LO with one-pion exchange: tensor-coupled 3S1-3D1, isospin-breaking 1S0, four channels
    "lo_j1_J3_n8": dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=8, Nq_WP=8, Nphi=16,
                        Nx=16, lab_energies="10"),
    # Malfliet-Tjon with all partial waves up to j=2 (non-interacting higher waves), two energies
    "mt_j2_J1_n8": dict(potential_model="malfliet_tjon", J_2N_max=2, two_J_3N_max=1, Np_WP=8, Nq_WP=8, Nphi=16,
                        Nx=16, lab_energies="5,30"),
}


def read_meta(path):
    meta = {"channels": []}
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "E_bound":
                meta["E_bound"] = float(tok[1])
            elif tok[0] == "chn":
                d = dict(zip(tok[::2], tok[1::2]))
                meta["channels"].append({k: (float(v) if "." in v or "e" in v else int(v)) for k, v in d.items()})
            elif tok[0] == "energies":
                v = tok[1:]
                meta["T_lab"] = np.array([float(x) for x in v[0::3]])
                meta["E_com"] = np.array([float(x) for x in v[1::3]])
                meta["q_idx"] = np.array([int(x) for x in v[2::3]], dtype=np.int32)
    return meta


def run_case(name, opts):
    with tempfile.TemporaryDirectory() as out:
        args = [REF_BIN, "dump", out, "--solver=replica"] + [f"{k}={v}" for k, v in opts.items()]
        subprocess.run(args, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
        meta = read_meta(os.path.join(out, "meta.txt"))

        def rd(fname, dtype):
            p = os.path.join(out, fname + ".bin")
            return np.fromfile(p, dtype=dtype) if os.path.exists(p) else np.zeros(0, dtype=dtype)

        data = {
            "opts": np.array([f"{k}={v}" for k, v in opts.items()]),
            "E_bound": np.array(meta["E_bound"]),
            "T_lab": meta["T_lab"], "E_com": meta["E_com"], "q_idx": meta["q_idx"],
            "p_WP": rd("p_WP", np.float64), "q_WP": rd("q_WP", np.float64),
            "V_unco": rd("V_unco", np.float64), "V_coup": rd("V_coup", np.float64),
            "C_unco": rd("C_unco", np.float64), "C_coup": rd("C_coup", np.float64),
            "e_unco": rd("e_unco", np.float64), "e_coup": rd("e_coup", np.float64),
            "n_chn": np.array(len(meta["channels"])),
        }
        for ch in meta["channels"]:
            c = ch["chn"]
            t = f"_c{c}"
            data["pw" + t] = rd("pw" + t, np.int32).reshape(-1, 9)
            data["p123_row" + t] = rd("p123_row" + t, np.int32)
            data["p123_col" + t] = rd("p123_col" + t, np.int32)
            data["p123_val" + t] = rd("p123_val" + t, np.float64)
            data["G" + t] = rd("G" + t, np.complex128)
            data["U" + t] = rd("U" + t, np.complex128)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print(name, "channels", len(meta["channels"]), "n", [ch["n"] for ch in meta["channels"]],
              "nnz", [ch["nnz"] for ch in meta["channels"]])


def run_pade(name, opts):
    """U of the reference's default production path (Pade-resummed Neumann
    series, CPP/solve_faddeev.cpp:440-1444) for the same case, written to
    <name>_pade.npz as U_pade_c<k>."""
    with tempfile.TemporaryDirectory() as out:
        args = [REF_BIN, "dump", out, "--solver=pade"] + [f"{k}={v}" for k, v in opts.items()]
        subprocess.run(args, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
        meta = read_meta(os.path.join(out, "meta.txt"))
        data = {}
        for ch in meta["channels"]:
            c = ch["chn"]
            data[f"U_pade_c{c}"] = np.fromfile(os.path.join(out, f"U_c{c}.bin"), dtype=np.complex128)
        np.savez_compressed(os.path.join(HERE, f"{name}_pade.npz"), **data)
        print(name, "pade channels", len(meta["channels"]))


PADE_CASES = ["mt_swave_n16", "lo_j1_J3_n8"]

if __name__ == "__main__":
    if not os.path.exists(REF_BIN):
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` first")
    only_pade = "--pade" in sys.argv
    for name, opts in CASES.items():
        if not only_pade:
            run_case(name, opts)
        if name in PADE_CASES:
            run_pade(name, opts)
