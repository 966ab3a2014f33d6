"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs oracle/_ref/tictac_ref (the reference's own CPP/ sources compiled
against the shims in oracle/ref/shim, see oracle/Makefile) on small
configurations and packs every stage it dumps (partial-wave tables, WP
boundaries, V, C, SWP energies, P123 in the reference's row-major COO order,
resolvents, on-shell U) into one .npz per case.

    make -C oracle ref && python tests/golden/make_golden.py [--pade | --large]

(--pade regenerates only the Pade fixtures <case>_pade.npz; --large only the
summary fixtures of the bench-sized cases, <case>.npz with U and checksums;
--breakup only the breakup fixtures <case>_breakup.npz; --custom-grid only the
custom-grid fixtures; --tables only the elastic U tables <case>_tables.npz.)

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

# Bench-sized cases: too large to store P123 and G, so the fixture keeps the
# on-shell U of every channel (the reference's zgetrf + zgetrs with nrhs = n)
# and order-independent checksums of P123 and G.
LARGE_CASES = {
    # the bench workload's basis (j <= 3, J <= 7/2, both parities, chiral LO) at
    # Np = Nq = 12: eight channels, n = 3,888 .. 9,072, 8 - 18 panels of 512
    "lo_j3_J7_n12": dict(potential_model="LO_internal", J_2N_max=3, two_J_3N_max=7, Np_WP=12, Nq_WP=12,
                         lab_energies="10"),
}


def pattern_hash(row, col, n):
    """Order-independent 64-bit hash of a sparsity pattern: the wrapping sum of
    a 64-bit mix of each key row * n + col."""
    k = row.astype(np.uint64) * np.uint64(n) + col.astype(np.uint64)
    with np.errstate(over="ignore"):
        k = (k ^ (k >> np.uint64(31))) * np.uint64(0x9E3779B97F4A7C15)
        k = (k ^ (k >> np.uint64(29))) * np.uint64(0xBF58476D1CE4E5B9)
        k = k ^ (k >> np.uint64(32))
        return int(np.sum(k, dtype=np.uint64))


def value_checksums(row, col, val, n):
    """Weighted sums of the values with weights fixed by the position
    (sum v, sum v * w(row, col) with w in [1, 2), sum |v|), compared to a
    relative tolerance."""
    w = 1.0 + ((row.astype(np.float64) * 0.6180339887498949 + col.astype(np.float64) * 0.4142135623730951) % 1.0)
    return np.array([np.sum(val), np.sum(val * w), np.sum(np.abs(val))])


def vector_checksums(G):
    """The same for a complex vector indexed by position."""
    return np.array([np.sum(G), np.sum(G * (1.0 + (np.arange(len(G)) % 7) / 7.0)), np.sum(np.abs(G))])


def run_large(name, opts):
    with tempfile.TemporaryDirectory() as out:
        args = [REF_BIN, "dump", out, "--solver=replica"] + [f"{k}={v}" for k, v in opts.items()]
        subprocess.run(args, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
        meta = read_meta(os.path.join(out, "meta.txt"))
        data = {"opts": np.array([f"{k}={v}" for k, v in opts.items()]), "E_bound": np.array(meta["E_bound"]),
                "T_lab": meta["T_lab"], "E_com": meta["E_com"], "q_idx": meta["q_idx"],
                "n_chn": np.array(len(meta["channels"]))}
        for ch in meta["channels"]:
            c, n = ch["chn"], ch["n"]
            t = f"_c{c}"
            row = np.fromfile(os.path.join(out, f"p123_row{t}.bin"), dtype=np.int32)
            col = np.fromfile(os.path.join(out, f"p123_col{t}.bin"), dtype=np.int32)
            val = np.fromfile(os.path.join(out, f"p123_val{t}.bin"), dtype=np.float64)
            G = np.fromfile(os.path.join(out, f"G{t}.bin"), dtype=np.complex128)
            data["n" + t] = np.array(n)
            data["nnz" + t] = np.array(len(val))
            data["p123_hash" + t] = np.array(pattern_hash(row, col, n), dtype=np.uint64)
            data["p123_sums" + t] = value_checksums(row, col, val, n)
            data["G_sums" + t] = vector_checksums(G)
            data["U" + t] = np.fromfile(os.path.join(out, f"U{t}.bin"), dtype=np.complex128)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print(name, "channels", len(meta["channels"]), "n", [ch["n"] for ch in meta["channels"]],
              "nnz", [ch["nnz"] for ch in meta["channels"]])

# Breakup channels (include_breakup_channels=true, Pade path): per channel the
# cells find_on_shell_bins located (bu_start, bu_cells), their amplitudes
# U_BU[d * num + b], the elastic U of the same run and, for the channels named
# in "tables", the reference's own breakup table text.  Channel 3 of
# lo_j1_J3_n8 is left out: there the reference's Pade loop stops when the
# elastic plus breakup elements converged equal the number of elastic elements
# (CPP/solve_faddeev.cpp:921) with elastic elements still open, and reads an
# unset approximant index for them (the run ends in a segmentation fault).
BREAKUP_CASES = {
    "mt_swave_n16": dict(channels=[0], tables=[0]),
    "lo_j1_J3_n8": dict(channels=[0, 1, 2], tables=[0]),
}


def run_breakup(name, opts, channels, tables):
    data = {"channels": np.array(channels, dtype=np.int32)}
    for c in channels:
        with tempfile.TemporaryDirectory() as out:
            args = [REF_BIN, "dump", out, "--solver=pade", f"--channel={c}", "include_breakup_channels=true"] + \
                [f"{k}={v}" for k, v in opts.items()]
            subprocess.run(args, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                           env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
            t = f"_c{c}"
            data["bu_start" + t] = np.fromfile(os.path.join(out, f"bu_start{t}.bin"), dtype=np.int32)
            data["bu_cells" + t] = np.fromfile(os.path.join(out, f"bu_cells{t}.bin"), dtype=np.int32).reshape(-1, 3)
            data["U_BU" + t] = np.fromfile(os.path.join(out, f"U_BU{t}.bin"), dtype=np.complex128)
            data["U_pade" + t] = np.fromfile(os.path.join(out, f"U{t}.bin"), dtype=np.complex128)
            if c in tables:
                with open(os.path.join(out, f"U_BU{t}.txt")) as f:
                    data["table" + t] = np.array(f.read())
    np.savez_compressed(os.path.join(HERE, f"{name}_breakup.npz"), **data)
    print(name, "breakup channels", channels, "cells", [len(data[f"bu_cells_c{c}"]) for c in channels])


def run_tables(name, opts):
    """The reference's elastic U table (store_U_matrix_elements_txt) of every
    channel of a case, with the U it was written from, as <name>_tables.npz."""
    with tempfile.TemporaryDirectory() as out:
        args = [REF_BIN, "dump", out, "--solver=replica"] + [f"{k}={v}" for k, v in opts.items()]
        subprocess.run(args, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
        meta = read_meta(os.path.join(out, "meta.txt"))
        data = {}
        for ch in meta["channels"]:
            t = f"_c{ch['chn']}"
            data["U" + t] = np.fromfile(os.path.join(out, f"U{t}.bin"), dtype=np.complex128)
            with open(os.path.join(out, f"U_table{t}.txt")) as f:
                data["table" + t] = np.array(f.read())
        np.savez_compressed(os.path.join(HERE, f"{name}_tables.npz"), **data)
        print(name, "tables of", len(meta["channels"]), "channels")


# Custom wave-packet grids (p_grid_type=custom, boundaries read from files,
# CPP/make_wp_states.cpp:46-75, disk_io_routines.cpp:977-994): the boundary
# files' text is kept in the fixture so that a test can write the same files.
CUSTOM_GRID_CASES = {
    "mt_swave_custom_n8": dict(
        opts=dict(potential_model="malfliet_tjon", swave_only="true", isospin_breaking_1S0="false",
                  tensor_force="false", J_2N_max=1, two_J_3N_max=1, Np_WP=8, Nq_WP=8, Nphi=16, Nx=16,
                  lab_energies="13", p_grid_type="custom", q_grid_type="custom"),
        p=[0.0, 8.0, 20.0, 45.0, 90.0, 160.0, 280.0, 500.0, 1000.0],
        q=[0.0, 6.5, 17.25, 35.0, 70.0, 125.5, 210.0, 400.0, 900.0]),
}


def run_custom_grid(name, opts, p, q):
    with tempfile.TemporaryDirectory() as out:
        texts = {}
        for key, vals in (("p", p), ("q", q)):
            texts[key] = "".join(f"{v!r}\n" for v in vals)
            with open(os.path.join(out, f"{key}_grid.dat"), "w") as f:
                f.write(texts[key])
        # not *.txt: the reference's argument parser takes any argument ending in
        # ".txt" for an input-list file (CPP/set_run_parameters.cpp:641-644)
        args = [REF_BIN, "dump", out, "--solver=replica", f"p_grid_filename={out}/p_grid.dat",
                f"q_grid_filename={out}/q_grid.dat"] + [f"{k}={v}" for k, v in opts.items()]
        subprocess.run(args, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
        meta = read_meta(os.path.join(out, "meta.txt"))

        def rd(fname, dtype):
            return np.fromfile(os.path.join(out, fname + ".bin"), dtype=dtype)

        data = {"opts": np.array([f"{k}={v}" for k, v in opts.items()]), "p_grid_text": np.array(texts["p"]),
                "q_grid_text": np.array(texts["q"]), "E_bound": np.array(meta["E_bound"]), "T_lab": meta["T_lab"],
                "E_com": meta["E_com"], "q_idx": meta["q_idx"], "p_WP": rd("p_WP", np.float64),
                "q_WP": rd("q_WP", np.float64), "V_unco": rd("V_unco", np.float64),
                "C_unco": rd("C_unco", np.float64), "e_unco": rd("e_unco", np.float64),
                "n_chn": np.array(len(meta["channels"]))}
        for ch in meta["channels"]:
            t = f"_c{ch['chn']}"
            data["pw" + t] = rd("pw" + t, np.int32).reshape(-1, 9)
            data["p123_row" + t] = rd("p123_row" + t, np.int32)
            data["p123_col" + t] = rd("p123_col" + t, np.int32)
            data["p123_val" + t] = rd("p123_val" + t, np.float64)
            data["U" + t] = rd("U" + t, np.complex128)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print(name, "custom grids, channels", len(meta["channels"]))


if __name__ == "__main__":
    if not os.path.exists(REF_BIN):
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` first")
    if "--large" in sys.argv:
        for name, opts in LARGE_CASES.items():
            run_large(name, opts)
        sys.exit(0)
    if "--tables" in sys.argv:
        for name in ("mt_swave_n16", "lo_j1_J3_n8"):
            run_tables(name, CASES[name])
        sys.exit(0)
    if "--custom-grid" in sys.argv:
        for name, case in CUSTOM_GRID_CASES.items():
            run_custom_grid(name, **case)
        sys.exit(0)
    if "--breakup" in sys.argv:
        for name, sel in BREAKUP_CASES.items():
            run_breakup(name, CASES[name], **sel)
        sys.exit(0)
    only_pade = "--pade" in sys.argv
    for name, opts in CASES.items():
        if not only_pade:
            run_case(name, opts)
        if name in PADE_CASES:
            run_pade(name, opts)
