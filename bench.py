#!/usr/bin/env python
"""Throughput of the WPCD elastic Faddeev solve (P123 -> A -> LU -> refined U).

Workload (default): the configuration the headline metric is quoted on --
two-body j <= 3, all 3N channels J^pi = 1/2+- .. 7/2+-, Np_WP = Nq_WP = 30,
T_lab = 10 MeV (two on-shell q bins), with the chiral LO one-pion-exchange
potential standing in for N3LO-Idaho (which exists only as Fortran in the
reference; the solve cost depends on the shapes only).  Eight channels,
n = 24,300 .. 56,700.  One step = both on-shell energies for all channels:
A = C^T (2 P123)(V C) built from the resident P123, 1 - A G_E formed and
LU-factorised per energy, on-shell columns solved and refined to 1e-12.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); rank r solves its own pair of
on-shell energies (T_lab = 10 + 6 r MeV) for all channels -- independent
replicas over the energy scan, no collective on the data path (weak scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "tic-tac_b200", "python"))

CONFIGS = {
    # the metric's configuration (see module docstring)
    "j3_J7_n30": dict(potential_model="LO_internal", J_2N_max=3, two_J_3N_max=7, Np_WP=30, Nq_WP=30),
    # same basis at Np=Nq=12 (largest channel n = 9072, ~0.7 GB per matrix): profiler captures
    "j3_J7_n12": dict(potential_model="LO_internal", J_2N_max=3, two_J_3N_max=7, Np_WP=12, Nq_WP=12),
    # small case for quick checks of this script
    "j1_J3_n12": dict(potential_model="LO_internal", J_2N_max=1, two_J_3N_max=3, Np_WP=12, Nq_WP=12),
}
METRIC = "energies/sec, mixed+refined vs FP64 on B200 at <=1e-10 rel err in on-shell U"


def load_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return (d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0),
                "measured")
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) >= 9:
                for k, nm in enumerate(names):
                    if s[5 + k].lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def step_flops(ns, nE):
    return sum(nE * 8.0 / 3.0 * float(n) ** 3 for n in ns)


# DRAM traffic of the tensor-core update per algorithmic byte (C read + written
# as complex64, L and U panels read once): dram__bytes_read.sum +
# dram__bytes_write.sum over 16 M N + 8 (M + N) K for two launches (M = N = 7536
# and 7280, K = 256) of the n = 9072 capture in profiles/k_lu_update_tc_n9072.md
# (926.4 / 939.5 MB and 861.2 / 877.8 MB); traffic grows with the tile count, so
# the ratio scales the bench's mean launch to a per-launch traffic figure.
TC_TRAFFIC_PER_ALGO_BYTE = 0.984


def roofline_of(kern, timed_ms, ms_step, ns, nE):
    """Roofline of the dominant kernel class over the timed region: algorithmic
    flops (or bytes) per launch over the CUDA-event time per launch."""
    hbm, tf_burst, tf_sust, peak_kind = load_peaks()
    kernels = {}
    for name, k in kern.items():
        if k["launches"]:
            kernels[name] = {"launches": k["launches"], "ms": round(k["ms"], 3),
                             "share_of_timed": round(k["ms"] / timed_ms, 4),
                             "tflops": round(k["flops"] / (k["ms"] * 1e-3) / 1e12, 2) if k["ms"] else None,
                             "gbs": round(k["bytes"] / (k["ms"] * 1e-3) / 1e9, 1) if k["ms"] else None}
    dom = max(kern, key=lambda nm: kern[nm]["ms"])
    k = kern[dom]
    if k["launches"] == 0:
        return None, kernels
    per_launch_s = k["ms"] * 1e-3 / k["launches"]
    if dom == "tc_update":
        # complex64 product in BF16x3: 3 bf16 tensor products per fp32-accurate
        # product, so the tensor roofline for algorithmic flops is peak / 3;
        # the kernel runs inside a seconds-long step -> sustained figure
        achieved = k["flops"] / k["launches"] / per_launch_s / 1e12
        peak = tf_sust / 3.0
        traffic = None
        if TC_TRAFFIC_PER_ALGO_BYTE:
            traffic = TC_TRAFFIC_PER_ALGO_BYTE * k["bytes"] / k["launches"]
        roof = {"bound": "tensor", "achieved": round(achieved, 2), "peak": round(peak, 1), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": "k_lu_update_tc (complex64 trailing update C -= L U, BF16x3 on tcgen05)",
                "flops_per_launch": k["flops"] / k["launches"], "ms_per_launch": round(per_launch_s * 1e3, 3),
                "peak_source": f"{peak_kind} bf16_tflops_sustained {tf_sust} / 3 (BF16x3 split factor)"}
    else:
        achieved = k["bytes"] / k["launches"] / per_launch_s / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "traffic": None, "kernel": dom,
                "peak_source": f"{peak_kind} hbm_gbs"}
    roof["step_lu_tflops"] = round(step_flops(ns, nE) / (ms_step * 1e-3) / 1e12, 2)
    return roof, kernels


def run_ours(args, world, rank, local, pg):
    import tictac_b200 as tt
    os.environ.setdefault("CUDA_VISIBLE_DEVICES", os.environ.get("CUDA_VISIBLE_DEVICES", ""))
    cfg = dict(CONFIGS[args.config])
    cfg["lab_energies"] = str(10.0 + 6.0 * rank)
    prec = tt.PRECISION_MIXED if args.precision == "mixed" else tt.PRECISION_FP64
    t_setup = time.perf_counter()
    run = tt.Run(**cfg)
    chans = [int(c) for c in args.channels.split(",")] if args.channels else list(range(run.num_channels))
    nch = len(chans)
    infos = [run.channel_info(c) for c in chans]
    T_lab, E_com, q_idx = run.energies()
    nE = len(T_lab)
    nnz = [run.build_P123(c) for c in chans]  # resident for the whole run
    t_setup = time.perf_counter() - t_setup

    def one_step():
        Us = []
        for c in chans:
            run.build_A(c)
            run.build_resolvent(c)
            U, rep = run.solve(c, prec)
            Us.append(U)
            run.release_A(c)
        return Us

    for _ in range(args.warmup):
        one_step()
    barrier(pg)
    times = []
    launches0 = tt.kernel_launches()
    tt.profile_begin()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            run.timer_start()
            one_step()
            times.append(run.timer_stop())
    kern = tt.profile_end()
    launches = tt.kernel_launches() - launches0
    barrier(pg)
    ms_step = allreduce_max(pg, float(np.mean(times)))
    energies_per_step = nE * world
    value = energies_per_step / (ms_step * 1e-3)
    roofline, kernels = roofline_of(kern, float(np.sum(times)), ms_step, [i["n"] for i in infos], nE)

    # end to end through the drop-in C-ABI call with host buffers
    e2e = None
    if args.e2e_steps > 0:
        host = []
        Np = Nq = cfg["Np_WP"]
        e_unco = run.host_array(7)
        e_coup = run.host_array(8)
        C_unco = run.host_array(5)
        C_coup = run.host_array(6)
        V_unco = run.host_array(3)
        V_coup = run.host_array(4)
        q_WP = run.host_array(2)
        n_unco = len(e_unco) // (Np + 1)
        n_coup = len(e_coup) // (2 * (Np + 1))
        swp = tt.SWP(Np, Nq, n_unco, n_coup, run.E_bound, e_unco, e_coup, C_unco, C_coup, q_WP)
        for i, c in enumerate(chans):
            rowptr, col, val = run.P123_csr(c, nnz[i])
            n = infos[i]["n"]
            rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rowptr))
            order = np.lexsort((rows, col))
            colptr = np.zeros(n + 1, dtype=np.uint64)
            np.add.at(colptr, col + 1, 1)
            colptr = np.cumsum(colptr).astype(np.uint64)
            run.build_resolvent(c)
            G = run.G(c).reshape(-1)
            pwt = run.host_array(0, c).reshape(-1, 9)
            deut = [a for a in range(len(pwt)) if tuple(pwt[a, :4]) == (0, 1, 1, 0)]
            host.append((G, val[order].copy(), rows[order].copy(), colptr, tt.PW(pwt, cfg["J_2N_max"]), deut))
            run.release(c)
        # inputs live in pinned host memory, as a caller streaming channels would keep them
        import torch

        pinned = []

        def pin(a):
            a = np.ascontiguousarray(a)
            t = torch.empty(max(1, a.nbytes), dtype=torch.uint8, pin_memory=True)
            v = t.numpy()[:a.nbytes].view(a.dtype).reshape(a.shape)
            v[...] = a
            pinned.append(t)
            return v

        host = [tuple(pin(x) if isinstance(x, np.ndarray) else x for x in h) for h in host]
        V_unco, V_coup = pin(V_unco), pin(V_coup)
        h2d = sum(h[0].nbytes + h[1].nbytes + h[2].nbytes + h[3].nbytes for h in host) + \
            nch * (V_unco.nbytes + V_coup.nbytes + C_unco.nbytes + C_coup.nbytes + e_unco.nbytes + e_coup.nbytes)
        d2h = sum(16 * nE * len(h[5]) ** 2 for h in host)

        def e2e_step():
            for (G, v, r, cp, pw, deut) in host:
                tt.solve_faddeev(G, v, r, cp, V_unco, V_coup, swp, q_idx, deut, pw, precision=prec)

        e2e_step()
        barrier(pg)
        te = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            e2e_step()
            te.append(time.perf_counter() - t0)
        t_e2e = allreduce_max(pg, float(np.mean(te)))
        e2e = {"value": round(energies_per_step / t_e2e, 6), "unit": "energies/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "timer": "host perf_counter around the synchronous C-ABI call"}
    # the metric's comparison: mixed+refined against the plain FP64 solve on the
    # smallest channel (same inputs, same energies), outside the timed region
    fp64 = None
    if args.fp64_check and prec == tt.PRECISION_MIXED:
        i = min(range(nch), key=lambda k: infos[k]["n"])
        c = chans[i]
        run.build_A(c)
        run.build_resolvent(c)
        Um, rm = run.solve(c, tt.PRECISION_MIXED)
        U64, r64 = run.solve(c, tt.PRECISION_FP64)
        t_m = rm["ms_form"] + rm["ms_factor"] + rm["ms_solve"] + rm["ms_refine"]
        t_64 = r64["ms_form"] + r64["ms_factor"] + r64["ms_solve"] + r64["ms_refine"]
        fp64 = {"channel": c, "n": infos[i]["n"], "mixed_ms": round(t_m, 1), "fp64_ms": round(t_64, 1),
                "speedup": round(t_64 / t_m, 2), "refine_iters": rm["refine_iters"],
                "max_rel_diff_U": float(np.max(np.abs(Um - U64)) / np.max(np.abs(U64)))}
        # adjoint: dU/dLEC for the potential's contact constants on the same channel
        nl = len(run.lecs())
        if nl:
            dV = [run.lec_derivative(k) for k in range(nl)]
            Ua, dU, ra = run.solve_adjoint(c, np.stack([d[0] for d in dV]), np.stack([d[1] for d in dV]),
                                           tt.PRECISION_MIXED)
            t_f = ra["ms_form"] + ra["ms_factor"] + ra["ms_solve"] + ra["ms_refine"]
            fp64["adjoint"] = {"n_theta": nl, "forward_ms": round(t_f, 1), "adjoint_ms": round(ra["ms_adjoint"], 1),
                               "adjoint_over_forward": round(ra["ms_adjoint"] / t_f, 3),
                               "adjoint_refine_iters": ra["adjoint_refine_iters"],
                               "max_abs_dU_dLEC": float(np.max(np.abs(dU)))}
        # the reference's production path: Pade-resummed Neumann series (about 1e-6)
        Up, rpd = run.solve(c, tt.PRECISION_PADE)
        fp64["pade"] = {"ms": round(rpd["ms_solve"], 1), "order": rpd["refine_iters"],
                        "max_rel_diff_U_vs_fp64": float(np.max(np.abs(Up - U64)) / np.max(np.abs(U64)))}
        run.release_A(c)
    return dict(value=value, ms_step=ms_step, clocks=clk.summary(), roofline=roofline, kernels=kernels, e2e=e2e,
                infos=infos, nE=nE, nnz=nnz, t_setup=t_setup, times=times, launches=launches, fp64=fp64)


REF_SAMPLE_N = 12


def reference_sample(args, sample_N=REF_SAMPLE_N, channel=None):
    """Time the reference's own dense LAPACK solve (oracle/_ref/tictac_ref,
    OpenMP + OpenBLAS on all host cores) on one channel of the same physics at
    Np_WP = Nq_WP = sample_N and scale to the workload by n^3."""
    binp = os.path.join(HERE, "oracle", "_ref", "tictac_ref")
    if not os.path.exists(binp):
        return None, "oracle/_ref/tictac_ref not built"
    cfg = dict(CONFIGS[args.config])
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as out:
        opts = [f"{k}={v}" for k, v in cfg.items() if k not in ("Np_WP", "Nq_WP")]
        opts += [f"Np_WP={sample_N}", f"Nq_WP={sample_N}", "lab_energies=10"]
        ch = channel if channel is not None else 0
        cmd = [binp, "time", out, f"--channel={ch}"] + opts
        t0 = time.perf_counter()
        subprocess.run(cmd, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(cores)), timeout=900)
        wall = time.perf_counter() - t0
        t = {}
        with open(os.path.join(out, "meta.txt")) as f:
            for line in f:
                tok = line.split()
                if tok and tok[0] == "timing":
                    t = dict(zip(tok[1::2], tok[2::2]))
                if tok and tok[0] == "chn":
                    meta = dict(zip(tok[::2], tok[1::2]))
    n_s = int(t["n"])
    nE = int(meta["nE"])
    per_energy = (float(t["t_A"]) + float(t["t_getrf_getrs"])) / nE
    return dict(n_sample=n_s, per_energy_s=per_energy, t_A=float(t["t_A"]) / nE,
                t_lu=float(t["t_getrf_getrs"]) / nE, t_fair=float(t["t_fair"]) / nE,
                t_p123=float(meta["t_p123"]), cores=cores, wall=wall), None


def cpu_phases(ref, infos):
    """Per-phase seconds of the reference sample (per energy, P123 once per
    channel) and the energies/s a fairer CPU path would reach: the same A
    columns, then zgetrf + zgetrs with only the nd on-shell right-hand sides
    instead of nrhs = n, extrapolated by n^3 like the value."""
    fair = 1.0 / sum((ref["t_A"] + ref["t_fair"]) * (i["n"] / ref["n_sample"]) ** 3 for i in infos)
    return {"sample_n": ref["n_sample"], "p123_s": round(ref["t_p123"], 4), "A_columns_s": round(ref["t_A"], 4),
            "zgetrf_zgetrs_nrhs_n_s": round(ref["t_lu"], 4), "zgetrf_zgetrs_nrhs_nd_s": round(ref["t_fair"], 4),
            "fair_value": fair}


def cpu_value_for(infos, ref):
    # seconds per energy for all channels of the workload, scaled by n^3
    s = sum(ref["per_energy_s"] * (i["n"] / ref["n_sample"]) ** 3 for i in infos)
    return 1.0 / s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=list(CONFIGS), default="j3_J7_n30")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-check", type=int, default=1, help="time FP64 vs mixed on the smallest channel")
    ap.add_argument("--channels", default="", help="comma list of channel indices to step (default: all)")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    cfg = CONFIGS[args.config]
    config = {"workload": f"{args.config}: LO-OPEP (stands in for N3LO-Idaho), j<=3, J<=7/2 both parities, "
                          f"Np=Nq={cfg['Np_WP']}, T_lab=10 MeV (rank r: 10+6r MeV)",
              "channels_per_step": None, "energies_per_rank": None, "parallelism": f"replicas x{world}",
              "l2": "inputs larger than L2 (A is 25.7 GB for the largest channel)"}

    if args.impl == "reference":
        if rank != 0:
            return
        import tictac_b200 as tt
        run = tt.Run(**dict(cfg, lab_energies="10"))
        infos = [run.channel_info(c) for c in range(run.num_channels)]
        nE = len(run.energies()[0])
        run.close()
        config["channels_per_step"] = len(infos)
        config["energies_per_rank"] = nE
        config["n_per_channel"] = [i["n"] for i in infos]
        samples = []
        for _ in range(args.warmup + max(1, args.steps)):
            r2, why = reference_sample(args)
            if r2 is None:
                print(json.dumps({"impl": "reference", "unavailable": why}))
                return
            samples.append(r2)
        ref = dict(samples[-1])
        for k in ("per_energy_s", "t_A", "t_lu", "t_fair"):
            ref[k] = float(np.mean([x[k] for x in samples[args.warmup:]]))
        v = cpu_value_for(infos, ref)
        sample = (f"reference dense LAPACK solve (A columns + zgetrf + zgetrs nrhs=n) of channel 0 at "
                  f"Np=Nq={REF_SAMPLE_N} (n={ref['n_sample']}), T_lab=10 MeV, {ref['cores']} threads, "
                  f"extrapolated by n^3 to every channel of the workload")
        print(json.dumps({"metric": METRIC, "value": v, "unit": "energies/s", "impl": "reference", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_step": nE / v * 1e3,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
                          "data": "synthetic (seeded LO potential)", "config": config,
                          "cpu_baseline": {"value": v, "unit": "energies/s", "cores": ref["cores"],
                                           "kind": "reference", "sample": sample,
                                           "phases": cpu_phases(ref, infos)},
                          "e2e": {"value": v, "unit": "energies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    r = run_ours(args, world, rank, local, pg)
    if rank == 0:
        config["channels_per_step"] = len(r["infos"])
        config["energies_per_rank"] = r["nE"]
        config["n_per_channel"] = [i["n"] for i in r["infos"]]
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            ref, why = reference_sample(args)
            if ref is not None:
                v = cpu_value_for(r["infos"], ref)
                cpu = {"value": v, "unit": "energies/s", "cores": ref["cores"], "kind": "reference",
                       "sample": f"reference dense LAPACK solve of channel 0 at Np=Nq={REF_SAMPLE_N} (n={ref['n_sample']}), "
                                 f"scaled by n^3 to all {len(r['infos'])} channels",
                       "phases": cpu_phases(ref, r["infos"])}
        out = {"metric": METRIC, "value": round(r["value"], 6), "unit": "energies/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_step": round(r["ms_step"], 3),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "complex64 LU (BF16x3 tcgen05) + FP64 refinement" if args.precision == "mixed" else "complex128",
               "data": "synthetic (chiral LO potential on the reference's default Chebyshev WP grid)",
               "config": config, "clocks": r["clocks"], "roofline": r["roofline"], "cpu_baseline": cpu,
               "e2e": r["e2e"], "gpu_launches": int(r["launches"]),
               "channel_solves_per_s": round(len(r["infos"]) * r["nE"] * world / (r["ms_step"] * 1e-3), 4),
               "kernels": r["kernels"], "fp64_comparison": r["fp64"], "setup_s": round(r["t_setup"], 3)}
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
