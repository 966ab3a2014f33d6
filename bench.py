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

Multi-GPU: one process per GPU (torchrun).  On N GPUs the workload is a scan
of N lab energies with 2N distinct on-shell bins; its (channel, energies)
items (each channel's bins in pairs, weighted by n^3) are assigned to the
ranks longest-processing-time first, each rank builds P123 and A only for the
channels it owns, and the U arrays are gathered on rank 0 in the reference's
layout.  No collective on the data path (weak scaling: the items grow with N).

--impl reference times the reference's own dense LAPACK path (the compiled
reference, oracle/_ref/tictac_ref) on the host cores; it loads nothing of this
repository's library.
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
    # the batched energy scan: j <= 2, J <= 5/2 (six channels, n = 10,944 .. 20,160), Np = Nq = 24,
    # 64 lab energies drawn uniformly in 1-200 MeV (seed 2024) collapsing to their distinct on-shell
    # bins; each channel's bins factored four at a time; LO-OPEP stands in for Nijmegen-I
    "j2_J5_n24_scan64": dict(potential_model="LO_internal", J_2N_max=2, two_J_3N_max=5, Np_WP=24, Nq_WP=24),
}
# lab energies of the scan configurations: (count, low MeV, high MeV, seed)
SCANS = {"j2_J5_n24_scan64": (64, 1.0, 200.0, 2024)}
# phase times of a solve report (build A, form 1 - A G, factor, substitute, refine)
PHASES = ("ms_A", "ms_form", "ms_factor", "ms_solve", "ms_refine")
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
        pw = [float(s[3]) for s in self.samples if len(s) >= 9 and s[3].replace(".", "").isdigit()]
        capped = [s[8].lower() == "active" for s in self.samples if len(s) >= 9]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "sm_mhz_p10_p90": [float(np.percentile(sm, 10)), float(np.percentile(sm, 90))] if sm else None,
                "power_w_median": float(np.median(pw)) if pw else None,
                "power_cap_share": round(sum(capped) / len(capped), 3) if capped else None}


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


# DRAM traffic of the tensor-core update (CTA pairs, TF32) per algorithmic byte
# (C read + written as complex64, L and U panels read once):
# dram__bytes_read.sum + dram__bytes_write.sum over 16 M N + 8 (M + N) K for
# the first trailing update of the n = 9072 channel (M = N = 8560, K = 512) in
# an ncu capture: (974.5 + 560.5) MB / 1242.5 MB; traffic grows with the tile
# count, so the ratio scales the bench's mean launch to a per-launch figure.
TC_TRAFFIC_PER_ALGO_BYTE = 1.235


# Tensor work per algorithmic complex flop of each product and the kernel
# that runs it: BF16x3 takes 3 bf16 products; TF32 one product at half the
# bf16 rate
PRODUCTS = {
    "bf16x3": (3.0, "k_lu_update_tc2<BF16X3> (complex64 C -= L U, real-row form, BF16x3 on tcgen05)"),
    "tf32": (2.0, "k_lu_update_tc2<TF32> (complex64 C -= L U, real-row form, TF32 on tcgen05)"),
    "bf16x3_n128": (3.0, "k_lu_update_tc (complex64 C -= L U, four real products, BF16x3 on tcgen05)"),
}


def roofline_of(kern, timed_ms, ms_step, ns, nE, product="bf16x3", pairs=True):
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
    # launch gaps and kernels outside the classes: the rest of the timed region
    kernels["unattributed"] = {"share_of_timed": round(1.0 - sum(k["ms"] for k in kern.values()) / timed_ms, 4)}
    if ms_step != timed_ms:
        # the breakdown step records an event pair around every launch class, which
        # slows the host's launch stream; against a plain timed step:
        kernels["unattributed"]["share_of_plain_step"] = round(
            max(0.0, 1.0 - sum(k["ms"] for k in kern.values()) / ms_step), 4)
    dom = max(kern, key=lambda nm: kern[nm]["ms"])
    k = kern[dom]
    if k["launches"] == 0:
        return None, kernels
    per_launch_s = k["ms"] * 1e-3 / k["launches"]
    if dom == "tc_update":
        # the tensor roofline for algorithmic flops is the bf16 peak over the
        # product's cost factor; the kernel runs inside a seconds-long step,
        # so the sustained figure
        factor, kname = PRODUCTS[product]
        if pairs:
            kname = kname.replace("k_lu_update_tc2<", "k_lu_update_tc2_pair<").replace(
                " on tcgen05)", " on tcgen05, CTA pairs)")
        achieved = k["flops"] / k["launches"] / per_launch_s / 1e12
        peak = tf_sust / factor
        traffic = None
        if TC_TRAFFIC_PER_ALGO_BYTE:
            traffic = TC_TRAFFIC_PER_ALGO_BYTE * k["bytes"] / k["launches"]
        roof = {"bound": "tensor", "achieved": round(achieved, 2), "peak": round(peak, 1), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": kname,
                "flops_per_launch": k["flops"] / k["launches"], "ms_per_launch": round(per_launch_s * 1e3, 3),
                "peak_source": f"{peak_kind} bf16_tflops_sustained {tf_sust} / {factor:g} ({product} product)"}
    else:
        achieved = k["bytes"] / k["launches"] / per_launch_s / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "traffic": None, "kernel": dom,
                "peak_source": f"{peak_kind} hbm_gbs"}
    roof["step_lu_tflops"] = round(step_flops(ns, nE) / (ms_step * 1e-3) / 1e12, 2)
    return roof, kernels


def scan_lab_energies(cfg, world, name=""):
    """Lab energies of the workload at `world` GPUs: T_lab = 10 MeV (two
    on-shell bins) on one GPU; on N GPUs the scan continues with N - 1 further
    lab energies placed between the next pairs of bin mid-points, so every lab
    energy brings two new on-shell bins (2N bins in all) and the (channel,
    energy) items grow with N."""
    if name in SCANS:
        count, lo, hi, seed = SCANS[name]
        return sorted(float(x) for x in np.random.default_rng(seed).uniform(lo, hi, count))
    if world == 1:
        return [10.0]
    import tictac_b200 as tt
    probe = tt.Run(**dict(cfg, lab_energies=",".join(str(x) for x in np.arange(1.0, 400.0, 0.5))))
    T, _, _ = probe.energies()
    probe.close()
    T = list(T)
    k0 = next(i for i in range(len(T) - 1) if T[i] <= 10.0 <= T[i + 1])
    if k0 + 2 * world > len(T):
        raise SystemExit(f"the q grid has no {2 * world} on-shell bins above 10 MeV")
    return [10.0] + [0.5 * (T[k0 + 2 * r] + T[k0 + 2 * r + 1]) for r in range(1, world)]


def elem_rel(a, b, floor=1e-6):
    """Relative error of every element of a against b (elements below `floor`
    of max|b| are zero by symmetry up to rounding and measured against it)."""
    a, b = np.asarray(a).reshape(-1), np.asarray(b).reshape(-1)
    if b.size == 0:
        return 0.0
    den = np.maximum(np.abs(b), floor * float(np.max(np.abs(b))))
    return float(np.max(np.abs(a - b) / np.where(den > 0, den, 1e-300)))


def run_ours(args, world, rank, local, pg):
    import tictac_b200 as tt
    from tictac_b200 import shard
    cfg = dict(CONFIGS[args.config])
    lab = scan_lab_energies(cfg, world, args.config)
    cfg["lab_energies"] = ",".join(f"{x:.12g}" for x in lab)
    cfg["tc_product"] = args.tc_product
    cfg["panel_order"] = args.panel_order
    cfg["panel_width"] = args.panel_width
    cfg["inverse_block"] = args.inverse_block
    cfg["cta_pairs"] = "true" if args.cta_pairs else "false"
    cfg["mid_panel"] = args.mid_panel
    prec = tt.PRECISION_MIXED if args.precision == "mixed" else tt.PRECISION_FP64
    t_setup = time.perf_counter()
    run = tt.Run(**cfg)
    all_chans = [int(c) for c in args.channels.split(",")] if args.channels else list(range(run.num_channels))
    infos_all = [run.channel_info(c) for c in range(run.num_channels)]
    T_lab, E_com, q_idx = run.energies()
    nE = len(T_lab)
    # (channel, energies) items over the ranks, longest processing time first
    group = 4 if args.config in SCANS else 2  # energies factored together per channel
    plans = shard.plan([infos_all[c]["n"] for c in all_chans], nE, world, group=group)
    mine = {all_chans[i]: js for i, js in plans[rank].items()}
    infos = [infos_all[c] for c in all_chans]
    # P123 of this rank's channels, built once on the device and resident for the
    # whole run (setup, not part of a step): device time per channel
    nnz, p123_ms = {}, {}
    for c in mine:
        run.timer_start()
        nnz[c] = run.build_P123(c)
        p123_ms[c] = run.timer_stop()
    p123_stage = {"ms_total": round(sum(p123_ms.values()), 1), "nnz_total": int(sum(nnz.values())),
                  "per_channel": {str(c): {"n": infos_all[c]["n"], "nnz": int(nnz[c]), "ms": round(p123_ms[c], 1)}
                                  for c in mine}}
    t_setup = time.perf_counter() - t_setup

    phases = {}  # per channel: the solve report's phase times of the latest step

    def one_step():
        Us = {}
        for c, js in mine.items():
            ms_A = run.build_A(c)
            U, rep = run.solve_energies(c, js, prec)
            Us[c] = (js, U)
            phases[c] = {k: round(rep[k], 1) for k in PHASES}
            phases[c]["ms_A"] = round(ms_A, 1)  # host clock around the A build, allocation included
            run.release_A(c)
        return Us

    for _ in range(args.warmup):
        one_step()
    barrier(pg)
    times = []
    launches0 = tt.kernel_launches()
    # the timed steps record events only around the roofline kernel's launches
    tt.profile_begin(["tc_update"])
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            run.timer_start()
            Us = one_step()
            times.append(run.timer_stop())
    step_phases = {str(c): dict(v) for c, v in phases.items()}
    kern = tt.profile_end()
    launches = tt.kernel_launches() - launches0
    barrier(pg)
    ms_step = allreduce_max(pg, float(np.mean(times)))
    energies_per_step = nE  # every channel at every on-shell energy of the scan, over all ranks
    value = energies_per_step / (ms_step * 1e-3)
    items = [infos_all[c]["n"] for c, js in mine.items() for _ in js]
    roofline, _ = roofline_of(kern, float(np.sum(times)), float(np.mean(times)), items, 1, args.tc_product,
                              bool(args.cta_pairs))
    # breakdown: one more step with every kernel class timed (not part of the value)
    kernels = None
    if args.breakdown:
        tt.profile_begin()
        run.timer_start()
        one_step()
        t_bd = run.timer_stop()
        _, kernels = roofline_of(tt.profile_end(), t_bd, float(np.mean(times)), items, 1, args.tc_product,
                                 bool(args.cta_pairs))
        kernels["step_ms"] = round(t_bd, 1)
        kernels["per_channel_phases_ms"] = {str(c): phases[c] for c in mine}
    # U of every (channel, energy) gathered on rank 0 in the reference's layout
    gathered = shard.gather_to_rank0(pg, Us)
    U_all = None
    if rank == 0:
        U_all = shard.assemble_U(gathered, [infos_all[c]["n_deuteron"] if c in all_chans else 0
                                            for c in range(run.num_channels)], nE)

    # end to end through the drop-in C-ABI call with host buffers, this rank's items
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
        for c, js in mine.items():
            rowptr, col, val = run.P123_csr(c, nnz[c])
            n = infos_all[c]["n"]
            rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rowptr))
            order = np.lexsort((rows, col))
            colptr = np.zeros(n + 1, dtype=np.uint64)
            np.add.at(colptr, col + 1, 1)
            colptr = np.cumsum(colptr).astype(np.uint64)
            run.build_resolvent(c)
            G = run.G(c).reshape(nE, n)[js].reshape(-1)
            pwt = run.host_array(0, c).reshape(-1, 9)
            deut = [a for a in range(len(pwt)) if tuple(pwt[a, :4]) == (0, 1, 1, 0)]
            host.append((G, val[order].copy(), rows[order].copy(), colptr, tt.PW(pwt, cfg["J_2N_max"]), deut,
                         q_idx[js]))
            run.release_A(c)  # A and G; P123 stays resident for the FP64 comparison below
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
            len(host) * (V_unco.nbytes + V_coup.nbytes + C_unco.nbytes + C_coup.nbytes + e_unco.nbytes +
                         e_coup.nbytes)
        d2h = sum(16 * len(h[6]) * len(h[5]) ** 2 for h in host)

        def e2e_step():
            for (G, v, r, cp, pw, deut, qs) in host:
                tt.solve_faddeev(G, v, r, cp, V_unco, V_coup, swp, qs, deut, pw, precision=prec)

        e2e_step()
        barrier(pg)
        te = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            e2e_step()
            te.append(time.perf_counter() - t0)
        t_e2e = allreduce_max(pg, float(np.mean(te)))
        e2e = {"value": round(energies_per_step / t_e2e, 6), "unit": "energies/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "timer": "host perf_counter around the synchronous C-ABI calls"}
    # the metric's comparison: the same step in FP64 against the mixed+refined
    # solve, every channel (or the smallest with --fp64-check 1), with the
    # relative error of every on-shell U element
    fp64 = None
    if args.fp64_check and prec == tt.PRECISION_MIXED and world == 1:
        cmp_chans = all_chans if args.fp64_check >= 2 else [min(all_chans, key=lambda c: infos_all[c]["n"])]
        rows, t_mix, t_64, worst = [], 0.0, 0.0, 0.0
        for c in cmp_chans:
            cache0 = tt.cached_device_memory()
            run.timer_start()
            h0 = time.perf_counter()
            ms_A = run.build_A(c)
            h1 = time.perf_counter()
            run.build_resolvent(c)
            h2 = time.perf_counter()
            Um, rm = run.solve(c, tt.PRECISION_MIXED)
            h3 = time.perf_counter()
            tm = run.timer_stop()
            host_ms = {"build_A": round(ms_A, 1), "build_A_call": round(1e3 * (h1 - h0), 1),
                       "resolvent": round(1e3 * (h2 - h1), 1), "solve_call": round(1e3 * (h3 - h2), 1),
                       "cached_gb_before": round(cache0 / 1e9, 1)}
            run.timer_start()
            run.build_A(c)
            run.build_resolvent(c)
            U64, r64 = run.solve(c, tt.PRECISION_FP64)
            t64 = run.timer_stop()
            err = elem_rel(Um, U64)
            worst = max(worst, err)
            t_mix += tm
            t_64 += t64
            rows.append({"channel": c, "n": infos_all[c]["n"], "mixed_ms": round(tm, 1), "fp64_ms": round(t64, 1),
                         "speedup": round(t64 / tm, 2), "refine_iters": rm["refine_iters"],
                         "final_correction": rm["final_correction"], "max_elem_rel_err_U": err,
                         "mixed_phases_ms": {k: round(rm[k], 1) for k in PHASES},
                         "mixed_host_ms": host_ms,
                         "fp64_lu_tflops": round(8.0 / 3.0 * infos_all[c]["n"] ** 3 * nE / (r64["ms_factor"] * 1e-3)
                                                 / 1e12, 2)})
            if c != cmp_chans[0]:
                run.release_A(c)
        fp64 = {"channels": len(cmp_chans), "mixed_ms": round(t_mix, 1), "fp64_ms": round(t_64, 1),
                "fp64_value": nE / (t_64 * 1e-3) if len(cmp_chans) == len(all_chans) else None,
                "speedup": round(t_64 / t_mix, 2), "max_elem_rel_err_U": worst, "per_channel": rows}
        c = cmp_chans[0]
        # adjoint: dU/dLEC for the potential's contact constants on the first channel
        nl = len(run.lecs())
        if nl:
            dV = [run.lec_derivative(k) for k in range(nl)]
            Ua, dU, ra = run.solve_adjoint(c, np.stack([d[0] for d in dV]), np.stack([d[1] for d in dV]),
                                           tt.PRECISION_MIXED)
            t_f = ra["ms_form"] + ra["ms_factor"] + ra["ms_solve"] + ra["ms_refine"]
            fp64["adjoint"] = {"channel": c, "n_theta": nl, "forward_ms": round(t_f, 1),
                               "adjoint_ms": round(ra["ms_adjoint"], 1),
                               "adjoint_over_forward": round(ra["ms_adjoint"] / t_f, 3),
                               "adjoint_refine_iters": ra["adjoint_refine_iters"],
                               "max_abs_dU_dLEC": float(np.max(np.abs(dU)))}
        # the reference's production path: Pade-resummed Neumann series (about 1e-6)
        Up, rpd = run.solve(c, tt.PRECISION_PADE)
        U64, _ = run.solve(c, tt.PRECISION_FP64)
        fp64["pade"] = {"channel": c, "ms": round(rpd["ms_solve"], 1), "order": rpd["refine_iters"],
                        "max_rel_diff_U_vs_fp64": float(np.max(np.abs(Up - U64)) / np.max(np.abs(U64)))}
        run.release_A(c)
    return dict(value=value, ms_step=ms_step, clocks=clk.summary(), roofline=roofline, kernels=kernels, e2e=e2e,
                infos=infos, nE=nE, nnz=nnz, t_setup=t_setup, times=times, launches=launches, fp64=fp64,
                lab=lab, plan=plans, U_all=U_all, step_phases=step_phases, p123=p123_stage)


# Np = Nq of the reference's timed sample: channel 0 of the workload's basis at
# this grid (n = 6,075 for j <= 3, J <= 7/2), about 10 s per step of both
# on-shell energies on 16 host threads, so 25 steps stay within minutes
REF_SAMPLE_N = 15
REF_BIN = os.path.join(HERE, "oracle", "_ref", "tictac_ref")


def _ref_opts(cfg, N, energies="10"):
    opts = [f"{k}={v}" for k, v in cfg.items() if k not in ("Np_WP", "Nq_WP")]
    return opts + [f"Np_WP={N}", f"Nq_WP={N}", f"lab_energies={energies}"]


def _read_meta(path):
    chans, steps, timing = [], [], {}
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "chn":
                chans.append({k: float(v) if "." in v or "e" in v else int(v) for k, v in zip(tok[::2], tok[1::2])})
            elif tok[0] == "step":
                steps.append(dict(zip(tok[::2], [float(x) for x in tok[1::2]])))
            elif tok[0] == "timing":
                timing = dict(zip(tok[1::2], tok[2::2]))
    return chans, steps, timing


def reference_info(cfg, lab):
    """Channel sizes, on-shell energies and deuteron states of the workload from
    the reference build's own state-space set-up (tictac_ref info)."""
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/tictac_ref not built"
    energies = ",".join(f"{x:.12g}" for x in lab)
    with tempfile.TemporaryDirectory() as out:
        subprocess.run([REF_BIN, "info", out] + _ref_opts(cfg, cfg["Np_WP"], energies), check=True, cwd=out,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=600)
        chans, _, _ = _read_meta(os.path.join(out, "meta.txt"))
    return [{"n": c["n"], "nE": c["nE"], "nd": c["nd"]} for c in chans], None


def reference_sample(cfg, steps, sample_N=REF_SAMPLE_N, channel=0):
    """The reference's own dense LAPACK solve (oracle/_ref/tictac_ref: A columns,
    then per energy L = 1 - A G, R = A, zgetrf + zgetrs with nrhs = n; OpenMP +
    OpenBLAS on all host cores) of one channel of the workload's basis at
    Np = Nq = sample_N, set up once and timed for `steps` repetitions."""
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/tictac_ref not built"
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as out:
        cmd = [REF_BIN, "time", out, f"--channel={channel}", f"--repeat={steps}"] + _ref_opts(cfg, sample_N)
        t0 = time.perf_counter()
        subprocess.run(cmd, check=True, cwd=out, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(cores)), timeout=3000)
        wall = time.perf_counter() - t0
        chans, st, t = _read_meta(os.path.join(out, "meta.txt"))
    meta = chans[0]
    nE = int(meta["nE"])
    return dict(n_sample=int(t["n"]), nE=nE, step_s=[x["t"] for x in st], t_A=float(t["t_A"]),
                t_fair=float(t["t_fair"]) / nE, t_p123=float(meta["t_p123"]), cores=cores, wall=wall,
                sample_N=sample_N), None


def reference_value(ref, infos, timed):
    """Energies/s of the reference path over the workload from the sample's
    timed steps: per energy, the A columns (rebuilt for every energy, as the
    reference's faddeev_dense_solver does, scaled by n^2 Np) and the L/R
    formation and LAPACK solve (scaled by n^3) for every channel."""
    n_s, N_s = ref["n_sample"], ref["sample_N"]
    lu = float(np.mean(timed)) / ref["nE"]
    factor = sum((i["n"] / n_s) ** 3 for i in infos)
    a_factor = sum((i["n"] / n_s) ** 2 * (i["N"] / N_s) for i in infos)
    per_energy = lu * factor + ref["t_A"] * a_factor
    fair = ref["t_fair"] * factor + ref["t_A"] * a_factor
    return 1.0 / per_energy, {"sample_n": n_s, "sample_Np_Nq": N_s, "extrapolation_factor_n3": round(factor, 1),
                              "p123_s": round(ref["t_p123"], 4), "A_columns_s": round(ref["t_A"], 4),
                              "form_zgetrf_zgetrs_nrhs_n_s_per_energy": round(lu, 4),
                              "zgetrf_zgetrs_nrhs_nd_s_per_energy": round(ref["t_fair"], 4),
                              "fair_value": 1.0 / fair}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=list(CONFIGS), default="j3_J7_n30")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--tc-product", choices=list(PRODUCTS), default="tf32",
                    help="tensor-core product of the complex64 LU")
    ap.add_argument("--panel-order", choices=["recursive", "blocked"], default="blocked",
                    help="LU panels by recursive halving or in 32-column steps")
    ap.add_argument("--panel-width", type=int, default=0, help="LU panel width (0: the library's table)")
    ap.add_argument("--cta-pairs", type=int, default=1, help="tensor-core updates on CTA pairs (cta_group::2)")
    ap.add_argument("--mid-panel", type=int, default=128,
                    help="blocked panels in mid-panels of this many columns (0: one level)")
    ap.add_argument("--inverse-block", type=int, default=0,
                    help="largest unit-lower block solved through its explicit inverse (0: the library's default)")
    ap.add_argument("--breakdown", type=int, default=1,
                    help="one extra step with every kernel class timed, for the per-class breakdown")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-check", type=int, default=2,
                    help="FP64 step against mixed: 0 off, 1 smallest channel, 2 every channel")
    ap.add_argument("--channels", default="", help="comma list of channel indices to step (default: all)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.config in SCANS:
        count, lo, hi, seed = SCANS[args.config]
        energies_text = (f"{count} lab energies drawn uniformly in {lo:g}-{hi:g} MeV (seed {seed}), their distinct "
                         f"on-shell bins factored four per channel at a time, split over the N GPUs")
    else:
        energies_text = ("T_lab=10 MeV on one GPU (two on-shell bins); on N GPUs a scan of N lab energies with 2N "
                         "distinct on-shell bins")
    config = {"workload": f"{args.config}: LO-OPEP (stands in for N3LO-Idaho), j<={cfg['J_2N_max']}, "
                          f"J<={cfg['two_J_3N_max']}/2 both parities, Np=Nq={cfg['Np_WP']}, {energies_text}",
              "channels_per_step": None, "energies_per_step": None,
              "parallelism": f"(channel, energy) items over {world} GPU(s), longest processing time first",
              "l2": "inputs larger than L2 (a channel's FP64 A is n x n doubles: 0.66 GB at n = 9,072, 25.7 GB at "
                    "n = 56,700; the L2 holds 126 MB)"}

    if args.impl == "reference":
        # the reference's own CPU path; nothing of this repository's library is loaded
        if int(os.environ.get("RANK", "0")) != 0:
            return
        lab = scan_lab_energies(cfg, 1, args.config) if args.config in SCANS else [10.0]
        infos, why = reference_info(cfg, lab)
        if infos is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        for i in infos:
            i["N"] = cfg["Np_WP"]
        nE = infos[0]["nE"]
        ref, why = reference_sample(cfg, args.warmup + max(1, args.steps))
        if ref is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        timed = ref["step_s"][args.warmup:]
        v, phases = reference_value(ref, infos, timed)
        config["channels_per_step"] = len(infos)
        config["energies_per_step"] = nE
        config["n_per_channel"] = [i["n"] for i in infos]
        sample = (f"reference dense LAPACK solve (A columns, then per energy L/R formation + zgetrf + zgetrs "
                  f"nrhs=n) of channel 0 at Np=Nq={ref['sample_N']} (n={ref['n_sample']}), both on-shell "
                  f"energies of T_lab=10 MeV per step, {ref['cores']} threads; extrapolated to the workload by "
                  f"sum over channels of (n/{ref['n_sample']})^3 = {phases['extrapolation_factor_n3']}")
        print(json.dumps({"metric": METRIC, "value": v, "unit": "energies/s", "impl": "reference", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup,
                          "ms_step": round(float(np.mean(timed)) * 1e3, 3),
                          "ms_step_note": "measured time of one sample step (n above); value is extrapolated",
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
                          "data": "synthetic (seeded LO potential)", "config": config,
                          "cpu_baseline": {"value": v, "unit": "energies/s", "cores": ref["cores"],
                                           "kind": "reference", "sample": sample, "phases": phases},
                          "e2e": {"value": v, "unit": "energies/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    world, rank, local, pg = dist_setup()
    r = run_ours(args, world, rank, local, pg)
    if rank == 0:
        config["channels_per_step"] = len(r["infos"])
        config["energies_per_step"] = r["nE"]
        config["lab_energies_mev"] = [round(x, 6) for x in r["lab"]]
        config["n_per_channel"] = [i["n"] for i in r["infos"]]
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            infos = [dict(i, N=cfg["Np_WP"]) for i in r["infos"]]
            ref, why = reference_sample(cfg, 1)
            if ref is not None:
                v, phases = reference_value(ref, infos, ref["step_s"])
                cpu = {"value": v, "unit": "energies/s", "cores": ref["cores"], "kind": "reference",
                       "sample": f"reference dense LAPACK solve of channel 0 at Np=Nq={ref['sample_N']} "
                                 f"(n={ref['n_sample']}), one step of both energies, extrapolated by "
                                 f"{phases['extrapolation_factor_n3']} (sum of (n/n_sample)^3) to all "
                                 f"{len(infos)} channels",
                       "phases": phases}
        fp = r["fp64"]
        prod = args.tc_product
        out = {"metric": METRIC, "value": round(r["value"], 6), "unit": "energies/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_step": round(r["ms_step"], 3),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": (f"complex64 LU (tcgen05 {prod} products) + FP64 refinement" if args.precision == "mixed"
                         else "complex128"),
               "data": "synthetic (chiral LO potential on the reference's default Chebyshev WP grid)",
               "config": config, "clocks": r["clocks"], "roofline": r["roofline"], "cpu_baseline": cpu,
               "e2e": r["e2e"], "gpu_launches": int(r["launches"]),
               "mixed_over_fp64": (round(r["value"] / fp["fp64_value"], 3)
                                   if fp and fp.get("fp64_value") else None),
               "max_elem_rel_err_U_vs_fp64": fp["max_elem_rel_err_U"] if fp else None,
               "channel_solves_per_s": round(len(r["infos"]) * r["nE"] / (r["ms_step"] * 1e-3), 4),
               "kernels": r["kernels"], "fp64_comparison": fp, "setup_s": round(r["t_setup"], 3),
               "timed_steps_ms": [round(t, 1) for t in r["times"]],
               "p123_build": r["p123"],
               "last_timed_step_phases_ms": r["step_phases"],
               "U_gathered": {"channels": len(r["U_all"]), "energies": r["nE"],
                              "layout": "U[d' nd nE + d nE + j] per channel on rank 0"}}
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()

if __name__ == "__main__":
    main()
