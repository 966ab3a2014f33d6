"""Panel-width tuning of the complex64 LU on the GPU at hand.

For every channel of a run (matrix order n) and every tensor-core product, the
mixed-precision solve of the first on-shell energies is timed with each
candidate panel width; the fastest width per (product, n) becomes a row of
``csrc/host/tt_panel_table.h`` (``--write``), which the library consults when
the run leaves ``panel_width`` at 0.  Widths are multiples of 32 up to 512;
every width gives the same U within the refinement tolerance, only the time
differs.

    python -m tictac_b200.autotune                      # print the table
    python -m tictac_b200.autotune --write              # and rewrite the header
"""
import argparse
import json
import os

import numpy as np

import tictac_b200 as tt

PRODUCTS = {"tf32": 2, "bf16x3": 3}
HEADER = os.path.normpath(os.path.join(os.path.dirname(__file__), "..", "..", "csrc", "host", "tt_panel_table.h"))


def time_widths(run, chans, energies, widths, product, reps):
    """{n: {width: fastest ms of reps}} of build_A + mixed solve per channel (the fastest repetition: clock dips
    under the power cap only ever add time)."""
    run.set_solve_option("tc_product", {v: k for k, v in PRODUCTS.items()}[product])
    out = {}
    for c in chans:
        n = run.channel_info(c)["n"]
        res = {}
        for w in widths:
            run.set_solve_option("panel_width", w)
            ms = []
            for r in range(reps + 1):  # the first solve warms up
                run.timer_start()
                run.build_A(c)
                run.solve_energies(c, energies, tt.PRECISION_MIXED)
                t = run.timer_stop()
                run.release_A(c)
                if r:
                    ms.append(t)
            res[w] = float(np.min(ms))
        out[n] = res
    run.set_solve_option("panel_width", 0)
    return out


def table_rows(timings):
    """Header rows (product, n_max, width): the best width per measured n, each row reaching halfway to the next
    measured n, the last one without bound."""
    rows = []
    for pname, per_n in timings.items():
        ns = sorted(per_n)
        best = [min(per_n[n], key=per_n[n].get) for n in ns]
        for i, n in enumerate(ns):
            n_max = (n + ns[i + 1]) // 2 if i + 1 < len(ns) else 1 << 30
            if rows and rows[-1][0] == PRODUCTS[pname] and rows[-1][2] == best[i]:
                rows[-1] = (rows[-1][0], n_max, best[i])  # merge equal neighbours
            else:
                rows.append((PRODUCTS[pname], n_max, best[i]))
    return rows


def render_header(rows, note):
    body = "\n".join(f"    {{{p}, {'1 << 30' if m == 1 << 30 else m}, {w}}}," for p, m, w in rows)
    return f"""// Complex64 LU panel width by matrix order and tensor-core product, measured
// on a B200 by tictac_b200.autotune (python -m tictac_b200.autotune --write):
// the first row whose product matches and whose n_max >= n gives the width.
// Products: 1 BF16x3 N=128 tiles, 2 TF32, 3 BF16x3 real-row.
// {note}
#pragma once

namespace tt {{

struct PanelWidthRow {{
  int product;
  int n_max;
  int width;
}};

constexpr PanelWidthRow kPanelWidthTable[] = {{
{body}
    {{1, 1 << 30, 512}},
}};

}}  // namespace tt
"""


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--Np", type=int, default=24, help="Np_WP = Nq_WP of the tuning run")
    ap.add_argument("--J2N", type=int, default=3, help="J_2N_max")
    ap.add_argument("--two-J3N", type=int, default=7, help="two_J_3N_max")
    ap.add_argument("--widths", default="256,384,512")
    ap.add_argument("--products", default="tf32,bf16x3")
    ap.add_argument("--energies", type=int, default=2, help="on-shell energies factored together")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--write", action="store_true", help="rewrite csrc/host/tt_panel_table.h")
    args = ap.parse_args(argv)
    widths = [int(w) for w in args.widths.split(",")]
    if any(w <= 0 or w > 512 or w % 32 for w in widths):
        raise SystemExit("panel widths are multiples of 32 up to 512")
    lab = ",".join(str(10.0 + 3.0 * i) for i in range(args.energies))
    run = tt.Run(potential_model="LO_internal", J_2N_max=args.J2N, two_J_3N_max=args.two_J3N, Np_WP=args.Np,
                 Nq_WP=args.Np, lab_energies=lab)
    nE = len(run.energies()[0])
    energies = list(range(min(nE, args.energies)))
    chans = list(range(run.num_channels))
    for c in chans:
        run.build_P123(c)
    timings = {p: time_widths(run, chans, energies, widths, PRODUCTS[p], args.reps) for p in args.products.split(",")}
    rows = table_rows(timings)
    print(json.dumps({"timings_ms": {p: {str(n): t for n, t in d.items()} for p, d in timings.items()},
                      "rows": rows}))
    if args.write:
        note = (f"Tuned on J_2N_max={args.J2N}, two_J_3N_max={args.two_J3N}, Np=Nq={args.Np}, "
                f"{len(energies)} energies, widths {args.widths}.")
        with open(HEADER, "w") as f:
            f.write(render_header(rows, note))
    run.close()


if __name__ == "__main__":
    main()
