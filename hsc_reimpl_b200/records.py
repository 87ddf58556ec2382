"""Solve evidence: the ``hsc_stats.jsonl`` collector and a system dump / replay tool.

``SolverRecords`` follows the experiment drivers' collector
(reproduction/experiments/vehicle_full_pass/storage.py:17-62): it copies each
complete line of the native ``hsc_stats.jsonl`` (written by
``linear_hsc.cu:420-431``, here by ``LinearHSC.do_solve`` and the C++ shim)
exactly once into a destination log, keeps the same running summary (solves,
fallbacks, maxima of residuals / iterations / contacts / ACA error / rank /
Neumann doublings, minima of rank and doublings) and raises on any solve that
was not an accepted ``linear_hsc`` result -- the reference's "no fallback"
rule.  A trailing line without its newline is left for the next call.

``dump_system`` / ``load_system`` store one Newton system exactly as the solver
received it (one-triangle BCOO, column-major blocks, ``b``, the dof layout),
with the options, the stats record and the solution of the original solve.
``replay`` re-solves dumped systems -- with the recorded options or with
overrides (precision, rank cap, tile width ...) -- and reports, per system, the
recorded against the replayed iteration count, rank and full residual and the
distance between the two solutions.  ``LinearHSC(dump_systems=True)`` writes a
dump per solve under ``<workspace>/systems/``.

    python -m hsc_reimpl_b200.records summary <hsc_stats.jsonl> <copy.jsonl>
    python -m hsc_reimpl_b200.records replay <workspace or .npz ...> [--precision fp32] [--max-rank 64]
"""
from __future__ import annotations

import argparse
import dataclasses
import glob
import json
import os
from pathlib import Path

import numpy as np

SUMMARY_MAX = (
    ("max_schur_relative_residual", "schur_relative_residual"),
    ("max_full_relative_residual", "full_relative_residual"),
    ("max_pcg_iterations", "pcg_iterations"),
    ("max_mesh_contacts", "active_mesh_contacts"),
    ("max_ground_contacts", "active_ground_contacts"),
    ("max_aca_error", "aca_relative_error"),
    ("max_rank", "rank"),
    ("max_neumann_doublings", "neumann_doublings"),
)
SUMMARY_MIN = (("min_rank", "rank"), ("min_neumann_doublings", "neumann_doublings"))


class UnacceptedSolve(RuntimeError):
    pass


class SolverRecords:
    """Incremental copy + summary of a native ``hsc_stats.jsonl`` (storage.py:17-62)."""

    def __init__(self, native, destination):
        self.native = Path(native)
        self.destination = Path(destination)
        self.offset = 0
        self.summary = {
            "linear_solves": 0, "fallbacks": 0,
            "max_schur_relative_residual": 0.0, "max_full_relative_residual": 0.0,
            "max_pcg_iterations": 0, "max_mesh_contacts": 0,
            "max_ground_contacts": 0, "max_aca_error": 0.0,
            "min_rank": None, "max_rank": 0,
            "min_neumann_doublings": None, "max_neumann_doublings": 0,
        }

    def collect(self):
        """New complete records since the last call (copied to the destination as read)."""
        rows = []
        if not self.native.exists():
            return rows
        with self.native.open("rb") as src, self.destination.open("ab") as dst:
            src.seek(self.offset)
            while True:
                line = src.readline()
                if not line or not line.endswith(b"\n"):
                    break
                row = json.loads(line)
                dst.write(line)
                self.offset = src.tell()
                rows.append(row)
                s = self.summary
                s["linear_solves"] += 1
                s["fallbacks"] += int(row["fallback"])
                if row["solver"] != "linear_hsc" or row["fallback"] or not row["accepted"]:
                    raise UnacceptedSolve("HSC returned an unaccepted solve or a fallback: "
                                          f"frame {row.get('frame')} newton {row.get('newton')}")
                for out, key in SUMMARY_MAX:
                    s[out] = max(s[out], row[key])
                for out, key in SUMMARY_MIN:
                    s[out] = row[key] if s[out] is None else min(s[out], row[key])
        return rows


# --------------------------------------------------------------------------- dumps

def _np(t):
    return t.detach().cpu().numpy() if hasattr(t, "detach") else np.asarray(t)


def dump_system(path, system, options=None, record=None, x=None):
    """One system as the solver saw it (``DeviceSystem`` or host ``HSCSystem``) -> ``.npz``."""
    if hasattr(system, "values"):       # DeviceSystem: column-major (nnzb, 9)
        rows, cols, vals, b = _np(system.rows), _np(system.cols), _np(system.values), _np(system.b)
    else:                               # HSCSystem
        rows, cols, vals, b = system.rows, system.cols, system.values_colmajor(), system.b
    extra = {}
    if x is not None:
        extra["x"] = np.asarray(_np(x), dtype=np.float64)
    opts = dataclasses.asdict(options) if options is not None else {}
    np.savez(path, rows=np.asarray(rows, np.int32), cols=np.asarray(cols, np.int32),
             values=np.asarray(vals, np.float64).reshape(-1, 9), b=np.asarray(b, np.float64),
             nblock=np.int64(system.nblock), layout=np.asarray(system.layout, np.int64),
             options=json.dumps(opts), record=json.dumps(record or {}), **extra)


def load_system(path, device="cuda"):
    """(DeviceSystem, options dict, record dict, recorded x or None)."""
    from .solver import DeviceSystem
    import torch
    z = np.load(path, allow_pickle=False)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    ds = DeviceSystem(t(z["rows"]), t(z["cols"]), t(z["values"]), int(z["nblock"]),
                      tuple(int(v) for v in z["layout"]), t(z["b"]))
    return (ds, json.loads(str(z["options"])), json.loads(str(z["record"])),
            z["x"] if "x" in z.files else None)


def options_from_dict(d, **overrides):
    from .solver import HSCOptions
    known = {f.name for f in dataclasses.fields(HSCOptions)}
    kw = {k: v for k, v in d.items() if k in known}
    if isinstance(kw.get("poly_weights"), list):
        kw["poly_weights"] = tuple(kw["poly_weights"])
    kw.update({k: v for k, v in overrides.items() if v is not None})
    return HSCOptions(**kw)


def dump_files(paths):
    out = []
    for p in paths:
        if os.path.isdir(p):
            out += sorted(glob.glob(os.path.join(p, "systems", "*.npz")) + glob.glob(os.path.join(p, "*.npz")))
        else:
            out.append(p)
    return out


def replay(paths, ctx=None, **overrides):
    """Re-solve dumped systems in file order on one context; one comparison row per system."""
    from .solver import HSCContext
    from .learned import MODEL_PATH, load_model
    rows = []
    own = ctx is None
    for path in dump_files(paths):
        ds, opts, rec, x_rec = load_system(path)
        o = options_from_dict(opts, **overrides)
        if ctx is None:
            ctx = HSCContext(o)
        else:
            ctx.set_options(o)
        if o.learned:
            ctx.set_learned_model(load_model(MODEL_PATH)[0])
        x, s = ctx.solve(ds, raise_on_error=False)
        xr = x.detach().cpu().numpy()
        row = {"file": os.path.basename(path), "status": s["status"],
               "pcg_iterations": s["pcg_iterations"], "recorded_pcg_iterations": rec.get("pcg_iterations"),
               "rank": s["rank"], "recorded_rank": rec.get("rank"),
               "full_relative_residual": s["full_relative_residual"],
               "recorded_full_relative_residual": rec.get("full_relative_residual"),
               "accepted": bool(s["accepted"]), "total_ms": s["total_ms"]}
        if x_rec is not None:
            row["x_relative_difference"] = float(np.linalg.norm(xr - x_rec) / max(np.linalg.norm(x_rec), 1e-300))
            row["x_bitwise_equal"] = bool(np.array_equal(xr, x_rec))
        rows.append(row)
    if own and ctx is not None:
        ctx.close()
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("summary")
    a.add_argument("native")
    a.add_argument("destination")
    r = sub.add_parser("replay")
    r.add_argument("paths", nargs="+")
    r.add_argument("--precision", choices=("fp64", "fp32", "bf16"))
    r.add_argument("--max-rank", type=int)
    r.add_argument("--threads-per-row", type=int)
    r.add_argument("--neumann-order", type=int)
    r.add_argument("--residual-replacement", type=int)
    args = ap.parse_args(argv)
    if args.cmd == "summary":
        rec = SolverRecords(args.native, args.destination)
        rec.collect()
        print(json.dumps(rec.summary))
        return 0
    rows = replay(args.paths, precision=args.precision, max_rank=args.max_rank,
                  threads_per_row=args.threads_per_row, neumann_order=args.neumann_order,
                  residual_replacement=args.residual_replacement)
    for row in rows:
        print(json.dumps(row))
    return 0 if all(r["accepted"] for r in rows) else 1


if __name__ == "__main__":
    raise SystemExit(main())
