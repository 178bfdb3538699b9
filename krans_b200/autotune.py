"""Autotuner of the batched persistent launch (krans_solve_batch and the
server's launches).

The knobs (krans_batch_tuning, include/krans_cuda.h) decide which kind of
team a request of a given size runs on and how the solvers' SpMV spreads a
row over threads:
  cluster_size   blocks per big thread-block cluster
  cluster_min    m + n from which a request runs on a cluster (else one block)
  pair_max       m + n below which a cluster request runs on a 2-block cluster
                 of the second launch beside the big clusters
  lanes[6]       threads per row for operands of mean row length <= 3, 8, 16,
                 32, 64 and above

tune() searches them one at a time (coordinate descent, each knob over a
short list of candidates around the built-in value, in the order above) on
probe batches drawn from the batched workload's generator with seeds the
benchmark does not use, keeping a candidate only when it is faster by more
than the noise margin. The winners are written to
krans_b200/tuning/<device>.json together with every trial; Context() applies
the table of its device when one exists.

    python -m krans_b200.autotune [--batch 256] [--probes 1]
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
from typing import Dict, List, Optional

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_DIR = os.path.join(HERE, "tuning")
DEFAULTS = {"cluster_min": 16384, "pair_max": 120000, "cluster_size": 8, "lanes": [1, 2, 4, 8, 16, 32]}
CANDIDATES = [
    ("cluster_size", [8, 4]),
    ("cluster_min", [16384, 8192, 32768]),
    ("pair_max", [120000, 60000, 250000]),
    ("lanes[1]", [2, 1, 4]),   # mean row length in (3, 8]: incidence transposes (degree ~6)
    ("lanes[0]", [1, 2]),      # mean row length <= 3: shift operators, incidence rows
]
MARGIN = 0.02  # a candidate must beat the incumbent by 2% to replace it


def device_key(name: str, sms: int) -> str:
    return "".join(c if c.isalnum() else "_" for c in name).strip("_") + f"_{sms}sm"


def table_path(name: str, sms: int) -> str:
    return os.path.join(TABLE_DIR, device_key(name, sms) + ".json")


def knobs_with(knobs: Dict, key: str, value) -> Dict:
    out = {"cluster_min": knobs["cluster_min"], "pair_max": knobs["pair_max"],
           "cluster_size": knobs["cluster_size"], "lanes": list(knobs["lanes"])}
    if key.startswith("lanes["):
        out["lanes"][int(key[6:-1])] = value
    else:
        out[key] = value
    return out


def apply(ctx, knobs: Dict):
    ctx.set_batch_tuning(cluster_min=knobs["cluster_min"], pair_max=knobs["pair_max"],
                         cluster_size=knobs["cluster_size"], lanes=knobs["lanes"])


def validate(table: Dict) -> Dict:
    """The knobs of a table file, checked against the C ABI's ranges."""
    k = table["knobs"]
    if not (int(k["cluster_min"]) > 0 and int(k["pair_max"]) > 0 and 2 <= int(k["cluster_size"]) <= 16):
        raise ValueError("tuning table: size thresholds or cluster size out of range")
    lanes = [int(x) for x in k["lanes"]]
    if len(lanes) != 6 or any(x < 1 or x > 32 or (x & (x - 1)) for x in lanes):
        raise ValueError("tuning table: lanes must be 6 powers of two up to 32")
    return {"cluster_min": int(k["cluster_min"]), "pair_max": int(k["pair_max"]),
            "cluster_size": int(k["cluster_size"]), "lanes": lanes}


def load(name: str, sms: int) -> Optional[Dict]:
    p = table_path(name, sms)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        t = json.load(f)
    t["knobs"] = validate(t)
    t["path"] = os.path.relpath(p, os.path.dirname(HERE))
    return t


def device_of(ctx):
    import torch
    prop = torch.cuda.get_device_properties(ctx.device)
    return prop.name, int(prop.multi_processor_count)


def apply_cached(ctx) -> Optional[str]:
    """Apply the table of ctx's device if one exists; returns its path."""
    try:
        name, sms = device_of(ctx)
    except Exception:
        return None
    t = load(name, sms)
    if t is None:
        return None
    apply(ctx, t["knobs"])
    return t["path"]


def search(evaluate, start: Dict, candidates=CANDIDATES, margin: float = MARGIN):
    """Coordinate descent: for each knob in turn, evaluate its candidates with
    the other knobs at their current best and keep the fastest, unless it
    beats the incumbent by less than `margin`. evaluate(knobs) -> solves/s.
    Returns (best knobs, its rate, trials)."""
    best = knobs_with(start, "cluster_min", start["cluster_min"])
    trials: List[Dict] = []
    cache = {}

    def ev(k):
        key = json.dumps(k, sort_keys=True)
        if key not in cache:
            cache[key] = float(evaluate(k))
            trials.append({"knobs": k, "solves_per_s": cache[key]})
        return cache[key]

    best_v = ev(best)
    for name, values in candidates:
        for v in values:
            k = knobs_with(best, name, v)
            r = ev(k)
            if r > best_v * (1.0 + margin):
                best, best_v = k, r
    return best, best_v, trials


def tune(ctx, batch: int = 256, probes: int = 1, seed: int = 7000) -> Dict:
    """Measure the knobs on `probes` batches of the batched workload and
    return the table (not yet saved)."""
    import numpy as np
    from . import generators as G
    from .api import CudaCsrMatrixAdapter, CyclicLanczosOptions, Precision
    from .serving import SolveRequest, solve_batch

    def L(A):
        A2 = A.multiply(A)
        return float(np.sqrt(max(A2.sum(axis=0).max(), A2.sum(axis=1).max())))

    sets = []
    for b in range(probes):
        insts = G.batch_instances(batch, seed=seed + b, kernel=False)
        mats = [CudaCsrMatrixAdapter.from_scipy(ctx, i.A, fp32=True) for i in insts]
        opts = [CyclicLanczosOptions(k=i.k, tol_abs=1e-12 * L(i.A), tol_rel=0.0, cg_maxit=1000,
                                     precision=Precision.MIXED) for i in insts]
        sets.append((mats, opts))

    def evaluate(knobs):
        apply(ctx, knobs)
        n, ms = 0, 0.0
        for mats, opts in sets:
            reqs = [SolveRequest(M, o, seed=1 + j, rng_mode="philox") for j, (M, o) in enumerate(zip(mats, opts))]
            ms += solve_batch(ctx, reqs)
            n += len(reqs)
        return n / (ms / 1e3)

    evaluate(DEFAULTS)  # warm-up (module load, first touch of the matrices)
    best, best_v, trials = search(evaluate, DEFAULTS)
    apply(ctx, best)
    name, sms = device_of(ctx)
    return {"device": name, "sms": sms, "library": ctx.lib.krans_version().decode(),
            "date": datetime.date.today().isoformat(),
            "probe": {"workload": "batched uneven null-space solves (shift and incidence, n log-uniform in "
                                  "[1e3, 2e5]), mixed precision, tol_abs = 1e-12 L", "batch": batch,
                      "probes": probes, "seed": seed},
            "metric": "solves/s of the probe batches (device time)", "knobs": best,
            "best_solves_per_s": best_v, "default_solves_per_s": trials[0]["solves_per_s"], "trials": trials}


def save(table: Dict) -> str:
    os.makedirs(TABLE_DIR, exist_ok=True)
    p = table_path(table["device"], table["sms"])
    with open(p, "w") as f:
        json.dump({k: v for k, v in table.items() if k != "path"}, f, indent=1)
    return p


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--probes", type=int, default=1)
    ap.add_argument("--seed", type=int, default=7000)
    a = ap.parse_args()
    from .api import Context
    ctx = Context(a.device, tuning=False)
    t = tune(ctx, a.batch, a.probes, a.seed)
    p = save(t)
    print(json.dumps({"table": p, "knobs": t["knobs"], "best_solves_per_s": t["best_solves_per_s"],
                      "default_solves_per_s": t["default_solves_per_s"], "trials": len(t["trials"])}))


if __name__ == "__main__":
    main()
