"""Tunes the launch shapes on this GPU and writes the JSON table the package
applies at import (xmss_b200/tuning.json):

    python -m xmss_b200.tune [--count 4096] [--out PATH] [--trees-only]

One representative parameter set per (func, n) family is tuned by the
library's autotuner (xmss_b200_autotune: verify and chain CTA sizes, the
split of large verify batches); then the tree-building shape of every
parameter set in TREE_SETS (xmss_b200_autotune_tree: in-CTA subtree height,
chains per warp and the build size from which the in-CTA form is used).
The table holds the chosen shapes and the trials they were chosen from."""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import xmss_b200 as xb  # noqa: E402

# one parameter set per (func, n) family
REPRESENTATIVES = ("XMSS-SHA2_10_192", "XMSS-SHA2_10_256", "XMSS-SHA2_10_512", "XMSS-SHAKE_10_256",
                   "XMSS-SHAKE256_10_192", "XMSS-SHAKE256_10_256", "XMSS-SHAKE_10_512")
# parameter sets whose subtree-building shape is tuned (the sets of the
# keygen, mix and serving workloads and the family representatives)
TREE_SETS = ("XMSS-SHA2_10_256", "XMSS-SHA2_16_256", "XMSS-SHA2_20_256", "XMSS-SHA2_10_512", "XMSS-SHAKE_10_256",
             "XMSSMT-SHA2_20/2_256", "XMSSMT-SHA2_40/4_256", "XMSS-SHA2_10_192", "XMSS-SHAKE256_10_192",
             "XMSS-SHAKE256_10_256", "XMSS-SHAKE_10_512")


def _oid(name: str):
    mt = name.startswith("XMSSMT")
    return (xb.xmssmt_str_to_oid(name) if mt else xb.xmss_str_to_oid(name)), mt


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=4096, help="signatures of the verify batch")
    ap.add_argument("--out", default=xb.TUNING_PATH)
    ap.add_argument("--trees-only", action="store_true", help="keep the family shapes; tune the tree shapes")
    args = ap.parse_args()
    xb.init(0)
    old = json.load(open(args.out)) if os.path.exists(args.out) else {}
    reports = dict(old.get("notes", {}).get("trials", {})) if args.trees_only else {}
    if not args.trees_only:
        for name in REPRESENTATIVES:
            best, report = xb.autotune(xb.xmss_str_to_oid(name), False, args.count)
            reports[name] = report
            print(name, best, flush=True)
    tree_reports = {}
    for name in TREE_SETS:
        oid, mt = _oid(name)
        best, report = xb.autotune_tree(oid, mt)
        tree_reports[name] = report
        print(name, best, flush=True)
    xb.save_tuning(args.out, notes={"count": args.count, "trials": reports, "tree_trials": tree_reports},
                   sets=[_oid(n) for n in TREE_SETS])
    print("wrote", args.out)


if __name__ == "__main__":
    main()
