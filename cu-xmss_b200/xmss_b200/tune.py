"""Tunes the launch shapes of every hash family on this GPU and writes the
JSON table the package applies at import (xmss_b200/tuning.json):

    python -m xmss_b200.tune [--count 4096] [--out PATH]

One representative parameter set per family is tuned by the library's
autotuner (xmss_b200_autotune); the table holds the chosen shapes and the
trials they were chosen from."""
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


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=4096, help="signatures of the verify batch")
    ap.add_argument("--out", default=xb.TUNING_PATH)
    args = ap.parse_args()
    xb.init(0)
    reports = {}
    for name in REPRESENTATIVES:
        oid = xb.xmss_str_to_oid(name)
        best, report = xb.autotune(oid, False, args.count)
        reports[name] = report
        print(name, best, flush=True)
    xb.save_tuning(args.out, notes={"count": args.count, "trials": reports})
    print("wrote", args.out)


if __name__ == "__main__":
    main()
