"""Extract the reference's regression anchors into reference_regression.json.

The reference's app regression tests (``regressions.sh`` beside each app) run the
app with ``-F regression.ini`` plus command-line overrides and compare three
counters with ``regression_values_N.csv`` (src/fclaw2d_finalize.c:119-165).  The
options in force are the app's ``fclaw_options.ini`` overridden by
``regression.ini`` overridden by the command line (src/fclaw_base.c:759-800).
This script reads those files from the reference tree and writes, per case, the
merged option values the build's runs need and the expected counters.

    FCB_REFERENCE_TREE=<path to the reference checkout> python tests/golden/make_regression_values.py
"""
from __future__ import annotations

import json
import os
import re
import sys

CASES = [
    # (name, app dir, ini, command-line overrides, values csv)
    ("swirl_claw46", "applications/clawpack/advection/2d/swirl", "regression.ini",
     {"user:claw-version": "4"}, "regression_values_0.csv"),
    ("radialdam_claw46", "applications/clawpack/shallow/2d/radialdam", "regression.ini",
     {"user:claw-version": "4", "user:example": "0"}, "regression_values_0.csv"),
]

KEYS = {
    "clawpatch": ["mx", "my", "mbc", "meqn", "maux", "refinement-criteria", "threshold-variable"],
    "options": ["minlevel", "maxlevel", "regrid_interval", "refine_threshold", "coarsen_threshold",
                "smooth-refine", "smooth-level", "tfinal", "initial_dt", "use_fixed_dt", "max_cfl",
                "desired_cfl", "outstyle", "nout", "subcycle", "time-sync", "ax", "bx", "ay", "by", "manifold"],
    "clawpack46": ["order", "mcapa", "mwaves", "mthlim", "mthbc"],
    "user": ["period", "claw-version", "example", "g", "x0", "y0", "r0", "hin", "hout"],
}


def read_ini(path: str) -> dict:
    out, sec = {}, None
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            m = re.match(r"\[(.+)\]", line)
            if m:
                sec = m.group(1).strip().lower()
                continue
            if "=" in line and sec:
                k, v = line.split("=", 1)
                out[(sec, k.strip().lower())] = v.strip()
    return out


def main() -> None:
    ref = os.environ.get("FCB_REFERENCE_TREE")
    if not ref or not os.path.isdir(ref):
        sys.exit("set FCB_REFERENCE_TREE to the reference checkout")
    cases = {}
    for name, app, ini, cli, csv in CASES:
        d = os.path.join(ref, app)
        opts = read_ini(os.path.join(d, "fclaw_options.ini"))
        opts.update(read_ini(os.path.join(d, ini)))
        for k, v in cli.items():
            sec, key = k.split(":")
            opts[(sec, key)] = v
        merged = {}
        for sec, keys in KEYS.items():
            for k in keys:
                if (sec, k) in opts:
                    merged[f"{sec}:{k}"] = opts[(sec, k)]
        expected = {}
        with open(os.path.join(d, csv)) as f:
            for line in f:
                k, v = line.strip().split(",")
                expected[k] = int(v)
        cases[name] = {"source": f"{app}/{ini} + fclaw_options.ini + {cli}", "values_file": f"{app}/{csv}",
                       "options": merged, "expected": expected}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_regression.json")
    with open(out, "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)
    print(out)


if __name__ == "__main__":
    main()
