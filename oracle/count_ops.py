"""Floating-point operation counts of IMPLSCH per spectral bin, from the
oracle instantiated with a counting number type, for the regional ST6 and
ST4 workloads; writes profiles/op_counts.json, which bench.py reads for the
FP32 roofline of IMPLSCH.  Test infrastructure: it runs the oracle only.

    python oracle/count_ops.py [--points 256]   (or python -m oracle.count_ops)

The counted state is the one the parity tests use: the workload's start
spectrum after three source steps of the oracle (spectra with a developed
tail, cut-off indices and LFACTOR iterations in their usual ranges).
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[0] = ROOT  # run as a script: import the oracle package, not oracle/oracle.py


def count(name, scale, npoints, seed=7):
    from oracle import oracle
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale)
    o = oracle.Oracle(w.cfg)
    o.set_grid(w.grid)
    o.set_fields(w.depth)
    o.prepare_propagation()
    o.prepare_source()
    indep = o.indep()
    f = w.spectrum_f().astype(float)
    tw, us, zz = (a.astype(float) for a in (w.tauw, w.ustar, w.z0))
    for _ in range(3):
        f, tw, us, zz, _ = o.implsch(f, w.u10, w.udir, tw, us, zz, w.roairn, w.wstar, w.depth, indep)
        for _ in range(w.sub_steps):
            f = o.propags(f)
    rng = np.random.default_rng(seed)
    pts = np.sort(rng.choice(w.nsea, size=min(npoints, w.nsea), replace=False))
    sl = lambda a: np.asarray(a)[pts]
    c = o.count_implsch(np.asfortranarray(f[pts]), sl(w.u10), sl(w.udir), sl(tw), sl(us), sl(zz), sl(w.roairn),
                        sl(w.wstar), sl(w.depth), sl(indep))
    bins = len(pts) * w.cfg["kl"] * w.cfg["ml"]
    per_bin = {k: v / bins for k, v in c.items()}
    flops = c["add"] + c["mul"] + c["div"] + c["sqrt"] + c["trans"]
    return {"workload": f"{name} at scale {scale}", "iphys": w.cfg["iphys"], "kl": w.cfg["kl"], "ml": w.cfg["ml"],
            "points": len(pts), "per_bin": per_bin, "flops_per_bin": flops / bins,
            "note": "flops = additions + multiplications + divisions + square roots + transcendentals (1 each); "
                    "comparisons are listed but not counted as flops"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=256)
    a = ap.parse_args()
    out = {"implsch_c1": count("c1", 0.05, a.points), "implsch_c2": count("c2", 0.1, a.points),
           "implsch_c0": count("c0", 0.5, a.points),
           "how": "oracle/count_ops.py: the oracle's IMPLSCH restatement instantiated with a counting number type "
                  "(oracle/oracle_count.hpp) on sampled points after three source steps"}
    path = os.path.join(ROOT, "profiles", "op_counts.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
