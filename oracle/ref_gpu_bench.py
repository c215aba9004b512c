"""Reference GASAL2 on the GPU, timed on the benchmark workloads, and a
full-size parity check of the CUDA path against it.

TEST INFRASTRUCTURE ONLY (needs a GPU and oracle/_ref built by
`make -C oracle ref`):

    python oracle/ref_gpu_bench.py --workload w1 [--pairs N]
    python oracle/ref_gpu_bench.py --workload w2 --pairs 20000
    python oracle/ref_gpu_bench.py --workload w3 --pairs 20000   # ksw, z-drop 0
    python oracle/ref_gpu_bench.py --workload w4 --pairs 8000    # mixed 50-5000 bp

Runs the unmodified reference library compiled for sm_100a
(oracle/_ref/libgasal_ref_mql{304,2048,8192}.so) through its own C++ API
(gasal_aln_async -> gasal_is_aln_async_done, timed on the host around those
two calls, averaged over --repeats), then this repository's library on the
same batches through gb_align, and prints one JSON line with both rates and
the number of result values that differ (0 expected).

The reference's ksw kernel hard-codes z-drop 0, so w3 and w4's ksw launch
run with z-drop 0 here.  Its traceback matrix is max_q * max_t * n, so w4's
traceback launch is capped at 800 pairs.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from gasal_b200 import workloads as W  # noqa: E402
from gasal_b200 import lib as gl  # noqa: E402
from gasal_b200.capi import Params, GLOBAL, KSW, WITH_TB  # noqa: E402
from oracle.bindings import ref_gpu_align  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="w1", choices=["w1", "w2", "w3", "w4"])
    ap.add_argument("--pairs", type=int, default=0)
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args()
    if args.workload == "w1":
        parts = W.workload1(args.pairs or 1_000_000)
        mql = 304
    elif args.workload == "w2":
        parts = [(Params(algo=GLOBAL, start_pos=WITH_TB), W.workload2(args.pairs or 20000))]
        mql = 2048
    elif args.workload == "w3":
        parts = [(Params(algo=KSW), W.workload3(args.pairs or 20000))]
        mql = 2048
    else:
        parts = []
        for p, b in W.workload4(args.pairs or 8000):
            if p.start_pos == WITH_TB:
                b = b.subset(np.arange(min(b.n, 800)))
            if p.algo == KSW:
                p = Params(algo=KSW)
            parts.append((p, b))
        mql = 8192
    gl.set_reference_max_query_len(mql)
    ref_ms = 0.0
    ours_ms = 0.0
    diffs = 0
    checked = 0
    n = 0
    for p, b in parts:
        out_ref, ms = ref_gpu_align(p, b, mql=mql, repeats=args.repeats)
        ref_ms += ms
        t0 = time.time()
        out = gl.align(p, b)
        ours_ms += (time.time() - t0) * 1e3
        for k, v in out_ref.as_dict(p).items():
            g = out.as_dict(p)[k]
            if k == "cigar":  # only the bytes each pair owns
                for i in range(b.n):
                    o, c = int(b.q_off[i]), int(out.n_cigar[i])
                    if c <= (int(b.q_len[i]) + 7) // 8 * 8:
                        diffs += int(np.count_nonzero(g[o:o + c] != v[o:o + c]))
                        checked += c
            else:
                diffs += int(np.count_nonzero(g != v))
                checked += v.size
        n += b.n
    print(json.dumps({"workload": args.workload, "pairs": n,
                      "reference_gpu_pairs_per_s": n / (ref_ms * 1e-3),
                      "reference_gpu_ms": ref_ms,
                      "note": "reference: host time from gasal_aln_async to gasal_is_aln_async_done()==0, "
                              "H2D of the staged batch, kernels and D2H included; sm_100a build, "
                              f"MAX_QUERY_LEN={mql}",
                      "ours_gb_align_ms_incl_setup": ours_ms,
                      "values_checked": checked, "values_different": diffs}), flush=True)


if __name__ == "__main__":
    main()
