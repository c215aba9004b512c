"""The reference's own caller as the drop-in check.

test_prog/test_prog.cpp from the reference is compiled unmodified twice by
oracle/Makefile (`make -C oracle ref`): once against this repository's
include/gasal_header.h and libgasal_b200.so, once against the reference
headers and the reference library built for sm_100a.  Both run on the
reference's 20,000-pair sample with the option sets of test_prog/Makefile
(`-p -y local`) and the other algorithm / start / second-best / semi-global
modes, and must print the same results.  Lines are compared as a sorted list:
test_prog prints each stream's batch when that stream completes, so the batch
order can differ between runs.

One exception, the reference's own undefined behaviour: its GLOBAL traceback
starts one past the last cell (src/kernels/get_tb.h:21-23) and, when a length
is a multiple of 8, reads a tile row that no kernel wrote.  test_prog reuses
one tile buffer for every batch, so the reference's CIGAR for those pairs
depends on the previous batch's leftovers (this library writes two zero tile
rows per pair instead).  For `-y global -t` such pairs are set aside; every
other line must match, and every differing line must be one of them.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TP = os.path.join(ROOT, "oracle", "_ref", "tp")
OURS = os.path.join(TP, "test_prog_ours")
REF = os.path.join(TP, "test_prog_ref")
FILES = [os.path.join(TP, "query_batch.fasta"), os.path.join(TP, "target_batch.fasta")]

OPTION_SETS = [
    "-p -y local",
    "-p -y local -s --second-best",
    "-p -y local -t",
    "-p -y global",
    "-p -y global -t",
    "-p -y semi_global -x TARGET TARGET -s",
    "-p -y semi_global -x NONE QUERY",
    "-p -y local -s -n 2",
    "-p -y local -a 2 -b 3 -q 5 -r 2 -s",
]


def _lengths():
    """(query, target) lengths per pair, parsed as test_prog parses the FASTA."""
    out = []
    for path in FILES:
        lens, cur = [], None
        for line in open(path):
            line = line.rstrip("\n")
            if line[:1] in (">", "<", "/", "+"):
                if cur is not None:
                    lens.append(cur)
                cur = 0
            else:
                cur += len(line)
        lens.append(cur)
        out.append(lens)
    return list(zip(*out))


def _run(binary, opts):
    r = subprocess.run([binary] + opts.split() + FILES, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"{os.path.basename(binary)} {opts}: rc {r.returncode}\n{r.stderr[-2000:]}"
    return r.stdout.splitlines()


@pytest.mark.skipif(not all(os.path.exists(p) for p in [OURS, REF] + FILES),
                    reason="test_prog builds missing (make -C oracle ref, where the reference tree is present)")
@pytest.mark.parametrize("opts", OPTION_SETS)
def test_reference_test_prog_prints_the_same(opts):
    ours = _run(OURS, opts)
    ref = _run(REF, opts)
    assert len(ref) == 20000, f"reference printed {len(ref)} lines"
    assert len(ours) == len(ref)
    if "global" in opts.split() and "-t" in opts.split():
        lens = _lengths()
        undefined = {str(i + 1) for i, (ql, tl) in enumerate(lens) if ql % 8 == 0 or tl % 8 == 0}
        key = lambda line: line.split("\t", 1)[0].split("=", 1)[1]
        o = {key(l): l for l in ours}
        r = {key(l): l for l in ref}
        assert o.keys() == r.keys()
        diff = [k for k in r if o[k] != r[k]]
        assert all(k in undefined for k in diff), [(o[k], r[k]) for k in diff if k not in undefined][:3]
        assert len(undefined) < len(r) // 5
        return
    so, sr = sorted(ours), sorted(ref)
    diff = [(a, b) for a, b in zip(so, sr) if a != b]
    assert not diff, f"{len(diff)} differing lines, first: {diff[0]}"
