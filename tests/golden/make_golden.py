"""Generates the golden fixtures in this directory from the reference.

Run here, where the reference sources exist (the GPU box never reads them):

    make -C oracle                      # builds oracle/_ref from the reference sources
    python tests/golden/make_golden.py [--reference /path/to/reference]

What it writes (all small):
  tagmatch_fixtures.txt   the F/Q filter strings of the reference's
                          test/test_tagmatch.cc and test/test_partitioning.cc
                          (read as text) plus, for test_tagmatch's F/Q, the
                          expected key sets as printed by the reference's own
                          test_matcher binary (keys = filter index).
  io_vectors.json         test/test_io.cc's ASCII -> 24-byte known answers.
  partitions.json         the reference partitioner's output (oracle/_ref/
                          ref_partition) on the test_partitioning fixtures and
                          on seeded random tables.
  matcher_small.npz       the reference test_matcher on small seeded
                          workloads (full per-query key lists).
  config0_digest.npz      per-query (count, multiset hash) digests of the
                          reference test_matcher on the 1M-filter x 10K-query
                          workload (match and match_unique).
"""
import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from tagmatch_b200 import workload  # noqa: E402
from tagmatch_b200.tagmatch import filter_from_string  # noqa: E402


def parse_filter_array(src, name):
    m = re.search(r"static const filter_t " + name + r"\[\] = \{(.*?)\};", src, re.S)
    return re.findall(r'filter_t\("([01]+)"\)', m.group(1))


def parse_test_io(src):
    cases = []
    for m in re.finditer(r'check_binary_encoding\("([01]+)", "((?:\\[0-7]{1,3})+)", (\d+)\)', src):
        raw = m.group(2)
        vals = [int(x, 8) for x in re.findall(r"\\([0-7]{1,3})", raw)]
        cases.append({"ascii": m.group(1), "bytes": vals})
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TAGMATCH_REF"),
                    help="reference source tree (default: $TAGMATCH_REF)")
    ap.add_argument("--skip-config0", action="store_true")
    args = ap.parse_args()
    ref = args.reference
    if not ref:
        raise SystemExit("give the reference source tree with --reference or TAGMATCH_REF")
    if not oracle.have_ref():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle REF=...` first")

    tt = open(os.path.join(ref, "test", "test_tagmatch.cc")).read()
    tp = open(os.path.join(ref, "test", "test_partitioning.cc")).read()
    tio = open(os.path.join(ref, "test", "test_io.cc")).read()
    F, Q = parse_filter_array(tt, "F"), parse_filter_array(tt, "Q")
    PF, PQ = parse_filter_array(tp, "F"), parse_filter_array(tp, "Q")

    # expected match_unique sets for test_tagmatch's misc_subsets, from the
    # reference's own sequential matcher (keys = filter index)
    fw = np.stack([filter_from_string(s) for s in F])
    qw = np.stack([filter_from_string(s) for s in Q])
    ko = np.arange(len(F) + 1, dtype=np.uint32)
    keys = np.arange(len(F), dtype=np.uint32)
    off, ks = oracle.run_ref_matcher(fw, ko, keys, qw, unique=True)
    with open(os.path.join(HERE, "tagmatch_fixtures.txt"), "w") as out:
        out.write("# filter strings from the reference's test/test_tagmatch.cc (F, Q) and\n")
        out.write("# test/test_partitioning.cc (PF, PQ); E lines: reference test_matcher's\n")
        out.write("# match_unique result for Q[i] against F (key j = F[j]).  Generated by make_golden.py.\n")
        for i, s in enumerate(F):
            out.write(f"F {i} {s}\n")
        for i, s in enumerate(Q):
            out.write(f"Q {i} {s}\n")
        for i, s in enumerate(PF):
            out.write(f"PF {i} {s}\n")
        for i, s in enumerate(PQ):
            out.write(f"PQ {i} {s}\n")
        for i in range(len(Q)):
            vals = " ".join(str(int(k)) for k in ks[int(off[i]):int(off[i + 1])])
            out.write(f"E {i} {vals}\n".rstrip() + "\n")

    with open(os.path.join(HERE, "io_vectors.json"), "w") as out:
        json.dump(parse_test_io(tio), out, indent=1)

    # reference partitioner outputs
    parts = {"fixtures": [], "random": []}
    pfw = np.stack([filter_from_string(s) for s in PF])
    pqw = np.stack([filter_from_string(s) for s in PQ])
    for name, fl, maxp in [("small_fib_no_part", pqw[:3], 5), ("small_fib_part", pfw[:3], 5),
                           ("large_fib_part", pfw, 3), ("large_fib_permutation", np.concatenate([pfw, pqw]), 4)]:
        p, m, s = oracle.run_ref_partition(fl, maxp)
        parts["fixtures"].append({"name": name, "max_p": maxp, "filters": fl.tolist(), "partition_of": p.tolist(),
                                  "masks": m.tolist(), "sizes": s.tolist()})
    for seed, n, maxp in [(11, 200, 16), (12, 1000, 64), (13, 5000, 300), (14, 20000, 1000), (15, 3000, 7)]:
        f, _, _ = workload.generate_filters(n, seed)
        p, m, s = oracle.run_ref_partition(f, maxp)
        parts["random"].append({"seed": seed, "n": n, "max_p": maxp, "partition_of": p.tolist(),
                                "masks": m.tolist(), "sizes": s.tolist()})
    with open(os.path.join(HERE, "partitions.json"), "w") as out:
        json.dump(parts, out)

    # small seeded workloads through the reference test_matcher
    small = {}
    for tag, (n, nq, seed) in {"a": (2000, 300, 21), "b": (20000, 500, 22)}.items():
        f, ko_, k_ = workload.generate_filters(n, seed)
        q = workload.generate_queries(nq, f, seed)
        o1, k1 = oracle.run_ref_matcher(f, ko_, k_, q, unique=False)
        o2, k2 = oracle.run_ref_matcher(f, ko_, k_, q, unique=True)
        small.update({f"{tag}_n": n, f"{tag}_nq": nq, f"{tag}_seed": seed, f"{tag}_off": o1, f"{tag}_keys": k1,
                      f"{tag}_uoff": o2, f"{tag}_ukeys": k2})
    np.savez_compressed(os.path.join(HERE, "matcher_small.npz"), **small)

    # the 1M x 10K workload: digests of the reference's own matcher output
    if not args.skip_config0:
        f, ko_, k_, q = workload.config("config0")
        o1, k1 = oracle.run_ref_matcher(f, ko_, k_, q, unique=False)
        c1, h1 = oracle.digest(o1, k1)
        uo = np.zeros_like(o1)
        uk = []
        for i in range(q.shape[0]):
            u = np.unique(k1[int(o1[i]):int(o1[i + 1])])
            uk.append(u)
            uo[i + 1] = uo[i] + u.size
        c2, h2 = oracle.digest(uo, np.concatenate(uk) if uk else np.zeros(0, np.uint32))
        fh = oracle._fin64(f.astype(np.uint64).reshape(-1)).sum(dtype=np.uint64)
        qh = oracle._fin64(q.astype(np.uint64).reshape(-1)).sum(dtype=np.uint64)
        np.savez_compressed(os.path.join(HERE, "config0_digest.npz"), count=c1, hash=h1, ucount=c2, uhash=h2,
                            filters_hash=np.uint64(fh), queries_hash=np.uint64(qh), n_keys=np.uint64(k_.size))


if __name__ == "__main__":
    main()
