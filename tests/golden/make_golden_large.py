"""Reference goldens for the two full-size workloads that take the reference
CPU path tens of minutes: written to large.json in this directory.

Runs in a container that holds the reference sources; IG_REFERENCE must name
that checkout.  Uses oracle/_ref/ref_driver (oracle/Makefile, target `ref`),
i.e. the reference's own C++ FillAdjList / AdjList / SolveIndependentSet:

  vt16         1,000,000 VT-style n=16 words (workloads.vt16_words, seed 16),
               editDist 5.  FillAdjList (src/SparseMat.cpp:567-615) on
               `--threads` threads gives the edge set (independent of the
               thread count); its (u<v) pair list, rows then columns
               ascending, is hashed.  The T=1 codebook is the FindMinDel loop
               over AdjList::FromBinaryFile of that pair file (the loader of
               the reference's GPU path, whose neighbour order equals
               FillAdjList's with one thread).
  clustered14  the 64 Zipf clusters of workloads.clustered14() (1,000,000
               n=14 words, editDist 4).  Each cluster is solved by the
               reference's SolveIndependentSet (src/SparseMat.cpp:784-851) with
               one FillAdjList thread -- the thread count its cluster worker
               pool passes when 16 workers share 16 threads (:985-1000).  Per
               cluster: size, matrix ones, codebook length and the sha256 of
               the codebook as int32 word ids within the cluster.

Usage:  IG_REFERENCE=<reference checkout> python tests/golden/make_golden_large.py [--only vt16|clustered14]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from indexgen_b200 import workloads as W  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
OUT = os.path.join(HERE, "large.json")


def sh(*args, cwd=None) -> str:
    r = subprocess.run([str(a) for a in args], check=True, capture_output=True, text=True, cwd=cwd)
    return r.stdout


def last_json(out: str) -> dict:
    return json.loads([l for l in out.splitlines() if l.startswith("{")][-1])


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def write_cands(path, words, L):
    with open(path, "w") as f:
        f.write("\n".join(W.to_strings(words, L)) + "\n")


def make_vt16(tmp, threads):
    words = W.vt16_words(1_000_000, 16)
    cfile = os.path.join(tmp, "vt16.txt")
    write_cands(cfile, words, 16)
    efile = os.path.join(tmp, "vt16_edges.bin")
    t0 = time.time()
    info = last_json(sh(DRIVER, "edges", cfile, 5, threads, efile, cwd=tmp))
    t_fill = time.time() - t0
    e = np.fromfile(efile, dtype="<i4").reshape(-1, 2)
    assert len(e) == info["edges"]
    sfile = os.path.join(tmp, "vt16_sel.bin")
    g = last_json(sh(DRIVER, "gpuload", len(words), efile, sfile, cwd=tmp))
    sel = np.fromfile(sfile, dtype="<i4")[1:]
    deg = np.bincount(e.reshape(-1), minlength=len(words))
    rec = {"L": 16, "min_ed": 5, "seed": 16, "N": int(len(words)), "words_sha256": sha(words.astype("<u4")),
           "edges": int(len(e)), "edges_sha256": sha(e), "degree_sha256": sha(deg.astype("<i8")),
           "ones": int(g["ones"]), "codebook_t1": int(len(sel)), "codebook_t1_sha256": sha(sel.astype("<i4")),
           "codebook_t1_head": sel[:64].tolist(), "fill_threads": threads, "fill_seconds": round(t_fill, 1)}
    print("vt16:", rec["N"], "words,", rec["edges"], "edges, codebook", rec["codebook_t1"], f"({t_fill:.0f} s)")
    return rec


def solve_cluster(args):
    tmp, c, words = args
    cfile = os.path.join(tmp, f"c{c}.txt")
    write_cands(cfile, words, 14)
    sfile = os.path.join(tmp, f"s{c}.bin")
    info = last_json(sh(DRIVER, "solve", cfile, 4, 1, sfile, cwd=tmp))
    s = np.fromfile(sfile, dtype="<i4")
    assert s[0] == len(s) - 1
    sel = s[1:]
    return c, {"N": int(len(words)), "words_sha256": sha(np.asarray(words, "<u4")), "ones": int(info["ones"]),
               "codebook": int(len(sel)), "codebook_sha256": sha(sel.astype("<i4"))}


def make_clustered14(tmp, procs):
    clusters = W.clustered14()
    t0 = time.time()
    out = [None] * len(clusters)
    order = sorted(range(len(clusters)), key=lambda c: -len(clusters[c]))
    with cf.ThreadPoolExecutor(procs) as ex:
        for c, rec in ex.map(solve_cluster, [(tmp, c, clusters[c]) for c in order]):
            out[c] = rec
    dt = time.time() - t0
    print("clustered14:", len(clusters), "clusters,", sum(r["codebook"] for r in out), "codewords", f"({dt:.0f} s)")
    return {"L": 14, "min_ed": 4, "k": len(clusters), "total": int(sum(len(c) for c in clusters)),
            "fill_threads_per_cluster": 1, "clusters": out}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=("vt16", "clustered14"))
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 8)
    a = ap.parse_args()
    if not os.environ.get("IG_REFERENCE"):
        sys.exit("IG_REFERENCE must name the reference checkout (the driver is built from it)")
    if not os.path.exists(DRIVER):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref",
                        f"REF={os.environ['IG_REFERENCE']}"], check=True)
    info = json.load(open(OUT)) if os.path.exists(OUT) else {}
    with tempfile.TemporaryDirectory() as tmp:
        if a.only in (None, "clustered14"):
            info["clustered14"] = make_clustered14(tmp, a.threads)
            json.dump(info, open(OUT, "w"), indent=1)
        if a.only in (None, "vt16"):
            info["vt16"] = make_vt16(tmp, a.threads)
            json.dump(info, open(OUT, "w"), indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
