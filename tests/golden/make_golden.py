"""Regenerate the golden fixtures in this directory from the REFERENCE's own code.

Runs in a container that holds the reference sources; IG_REFERENCE must name
that checkout.  It builds oracle/_ref/ref_driver from those
sources (oracle/Makefile, target `ref`) and records what the reference's C++
path outputs:

  uniform11.npz   the CPU-runnable workload (20,000 uniform n=11 strings, seed
                  12345, maxRun 3, GC [0.3,0.7], editDist 3): candidates, sorted
                  (u<v) edges, and the SolveIndependentSet codebooks (as vertex
                  ids) for FillAdjList thread counts 16, 8 and 1.
  small_cases.npz seeded small sets for n = 4..16, editDist 2..5 with planted
                  near neighbours and duplicates: edges, codebooks for T=1 and
                  T=3, and the reference's own neighbour lists m[] at T=3.
  predicate.npz   20,000 (a, b, minED) queries answered by
                  EditDistanceBandedAtLeast (include/EditDistance.hpp:368).
  linear.json     the LinearCode candidate lists of the shipped codebook header
                  Codebooks/N11/N11-ED3-GC0.3-0.7-RUN0.txt (N and "Number of Ones")
                  and of the n=12 editDist 4 [12,9,3]+coset workload (N, edges,
                  sha256 of edges and of the T=1 codebook built through
                  AdjList::FromBinaryFile, the reference GPU path's loader).
  shipped.npz     the first 1,500 words of a few shipped codebooks, which must
                  contain no conflicting pair.

Usage:  python tests/golden/make_golden.py [--skip-large]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from indexgen_b200 import workloads as W  # noqa: E402

REF = os.environ.get("IG_REFERENCE", "")
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def sh(*args, cwd=None) -> str:
    r = subprocess.run([str(a) for a in args], check=True, capture_output=True, text=True, cwd=cwd)
    return r.stdout


def last_json(out: str) -> dict:
    return json.loads([l for l in out.splitlines() if l.startswith("{")][-1])


def write_cands(path, words, L):
    with open(path, "w") as f:
        f.write("\n".join(W.to_strings(words, L)) + "\n")


def read_i32(path):
    return np.fromfile(path, dtype="<i4")


def ref_edges(tmp, words, L, d, T=8):
    cf = os.path.join(tmp, "c.txt")
    write_cands(cf, words, L)
    ef = os.path.join(tmp, "e.bin")
    info = last_json(sh(DRIVER, "edges", cf, d, T, ef, cwd=tmp))
    e = read_i32(ef).reshape(-1, 2)
    assert len(e) == info["edges"] and info["ones"] == 2 * len(e)
    return e


def ref_solve(tmp, words, L, d, T):
    cf = os.path.join(tmp, "c.txt")
    write_cands(cf, words, L)
    of = os.path.join(tmp, "s.bin")
    sh(DRIVER, "solve", cf, d, T, of, cwd=tmp)
    s = read_i32(of)
    assert s[0] == len(s) - 1
    return s[1:].astype(np.int32)


def ref_adj(tmp, words, L, d, T):
    cf = os.path.join(tmp, "c.txt")
    write_cands(cf, words, L)
    of = os.path.join(tmp, "a.bin")
    sh(DRIVER, "adj", cf, d, T, of, cwd=tmp)
    raw = read_i32(of)
    n = int(raw[0])
    ptr = np.zeros(n + 1, np.int64)
    lists = []
    k = 1
    for i in range(n):
        deg = int(raw[k])
        lists.append(raw[k + 1 : k + 1 + deg])
        ptr[i + 1] = ptr[i] + deg
        k += 1 + deg
    adj = np.concatenate(lists).astype(np.int32) if lists else np.zeros(0, np.int32)
    return ptr, adj


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def mutate(rng, digits, n_edits):
    """Apply n_edits random substitutions / (delete+insert) pairs, keeping length."""
    s = list(digits)
    L = len(s)
    for _ in range(n_edits):
        op = rng.integers(0, 3)
        if op == 0:
            p = rng.integers(0, L)
            s[p] = (s[p] + rng.integers(1, 4)) % 4
        else:
            p = rng.integers(0, L)
            del s[p]
            q = rng.integers(0, L)
            s.insert(q, int(rng.integers(0, 4)))
    return s


def planted_set(rng, L, n_base, per_base):
    base = rng.integers(0, 4, size=(n_base, L))
    rows = []
    for b in base:
        rows.append(list(b))
        for _ in range(per_base):
            rows.append(mutate(rng, b, int(rng.integers(0, 5))))
    rows = np.array(rows)
    rng.shuffle(rows)
    return W.pack_digits(rows)


def make_uniform11(tmp):
    w = W.uniform11_candidates()
    assert len(w) == 14375
    e = ref_edges(tmp, w, 11, 3, T=8)
    sel = {T: ref_solve(tmp, w, 11, 3, T) for T in (16, 8, 1)}
    np.savez_compressed(os.path.join(HERE, "uniform11.npz"), words=w, L=11, min_ed=3, edges=e.astype(np.int32),
                        sel16=sel[16], sel8=sel[8], sel1=sel[1])
    print("uniform11:", len(w), "words,", len(e), "edges, codebooks", {k: len(v) for k, v in sel.items()})


def make_small(tmp):
    rng = np.random.default_rng(20251203)
    out = {}
    cases = [(L, d) for L in (10, 11, 12, 13, 14, 15, 16) for d in (3, 4, 5)]
    cases += [(4, 2), (6, 3), (8, 2), (9, 4), (16, 2)]
    for L, d in cases:
        w = planted_set(rng, L, 90, 3)
        # a few exact duplicates
        w = np.concatenate([w, w[rng.integers(0, len(w), 6)]])
        e = ref_edges(tmp, w, L, d)
        s1 = ref_solve(tmp, w, L, d, 1)
        s3 = ref_solve(tmp, w, L, d, 3)
        ap, adj = ref_adj(tmp, w, L, d, 3)
        key = f"L{L}_d{d}"
        out[key + "_words"] = w
        out[key + "_edges"] = e.astype(np.int32)
        out[key + "_sel1"] = s1
        out[key + "_sel3"] = s3
        out[key + "_adj3_ptr"] = ap
        out[key + "_adj3"] = adj
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **out)
    print("small_cases:", len(cases), "cases")


def make_predicate(tmp):
    rng = np.random.default_rng(7)
    qa, qb, ql, qd = [], [], [], []
    for i in range(20000):
        L = int(rng.integers(1, 17))
        a = rng.integers(0, 4, size=L)
        b = np.array(mutate(rng, a, int(rng.integers(0, 7)))) if rng.random() < 0.8 else rng.integers(0, 4, size=L)
        qa.append(W.pack_digits(a[None, :])[0])
        qb.append(W.pack_digits(b[None, :])[0])
        ql.append(L)
        qd.append(int(rng.integers(1, 7)))
    qf = os.path.join(tmp, "q.txt")
    with open(qf, "w") as f:
        for a, b, L, d in zip(qa, qb, ql, qd):
            f.write(f"{W.to_strings([a], L)[0]} {W.to_strings([b], L)[0]} {d}\n")
    of = os.path.join(tmp, "q.bin")
    sh(DRIVER, "predfile", qf, of, cwd=tmp)
    res = np.fromfile(of, dtype=np.uint8)
    assert len(res) == len(qa)
    np.savez_compressed(os.path.join(HERE, "predicate.npz"), a=np.array(qa, np.uint32), b=np.array(qb, np.uint32),
                        L=np.array(ql, np.int32), min_ed=np.array(qd, np.int32), at_least=res)
    print("predicate:", len(res), "queries,", int((res == 0).sum()), "below minED")


def make_linear(tmp, skip_large):
    info = {}
    cfg = {
        "core": {"lenStart": 11, "lenEnd": 11, "editDist": 3},
        "constraints": {"maxRun": 0, "minGC": 0.3, "maxGC": 0.7},
        "performance": {"threads": 8, "saveInterval": 0, "use_gpu": False},
        "method": {"name": "LinearCode", "linearCode": {
            "minHD": 3, "biasMode": "manual", "rowPermMode": "manual", "colPermMode": "manual",
            "bias": [3, 0, 2, 3, 1, 1, 1, 3, 2, 3, 3], "rowPerm": [4, 0, 5, 1, 6, 3, 7, 2],
            "colPerm": [8, 9, 6, 10, 3, 5, 0, 4, 7, 2, 1]}},
    }
    jf = os.path.join(tmp, "n11.json")
    json.dump(cfg, open(jf, "w"))
    cf = os.path.join(tmp, "n11.txt")
    sh(DRIVER, "gen", jf, cf, cwd=tmp)
    words = W.from_strings([l.strip() for l in open(cf) if l.strip()])
    e = ref_edges(tmp, words, 11, 3)
    info["n11_header"] = {"source": "Codebooks/N11/N11-ED3-GC0.3-0.7-RUN0.txt", "L": 11, "min_ed": 3,
                          "max_run": 0, "min_gc": 0.3, "max_gc": 0.7,
                          "bias": cfg["method"]["linearCode"]["bias"],
                          "row_perm": cfg["method"]["linearCode"]["rowPerm"],
                          "col_perm": cfg["method"]["linearCode"]["colPerm"],
                          "N": int(len(words)), "words_sha256": sha(words.astype("<u4")),
                          "edges": int(len(e)), "edges_sha256": sha(e.astype("<i4"))}
    print("n11 header:", info["n11_header"]["N"], info["n11_header"]["edges"])
    cfg2 = {
        "core": {"lenStart": 12, "lenEnd": 12, "editDist": 4},
        "constraints": {"maxRun": 3, "minGC": 0.3, "maxGC": 0.7},
        "performance": {"threads": 8, "saveInterval": 0, "use_gpu": False},
        "method": {"name": "LinearCode", "linearCode": {"minHD": 3, "biasMode": "random", "randomSeed": 20251203}},
    }
    jf = os.path.join(tmp, "l12.json")
    json.dump(cfg2, open(jf, "w"))
    cf = os.path.join(tmp, "l12.txt")
    sh(DRIVER, "gen", jf, cf, cwd=tmp)
    words = W.from_strings([l.strip() for l in open(cf) if l.strip()])
    rec = {"L": 12, "min_ed": 4, "seed": 20251203, "N": int(len(words)), "words_sha256": sha(words.astype("<u4"))}
    if not skip_large:
        e = ref_edges(tmp, words, 12, 4, T=os.cpu_count() or 8)
        ef = os.path.join(tmp, "l12_edges.bin")
        e.astype("<i4").tofile(ef)
        sf = os.path.join(tmp, "l12_sel.bin")
        g = last_json(sh(DRIVER, "gpuload", len(words), ef, sf, cwd=tmp))
        sel = read_i32(sf)[1:]
        deg = np.bincount(e.reshape(-1), minlength=len(words))
        rec.update({"edges": int(len(e)), "edges_sha256": sha(e.astype("<i4")),
                    "degree_sha256": sha(deg.astype("<i8")),
                    "codebook_t1": int(len(sel)), "codebook_t1_sha256": sha(sel.astype("<i4")),
                    "codebook_t1_head": sel[:64].tolist(), "ones": int(g["ones"])})
        print("linear12:", rec["N"], rec["edges"], rec["codebook_t1"])
    else:
        old = json.load(open(os.path.join(HERE, "linear.json"))) if os.path.exists(os.path.join(HERE, "linear.json")) else {}
        rec.update({k: v for k, v in old.get("linear12", {}).items() if k not in rec})
    info["linear12"] = rec
    json.dump(info, open(os.path.join(HERE, "linear.json"), "w"), indent=1)


def parse_codebook(path):
    words, L, d = [], None, None
    with open(path) as f:
        body = False
        for line in f:
            line = line.strip()
            if line.startswith("Code Length:"):
                L = int(line.split()[-1])
            if line.startswith("Min Codebook Edit Distance:"):
                d = int(line.split()[-1])
            if line.startswith("====="):
                body = True
                continue
            if body and line:
                words.append(line)
    return words, L, d


def make_shipped(tmp):
    files = ["Codebooks/N11/N11-ED3-GC0.3-0.7-RUN0.txt", "Codebooks/N12/N12-ED4-GC0.3-0.7-RUN0.txt",
             "Codebooks/N14/N14-ED5-GC0.3-0.7-RUN0.txt", "Codebooks/N16/N16-ED5-GC0.3-0.7-RUN0.txt"]
    out = {}
    for rel in files:
        p = os.path.join(REF, rel)
        if not os.path.exists(p):
            print("missing", rel)
            continue
        words, L, d = parse_codebook(p)
        w = W.from_strings(words[:1500])
        e = ref_edges(tmp, w, L, d)
        assert len(e) == 0, rel
        key = os.path.basename(rel).split("-RUN")[0].replace(".", "p").replace("-", "_")
        out[key + "_words"] = w
        out[key + "_meta"] = np.array([L, d], np.int32)
    np.savez_compressed(os.path.join(HERE, "shipped.npz"), **out)
    print("shipped:", sorted(k for k in out if k.endswith("_meta")))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-large", action="store_true")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    if not REF:
        sys.exit("IG_REFERENCE must name the reference checkout")
    sh("make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}")
    with tempfile.TemporaryDirectory() as tmp:
        steps = {"uniform11": lambda: make_uniform11(tmp), "small": lambda: make_small(tmp),
                 "predicate": lambda: make_predicate(tmp), "shipped": lambda: make_shipped(tmp),
                 "linear": lambda: make_linear(tmp, a.skip_large)}
        for k, f in steps.items():
            if not a.only or k in a.only.split(","):
                f()


if __name__ == "__main__":
    main()
