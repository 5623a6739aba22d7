"""The reference's own C++ program (src/IndexGen.cpp) on the library.

oracle/Makefile (target `host`, built in a container that holds the
reference sources) links the reference's unmodified objects three ways:
IndexGen_ref (as shipped), IndexGen_ref_seeded (RandomCluster replaced by a
seeded stand-in so clustered runs repeat) and IndexGen_lib (also with
FillAdjListGPU replaced by indexgen_b200/host/FillAdjListGPU.cpp, linked
against libindexgen_cuda.so).  These tests run the programs end to end from
a JSON config, as a user of the reference would, and compare the codebook
files they write:

  * use_gpu=true on the library == use_gpu=false (the reference CPU path,
    FillAdjList with one thread, whose neighbour order the GPU loader
    reproduces), codebook lines and "Number of Ones in Matrix";
  * the unmodified program's script boundary (use_gpu=true runs
    $INDEXGEN_PYTHON $INDEXGEN_ROOT/src/gpu_graph_generator.py) on
    indexgen_b200/gpu_graph_generator.py gives the same codebook, and so does
    its VerifyDist GPU branch (same script);
  * the clustered loop (src/SparseMat.cpp:927-1095), whose worker pool calls
    FillAdjListGPU from 16 threads on one shared context, equals the CPU run
    with the same clusters;
  * the library's resident clustered solve (ig_cluster_solve) equals the
    reference's own loop: codebook and the size after every iteration;
  * the n=12 editDist-4 [12,9,3] GF(4) workload generated by the program's own
    LinearCode generator gives the reference's T=1 codebook (tests/golden).
"""
import glob
import hashlib
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

HOST = os.path.join(ROOT, "oracle", "_ref", "host")
BIN = {k: os.path.join(HOST, "IndexGen_" + k) for k in ("ref", "ref_seeded", "lib")}


def need(*kinds):
    for k in kinds:
        if not os.path.exists(BIN[k]):
            pytest.skip(f"{BIN[k]} not built (make -C oracle host REF=<reference checkout>)")


def uniform11_file(tmp_path):
    """Config 1's input as a FileRead file: 20,000 uniform n=11 strings (seed
    12345), the reference's '===' separator line first."""
    from indexgen_b200 import workloads as W

    p = tmp_path / "cands.txt"
    if not p.exists():
        w = W.uniform_words(20000, 11, 12345)
        p.write_text("===\n" + "\n".join(W.to_strings(w, 11)) + "\n")
    return str(p)


def config(tmp_path, name, *, use_gpu, threads=1, length=11, min_ed=3, method=None, clustering=None, verify=False):
    cfg = {
        "dir": str(tmp_path / name),
        "core": {"lenStart": length, "lenEnd": length, "editDist": min_ed},
        "constraints": {"maxRun": 3, "minGC": 0.3, "maxGC": 0.7},
        "performance": {"threads": threads, "saveInterval": 0, "use_gpu": use_gpu, "max_gpu_memory_gb": 10.0},
        "method": method or {"name": "FileRead", "fileRead": {"input_file": uniform11_file(tmp_path)}},
        "verify": verify,
    }
    if clustering:
        cfg["clustering"] = clustering
    path = tmp_path / (name + ".json")
    path.write_text(json.dumps(cfg))
    return str(path), cfg["dir"]


def script_root(tmp_path):
    """An INDEXGEN_ROOT whose src/gpu_graph_generator.py is the two-line shim
    onto indexgen_b200.gpu_graph_generator."""
    src = tmp_path / "shim" / "src"
    src.mkdir(parents=True, exist_ok=True)
    (src / "gpu_graph_generator.py").write_text(
        f"import sys; sys.path.insert(0, {ROOT!r})\n"
        "from indexgen_b200.gpu_graph_generator import main; sys.exit(main())\n")
    return str(tmp_path / "shim")


def run(kind, cfg_path, out_dir, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([BIN[kind], "--config", cfg_path], capture_output=True, text=True, env=e, timeout=timeout,
                       cwd=os.path.dirname(cfg_path))
    assert r.returncode == 0, f"{kind} exited {r.returncode}:\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}"
    books = glob.glob(os.path.join(out_dir, "CodeSize-*.txt"))
    assert len(books) == 1, f"expected one codebook file in {out_dir}, found {books}"
    lines = open(books[0]).read().splitlines()
    end = max(i for i, l in enumerate(lines) if l.startswith("===="))
    ones = [int(l.split(":")[1]) for l in lines[:end] if l.startswith("Number of Ones in Matrix")]
    sizes = [int(s.replace(",", "")) for s in re.findall(r"Candidate set size = ([\d,]+)", r.stdout)]
    return {"codebook": lines[end + 1:], "ones": ones[0] if ones else None, "sizes": sizes, "log": r.stdout}


def sizes_after(res):
    """Size of the candidate set after each iteration of the clustered loop."""
    return res["sizes"][1:] + [len(res["codebook"])]


CLUSTERING = {"enabled": True, "k": 16, "verbose": True, "convergenceIterations": 3, "method": "random_cluster"}


@pytest.fixture(scope="module")
def cpu_plain(tmp_path_factory):
    """The reference CPU path on config 1 with one FillAdjList thread."""
    need("ref")
    tmp = tmp_path_factory.mktemp("cpu_plain")
    cfg, out = config(tmp, "cpu", use_gpu=False, threads=1)
    res = run("ref", cfg, out)
    assert len(res["codebook"]) == 7535 and res["ones"] == 41742  # the reference's own numbers
    return res


@pytest.fixture(scope="module")
def cpu_clustered(tmp_path_factory):
    need("ref_seeded")
    tmp = tmp_path_factory.mktemp("cpu_clustered")
    cfg, out = config(tmp, "cpu_cl", use_gpu=False, threads=16, clustering=CLUSTERING)
    return run("ref_seeded", cfg, out, env={"IG_CLUSTER_SEED": "7"})


def test_reference_cluster_loop_equals_oracle(cpu_clustered, oracle):
    """The oracle's restatement of the clustered loop is the reference's own
    loop (same seeded clusters): codebook and per-iteration sizes."""
    from indexgen_b200 import workloads as W

    w = W.uniform11_candidates()
    ids, sizes = oracle.cluster_solve(w, 11, 3, 16, 3, 7, 50)
    assert W.to_strings(w[ids], 11) == cpu_clustered["codebook"]
    assert sizes.tolist() == sizes_after(cpu_clustered)
    assert cpu_clustered["sizes"][0] == len(w)


def test_script_drop_in_usage_errors(tmp_path):
    """Wrong argument counts and values exit 1 with a message, as the
    reference script does (no device work)."""
    mod = [sys.executable, "-m", "indexgen_b200.gpu_graph_generator"]
    r = subprocess.run(mod + ["a", "b"], capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 1 and "Usage" in r.stdout
    r = subprocess.run(mod + ["a", "b", "three"], capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 1 and "bad argument" in r.stdout
    r = subprocess.run(mod + [str(tmp_path / "missing.txt"), str(tmp_path / "e.bin"), "3"], capture_output=True,
                       text=True, cwd=ROOT)
    assert r.returncode == 1 and "[Error]" in r.stdout


@pytest.mark.gpu
def test_program_on_library_equals_cpu_path(tmp_path, cpu_plain):
    need("lib")
    cfg, out = config(tmp_path, "lib", use_gpu=True, threads=16, verify=True)
    env = {"INDEXGEN_ROOT": script_root(tmp_path), "INDEXGEN_PYTHON": sys.executable}
    res = run("lib", cfg, out, env=env)
    assert "libindexgen_cuda:" in res["log"], "the program did not build its graph through the library"
    assert res["codebook"] == cpu_plain["codebook"]
    assert res["ones"] == cpu_plain["ones"]
    # VerifyDist's GPU branch runs the script drop-in on the codebook
    assert "Vector distance SUCCESS" in res["log"]


@pytest.mark.gpu
def test_unmodified_program_on_script_drop_in(tmp_path, cpu_plain):
    need("ref")
    cfg, out = config(tmp_path, "script", use_gpu=True, threads=16)
    env = {"INDEXGEN_ROOT": script_root(tmp_path), "INDEXGEN_PYTHON": sys.executable}
    res = run("ref", cfg, out, env=env)
    assert "[GPU] Done. Wrote" in res["log"]
    assert res["codebook"] == cpu_plain["codebook"]
    assert res["ones"] == cpu_plain["ones"]


@pytest.mark.gpu
def test_program_clustered_worker_pool_on_library(tmp_path, cpu_clustered):
    """16 workers of the clustered loop call FillAdjListGPU at once on one
    shared context; every iteration and the final codebook equal the CPU run."""
    need("lib")
    cfg, out = config(tmp_path, "lib_cl", use_gpu=True, threads=16, clustering=CLUSTERING)
    res = run("lib", cfg, out, env={"IG_CLUSTER_SEED": "7"})
    assert res["codebook"] == cpu_clustered["codebook"]
    assert res["sizes"] == cpu_clustered["sizes"]


@pytest.mark.gpu
def test_resident_cluster_solve_equals_reference_loop(cpu_clustered, igctx):
    from indexgen_b200 import cluster_solve
    from indexgen_b200 import workloads as W

    w = W.uniform11_candidates()
    ids, sizes = cluster_solve(w, 11, 3, 16, converge_iters=3, seed=7, ctx=igctx)
    assert W.to_strings(w[ids], 11) == cpu_clustered["codebook"]
    assert sizes.tolist() == sizes_after(cpu_clustered)


@pytest.mark.gpu
def test_program_linear12_on_library(tmp_path):
    """Config 2 end to end: the program's own LinearCode generator (biasMode
    random, seed 20251203), the graph on the library, the reference greedy."""
    need("lib")
    from indexgen_b200 import workloads as W

    gold = json.load(open(os.path.join(GOLDEN, "linear.json")))["linear12"]
    method = {"name": "LinearCode", "linearCode": {"minHD": 3, "biasMode": "random", "randomSeed": 20251203}}
    cfg, out = config(tmp_path, "lib12", use_gpu=True, threads=16, length=12, min_ed=4, method=method)
    res = run("lib", cfg, out, timeout=900)
    assert res["ones"] == 2 * gold["edges"] == gold["ones"]
    words = W.linear12_candidates()
    idx = {s: i for i, s in enumerate(W.to_strings(words, 12))}
    sel = np.array([idx[s] for s in res["codebook"]], dtype="<i4")
    assert len(sel) == gold["codebook_t1"]
    assert hashlib.sha256(sel.tobytes()).hexdigest() == gold["codebook_t1_sha256"]
