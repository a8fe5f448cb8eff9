"""Drop-in programs on the GPU: deterministic runs (fixed seed, fixed number of
generations) give the same result for every lookup structure -- the six
structures are bit-exact with each other -- and the same result twice."""
import os
import re
import subprocess

import numpy as np
import pytest

import ts_b200 as T
from conftest import PKG

pytestmark = pytest.mark.gpu
BIN = os.path.join(PKG, "bin")
ALGS = T.STRUCT_NAMES


@pytest.fixture(scope="module")
def instances(tmp_path_factory):
    if not os.path.exists(os.path.join(BIN, "mdp_csr")):
        subprocess.run(["make", "-s", "-C", PKG, "cli"], check=True)
    d = tmp_path_factory.mktemp("inst")
    u, v, w, _ = T.gen.erdos_renyi(500, 10.0, 5)
    mdp = d / "mdp.txt"
    with open(mdp, "w") as f:
        f.write(f"%%MatrixMarket\n500 500 {len(u)}\n")
        for a, b, c in zip(u, v, w):
            f.write(f"{a + 1} {b + 1} {c}\n")
    u, v, w, _ = T.gen.erdos_renyi(300, 8.0, 6)
    mx = d / "maxbs.txt"
    with open(mx, "w") as f:
        f.write(f"300 300 {len(u)}\n")
        for a, b, c in zip(u, v, w):
            f.write(f"{a + 1} {b + 1} {c / 1000:.3f}\n")
    return mdp, mx, d


def run(args):
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout, r.stderr


def mdp_summary(out):
    best = re.search(r"found best objective = (\S+)", out).group(1)
    iters = re.search(r"average number of iterations per run = (\S+)", out).group(1)
    trials = re.findall(r"finish \d+-th trial,nbr_gen = (\d+),best_cost = (\S+),", out)
    return best, iters, trials


def test_mdp_program_same_result_for_every_structure(gpu, instances):
    mdp, _, _ = instances
    ref = None
    for alg in ALGS:
        out, _ = run([os.path.join(BIN, f"mdp_{alg}"), str(mdp), "sparse", "100", "2", "--seed", "3",
                      "--gens", "2", "--iters", "300", "--m", "25", "--quiet"])
        s = mdp_summary(out)
        assert len(s[2]) == 2 and all(t[0] == "1" for t in s[2])
        if ref is None:
            ref = s
        assert s == ref, alg
    out2, _ = run([os.path.join(BIN, "mdp_csr"), str(mdp), "sparse", "100", "2", "--seed", "3",
                   "--gens", "2", "--iters", "300", "--m", "25", "--quiet"])
    assert mdp_summary(out2) == ref


def test_maxbs_program_same_result_for_every_structure(gpu, instances):
    _, mx, d = instances
    ref = None
    for alg in ALGS:
        part = d / f"part_{alg}.txt"
        out, _ = run([os.path.join(BIN, f"maxbs_{alg}"), str(mx), "-seed", "4", "-gens", "3", "-maxiter", "400",
                      "-piter", "40", "-gamma", "20", "-p", "4", "-out", str(part)])
        best = re.search(r"\(f_best\):\s+(\S+)", out).group(1)
        verify = re.search(r"fitness:\s+(\S+)", out).group(1)
        iters = re.search(r"Iteracoes total:\s+(\d+)", out).group(1)
        lines = part.read_text().splitlines()
        assert lines[0].startswith("# Particao encontrada por MACUT")
        p = np.array([int(x.split()[1]) for x in lines[2:]])
        assert len(p) == 300 and (p == 1).sum() == 150
        key = (best, verify, iters, tuple(p))
        if ref is None:
            ref = key
        assert key == ref, alg


def test_runner_runs_and_resumes(gpu, instances, tmp_path):
    _, mx, _ = instances
    g = tmp_path / "graphs"
    g.mkdir()
    (g / "tiny.txt").write_text(mx.read_text())
    res = tmp_path / "res"
    cmd = ["python", os.path.join(PKG, "cli", "run_experimentos.py"), "--problema", "maxbs", "--alg", "csr",
           "--repeticoes", "2", "--tempo", "1", "--maxiter", "200", "--grafos", str(g), "--resultados", str(res),
           "--seed", "9"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    logs = sorted((res / "maxbisection" / "CSR").glob("tiny_*.txt"))
    assert len(logs) == 2 and all(x.read_text().endswith("[EXPERIMENTOS] EXIT_CODE=0\n") for x in logs)
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert "retomadas: 2" in r.stdout
