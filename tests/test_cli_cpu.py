"""Drop-in programs on the CPU: instance readers (exact fixed-point weights,
the reference's data-set rules) and argument handling.  No GPU needed: the
programs parse and report without touching a device (--check-instance)."""
import os
import subprocess

import pytest

from conftest import PKG

BIN = os.path.join(PKG, "bin")


def run(args, **kw):
    return subprocess.run(args, capture_output=True, text=True, timeout=60, **kw)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not all(os.path.exists(os.path.join(BIN, b)) for b in ("mdp_csr", "maxbs_csr", "convert_mwis")):
        subprocess.run(["make", "-s", "-C", PKG, "cli"], check=True)


def check_mdp(path, dataset, *extra):
    r = run([os.path.join(BIN, "mdp_csr"), str(path), dataset, "1", "1", "--check-instance", *extra])
    assert r.returncode == 0, r.stderr
    return [int(x) for x in r.stdout.split()]


def test_mdp_sparse_one_based_self_loops_comments(tmp_path):
    f = tmp_path / "g.txt"
    f.write_text("%%MatrixMarket\n% comment\n\n5 5 4\n1 2 3\n2 2 9\n3 5 4\n4 1 1\n")
    n, m, e, scale, wsum, rounded = check_mdp(f, "sparse")
    # self-loop 2-2 dropped (GPU-MDP-CSR.cu:340); m = 100 for 'sparse'
    assert (n, m, e, scale, wsum, rounded) == (5, 100, 3, 1, 8, 0)


def test_mdp_mdg_zero_based_decimals_exact(tmp_path):
    f = tmp_path / "g.txt"
    f.write_text("4 2\n0 1 1.25\n0 2 2.5\n1 3 0.125\n2 3 10\n")
    n, m, e, scale, wsum, rounded = check_mdp(f, "MDG-a")
    assert (n, m, e, scale) == (4, 2, 4, 1000)
    assert wsum == 1250 + 2500 + 125 + 10000 and rounded == 0


def test_mdp_b2500_doubles_weights(tmp_path):
    f = tmp_path / "g.txt"
    f.write_text("3 2\n1 2 7\n2 3 -4\n")
    n, m, e, scale, wsum, _ = check_mdp(f, "b2500")
    assert (n, m, e, scale, wsum) == (3, 1000, 2, 1, 2 * (7 - 4))


def test_mdp_p3000_and_nenad_sizes(tmp_path):
    f = tmp_path / "g.txt"
    f.write_text("6 1\n1 6 2\n")
    assert check_mdp(f, "p30005000")[:3] == [6, 3, 1]
    f.write_text("6 1\n0 5 2\n")
    assert check_mdp(f, "nenad")[:3] == [6, 100, 1]
    assert check_mdp(f, "nenad", "--m", "2")[1] == 2


def test_mdp_bad_inputs(tmp_path):
    f = tmp_path / "g.txt"
    f.write_text("3 3 1\n1 9 2\n")
    r = run([os.path.join(BIN, "mdp_csr"), str(f), "sparse", "1", "1", "--check-instance"])
    assert r.returncode != 0 and "Read Date Error" in r.stderr
    r = run([os.path.join(BIN, "mdp_csr"), str(f), "nosuchset", "1", "1", "--check-instance"])
    assert r.returncode != 0 and "data set is wrong" in r.stderr
    r = run([os.path.join(BIN, "mdp_csr"), str(f), "sparse"])
    assert r.returncode == 0 and "Input the following parameters" in r.stdout


def test_maxbs_converter_format_thousandths(tmp_path):
    f = tmp_path / "g.txt"
    # converter output: (w_u + w_v) / 1000 with three decimals (convert_mwis.cpp:19-31)
    f.write_text("5 5 4\n1 2 1.085\n2 3 0.002\n3 3 4.000\n4 5 12.340\n")
    r = run([os.path.join(BIN, "maxbs_csr"), str(f), "-check-instance"])
    assert r.returncode == 0, r.stderr
    n, m, e, scale, wsum, rounded = [int(x) for x in r.stdout.split()]
    # self-loop kept (GPU-MAXBS-CSR.cu:160-166); m = floor(n/2)
    assert (n, m, e, scale, wsum, rounded) == (5, 2, 4, 1000, 1085 + 2 + 4000 + 12340, 0)


def test_maxbs_rounding_flag_and_options(tmp_path):
    f = tmp_path / "g.txt"
    f.write_text("3 3 1\n1 2 0.12345\n")
    r = run([os.path.join(BIN, "maxbs_csr"), str(f), "-check-instance"])
    assert r.returncode == 0
    assert r.stdout.split()[3:] == ["1000", "123", "1"]
    r = run([os.path.join(BIN, "maxbs_csr"), str(f), "-bogus"])
    assert r.returncode == 1 and "Opcao desconhecida" in r.stderr
    r = run([os.path.join(BIN, "maxbs_csr")])
    assert r.returncode == 1 and "Uso:" in r.stderr


def test_program_names_select_structures():
    for alg in ("csr", "hash", "wswap", "csr-bitset", "csr-bb", "csr-bitset-bb"):
        assert os.path.islink(os.path.join(BIN, f"mdp_{alg}"))
        assert os.path.islink(os.path.join(BIN, f"maxbs_{alg}"))


def test_runner_resume_marker_and_layout(tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location("runner", os.path.join(PKG, "cli", "run_experimentos.py"))
    R = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(R)
    log = tmp_path / "x_1.txt"
    log.write_text("Comando: x\n\nstuff\n[EXPERIMENTOS] EXIT_CODE=0\n")
    assert R.concluido(log)
    log.write_text("Comando: x\n\n[EXPERIMENTOS] EXIT_CODE=1\n")
    assert not R.concluido(log)
    g = tmp_path / "g.txt"
    g.write_text("7 7 0\n")
    assert R.quantidade_vertices(g) == 7
    g.write_text("7 8 0\n")
    with pytest.raises(ValueError):
        R.quantidade_vertices(g)
    assert R.ALGOS["csr-bb"] == "CSR-BuscaBinaria"


def _mwis_fixture(root, name, n, edges, weights):
    d = root / name
    d.mkdir(parents=True)
    (d / "conflict_graph.txt").write_text(f"{n} {len(edges)}\n" + "".join(f"{a} {b}\n" for a, b in edges))
    (d / "node_weights.txt").write_text("".join(f"{v} {wt}\n" for v, wt in weights))


def test_converter_known_answer(tmp_path):
    inp, out = tmp_path / "in", tmp_path / "out"
    # duplicates in both orientations, a negative weight sum, sums >= 1000
    _mwis_fixture(inp, "tiny", 4, [(2, 1), (1, 2), (3, 4), (4, 1), (3, 4), (1, 3)],
                  [(1, 1500), (2, 7), (3, -20), (4, 999)])
    r = run([os.path.join(BIN, "convert_mwis"), str(inp), str(out), "tiny"])
    assert r.returncode == 0, r.stderr
    assert "2 duplicatas removidas" in r.stdout
    assert (out / "tiny.txt").read_text() == (
        "4 4 4\n"
        "1 2 1.507\n"
        "1 3 1.480\n"
        "1 4 2.499\n"
        "3 4 0.979\n")
    _mwis_fixture(inp, "neg", 2, [(1, 2)], [(1, -1500), (2, -7)])
    r = run([os.path.join(BIN, "convert_mwis"), str(inp), str(out), "neg"])
    assert (out / "neg.txt").read_text() == "2 2 1\n1 2 -1.507\n"


def test_converter_errors(tmp_path):
    inp, out = tmp_path / "in", tmp_path / "out"
    _mwis_fixture(inp, "bad", 3, [(1, 4)], [(1, 1), (2, 2), (3, 3)])
    r = run([os.path.join(BIN, "convert_mwis"), str(inp), str(out), "bad"])
    assert r.returncode == 1 and "invalida" in r.stderr
    r = run([os.path.join(BIN, "convert_mwis")])
    assert r.returncode == 1 and "Uso:" in r.stderr


REF_CONVERTER = os.path.join(os.path.dirname(PKG), "oracle", "_ref", "convert_mwis")


@pytest.mark.skipif(not os.path.exists(REF_CONVERTER), reason="reference converter not built (oracle/build_ref.sh)")
def test_converter_matches_reference_converter(tmp_path):
    import numpy as np
    rng = np.random.default_rng(8)
    inp = tmp_path / "in"
    names = []
    for k in range(4):
        n = int(rng.integers(5, 400))
        m = int(rng.integers(1, 3 * n))
        a = rng.integers(1, n + 1, size=m)
        b = rng.integers(1, n + 1, size=m)
        keep = a != b
        edges = list(zip(a[keep].tolist(), b[keep].tolist()))
        edges += edges[: len(edges) // 4]  # duplicates
        wts = rng.integers(-5000, 10**9, size=n)
        _mwis_fixture(inp, f"i{k}", n, edges, [(v + 1, int(wts[v])) for v in range(n)])
        names.append(f"i{k}")
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    assert run([os.path.join(BIN, "convert_mwis"), str(inp), str(ours)]).returncode == 0
    assert run([REF_CONVERTER, str(inp), str(ref)]).returncode == 0
    for nm in names:
        assert (ours / f"{nm}.txt").read_bytes() == (ref / f"{nm}.txt").read_bytes(), nm
