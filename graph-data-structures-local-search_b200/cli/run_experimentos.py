#!/usr/bin/env python3
"""Experiment runner over the B200 drop-in programs (bin/mdp_<alg>, bin/maxbs_<alg>).

Same command line, log layout and resume rule as the reference runner
(src/run_experimentos.py:127-146): one log per (problem, structure, instance,
round) under <results>/<problem>/<Suffix>/<instance>_<round>.txt, each ending
with the marker "[EXPERIMENTOS] EXIT_CODE=<c>"; a log that ends with code 0 is
not run again unless --forcar.  Differences: the programs are built once by
``make`` (no per-structure nvcc call), Max Bisection runs whatever its pair
count (the pair index is 64-bit here, so the reference's int32 guard
:224-235 is gone), and a few options the synthetic configurations need are
passed through (--m, --seed, --iters, --tenure).
"""
from __future__ import annotations

import argparse
import subprocess
import sys
from pathlib import Path

ALGOS = {
    "csr": "CSR",
    "hash": "Hash",
    "wswap": "WSwap",
    "csr-bitset": "CSR-Bitset",
    "csr-bb": "CSR-BuscaBinaria",
    "csr-bitset-bb": "CSR-Bitset-BuscaBinaria",
}
PROBLEMAS = {"mdp": "mdp", "maxbs": "maxbisection"}
MARCADOR_OK = b"\n[EXPERIMENTOS] EXIT_CODE=0\n"
PKG = Path(__file__).resolve().parent.parent


def concluido(log: Path) -> bool:
    if not log.is_file():
        return False
    with log.open("rb") as f:
        f.seek(max(0, log.stat().st_size - 256))
        return f.read().endswith(MARCADOR_OK)


def quantidade_vertices(grafo: Path) -> int:
    with grafo.open("r", encoding="utf-8") as f:
        cab = f.readline().split()
    if len(cab) != 3:
        raise ValueError(f"Cabecalho invalido em {grafo}")
    n, n2, _ = map(int, cab)
    if n < 1 or n2 != n:
        raise ValueError(f"Cabecalho invalido em {grafo}")
    return n


def compilar(forcar: bool) -> bool:
    alvo = ["make", "-s", "-C", str(PKG)] + (["-B"] if forcar else [])
    r = subprocess.run(alvo, check=False)
    if r.returncode != 0:
        print(f"[ERRO] Falha na compilacao ({' '.join(alvo)})", flush=True)
        return False
    return True


def executar(comando: list[str], log: Path, cwd: Path) -> bool:
    with log.open("w", encoding="utf-8") as saida:
        saida.write("Comando: " + " ".join(comando) + "\n\n")
        saida.flush()
        try:
            codigo = subprocess.run(comando, cwd=cwd, stdout=saida, stderr=subprocess.STDOUT,
                                    check=False).returncode
        except OSError as erro:
            saida.write(f"\nFalha ao executar: {erro}\n")
            codigo = 127
        saida.write(f"\n[EXPERIMENTOS] EXIT_CODE={codigo}\n")
    return codigo == 0


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description="Executa MDP e Max Bisection nas instancias.")
    p.add_argument("--problema", choices=["todos", *PROBLEMAS], default="todos")
    p.add_argument("--alg", choices=["todos", *ALGOS], default="todos")
    p.add_argument("--instancia", help="Ex.: MR-D-01; padrao: todas")
    p.add_argument("--repeticoes", type=int, default=10)
    p.add_argument("--tempo", type=int, default=60)
    p.add_argument("--maxiter", type=int, default=1000000)
    p.add_argument("--maxt", type=int, default=200)
    p.add_argument("--forcar", action="store_true", help="Refaz as execucoes concluidas e recompila")
    p.add_argument("--grafos", default="graph_instances", help="pasta das instancias (*.txt)")
    p.add_argument("--resultados", default="Resultados", help="pasta dos logs")
    p.add_argument("--m", type=int, help="MDP: tamanho do conjunto (padrao do formato sparse: 100)")
    p.add_argument("--seed", type=int, help="semente fixa (padrao: relogio, como a referencia)")
    p.add_argument("--iters", type=int, help="MDP: iteracoes por busca tabu (padrao 50000)")
    p.add_argument("--tenure", help="ref ou fixed:T")
    a = p.parse_args(argv)
    if min(a.repeticoes, a.tempo, a.maxiter, a.maxt) < 1:
        p.error("Os parametros numericos devem ser positivos")

    pasta_grafos = Path(a.grafos)
    if a.instancia:
        grafos = [pasta_grafos / (Path(a.instancia).name.removesuffix(".txt") + ".txt")]
    else:
        grafos = sorted(pasta_grafos.glob("*.txt"))
    if not grafos or any(not g.is_file() for g in grafos):
        p.error(f"Instancias nao encontradas em {pasta_grafos}")
    problemas = list(PROBLEMAS) if a.problema == "todos" else [a.problema]
    algoritmos = list(ALGOS) if a.alg == "todos" else [a.alg]
    status = {"ok": 0, "erro": 0, "retomadas": 0, "compilacao": 0}
    total = len(grafos) * len(problemas) * len(algoritmos) * a.repeticoes
    print(f"Instancias: {len(grafos)} | Problemas: {len(problemas)} | Algoritmos: {len(algoritmos)} | "
          f"Repeticoes: {a.repeticoes}")
    print(f"Execucoes planejadas: {total}", flush=True)
    if not compilar(a.forcar):
        status["compilacao"] += 1
        print("\nResumo:", flush=True)
        for k, v in status.items():
            print(f"  {k}: {v}", flush=True)
        return 1
    extra_mdp, extra_maxbs = [], []
    if a.m:
        extra_mdp += ["--m", str(a.m)]
    if a.iters:
        extra_mdp += ["--iters", str(a.iters)]
    if a.tenure:
        extra_mdp += ["--tenure", a.tenure]
        extra_maxbs += ["-tenure", a.tenure]
    for problema in problemas:
        for alg in algoritmos:
            sufixo = ALGOS[alg]
            pasta = Path(a.resultados) / PROBLEMAS[problema] / sufixo
            pasta.mkdir(parents=True, exist_ok=True)
            exe = PKG / "bin" / f"{problema}_{alg}"
            for grafo in grafos:
                try:
                    quantidade_vertices(grafo)
                except (OSError, ValueError) as erro:
                    print(f"[ERRO] {erro}", flush=True)
                    status["erro"] += a.repeticoes
                    continue
                for rodada in range(1, a.repeticoes + 1):
                    log = pasta / f"{grafo.stem}_{rodada}.txt"
                    if not a.forcar and concluido(log):
                        status["retomadas"] += 1
                        continue
                    if problema == "mdp":
                        cmd = [str(exe), str(grafo.resolve()), "sparse", str(a.tempo), "1"] + extra_mdp
                        if a.seed is not None:
                            cmd += ["--seed", str(a.seed + rodada - 1)]
                    else:
                        cmd = [str(exe), str(grafo.resolve()), "-time", str(a.tempo), "-maxiter", str(a.maxiter),
                               "-maxt", str(a.maxt)] + extra_maxbs
                        if a.seed is not None:
                            cmd += ["-seed", str(a.seed + rodada - 1)]
                    print(f"[{problema.upper()} / {sufixo}] {grafo.stem} - rodada {rodada}/{a.repeticoes}",
                          flush=True)
                    if executar(cmd, log, pasta):
                        status["ok"] += 1
                    else:
                        status["erro"] += 1
                        print(f"[ERRO] Execucao falhou. Verifique {log}", flush=True)
    print("\nResumo:", flush=True)
    for k, v in status.items():
        print(f"  {k}: {v}", flush=True)
    return 1 if status["erro"] or status["compilacao"] else 0


if __name__ == "__main__":
    try:
        sys.exit(main())
    except KeyboardInterrupt:
        print("\nInterrompido. Execute o mesmo comando para retomar.", file=sys.stderr)
        sys.exit(130)
