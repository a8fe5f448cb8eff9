"""Pins the oracle to the reference's own CUDA programs.

The fixtures in tests/golden/ were recorded from the unmodified reference
programs (built from their sources with oracle/build_ref.sh, traced through
oracle/ref_shim.c) by tests/golden/make_golden.py on a B200.  For each case the
oracle must reproduce the reference's start solution and, iteration by
iteration, the ArgMax (flat index, value) the reference copied to the host,
plus every MaxBS perturbation gain.
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(p for p in glob.glob(os.path.join(HERE, "golden", "*.npz")) if "__" not in os.path.basename(p))


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    return z, meta


def instance(spec):
    import importlib.util
    spec_mod = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec_mod)
    spec_mod.loader.exec_module(mod)
    return mod.instance(spec)


def test_fixtures_present():
    assert len(GOLDEN) >= 6, "golden fixtures missing; run tests/golden/make_golden.py on a GPU box"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_reference_trace(path):
    z, meta = load(path)
    n, u, v, w = instance(meta["spec"])
    rp = meta["params"]
    K = meta["records"]
    assert not meta["programs_differing"], f"reference programs disagree: {meta['programs_differing']}"
    if meta["problem"] == "mdp":
        m = rp["m"]
        g = O.Graph(n, u, v, w, drop_self_loops=True)
        init = O.mdp_random_initial(n, m, rp["seed"])
        inside = np.zeros(n, bool)
        inside[init] = True
        start = np.concatenate([np.nonzero(inside)[0], np.nonzero(~inside)[0]])
        np.testing.assert_array_equal(start, z["init"])
        r = O.run(g, O.MDP, m=m, max_iter=K, tenure_policy=O.TENURE_REF, seed=rp["seed"],
                  initial=None, threads=1)
        tr = r.trace
        assert len(tr) == K, (len(tr), K)
        np.testing.assert_array_equal(tr["idx"], z["idx"])
        np.testing.assert_array_equal(tr["key"].astype(np.float64), z["value"])
    else:
        g = O.Graph(n, u, v, w, drop_self_loops=False)
        part = O.maxbs_random_partition(n, rp["seed"])
        start = np.concatenate([np.nonzero(part == 0)[0], np.nonzero(part == 1)[0]])
        np.testing.assert_array_equal(start, z["init"])
        r = O.run(g, O.MAXBS, max_iter=K, tenure_policy=O.TENURE_REF, maxt=rp["maxt"],
                  piter=rp["piter"], gamma=rp["gamma"], seed=rp["seed"], initial=None, threads=1)
        tr = r.trace
        moves = tr[tr["kind"] == O.REC_MOVE]
        assert len(moves) == K
        np.testing.assert_array_equal(moves["idx"], z["idx"])
        np.testing.assert_array_equal(moves["key"].astype(np.float64), z["value"])
        pert = tr[tr["kind"] == O.REC_PERTURB]
        n_moves_before = np.searchsorted(np.nonzero(tr["kind"] == O.REC_MOVE)[0],
                                         np.nonzero(tr["kind"] == O.REC_PERTURB)[0])
        # The traced reference process exits at its K-th ArgMax, before a
        # perturbation that would follow the last move.
        keep = n_moves_before < K
        np.testing.assert_array_equal(pert["key"][keep].astype(np.float64), z["perturb_value"])
        np.testing.assert_array_equal(n_moves_before[keep], z["perturb_at"])
