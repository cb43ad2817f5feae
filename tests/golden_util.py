"""Helpers to read the committed golden fixtures (made by tests/golden/make_golden.py)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Must match tests/golden/make_golden.py
CONFIGS = [
    (["222"], [1]),
    (["222"], [2]),
    (["232"], [1]),
    (["333"], [1]),
    (["222", "333"], [1, 1]),
    (["222", "232"], [1, 1]),
    (["424"], [1]),
    (["336"], [1]),
    (["323"], [1]),
    (["classical222_8_24"], [1]),
]
RUN_CONFIGS = [0, 1, 2, 3, 4, 6, 7]


def job_name(algs, levels):
    return "_".join(f"{a}-{l}" for a, l in zip(algs, levels))


def inputs(seed, m, n, k):
    rng = np.random.Generator(np.random.PCG64(seed))
    A = rng.uniform(-1.0, 1.0, size=(m, k))
    B = rng.uniform(-1.0, 1.0, size=(k, n))
    C = rng.uniform(-1.0, 1.0, size=(m, n))
    return np.asfortranarray(A), np.asfortranarray(B), np.asfortranarray(C)


def load_coeffs(algs, levels):
    with open(os.path.join(GOLDEN, f"coeffs_{job_name(algs, levels)}.json")) as fh:
        return json.load(fh)


def load_outputs(algs, levels):
    """-> (meta dict, {f'{pack}_{i}': array})"""
    g = np.load(os.path.join(GOLDEN, f"out_{job_name(algs, levels)}.npz"))
    meta = json.loads(str(g["meta"]))
    return meta, {k: g[k] for k in g.files if k != "meta"}


def golden_cases():
    """(algs, levels, pack, index, (m, n, k), seed, expected C)"""
    out = []
    for ci in RUN_CONFIGS:
        algs, levels = CONFIGS[ci]
        meta, arrs = load_outputs(algs, levels)
        for pack in meta["packs"]:
            for i, shp in enumerate(meta["shapes"]):
                out.append((algs, levels, pack, i, tuple(shp), meta["seed0"] + i, arrs[f"{pack}_{i}"]))
    return out


def plain_cases():
    g = np.load(os.path.join(GOLDEN, "out_plain.npz"))
    meta = json.loads(str(g["meta"]))
    return [(tuple(s), meta["seed0"] + i, g[f"plain_{i}"]) for i, s in enumerate(meta["shapes"])]
