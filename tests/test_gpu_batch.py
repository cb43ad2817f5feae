"""Batches (fmm_batch_create / fmm_batch_dgemm) through the C ABI.

A batch partitions every problem exactly as the single-problem entry point does and
applies the products to each C element in the same order, so its results must be
bit-identical to calling fmm_dgemm_dev (or the plain GEMM) per problem; the per-problem
result is itself checked against the oracle by the parity tests.  Here additionally:
one problem against the oracle, a CUDA-graph capture and replay, and the work-unit
accounting.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import algebra, build, runtime as rt  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    rt.load_library()


_plans = {}


def plan_for(name):
    if name is None:
        return None
    if name not in _plans:
        algs, levels = [], []
        for part in name.split("_"):
            a, lv = part.split("-")
            algs.append(a)
            levels.append(int(lv))
        _plans[name] = rt.Plan.from_levels(algs, levels)
    return _plans[name]


def operands(shapes, seed):
    g = torch.Generator(device=DEV).manual_seed(seed)
    As, Bs, Cs = [], [], []
    for m, n, k in shapes:
        As.append(rt.colmajor(m, k, device=DEV).uniform_(-1, 1, generator=g))
        Bs.append(rt.colmajor(k, n, device=DEV).uniform_(-1, 1, generator=g))
        Cs.append(rt.colmajor(m, n, device=DEV).uniform_(-1, 1, generator=g))
    return As, Bs, Cs


def one_by_one(shapes, names, As, Bs, Cs):
    out = []
    for (m, n, k), name, A, B, C in zip(shapes, names, As, Bs, Cs):
        c = C.clone()
        if name is None:
            rt.plain_gemm(A, B, c)
        else:
            rt.fmm_gemm(plan_for(name), A, B, c, "abc")
        out.append(c)
    return out


MIXED = [
    ((1030, 1001, 777), "222-1"),         # fringes on every side, k strip in the second launch
    ((517, 389, 263), "232-1"),
    ((700, 900, 1000), "222-1_333-1"),
    ((256, 256, 256), None),
    ((1, 1, 1), None),
    ((300, 257, 5), "333-1"),             # k smaller than the plan's k split: strips only
    ((2048, 2048, 2048), "222-1"),        # pre-summed operands (first launch)
    ((1100, 900, 1300), "222-2"),
    ((129, 4000, 64), None),
]


def test_batch_is_identical_to_one_call_per_problem():
    shapes = [s for s, _ in MIXED]
    names = [nm for _, nm in MIXED]
    As, Bs, Cs = operands(shapes, 1)
    want = one_by_one(shapes, names, As, Bs, Cs)
    batch = rt.Batch(shapes, [plan_for(nm) for nm in names])
    got = [c.clone() for c in Cs]
    batch.run(As, Bs, got)
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    for (shape, nm), w, g in zip(MIXED, want, got):
        assert torch.equal(w, g), (shape, nm, (w - g).abs().max().item())
    assert batch.units(0) > 0 and batch.units(1) > 0
    batch.close()


def test_batch_problem_matches_oracle(oracle_lib):
    m, n, k = 333, 290, 301
    A = np.asfortranarray(np.random.default_rng(3).uniform(-1, 1, (m, k)))
    B = np.asfortranarray(np.random.default_rng(4).uniform(-1, 1, (k, n)))
    C = np.asfortranarray(np.random.default_rng(5).uniform(-1, 1, (m, n)))
    want = C.copy(order="F")
    oracle_lib.bl_dgemm(A, B, want)
    dA = rt.colmajor(m, k, device=DEV).copy_(torch.from_numpy(A))
    dB = rt.colmajor(k, n, device=DEV).copy_(torch.from_numpy(B))
    dC = rt.colmajor(m, n, device=DEV).copy_(torch.from_numpy(C))
    p = plan_for("222-1")
    batch = rt.Batch([(m, n, k), (m, n, k)], [p, None])
    dC2 = dC.clone()
    batch.run([dA, dA], [dB, dB], [dC, dC2])
    torch.cuda.synchronize()
    bound = algebra.error_bound(p.algebra, m, n, k, 1.0, 1.0, 1.0)
    assert np.abs(dC.cpu().numpy() - want).max() <= 2 * bound
    assert np.linalg.norm(dC2.cpu().numpy() - want) / np.linalg.norm(want) <= 1e-13


def test_batch_runs_from_a_cuda_graph():
    shapes = [(640, 512, 384), (1030, 1001, 777), (96, 200, 1500)]
    names = [None, "222-1", "232-1"]
    As, Bs, Cs = operands(shapes, 7)
    want = one_by_one(shapes, names, As, Bs, Cs)
    batch = rt.Batch(shapes, [plan_for(nm) for nm in names])
    got = [c.clone() for c in Cs]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):  # warm-up outside the capture
        batch.run(As, Bs, [c.clone() for c in Cs], stream=s)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        batch.run(As, Bs, got)
    for c, c0 in zip(got, Cs):
        c.copy_(c0)
    g.replay()
    torch.cuda.synchronize()
    for w, x in zip(want, got):
        assert torch.equal(w, x)
    g.replay()  # a second replay adds the same update again
    torch.cuda.synchronize()
    for w, x, c0 in zip(want, got, Cs):
        assert torch.allclose(x - c0, 2 * (w - c0), rtol=1e-12, atol=1e-12)
    del g
    batch.close()


def test_batch_rejects_mismatched_operands():
    batch = rt.Batch([(64, 64, 64)])
    A = rt.colmajor(64, 32, device=DEV)
    with pytest.raises(rt.FmmError):
        batch.run([A], [A], [A])
    batch.close()


def test_batch_with_64_row_tiles_matches_oracle(oracle_lib):
    """Per-problem tile heights (fmm_batch_create_tiled): a 64-row tile gives each row of
    consumer warps half of its columns, every element getting a full tile's DMMAs in order, so
    the results match the oracle and equal single calls bit for bit."""
    shapes = [(700, 500, 640), (2048, 2048, 2048), (300, 257, 512), (1030, 1001, 777)]
    names = [None, "222-1", None, "222-1"]
    tiles = [64, 64, 128, 64]
    rngs = [np.random.default_rng(40 + i) for i in range(len(shapes))]
    host = [(np.asfortranarray(r.uniform(-1, 1, (m, k))), np.asfortranarray(r.uniform(-1, 1, (k, n))),
             np.asfortranarray(r.uniform(-1, 1, (m, n)))) for r, (m, n, k) in zip(rngs, shapes)]
    dev = [tuple(rt.colmajor(*x.shape, device=DEV).copy_(torch.from_numpy(x)) for x in h) for h in host]
    batch = rt.Batch(shapes, [plan_for(nm) for nm in names], tiles=tiles)
    batch.run([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev])
    torch.cuda.synchronize()
    batch.close()
    assert rt.load_library().fmm_device_status(1) == 0
    singles = one_by_one(shapes, names, [d[0] for d in dev], [d[1] for d in dev],
                         [rt.colmajor(*h[2].shape, device=DEV).copy_(torch.from_numpy(h[2])) for h in host])
    for (m, n, k), nm, (A, B, C), d, w in zip(shapes, names, host, dev, singles):
        assert torch.equal(d[2], w), (m, n, k, nm)
        want = C.copy(order="F")
        if nm is None:
            oracle_lib.bl_dgemm(A, B, want)
        else:
            pl = plan_for(nm).algebra
            dims, nterms, rows, cols, coefs = rt.plan_tables(pl)
            oracle_lib.fmm((dims, pl.rank, nterms, rows, cols, coefs), "abc", A, B, want)
        got = d[2].cpu().numpy()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-13, (m, n, k, nm)


def test_batch_rejects_unknown_tile_height():
    with pytest.raises(rt.FmmError):
        rt.Batch([(64, 64, 64)], tiles=[96])
