"""Batched solves: many independent systems of uneven n in one persistent
launch (captured in a CUDA graph), checked system by system against the
oracle: the factors against gefa_ref_nopvt's restatement in FP64 (relative
bound) and the solutions against the FP64 solve; every reference-generator
system must pass the reference's validation (residn < 1,
linpack_benchmark.hpp:416-417,465)."""
import numpy as np
import pytest

import oracle
from hpcc_fpga_b200 import batch as hb

FLT_EPS = float(np.finfo(np.float32).eps)


def test_batch_packing(lp):
    b = hb.Batch([3, 5, 8], [1, 2, 3])
    s = b.systems
    assert [x.lda for x in s] == [4, 8, 8]
    assert s[1].a_off == 3 * 4 and s[2].a_off == 3 * 4 + 5 * 8
    assert s[1].b_off == 4 and s[2].b_off == 4 + 2 * 8
    b.mat(1)[:] = 7.0
    assert np.all(b.A[s[1].a_off:s[1].a_off + 5 * 8].reshape(5, 8)[:, :5] == 7.0)
    assert b.rhs(2).shape == (3, 8)


def test_log_uniform_sizes(lp):
    n = hb.log_uniform_sizes(4096, 32, 1024, 7)
    assert n.min() >= 32 and n.max() <= 1024
    assert abs(np.median(np.log(n)) - 0.5 * (np.log(32) + np.log(1024))) < 0.1
    assert np.array_equal(n, hb.log_uniform_sizes(4096, 32, 1024, 7))


def _run(ctx, dev, b, cfg=None):
    dA, dB = dev.put(b.A), dev.put(b.B)
    st = ctx.batch_solve(b.systems, dA.data_ptr(), dB.data_ptr(), cfg)
    return dev.get(dA), dev.get(dB), st


def _check(b, A_out, B_out, ref_inputs):
    for i, s in enumerate(b.systems):
        A0, R0 = ref_inputs[i]
        lu = A_out[s.a_off:s.a_off + s.n * s.lda].reshape(s.n, s.lda)[:, :s.n]
        want = oracle.gefa_nopvt(A0.astype(np.float64))
        rel = np.abs(lu - want).max() / np.abs(want).max()
        assert rel < 64 * FLT_EPS * max(1.0, np.log2(s.n)), f"system {i} (n={s.n}) factor rel {rel}"
        X = B_out[s.b_off:s.b_off + s.nrhs * s.ldb].reshape(s.nrhs, s.ldb)[:, :s.n]
        for q in range(s.nrhs):
            x64 = oracle.gesl_nopvt(want, R0[q].astype(np.float64))
            x32 = oracle.gesl_nopvt(oracle.gefa_nopvt(A0), R0[q])
            tol = 8 * np.abs(x32 - x64).max() + 64 * FLT_EPS * np.abs(x64).max()
            assert np.abs(X[q] - x64).max() <= tol, f"system {i} (n={s.n}) rhs {q}"


@pytest.mark.gpu
def test_batch_mixed_sizes_against_oracle(ctx, dev):
    sizes = [1, 2, 5, 31, 32, 64, 100, 127, 128, 129, 200, 256, 257, 300, 513, 777, 1024]
    nrhs = [1, 2, 3, 1, 8, 16, 4, 2, 1, 5, 7, 3, 1, 2, 8, 1, 4]
    b = hb.Batch(sizes, nrhs)
    rng = np.random.default_rng(11)
    ref = []
    for i, n in enumerate(sizes):
        A, _, _ = oracle.gen_baseline(n, seed=100 + i, margin=1.0)
        b.mat(i)[:, :] = A
        b.rhs(i)[:, :] = rng.uniform(-1, 1, (nrhs[i], n)).astype(np.float32)
        ref.append((A.copy(), b.rhs(i).copy()))
    A_out, B_out, st = _run(ctx, dev, b)
    assert st["systems"] == len(sizes) and st["seconds"] > 0
    _check(b, A_out, B_out, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("nb", [16, 32])
@pytest.mark.parametrize("small", [64, 128])
def test_batch_configurations(ctx, dev, lp, nb, small):
    sizes = [48, 96, 160, 300, 600]
    b = hb.Batch(sizes, [2] * len(sizes))
    rng = np.random.default_rng(5)
    ref = []
    for i, n in enumerate(sizes):
        A, _, _ = oracle.gen_baseline(n, seed=200 + i)
        b.mat(i)[:, :] = A
        b.rhs(i)[:, :] = rng.uniform(-1, 1, (2, n)).astype(np.float32)
        ref.append((A.copy(), b.rhs(i).copy()))
    cfg = lp.LpBatchConfig()
    lp.lib().lp_batch_default_config(cfg)
    cfg.small_n_max = small
    for k in range(5):
        cfg.nb[k] = nb
    A_out, B_out, _ = _run(ctx, dev, b, cfg)
    _check(b, A_out, B_out, ref)


@pytest.mark.gpu
def test_batch_reference_generator_validates(ctx, dev):
    """Reference-generator systems (U(0,1), diagonal = row sum), b = A*ones:
    every solution passes the reference's residn < 1."""
    sizes = [16, 64, 128, 256, 512]
    b = hb.Batch(sizes, [1] * len(sizes))
    normb = []
    for i, n in enumerate(sizes):
        A, rhs, _, nb_ = oracle.gen_reference(n)
        b.mat(i)[:, :] = A
        b.rhs(i)[0, :] = rhs
        normb.append(nb_)
    _, B_out, _ = _run(ctx, dev, b)
    for i, s in enumerate(b.systems):
        x = B_out[s.b_off:s.b_off + s.n]
        residn, _ = oracle.residn(x, normb[i])
        assert residn < 1.0 and np.all(np.abs(x - 1.0) < 1e-3)


@pytest.mark.gpu
def test_batch_graph_replay_and_autotune(ctx, dev):
    b = hb.make_batch(count=96, lo=32, hi=1024, seed=7)
    dA, dB = dev.put(b.A), dev.put(b.B)
    st1 = ctx.batch_solve(b.systems, dA.data_ptr(), dB.data_ptr())
    X1 = dev.get(dB)
    dA.copy_(dev.put(b.A))
    dB.copy_(dev.put(b.B))
    dev.torch.cuda.synchronize()
    st2 = ctx.batch_solve(b.systems, dA.data_ptr(), dB.data_ptr())
    X2 = dev.get(dB)
    assert st1["graph_replayed"] == 0 and st2["graph_replayed"] == 1
    assert np.array_equal(X1, X2)
    dA.copy_(dev.put(b.A))
    dB.copy_(dev.put(b.B))
    dev.torch.cuda.synchronize()
    cfg = ctx.batch_autotune(b.systems, dA.data_ptr(), dB.data_ptr())
    assert cfg.small_n_max in (64, 128) and all(x in (16, 32) for x in cfg.nb)
    X0 = dev.get(dB)                      # autotune leaves the inputs untouched
    assert np.array_equal(X0, b.B)
    ctx.batch_solve(b.systems, dA.data_ptr(), dB.data_ptr())
    X3 = dev.get(dB)
    assert np.allclose(X3, X1, rtol=1e-4, atol=1e-5)


@pytest.mark.gpu
def test_batch_rejects_bad_systems(ctx, lp):
    bad = [lp.LpSystem(2048, 1, 2048, 2048, 0, 0)]
    with pytest.raises(lp.LpError) as e:
        ctx.batch_solve(bad, 1 << 20, 1 << 20)
    assert e.value.status == lp.LP_E_INVALID
    with pytest.raises(lp.LpError):
        ctx.batch_solve([lp.LpSystem(8, 17, 8, 8, 0, 0)], 1 << 20, 1 << 20)


def _refined_batch(lp, sizes, nrhs, seed=3):
    """A batch of seeded diagonally dominant systems whose FP64 right-hand
    sides have exact solutions: x_q = (q + 1) * ones."""
    b = hb.Batch(sizes, nrhs)
    B64 = np.zeros(b.B.shape, np.float64)
    for i, s in enumerate(b.systems):
        A, b64, _ = lp.generate_baseline(s.n, seed + i, 1.0)
        b.mat(i)[:, :] = A
        for q in range(s.nrhs):
            B64[s.b_off + q * s.ldb:s.b_off + q * s.ldb + s.n] = (q + 1) * b64
    return b, B64


def _x_of(b, X, i):
    s = b.systems[i]
    return X[s.b_off:s.b_off + s.nrhs * s.ldb].reshape(s.nrhs, s.ldb)[:, :s.n]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "bf16"])
def test_batch_refined_reaches_hpl_threshold(ctx, dev, lp, prec):
    """Every system of a mixed batch (whole-in-shared-memory and blocked
    sizes, 1..16 right-hand sides) refines in FP64 to the HPL threshold
    (gmres.c:182-193) inside the one launch, and the FP64-oracle error (the
    exact solutions are (q + 1) * ones) is far below FP32 accuracy."""
    sizes = [1, 7, 32, 100, 128, 129, 200, 256, 300, 513, 777, 1024]
    nrhs = [1, 2, 16, 3, 1, 5, 8, 1, 4, 2, 16, 3]
    b, B64 = _refined_batch(lp, sizes, nrhs)
    dA, dB = dev.put(b.A), dev.put(B64)
    dX = dev.empty(B64.shape, np.float64)
    st, its, res = ctx.batch_solve_ir(b.systems, dA.data_ptr(), dB.data_ptr(), dX.data_ptr(), prec, max_iters=10)
    X = dev.get(dX)
    assert st["systems"] == len(sizes)
    for i, s in enumerate(b.systems):
        x = _x_of(b, X, i)
        want = np.arange(1, s.nrhs + 1, dtype=np.float64)[:, None]
        err = np.abs(x - want).max() / want.max()
        assert res[i] <= 16.0, f"system {i} (n={s.n}): hpl {res[i]}"
        assert its[i] <= 5, f"system {i} (n={s.n}): {its[i]} refinements"
        assert err < 1e-10, f"system {i} (n={s.n}): err {err}"


@pytest.mark.gpu
def test_batch_bf16_factors_are_the_tensor_core_form(ctx, dev, lp):
    """The BF16 form's factors of a blocked-path system differ from the FP32
    form's by the BF16 rounding of the trailing updates (not more, not zero),
    while systems solved whole in shared memory are factored in FP32 by both."""
    sizes, nrhs = [64, 512], [1, 1]
    b, B64 = _refined_batch(lp, sizes, nrhs, seed=9)
    out = {}
    for prec in ("f32", "bf16"):
        dA, dB = dev.put(b.A), dev.put(B64)
        dX = dev.empty(B64.shape, np.float64)
        ctx.batch_solve_ir(b.systems, dA.data_ptr(), dB.data_ptr(), dX.data_ptr(), prec, max_iters=0)
        out[prec] = dev.get(dA)
    s0, s1 = b.systems
    small = slice(s0.a_off, s0.a_off + s0.n * s0.lda)
    big = slice(s1.a_off, s1.a_off + s1.n * s1.lda)
    assert np.array_equal(out["f32"][small], out["bf16"][small])
    d = np.abs(out["f32"][big] - out["bf16"][big]).max() / np.abs(out["f32"][big]).max()
    assert 0.0 < d < 2e-3, d


@pytest.mark.gpu
def test_batch_host_buffers_match_device_call_and_replay(ctx, dev, lp):
    """lp_batch_solve (host buffers) returns exactly what the device entry
    point returns, and the second device call replays the captured graph with
    identical results."""
    sizes, nrhs = [50, 130, 400, 900], [2, 1, 3, 8]
    b, B64 = _refined_batch(lp, sizes, nrhs, seed=21)
    A_host = b.A.copy()
    X_host, st_h, its_h, res_h = ctx.batch_solve_host(b.systems, A_host, B64, "bf16", max_iters=10)
    runs = []
    dA, dB = dev.put(b.A), dev.put(B64)
    dX = dev.empty(B64.shape, np.float64)
    for _ in range(2):  # the same buffers both times: the second call replays the graph
        dA.copy_(dev.torch.from_numpy(b.A).cuda())
        dX.zero_()
        dev.torch.cuda.synchronize()
        st, its, res = ctx.batch_solve_ir(b.systems, dA.data_ptr(), dB.data_ptr(), dX.data_ptr(), "bf16",
                                          max_iters=10)
        runs.append((dev.get(dA), dev.get(dX), st, its, res))
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][0], runs[1][0])
    assert runs[1][2]["graph_replayed"] == 1
    assert np.array_equal(X_host, runs[0][1]) and np.array_equal(A_host, runs[0][0])
    assert np.array_equal(its_h, runs[0][3]) and np.array_equal(res_h, runs[0][4])


@pytest.mark.gpu
def test_batch_refined_rejects_bad_arguments(ctx, dev, lp):
    b, B64 = _refined_batch(lp, [40], [1])
    dA, dB = dev.put(b.A), dev.put(B64)
    dX = dev.empty(B64.shape, np.float64)
    with pytest.raises(lp.LpError) as e:
        ctx.batch_solve_ir(b.systems, dA.data_ptr(), dB.data_ptr(), dX.data_ptr(), "fp8")
    assert e.value.status == lp.LP_E_INVALID
    with pytest.raises(lp.LpError) as e:
        ctx.batch_solve_ir(b.systems, dA.data_ptr(), dB.data_ptr(), dX.data_ptr(), "bf16", max_iters=-1)
    assert e.value.status == lp.LP_E_INVALID
