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
