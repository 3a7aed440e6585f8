"""GPU tests of the batched products (iarray_b200_batch_*): many independent float64
products of uneven sizes, ragged edge blocks, one grouped persistent launch replayed from a
CUDA graph.  Each output must be byte-identical to the single-product path
(iarray_linalg_matmul on the same operands and partition, same form): the grouped kernel
runs the same per-element accumulation order whatever tile configuration the autotuner
picks, and the encoder is deterministic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(ia, ctx, rng, count, lo=80, hi=300):
    # output chunks (48, 80) fit every output, as iarray_linalg_matmul requires
    As, Bs, cs, bs = [], [], [], []
    for _ in range(count):
        m, n = (int(x) for x in rng.integers(lo, hi + 1, 2))
        k = int(rng.integers(1, hi + 1))
        ca, ba = (64, 64), (16, 16)
        A = rng.uniform(-1, 1, (m, k))
        B = rng.uniform(-1, 1, (k, n))
        As.append(ia.Container.from_numpy(ctx, A, ca, ba))
        Bs.append(ia.Container.from_numpy(ctx, B, ca, ba))
        cs.append((48, 80))
        bs.append((16, 16))
    return As, Bs, cs, bs


@pytest.mark.parametrize("form", ["native", "split"])
def test_batch_matches_single_products(ia, form):
    ctx = ia.Context()
    if form == "split":
        ctx.set_form(ia.FORM_SPLIT, 14)      # the single products' moduli count: byte-identical results
    rng = np.random.default_rng(5)
    As, Bs, cs, bs = _problems(ia, ctx, rng, 12)
    batch = ia.Batch(ctx, As, Bs, cs, bs)
    info = batch.info()
    # grouped decode, product and encode: a few launches per stage for all problems
    assert 0 < info["graph_nodes"] <= 32, info
    if form == "native":
        assert info["tile_config"] in range(8)
        assert len(info["tune_ms"]) == 8
    else:
        assert info["tile_config"] == -1
    for rep in range(2):                                    # graph replays
        outs = batch.run()
        for i, c in enumerate(outs):
            ref = ia.matmul(ctx, As[i], Bs[i], cs[i], bs[i])
            assert c.chunks() == ref.chunks(), (rep, i)
            x, y = As[i].to_numpy(), Bs[i].to_numpy()
            np.testing.assert_allclose(c.to_numpy(), x @ y, rtol=1e-12, atol=1e-12)
            c.free()
            ref.free()
    batch.free()


def test_batch_uneven_sizes_with_empty_and_tiny_problems(ia):
    ctx = ia.Context()
    rng = np.random.default_rng(7)
    shapes = [(1, 1, 1), (1, 700, 3), (700, 1, 5), (3, 4, 700), (129, 257, 65), (0, 5, 5)]
    As, Bs, cs, bs = [], [], [], []
    for m, n, k in shapes:
        As.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (m, k)), (64, 64), (32, 32)))
        Bs.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (k, n)), (64, 64), (32, 32)))
        cs.append((100, 100))
        bs.append((25, 50))
    batch = ia.Batch(ctx, As, Bs, cs, bs)
    outs = batch.run()
    for i, c in enumerate(outs):
        x, y = As[i].to_numpy(), Bs[i].to_numpy()
        assert c.to_numpy().shape == (x.shape[0], y.shape[1])
        np.testing.assert_allclose(c.to_numpy(), x @ y, rtol=1e-12, atol=1e-12)
    batch.free()


@pytest.mark.parametrize("encoder", ["liblz4", "parallel"])
@pytest.mark.parametrize("mixed", [False, True])
def test_batch_encoders_and_mixed_partitions(ia, encoder, mixed):
    """One LZ4 launch encodes the streams of every output when they share one stream size
    (mixed=False); outputs of different block shapes are encoded one by one (mixed=True).
    Either way each output is byte-identical to the single-product path with the same
    encoder."""
    ctx = ia.Context(encoder=ia.ENCODER_PARALLEL if encoder == "parallel" else ia.ENCODER_LIBLZ4)
    rng = np.random.default_rng(11)
    As, Bs, cs, bs = [], [], [], []
    for i in range(6):
        # output chunks (48, 80) fit every output, as iarray_linalg_matmul requires
        m, n = (int(x) for x in rng.integers(80, 200, 2))
        k = int(rng.integers(1, 200))
        As.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (m, k)) * 50.0, (64, 64), (16, 16)))
        Bs.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (k, n)), (64, 64), (16, 16)))
        cs.append((48, 80))
        bs.append((16, 40) if mixed and i % 2 else (16, 16))
    batch = ia.Batch(ctx, As, Bs, cs, bs)
    for rep in range(2):
        outs = batch.run()
        for i, c in enumerate(outs):
            ref = ia.matmul(ctx, As[i], Bs[i], cs[i], bs[i])
            assert c.chunks() == ref.chunks(), (rep, i)
            c.free()
            ref.free()
    batch.free()


def test_batch_rejects_bad_operands(ia):
    ctx = ia.Context()
    a = ia.Container.from_numpy(ctx, np.ones((4, 5)), (4, 5), (2, 5))
    b = ia.Container.from_numpy(ctx, np.ones((6, 3)), (6, 3), (3, 3))
    with pytest.raises(ia.IArrayError) as e:
        ia.Batch(ctx, [a], [b], [(4, 3)], [(2, 3)])
    assert e.value.name == "INVALID_SHAPE"
    f = ia.Container.from_numpy(ctx, np.ones((5, 3), np.float32), (5, 3), (5, 3))
    a32 = ia.Container.from_numpy(ctx, np.ones((4, 5), np.float32), (4, 5), (2, 5))
    with pytest.raises(ia.IArrayError) as e:
        ia.Batch(ctx, [a32], [f], [(4, 3)], [(2, 3)])
    assert e.value.name == "INVALID_DTYPE"


def test_batch_split_autotunes_moduli_within_the_error_bar(ia):
    """With the context's moduli count automatic, the split batch picks the fastest count whose
    normwise error (against 16 moduli) stays within 4x the native FP64 product's."""
    ctx = ia.Context()
    ctx.set_form(ia.FORM_SPLIT)
    rng = np.random.default_rng(9)
    As, Bs, cs, bs = _problems(ia, ctx, rng, 10, lo=200, hi=600)
    batch = ia.Batch(ctx, As, Bs, cs, bs)
    t = batch.split_tuning()
    assert 12 <= t["nterms"] <= 16
    k = 16 - t["nterms"]
    assert t["tune_err"][k] <= 4 * t["err_native"]
    assert all(e >= 0 for e in t["tune_err"]) and t["err_native"] > 0
    outs = batch.run()
    num = den = 0.0
    for i, c in enumerate(outs):
        x, y = As[i].to_numpy(), Bs[i].to_numpy()
        ref = x @ y
        num += float(np.sum((c.to_numpy() - ref) ** 2))
        den += float(np.sum(ref ** 2))
        c.free()
    assert (num / den) ** 0.5 <= 1e-14
    # a second batch of the same shapes takes the cached choice without tuning
    batch2 = ia.Batch(ctx, As, Bs, cs, bs)
    t2 = batch2.split_tuning()
    assert t2["nterms"] == t["nterms"] and t2["tune_ms"] == [-1.0] * 5
    batch.free()
    batch2.free()
