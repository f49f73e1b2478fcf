"""Learned minimizer order: the network's CUDA forward/backward kernels against
the CPU oracle (oracle/mlp_oracle.py), the order table, the minimizer loads the
training data comes from, and what the trained order gains over the default
order on a held-out skewed genome."""
import numpy as np
import pytest

from conftest import partition_digest
from oracle import mlp_oracle
from tests_util import random_reads

U32 = 0xFFFFFFFF


def _counter(**kw):
    from rapidgkc_b200 import KmerCounter
    return KmerCounter(**kw)


# ---- CPU: the oracle and the host-side helpers ---------------------------

def test_oracle_gradient_matches_finite_differences():
    p = 4
    r = np.random.default_rng(0)
    P = mlp_oracle.init_params(p, 1).astype(np.float64)
    v = r.choice(4 ** p, 60, replace=False)
    t = r.normal(0, 1, 60)
    w = r.uniform(0.5, 2, 60)
    _, g = mlp_oracle.loss_and_grad(P, p, v, t, w)
    eps = 1e-6
    for i in r.choice(len(P), 200, replace=False):
        a, b = P.copy(), P.copy()
        a[i] += eps
        b[i] -= eps
        num = (mlp_oracle.loss_and_grad(a, p, v, t, w)[0] - mlp_oracle.loss_and_grad(b, p, v, t, w)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_order_mix_is_a_bijection_and_params_match_layout():
    from rapidgkc_b200 import order
    for p in (3, 6, 11):
        x = order.mix_bits(np.arange(4 ** p), 2 * p, order.ORDER_MIX_KEY)
        assert len(np.unique(x)) == 4 ** p and x.max() < 4 ** p
        assert order.param_count(p) == mlp_oracle.n_params(p)
    assert order.param_count(11) == 44 * 64 + 64 + 64 * 64 + 64 + 64 + 1


# ---- GPU: kernels against the oracle ---------------------------------------

def _random_params(p, seed):
    r = np.random.default_rng(seed)
    P = mlp_oracle.init_params(p, seed)
    return (P + r.normal(0, 0.05, len(P))).astype(np.float32)  # non-zero biases: mixed ReLU states


@pytest.mark.gpu
@pytest.mark.parametrize("p,n", [(11, 700), (11, 128), (5, 300), (3, 64)])
def test_mlp_gradient_matches_oracle(p, n):
    r = np.random.default_rng(p * 100 + n)
    params = _random_params(p, p)
    pm = r.choice(4 ** p, n, replace=False).astype(np.uint32)
    targets = np.zeros(4 ** p, np.float32)
    weights = np.zeros(4 ** p, np.float32)
    targets[pm] = r.normal(1.0, 2.0, n)
    weights[pm] = r.uniform(0.2, 3.0, n)
    norm = 1.0 / float(weights[pm].astype(np.float64).sum())
    with _counter(k=max(p, 15), p=p, partitions=4) as c:
        loss, grad = c.mlp_grad(params, pm, targets, weights, norm)
    L, g = mlp_oracle.loss_and_grad(params, p, pm, targets[pm], weights[pm])
    # FP32 sums of a few hundred terms against float64
    assert abs(loss - L) <= 1e-4 * max(1.0, abs(L))
    scale = np.abs(g).max()
    assert np.abs(grad - g).max() <= 1e-4 * scale + 1e-7


@pytest.mark.gpu
def test_mlp_scores_match_oracle_forward():
    p = 6
    params = _random_params(p, 3)
    with _counter(k=21, p=p, partitions=4) as c:
        s = c.mlp_scores(params)
    ref = mlp_oracle.forward(params, p, np.arange(4 ** p))
    assert np.abs(s - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.gpu
def test_mlp_training_fits_a_known_function():
    """Targets = number of A bases + 2 * [first base is C]: learnable from the
    one-hot input; Adam on all 4^p samples must get close."""
    p = 7
    v = np.arange(4 ** p)
    bases = np.stack([(v >> (2 * (p - 1 - i))) & 3 for i in range(p)], 1)
    t = ((bases == 0).sum(1) + 2.0 * (bases[:, 0] == 1)).astype(np.float32)
    params = mlp_oracle.init_params(p, 0)
    with _counter(k=21, p=p, partitions=4) as c:
        l0 = mlp_oracle.loss_and_grad(params, p, v, t)[0]
        trained, loss = c.mlp_train(params, t, None, epochs=30, batch=512, lr=3e-3, seed=1)
    l1 = mlp_oracle.loss_and_grad(trained, p, v, t)[0]
    assert l1 < 0.02 * l0 and l1 < 0.05
    assert abs(loss - l1) < 0.1  # the library's last-epoch loss is of the same size


@pytest.mark.gpu
def test_order_table_ranks_by_score():
    """The learned order: the K p-mers of highest score get levels that rise
    with the score (chosen last); all others level 0; ranks are distinct and
    their low 2p bits are the tie-break mix of the p-mer."""
    from rapidgkc_b200 import order
    p = 8
    K = 4 ** p // 4  # the default
    params = _random_params(p, 5)
    with _counter(k=21, p=p, partitions=8) as c:
        assert np.count_nonzero(c.mlp_order(params, heavy=1000) >> np.uint32(2 * p)) == 1000
        lut = c.mlp_order(params)
        s = c.mlp_scores(params)
    assert len(np.unique(lut)) == 4 ** p
    assert np.array_equal(lut & np.uint32(4 ** p - 1),
                          order.mix_bits(np.arange(4 ** p), 2 * p, order.ORDER_MIX_KEY).astype(np.uint32))
    level = (lut >> np.uint32(2 * p)).astype(np.int64)
    heavy = np.nonzero(level > 0)[0]
    assert len(heavy) == K
    assert s[heavy].min() >= np.sort(s)[-K]          # the top K by score
    o = heavy[np.argsort(s[heavy], kind="stable")]
    assert np.all(np.diff(level[o]) >= 0) and level.max() <= 2 ** (32 - 2 * p) - 2


@pytest.mark.gpu
def test_learned_order_matches_its_table(oracle):
    """Phase 1 with the learned order (read from its canonical table) gives
    the partitions the oracle gives with the exported rank table."""
    k, p, P = 31, 11, 64
    reads, offs = random_reads(41, 50_000, 4000, 150, 0.004)
    params = _random_params(p, 7)
    with _counter(k=k, p=p, partitions=P) as c:
        lut = c.mlp_order(params)
        c.add_reads(reads, offs)
        pb, ps, pk = c.store_stats()
        pbo, pso, pko, po, stream = oracle.skmgen(reads, offs, k, p, P, lut)
        assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
        for i in range(P):
            assert partition_digest(c.store_export(i)) == partition_digest(stream[int(po[i]):int(po[i + 1])])


@pytest.mark.gpu
def test_minimizer_loads_match_oracle(oracle):
    """Default order: the load of key v = k-mers whose minimizer is v."""
    k, p, P = 31, 11, 16
    reads, offs = random_reads(31, 4000, 3000, 150, 0.01)
    keys = np.concatenate([oracle.kmer_keys(reads[int(offs[i]):int(offs[i + 1])].tobytes(), k, p)
                           for i in range(len(offs) - 1)])
    ref = np.bincount(keys, minlength=4 ** p).astype(np.uint64)
    with _counter(k=k, p=p, partitions=P) as c:
        c.add_reads(reads, offs)
        loads = c.minimizer_loads()
        assert np.array_equal(loads, ref)
        lut = np.random.default_rng(2).permutation(4 ** p).astype(np.uint32)
        c.store_clear()
        c.set_order(lut)
        c.add_reads(reads, offs)
        keys2 = np.concatenate([oracle.kmer_keys(reads[int(offs[i]):int(offs[i + 1])].tobytes(), k, p, lut)
                                for i in range(len(offs) - 1)])
        assert np.array_equal(c.minimizer_loads(), np.bincount(keys2, minlength=4 ** p).astype(np.uint64))


@pytest.mark.gpu
def test_learned_order_gain_on_held_out_skewed_genome():
    """Trained on small skewed genomes of other seeds, the learned order lowers
    the max/mean partition load of a held-out genome against the default
    order, and the (k-mer, count) multiset stays identical."""
    import torch
    from rapidgkc_b200 import order, synth
    params, log = order.train_order("skewed_200m", seeds=range(1, 5), scale=0.01, iterations=2, partitions=256,
                                    epochs=3, batch=8192)
    reads, offs = synth.make_workload("skewed_200m", scale=0.01, seed=404)
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    res = {}
    with _counter(k=31, p=11, partitions=256) as c:
        for name in ("default", "learned"):
            c.set_order(None)
            if name == "learned":
                c.mlp_order(params)
            c.store_clear()
            c.add_reads(d_reads, d_offs)
            st = order.partition_stats(c)
            n, d = c.count(2, U32)
            km, ct = c.result()
            o = np.argsort(km)
            res[name] = (st, d, km[o], ct[o])
    (s0, d0, k0, c0), (s1, d1, k1, c1) = res["default"], res["learned"]
    assert d0 == d1 and np.array_equal(k0, k1) and np.array_equal(c0, c1)
    assert s1["maxmean_kmers"] < 0.9 * s0["maxmean_kmers"], (s0, s1, log.iterations)


@pytest.mark.gpu
def test_trained_network_beats_its_untrained_order():
    """What the trained network adds: the learned order against the same
    order with no network levels (every p-mer ranked by the pseudo-random mix
    alone), on a held-out skewed genome (seed 404, not among the training
    seeds).  The network's levels lower the max/mean partition load in bytes
    (the superkmer bytes phase 2 reads per partition) and the number of
    sub-buckets that overflow shared memory, with identical counts.  The
    max/mean load in k-mers is not asserted: its maximum is the partition of
    the longest poly-A / (AT)n / (CAG)n runs, whose every window holds only the
    run's own p-mers, so no order moves those k-mers."""
    import torch
    from rapidgkc_b200 import order, synth
    params = order.load_order(order.default_order_path(11))[0]
    reads, offs = synth.make_workload("skewed_200m", scale=0.02, seed=404)
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    res = {}
    with _counter(k=31, p=11, partitions=512) as c:
        for name in ("mix", "learned"):
            if name == "mix":
                c.set_order(order.mix_table(11))
            else:
                c.mlp_order(params)
            c.store_clear()
            c.add_reads(d_reads, d_offs)
            st = order.partition_stats(c)
            n, d = c.count(2, U32)
            relisted = c.timings()["overflowed_sub_buckets"]
            km, ct = c.result()
            o = np.argsort(km)
            res[name] = (st, relisted, d, km[o], ct[o])
    (s0, r0, d0, k0, c0), (s1, r1, d1, k1, c1) = res["mix"], res["learned"]
    assert d0 == d1 and np.array_equal(k0, k1) and np.array_equal(c0, c1)
    assert s1["maxmean_bytes"] < 0.97 * s0["maxmean_bytes"], (s0, s1)
    assert r1 < r0, (r0, r1, s0, s1)
