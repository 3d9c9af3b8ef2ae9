"""A J/K build split into rank slices (qcg_set_shard): the partial J and K of the slices, summed, equal the
whole build, for 2 and 3 slices, on one GPU (each slice is what one rank of a multi-GPU build computes); the
slices are cut at equal shares of the primitive-quartet work."""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, parallel, workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_slices_sum_to_the_whole_build(world):
    mol = W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)
    sh = B.even_tempered(mol)
    eng = api.Engine(sh)
    D = W.cluster_density(eng.nbf, nocc=10)
    J, K, _ = eng.fock_jk(D)
    Js, Ks = np.zeros_like(J), np.zeros_like(K)
    for r in range(world):
        eng.set_shard(r, world)
        Jr, Kr, _ = eng.fock_jk(D)
        assert np.abs(Jr).max() > 0
        Js += Jr
        Ks += Kr
    assert np.abs(Js - J).max() <= 1e-10 and np.abs(Ks - K).max() <= 1e-10
    eng.set_shard(0, 1)
    J1, _, _ = eng.fock_jk(D)
    assert np.abs(J1 - J).max() <= 1e-10


@pytest.mark.parametrize("world", [2, 3, 8])
def test_shards_balance_primitive_quartets_on_a_contracted_basis(world):
    """The slices are cut at equal shares of each class's primitive quartets: on contracted shells (1-3
    primitives, so quartets cost 1 to 81 primitive quartets) the ranks' primitive work is equal to within
    one quartet per class at each of a share's two cuts, while their quartet counts differ; the shares cover
    the build exactly."""
    pool = W.shell_pool(48, seed=W.SEED0 + 5000)
    eng = api.Engine(pool)
    eng.schwarz(1e-10)
    whole = eng.shard_work(0, 1)
    parts = [eng.shard_work(r, world) for r in range(world)]
    assert sum(p[0] for p in parts) == whole[0] and sum(p[1] for p in parts) == whole[1]
    prims = [p[1] for p in parts]
    assert max(prims) - min(prims) <= 2 * 21 * 81, prims
    quartets = [p[0] for p in parts]
    assert max(quartets) > min(quartets)
    # and the slices still sum to the whole build
    D = W.cluster_density(eng.nbf, nocc=40)
    J, K, _ = eng.fock_jk(D)
    Js, Ks = np.zeros_like(J), np.zeros_like(K)
    for r in range(world):
        eng.set_shard(r, world)
        Jr, Kr, _ = eng.fock_jk(D)
        Js += Jr
        Ks += Kr
    eng.set_shard(0, 1)
    assert np.abs(Js - J).max() <= 1e-10 and np.abs(Ks - K).max() <= 1e-10


def test_sharded_helper_without_a_process_group():
    import torch
    sh = B.even_tempered(W.water())
    eng = api.Engine(sh)
    n = eng.nbf
    D = torch.tensor(W.cluster_density(n, nocc=5), device="cuda")
    J, K = torch.empty_like(D), torch.empty_like(D)
    parallel.sharded_fock_jk(eng, D.data_ptr(), J.data_ptr(), K.data_ptr(), J, K)
    torch.cuda.synchronize()
    Jr, Kr, _ = api.Engine(sh).fock_jk(D.cpu().numpy())
    assert np.abs(J.cpu().numpy() - Jr).max() <= 1e-10


def test_bad_shard_rejected():
    eng = api.Engine(B.even_tempered(W.water()))
    for r, w in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(api.QcgError) as e:
            eng.set_shard(r, w)
        assert e.value.code == api.QCG_ERR_ARG
