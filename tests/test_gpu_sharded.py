"""One state sharded over 2^g shards on one GPU (quantumsimevo_b200/sharded.py,
execute_shards): each shard runs its local ops through the fused engine, and
the half-shard exchanges run as device copies between the shards.  This is the
multi-rank program with the transport replaced by in-process copies (no kernel
waits on another shard).  Amplitudes against the oracle and the unsharded
engine."""
import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import sharded as S
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Circuit, Device
from test_sharded_cpu import _mixed

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def _sharded(dev, n, g, ops, params=None):
    shards = [S.DeviceShard(n - g, r, dev) for r in range(1 << g)]
    pos = S.execute_shards(ops, n, g, shards, params)
    return S.logical_order([s.download() for s in shards], n, g, pos)


@pytest.mark.parametrize("g", [1, 2])
def test_sharded_on_one_gpu_matches_oracle(dev, g):
    n = 14
    ops = _mixed(n, 731 + g)
    got = _sharded(dev, n, g, ops)
    assert np.max(np.abs(got - O.run(n, ops))) <= TOL


def test_sharded_22q_matches_unsharded_engine(dev):
    n, g = 22, 2
    ops = np.concatenate([W.hrz_qft(n, seed=5), _mixed(n, 9)[:400]])
    got = _sharded(dev, n, g, ops)
    c = Circuit(n, device=dev, seed=1)
    c.add_ops(ops)
    c.execute()
    assert np.max(np.abs(got - c.get_state_vector())) <= TOL
