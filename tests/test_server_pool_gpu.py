"""The multi-device server pool (fmd_server_pool_*), on one GPU listed twice.

Two servers, each with its own host thread and batch, share the device; a
request goes to the server with the least outstanding work.  Every request
must finish with the same final thermo row and Rg as the same request run
alone (a replica's trajectory does not depend on where it ran or what ran
beside it), requests must land on both servers, and the pool-wide ids must
cover exactly the submitted requests."""
import numpy as np
import pytest

import fastmd_b200 as fm
from tests.util import run_conf

pytestmark = pytest.mark.gpu


def test_pool_spreads_requests_and_results_equal_alone():
    reqs = []
    for k, (nc, cl, steps) in enumerate([(10, 20, 300), (8, 50, 500), (20, 30, 200), (5, 100, 400), (12, 40, 350),
                                         (6, 50, 250)]):
        T = 0.8 + 0.05 * k
        conf = run_conf(ensemble=f"nvt_langevin {T} {T} 1.0 {k + 1}", nsteps=steps)
        gen = dict(nchains=nc, chain_length=cl, density=0.85, seed=200 + k, pushoff_steps=300)
        reqs.append((conf, gen))
    pool = fm.ServerPool(devices=[0, 0], max_replicas=3, hbm_budget_gb=8.0, steps_per_round=50)
    ids, where = [], []
    for conf, gen in reqs:
        rid, srv = pool.submit(conf, gen)
        ids.append(rid)
        where.append(srv)
    assert sorted(set(where)) == [0, 1]
    assert ids == list(range(1, len(reqs) + 1))
    pool.drain(600.0)
    got = {r.request_id: r for r in pool.poll(64)}
    st = pool.stats()
    pool.close()
    assert sorted(got) == ids and st["finished"] == len(reqs)
    for rid, (conf, gen) in zip(ids, reqs):
        r = got[rid]
        assert r.status == 0
        alone = fm.Batch(max_replicas=1, max_atoms=1 << 14)
        s = alone.add(conf, gen=gen)
        alone.run(10_000)
        assert alone.info(s).step == r.steps
        assert np.array_equal(alone.thermo(s).as_array(), np.asarray(r.thermo.as_array()))
        assert alone.rg(s) == r.rg
        alone.close()
