"""Seeded inputs of the single-call checks at the benchmark configurations, shared by the fixture script
(make_config_golden.py) and the tests: numpy's default_rng with one seed per input, so that every machine
draws the same arrays."""
import numpy as np

NSAMPLE = 8192


def config_inputs(seed, ne, nf):
    g = lambda k: np.random.default_rng([seed, k])
    return dict(E=g(1).uniform(1e-6, 1.0, ne), u=g(2).standard_normal(nf), r=g(3).standard_normal(nf),
                fsrc=(-g(4).uniform(0.0, 0.5, ne)).astype(np.float32),
                x=g(5).uniform(1e-3, 1.0, ne).astype(np.float32), ce=g(6).uniform(0.0, 2.0, ne),
                idx_f=np.sort(g(7).choice(nf, NSAMPLE, replace=False)),
                idx_e=np.sort(g(8).choice(ne, NSAMPLE, replace=False)))


def sample_indices(seed, k, n):
    return np.sort(np.random.default_rng([seed, k]).choice(n, NSAMPLE, replace=False))
