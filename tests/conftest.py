"""Shared test setup: the ``gpu`` marker, import paths and fixture loaders.

``-m "not gpu"`` runs on a CPU-only machine (oracle vs golden fixtures, plan
compiler vs oracle, library symbol checks); ``-m gpu`` runs the parity tests
of the CUDA paths against the oracle on a B200.
"""
import functools
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ('', 'oracle', 'tests'):
    path = os.path.join(ROOT, sub) if sub else ROOT
    if path not in sys.path:
        sys.path.insert(0, path)

GOLDEN = os.path.join(ROOT, 'tests', 'golden', 'qaoa_reference.json')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')


@functools.lru_cache(maxsize=1)
def golden():
    with open(GOLDEN) as f:
        return json.load(f)['workloads']


def golden_graph(name):
    """The workload's graph rebuilt with its generator (same node and
    adjacency order as when the fixture was made) and its fixture record."""
    import graphs
    w = golden()[name]
    G = graphs.by_name(name)
    assert [list(e) for e in G.edges()] == w['edges'], 'graph generator changed: ' + name
    return G, w


@pytest.fixture
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail('GPU test run without a CUDA device')
    return torch.device('cuda', 0)
