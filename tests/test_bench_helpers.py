"""Host-side helpers of the bench: the count of the count walk's candidate tests (the compute side
of its roofline line: every query against every point of the 3^3 stencil of its cell on the
reference's grid, checked against a brute-force count over point pairs on a small cloud), and the
NUMA placement of its pinned host buffers."""
import os
import sys

import numpy as np
import torch

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _brute(pos, h):
    ext = 2.0
    n = int(ext / h)
    if ext / h - n > 0:
        n -= 1
    n = max(n, 1)
    hc = ext / n
    if np.ceil(ext / hc) > ext / hc:
        hc *= 1 + 1e-4
    cnt = int(np.ceil(ext / hc))
    c = np.clip(np.floor((pos + np.float32(1.0)) / np.float32(hc)).astype(np.int64), 0, cnt - 1)  # float32, as the bench
    d = np.abs(c[:, None, :] - c[None, :, :]).max(-1)
    return int((d <= 1).sum())


def test_candidate_tests_match_brute_force():
    sys.path.insert(0, REPO)
    import bench
    g = torch.Generator().manual_seed(3)
    for n, h in ((700, 0.31), (1500, 0.2), (400, 0.9)):
        pos = torch.rand(n, 3, generator=g) * 2 - 1
        sup = torch.full((n,), h) * (0.9 + 0.2 * torch.rand(n, generator=g))
        want = _brute(pos.numpy(), float(sup.max()))
        assert bench.candidate_tests(pos, sup) == want


def test_near_gpu_restores_affinity(monkeypatch):
    """The bench's NUMA placement of pinned buffers runs the block on the GPU's local CPUs and
    puts the process's affinity back afterwards (here with a fake NVML answer)."""
    sys.path.insert(0, REPO)
    import bench
    before = os.sched_getaffinity(0)
    local = {min(before)}
    monkeypatch.setattr(bench, "gpu_local_cpus", lambda index: local)
    with bench.near_gpu(0) as near:
        assert near.cpus == local
        assert os.sched_getaffinity(0) == local
    assert os.sched_getaffinity(0) == before
    monkeypatch.setattr(bench, "gpu_local_cpus", lambda index: None)
    with bench.near_gpu(0):
        assert os.sched_getaffinity(0) == before
