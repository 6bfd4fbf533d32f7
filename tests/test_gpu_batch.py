"""Batched uneven images: the persistent launch captured in a CUDA graph
(BatchPlan) against direct launches and the oracle; autotuning; per-CTA
busy times for load imbalance."""

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core
from idi_b200.simulation.batch import BatchPlan
from tests.helpers import K64, atoms, rng, sphere

pytestmark = pytest.mark.gpu


def _batch(seed, counts):
    g0 = rng(seed)
    imgs = [atoms(sphere(g0, int(c), g0.uniform(0.005, 0.025)), g0.uniform(0, 2 * np.pi, int(c))) for c in counts]
    amp = g0.uniform(0.5, 1.5, int(sum(counts))).astype(np.float32)
    return imgs, amp


def test_batchplan_graph_replay_matches_direct_and_oracle():
    counts = [1000, 37, 0, 4000, 1500, 2, 800]
    geom = _core.make_geom([48, 40], 75.0, 1e5, K64, flags=nat.NF)
    og = oracle.geometry([48, 40], 75.0, 1e5, K64)
    plan = BatchPlan(counts, geom, nat.SPLIT, nat.OUT_C128, amplitudes="float32")
    for seed in (1, 2):  # two different batches through the same captured graph
        imgs, amp = _batch(seed, counts)
        at = torch.from_numpy(np.concatenate(imgs)).cuda()
        E = plan.run(at, torch.from_numpy(amp).cuda()).clone()
        off = np.concatenate([[0], np.cumsum(counts)])
        direct = _core.forward(at, off, geom, nat.SPLIT, nat.OUT_C128, amplitudes=torch.from_numpy(amp).cuda())
        torch.cuda.synchronize()
        plan.check()
        assert torch.equal(E, direct)
        E = E.cpu().numpy()
        for b, a in enumerate(imgs):
            if len(a) == 0:
                assert np.all(E[b] == 0)
                continue
            ref = oracle.wavefield(og, oracle.NF, a, amp[off[b]:off[b + 1]].astype(np.float64))
            assert np.abs(E[b] - ref).max() <= 2e-5 * np.sqrt(np.mean(np.abs(ref) ** 2))
    assert plan.config["threads"] in (64, 128, 256)
    busy = plan.cta_times()
    assert busy.size > 0 and np.all(busy > 0)
    plan.close()


def test_more_images_than_one_launch():
    """Batches above 512 images are split over launches by the library."""
    counts = [3] * 600
    imgs, _ = _batch(3, counts)
    at = np.concatenate(imgs)
    geom = _core.make_geom([4, 4], 75.0, 1e5, K64, flags=nat.NF)
    off = np.concatenate([[0], np.cumsum(counts)])
    E = _core.forward(torch.from_numpy(at).cuda(), off, geom, nat.DOUBLE, nat.OUT_C128).cpu().numpy()
    og = oracle.geometry([4, 4], 75.0, 1e5, K64)
    for b in (0, 511, 512, 599):
        assert np.abs(E[b] - oracle.wavefield(og, oracle.NF, imgs[b])).max() < 1e-12
