"""Channel sharding over ranks (one process per GPU), on CPU with gloo.

* the deterministic channel assignment partitions the channels and balances
  visibility counts;
* two gloo ranks each grid their own channels with the oracle and form the
  continuum residual with one all-reduce: the result equals the
  single-process sum over all channels;
* the step time reported is the maximum over ranks.

No GPU is used: the sharding and the exchange step are host logic.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import channels
import synth

WORLD = 2
NUM_CHANNELS = 5


def test_assignment_partitions_channels_and_balances_counts():
    counts = channels.flagged_counts(64, 3_916_800, seed=3)
    assert all(0.4 * 3_916_800 - 1 <= c <= 3_916_800 for c in counts)
    for world in (1, 2, 3, 4, 8):
        owned = channels.assign_channels(counts, world)
        flat = sorted(c for o in owned for c in o)
        assert flat == list(range(64))
        loads = [channels.rank_load(counts, o) for o in owned]
        # largest-first greedy: no rank exceeds the mean by more than one channel
        assert max(loads) - sum(loads) / world <= max(counts)
        assert owned == channels.assign_channels(counts, world)  # deterministic


def test_assignment_rejects_bad_input():
    with pytest.raises(ValueError):
        channels.assign_channels([1, 2], 0)
    with pytest.raises(ValueError):
        channels.assign_channels([1, -2], 2)
    assert channels.assign_channels([], 3) == [[], [], []]


def _channel_grid(ch: int):
    """Oracle std_gridding of channel ch of a small multi-channel workload."""
    import oracle as O

    o = O.Oracle("f64")
    w = synth.small_workload(seed=40 + ch, grid_size=64)
    g = o.std_gridding(w.cfg.grid_size, w.cfg.oversampling, w.gkernels, w.supports, w.uvw, w.vis,
                       w.cfg.uv_scale, w.cfg.w_scale)
    return np.asarray(g, dtype=np.float64)


def _worker(rank: int, port: int, counts, out_dir: str):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        mine = channels.assign_channels(counts, WORLD)[rank]
        acc = None
        for ch in mine:
            g = _channel_grid(ch)
            acc = g if acc is None else acc + g
        t = torch.from_numpy(acc if acc is not None else np.zeros_like(_channel_grid(0))).contiguous()
        channels.continuum_sum_(t)
        tmax = channels.max_over_ranks(1.0 + rank)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), t.numpy())
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{tmax} {' '.join(map(str, mine))}\n")
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_continuum_sum_matches_single_process(tmp_path, oracle64):
    counts = [int(synth.small_workload(seed=40 + ch, grid_size=64).num_vis) for ch in range(NUM_CHANNELS)]
    mp.start_processes(_worker, args=(_free_port(), counts, str(tmp_path)), nprocs=WORLD, join=True,
                       start_method="spawn")
    ref = sum(_channel_grid(ch) for ch in range(NUM_CHANNELS))
    owned = []
    for r in range(WORLD):
        got = np.load(tmp_path / f"rank{r}.npy")
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        tmax, *chs = (tmp_path / f"rank{r}.txt").read_text().split()
        assert float(tmax) == float(WORLD)  # max over ranks of 1 + rank
        owned += [int(c) for c in chs]
    assert sorted(owned) == list(range(NUM_CHANNELS))


CYCLES = 3


def _channel_data(ch: int):
    """Channel ch of a small multi-channel set with a seeded 0-60 % of its
    visibilities flagged (dropped), so channels differ in size."""
    w = synth.small_workload(seed=40 + ch, grid_size=64)
    keep = channels.flagged_counts(NUM_CHANNELS, w.num_vis, seed=9)[ch]
    w.uvw, w.vis = np.ascontiguousarray(w.uvw[:keep]), np.ascontiguousarray(w.vis[:keep])
    return w


def _cycle_residual(o, w, model_grid):
    """One channel's major-cycle visibility pass with the oracle: degrid the
    model grid (convolutional), subtract from the measured visibilities,
    grid the residual."""
    G, OS = w.cfg.grid_size, w.cfg.oversampling
    pred = o.std_degridding(G, OS, w.dkernels, w.supports, model_grid, w.uvw, w.cfg.uv_scale, w.cfg.w_scale,
                            nearest=False)
    delta = o.subtract_vis(w.vis, pred)
    return np.asarray(o.std_gridding(G, OS, w.gkernels, w.supports, w.uvw, delta, w.cfg.uv_scale, w.cfg.w_scale),
                      dtype=np.float64)


def _model_update(model_grid, continuum, nch):
    """The replicated step after the exchange (the same on every rank): a
    fixed-gain update of the model grid from the continuum residual."""
    return model_grid + 0.25 * continuum / nch


def _cycles_worker(rank: int, port: int, counts, out_dir: str):
    import torch
    import torch.distributed as dist
    import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        o = O.Oracle("f64")
        mine = channels.assign_channels(counts, WORLD)[rank]
        data = {ch: _channel_data(ch) for ch in mine}
        G = 64
        model = np.zeros((G * G, 2))
        for _ in range(CYCLES):
            acc = np.zeros((G * G, 2))
            for ch in mine:
                acc += _cycle_residual(o, data[ch], model)
            t = torch.from_numpy(acc).contiguous()
            channels.continuum_sum_(t)
            model = _model_update(model, t.numpy(), len(counts))
        np.save(os.path.join(out_dir, f"model{rank}.npy"), model)
        np.save(os.path.join(out_dir, f"cont{rank}.npy"), t.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_major_cycles_match_single_process(tmp_path, oracle64):
    """Channels dealt by visibility count (uneven), three major cycles of
    pass -> continuum all-reduce -> replicated model update: every rank ends
    with the single-process model and continuum residual."""
    counts = [int(_channel_data(ch).uvw.shape[0]) for ch in range(NUM_CHANNELS)]
    assert len(set(counts)) > 1
    mp.start_processes(_cycles_worker, args=(_free_port(), counts, str(tmp_path)), nprocs=WORLD, join=True,
                       start_method="spawn")
    G = 64
    model = np.zeros((G * G, 2))
    data = [_channel_data(ch) for ch in range(NUM_CHANNELS)]
    for _ in range(CYCLES):
        cont = sum(_cycle_residual(oracle64, d, model) for d in data)
        model = _model_update(model, cont, NUM_CHANNELS)
    for r in range(WORLD):
        np.testing.assert_allclose(np.load(tmp_path / f"model{r}.npy"), model, rtol=1e-12,
                                   atol=1e-12 * np.abs(model).max())
        np.testing.assert_allclose(np.load(tmp_path / f"cont{r}.npy"), cont, rtol=1e-12,
                                   atol=1e-12 * np.abs(cont).max())
