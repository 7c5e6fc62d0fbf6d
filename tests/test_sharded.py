"""One micrograph across ranks (gisspa_shard_*, sharded.py): the angle partition and the
merge of the per-pixel state on CPU ranks with the gloo backend (no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import gisspa
from sharded import ShardState, angle_ranges, merge_state


def test_angle_ranges_cover_the_sequence():
    for n in (0, 1, 7, 36, 72, 120, 72000):
        for world in (1, 2, 3, 4, 8):
            r = angle_ranges(n, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1 and sorted(sizes, reverse=True) == sizes


# Python statement of the library's peak key (include/gisspa.h, gisspa_shard_info): the
# order-preserving bits of the FP32 value above 0xFFFFFFFF - k, XOR 2^63, as int64.
def peak_key(value: np.ndarray, k: np.ndarray) -> np.ndarray:
    b = np.asarray(value, np.float32).view(np.uint32).astype(np.uint64)
    fk = np.where(b & 0x80000000, (~b) & 0xFFFFFFFF, b | 0x80000000)
    key = (fk << np.uint64(32)) | (np.uint64(0xFFFFFFFF) - np.asarray(k, np.uint64))
    key = np.where(np.asarray(k) < 0, np.uint64(0), key)
    return (key ^ np.uint64(1 << 63)).view(np.int64)


def unpack(key: np.ndarray):
    u = key.view(np.uint64) ^ np.uint64(1 << 63)
    hi = (u >> np.uint64(32)).astype(np.uint32)
    bits = np.where(hi & 0x80000000, hi & 0x7FFFFFFF, ~hi)
    k = (np.uint64(0xFFFFFFFF) - (u & np.uint64(0xFFFFFFFF))).astype(np.int64)
    return bits.astype(np.uint32).view(np.float32), np.where(u == 0, -1, k)


def test_peak_key_orders_value_then_lower_index():
    v = np.array([-3.0, -0.5, 0.0, 0.25, 0.25, 7.0], np.float32)
    k = np.array([5, 9, 3, 8, 2, 0])
    key = peak_key(v, k)
    # larger value -> larger key; equal values -> the lower index has the larger key
    assert key[0] < key[1] < key[2] < key[3] < key[4] < key[5]
    assert peak_key(np.float32([-np.inf]), np.array([-1]))[0] == np.iinfo(np.int64).min
    vv, kk = unpack(key)
    assert np.array_equal(vv, v) and np.array_equal(kk, k)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


N_PIX = 4096


def _partials(rank: int):
    rng = np.random.default_rng(100 + rank)
    s1 = rng.standard_normal(N_PIX)
    s2 = rng.random(N_PIX) * 10
    val = rng.integers(-4, 4, N_PIX).astype(np.float32) / 2  # many ties across ranks
    k = rank * 1000 + rng.integers(0, 1000, N_PIX)
    k[::97] = -1  # pixels this rank never reached
    return s1, s2, val, k


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s1, s2, val, k = _partials(rank)
    st = ShardState(torch.from_numpy(s1.copy()), torch.from_numpy(s2.copy()), torch.from_numpy(peak_key(val, k)))
    merge_state(st)
    q.put((rank, st.sum.numpy(), st.sum_sq.numpy(), st.key.numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_merge_state_two_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, a, b, c = q.get(timeout=120)
        res[r] = (a, b, c)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = [_partials(r) for r in range(world)]
    s1 = sum(p[0] for p in parts)
    s2 = sum(p[1] for p in parts)
    # single-GPU rule: the larger value wins, ties go to the lower (angle, template) index
    best_v = np.full(N_PIX, -np.inf, np.float32)
    best_k = np.full(N_PIX, -1)
    for _, _, v, k in parts:
        take = (k >= 0) & ((v > best_v) | ((v == best_v) & ((best_k < 0) | (k < best_k))))
        best_v = np.where(take, v, best_v)
        best_k = np.where(take, k, best_k)
    for r in range(world):
        a, b, c = res[r]
        assert np.allclose(a, s1, rtol=0, atol=1e-12) and np.allclose(b, s2, rtol=0, atol=1e-12)
        v, k = unpack(c)
        none = best_k < 0
        assert np.array_equal(k, best_k)
        assert np.array_equal(v[~none], best_v[~none])
