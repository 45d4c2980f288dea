"""Admission rule of the job server (sched.hpp), on the CPU: arrival order,
memory budget, and backfilling that never delays the head of the queue."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import HOSTMODEL_DIR, ROOT

SRC = os.path.join(HOSTMODEL_DIR, "sched_shim.cpp")
SO = os.path.join(HOSTMODEL_DIR, "_build", "libsched_shim.so")


@pytest.fixture(scope="module")
def sq():
    hdr = os.path.join(ROOT, "bt-am_b200", "csrc", "sched.hpp")
    if (not os.path.exists(SO) or os.path.getmtime(SO) < max(os.path.getmtime(SRC),
                                                             os.path.getmtime(hdr))):
        os.makedirs(os.path.dirname(SO), exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", SO, SRC],
                       check=True)
    L = ctypes.CDLL(SO)
    L.sq_create.restype = ctypes.c_void_p
    L.sq_create.argtypes = [ctypes.c_ulonglong]
    L.sq_destroy.argtypes = [ctypes.c_void_p]
    L.sq_push.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_ulonglong]
    L.sq_admit.restype = ctypes.c_longlong
    L.sq_admit.argtypes = [ctypes.c_void_p]
    L.sq_release.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong]
    L.sq_in_use.restype = ctypes.c_ulonglong
    L.sq_in_use.argtypes = [ctypes.c_void_p]
    L.sq_fits_ever.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong]
    return L


def test_fifo_within_budget(sq):
    q = sq.sq_create(100)
    for i, b in enumerate([30, 30, 30, 30]):
        sq.sq_push(q, i, b)
    assert [sq.sq_admit(q) for _ in range(4)] == [0, 1, 2, -1]
    assert sq.sq_in_use(q) == 90
    sq.sq_release(q, 30)
    assert sq.sq_admit(q) == 3
    sq.sq_destroy(q)


def test_backfill_leaves_room_for_head(sq):
    q = sq.sq_create(100)
    sq.sq_push(q, 0, 60)
    assert sq.sq_admit(q) == 0          # running: 60
    sq.sq_push(q, 1, 70)                # head, blocked (60 + 70 > 100)
    sq.sq_push(q, 2, 20)                # 60 + 70 + 20 > 100: may not overtake
    sq.sq_push(q, 3, 10)
    assert sq.sq_admit(q) == -1
    sq.sq_release(q, 60)                # running: 0
    assert sq.sq_admit(q) == 1          # head first
    assert sq.sq_admit(q) == 2          # 70 + 20 fits
    assert sq.sq_admit(q) == 3          # 90 + 10 fits
    sq.sq_destroy(q)


def test_small_jobs_overtake_only_with_room(sq):
    q = sq.sq_create(100)
    sq.sq_push(q, 0, 20)
    assert sq.sq_admit(q) == 0          # running: 20
    sq.sq_push(q, 1, 50)                # head fits: 70
    sq.sq_push(q, 2, 40)
    assert sq.sq_admit(q) == 1
    assert sq.sq_admit(q) == -1         # 70 + 40 > 100
    sq.sq_push(q, 3, 5)                 # behind a blocked head: 70 + 40 + 5 > 100
    assert sq.sq_admit(q) == -1
    sq.sq_release(q, 20)                # running: 50
    assert sq.sq_admit(q) == 2          # head 40 fits: 90
    assert sq.sq_admit(q) == 3          # 95
    assert sq.sq_in_use(q) == 95
    assert not sq.sq_fits_ever(q, 101) and sq.sq_fits_ever(q, 100)
    sq.sq_destroy(q)


def test_random_stream_never_overcommits_and_head_waits_boundedly(sq):
    """Seeded random arrivals and completions: memory in use never exceeds
    the budget, every job is admitted, and once a job is at the head no job
    admitted later than its arrival at the head is admitted unless the head
    still fits next to it."""
    rng = np.random.default_rng(3)
    budget = 1000
    q = sq.sq_create(budget)
    running = {}
    queue = []
    nxt = 0
    admitted = []
    for step in range(4000):
        if nxt < 600 and rng.random() < 0.6:
            b = int(rng.integers(1, 400))
            sq.sq_push(q, nxt, b)
            queue.append((nxt, b))
            nxt += 1
        if running and rng.random() < 0.5:
            k = list(running)[int(rng.integers(len(running)))]
            sq.sq_release(q, running.pop(k))
        while True:
            head = queue[0] if queue else None
            j = sq.sq_admit(q)
            if j < 0:
                break
            b = dict(queue)[j]
            if head is not None and j != head[0]:
                # an overtaking job leaves room for the head
                assert sum(running.values()) + head[1] + b <= budget
            queue = [e for e in queue if e[0] != j]
            running[j] = b
            admitted.append(j)
            assert sum(running.values()) <= budget
            assert sq.sq_in_use(q) == sum(running.values())
    while running:
        sq.sq_release(q, running.pop(next(iter(running))))
        while (j := sq.sq_admit(q)) >= 0:
            b = dict(queue)[j]
            queue = [e for e in queue if e[0] != j]
            running[j] = b
            admitted.append(j)
    assert sorted(admitted) == list(range(nxt))
    sq.sq_destroy(q)
