"""The request server: continuous batching of mixed requests.  Each result must be the
same alone and in the mix (within the tolerance of its payload), admission must refuse
what can never fit, and a small budget must serialise without losing requests."""
import threading
import time

import numpy as np
import pytest

import imagestack_b200 as ib
from imagestack_b200 import synth

RTOL_FP32 = 1e-5


def rel_err(a, b, floor_frac=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-30)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


def mixed_requests(count, seed):
    """Bilateral RGB (d=5), joint bilateral on a grey guide (d=3) and Gauss transforms."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        kind = i % 3
        w, h = int(rng.integers(48, 300)), int(rng.integers(48, 300))
        ss, sr = float(rng.uniform(4, 24)), float(rng.uniform(0.05, 0.3))
        img = synth.image(w, h, 3 if kind == 0 else 1, rects=4, seed=seed * 1000 + i)
        if kind == 0:
            reqs.append(dict(kind=ib.REQ_BILATERAL, image=img, ss=ss, sr=sr))
        elif kind == 1:
            ref = synth.luminance(synth.image(w, h, 3, rects=4, seed=seed * 2000 + i))
            reqs.append(dict(kind=ib.REQ_JOINT_BILATERAL, image=img, ref=ref, ss=ss, sr=sr))
        else:
            pos = np.concatenate([img, np.broadcast_to(np.arange(w, dtype=np.float32), (1, h, w)),
                                  np.broadcast_to(np.arange(h, dtype=np.float32)[:, None], (1, h, w))])
            vals = np.concatenate([img, np.ones((1, h, w), np.float32)])
            reqs.append(dict(kind=ib.REQ_GAUSS_TRANSFORM, image=np.ascontiguousarray(vals),
                             ref=np.ascontiguousarray(pos), sigmas=[sr, ss, ss]))
    return reqs


def direct(gpu, q, payload):
    """The same request through the single-call entry points."""
    if q["kind"] == ib.REQ_BILATERAL:
        out = q["image"].copy()
        gpu.Bilateral.apply(out, q["ss"], q["ss"], 0.0, q["sr"], payload=payload)
        return out
    if q["kind"] == ib.REQ_JOINT_BILATERAL:
        out = q["image"].copy()
        gpu.JointBilateral.apply(out, q["ref"], q["ss"], q["ss"], 0.0, q["sr"], payload=payload)
        return out
    return gpu.GaussTransform.apply(None, q["ref"], q["image"], q["sigmas"], payload=payload)


def submit(srv, q):
    out = np.full_like(q["image"], np.nan)
    t = srv.submit(q["kind"], q["image"], out, ref=q.get("ref"),
                   filter_width=q.get("ss", 0.0), color_sigma=q.get("sr", 0.0),
                   sigmas=q.get("sigmas"))
    return t, out


@pytest.mark.skipif(ib.device_count() > 0, reason="checks the no-GPU behaviour")
def test_server_needs_a_gpu():
    with pytest.raises(ib.PgpuError) as e:
        ib.Server(workers=2)
    assert e.value.code == ib.ERR_NO_DEVICE


@pytest.mark.gpu
@pytest.mark.parametrize("payload,tol", [("fp32", RTOL_FP32), ("fp16", 1e-3)])
def test_each_result_is_the_same_alone_and_in_the_mix(gpu, payload, tol):
    reqs = mixed_requests(30, seed=7)
    with gpu.Server(workers=4, max_batch=16, payload=payload) as srv:
        alone = []
        for q in reqs:                      # one at a time: every batch holds one request
            t, out = submit(srv, q)
            srv.wait(t)
            alone.append(out)
        srv.reset_stats()
        # the mix: everything at once from two client threads, plus a late wave that
        # arrives while the first batches run
        tickets = [None] * len(reqs)

        def client(idx):
            for i in idx:
                tickets[i] = submit(srv, reqs[i])
        th = [threading.Thread(target=client, args=(range(k, 20, 2),)) for k in (0, 1)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        time.sleep(0.002)
        for i in range(20, len(reqs)):
            tickets[i] = submit(srv, reqs[i])
        for t, _ in tickets:
            srv.wait(t)
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] < len(reqs)        # requests shared batches
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
    for q, a, (_, mixed) in zip(reqs, alone, tickets):
        assert np.isfinite(mixed).all()
        assert rel_err(mixed, a, floor_frac=1e-2 if payload != "fp32" else 1e-6) <= tol
        if payload == "fp32":
            assert rel_err(mixed, direct(gpu, q, payload)) <= RTOL_FP32


@pytest.mark.gpu
def test_admission_refuses_what_cannot_fit_and_serialises_under_a_small_budget(gpu):
    reqs = mixed_requests(9, seed=8)
    with gpu.Server(workers=3, payload="fp32", memory_budget=200 << 20) as srv:
        big = np.zeros((3, 2048, 2048), np.float32)
        with pytest.raises(gpu.PgpuError) as e:
            srv.submit(gpu.REQ_BILATERAL, big, big, filter_width=8.0, color_sigma=0.1)
        assert e.value.code == gpu.ERR_ADMISSION
        tickets = [submit(srv, q) for q in reqs]
        for t, _ in tickets:
            srv.wait(t)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["rejected"] == 1
        assert st["peak_bytes"] <= 200 << 20
    for q, (_, out) in zip(reqs, tickets):
        assert rel_err(out, direct(gpu, q, "fp32")) <= RTOL_FP32


@pytest.mark.gpu
def test_a_failing_request_is_reported_and_the_server_keeps_serving(gpu):
    """A Gauss transform whose positions leave the lattice's int16 key range fails inside
    the batch; wait() returns its error only after the worker's stream is idle (its output
    stays unwritten), and later requests are served normally."""
    import torch
    reqs = mixed_requests(3, seed=9)
    with gpu.Server(workers=2, payload="fp32") as srv:
        w, h = 64, 48
        pos = torch.full((3, h, w), 1e6, dtype=torch.float32).pin_memory().numpy()
        vals = torch.ones((2, h, w), dtype=torch.float32).pin_memory().numpy()
        out = torch.full((2, h, w), float("nan")).pin_memory().numpy()
        t = srv.submit(gpu.REQ_GAUSS_TRANSFORM, vals, out, ref=pos, sigmas=[1.0, 1.0, 1.0])
        with pytest.raises(gpu.PgpuError) as e:
            srv.wait(t)
        assert e.value.code == gpu.ERR_ARGUMENT
        assert np.isnan(out).all()
        tickets = [submit(srv, q) for q in reqs]
        for tk, _ in tickets:
            srv.wait(tk)
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == len(reqs)
    for q, (_, o) in zip(reqs, tickets):
        assert rel_err(o, direct(gpu, q, "fp32")) <= RTOL_FP32


@pytest.mark.gpu
def test_one_waiter_per_ticket(gpu):
    """Two threads waiting on one ticket: one gets the result, the other is refused with
    ERR_ARGUMENT (already being waited for, or already collected), never a crash."""
    q = mixed_requests(1, seed=10)[0]
    with gpu.Server(workers=1, payload="fp32") as srv:
        t, _ = submit(srv, q)
        codes = []

        def waiter():
            try:
                srv.wait(t)
                codes.append(0)
            except gpu.PgpuError as e:
                codes.append(e.code)
        th = [threading.Thread(target=waiter) for _ in range(2)]
        for x in th:
            x.start()
        for x in th:
            x.join()
    assert sorted(codes) == [0, gpu.ERR_ARGUMENT]
