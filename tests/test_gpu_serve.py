"""The request server (ipfc_server_*): continuous batching against a
device-memory budget.

Each request's result must be the same alone (its per-image call) and in
the mix (many requests in flight on several streams, batchable ones merged
into persistent launches): bit-identical, since the same kernels run either
way.  Admission must respect the slot limit, the budget and the arrival
times.
"""
import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
from imageprocessingflex_b200 import mix
from imageprocessingflex_b200 import serve as S

pytestmark = pytest.mark.gpu


def _pinned(shape, dtype, seed=None):
    import torch

    t = torch.empty(shape, dtype=dtype).pin_memory()
    if seed is not None:
        g = torch.Generator()
        g.manual_seed(seed)
        t.copy_(torch.randint(0, 256, shape, dtype=torch.int32, generator=g).to(dtype))
    return t


def _requests(n, seed, hi=320):
    rng = np.random.default_rng(seed)
    taps = mix.filter2d_taps()
    out = []
    for i in range(n):
        w, h = (int(v) for v in rng.integers(1, hi, size=2))
        c = int(rng.choice([1, 3]))
        op = ["gaussian", "sobel", "median", "filter2d", "erode", "dilate", "box", "gaussian"][i % 8]
        p = {}
        if op == "gaussian":
            p = {"sigma_x": float(rng.uniform(0.5, 4.0))}
        elif op == "sobel":
            dx = int(rng.random() < 0.5)
            p = {"dx": dx, "dy": 1 - dx, "ksize": 3}
        elif op == "median":
            p = {"ksize": 5}
        elif op == "filter2d":
            p = {"kernel": taps}
        elif op in ("erode", "dilate"):
            p = {"ksize": 3}
        else:
            p = {"ksize": 5}
        out.append((op, w, h, c, p))
    return out


def _alone(op, x, p):
    if op == "gaussian":
        return ipf.gaussianBlur(x, p["sigma_x"])
    if op == "sobel":
        return ipf.sobel(x, p["dx"], p["dy"], 3)
    if op == "median":
        return ipf.medianBlur(x, p["ksize"])
    if op == "filter2d":
        return ipf.filter2D(x, p["kernel"])
    if op == "box":
        return ipf.blur(x, p["ksize"])
    se = np.ones((p["ksize"], p["ksize"]), np.uint8)
    return ipf.erode(x, se) if op == "erode" else ipf.dilate(x, se)


def _serve(server, reqs, seed):
    import torch

    jobs = []
    for i, (op, w, h, c, p) in enumerate(reqs):
        shape = (h, w, c) if c > 1 else (h, w)
        src = _pinned(shape, torch.uint8, seed + i)
        dst = _pinned(shape, torch.float32 if op == "sobel" else torch.uint8)
        server.submit(op, src, dst, **p)
        jobs.append((op, src, dst, p))
    server.drain(120000)
    comps = server.poll(100000)
    assert len(comps) == len(reqs) and all(cp.status == 0 for cp in comps)
    return jobs, comps


@pytest.mark.parametrize("cfg", [{}, {"max_inflight": 5, "streams": 3}, {"max_inflight": 1, "streams": 1, "batch": False}],
                         ids=["continuous", "few-slots", "plain"])
def test_results_same_alone_and_in_the_mix(gpu, cfg):
    reqs = _requests(80, seed=3)
    with S.Server(**cfg) as server:
        jobs, comps = _serve(server, reqs, 1000)
        st = server.stats()
    for op, src, dst, p in jobs:
        want = _alone(op, src.numpy(), p)
        np.testing.assert_array_equal(dst.numpy(), want, err_msg=op)
    assert st["max_inflight"] <= cfg.get("max_inflight", 64)
    if cfg.get("batch", True) and cfg.get("max_inflight", 64) > 1:
        assert st["batched"] > 0 and st["batch_launches"] > 0


def test_device_images_and_arrival_times(gpu):
    import torch

    with S.Server() as server:
        x = torch.randint(0, 256, (97, 131, 3), dtype=torch.uint8, device="cuda")
        y = torch.empty_like(x)
        t0 = server.now()
        server.submit("gaussian", x, y, t0 + 0.2, sigma_x=2.0)
        server.drain(60000)
        (c,) = server.poll()
        assert c.status == 0 and c.admitted >= c.arrival - 1e-6 and c.done >= c.arrival
        assert c.arrival == pytest.approx(t0 + 0.2)
        assert torch.equal(y, ipf.gaussianBlur(x, 2.0))


def test_budget_admission(gpu):
    import torch

    # 1 MiB budget: small requests pass, one that can never fit fails
    with S.Server(budget_bytes=1 << 20, max_inflight=8, streams=2) as server:
        small = [(_pinned((64, 64), torch.uint8, i), _pinned((64, 64), torch.uint8)) for i in range(20)]
        for s_, d_ in small:
            server.submit("median", s_, d_, ksize=3)
        big_s, big_d = _pinned((1024, 1024), torch.uint8, 7), _pinned((1024, 1024), torch.uint8)
        tb = server.submit("gaussian", big_s, big_d, sigma_x=1.0)
        server.drain(60000)
        comps = {c.ticket: c for c in server.poll(100)}
        st = server.stats()
    assert comps[tb].status == 2  # IPFC_ERR_NOMEM
    assert sum(1 for c in comps.values() if c.status == 0) == 20
    assert st["max_bytes"] <= 1 << 20
    for s_, d_ in small:
        np.testing.assert_array_equal(d_.numpy(), ipf.medianBlur(s_.numpy(), 3))
