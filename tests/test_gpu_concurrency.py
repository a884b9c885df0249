"""One shared plan used from many host threads and several streams at once.

The reference's plans are Arc-shared and Send + Sync: apollo-stft runs Rayon
over one FftPlan1D (crates/apollo-stft/src/application/execution/plan/stft/
dimension_1d.rs:225-239), and the plan cache hands the same plan to every
caller (crates/apollo-fft/src/application/orchestration/cache/plans.rs).  Here
every result computed concurrently must equal, bit for bit, the result of the
same input computed alone (the kernels use no atomics, so a transform is
deterministic).
"""
import threading

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# a single-CTA length, a Bluestein prime, the four-step split (plan workspace)
# and a 3D shape whose middle pass runs on the lanes kernels
CASES = [([1000], 3), ([4099], 2), ([1 << 16], 2), ([24, 30, 40], 1)]


def _inputs(dims, batch, count, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims)) * batch
    return [(rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex128) for _ in range(count)]


@pytest.mark.parametrize("dims,batch", CASES)
def test_host_calls_from_eight_threads(afc, cuda, dims, batch):
    plan = afc.CudaPlan(dims, precision="f64", batch=batch)  # the cached plan every caller shares
    xs = _inputs(dims, batch, 8, seed=len(dims) * 1000 + dims[0])
    alone = [(plan.execute_host(x), plan.execute_host(x, inverse=True)) for x in xs]
    results = [None] * len(xs)
    errors = []
    start = threading.Barrier(len(xs))

    def worker(i):
        try:
            other = afc.CudaPlan(dims, precision="f64", batch=batch)  # same cached plan object
            start.wait()
            out = []
            for _ in range(3):
                out.append((other.execute_host(xs[i]), other.execute_host(xs[i], inverse=True)))
            results[i] = out
        except Exception as exc:  # pragma: no cover - reported below
            errors.append(repr(exc))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(xs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for i, runs in enumerate(results):
        assert runs is not None
        for fwd, inv in runs:
            assert np.array_equal(fwd, alone[i][0]), (dims, i)
            assert np.array_equal(inv, alone[i][1]), (dims, i)


def test_device_calls_on_two_streams(afc, cuda):
    dims, batch = [1 << 16], 4
    plan = afc.CudaPlan(dims, precision="f64", batch=batch)
    assert plan.workspace_size() > 0  # the four-step intermediate lives in a plan workspace
    g = torch.Generator(device="cuda").manual_seed(21)
    xs = [torch.randn(batch * dims[0], dtype=torch.complex128, device=cuda, generator=g) for _ in range(2)]
    alone = [plan.execute(x).reshape(-1).clone() for x in xs]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [[torch.empty_like(xs[0]) for _ in range(6)] for _ in range(2)]
    for s in streams:
        s.wait_stream(torch.cuda.current_stream())
    # interleave enqueues on the two streams: each stream's calls would overwrite
    # the other's intermediate if they shared one workspace without ordering
    for k in range(6):
        for j, s in enumerate(streams):
            with torch.cuda.stream(s):
                plan.execute(xs[j], out=outs[j][k], stream=s.cuda_stream)
    torch.cuda.synchronize()
    for j in range(2):
        for o in outs[j]:
            assert torch.equal(o, alone[j])


def test_batch_plan_on_two_streams(afc, cuda):
    lens = np.array([256, 4096, 97, 1031, 65536, 12000], dtype=np.int64)
    bp = afc.BatchPlan(lens, precision="f32")
    g = torch.Generator(device="cuda").manual_seed(22)
    xs = [torch.randn(int(lens.sum()), dtype=torch.complex64, device=cuda, generator=g) for _ in range(2)]
    alone = [bp.execute(x, mode=1).clone() for x in xs]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [[torch.empty_like(xs[0]) for _ in range(4)] for _ in range(2)]
    for s in streams:
        s.wait_stream(torch.cuda.current_stream())
    for k in range(4):
        for j, s in enumerate(streams):
            with torch.cuda.stream(s):
                bp.execute(xs[j], out=outs[j][k], mode=1 if k % 2 else 2, stream=s.cuda_stream)
    torch.cuda.synchronize()
    for j in range(2):
        for o in outs[j]:
            assert torch.equal(o, alone[j]) or (torch.linalg.vector_norm(o - alone[j]) /
                                                 torch.linalg.vector_norm(alone[j])).item() < 1e-6
