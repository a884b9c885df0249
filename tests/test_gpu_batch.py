"""Uneven batches (many lengths in one call) against the f64 oracle.

The persistent kernel (mode 0 in a CUDA graph, mode 2 without) and the
per-length plain launches (mode 1) must agree with the oracle per lane:
f32 relative L2 <= 1e-5, f64 <= 1e-12."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


def lanes_of(packed, lengths):
    offs = np.concatenate([[0], np.cumsum(lengths)[:-1]])
    return [packed[o:o + n] for o, n in zip(offs, lengths)]


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_golden_uneven_batch(afc, cuda, mode):
    lens = GOLD["c3_lengths"]
    x = torch.from_numpy(GOLD["c3_x"]).cuda()
    bp = afc.BatchPlan(lens, precision="f32")
    y = bp.execute(x, mode=mode).cpu().numpy()
    for got, ref, n in zip(lanes_of(y, lens), lanes_of(GOLD["c3_fwd64"], lens), lens):
        assert rel_l2(got, ref) < 1e-5, n


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_workload_lengths_vs_numpy(afc, cuda, prec):
    from apollofft_b200 import workloads as W
    lens = W.c3_lengths(count=300, seed=33)
    x = W.c3_values(lens, seed=33).astype(np.complex64 if prec == "f32" else np.complex128)
    bp = afc.BatchPlan(lens, precision=prec)
    xt = torch.from_numpy(x).cuda()
    y = bp.execute(xt, mode=0).cpu().numpy()
    yi = bp.execute(torch.from_numpy(y).cuda(), mode=0, inverse=True).cpu().numpy()
    tol = 1e-5 if prec == "f32" else 1e-12
    for got, back, src, n in zip(lanes_of(y, lens), lanes_of(yi, lens), lanes_of(x, lens), lens):
        ref = np.fft.fft(src.astype(np.complex128))
        assert rel_l2(got, ref) < tol, n
        assert rel_l2(back, src) < tol, n
    # graph replay with the same buffers gives the same result
    y2 = bp.execute(xt, mode=0).cpu().numpy()
    assert np.array_equal(y, y2)


def test_batch_modes_agree_on_repeats(afc, cuda):
    lens = np.array([256, 256, 4096, 97, 97, 97, 1031, 65536, 12000, 7, 1], dtype=np.int64)
    rng = np.random.default_rng(9)
    x = (rng.standard_normal(lens.sum()) + 1j * rng.standard_normal(lens.sum())).astype(np.complex64)
    bp = afc.BatchPlan(lens, precision="f32")
    xt = torch.from_numpy(x).cuda()
    outs = [bp.execute(xt, mode=m).cpu().numpy() for m in (0, 1, 2)]
    for o in outs[1:]:
        assert rel_l2(o, outs[0]) < 1e-6
    for got, src in zip(lanes_of(outs[0], lens), lanes_of(x, lens)):
        assert rel_l2(got, np.fft.fft(src.astype(np.complex128))) < 1e-5


def test_plan_creation_leaves_no_stale_error(afc, cuda):
    """A batch plan whose shared-memory group is large (here 8 lanes of 16384
    points) is tuned on a scratch buffer sized from that group; the plan's
    first launch, straight after creation, must succeed (a failed optional
    allocation during creation once surfaced as an out-of-memory error of the
    next launch)."""
    lens = np.array([16384] * 8 + [4096, 97, 1031], dtype=np.int64)
    rng = np.random.default_rng(21)
    x = (rng.standard_normal(lens.sum()) + 1j * rng.standard_normal(lens.sum())).astype(np.complex64)
    xt = torch.from_numpy(x).cuda()
    bp = afc.BatchPlan(lens, precision="f32")
    for mode in (2, 0, 0):
        y = bp.execute(xt, mode=mode).cpu().numpy()
        for got, src in zip(lanes_of(y, lens), lanes_of(x, lens)):
            assert rel_l2(got, np.fft.fft(src.astype(np.complex128))) < 1e-5
