"""Small single-GPU cases of each measured workload, for profiler captures.

Each case builds its plan, runs the transform `--reps` times on seeded device
data and exits 0; wrap it in a profiler, e.g.

    python -m apollofft_b200.profile_cases c4 --rows 8192 --precision tc_fp16
    ncu --set full --clock-control none -k regex:tc_fft_kernel -c 1 \
        -o prof python -m apollofft_b200.profile_cases c4 --rows 8192 --precision tc_fp16

Cases (inputs larger than the 126 MB L2 where the workload allows):
  c1  64 x 4096 complex128 forward + inverse
  c2  3D C2C forward + inverse of --shape (default 128,256,256) at --precision f64|f32
  c3  the 4096-length uneven complex64 batch, --mode 0 (graph) | 1 (per length) | 2 (persistent)
  c4  --rows x 4096 complex64 forward at --precision f32 | tc_bf16 | tc_fp16
  c5  --batch x 2048 x 2048 real f32 R2C (full spectrum) forward + adjoint
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--shape", default="128,256,256")
    ap.add_argument("--precision", default=None)
    ap.add_argument("--rows", type=int, default=8192)
    ap.add_argument("--mode", type=int, default=2)
    ap.add_argument("--batch", type=int, default=2)
    a = ap.parse_args(argv)

    import torch
    import apollofft_b200 as afc
    from apollofft_b200 import workloads as W

    g = torch.Generator(device="cuda").manual_seed(7)
    if a.case == "c1":
        x = torch.from_numpy(W.c1_input()).cuda()
        p = afc.CudaPlan([4096], precision="f64", batch=64)
        y = torch.empty_like(x)
        for _ in range(a.reps):
            p.execute(x, out=y)
            p.execute(y, out=x, inverse=True)
    elif a.case == "c2":
        prec = a.precision or "f64"
        shape = [int(v) for v in a.shape.split(",")]
        dt = torch.complex128 if prec == "f64" else torch.complex64
        x = torch.randn(shape, dtype=dt, device="cuda", generator=g)
        p = afc.CudaPlan(shape, precision=prec)
        y = torch.empty_like(x)
        for _ in range(a.reps):
            p.execute(x, out=y)
            p.execute(y, out=x, inverse=True)
    elif a.case == "c3":
        lens = W.c3_lengths()
        x = torch.from_numpy(W.c3_values(lens)).cuda()
        bp = afc.BatchPlan(lens, precision="f32")
        y = torch.empty_like(x)
        for _ in range(a.reps):
            bp.execute(x, out=y, mode=a.mode)
    elif a.case == "c4":
        prec = a.precision or "f32"
        x = torch.randn(a.rows, 4096, dtype=torch.complex64, device="cuda", generator=g)
        p = afc.CudaPlan([4096], precision=prec, batch=a.rows)
        y = torch.empty_like(x)
        for _ in range(a.reps):
            p.execute(x, out=y)
    else:
        from apollofft_b200 import autograd as AG
        img = torch.randn(a.batch, 2048, 2048, dtype=torch.float32, device="cuda", generator=g, requires_grad=True)
        for _ in range(a.reps):
            X = AG.rfft2(img, half=False)
            (X.abs() ** 2).sum().backward()
    torch.cuda.synchronize()
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
