"""Micro-benchmark of the surrogate network's tensor-core kernels: prediction throughput
over `rows` inputs and the time of one training step (a replay of the captured step).

    python u-cuda_b200/ucb/mlp_bench.py [rows] [train_steps]
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import torch  # noqa: E402  (device memory only)

import ucb  # noqa: E402


def main(rows: int = 1 << 20, steps: int = 200) -> None:
    eng = ucb.Engine(0)
    net = ucb.Mlp(eng, fourier=64, hidden=256, layers=4, batch=8192, train_steps=steps)
    u = torch.rand(rows, 2, device="cuda")
    mean = torch.empty(rows, device="cuda")
    sd = torch.empty(rows, device="cuda")
    for _ in range(3):
        torch.cuda.synchronize()
        t = time.perf_counter()
        net.predict(u.data_ptr(), rows, mean.data_ptr(), sd.data_ptr())
        torch.cuda.synchronize()
        print(f"predict rows {rows} ms {(time.perf_counter() - t) * 1e3:.3f}", flush=True)
    y = torch.sin(5 * u[:, 0])
    for _ in range(2):
        torch.cuda.synchronize()
        t = time.perf_counter()
        loss = net.fit(u.data_ptr(), y.data_ptr(), rows)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t) * 1e3
        print(f"fit steps {steps} ms {ms:.1f} per step {ms / max(steps, 1):.4f} loss {loss:.5f}", flush=True)
    net.close()
    eng.close()


if __name__ == "__main__":
    main(*(int(a) for a in sys.argv[1:3]))
