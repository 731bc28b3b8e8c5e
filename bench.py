"""Benchmark of the B200 lab-fill + stencil path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workloads (synthetic inputs of the shapes named in the reference's benchmark
descriptions; FP64 unless stated):

  c1     128^3 cells = 8^3 blocks of 16^3, one scalar, lab (-1,2) + 7-point
         Laplacian + central gradient fused (one kernel per step).

A step is one pass of the path over the whole grid.  ``value`` is whole-job
Gcell-updates/s with inputs resident in HBM (kernel time from CUDA events on
the launching stream); ``e2e`` is the same metric through the C ABI with the
input uploaded from pinned host memory and the outputs read back every step.
Multi-GPU runs are independent replicas (the path does not shard across GPUs
in this build): scaling "weak", value = all ranks' cells / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return dict(hbm_gbs=float(d["hbm_gbs"]), src="measured")
    return dict(hbm_gbs=6650.0, src="fallback")


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- dist helpers
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, value: float) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- inputs
def c1_field(nb, n, block_stride, seed=1234):
    """u = sin(2 pi x) sin(2 pi y) cos(2 pi z) + U(-1e-3, 1e-3) at cell centres,
    in the grid layout (blocks x-fastest, 32-byte padded)."""
    nbk = int(np.prod(nb))
    cells = int(np.prod(n))
    h = [1.0 / (nb[d] * n[d]) for d in range(3)]
    xs = [(np.arange(nb[d] * n[d]) + 0.5) * h[d] for d in range(3)]
    sx, sy, cz = np.sin(2 * np.pi * xs[0]), np.sin(2 * np.pi * xs[1]), np.cos(2 * np.pi * xs[2])
    g = cz[:, None, None] * sy[None, :, None] * sx[None, None, :]
    g = g.reshape(nb[2], n[2], nb[1], n[1], nb[0], n[0]).transpose(0, 2, 4, 1, 3, 5)
    out = np.zeros((nbk, block_stride))
    out[:, :cells] = g.reshape(nbk, cells)
    rng = np.random.default_rng(seed)
    out[:, :cells] += rng.uniform(-1e-3, 1e-3, size=(nbk, cells))
    return out.reshape(-1)


# --------------------------------------------------------------- workloads
class C1:
    name = "c1"
    desc = "lab(-1,2)+7pt Laplacian+central gradient, 128^3 cells as 8^3 blocks of 16^3, FP64"
    nb, n = (8, 8, 8), (16, 16, 16)
    bytes_per_cell = 40  # 8 B read + 4 x 8 B written
    dtype = "f64"

    def __init__(self):
        import torch

        import cubismnova_b200 as cn
        self.cn, self.torch = cn, torch
        self.u = cn.Grid.Cartesian(self.nb, self.n)
        self.host = c1_field(self.nb, self.n, self.u.block_stride)
        self.u.upload(self.host)
        self.lap = cn.Grid.Cartesian(self.nb, self.n)
        self.grad = cn.Grid.Cartesian(self.nb, self.n, ncomp=3)
        self.cells = int(np.prod(self.nb)) * int(np.prod(self.n))
        self.flush_buf = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
        self.u.sync_bcs()
        # pinned host buffers for the end-to-end leg
        self.h_in = torch.from_numpy(self.host).pin_memory()
        self.h_out = [torch.empty(self.u.comp_stride, dtype=torch.float64).pin_memory() for _ in range(4)]

    def needs_flush(self):
        return True

    def flush(self, stream):
        with self.torch.cuda.stream(stream):
            self.flush_buf.fill_(1.0)

    def step(self, stream):
        self.cn.ops.lap_grad(self.u, self.lap, self.grad, stream=stream)

    launches_per_step = 1

    def e2e_step(self, stream):
        import ctypes as C
        lib = self.cn._lib.lib()
        sh = C.c_void_p(stream.cuda_stream)
        nbytes = self.u.comp_stride * 8
        self.cn._lib.check(lib.cn_grid_upload(self.u.handle, 0, C.c_void_p(self.h_in.data_ptr()), nbytes, sh))
        self.step(stream)
        self.cn._lib.check(lib.cn_grid_download(self.lap.handle, 0, C.c_void_p(self.h_out[0].data_ptr()),
                                                nbytes, sh))
        for d in range(3):
            self.cn._lib.check(lib.cn_grid_download(self.grad.handle, d,
                                                    C.c_void_p(self.h_out[1 + d].data_ptr()), nbytes, sh))
        return nbytes, 4 * nbytes

    def cpu_sample(self, threads, budget_s=10.0):
        """Reference FieldLab + loops (oracle/_ref) on all blocks, repeated."""
        import oracle as O
        h = 1.0 / 128
        kind = "reference" if O.ref_available() else "port"
        if kind == "reference":
            t, _, _ = O.ref_c1_sweep(self.host, self.nb, self.n, (1 / h / h,) * 3, (1 / h,) * 3,
                                     threads=threads, reps=3)
        else:
            t0 = time.perf_counter()
            O.laplacian_f64(self.host, self.nb, self.n, {}, (1 / h / h,) * 3)
            O.gradient_f64(self.host, self.nb, self.n, {}, (1 / h,) * 3)
            t = time.perf_counter() - t0
            threads = 1
        return dict(value=self.cells / t / 1e9, unit="Gcell-updates/s", cores=threads, kind=kind,
                    sample=f"full 128^3 sweep (lab+Laplacian+gradient), best of 3, {threads} threads",
                    seconds_per_sweep=t)


WORKLOADS = {"c1": C1}
DEFAULT_WORKLOAD = "c1"


# ------------------------------------------------------------------- main
def run_ours(args, world, rank, local, pg):
    import torch
    torch.cuda.set_device(local)
    W = WORKLOADS[args.workload]()
    stream = torch.cuda.Stream()
    peaks = measured_peaks()
    # warm-up
    for _ in range(args.warmup):
        if W.needs_flush():
            W.flush(stream)
        W.step(stream)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(pg)
    torch.cuda.synchronize()
    for i in range(args.steps):
        if W.needs_flush():
            W.flush(stream)
        starts[i].record(stream)
        W.step(stream)
        ends[i].record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    clocks = sampler.stop()
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms_local = float(np.sum(per))
    ms = max_over_ranks(pg, ms_local)
    ms_per_step = ms / args.steps
    value = W.cells * world * args.steps / (ms / 1e3) / 1e9
    # roofline of the dominant (here: only) kernel per launch
    launch_ms = ms_local / (args.steps * W.launches_per_step)
    cells_per_launch = W.cells / W.launches_per_step
    achieved = W.bytes_per_cell * cells_per_launch / (launch_ms / 1e3) / 1e9
    roof = dict(bound="hbm", achieved=round(achieved, 1), peak=peaks["hbm_gbs"], unit="GB/s",
                frac=round(achieved / peaks["hbm_gbs"], 4), traffic=args.traffic,
                peak_source=peaks["src"], algorithmic_bytes_per_cell=W.bytes_per_cell)
    # end to end through the C ABI with host buffers
    for _ in range(2):
        W.e2e_step(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ek = max(3, args.steps // 2)
    barrier(pg)
    e0.record(stream)
    hb = db = 0
    for _ in range(ek):
        hb, db = W.e2e_step(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(pg, e0.elapsed_time(e1)) / ek
    e2e = dict(value=round(W.cells * world / (e2e_ms / 1e3) / 1e9, 4), unit="Gcell-updates/s",
               h2d_bytes_per_step=hb, d2h_bytes_per_step=db, ms_per_step=round(e2e_ms, 4))
    out = dict(metric="Gcell-updates/s", value=round(value, 4), unit="Gcell-updates/s", n_gpus=world,
               steps=args.steps, warmup=args.warmup, ms_per_step=round(ms_per_step, 5),
               higher_is_better=True, scaling="weak", vs_baseline=None, dtype=W.dtype, data="synthetic",
               config=dict(workload=W.desc, name=W.name, cells=W.cells, blocks=list(W.nb),
                           block_cells=list(W.n), parallelism=f"replicas x{world}",
                           l2="flushed between steps (untimed 252 MB write)" if W.needs_flush()
                           else "inputs larger than L2"),
               roofline=roof, e2e=e2e, clocks=clocks, gpu_launches=W.launches_per_step * args.steps)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = W.cpu_sample(os.cpu_count() or 1)
    return out


def run_reference(args, world, rank):
    if rank != 0:
        return None
    W = WORKLOADS[args.workload]
    import oracle as O
    threads = os.cpu_count() or 1
    w = W.__new__(W)
    w.cells = int(np.prod(W.nb)) * int(np.prod(W.n))
    w.host = c1_field(W.nb, W.n, O.block_stride(W.n, np.float64))
    for _ in range(args.warmup):
        w.cpu_sample(threads)
    vals, secs = [], []
    for _ in range(args.steps):
        r = w.cpu_sample(threads)
        vals.append(r["value"])
        secs.append(r["seconds_per_sweep"])
    v = float(np.median(vals))
    base = dict(value=round(v, 4), unit="Gcell-updates/s", cores=r["cores"], kind=r["kind"], sample=r["sample"])
    return dict(impl="reference", metric="Gcell-updates/s", value=round(v, 4), unit="Gcell-updates/s",
                n_gpus=world, steps=args.steps, warmup=args.warmup, ms_per_step=round(1e3 * float(np.median(secs)), 4),
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype=W.dtype, data="synthetic",
                config=dict(workload=W.desc, name=W.name, cells=w.cells, parallelism="host threads"),
                cpu_baseline=base,
                e2e=dict(value=round(v, 4), unit="Gcell-updates/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu DRAM bytes per launch of the dominant kernel, if measured")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # the reference arm is the host CPU path: rank 0 alone runs it
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        out = run_reference(args, world, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        out = run_ours(args, world, rank, local, pg)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
