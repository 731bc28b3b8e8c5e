"""Benchmark of the B200 lab-fill + stencil path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workloads (synthetic inputs of the shapes named in the reference's benchmark
descriptions; FP64 unless stated):

  c2     (default, the headline) compressible Euler, 512^3 cells = 16^3 blocks
         of 32^3, 5 conserved variables, FP64: one SSP-RK3 step = 3 fused
         kernels, each lab(-3,4) + WENO5-JS + Rusanov + flux divergence + the
         stage update; BCs x periodic, y absorbing, z Dirichlet (far field).
         Metric counts cell-updates per RK stage.
  c4     the same Euler step at 1024^3 cells (32^3 blocks of 32^3), FP32.
  c3     two-level AMR layout, 2048 blocks drawn by seed from 8^3/16^3/32^3
         cells (50/35/15 %), FP64 Euler, one CUDA graph (3 persistent
         launches) per SSP-RK3 step.
  c1     128^3 cells = 8^3 blocks of 16^3, one scalar, lab (-1,2) + 7-point
         Laplacian + central gradient fused (one kernel per step).
  c5     variable-coefficient Poisson div(k grad p) = f, 256^3 cells = 8^3
         blocks of 32^3: one step = one multigrid solve from zero to relative
         residual 1e-8 (metric: cells solved per second); the learned
         smoother's solve is reported beside it.
  lab    FieldLab::loadData of every block of the c2 state (cn_lab_fill, one
         launch per component), stencil (-3,4): the explicit ghost fill.
  io / io_read   the Field2AOS / AOS2Field gathers of CartesianWriteHDF /
         CartesianReadHDF (512^3 cells, 3 components).

A step is one pass of the path over the whole grid.  ``value`` is whole-job
Gcell-updates/s with inputs resident in HBM (kernel time from CUDA events on
the launching stream); ``e2e`` is the same metric through the C ABI with the
input uploaded from pinned host memory and the outputs read back every step.
Multi-GPU runs are independent replicas (the path does not shard across GPUs
in this build): scaling "weak", value = all ranks' cells / max-over-ranks time.

The default run (c2 at N = 1) then times the other workloads briefly on the
same GPU (``companions``: 3 warm-up and 5 timed steps each; --no-companions
skips them, as profiling runs do).
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
def dist_setup(args, backend=None):
    """One process per GPU under torchrun (RANK / LOCAL_RANK / WORLD_SIZE);
    NCCL unless `backend` says otherwise (the CPU tests use gloo)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = backend or "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, value: float) -> float:
    """Largest value over the ranks (device times: the job's time is the slowest rank's)."""
    if pg is None:
        return value
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
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
        self.updates_per_step = self.cells
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

    def step(self, stream, events=None):
        if events is not None:
            events[0].record(stream)
        self.cn.ops.lap_grad(self.u, self.lap, self.grad, stream=stream)
        if events is not None:
            events[1].record(stream)

    launches_per_step = 1
    bytes_per_cell_step = 40
    # DRAM bytes per cell per step from one ncu capture (dram__bytes_read.sum +
    # dram__bytes_write.sum, mean of 3 launches) of this workload: the field
    # (16.8 MB) is read from DRAM, the 67 MB of results mostly stay dirty in the
    # 126 MB L2 and are written back during the flush that follows
    traffic_per_cell_step = 11.12
    traffic_source = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of fd_kernel on this workload, "
                      "mean of 3 launches; results stay dirty in L2 and are written back during the flush")

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

    @classmethod
    def cpu_sample_static(cls, threads, reps=3):
        """Reference FieldLab + Laplacian/gradient loops (oracle/_ref) on the
        full grid, or the C oracle without the reference build."""
        import oracle as O
        host = c1_field(cls.nb, cls.n, O.block_stride(cls.n, np.float64))
        cells = int(np.prod(cls.nb)) * int(np.prod(cls.n))
        h = 1.0 / 128
        kind = "reference" if O.ref_available() else "port"
        if kind == "reference":
            t, _, _ = O.ref_c1_sweep(host, cls.nb, cls.n, (1 / h / h,) * 3, (1 / h,) * 3,
                                     threads=threads, reps=reps)
        else:
            t0 = time.perf_counter()
            O.laplacian_f64(host, cls.nb, cls.n, {}, (1 / h / h,) * 3)
            O.gradient_f64(host, cls.nb, cls.n, {}, (1 / h,) * 3)
            t = time.perf_counter() - t0
            threads = 1
        return dict(value=cells / t / 1e9, unit="Gcell-updates/s", cores=threads, kind=kind,
                    sample=f"full 128^3 sweep (lab+Laplacian+gradient), best of {reps}, {threads} threads",
                    seconds_per_sweep=t)

    def cpu_sample(self, threads):
        """About 10 s of host work: the full sweep, repeated."""
        t1 = self.cpu_sample_static(threads, reps=1)["seconds_per_sweep"]
        return self.cpu_sample_static(threads, reps=int(min(2000, max(1, 10.0 / t1))))


# FP64/FP32 operations per cell and RK stage of the Euler kernel (fma = 2,
# div = sqrt = 1), each cell and face counted once: per direction and
# variable the cell's WENO5 smoothness indicators and weight products (42;
# FP32 45 with the three power-of-two rescaling products) and its left- and
# right-biased states (24 each); per face the divisions of the five
# variables' states (variables paired, 2 x 14 + 6 = 34) and the Rusanov flux
# (74); per cell the primitive conversion (12), the flux differences (40) and
# the stage update (20).  Integer instructions and work the kernel repeats at
# tile and run edges are not counted.
EULER_FLOPS_PER_CELL_STAGE = {"f64": 3 * (5 * (42 + 24 + 24) + 34 + 74) + 12 + 40 + 20,
                              "f32": 3 * (5 * (45 + 24 + 24) + 34 + 74) + 12 + 40 + 20}


def euler_host_state(nb, n, block_stride, gamma=1.4, seed=1234):
    """The Euler pulse recipe on the host (numpy), grid layout, for CPU samples."""
    nbk = int(np.prod(nb))
    cells = int(np.prod(n))
    h = [1.0 / (nb[d] * n[d]) for d in range(3)]
    xs = [(np.arange(nb[d] * n[d]) + 0.5) * h[d] for d in range(3)]
    r2 = ((xs[2][:, None, None] - 0.5) ** 2 + (xs[1][None, :, None] - 0.5) ** 2 +
          (xs[0][None, None, :] - 0.5) ** 2)
    rho = 1.0 + 0.5 * np.exp(-r2 / (2 * 0.1 * 0.1))
    rho = rho.reshape(nb[2], n[2], nb[1], n[1], nb[0], n[0]).transpose(0, 2, 4, 1, 3, 5).reshape(nbk, cells)
    rng = np.random.default_rng(seed)
    vel = (rng.random((3, nbk, cells)) * 2 - 1) * 1e-2
    U = np.zeros((5, nbk, block_stride))
    U[0, :, :cells] = rho
    U[1:4, :, :cells] = rho[None] * vel
    U[4, :, :cells] = 1.0 / (gamma - 1.0) + 0.5 * rho * (vel ** 2).sum(0)
    return U.reshape(5, -1)


def euler_bclists_host(nb, gamma=1.4):
    ff = (1.0, 0.0, 0.0, 0.0, 1.0 / (gamma - 1.0))
    out = []
    for c in range(5):
        d = {}
        for b in range(int(np.prod(nb))):
            bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
            lst = []
            if bi[1] == 0:
                lst.append((1, 0, 2, 0.0))
            if bi[1] == nb[1] - 1:
                lst.append((1, 1, 2, 0.0))
            if bi[2] == 0:
                lst.append((2, 0, 1, ff[c]))
            if bi[2] == nb[2] - 1:
                lst.append((2, 1, 1, ff[c]))
            if lst:
                d[b] = lst
        out.append(d)
    return out


class Euler:
    """SSP-RK3 step of the compressible Euler equations (three fused stage kernels)."""
    stages = 3
    launches_per_step = 3
    bytes_per_cell_step = 80 + 120 + 120  # stage 1 reads U, writes U1; stages 2, 3 also read U^n
    # DRAM bytes per cell per step of the three stage launches from one ncu
    # capture on 8x8x4 blocks of 32^3 (8.4 M cells, inputs 5x larger than L2),
    # scaled to the workload's cells: traffic grows with the cells processed
    traffic_per_cell_step = 327.80
    traffic_source = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 3 stage_kernel launches "
                      "of one step on 8x8x4 blocks of 32^3, per cell, scaled by the workload's cells")
    sample_nb = (4, 4, 4)  # CPU sample grid: 64 blocks of the same block size

    def __init__(self):
        import torch

        import cubismnova_b200 as cn
        self.cn, self.torch = cn, torch
        npdt = np.float64 if self.dtype == "f64" else np.float32
        self.U = cn.Grid.Cartesian(self.nb, self.n, ncomp=5, dtype=npdt)
        self.w1, self.w2 = cn.euler.like(self.U), cn.euler.like(self.U)
        cn.workloads.euler_pulse(self.U)
        cn.workloads.euler_bcs(self.U)
        self.U.sync_bcs()
        self.dt = cn.euler.cfl_dt(self.U, 0.3)
        self.cells = int(np.prod(self.nb)) * int(np.prod(self.n))
        self.updates_per_step = self.cells * self.stages
        self.flops_per_cell_stage = EULER_FLOPS_PER_CELL_STAGE[self.dtype]
        self.h_state = None

    def needs_flush(self):
        return False  # 5 components x cells x itemsize >> 126 MB of L2

    def step(self, stream, events=None):
        if events is None:
            self.cn.euler.rk3_step(self.U, self.w1, self.w2, self.dt, stream=stream)
            return
        e = self.cn.euler
        events[0].record(stream)
        e.rk3_stage(self.U, self.U, None, self.w1, 1, self.dt, stream=stream)
        events[1].record(stream)
        e.rk3_stage(self.U, self.w1, self.U, self.w2, 2, self.dt, stream=stream)
        events[2].record(stream)
        e.rk3_stage(self.U, self.w2, self.U, self.U, 3, self.dt, stream=stream)
        events[3].record(stream)

    def e2e_step(self, stream):
        import ctypes as C
        lib = self.cn._lib.lib()
        torch = self.torch
        nbytes = self.U.comp_stride * self.U.dtype.itemsize
        if self.h_state is None:
            tdt = torch.float64 if self.dtype == "f64" else torch.float32
            self.h_state = torch.empty((5, self.U.comp_stride), dtype=tdt).pin_memory()
            for c in range(5):
                self.h_state[c].copy_(torch.from_numpy(self.U.download(c)))
        sh = C.c_void_p(stream.cuda_stream)
        for c in range(5):
            self.cn._lib.check(lib.cn_grid_upload(self.U.handle, c, C.c_void_p(self.h_state[c].data_ptr()),
                                                  nbytes, sh))
        self.step(stream)
        for c in range(5):
            self.cn._lib.check(lib.cn_grid_download(self.U.handle, c, C.c_void_p(self.h_state[c].data_ptr()),
                                                    nbytes, sh))
        return 5 * nbytes, 5 * nbytes

    e2e_path = ("C ABI, device states in turn (three when the node's pinned host copies fit in 48 GB, else two): "
                "step i+1's upload (cn_grid_upload from pinned host) and step i-1's download "
                "(cn_grid_download to pinned host) run on their own streams while step i runs; "
                "the stage work grids are shared")

    # pinned host memory the pipelined leg may hold on one node, all ranks
    E2E_PINNED_BUDGET = 48e9
    ranks_per_node = 1

    def e2e_slots(self):
        """Device states (each with a pinned host copy) the pipelined leg
        uses: three when the node's ranks' host copies fit the budget, else
        two, else one (the pipelined leg is then not run)."""
        state = 5 * self.U.comp_stride * self.U.dtype.itemsize
        for n in (3, 2):
            if n * state * self.ranks_per_node <= self.E2E_PINNED_BUDGET:
                return n
        return 1

    def e2e_pipelined(self, stream, k):
        """k independent steps (each: 5 components uploaded from pinned host
        memory, one SSP-RK3 step, 5 components downloaded) over several
        device states, so that the copy engines (one per direction) overlap
        the compute of the neighbouring steps.  With two states a state's
        upload -> step -> download chain serialises (its next upload waits
        for its download); three let the copies run back to back.  Returns
        bytes per step."""
        import ctypes as C
        torch, lib, cn = self.torch, self.cn._lib.lib(), self.cn
        nbytes = self.U.comp_stride * self.U.dtype.itemsize
        if self.h_state is None:
            self.e2e_step(stream)
            stream.synchronize()
        if getattr(self, "pipe", None) is None:
            nslots = self.e2e_slots()
            Us, hs = [self.U], [self.h_state]
            for _ in range(nslots - 1):
                U2 = cn.Grid.Cartesian(self.nb, self.n, ncomp=5, dtype=self.U.dtype)
                cn.workloads.euler_bcs(U2)
                U2.sync_bcs()
                h2 = torch.empty_like(self.h_state).pin_memory()
                h2.copy_(self.h_state)
                Us.append(U2)
                hs.append(h2)
            self.pipe = dict(U=Us, h=hs, s_in=torch.cuda.Stream(), s_out=torch.cuda.Stream())
        P = self.pipe
        s_in, s_out = P["s_in"], P["s_out"]
        nslots = len(P["U"])
        start = torch.cuda.Event()
        start.record(stream)
        s_in.wait_event(start)
        s_out.wait_event(start)
        freed = [None] * nslots
        for i in range(k):
            j = i % nslots
            U, h = P["U"][j], P["h"][j]
            if freed[j] is not None:
                s_in.wait_event(freed[j])  # the slot's previous result is home
            sh = C.c_void_p(s_in.cuda_stream)
            for c in range(5):
                cn._lib.check(lib.cn_grid_upload(U.handle, c, C.c_void_p(h[c].data_ptr()), nbytes, sh))
            up = torch.cuda.Event()
            up.record(s_in)
            stream.wait_event(up)
            cn.euler.rk3_step(U, self.w1, self.w2, self.dt, stream=stream)
            done = torch.cuda.Event()
            done.record(stream)
            s_out.wait_event(done)
            sh = C.c_void_p(s_out.cuda_stream)
            for c in range(5):
                cn._lib.check(lib.cn_grid_download(U.handle, c, C.c_void_p(h[c].data_ptr()), nbytes, sh))
            freed[j] = torch.cuda.Event()
            freed[j].record(s_out)
        for ev in freed:
            if ev is not None:
                stream.wait_event(ev)
        return 5 * nbytes, 5 * nbytes

    @classmethod
    def cpu_sample_static(cls, threads, reps=2, nb=None):
        """One SSP-RK3 stage (stage 2: lab + WENO + Rusanov + update reading U^n)
        over a sample grid of the same block size and BC pattern (default 4^3
        blocks), best of `reps`, on the reference FieldLab (oracle/_ref) or,
        without it, the C oracle."""
        import oracle as O
        nb, n = tuple(nb or cls.sample_nb), cls.n
        stride = O.block_stride(n, np.float64)
        U = euler_host_state(nb, n, stride)
        bcl = euler_bclists_host(nb)
        h = [1.0 / (nb[d] * n[d]) for d in range(3)]
        cells = int(np.prod(nb)) * int(np.prod(n))
        if O.ref_available():
            kind = "reference"
            t, _ = O.ref_euler_stage(U, U, nb, n, bcl, 2, 1e-4, 1.4, h, threads=threads, reps=reps)
        else:
            kind = "port"
            best = 1e300
            for _ in range(reps):
                t0 = time.perf_counter()
                O.euler_stage(U, U, nb, n, bcl, 2, 1e-4, 1.4, h, threads=threads)
                best = min(best, time.perf_counter() - t0)
            t = best
        return dict(value=cells / t / 1e9, unit="Gcell-updates/s", cores=threads, kind=kind,
                    sample=(f"one SSP-RK3 stage (lab(-3,4)+WENO5+Rusanov+update, FP64) on "
                            f"{nb[0]}x{nb[1]}x{nb[2]} blocks of {n[0]}^3 cells, same BCs, "
                            f"best of {reps}, {threads} threads"),
                    seconds_per_sweep=t)

    cpu_nb = (8, 8, 4)  # blocks of the CPU sample (cpu_baseline and the reference arm)

    def cpu_sample(self, threads):
        """About 10 s of host work: the stage on 8x8x4 blocks, repeated."""
        t1 = self.cpu_sample_static(threads, reps=1, nb=self.cpu_nb)["seconds_per_sweep"]
        return self.cpu_sample_static(threads, reps=int(min(100, max(1, 10.0 / t1))), nb=self.cpu_nb)


class C2(Euler):
    name = "c2"
    desc = ("Euler SSP-RK3 step, 512^3 cells as 16^3 blocks of 32^3, 5 vars, FP64, "
            "lab(-3,4)+WENO5-JS+Rusanov+divergence fused with the stage update; "
            "BCs x periodic, y absorbing, z Dirichlet")
    nb, n = (16, 16, 16), (32, 32, 32)
    dtype = "f64"


class C4(Euler):
    name = "c4"
    desc = ("Euler SSP-RK3 step, 1024^3 cells as 32^3 blocks of 32^3, 5 vars, FP32 storage "
            "and arithmetic, same fused kernels and BCs")
    nb, n = (32, 32, 32), (32, 32, 32)
    dtype = "f32"
    bytes_per_cell_step = (80 + 120 + 120) // 2
    # capture on 8x8x4 blocks (168 MB of state, comparable to L2, so slightly
    # under the full-size figure)
    traffic_per_cell_step = 156.84


class C3:
    autotune = True  # bench.py --no-autotune: the default schedule (profiling runs)
    fixed_schedule = None  # bench.py --amr-schedule ORDER CTAS TX TY TZ
    """Batched two-level AMR step: 2048 blocks whose sizes are drawn by seed
    from {8^3: 50 %, 16^3: 35 %, 32^3: 15 %} (workloads.amr_layout: about
    13.5 M cells, a level-0 tiling refined in a seeded ball), level-interface
    ghosts by trilinear prolongation and conservative restriction, FP64
    Euler; each SSP-RK3 step is one CUDA graph of three persistent launches
    over the tile work list, schedule chosen by the autotuner."""
    name = "c3"
    desc = ("AMR Euler SSP-RK3 step, 2048 blocks drawn by seed from {8^3: 50%, 16^3: 35%, 32^3: 15%} cells on "
            "2 levels (ratio 2), FP64, interface ghosts by trilinear prolongation / conservative restriction, "
            "one CUDA graph per step (3 persistent launches), autotuned schedule")
    dtype = "f64"
    stages = 3
    launches_per_step = 3
    bytes_per_cell_step = 320
    traffic_per_cell_step = 394.0
    traffic_source = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 3 stage_kernel launches of one "
                      "step on this layout (5302 MB per step), per cell and scaled to a launch")
    nb, n = ("amr", "amr")

    def __init__(self):
        import torch

        import cubismnova_b200 as cn
        self.cn, self.torch = cn, torch
        l, c, o, F = cn.workloads.amr_layout()
        self.U = cn.amr.AmrGrid(l, c, o, F)
        self.layout = dict(blocks=len(l), box_level1_cells=list(F),
                           level1_blocks=[int(np.sum((l == 1) & (c == k))) for k in (8, 16, 32)],
                           level0_blocks=[int(np.sum((l == 0) & (c == k))) for k in (8, 16, 32)])
        self.w1, self.w2 = self.U.like(), self.U.like()
        cn.workloads.euler_pulse_amr(self.U)
        self.cells = self.U.total_cells
        self.updates_per_step = self.cells * self.stages
        self.flops_per_cell_stage = EULER_FLOPS_PER_CELL_STAGE[self.dtype]
        self.nb, self.n = (len(l),), tuple(int(e) for e in F)
        # CFL on the fine level (h = 1/Lx), sound speed of the pulse state < 1.3
        self.dt = 0.3 / (3 * 1.3 * F[0])
        def work_tile(shape):
            return (f"{8 * shape[0]}x{8 * shape[1]}x{8 * shape[2]} cells "
                    f"({shape[0]}x{shape[1]}x{shape[2]} tiles of 8^3, clipped to the block)")
        if self.fixed_schedule is not None:
            order, ctas, shape = self.fixed_schedule[0], self.fixed_schedule[1], tuple(self.fixed_schedule[2:])
            for g in (self.U, self.w1, self.w2):
                g.set_schedule(order, ctas, shape=shape)
            self.schedule = dict(order=["block order", "largest blocks first", "Morton"][order], ctas=ctas,
                                 work_tile=work_tile(shape), autotuned=False)
        elif self.autotune:
            order, ctas, ms = cn.amr.autotune(self.U, self.w1, self.w2, self.dt, reps=2)
            self.schedule = dict(order=["block order", "largest blocks first", "Morton"][order], ctas=ctas,
                                 work_tile=work_tile(self.U.work_shape()), ms_per_step=round(ms, 3))
        else:
            self.schedule = dict(order="largest blocks first", ctas=0, work_tile=work_tile((1, 1, 1)),
                                 autotuned=False)
        cn.workloads.euler_pulse_amr(self.U)
        self.stream = torch.cuda.Stream()
        cn.amr.rk3_step(self.U, self.w1, self.w2, self.dt, stream=self.stream)  # eager once before capture
        self.stream.synchronize()
        cn.workloads.euler_pulse_amr(self.U)
        self.graph = cn.amr.Graph.capture(
            lambda: cn.amr.rk3_step(self.U, self.w1, self.w2, self.dt, stream=self.stream), self.stream)
        self.h_state = None
        self.desc = self.desc + f"; layout {self.layout}; schedule {self.schedule}"

    def needs_flush(self):
        return False

    def step(self, stream, events=None):
        if events is not None:
            events[0].record(stream)
        self.graph.launch(stream)
        if events is not None:
            for e in events[1:]:
                e.record(stream)

    def e2e_step(self, stream):
        torch = self.torch
        if self.h_state is None:
            self.h_state = torch.empty((5, self.U.comp_stride), dtype=torch.float64).pin_memory()
            for k in range(5):
                self.h_state[k].copy_(self.U.tensor(k))
        with torch.cuda.stream(stream):
            for k in range(5):
                self.U.tensor(k).copy_(self.h_state[k], non_blocking=True)
            self.graph.launch(stream)
            for k in range(5):
                self.h_state[k].copy_(self.U.tensor(k), non_blocking=True)
        nbytes = 5 * self.U.comp_stride * 8
        return nbytes, nbytes

    @classmethod
    def cpu_sample_static(cls, threads, reps=1):
        """The C oracle (no reference AMR code exists) on the small two-level
        layout (99 blocks, 104 k cells), one RK3 stage, blocks spread over all
        host threads (OpenMP)."""
        import oracle as O

        from cubismnova_b200 import workloads as WL
        l, c, o, F = WL.amr_small_layout()
        blk, tot = O.amr_blocks(l, c, o, F)
        rng = np.random.default_rng(0)
        U = np.zeros((5, tot))
        U[0] = 1 + 0.1 * rng.random(tot)
        U[4] = 2.5
        best = 1e300
        for _ in range(max(1, reps)):
            t0 = time.perf_counter()
            O.amr_stage(U, U, blk, F, 2, 1e-4, 1.4)
            best = min(best, time.perf_counter() - t0)
        ncpu = len(os.sched_getaffinity(0))
        return dict(value=tot / best / 1e9, unit="Gcell-updates/s", cores=ncpu, kind="port",
                    sample=f"one SSP-RK3 stage of the C oracle on the small two-level layout ({len(l)} blocks, "
                           f"{tot} cells), {ncpu} threads, best of {max(1, reps)}",
                    seconds_per_sweep=best)

    def cpu_sample(self, threads):
        """About 10 s of host work: the stage repeated."""
        t1 = self.cpu_sample_static(threads, reps=1)["seconds_per_sweep"]
        return self.cpu_sample_static(threads, reps=int(min(500, max(1, 10.0 / t1))))


def poisson_host(nb, n, seed=1234, sigma=0.5, count=32):
    """Host (numpy) Poisson problem of the same construction as the device
    workload generators: k = 3-cell box filter of exp(N(0, sigma^2)), f = sum
    of Gaussians minus its mean; both FP32 in block layout."""
    import oracle as O
    rng = np.random.default_rng(seed)
    G = [nb[d] * n[d] for d in range(3)]
    a = np.exp(rng.standard_normal((G[2], G[1], G[0])) * sigma)
    for ax in range(3):
        a = (np.roll(a, 1, ax) + a + np.roll(a, -1, ax)) / 3.0
    xs = [(np.arange(G[d]) + 0.5) / G[d] for d in range(3)]
    f = np.zeros((G[2], G[1], G[0]))
    for _ in range(count):
        c, w, amp = rng.random(3), 0.02 + 0.06 * rng.random(), -1.0 + 2.0 * rng.random()
        d2 = []
        for d in range(3):
            t = xs[d] - c[d]
            t = t - np.round(t)
            d2.append(t * t)
        f += amp * np.exp(-(d2[2][:, None, None] + d2[1][None, :, None] + d2[0][None, None, :]) / (2 * w * w))
    f -= f.mean()
    s = O.block_stride(n, np.float32)
    cells = int(np.prod(n))

    def blocks(g):
        v = g.reshape(nb[2], n[2], nb[1], n[1], nb[0], n[0]).transpose(0, 2, 4, 1, 3, 5).reshape(-1, cells)
        out = np.zeros((v.shape[0], s), dtype=np.float32)
        out[:, :cells] = v
        return out.reshape(-1)
    return blocks(a), blocks(f)


class C5:
    """Multigrid solve of div(k grad p) = f (periodic, variable k) to a
    relative residual of 1e-8: FP32 V-cycles (2+2 weighted-Jacobi sweeps,
    omega 6/7, fused residual restriction, trilinear prolongation, FP64 CG on
    the coarsest level) inside an FP64 defect correction; one step is a whole
    solve from p = 0.  The learned smoother (trained untimed on this problem's
    residual patches, replacing Jacobi on the finest level) is timed beside it
    and reported in the config."""
    nn_training = "tensor"  # bench.py --nn-training fp32: the CUDA-core training path
    # Jacobi damping: 6/7 minimises the largest amplification of the
    # high-frequency error modes for the 7-point operator in 3-D (standard
    # local Fourier analysis of damped Jacobi); measured on this problem: 15
    # V(2,2) cycles, 23.4 ms, against 16 cycles, 25.0 ms at omega 0.8
    omega = 6.0 / 7.0
    nu = (2, 2)  # pre- and post-smoothing sweeps (bench.py --mg-nu, --mg-omega)
    name = "c5"
    desc = ("Poisson div(k grad p) = f, 256^3 cells as 8^3 blocks of 32^3, k = box-filtered lognormal "
            "(sigma 0.5), f = 32 Gaussians; multigrid V(2,2) weighted Jacobi (omega 6/7), FP32 cycles in "
            "FP64 defect correction, solved from zero to relative residual 1e-8")
    nb, n = (8, 8, 8), (32, 32, 32)
    dtype = "f32"
    metric = unit = "Gcell/s solved to 1e-8"
    launches_per_step = 1  # the events bracket the whole solve
    with_learned = True
    roofline_scope = ("whole solve (all kernels and the per-cycle host check of the residual norm) against "
                      "its compulsory HBM bytes")
    rtol = 1e-8
    sample_nb = (2, 2, 2)

    def __init__(self):
        import torch

        import cubismnova_b200 as cn
        self.cn, self.torch = cn, torch
        self.k = cn.Grid.Cartesian(self.nb, self.n, dtype=np.float32)
        cn.workloads.poisson_coefficient(self.k, seed=1)
        self.f = cn.Grid.Cartesian(self.nb, self.n, dtype=np.float32)
        cn.workloads.poisson_rhs(self.f, seed=2)
        self.p64 = cn.Grid.Cartesian(self.nb, self.n, dtype=np.float64)
        self.mg = cn.mg.Multigrid(self.k, nu1=self.nu[0], nu2=self.nu[1], omega=self.omega)
        om = "6/7" if abs(self.omega - 6.0 / 7.0) < 1e-12 else f"{self.omega:g}"
        self.desc = self.desc.replace("V(2,2) weighted Jacobi (omega 6/7)",
                                      f"V({self.nu[0]},{self.nu[1]}) weighted Jacobi (omega {om})")
        self.cells = int(np.prod(self.nb)) * int(np.prod(self.n))
        self.updates_per_step = self.cells
        self.cycles, self.relres = self.mg.solve(self.f, self.p64, self.rtol, max_cycles=100)
        torch.cuda.synchronize()
        # kernels per solve: initial residual (2), per cycle 6 per non-coarsest
        # level + coarsest CG + accumulate + residual (2)
        L = self.mg.nlevels
        self.gpu_launches_per_step = 2 + self.cycles * (6 * (L - 1) + 4)
        # compulsory HBM bytes per fine cell (FP32 4 B, FP64 8 B): a V(2,2)
        # level pass moves 81 B per level cell (Jacobi from zero 12, Jacobi 16
        # x 3, residual restriction 12.5, prolongation 8.5), the coarsest CG
        # 12 B, accumulate + FP64 residual 40 B per fine cell; 28 B once
        ncl = [self.cells // 8 ** l for l in range(L)]
        per_cycle = 81 * sum(ncl[:-1]) + 12 * ncl[-1] + 40 * ncl[0]
        self.bytes_per_cell_step = (28 * self.cells + self.cycles * per_cycle) / self.cells
        self.learned = self._learned() if self.with_learned else None
        self.desc = self.desc + f"; {L} levels, {self.cycles} cycles (relres {self.relres:.2e})"
        self.h_f = self.h_p = None

    # learned-smoother schedules timed beside the plain solve: (name, pre
    # mask, post mask, pre applications, post applications); -1 = nu1 / nu2
    LEARNED_SCHEDULES = (
        ("learned pre + post on the finest level, 2 + 2 applications", 1, 1, -1, -1),
        ("learned pre + post on the finest level, 1 + 1", 1, 1, 1, 1),
        ("learned post on the finest level (1), Jacobi pre (2)", 0, 1, -1, 1),
        ("learned post on the finest level (2), Jacobi pre (2)", 0, 1, -1, 2),
        ("learned pre on the finest level (1), Jacobi post (2)", 1, 0, 1, -1),
    )

    def _learned(self):
        """Train the learned smoother (untimed in the metric; its wall time is
        reported) on 2000 residual/error pairs of the plain V-cycle, then time
        solves with it under each schedule of LEARNED_SCHEDULES and the plain
        solve, on the same problem."""
        cn, torch = self.cn, self.torch
        try:
            x, k, r, P = cn.learned.collect_patches(self.mg, self.f, cycles=8, per_snapshot=125, max_patches=2000,
                                                    seed=5)
            npatch = int(x.shape[0])
            ih2 = 1.0 / self.k.getCellSize()[0] ** 2
            # untimed warm-up on a throwaway network: first launches of the
            # training kernels (module loading) and the host paths
            scratch = cn.learned.LearnedSmoother(seed=9, omega=0.8, init_scale=1e-3)
            scratch.set_training(self.nn_training)
            scratch.train(x[:64], k[:64], r[:64], P, ih2, epochs=1, batch=32, lr=2e-3, seed=1)
            scratch.close()
            nn = cn.learned.LearnedSmoother(seed=1, omega=0.8, init_scale=1e-3)
            nn.set_training(self.nn_training)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            loss = nn.train(x, k, r, P, ih2, epochs=8, batch=32, lr=2e-3, seed=2)
            torch.cuda.synchronize()
            train_s = time.perf_counter() - t0
            del x, k, r
            p = cn.Grid.Cartesian(self.nb, self.n, dtype=np.float64)

            def timed(m2):
                m2.solve(self.f, p, self.rtol, max_cycles=60)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                cyc, rel = m2.solve(self.f, p, self.rtol, max_cycles=60)
                e1.record()
                torch.cuda.synchronize()
                return dict(cycles=cyc, relres=float(rel), ms_per_solve=round(e0.elapsed_time(e1), 3))

            table = [dict(schedule="plain Jacobi V(2,2)",
                          **timed(cn.mg.Multigrid(self.k, nu1=2, nu2=2, omega=self.omega)))]
            for name, pre, post, na, nb in self.LEARNED_SCHEDULES:
                m2 = cn.mg.Multigrid(self.k, nu1=2, nu2=2, omega=self.omega)
                cn.learned.use_in(m2, nn, level_mask=pre, post_mask=post, pre_apps=na, post_apps=nb)
                table.append(dict(schedule=name, **timed(m2)))
                del m2
            ok = [t for t in table[1:] if t["relres"] <= self.rtol]
            best = min(ok, key=lambda t: t["ms_per_solve"]) if ok else None
            nbatches = 8 * (npatch // 32)
            return dict(train_patches=npatch, train_loss=round(float(loss), 4),
                        train_seconds=round(train_s, 2), train_ms_per_batch=round(1e3 * train_s / nbatches, 3),
                        training=("hidden layer forward, data and weight gradients on tcgen05 (BF16 operands, "
                                  "FP32 accumulation); first and last layers on the CUDA cores"
                                  if self.nn_training == "tensor" else "FP32 on the CUDA cores throughout")
                        + "; 8 epochs of batches of 32, Adam",
                        schedules=table,
                        best=best["schedule"] if best else None,
                        ms_per_solve=best["ms_per_solve"] if best else None,
                        cycles=best["cycles"] if best else None,
                        smoother="3-layer 3^3 conv net, 16 channels, BF16 tensor-core inference")
        except Exception as e:  # reported, not fatal: the plain solve is the metric
            return dict(error=str(e)[:200])

    def needs_flush(self):
        return False  # 256^3 FP32 + FP64 grids and the hierarchy exceed the 126 MB L2

    def step(self, stream, events=None):
        if events is not None:
            events[0].record(stream)
        self.mg.solve(self.f, self.p64, self.rtol, max_cycles=100, stream=stream)
        if events is not None:
            events[1].record(stream)

    def e2e_step(self, stream):
        import ctypes as C
        torch, lib = self.torch, self.cn._lib.lib()
        fb = self.f.comp_stride * 4
        pb = self.p64.comp_stride * 8
        if self.h_f is None:
            self.h_f = torch.from_numpy(self.f.download(0)).pin_memory()
            self.h_p = torch.empty(self.p64.comp_stride, dtype=torch.float64).pin_memory()
        sh = C.c_void_p(stream.cuda_stream)
        self.cn._lib.check(lib.cn_grid_upload(self.f.handle, 0, C.c_void_p(self.h_f.data_ptr()), fb, sh))
        self.step(stream)
        self.cn._lib.check(lib.cn_grid_download(self.p64.handle, 0, C.c_void_p(self.h_p.data_ptr()), pb, sh))
        return fb, pb

    @classmethod
    def cpu_sample_static(cls, threads, reps=1):
        """The C oracle's multigrid (same algorithm; the cell loops spread over
        all host threads with OpenMP, the coarsest CG on one) solving a 64^3
        problem of the same construction (2^3 blocks of 32^3) to 1e-8."""
        import oracle as O
        nb, n = cls.sample_nb, cls.n
        k, f = poisson_host(nb, n)
        cells = int(np.prod(nb)) * int(np.prod(n))
        best, cyc = 1e300, 0
        for _ in range(max(1, reps)):
            t0 = time.perf_counter()
            _, cyc, rel = O.mg_solve(k, f, nb, n, 1.0 / (nb[0] * n[0]), omega=cls.omega, rtol=cls.rtol,
                                     max_cycles=40)
            best = min(best, time.perf_counter() - t0)
        ncpu = len(os.sched_getaffinity(0))
        return dict(value=cells / best / 1e9, unit=cls.unit, cores=ncpu, kind="port",
                    sample=(f"C oracle multigrid, {nb[0] * n[0]}^3 cells ({nb[0]}^3 blocks of {n[0]}^3), "
                            f"{cyc} cycles to relres {rel:.1e}, {ncpu} threads, best of {max(1, reps)}"),
                    seconds_per_sweep=best)

    def cpu_sample(self, threads):
        return self.cpu_sample_static(threads)


class LAB:
    """FieldLab::loadData of every block (Cartesian::loadLab over the grid,
    Block/FieldLab.h:180-224; ``cn_lab_fill`` over a block range, one launch
    per component): the C2 state (512^3 cells as 16^3 blocks of 32^3, FP64,
    5 components, x periodic, y absorbing, z Dirichlet), stencil (-3, 4)
    non-tensorial: 38^3 labs whose 6 x 3 x 32^2 face ghosts are written and
    whose edges and corners stay undefined, as in the reference."""
    name = "lab"
    desc = ("FieldLab::loadData of all 4096 blocks (cn_lab_fill, one launch per component): C2 state, 512^3 "
            "cells as 16^3 blocks of 32^3, 5 FP64 components, stencil (-3,4) non-tensorial, BCs x periodic, "
            "y absorbing, z Dirichlet; 38^3 labs")
    nb, n = (16, 16, 16), (32, 32, 32)
    dtype = "f64"
    metric = unit = "Gcell/s"
    launches_per_step = 5
    # per block cell and component: the block's cell read (8 B) and its share
    # of the written lab cells, (32^3 + 6 x 3 x 32^2) / 32^3 x 8 B = 12.5 B;
    # ghost cells read from neighbours are re-reads and not counted
    bytes_per_cell_step = 5 * (8 + 8 * (32 ** 3 + 6 * 3 * 32 ** 2) / 32 ** 3)
    # DRAM bytes per cell of one ncu capture of a launch on 8x8x8 blocks of
    # 32^3 (147.6 MB read + 163.6 MB written for 16.8 M cells, mean of 3
    # launches), times the 5 launches of a step; traffic grows with the
    # blocks processed
    traffic_per_cell_step = 92.7
    traffic_source = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of lab_fill_rows_kernel on 8x8x8 blocks "
                      "of 32^3 (mean of 3 launches), per cell, times the 5 launches of a step")
    cpu_nb = (8, 8, 4)

    def __init__(self):
        import torch

        import cubismnova_b200 as cn
        self.cn, self.torch = cn, torch
        self.U = cn.Grid.Cartesian(self.nb, self.n, ncomp=5)
        cn.workloads.euler_pulse(self.U)
        cn.workloads.euler_bcs(self.U)
        self.U.sync_bcs()
        self.stencil = cn.Core.Stencil(-3, 4, False)
        self.labs = cn.ops.load_labs(self.U, self.stencil, comp=0)
        self.cells = int(np.prod(self.nb)) * int(np.prod(self.n))
        self.updates_per_step = 5 * self.cells
        self.h_state = None
        self.h_labs = None

    def needs_flush(self):
        return False  # 1.07 GB read and 1.8 GB written per launch

    def step(self, stream, events=None):
        for c in range(5):
            if events is not None:
                events[c].record(stream)
            self.cn.ops.load_labs(self.U, self.stencil, out=self.labs, comp=c, stream=stream)
        if events is not None:
            events[5].record(stream)

    def e2e_step(self, stream):
        """Each component uploaded from pinned host memory, its labs filled
        and downloaded to pinned host memory."""
        import ctypes as C
        torch = self.torch
        lib = self.cn._lib.lib()
        nbytes = self.U.comp_stride * 8
        if self.h_state is None:
            self.h_state = torch.empty((5, self.U.comp_stride), dtype=torch.float64).pin_memory()
            for c in range(5):
                self.h_state[c].copy_(self.U.tensor(c).reshape(-1))
            self.h_labs = torch.empty(self.labs.shape, dtype=self.labs.dtype).pin_memory()
        sh = C.c_void_p(stream.cuda_stream)
        for c in range(5):
            self.cn._lib.check(lib.cn_grid_upload(self.U.handle, c, C.c_void_p(self.h_state[c].data_ptr()),
                                                  nbytes, sh))
            self.cn.ops.load_labs(self.U, self.stencil, out=self.labs, comp=c, stream=stream)
            with torch.cuda.stream(stream):
                self.h_labs.copy_(self.labs, non_blocking=True)
        return 5 * nbytes, 5 * self.labs.numel() * 8

    @classmethod
    def cpu_sample_static(cls, threads, reps=1, nb=None):
        """The reference's FieldLab::loadData (oracle/_ref) of every block of a
        8x8x4-block grid of 32^3 with the C2 BCs, all 5 components, on
        `threads` host threads with one lab each (the loadLab pattern of the
        reference's own threaded tests); the C oracle, one lab at a time,
        without the reference build."""
        import ctypes as C

        import oracle as O
        nb = tuple(nb or cls.cpu_nb)
        n = cls.n
        stride = O.block_stride(n, np.float64)
        U = euler_host_state(nb, n, stride)
        bcl = euler_bclists_host(nb)
        nblocks = int(np.prod(nb))
        kind = "reference" if O.ref_available() else "port"
        if kind == "reference":
            best = O.ref_lab_sweep(U, nb, n, bcl, 3, 3, threads=threads, reps=max(1, reps))
        else:
            threads = 1
            g = O.make_geom(nb, n, (3, 3, 3), (3, 3, 3), False, stride)
            E = [n[d] + 6 for d in range(3)]
            lab = np.zeros((E[2], E[1], E[0]))
            w = np.zeros((E[2], E[1], E[0]), dtype=np.uint8)
            best = 1e300
            for _ in range(max(1, reps)):
                t0 = time.perf_counter()
                for c in range(5):
                    off, ents = O.bc_arrays(nblocks, bcl[c])
                    for b in range(nblocks):
                        O.lib().or_lab_fill_f64(C.byref(g), O._ptr(np.ascontiguousarray(U[c])), O._ptr(off), ents,
                                                C.c_int(b), O._ptr(lab), O._ptr(w))
                best = min(best, time.perf_counter() - t0)
        cells = nblocks * int(np.prod(n)) * 5
        return dict(value=cells / best / 1e9, unit="Gcell/s", cores=threads, kind=kind,
                    sample=f"labs of all {nblocks} blocks of 32^3 ({nb[0]}x{nb[1]}x{nb[2]}) x 5 components, "
                           f"stencil (-3,4), C2 BCs, {threads} threads, best of {max(1, reps)}",
                    seconds_per_sweep=best)

    def cpu_sample(self, threads):
        """About 10 s of host work: the sample repeated."""
        t1 = self.cpu_sample_static(threads, reps=1)["seconds_per_sweep"]
        return self.cpu_sample_static(threads, reps=int(min(500, max(1, 10.0 / t1))))


class IOW:
    """Grid -> file buffer of IO::CartesianWriteHDF<float> (IO/CartesianHDF.h:76-80,
    Field2AOS of IO/FieldAOS.h:79-101): a rank-1 FP64 cell grid gathered into
    one (z, y, x, 3) FP32 array-of-structures buffer."""
    name = "io"
    desc = ("Field2AOS block loop of CartesianWriteHDF<float>: 3-component FP64 cell grid, 512^3 cells as "
            "16^3 blocks of 32^3, into one (z, y, x, 3) FP32 file buffer")
    nb, n = (16, 16, 16), (32, 32, 32)
    dtype = "f64"
    metric = unit = "Gcell/s"
    launches_per_step = 1
    bytes_per_cell_step = 36  # 3 x 8 B read, 3 x 4 B written
    cpu_blocks = (8, 8, 4)

    def __init__(self):
        import torch

        import cubismnova_b200 as cn
        self.cn, self.torch = cn, torch
        self.u = cn.Grid.Cartesian(self.nb, self.n, ncomp=3)
        gen = torch.Generator(device="cuda").manual_seed(1234)
        for c in range(3):
            self.u.tensor(c).uniform_(-1.0, 1.0, generator=gen)
        top = [self.nb[d] * self.n[d] for d in range(3)]
        self.buf = torch.empty((top[2], top[1], top[0], 3), dtype=torch.float32, device="cuda")
        self.cells = int(np.prod(top))
        self.updates_per_step = self.cells
        # pinned host copies for the end-to-end leg: the grid's components in
        # the reference layout and the file buffer
        self.h_in = [self.u.tensor(c).cpu().pin_memory() for c in range(3)]
        self.h_out = torch.empty(self.buf.shape, dtype=torch.float32).pin_memory()

    def needs_flush(self):
        return False  # 3.2 GB of input, 1.6 GB of output: far larger than L2

    def step(self, stream, events=None):
        if events is not None:
            events[0].record(stream)
        self.cn.IO.Field2AOS(self.u, file_dtype=np.float32, out=self.buf, stream=stream)
        if events is not None:
            events[1].record(stream)

    def e2e_step(self, stream):
        import ctypes as C
        lib = self.cn._lib.lib()
        sh = C.c_void_p(stream.cuda_stream)
        nbytes = self.u.comp_stride * 8
        for c in range(3):
            self.cn._lib.check(lib.cn_grid_upload(self.u.handle, c, C.c_void_p(self.h_in[c].data_ptr()), nbytes, sh))
        self.step(stream)
        with self.torch.cuda.stream(stream):
            self.h_out.copy_(self.buf, non_blocking=True)
        return 3 * nbytes, self.buf.numel() * 4

    E2E_PINNED_BUDGET = 48e9
    ranks_per_node = 1
    e2e_path = ("C ABI, device slots in turn: step i+1's upload (cn_grid_upload from pinned host) and step "
                "i-1's download of the file buffer to pinned host run on their own streams while step i "
                "gathers (cn_grid_to_aos)")

    def _pinned_bytes(self, n):
        """Pinned host bytes of n slots: the shared input copy plus one output per slot."""
        return 3 * self.u.comp_stride * 8 + n * self.buf.numel() * 4

    def e2e_slots(self):
        for n in (3, 2):
            if self._pinned_bytes(n) * self.ranks_per_node <= self.E2E_PINNED_BUDGET:
                return n
        return 1

    def _new_slot(self):
        torch = self.torch
        u = self.cn.Grid.Cartesian(self.nb, self.n, ncomp=3)
        return dict(u=u, buf=torch.empty_like(self.buf), out=torch.empty_like(self.h_out).pin_memory())

    def _slot0(self):
        return dict(u=self.u, buf=self.buf, out=self.h_out)

    def _upload(self, slot, s):
        import ctypes as C
        lib = self.cn._lib.lib()
        for c in range(3):
            self.cn._lib.check(lib.cn_grid_upload(slot["u"].handle, c, C.c_void_p(self.h_in[c].data_ptr()),
                                                  self.u.comp_stride * 8, C.c_void_p(s.cuda_stream)))

    def _compute(self, slot, s):
        self.cn.IO.Field2AOS(slot["u"], file_dtype=np.float32, out=slot["buf"], stream=s)

    def _download(self, slot, s):
        with self.torch.cuda.stream(s):
            slot["out"].copy_(slot["buf"], non_blocking=True)

    def _bytes(self):
        return 3 * self.u.comp_stride * 8, self.buf.numel() * 4

    def e2e_pipelined(self, stream, k):
        """k independent steps (upload, gather or scatter, download) over
        several device slots so that both copy directions overlap the
        neighbouring steps' kernels.  A slot's next upload waits until its
        kernel has read it, its next kernel until its result is home."""
        torch = self.torch
        if getattr(self, "pipe", None) is None:
            slots = [self._slot0()] + [self._new_slot() for _ in range(self.e2e_slots() - 1)]
            self.pipe = dict(slots=slots, s_in=torch.cuda.Stream(), s_out=torch.cuda.Stream())
        P = self.pipe
        s_in, s_out, slots = P["s_in"], P["s_out"], P["slots"]
        start = torch.cuda.Event()
        start.record(stream)
        s_in.wait_event(start)
        s_out.wait_event(start)
        used, home = [None] * len(slots), [None] * len(slots)
        for i in range(k):
            j = i % len(slots)
            if used[j] is not None:
                s_in.wait_event(used[j])
            self._upload(slots[j], s_in)
            up = torch.cuda.Event()
            up.record(s_in)
            stream.wait_event(up)
            if home[j] is not None:
                stream.wait_event(home[j])
            self._compute(slots[j], stream)
            used[j] = torch.cuda.Event()
            used[j].record(stream)
            s_out.wait_event(used[j])
            self._download(slots[j], s_out)
            home[j] = torch.cuda.Event()
            home[j].record(s_out)
        for ev in home:
            if ev is not None:
                stream.wait_event(ev)
        return self._bytes()

    @classmethod
    def cpu_sample_static(cls, threads, reps=3):
        """The reference's Field2AOS block loop (oracle/_ref, OpenMP over
        blocks as CartesianWriteHDF) on 8x8x4 blocks of 32^3, or the oracle
        restatement without the reference build."""
        import oracle as O
        from oracle import aos as A
        nb, n = cls.cpu_blocks, cls.n
        stride = O.block_stride(n, np.float64)
        rng = np.random.default_rng(1234)
        data = rng.uniform(-1.0, 1.0, size=(3, int(np.prod(nb)) * stride))
        top = [nb[d] * n[d] for d in range(3)]
        buf = np.empty(int(np.prod(top)) * 3, dtype=np.float32)
        cells = int(np.prod(top))
        if O.ref_available():
            t, _ = O.ref_field_aos(data, nb, n, 0, stride, (0, 0, 0), top, np.float32, buf, to_aos=True,
                                   threads=threads, reps=reps)
            kind = "reference"
        else:
            t0 = time.perf_counter()
            for _ in range(reps):
                A.grid_to_aos(list(data), nb, n, 0, stride, (0, 0, 0), top, buf)
            t = (time.perf_counter() - t0) / reps
            kind, threads = "port", 1
        return dict(value=cells / t / 1e9, unit="Gcell/s", cores=threads, kind=kind,
                    sample=f"Field2AOS of 3 FP64 components into FP32 AoS on {nb[0]}x{nb[1]}x{nb[2]} blocks of "
                           f"32^3 ({cells / 1e6:.1f} M cells), best of {reps}, {threads} threads",
                    seconds_per_sweep=t)

    def cpu_sample(self, threads):
        t1 = self.cpu_sample_static(threads, reps=1)["seconds_per_sweep"]
        return self.cpu_sample_static(threads, reps=int(min(200, max(3, 10.0 / t1))))


class IOR(IOW):
    """File buffer -> grid of IO::CartesianReadHDF<float> (IO/CartesianHDF.h:182-186,
    AOS2Field of IO/FieldAOS.h:103-124): one (z, y, x, 3) FP32 buffer scattered
    into a rank-1 FP64 cell grid."""
    name = "io_read"
    desc = ("AOS2Field block loop of CartesianReadHDF<float>: one (z, y, x, 3) FP32 file buffer into a "
            "3-component FP64 cell grid, 512^3 cells as 16^3 blocks of 32^3")
    bytes_per_cell_step = 36  # 3 x 4 B read, 3 x 8 B written

    def __init__(self):
        super().__init__()
        self.cn.IO.Field2AOS(self.u, file_dtype=np.float32, out=self.buf)
        self.torch.cuda.synchronize()
        self.h_file = self.buf.cpu().pin_memory()
        self.h_grid = [self.torch.empty_like(self.h_in[c]).pin_memory() for c in range(3)]

    def step(self, stream, events=None):
        if events is not None:
            events[0].record(stream)
        self.cn.IO.AOS2Field(self.buf, self.u, stream=stream)
        if events is not None:
            events[1].record(stream)

    e2e_path = ("C ABI, device slots in turn: step i+1's upload of the file buffer from pinned host and step "
                "i-1's download of the grid (cn_grid_download to pinned host) run on their own streams while "
                "step i scatters (cn_grid_from_aos)")

    def _pinned_bytes(self, n):
        return self.buf.numel() * 4 + n * 3 * self.u.comp_stride * 8

    def _new_slot(self):
        torch = self.torch
        return dict(u=self.cn.Grid.Cartesian(self.nb, self.n, ncomp=3), buf=torch.empty_like(self.buf),
                    out=[torch.empty_like(self.h_in[c]).pin_memory() for c in range(3)])

    def _slot0(self):
        return dict(u=self.u, buf=self.buf, out=self.h_grid)

    def _upload(self, slot, s):
        with self.torch.cuda.stream(s):
            slot["buf"].copy_(self.h_file, non_blocking=True)

    def _compute(self, slot, s):
        self.cn.IO.AOS2Field(slot["buf"], slot["u"], stream=s)

    def _download(self, slot, s):
        import ctypes as C
        lib = self.cn._lib.lib()
        for c in range(3):
            self.cn._lib.check(lib.cn_grid_download(slot["u"].handle, c, C.c_void_p(slot["out"][c].data_ptr()),
                                                    self.u.comp_stride * 8, C.c_void_p(s.cuda_stream)))

    def _bytes(self):
        return self.buf.numel() * 4, 3 * self.u.comp_stride * 8

    def e2e_step(self, stream):
        import ctypes as C
        lib = self.cn._lib.lib()
        sh = C.c_void_p(stream.cuda_stream)
        with self.torch.cuda.stream(stream):
            self.buf.copy_(self.h_file, non_blocking=True)
        self.step(stream)
        nbytes = self.u.comp_stride * 8
        for c in range(3):
            self.cn._lib.check(lib.cn_grid_download(self.u.handle, c, C.c_void_p(self.h_grid[c].data_ptr()),
                                                    nbytes, sh))
        return self.buf.numel() * 4, 3 * nbytes

    @classmethod
    def cpu_sample_static(cls, threads, reps=3):
        """The reference's AOS2Field block loop (oracle/_ref) on 8x8x4 blocks
        of 32^3, or the oracle restatement without the reference build."""
        import oracle as O
        from oracle import aos as A
        nb, n = cls.cpu_blocks, cls.n
        stride = O.block_stride(n, np.float64)
        top = [nb[d] * n[d] for d in range(3)]
        cells = int(np.prod(top))
        rng = np.random.default_rng(1234)
        buf = rng.uniform(-1.0, 1.0, size=cells * 3).astype(np.float32)
        data = np.zeros((3, int(np.prod(nb)) * stride))
        if O.ref_available():
            t, _ = O.ref_field_aos(data, nb, n, 0, stride, (0, 0, 0), top, np.float32, buf, to_aos=False,
                                   threads=threads, reps=reps)
            kind = "reference"
        else:
            t0 = time.perf_counter()
            for _ in range(reps):
                A.aos_to_grid(buf, list(data), nb, n, 0, stride, (0, 0, 0), top)
            t = (time.perf_counter() - t0) / reps
            kind, threads = "port", 1
        return dict(value=cells / t / 1e9, unit="Gcell/s", cores=threads, kind=kind,
                    sample=f"AOS2Field of an FP32 AoS buffer into 3 FP64 components on {nb[0]}x{nb[1]}x{nb[2]} "
                           f"blocks of 32^3 ({cells / 1e6:.1f} M cells), best of {reps}, {threads} threads",
                    seconds_per_sweep=t)


WORKLOADS = {"c1": C1, "c2": C2, "c3": C3, "c4": C4, "c5": C5, "io": IOW, "io_read": IOR, "lab": LAB}
DEFAULT_WORKLOAD = "c2"


# ------------------------------------------------------------------- main
def run_ours(args, world, rank, local, pg):
    import torch

    from cubismnova_b200 import _lib
    torch.cuda.set_device(local)
    cls = WORKLOADS[args.workload]
    if getattr(args, "no_learned", False) and hasattr(cls, "with_learned"):
        cls = type(cls.__name__, (cls,), {"with_learned": False})
    if args.blocks:
        cls = type(cls.__name__, (cls,), {"nb": tuple(args.blocks),
                                          "desc": cls.desc + f" [reduced: {tuple(args.blocks)} blocks]"})
    if getattr(args, "mg_omega", None) is not None and hasattr(cls, "omega"):
        cls = type(cls.__name__, (cls,), {"omega": args.mg_omega})
    if getattr(args, "mg_nu", None) is not None and hasattr(cls, "nu"):
        cls = type(cls.__name__, (cls,), {"nu": tuple(args.mg_nu)})
    if getattr(args, "nn_training", None) and hasattr(cls, "nn_training"):
        cls = type(cls.__name__, (cls,), {"nn_training": args.nn_training})
    if getattr(args, "amr_schedule", None) is not None and hasattr(cls, "fixed_schedule"):
        cls = type(cls.__name__, (cls,), {"fixed_schedule": tuple(args.amr_schedule)})
    if getattr(args, "no_autotune", False) and hasattr(cls, "autotune"):
        cls = type(cls.__name__, (cls,), {"autotune": False})
    W = cls()
    stream = torch.cuda.Stream()
    peaks = measured_peaks()
    L = W.launches_per_step
    # warm-up
    for _ in range(args.warmup):
        if W.needs_flush():
            W.flush(stream)
        W.step(stream)
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(L + 1)] for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(pg)
    torch.cuda.synchronize()
    for i in range(args.steps):
        if W.needs_flush():
            W.flush(stream)
        W.step(stream, ev[i])
    torch.cuda.synchronize()
    barrier(pg)
    clocks = sampler.stop()
    launch_ms = np.array([[ev[i][k].elapsed_time(ev[i][k + 1]) for k in range(L)] for i in range(args.steps)])
    ms_local = float(launch_ms.sum())
    ms = max_over_ranks(pg, ms_local)
    ms_per_step = ms / args.steps
    metric = getattr(W, "metric", "Gcell-updates/s")
    unit = getattr(W, "unit", "Gcell-updates/s")
    value = W.updates_per_step * world * args.steps / (ms / 1e3) / 1e9
    # roofline of the dominant kernel (every launch of a step is that kernel)
    avg_launch_s = ms_local / (args.steps * L) / 1e3
    bytes_per_launch = W.bytes_per_cell_step * W.cells / L
    achieved = bytes_per_launch / avg_launch_s / 1e9
    roof = dict(bound="hbm", achieved=round(achieved, 1), peak=peaks["hbm_gbs"], unit="GB/s",
                frac=round(achieved / peaks["hbm_gbs"], 4),
                traffic=(args.traffic if args.traffic is not None else
                         int(W.traffic_per_cell_step * W.cells / L) if getattr(W, "traffic_per_cell_step", None)
                         else None),
                peak_source=peaks["src"] + " (MEASURED_PEAKS.json hbm_gbs)" if peaks["src"] == "measured"
                else "fallback 6.65 TB/s",
                algorithmic_bytes_per_launch=int(bytes_per_launch),
                algorithmic_bytes_per_cell_step=W.bytes_per_cell_step,
                launch_ms_mean=[round(float(x), 4) for x in launch_ms.mean(0)])
    if getattr(W, "roofline_scope", None):
        roof["scope"] = W.roofline_scope
    if args.traffic is None and getattr(W, "traffic_per_cell_step", None):
        roof["traffic_source"] = W.traffic_source
    flops = getattr(W, "flops_per_cell_stage", None)
    if flops:
        dt_code = _lib.CN_FLOAT64 if W.dtype == "f64" else _lib.CN_FLOAT32
        peak_tf = _lib.fma_peak_tflops(dt_code)
        ach_tf = flops * W.updates_per_step / (ms_local / args.steps / 1e3) / 1e12
        roof["alu"] = dict(bound="fp64" if W.dtype == "f64" else "fp32", achieved=round(ach_tf, 2),
                           peak=round(peak_tf, 2), unit="TFLOP/s", frac=round(ach_tf / peak_tf, 4),
                           peak_source="measured by cn_calib_fma_peak (independent FMA chains)",
                           flops_per_cell_stage=flops)
    # end to end through the C ABI with host buffers: every step uploads its
    # input from pinned host memory and downloads its result
    ek = max(3, min(args.steps // 2, 10))

    def timed_e2e(run, k):
        run(2)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(pg)
        e0.record(stream)
        hb, db = run(k)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(pg, e0.elapsed_time(e1)) / k, hb, db

    def serial(k):
        hb = db = 0
        for _ in range(k):
            hb, db = W.e2e_step(stream)
        return hb, db

    serial_ms, hb, db = timed_e2e(serial, ek)
    e2e_ms, path = serial_ms, "C ABI: cn_grid_upload from pinned host, the step, cn_grid_download to pinned host"
    W.ranks_per_node = int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
    if getattr(W, "e2e_pipelined", None) and not args.e2e_serial and W.e2e_slots() >= 2:
        # the pipeline's fill and drain (one upload, one download) are inside
        # the timed region: run as many steps as the main timed region
        e2e_ms, hb, db = timed_e2e(lambda k: W.e2e_pipelined(stream, k), max(ek, args.steps))
        path = W.e2e_path
    e2e = dict(value=round(W.updates_per_step * world / (e2e_ms / 1e3) / 1e9, 4), unit=unit,
               h2d_bytes_per_step=hb, d2h_bytes_per_step=db, ms_per_step=round(e2e_ms, 4), path=path)
    if e2e_ms != serial_ms:
        e2e["serial"] = dict(value=round(W.updates_per_step * world / (serial_ms / 1e3) / 1e9, 4),
                             ms_per_step=round(serial_ms, 4),
                             path="upload, step and download in order on one stream")
    out = dict(metric=metric, value=round(value, 4), unit=unit, n_gpus=world,
               steps=args.steps, warmup=args.warmup, ms_per_step=round(ms_per_step, 5),
               higher_is_better=True, scaling="weak", vs_baseline=None, dtype=W.dtype, data="synthetic",
               config=dict(workload=W.desc, name=W.name, cells=W.cells, updates_per_step=W.updates_per_step,
                           blocks=list(W.nb), block_cells=list(W.n), parallelism=f"replicas x{world}",
                           l2="flushed between steps (untimed 252 MB write)" if W.needs_flush()
                           else "inputs larger than L2 (no flush)"),
               roofline=roof, e2e=e2e, clocks=clocks,
               gpu_launches=int(getattr(W, "gpu_launches_per_step", L)) * args.steps)
    if getattr(W, "learned", None) is not None:
        out["config"]["learned_smoother"] = W.learned
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = W.cpu_sample(os.cpu_count() or 1)
    if world == 1 and args.workload == DEFAULT_WORKLOAD and not args.no_companions and not args.blocks:
        W = None
        import gc
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        out["companions"] = run_companions(args, local)
    return out


# The other workloads, timed briefly on the same GPU after the main one so
# that one default run measures them all (rank 0 at N = 1 only).
COMPANIONS = ("c1", "c4", "c5", "c3", "lab")


def run_companions(args, local):
    """Device-timed short runs of COMPANIONS: 3 warm-up steps, then
    args.companion_steps steps (L2 handled as in the main run); value,
    roofline fractions against the measured peaks, and each workload's own
    extras (the C5 learned-smoother table, the C3 layout and schedule)."""
    import gc

    import torch

    from cubismnova_b200 import _lib
    peaks = measured_peaks()
    res = {}
    for name in COMPANIONS:
        t0 = time.perf_counter()
        W = None
        try:
            W = WORKLOADS[name]()
            stream = torch.cuda.Stream()
            L = W.launches_per_step
            for _ in range(3):
                if W.needs_flush():
                    W.flush(stream)
                W.step(stream)
            torch.cuda.synchronize()
            k = max(1, args.companion_steps)
            ev = [[torch.cuda.Event(enable_timing=True) for _ in range(L + 1)] for _ in range(k)]
            for i in range(k):
                if W.needs_flush():
                    W.flush(stream)
                W.step(stream, ev[i])
            torch.cuda.synchronize()
            launch_ms = np.array([[ev[i][j].elapsed_time(ev[i][j + 1]) for j in range(L)] for i in range(k)])
            ms = float(launch_ms.sum())
            unit = getattr(W, "unit", "Gcell-updates/s")
            d = dict(metric=getattr(W, "metric", unit), value=round(W.updates_per_step * k / (ms / 1e3) / 1e9, 4),
                     unit=unit, dtype=W.dtype, ms_per_step=round(ms / k, 4), steps=k, warmup=3, cells=W.cells,
                     workload=W.desc)
            ach = W.bytes_per_cell_step * W.cells / L / (ms / (k * L) / 1e3) / 1e9
            d["hbm"] = dict(achieved_gbs=round(ach, 1), frac=round(ach / peaks["hbm_gbs"], 4),
                            algorithmic_bytes_per_cell_step=W.bytes_per_cell_step)
            if getattr(W, "traffic_per_cell_step", None):
                d["hbm"]["traffic_per_cell_step"] = W.traffic_per_cell_step
                d["hbm"]["traffic_source"] = W.traffic_source
            flops = getattr(W, "flops_per_cell_stage", None)
            if flops:
                peak_tf = _lib.fma_peak_tflops(_lib.CN_FLOAT64 if W.dtype == "f64" else _lib.CN_FLOAT32)
                tf = flops * W.updates_per_step / (ms / k / 1e3) / 1e12
                d["alu"] = dict(achieved_tflops=round(tf, 2), peak_tflops=round(peak_tf, 2),
                                frac=round(tf / peak_tf, 4))
            if getattr(W, "learned", None) is not None:
                d["learned_smoother"] = W.learned
            for extra in ("layout", "schedule"):
                if getattr(W, extra, None) is not None:
                    d[extra] = getattr(W, extra)
        except Exception as e:  # reported, not fatal: the main line stands
            d = dict(error=str(e)[:300])
        d["wall_seconds"] = round(time.perf_counter() - t0, 1)
        res[name] = d
        del W
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return res


def run_reference(args, world, rank):
    if rank != 0:
        return None
    W = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    # the sample of the cpu_baseline leg (same blocks), best of 3 per step
    kw = {"nb": W.cpu_nb} if hasattr(W, "cpu_nb") else {}
    for _ in range(args.warmup):
        W.cpu_sample_static(threads, reps=1, **kw)
    vals, secs = [], []
    r = None
    for _ in range(args.steps):
        r = W.cpu_sample_static(threads, reps=3, **kw)
        vals.append(r["value"])
        secs.append(r["seconds_per_sweep"])
    v = float(np.median(vals))
    unit = r["unit"]
    base = dict(value=round(v, 6), unit=unit, cores=r["cores"], kind=r["kind"], sample=r["sample"])
    return dict(impl="reference", metric=getattr(W, "metric", unit), value=round(v, 6), unit=unit,
                n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=round(1e3 * float(np.median(secs)), 4), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype=W.dtype, data="synthetic",
                config=dict(workload=W.desc, name=W.name, parallelism=f"{threads} host threads, rank 0 only"),
                cpu_baseline=base,
                e2e=dict(value=round(v, 6), unit=unit, h2d_bytes_per_step=0, d2h_bytes_per_step=0))


def accuracy_fp32(args):
    """FP32 against FP64 on the C4 geometry (1024^3 cells as 32^3 blocks of
    32^3, the C2 pulse, BCs and CFL 0.3 time step from the FP64 state), both
    on the GPU: `--acc-steps` SSP-RK3 steps each, then L1 / Linf of the
    difference per conserved variable (relative to max |state| of rho and E)
    and the drift of the FP64 integrals of mass and energy.  The two states
    and their work grids (193 GB) do not fit one GPU together, so the FP64 run
    goes first and its final state waits in host memory."""
    import torch

    import cubismnova_b200 as cn
    nb = tuple(args.blocks) if args.blocks else C4.nb
    n = C4.n
    cells = int(np.prod(n))
    steps = args.acc_steps

    def make(dtype):
        U = cn.Grid.Cartesian(nb, n, ncomp=5, dtype=dtype)
        cn.workloads.euler_pulse(U)
        torch.cuda.empty_cache()  # the pulse's FP64 temporaries
        cn.workloads.euler_bcs(U)
        U.sync_bcs()
        return U, cn.euler.like(U), cn.euler.like(U)

    def integrals(U):
        vol = float(np.prod(U.getCellSize()))
        return [float(U.tensor(c)[:, :cells].sum(dtype=torch.float64)) * vol for c in range(5)]

    out = dict(impl="accuracy", workload=f"{nb[0] * n[0]}x{nb[1] * n[1]}x{nb[2] * n[2]} cells as "
                                        f"{nb[0]}x{nb[1]}x{nb[2]} blocks of 32^3, Euler pulse, C2 BCs",
               rk3_steps=steps)
    runs = {}
    host64 = None
    dt = None
    for name, dtype in (("f64", np.float64), ("f32", np.float32)):
        U, w1, w2 = make(dtype)
        if dt is None:
            dt = cn.euler.cfl_dt(U, 0.3)
        s0 = integrals(U)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sums = None
        for i in range(steps):
            sums = cn.euler.rk3_step(U, w1, w2, dt, want_sums=(i == steps - 1))
        e1.record()
        torch.cuda.synchronize()
        runs[name] = dict(ms_per_step=round(e0.elapsed_time(e1) / steps, 3),
                          mass_drift=(sums[0] - s0[0]) / s0[0], energy_drift=(sums[4] - s0[4]) / s0[4],
                          momentum_change=[sums[c] - s0[c] for c in (1, 2, 3)])
        if name == "f64":
            host64 = [U.tensor(c)[:, :cells].cpu() for c in range(5)]
            del U, w1, w2
            torch.cuda.empty_cache()
        else:
            scale = max(float(host64[0].abs().max()), float(host64[4].abs().max()))
            err = []
            for c in range(5):
                a = host64[c].cuda()
                a.sub_(U.tensor(c)[:, :cells].double()).abs_()
                err.append(dict(var=c, L1=float(a.mean()) / scale, Linf=float(a.max()) / scale))
                del a
                torch.cuda.empty_cache()
            del U, w1, w2
    out.update(dt=dt, runs=runs, fp32_vs_fp64=err,
               note="errors relative to max(|rho|, |E|) of the FP64 state; drifts are (I_end - I_0) / I_0 "
                    "of the FP64 integrals that the stage kernels accumulate")
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-serial", action="store_true",
                    help="time the end-to-end leg with upload, step and download in order on one stream only")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu DRAM bytes per launch of the dominant kernel, if measured")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-companions", action="store_true",
                    help="skip the short runs of the other workloads that follow the default one")
    ap.add_argument("--companion-steps", type=int, default=5, help="timed steps of each companion workload")
    ap.add_argument("--no-learned", action="store_true",
                    help="c5: skip training and timing the learned smoother")
    ap.add_argument("--mg-omega", type=float, default=None, help="c5: Jacobi damping (default 6/7)")
    ap.add_argument("--mg-nu", type=int, nargs=2, default=None, help="c5: pre- and post-smoothing sweeps (default 2 2)")
    ap.add_argument("--nn-training", default=None, choices=["tensor", "fp32"],
                    help="c5: training arithmetic of the learned smoother (default tensor)")
    ap.add_argument("--amr-schedule", type=int, nargs=5, default=None, metavar=("ORDER", "CTAS", "TX", "TY", "TZ"),
                    help="c3: a fixed schedule instead of the autotuner's (order 0-2, persistent CTAs, "
                         "work tile of TX x TY x TZ 8^3 tiles, each 1/2/4)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="c3: keep the default schedule instead of autotuning it (profiling runs)")
    ap.add_argument("--blocks", type=int, nargs=3, default=None,
                    help="override the block counts (reduced grids for profiling runs)")
    ap.add_argument("--accuracy", action="store_true",
                    help="FP32 vs FP64 accuracy study on the C4 geometry (no timing line)")
    ap.add_argument("--acc-steps", type=int, default=100, help="--accuracy: SSP-RK3 steps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.accuracy:
        accuracy_fp32(args)
        return
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
