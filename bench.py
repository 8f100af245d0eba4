"""Benchmark: refactorization + FP64-refined solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mesh|nodal|batch]

One step = refactorize with a new value set of the same pattern (values placed
into the LU layout on the GPU, FP32 factorization) + FP64-refined solve of the
step's right-hand sides to the workload's residual tolerance.  ``value`` is
solves per second over all GPUs with inputs resident in HBM; ``e2e`` is the
same through the public API with host buffers (copies inside the timed
region).  ``--impl reference`` times NICSLU, the reference's own CPU solver,
on the same workload on this host's cores (rank 0 only).

Workloads (seeded synthetic matrices):
  mesh   700 x 700 resistive power grid, n = 490,000, 1 right-hand side,
         refinement to 1e-12 (default);
  nodal  nodal-analysis matrix n = 4,960, 1 right-hand side, 1e-10;
  batch  256 value sets of one n = 20,000 nodal pattern, 4 right-hand sides
         each, 1e-10.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "glu-hcu_b200"))

METRIC = "refactor ms & batched solves/s at 1e-10 FP64 residual vs plain FP32 on B200"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="mesh", choices=["mesh", "nodal", "batch", "uneven", "adjoint"])
    p.add_argument("--adjoint-n", type=int, default=100000, help="order of the differentiation workload")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="skip timing the reference's own numeric.cu (LUonDevice) on the mesh's arrays")
    p.add_argument("--reference-gpu", action="store_true", help=argparse.SUPPRESS)  # the default now
    p.add_argument("--no-batch-record", action="store_true",
                   help="skip the batched same-pattern sub-record of the mesh line")
    p.add_argument("--side", type=int, default=700, help="mesh side (workload mesh)")
    p.add_argument("--batch", type=int, default=256, help="value sets of the batch workload")
    p.add_argument("--uneven-max-n", type=int, default=50000, help="largest system of the uneven workload")
    return p.parse_args()


def workload(name, side=700, batch=256):
    from pyglu import synth

    if name == "mesh":
        A = synth.config1(side=side)
        return dict(A=A, batch=1, nrhs=1, tol=1e-12, values=2,
                    desc=f"power-grid mesh {side}x{side}, n={side * side}, 1 RHS, refine to 1e-12",
                    b=lambda n, k, s: synth.rhs_loads(n, seed=s)[None, :])
    if name == "nodal":
        A = synth.config0()
        return dict(A=A, batch=1, nrhs=1, tol=1e-10, values=2,
                    desc="nodal matrix n=4960, 1 RHS, refine to 1e-10",
                    b=lambda n, k, s: synth.rhs_uniform(n, k, seed=s))
    if name == "uneven":  # the reference arm times one system of the set (its largest)
        n, k, sd = max(synth.config3_systems(count=64, seed=0, n_range=(2000, 50000), rhs_range=(1, 64)))
        A = synth.nodal(n, seed=sd)
        return dict(A=A, batch=1, nrhs=k, tol=1e-10, values=2,
                    desc=f"largest system of the uneven batch, n={n}, {k} RHS, refine to 1e-10",
                    b=lambda n, k, s: synth.rhs_uniform(n, k, seed=s))
    A = synth.config2_pattern()
    return dict(A=A, batch=batch, nrhs=4, tol=1e-10, values=1,
                desc=f"{batch} value sets of one nodal pattern n=20000, 4 RHS each, refine to 1e-10",
                b=lambda n, k, s: synth.rhs_uniform(n, k, seed=s))


class Clocks:
    """SM clock, power and clock-event reasons of this rank's GPU, sampled
    during the timed region.

    NVML is polled every 10 ms from a thread, so a timed region of a few
    hundred milliseconds still gets a dozen readings, plus one reading at
    start and one at stop.  The device is found by the PCI bus id of the CUDA
    device, so the reading is of the GPU the kernels run on whatever device
    numbering CUDA_VISIBLE_DEVICES sets.  Without NVML the same fields come
    from ``nvidia-smi -lms 200``.  Only reads: nothing here sets a clock."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    PERIOD_S = 0.010

    def __init__(self, index):
        self.index = index
        self.rows = []          # (sm_mhz, max_mhz, watts, {reason names})
        self.proc = None
        self.nvml = None
        self.handle = None
        self.source = None
        self.halt = threading.Event()
        self.thread = None

    def _bus_id(self):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.index)
            return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            return None

    def _nvml_sample(self):
        nv, h = self.nvml, self.handle
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                          float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                          nv.nvmlDeviceGetPowerUsage(h) / 1e3,
                          {n for n, b in zip(self.NAMES, bits) if mask & b}))

    def _nvml_loop(self):
        while not self.halt.wait(self.PERIOD_S):
            try:
                self._nvml_sample()
            except Exception:
                return

    def start(self):
        bus = self._bus_id()
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nvml = nv
            try:
                self.handle = nv.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.handle = nv.nvmlDeviceGetHandleByIndex(self.index)
            self._nvml_sample()
            self.source = "nvml"
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
            self.rows = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={bus or self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            self.thread = threading.Thread(target=self._smi_read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _smi_read(self):
        def num(s):
            try:
                return float(s)
            except ValueError:
                return None
        for line in self.proc.stdout:
            r = [c.strip() for c in line.split(",")]
            if len(r) < 9:
                continue
            self.rows.append((num(r[1]), num(r[2]), num(r[3]),
                              {n for i, n in enumerate(self.NAMES) if r[5 + i] == "Active"}))

    def stop(self):
        if self.nvml is not None:
            self.halt.set()
            self.thread.join(timeout=5)
            try:
                self._nvml_sample()
            except Exception:
                pass
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)
        else:
            return None
        if not self.rows:
            return None
        sm = [r[0] for r in self.rows if r[0] is not None]
        mx = [r[1] for r in self.rows if r[1] is not None]
        w = [r[2] for r in self.rows if r[2] is not None]
        reasons = sorted(set().union(*(r[3] for r in self.rows)))
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "sm_min_mhz": min(sm) if sm else None,
                "power_w_median": float(np.median(w)) if w else None,
                "reasons": reasons, "samples": len(self.rows), "source": self.source}


def dist_setup(args):
    """One process per GPU (torchrun env); NCCL, or gloo on a host without GPUs
    (the reference arm's CPU ranks)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        # ranks meet only at the timing barriers and the max-over-ranks reduction;
        # the longest legitimate skew is setup + warm-up of the batch workload
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x, pg, device):
    """The maximum of x over all ranks (a device tensor under NCCL, a host
    tensor under gloo)."""
    if pg is None:
        return x
    import torch

    if pg.get_backend() != "nccl":
        device = "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, solves_per_rank, ms_max):
    """Solves per second of the whole job: every rank's solves over the
    slowest rank's time per step."""
    return world * solves_per_rank / (ms_max / 1e3)


def cpu_reference(W, steps, warmup, sample_only=False):
    """NICSLU (reference CPU code) refactor + solve + refine on this host."""
    import oracle
    from pyglu import synth

    data, indices, indptr, n = W["A"]
    threads = os.cpu_count() or 1
    vals = synth.perturb_values(data, indices, indptr, n, count=2, seed=7)
    b = W["b"](n, W["nrhs"], 11)
    nl = oracle.RefNicsLU(data, indices, indptr, n, threads)
    per_step_solves = W["nrhs"] if sample_only or W["batch"] == 1 else W["nrhs"]

    x_check = {}

    def step(i):
        nl.refactor(vals[i % 2])
        for k in range(W["nrhs"]):
            x = nl.solve(b[k])
            nl.refine(x, b[k], W["tol"], 10)
            if i % 2 == 0 and k == 0:
                x_check["x"] = np.array(x, dtype=np.float64, copy=True)

    for i in range(warmup):
        step(i)
    t0 = time.perf_counter()
    for i in range(steps):
        step(i)
    dt = (time.perf_counter() - t0) / steps
    sample = (f"{steps} step(s) of NICSLU ReFactorize_MT + Solve + Refine on one value set "
              f"({per_step_solves} RHS) of the workload matrix")
    if not x_check:  # the timed steps factored value set 1 only
        nl.refactor(vals[0])
        x = nl.solve(b[0])
        nl.refine(x, b[0], W["tol"], 10)
        x_check["x"] = np.array(x, dtype=np.float64, copy=True)
    return per_step_solves / dt, dt, threads, sample, x_check["x"]


def run_uneven(args, world, rank, local, pg):
    """Uneven batch: 64 independent nodal systems of different sizes (n
    log-uniform in [2,000, 50,000]), each with 1-64 right-hand sides,
    refactored and FP64-refined together (UnevenBatch: every system's kernels
    on one of 16 streams from one host thread, one host wait per
    factorization round and per refinement step; host buffers)."""
    import torch

    import pyglu
    from pyglu import synth

    torch.cuda.set_device(local)
    specs = synth.config3_systems(count=64, seed=0, n_range=(2000, args.uneven_max_n), rhs_range=(1, 64))
    systems = [synth.nodal(n, seed=sd) for n, k, sd in specs]
    bs = [synth.rhs_uniform(n, k, seed=sd).T.copy() for n, k, sd in specs]
    vals = [synth.perturb_values(*A, count=2, seed=7) for A in systems]
    t_setup = time.perf_counter()
    ub = pyglu.UnevenBatch(systems, streams=16, workers=16, device=local)
    t_setup = time.perf_counter() - t_setup
    solves = sum(k for _, k, _ in specs)

    def step(i):
        ub.refactor([v[i % 2] for v in vals])
        return ub.solve(bs, tol=1e-10)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        xs = step(i)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    if pg:
        pg.barrier()
    ms = max_over_ranks(ms, pg, torch.device("cuda", local))
    res = max(st["residual"] for st in ub.last_refine)
    h2d = sum(v[0].nbytes for v in vals) + sum(b.nbytes for b in bs)
    d2h = sum(x.nbytes for x in xs)
    value = whole_job_value(world, solves, ms)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"64 nodal systems, n log-uniform in [2,000, {args.uneven_max_n:,}], "
                                   "1-64 RHS each, refine to 1e-10",
                       "systems": len(specs), "rhs_total": solves, "n_total": sum(n for n, _, _ in specs),
                       "nnz_lu_total": int(sum(lu.analysis.nnz_lu for lu in ub.lus)),
                       "setup_s": t_setup, "parallelism": f"16 streams x{world}"},
            "residual": res, "refine_dtype": "f64",
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "note": "the uneven batch is driven through host buffers; value is already end to end"},
            "roofline": None, "gpu_launches": None, "clocks": None}
    if rank == 0:
        print(json.dumps(line))


def run_adjoint(args, local):
    """The differentiation workload: the nodal generator with band 24 and 5%
    unsymmetric rows at n = args.adjoint_n, loss = w.x with w standard normal,
    FP32 factor + FP64-refined solve forward, the hand-written adjoint
    (transposed refined solves, -lambda_i x_j on A's pattern) backward.
    Checked against FP64 central differences (relative step 1e-6) on 64
    random nonzeros and 64 random entries of b, each quotient evaluated
    through an identity that needs no subtraction of the two function values
    (refactorizations at the perturbed values and refined solves), and, at
    n = 2,000, against the gradient of a dense torch.linalg.solve of the same
    system."""
    import scipy.sparse as sp
    import torch

    import pyglu
    from pyglu import synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    out = {"metric": "adjoint gradient max relative error vs FP64 central differences", "unit": "relative",
           "higher_is_better": False, "data": "synthetic", "dtype": "f32 factor, f64 refinement",
           "n_gpus": 1, "config": {"workload": f"nodal generator n={args.adjoint_n:,}, band 24, "
                                               "5% unsymmetric rows, loss w.x"}}
    t0 = time.perf_counter()
    A = synth.config4(n=args.adjoint_n, seed=0)
    data, indices, indptr, n = A
    lu = pyglu.GLUFactorization(*A, device=local)
    out["config"].update(nnz_lu=int(lu.analysis.nnz_lu), dense_tail=int(lu.stats["dense_tail"]),
                         setup_s=time.perf_counter() - t0)
    rng = np.random.default_rng(1)
    w = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device=dev)
    vals = torch.tensor(data, dtype=torch.float64, device=dev, requires_grad=True)
    b = torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, device=dev, requires_grad=True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    x = pyglu.sparse_solve(vals, b, lu, tol=1e-15, maxiter=40)
    loss = (w * x).sum()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    loss.backward()
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    out.update(forward_ms=(t2 - t1) * 1e3, backward_ms=(t3 - t2) * 1e3)
    gv, gb = vals.grad.cpu().numpy(), b.grad.cpu().numpy()
    wn, bn, f0 = w.cpu().numpy(), b.detach().cpu().numpy(), abs(float(loss.detach()))

    # central quotients at relative step 1e-6, evaluated without subtracting
    # the two function values (they agree to more digits than FP64 holds):
    # nonzero q = (i, j): (f(+) - f(-)) / 2h == -x(-)_j lambda(+)_i exactly;
    # entry i of b: f is linear in b, the quotient is w . A^-1 e_i exactly
    # FP64 refinement stalls near 1e-15 on this system: a few steps past 1e-14
    # change nothing measurable
    kw = dict(refine=True, tol=1e-14, maxiter=10)
    cols = np.repeat(np.arange(n), np.diff(indptr))
    rs = np.random.default_rng(2)
    errs_v, iters = [], []
    t4 = time.perf_counter()
    for q in rs.choice(len(data), 64, replace=False):
        i, j = indices[q], cols[q]
        h = 1e-6 * abs(data[q])
        vp, vm = data.copy(), data.copy()
        vp[q] += h
        vm[q] -= h
        lam_p = lu.refactor(vp).solve(wn, trans="T", **kw)
        iters.append(lu.last_refine["iterations"])
        x_m = lu.refactor(vm).solve(bn, **kw)
        iters.append(lu.last_refine["iterations"])
        fd = -x_m[j] * lam_p[i]
        errs_v.append(abs(fd - gv[q]) / abs(fd))
    lu.refactor(data)
    idx = rs.choice(n, 64, replace=False)
    E = np.zeros((n, 64))
    E[idx, np.arange(64)] = 1.0
    fd_b = wn @ lu.solve(E, **kw)
    errs_b = list(np.abs(fd_b - gb[idx]) / np.abs(fd_b))
    out["fd_s"] = time.perf_counter() - t4
    out["value"] = float(max(errs_v + errs_b))
    out["fd"] = {"nonzeros": {"checked": len(errs_v), "max_rel": float(max(errs_v)),
                              "median_rel": float(np.median(errs_v)), "refine_iterations_max": int(max(iters)),
                              "refine_iterations_median": float(np.median(iters))},
                 "b": {"checked": len(errs_b), "max_rel": float(max(errs_b)), "median_rel": float(np.median(errs_b))},
                 "sample": "64 random nonzeros, 64 random entries of b",
                 "step": "1e-6 relative", "bar": 1e-6,
                 "evaluation": "nonzero (i, j): -x(v - h)_j lambda(v + h)_i; b entry i: w . A^-1 e_i "
                               "(both equal the central quotient exactly)"}
    # dense gradient at n = 2,000
    A2 = synth.config4(n=2000, seed=1)
    d2, i2, p2, n2 = A2
    lu2 = pyglu.GLUFactorization(*A2, device=local)
    w2 = torch.tensor(rng.standard_normal(n2), dtype=torch.float64, device=dev)
    v2 = torch.tensor(d2, dtype=torch.float64, device=dev, requires_grad=True)
    b2 = torch.tensor(rng.uniform(-1, 1, n2), dtype=torch.float64, device=dev, requires_grad=True)
    (w2 * pyglu.sparse_solve(v2, b2, lu2, tol=1e-15, maxiter=40)).sum().backward()
    M = torch.tensor(sp.csc_matrix((d2, i2, p2), shape=(n2, n2)).toarray(), dtype=torch.float64, requires_grad=True)
    bb = b2.detach().cpu().clone().requires_grad_(True)
    (w2.cpu() * torch.linalg.solve(M, bb)).sum().backward()
    cols = np.repeat(np.arange(n2), np.diff(p2))
    gd = M.grad.numpy()[i2, cols]
    gv2 = v2.grad.cpu().numpy()
    big = np.abs(gd) > 1e-9 * np.abs(gd).max()
    out["dense_n2000"] = {"values_max_rel": float((np.abs(gv2 - gd)[big] / np.abs(gd)[big]).max()),
                          "b_max_rel": float((np.abs(b2.grad.cpu().numpy() - bb.grad.numpy()) /
                                              np.maximum(np.abs(bb.grad.numpy()), 1e-300)).max())}
    out["wall_s"] = time.perf_counter() - t0
    print(json.dumps(out))


def plain_form(W, vals, local, nrhs, tensor_cores=False):
    """The plain unbatched, unrefined FP32 form on the batch's pattern: one
    value set factored alone, then one FP32 solve of its right-hand sides,
    device-resident, timed per matrix.  Without ``tensor_cores`` every update
    is FP32 FMA (the reference's arithmetic); with it the dense tail updates
    on the tensor cores as in the batched form."""
    import torch

    import pyglu
    from pyglu import _capi

    data, indices, indptr, n = W["A"]
    lu = pyglu.GLUFactorization(vals[0], indices, indptr, n, device=local)
    eng = _capi.engine()
    tu = _capi.Tuning()
    _capi.check(eng.glu_get_tuning(lu.handle, _capi.C.byref(tu)))
    if not tensor_cores:
        tu.dense_tc_min = 0
        _capi.check(eng.glu_set_tuning(lu.handle, _capi.C.byref(tu)))
    dev = torch.device("cuda", local)
    d = [torch.tensor(vals[i], dtype=torch.float64, device=dev) for i in range(2)]
    b = torch.tensor(W["b"](n, nrhs, 11), dtype=torch.float32, device=dev)
    x = torch.empty_like(b)
    ts = []
    for i in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lu.refactor_device(d[i % 2])
        lu.solve_device(b, x, refine=False)
        e1.record()
        torch.cuda.synchronize()
        if i >= 2:
            ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    form = ("one value set: FP32 refactor + FP32 solve of its right-hand sides, no refinement, "
            + ("dense tail on the tensor cores (three-part BF16 split, FP32 accuracy)" if tensor_cores else "all updates FP32 FMA"))
    return {"value": nrhs / (ms / 1e3), "unit": "solves/s", "ms_per_matrix": ms, "form": form}


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    if args.workload == "adjoint":
        if rank == 0 and args.impl == "ours":
            run_adjoint(args, local)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no differentiation"}))
        if pg:
            pg.destroy_process_group()
        return
    if args.workload == "uneven" and args.impl == "ours":
        run_uneven(args, world, rank, local, pg)
        if pg:
            pg.destroy_process_group()
        return
    W = workload(args.workload, args.side, args.batch)
    if args.impl == "reference":
        if rank != 0:  # rank 0 alone times the reference; no collective follows
            if pg:
                pg.destroy_process_group()
            return
        v, dt, thr, sample, _ = cpu_reference(W, args.steps, args.warmup)
        line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": W["desc"], "solver": "NICSLU (reference CPU code)"},
                "cpu_baseline": {"value": v, "unit": "solves/s", "cores": thr, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        if pg:
            pg.destroy_process_group()
        return

    line = run_ours(args, W, world, rank, local, pg, args.steps, args.warmup, full=True)
    if rank == 0 and world == 1 and args.workload == "mesh" and not args.no_batch_record:
        line["batch"] = batch_record(args, world, rank, local, pg)
    if rank == 0:
        print(json.dumps(line))
    if pg:
        pg.destroy_process_group()


def batch_record(args, world, rank, local, pg, steps=2, warmup=3):
    """The batched same-pattern workload (256 value sets of one n = 20,000
    pattern, 4 right-hand sides each) at a couple of steps, with the plain
    per-matrix FP32 form beside it, as a sub-record of the default line."""
    import gc

    import torch

    gc.collect()
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    try:
        b = run_ours(args, workload("batch"), world, rank, local, pg, steps, warmup, full=False)
    except Exception as e:  # pragma: no cover
        return {"error": str(e)}
    keep = ("value", "unit", "ms_per_step", "refactor_ms", "solve_refined_ms", "residual", "residual_inf",
            "refine_iterations", "plain_form", "plain_form_tc", "factor_roofline", "roofline", "gpu_launches")
    out = {k: b[k] for k in keep if k in b}
    out.update(steps=steps, warmup=warmup, workload=b["config"]["workload"], config=b["config"],
               wall_s=time.perf_counter() - t0)
    gc.collect()
    torch.cuda.empty_cache()
    return out


def run_ours(args, W, world, rank, local, pg, nsteps, nwarmup, full=True):
    """One workload through our engine: the timed steps (device-resident
    inputs), then -- with ``full`` -- the end-to-end pass through the public
    API, the CPU baseline and the reference's numeric.cu.  Returns the JSON
    line as a dict."""
    import torch

    import pyglu
    from pyglu import _capi, synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    data, indices, indptr, n = W["A"]
    B, nrhs = W["batch"], W["nrhs"]
    nvals = max(W["values"], 1)
    vals = synth.perturb_values(data, indices, indptr, n, count=max(B, 2), seed=7)
    if B == 1:
        lu = pyglu.GLUFactorization(vals[0], indices, indptr, n, device=local)
        handle = lu.handle
    else:
        lu = pyglu.BatchedGLU(indices, indptr, n, vals[:B], device=local)
        handle = lu.handle
    an = lu._an
    eng = _capi.engine()
    stream = torch.cuda.current_stream(dev)
    sp_ = _capi.C.c_void_p(stream.cuda_stream)
    # device-resident inputs: value sets and right-hand sides
    if B == 1:
        d_vals = [torch.tensor(vals[i], dtype=torch.float64, device=dev) for i in range(nvals)]
    else:
        d_vals = [torch.tensor(vals[:B], dtype=torch.float64, device=dev)]
    b_host = np.ascontiguousarray(np.broadcast_to(W["b"](n, nrhs, 11), (B, nrhs, n)))
    d_b = torch.tensor(b_host, dtype=torch.float64, device=dev)
    d_x = torch.empty_like(d_b)
    rst = _capi.RefineStats()
    st = _capi.Stats()

    def step(i):
        v = d_vals[i % len(d_vals)]
        _capi.check(eng.glu_load_source_values(handle, 0, B, _capi.C.c_void_p(v.data_ptr()), _capi.GLU_DEVICE, sp_))
        _capi.check(eng.glu_factor(handle, 0, B, 0, sp_), "factor")
        s = eng.glu_solve_refined(handle, 0, B, nrhs, _capi.C.c_void_p(d_b.data_ptr()),
                                  _capi.C.c_void_p(d_x.data_ptr()), W["tol"], 10, 0, _capi.GLU_DEVICE,
                                  _capi.C.byref(rst), sp_)
        if s not in (0, _capi.GLU_ERR_NOT_CONVERGED):
            _capi.check(s, "refined solve")

    for i in range(nwarmup):
        step(i)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fact_ms = []
    launches = 0
    ev0.record(stream)
    for i in range(nsteps):
        step(i)
        eng.glu_get_stats(handle, _capi.C.byref(st))
        fact_ms.append(st.last_factor_ms)
        # this library's kernels of the step: value placement, factorization, refined solve
        launches += 1 + int(st.factor_launches) + int(st.solve_launches)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if pg:
        pg.barrier()
    ms = ev0.elapsed_time(ev1) / nsteps
    ms = max_over_ranks(ms, pg, dev)
    solves = B * nrhs
    value = whole_job_value(world, solves, ms)
    residual = rst.residual
    iters = rst.iterations

    # plain FP32 form: factor + unrefined solve per matrix (for the comparison)
    eng.glu_get_stats(handle, _capi.C.byref(st))
    factor_ms = float(np.median(fact_ms))
    # solve-only time (refined), device events
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s = eng.glu_solve_refined(handle, 0, B, nrhs, _capi.C.c_void_p(d_b.data_ptr()), _capi.C.c_void_p(d_x.data_ptr()),
                              W["tol"], 10, 0, _capi.GLU_DEVICE, _capi.C.byref(rst), sp_)
    e1.record(stream)
    torch.cuda.synchronize()
    solve_ms = e0.elapsed_time(e1)

    # refined solution of value set 0, RHS 0, for the forward-error check
    x_check = None
    if B == 1:
        _capi.check(eng.glu_load_source_values(handle, 0, 1, _capi.C.c_void_p(d_vals[0].data_ptr()), _capi.GLU_DEVICE, sp_))
        _capi.check(eng.glu_factor(handle, 0, 1, 0, sp_), "factor")
        s = eng.glu_solve_refined(handle, 0, 1, nrhs, _capi.C.c_void_p(d_b.data_ptr()), _capi.C.c_void_p(d_x.data_ptr()),
                                  W["tol"], 10, 0, _capi.GLU_DEVICE, _capi.C.byref(rst), sp_)
        torch.cuda.synchronize()
        x_check = d_x[0, 0].double().cpu().numpy().copy()

    # e2e through the public API with host buffers
    e2e_steps = max(1, min(nsteps, 5))
    if not full:
        e2e_ms, h2d, d2h = None, 0, 0
    elif B == 1:
        # one untimed pass: first-call allocations of the host-buffer path
        lu.refactor(vals[0])
        lu.solve(b_host[0].T if nrhs > 1 else b_host[0, 0], refine=True, tol=W["tol"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        for i in range(e2e_steps):
            lu.refactor(vals[i % nvals])
            x = lu.solve(b_host[0].T if nrhs > 1 else b_host[0, 0], refine=True, tol=W["tol"])
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3) / e2e_steps
        h2d = vals[0].nbytes + b_host[0].nbytes
        d2h = b_host[0].nbytes
    else:
        lu.refactor(vals[:B])
        lu.solve(b_host, tol=W["tol"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(e2e_steps):
            lu.refactor(vals[:B])
            X = lu.solve(b_host, tol=W["tol"])
        torch.cuda.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
        h2d = vals[:B].nbytes + b_host.nbytes
        d2h = b_host.nbytes
    e2e_value = None
    if e2e_ms is not None:
        e2e_ms = max_over_ranks(e2e_ms, pg, dev)
        e2e_value = whole_job_value(world, solves, e2e_ms)

    # roofline of the factorization (all its kernels, one launch sequence)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    nnz_lu = an.nnz_lu
    flops = st.factor_flops * B
    # dominant kernel, timed live: one more factorization with CUDA events
    # around every launch on the factor stream
    _capi.check(eng.glu_profile_enable(handle, 1))
    _capi.check(eng.glu_load_source_values(handle, 0, B, _capi.C.c_void_p(d_vals[0].data_ptr()), _capi.GLU_DEVICE, sp_))
    _capi.check(eng.glu_factor(handle, 0, B, 0, sp_), "factor")
    torch.cuda.synchronize()
    kt = _capi.kernel_times(handle)
    _capi.check(eng.glu_profile_enable(handle, 0))
    dom = max(kt, key=lambda k: kt[k][0])
    dom_ms, dom_n = kt[dom]
    pat = an.pattern()
    cp, dg = pat["sym_c_ptr"].astype(np.int64), pat["l_col_ptr"].astype(np.int64)
    rp, rd = pat["csr_r_ptr"].astype(np.int64), pat["csr_diag_ptr"].astype(np.int64)
    m_t = int(st.dense_tail)
    t_s = n - m_t
    Lk, Uk = cp[1:] - dg - 1, rp[1:] - rd - 1
    steps_k0 = np.arange(0, m_t, 64)
    mp = np.maximum(m_t - steps_k0 - 64, 0).astype(np.float64)
    if dom in ("k_factor_level", "k_factor_chain", "k_scale_level"):
        # one FP32 read-modify-write of the target per update, L(:,k) read per target
        upd = float((Lk[:t_s] * Uk[:t_s]).sum())
        dom_bytes = 8.0 * upd * B
        dom_flops = 2.0 * upd * B
    elif dom in ("k_dense_update", "k_dense_update_tc"):
        # C read and written once per launch, the panels' L21 / U12 read once
        # (the launches the engine made, summed over the value sets)
        dom_bytes = float(st.dense_update_bytes)
        dom_flops = float(st.dense_update_flops)
    elif dom == "k_sn_update":
        # L21 and U12 read once, every m x nt output read and written, positions read
        dom_bytes = float(st.sn_update_bytes) * B
        dom_flops = float(st.sn_update_flops) * B
    elif dom in ("k_sn_panel", "k_sn_diag"):
        dom_bytes = float(st.sn_panel_bytes) * B
        dom_flops = 0.0
    else:  # panel: diagonal block + L21 rows + U12 columns read and written
        dom_bytes = float((8.0 * (64 * 64 + 2 * 64 * mp)).sum()) * B
        dom_flops = float((2.0 * 64 * 64 * mp).sum()) * B
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    # DRAM traffic per launch: ncu's dram__bytes_read.sum + dram__bytes_write.sum
    # over all k_sn_update launches of a factorization of the 300x300 mesh was
    # 2.79x their algorithmic bytes (reads; the writes reach DRAM from L2 after
    # the launches and are not attributed to them); the full-size launch is
    # scaled by that
    traffic = None
    traffic_note = None
    if dom == "k_sn_update" and dom_n:
        traffic = 2.79 * dom_bytes / dom_n
        traffic_note = "ncu dram bytes (read+write) of k_sn_update on the 300x300 mesh, scaled by algorithmic bytes"
    sn_alg = {"sn_update_algorithmic_bytes": float(st.sn_update_bytes) * B,
              "sn_update_flops": float(st.sn_update_flops) * B}
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    peak_c = _capi.C.c_double(0.0)
    fp32_meas = fp32_peak
    if eng.glu_measure_fp32_peak(local, _capi.C.byref(peak_c)) == 0 and peak_c.value > 0:
        fp32_meas = peak_c.value
    # whole-refactorization roofline, both bounds: HBM with 16 B per LU entry
    # ((8 B + 8) per entry for a batch of B) and FP32 with sum |L_k| + 2|L_k||U_k|
    fac_bytes = (16.0 * nnz_lu) if B == 1 else (8.0 * B + 8.0) * nnz_lu
    fac_gbs = fac_bytes / (factor_ms / 1e3) / 1e9
    fac_tf = flops / (factor_ms / 1e3) / 1e12
    factor_roof = {"hbm": {"algorithmic_bytes": fac_bytes, "achieved_gbs": fac_gbs, "peak_gbs": hbm,
                           "frac": fac_gbs / hbm},
                   "fp32": {"flops": flops, "achieved_tflops": fac_tf, "peak_tflops": fp32_meas,
                            "peak_source": "measured FFMA microbenchmark (glu_measure_fp32_peak)",
                            "frac": fac_tf / fp32_meas},
                   "binding": "fp32" if fac_tf / fp32_meas >= fac_gbs / hbm else "hbm",
                   "levels": int(st.num_lev), "supernode_levels": int(st.sn_levels),
                   "levels_per_s": st.num_lev / (factor_ms / 1e3)}
    # refined solve: each FP32 solve reads the factors once (8 B per LU entry)
    # plus 16 B per unknown per RHS, each residual 12 B per A entry per RHS
    nnz_a = len(data)
    nsolves = iters + 1
    sol_bytes = B * (nsolves * (8.0 * nnz_lu + 16.0 * n * nrhs) + iters * 12.0 * nnz_a * nrhs)
    solve_roof = {"algorithmic_bytes": sol_bytes, "achieved_gbs": sol_bytes / (solve_ms / 1e3) / 1e9,
                  "frac": sol_bytes / (solve_ms / 1e3) / 1e9 / hbm, "fp32_solves": nsolves, "residuals": iters}
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": traffic, "traffic_source": traffic_note, "kernel": dom, "launches": dom_n,
            "kernel_ms": dom_ms, **sn_alg,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "algorithmic_bytes": dom_bytes,
            "fp32_tflops": dom_flops / (dom_ms / 1e3) / 1e12 if dom_ms > 0 else 0.0,
            "fp32_peak_tflops_derived": fp32_peak,
            "fp32_frac_of_derived": (dom_flops / (dom_ms / 1e3) / 1e12) / fp32_peak if dom_ms > 0 else 0.0,
            "factor_breakdown_ms": {k: round(v[0], 4) for k, v in kt.items() if v[1]},
            "factor_fp32_tflops": flops / (factor_ms / 1e3) / 1e12}

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": nsteps,
            "warmup": nwarmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": W["desc"], "n": n, "nnz_lu": nnz_lu, "batch": B, "nrhs": nrhs,
                       "levels": st.num_lev, "dense_tail": st.dense_tail, "supernodes": st.supernodes,
                       "supernode_levels": st.sn_levels, "deferred_coupling_columns": st.couple_columns,
                       "l2": "inputs larger than L2",
                       "parallelism": f"replicas x{world}" if B == 1 else f"batch x{world}"},
            "refactor_ms": factor_ms, "solve_refined_ms": solve_ms, "residual": residual,
            "refine_iterations": iters, "refine_dtype": "f64",
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": roof, "factor_roofline": factor_roof, "solve_roofline": solve_roof,
            "residual_inf": rst.residual_inf,
            "gpu_launches": launches, "clocks": clk}
    if B > 1:
        line["plain_form"] = plain_form(W, vals, local, nrhs)
        line["plain_form"]["batched_over_plain"] = value / line["plain_form"]["value"]
        line["plain_form_tc"] = plain_form(W, vals, local, nrhs, tensor_cores=True)
        line["plain_form_tc"]["batched_over_plain"] = value / line["plain_form_tc"]["value"]
    if full and rank == 0 and world == 1 and B == 1 and not args.no_reference_gpu:
        line["reference_numeric_cu"] = reference_numeric_cu(an, lu, vals[0], n, factor_ms)
    if full and rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle

            if oracle.ref_available():
                v, dt, thr, sample, x_ref = cpu_reference(W, 1, 0, sample_only=True)
                line["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": thr, "kind": "reference",
                                        "sample": sample}
                if B == 1 and x_check is not None:
                    # forward error of the GPU's refined solution against NICSLU's
                    # FP64 refined solution of the same system (value set 0, RHS 0)
                    dx = x_check - x_ref
                    line["forward_error"] = {
                        "vs": "NICSLU FP64 factor + refinement on the host",
                        "rel_2": float(np.linalg.norm(dx) / np.linalg.norm(x_ref)),
                        "rel_inf": float(np.abs(dx).max() / np.abs(x_ref).max())}
        except Exception as e:  # pragma: no cover
            line["cpu_baseline"] = {"error": str(e)}
    return line


def reference_numeric_cu(an, lu, val0, n, ours_refactor_ms):
    """The reference's own numeric.cu (LUonDevice, built for sm_100a from the
    reference tree) on the same arrays and values: its "Total GPU time"
    (allocations, copies in and out, factorization: numeric.cu:431-625), the
    span of the same allocations and copies alone, and their difference, the
    factorization alone."""
    try:
        import oracle

        if not oracle.ref_gpu_available():
            return {"unavailable": "oracle/_ref/libglu_ref_gpu.so not built"}
        p = an.pattern()
        lp, li = lu.levels()
        placed = np.zeros(an.nnz_lu, np.float32)
        placed[an.src_slot] = (val0 * an.src_scale).astype(np.float32)
        # keep its n-long scratch columns below 2^32 elements (numeric.cu:44,82,99)
        keep = 0
        if n * 8000 > (1 << 31):
            keep = (4 << 30) + 12 * an.nnz_lu + (64 << 20) + 8000 * 4 * n
        t0 = time.perf_counter()
        copy = []
        ref_val, total = oracle.ref_luondevice(p, placed, lp, li, keep_free_bytes=keep, copy_span=copy)
        wall = (time.perf_counter() - t0) * 1e3
        ours = lu.lu_values()
        cp = p["sym_c_ptr"].astype(np.int64)
        d = np.abs(ours.astype(np.float64) - ref_val)
        starts = cp[:-1][np.diff(cp) > 0]
        rel = np.maximum.reduceat(d, starts) / np.maximum(np.maximum.reduceat(np.abs(ref_val.astype(np.float64)),
                                                                              starts), 1e-300)
        factor_only = total - copy[0]
        return {"total_gpu_ms": total, "copy_span_ms": copy[0], "factor_only_ms": factor_only,
                "includes": "total: its allocations, copies in and out and the factorization (numeric.cu:431-625); "
                            "factor_only: total minus the same allocations and copies timed alone",
                "wall_ms": wall, "ballast_free_bytes": keep, "ours_refactor_ms": ours_refactor_ms,
                "speedup_vs_factor_only": factor_only / ours_refactor_ms,
                "speedup_vs_total": total / ours_refactor_ms,
                "factor_col_max_rel_vs_ours": float(rel.max()),
                "note": "ours: the value set of the last profiled factorization is value set 0 of the workload"}
    except Exception as e:  # pragma: no cover
        return {"error": str(e)}


if __name__ == "__main__":
    main()
