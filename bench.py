"""Benchmark: node-steps/s of the explicit meshfree step on the 1M-node Taylor bar.

Workload: copper Taylor bar D = 6.4 mm, L = 32.4 mm on a 0.1 mm jittered
lattice (1,042,925 nodes), linear-basis RKPM, cubic B-spline box support
2.0 h, direct nodal integration, J2 with linear hardening, v0 = 227 m/s
into a rigid wall, fixed CFL-0.5 step.  A "step" is one explicit step of
the whole bar (force, return mapping, central-difference update).  The
inputs (shape-function stacks, ~4 GB) are far larger than L2 (126 MB), so
no L2 flush is needed between steps.

`value` = node-steps/s of the mixed-precision path (the headline form),
`fp64_value` the plain FP64 drop-in; both device-timed with CUDA events on
the library's stream.  `e2e` drives the same job through the public C ABI
from host buffers: model upload, step-0 search and shapes, K steps with the
per-step scalars MAIN writes (energies, reaction force) read back to the
host every step, and the end-state download, all inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: replicas only (one independent bar per rank), weak scaling.
"""
import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-steps/s, 1M-node Taylor bar: mixed+learned vs plain FP64 at <=1e-3 err"
UNIT = "node-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--h", type=float, default=0.1e-3, help="lattice spacing (m)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=0, help="CPU baseline sample steps (0 = auto)")
    ap.add_argument("--modes", default="fp64,mixed", help="order in which the precision modes run")
    ap.add_argument("--full-steps", type=int, default=2000,
                    help="steps of the accuracy runs (FP64 vs mixed end states); 0 skips them")
    ap.add_argument("--rate-h", type=float, default=0.08e-3,
                    help="lattice spacing of the rate-dependent bar of the learned-start runs; 0 skips them")
    ap.add_argument("--rate-steps", type=int, default=2000, help="steps of the rate-dependent runs")
    return ap.parse_args()


def dist_setup(n):
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return rank, world, dist
    return rank, world, None


def max_over_ranks(v, dist):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


class Clocks:
    """SM clock and throttle reasons sampled during the timed region: NVML
    from a background thread every 2 ms (the region can be tens of ms)."""
    HW_SLOW, SW_POWER, HW_THERMAL, SW_THERMAL = 0x8, 0x4, 0x40, 0x20

    def __init__(self):
        import threading
        self.samples, self.reasons, self.smax = [], 0, None
        self.stop_evt = threading.Event()
        self.t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(int(os.environ.get("LOCAL_RANK", 0)))
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        while not self.stop_evt.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                self.reasons |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        import threading
        if self.nv is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()

    def stop(self):
        if self.t is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["unsampled"], samples=0)
        self.stop_evt.set()
        self.t.join()
        names = []
        for bit, nm in ((self.HW_SLOW, "hw_slowdown"), (self.HW_THERMAL, "hw_thermal_slowdown"),
                        (self.SW_THERMAL, "sw_thermal_slowdown"), (self.SW_POWER, "sw_power_cap")):
            if self.reasons & bit:
                names.append(nm)
        return dict(sm_mhz=statistics.median(self.samples) if self.samples else None, sm_max_mhz=self.smax,
                    reasons=names, samples=len(self.samples))


def measured_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kernel_bytes(n, nnz, mixed):
    """Algorithmic bytes per launch of each per-step kernel (every array
    touched once; neighbour data counted once per owning node)."""
    g = 12 if mixed else 24          # three gradient components per CSR entry
    t = 36 if mixed else 72          # T_i (3x3) per node
    defgrad = nnz * (4 + g) + n * (8 + 48 + 24 + 144)           # col + grad; rowptr, u and du, sum grad, F/G0 out
    stress = n * (144 + 192 + 16 + 8 + 8 + 8 + 2 + t)           # F/G0, sigma+eps rw, eps_p rw, eq, wvel, vol, mat, T
    force = nnz * (4 + g) + n * (8 + t + 3 + 24 + 24 + 48 + 48 + 24 + 48 + 48 + 24)  # trow + grad^T; T, fixity,
    return dict(defgrad=defgrad, stress=stress, force=force)     # mass, fint, fext rw, vel rw, acl, dsp rw, tot rw, pr


def survey_step_bytes(k, mixed):
    """Whole-step algorithmic bytes per node-step: 36k + 600 (FP64), 20k + 484 (mixed)."""
    return (20 * k + 484) if mixed else (36 * k + 600)


def run_ours(args, rank, world, dist):
    import taylor_b200
    from taylor_b200 import _lib, cases, mega
    case = cases.taylor_bar(h=args.h, seed=1 + rank)
    n = case["n"]
    p = _lib.params(**cases.param_kwargs(case))
    m = mega.Mega(case, p)
    t0 = time.perf_counter()
    info = m.search_and_shapes(download=False)
    step0_s = time.perf_counter() - t0
    nnz = info["nnz"]
    kmean = nnz / n
    # the CFL step from the neighbour lists (host-side, once)
    nb = m.search_and_shapes(download=True)
    dt = cases.stable_dt(case, nb["gn"], nb["gstart"], nb["gstack"])
    del nb
    res = {}
    for mode in args.modes.split(","):
        m.step(args.warmup, dt, mode=mode)
        barrier(dist)
        clk = Clocks()
        clk.start()
        l0 = m.kernel_launches()
        ms = m.step_timed(args.steps, dt, mode=mode)
        launches = m.kernel_launches() - l0
        clocks = clk.stop()
        ms = max_over_ranks(ms, dist)
        kt = m.kernel_times(max(3, args.steps // 2), dt, mode=mode)
        res[mode] = dict(ms=ms, clocks=clocks, launches=launches, kt=[float(x) for x in kt])
    s = m.scalars()
    dev_bytes = m.device_bytes()
    m.close()

    # end to end through the public API from host buffers
    barrier(dist)
    t0 = time.perf_counter()
    e = mega.Mega(case, p)
    e.search_and_shapes()
    d2h = 0
    for _ in range(args.steps):
        e.step(1, dt, mode="mixed")
        sc = e.scalars()           # ENERGY_INFO.OUT / TOTAL_FORCE.OUT / TIME.OUT of MAIN, every step
        d2h += 8 * 12
    xend = e.download(_lib.F_COO_CURRENT)
    epend = e.download(_lib.F_EPS)
    d2h += xend.nbytes + epend.nbytes
    e.close()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    h2d = sum(np.asarray(case[k]).nbytes for k in ("coo", "win", "vol", "mass", "ebc", "vinit", "props", "mat_type",
                                                     "body_id", "sm_len"))
    peak, peak_kind = measured_peak()
    acc = accuracy(case, p, dt, args.full_steps) if args.full_steps > 0 else None
    lrn = learned_runs(args, rank) if args.rate_h > 0 else None
    out = dict(case=case, n=n, nnz=nnz, kmean=kmean, dt=dt, res=res, step0_s=step0_s, e2e_s=e2e_s, h2d=h2d,
               d2h=d2h, peak=peak, peak_kind=peak_kind, scalars=s, dev_bytes=dev_bytes, accuracy=acc, learned=lrn)
    return out


STATE_FIELDS = (1, 2, 3, 4, 6, 7, 8, 9)  # dsp, dsp_tot, vel, acl, fext, stress, strain, eps


def accuracy(case, p, dt, steps):
    """FP64 and mixed runs of `steps` steps from impact: end-state length,
    mushroom radius and peak plastic strain, and (from the FP64 end state)
    the relative L2 difference of one step's nodal forces."""
    from taylor_b200 import _lib, cases, mega
    m = mega.Mega(case, p)
    m.search_and_shapes()
    m.step(steps, dt, mode="fp64")
    ref = cases.bar_metrics(case, m.download(_lib.F_COO_CURRENT), m.download(_lib.F_EPS))
    state = {f: m.download(f) for f in STATE_FIELDS}
    m.step(1, dt, mode="fp64")
    f64 = m.download(_lib.F_FINT)
    for f, v in state.items():
        m.upload(f, v)
    m.step(1, dt, mode="mixed")
    f32 = m.download(_lib.F_FINT)
    m.close()
    del state
    q = mega.Mega(case, p)
    q.search_and_shapes()
    q.step(steps, dt, mode="mixed")
    mix = cases.bar_metrics(case, q.download(_lib.F_COO_CURRENT), q.download(_lib.F_EPS))
    q.close()
    rel = {k: abs(mix[k] - ref[k]) / abs(ref[k]) for k in ref}
    return dict(steps=steps, fp64=ref, mixed=mix, mixed_rel_err=rel,
                force_rel_l2_one_step=float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64)))


RATE_LAW = (90e6, 292e6, 0.31, 0.025, 1.0)  # A, B, n, C, epsdot0 of the power-law rate-dependent hardening


def learned_runs(args, rank):
    """Rate-dependent bar: plain FP64, plain mixed and mixed + learned start
    from impact for the same steps.  The learned context logs return-mapping
    samples during the first quarter (plain Newton), trains the network on
    them on the device, then continues with the learned start; the other
    two run plain throughout.  Times cover the last three quarters."""
    from taylor_b200 import _lib, cases, mega
    case = cases.taylor_bar(h=args.rate_h, rate_law=RATE_LAW, seed=7 + rank)
    n = case["n"]
    p = _lib.params(**cases.param_kwargs(case, newton_max_iter=60, newton_rtol=1e-10))
    total = args.rate_steps
    first = total // 4
    rest = total - first
    runs = {}
    dt = None
    for name, mode, learn in (("fp64", "fp64", False), ("mixed", "mixed", False), ("mixed_learned", "mixed", True)):
        m = mega.Mega(case, p)
        m.search_and_shapes()
        if dt is None:
            nb = m.search_and_shapes(download=True)
            dt = cases.stable_dt(case, nb["gn"], nb["gstart"], nb["gstack"])
            del nb
        info = {}
        if learn:
            m.log_rate_samples(cap=10_000_000, stride=4, seed=3)
        m.step(first, dt, mode=mode)
        if learn:
            t0 = time.perf_counter()
            th, loss = m.train_surrogate(mega.mlp_init(5), epochs=6, batch=8192, lr=2e-3, seed=9)
            info.update(train_s=time.perf_counter() - t0, samples=int(min(10_000_000, _held_count(m))),
                        loss_first_epoch=float(loss[0]), loss_last_epoch=float(loss[-1]))
            m.log_rate_samples(0)
            del th
        s0 = m.scalars()
        clk = Clocks()
        clk.start()
        ms = m.step_timed(rest, dt, mode=mode, learned=learn)
        info["clocks"] = clk.stop()
        s1 = m.scalars()
        it = s1["newton_iters_total"] - s0["newton_iters_total"]
        pl = s1["plastic_nodes_total"] - s0["plastic_nodes_total"]
        kt = m.kernel_times(3, dt, mode=mode, learned=learn)
        end = cases.bar_metrics(case, m.download(_lib.F_COO_CURRENT), m.download(_lib.F_EPS))
        m.close()
        info.update(ms_per_step=ms / rest, node_steps_per_s=n * rest / (ms / 1e3), newton_iters=int(it),
                    plastic_updates=int(pl), iters_per_plastic_update=it / max(pl, 1),
                    stress_kernel_ms=float(kt[1]), end_state=end)
        runs[name] = info
    ref = runs["fp64"]["end_state"]
    for name in ("mixed", "mixed_learned"):
        e = runs[name]["end_state"]
        runs[name]["rel_err_vs_fp64"] = {k: abs(e[k] - ref[k]) / abs(ref[k]) for k in ref}
    return dict(workload=f"rate-dependent taylor_bar h={args.rate_h*1e3:.3g}mm", nodes=n, dt=dt, steps=total,
                timed_steps=rest, rate_law=dict(A=RATE_LAW[0], B=RATE_LAW[1], n=RATE_LAW[2], C=RATE_LAW[3],
                                                epsdot0=RATE_LAW[4]), newton_rtol=1e-10, runs=runs,
                mixed_learned_over_fp64=runs["fp64"]["ms_per_step"] / runs["mixed_learned"]["ms_per_step"],
                iteration_reduction=1.0 - runs["mixed_learned"]["iters_per_plastic_update"]
                / runs["mixed"]["iters_per_plastic_update"])


def _held_count(m):
    import ctypes as C
    from taylor_b200 import _lib
    k = C.c_int64(0)
    _lib.check(_lib.lib().mega_rate_samples(m.h, None, 0, C.byref(k)), "rate_samples")
    return k.value


def cpu_baseline(case, steps, nthreads):
    from oracle import oracle as O
    from taylor_b200 import cases
    p = O.params(**cases.param_kwargs(case))
    r = O.Run(case, p, nthreads=nthreads)
    dt = cases.stable_dt(case, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    r.step(1, dt)
    t0 = time.perf_counter()
    r.step(steps, dt)
    el = time.perf_counter() - t0
    return case["n"] * steps / el, el


def main():
    args = parse()
    rank, world, dist = dist_setup(args.gpus)
    if args.impl == "reference":
        if rank != 0:
            return
        from taylor_b200 import cases
        case = cases.taylor_bar(h=args.h, seed=1)
        nthreads = os.cpu_count() or 1
        steps = args.cpu_steps or max(1, min(args.steps, 10))
        for _ in range(0):
            pass
        val, el = cpu_baseline(case, steps, nthreads)
        line = dict(metric=METRIC, value=val, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                    ms_per_step=1e3 * el / steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64", data="synthetic", impl="reference",
                    config=dict(workload=f"taylor_bar_1M h={args.h*1e3:.3g}mm n={case['n']}", nodes=case["n"],
                                sample=f"{steps} explicit steps after step 0 (reference arm: C++ OpenMP "
                                       f"restatement of MEGA, the Fortran reference cannot be compiled here)"),
                    cpu_baseline=dict(value=val, unit=UNIT, cores=nthreads, kind="port",
                                      sample=f"{steps} steps of the {case['n']}-node bar"),
                    e2e=dict(value=val, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line))
        return

    r = run_ours(args, rank, world, dist)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    n, nnz, K = r["n"], r["nnz"], args.steps
    mix = r["res"].get("mixed") or r["res"]["fp64"]
    f64 = r["res"].get("fp64") or mix
    value = world * n * K / (mix["ms"] / 1e3)
    fp64_value = world * n * K / (f64["ms"] / 1e3)
    # roofline of the dominant kernel (mixed path, the headline)
    kb = kernel_bytes(n, nnz, mixed=True)
    names = ["defgrad", "stress", "force"]
    kt = mix["kt"]
    dom = int(np.argmax(kt))
    achieved = kb[names[dom]] / (kt[dom] / 1e3) / 1e9
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = prof.get(f"mixed_{names[dom]}_bytes_per_launch")
    except Exception:
        pass
    roof = dict(bound="hbm", kernel=f"k_{names[dom]} (mixed)", achieved=achieved, peak=r["peak"], unit="GB/s",
                frac=achieved / r["peak"], traffic=traffic, peak_source=r["peak_kind"],
                all_kernels={nm: dict(ms=kt[i], gbs=kb[nm] / (kt[i] / 1e3) / 1e9,
                                      frac=kb[nm] / (kt[i] / 1e3) / 1e9 / r["peak"]) for i, nm in enumerate(names)},
                fp64_kernels={nm: dict(ms=f64["kt"][i],
                                       gbs=kernel_bytes(n, nnz, False)[nm] / (f64["kt"][i] / 1e3) / 1e9)
                              for i, nm in enumerate(names)},
                step_bytes_per_node_survey=dict(fp64=survey_step_bytes(nnz / n, False),
                                                mixed=survey_step_bytes(nnz / n, True)))
    cpu = None
    if not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        steps = args.cpu_steps or 5
        val, el = cpu_baseline(r["case"], steps, nthreads)
        cpu = dict(value=val, unit=UNIT, cores=nthreads, kind="port",
                   sample=f"{steps} explicit steps of the same {n}-node bar after step 0, C++ OpenMP restatement "
                          f"of MEGA with per-thread FINT_TEMP buffers (the Fortran reference cannot be compiled here)")
    e2e_val = world * n * K / r["e2e_s"]
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=K, warmup=args.warmup,
        ms_per_step=mix["ms"] / K, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32+f64",
        data="synthetic (seeded jittered lattice of the 0.1 mm copper bar, random-free material data)",
        config=dict(workload=f"taylor_bar_1M h={args.h*1e3:.3g}mm", nodes=n, nnz=nnz, mean_neighbours=nnz / n,
                    dt=r["dt"], parallelism=f"replicas{world}", l2="inputs larger than L2 (no flush needed)",
                    step0_search_shapes_s=r["step0_s"], device_bytes=r["dev_bytes"]),
        fp64_value=fp64_value, fp64_ms_per_step=f64["ms"] / K, mixed_over_fp64=value / fp64_value,
        roofline=roof, cpu_baseline=cpu,
        e2e=dict(value=e2e_val, unit=UNIT, h2d_bytes_per_step=r["h2d"] / K, d2h_bytes_per_step=r["d2h"] / K,
                 note="model upload + step 0 + K steps with per-step scalar readback + end-state download"),
        gpu_launches=mix["launches"], clocks=mix["clocks"], clocks_fp64=f64["clocks"],
        newton_iters_last_step=r["scalars"]["newton_iters"], plastic_nodes_last_step=r["scalars"]["plastic_nodes"],
        accuracy=r["accuracy"], learned=r["learned"])
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
