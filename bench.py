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
host every step, and the end-state download, all inside the timed region
(after one untimed job of the same size, so that the device memory pool and
the pinned staging buffer have reached the job's sizes).

Further sections of the same line (each skippable by its flag):
  accuracy      FP64 vs mixed end states after --full-steps steps
  learned       the 2M-node rate-dependent bar: FP64, mixed, mixed with the
                textbook Newton start, mixed with the learned start
  peridynamics  the 2.56M-particle bond-based plate (--pmb-nx)
  nsni          the same bar with stabilised nodal integration: timing in
                both precisions and --nsni-steps from impact
  pre_model     device mesh pre-processing of a --pre-nodes^3 hexahedral box
  batch         --batch-bars bars of uneven size in one context vs one
                context per bar
  cpu_baseline  the C++ OpenMP restatement of the reference on the host

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
    ap.add_argument("--cpu-steps", type=int, default=0, help="timed steps of the CPU baseline (0 = --steps)")
    ap.add_argument("--modes", default="fp64,mixed", help="order in which the precision modes run")
    ap.add_argument("--full-steps", type=int, default=600,
                    help="steps of the accuracy runs (FP64 vs mixed end states); 0 skips them")
    ap.add_argument("--rate-h", type=float, default=0.08e-3,
                    help="lattice spacing of the rate-dependent bar of the learned-start runs; 0 skips them")
    ap.add_argument("--rate-steps", type=int, default=600, help="steps of the rate-dependent runs")
    ap.add_argument("--pmb-nx", type=int, default=400,
                    help="in-plane particles per side of the bond-based peridynamics plate; 0 skips it")
    ap.add_argument("--pmb-steps", type=int, default=4000, help="steps of the peridynamics run")
    ap.add_argument("--nsni-steps", type=int, default=2000,
                    help="steps of the stabilised-nodal-integration runs of the same bar; 0 skips them")
    ap.add_argument("--pre-nodes", type=int, default=100,
                    help="nodes per side of the hexahedral mesh of the pre-processing run; 0 skips it")
    ap.add_argument("--batch-bars", type=int, default=256, help="bars of the batched run; 0 skips it")
    ap.add_argument("--batch-steps", type=int, default=1500, help="timed steps of the batched and sequential runs")
    return ap.parse_args()


def dist_setup(n, backend="nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): the
    process group carries only the barriers and the max-over-ranks timing
    (replicas: every rank steps its own bar, no data-path collective)."""
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return rank, world, dist
    return rank, world, None


def max_over_ranks(v, dist):
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
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


def rel_err(x, ref):
    """|x - ref| / |ref| per measure (the absolute difference where ref is 0)."""
    return {k: abs(x[k] - ref[k]) / abs(ref[k]) if ref[k] != 0 else abs(x[k] - ref[k]) for k in ref}


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo), for the CPU baselines."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def workload_name(h, n):
    """The workload string both arms report for the same bar."""
    return f"taylor_bar_1M h={h*1e3:.3g}mm n={n} direct nodal integration"


def kernel_bytes(n, nnz, mixed):
    """Algorithmic bytes per launch of each per-step kernel (every array
    touched once; neighbour data counted once per owning node)."""
    g = 12 if mixed else 24          # three gradient components per CSR entry
    t = 36 if mixed else 72          # T_i (3x3) per node
    fg = 72 if mixed else 144        # F (less its identity in mixed) and G0 per node
    defgrad = nnz * (4 + g) + n * (8 + 48 + 24 + fg)            # col + grad; rowptr, u and du, sum grad, F/G0 out
    stress = n * (fg + 192 + 16 + 8 + 8 + 8 + 2 + t)            # F/G0, sigma+eps rw, eps_p rw, eq, wvel, vol, mat, T
    force = nnz * (4 + g) + n * (8 + t + 3 + 24 + 24 + 48 + 48 + 24 + 48 + 48 + 24)  # trow + grad^T; T, fixity,
    return dict(defgrad=defgrad, stress=stress, force=force)     # mass, fint, fext rw, vel rw, acl, dsp rw, tot rw, pr


def nsni_step_bytes(n, nnz, mixed):
    """Algorithmic bytes of one NSNI step (every array touched once): the
    DNI kernels on the seven-point lists (kernel_bytes), the six second
    derivatives S of every entry in both gathers (6 s bytes each, s = 4
    mixed or 8; the FP64 NSNI gathers also read each entry's row / column
    index, 4 bytes, and k_nsni_h gathers the increment, 24 per node, which
    the mixed gathers have staged already), H (18 doubles written, read),
    the stress gradients (18 doubles read and written), the force weights
    (18 floats / doubles written, read), the stress before the step (6
    doubles copied and read) and, in FP64, the stabilisation force (3
    doubles written, read)."""
    kb = kernel_bytes(n, nnz, mixed)
    s = 4 if mixed else 8
    w = 80 if mixed else 144
    per_entry = 2 * (6 * s) if mixed else 2 * (4 + 6 * s)
    per_node = 2 * 144 + 2 * 144 + 2 * w + 3 * 48 + (0 if mixed else 24 + 2 * 24)
    return kb["defgrad"] + kb["stress"] + kb["force"] + nnz * per_entry + n * per_node


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
    tuned = {}
    for mode in args.modes.split(","):
        (vd, vf), tms = m.autotune(dt, mode=mode, reps=5)  # launch variants of the two gathers
        tuned[mode] = dict(defgrad_variant=vd, force_variant=vf, defgrad_ms=[float(x) for x in tms[0]],
                           force_ms=[float(x) for x in tms[1]])
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

    # end to end through the public API from host buffers: one untimed job
    # first (the device memory pool and the pinned staging buffer reach the
    # job's sizes), then the timed one
    def job(steps):
        t0 = time.perf_counter()
        e = mega.Mega(case, p)
        e.set_precisions(fp64=False, mixed=True)   # the job steps in mixed precision only
        t1 = time.perf_counter()
        e.search_and_shapes()
        t2 = time.perf_counter()
        d2h = 0
        for _ in range(steps):
            e.step(1, dt, mode="mixed")
            e.scalars()            # ENERGY_INFO.OUT / TOTAL_FORCE.OUT / TIME.OUT of MAIN, every step
            d2h += 8 * 12
        t3 = time.perf_counter()
        xend = e.download(_lib.F_COO_CURRENT)
        epend = e.download(_lib.F_EPS)
        d2h += xend.nbytes + epend.nbytes
        e.close()
        t4 = time.perf_counter()
        return (t0, t1, t2, t3, t4), d2h

    job(args.warmup)
    barrier(dist)
    (t0, t1, t2, t3, t4), d2h = job(args.steps)
    e2e_s = max_over_ranks(t4 - t0, dist)
    e2e_parts = dict(upload_s=t1 - t0, search_shapes_s=t2 - t1, steps_s=t3 - t2, download_close_s=t4 - t3)
    h2d = sum(np.asarray(case[k]).nbytes for k in ("coo", "win", "vol", "mass", "ebc", "vinit", "props", "mat_type",
                                                     "body_id", "sm_len"))
    peak, peak_kind = measured_peak()
    acc = lrn = None
    try:
        acc = accuracy(case, p, dt, args.full_steps) if args.full_steps > 0 else None
    except Exception as ex:  # reported in the JSON line, the timing above stands
        acc = dict(error=str(ex))
    try:
        lrn = learned_runs(args, rank) if args.rate_h > 0 else None
    except Exception as ex:
        lrn = dict(error=str(ex))
    try:
        pmb = pmb_run(args) if args.pmb_nx > 0 else None
    except Exception as ex:
        pmb = dict(error=str(ex))
    try:
        nsni = nsni_run(case, dt, args) if args.nsni_steps > 0 else None
    except Exception as ex:
        nsni = dict(error=str(ex))
    try:
        pre = pre_model_run(args) if args.pre_nodes > 0 else None
    except Exception as ex:
        pre = dict(error=str(ex))
    try:
        batch = batch_run(args) if args.batch_bars > 0 else None
    except Exception as ex:
        batch = dict(error=str(ex))
    out = dict(case=case, n=n, nnz=nnz, kmean=kmean, dt=dt, res=res, step0_s=step0_s, e2e_s=e2e_s, h2d=h2d,
               d2h=d2h, peak=peak, peak_kind=peak_kind, scalars=s, dev_bytes=dev_bytes, accuracy=acc, learned=lrn, pmb=pmb,
               nsni=nsni, pre_model=pre, batch=batch,
               tuned=tuned,
               e2e_parts=e2e_parts)
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
    rel = rel_err(mix, ref)
    return dict(steps=steps, fp64=ref, mixed=mix, mixed_rel_err=rel,
                force_rel_l2_one_step=float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64)))


def nsni_run(case, dt, args):
    """The same bar with stabilised nodal integration (ITYPE_INT = 2):
    set-up time, device-timed steps in both precisions, then FP64 and mixed
    runs from impact for --nsni-steps steps (the horizon direct nodal
    integration does not reach on this lattice) with their end states, and
    two more FP64 runs whose initial velocity differs by one part in 1e12
    and in 1e7: how far the end-state measures move under a perturbation at
    the FP64 and at the FP32 noise level (their conditioning), the
    yardstick for the mixed run's error.  The step is 0.8 of the timing
    runs' (0.4 x 0.9 h / c): at 0.5 x 0.9 h / c the compressed wall region
    runs at the edge of stability over 2,000 steps and the largest nodal
    strain moves by 1e-2 under the 1e-12 perturbation."""
    from taylor_b200 import _lib, cases, mega
    p = _lib.params(**cases.param_kwargs(case, itype_int=2))
    dt = 0.8 * dt
    out = dict(steps=args.nsni_steps, dt=dt)
    for mode in ("mixed", "fp64"):
        t0 = time.perf_counter()
        m = mega.Mega(case, p)
        res = m.search_and_shapes()
        setup_s = time.perf_counter() - t0
        m.autotune(dt, mode=mode, reps=3)
        m.step(args.warmup, dt, mode=mode)
        clk = Clocks()
        clk.start()
        ms = m.step_timed(args.steps, dt, mode=mode)
        clocks = clk.stop()
        st = m.step(args.nsni_steps - args.warmup - args.steps, dt, mode=mode, allow_status=True)
        end = cases.bar_metrics(case, m.download(_lib.F_COO_CURRENT), m.download(_lib.F_EPS))
        peak, _ = measured_peak()
        sb = nsni_step_bytes(case["n"], int(res["nnz"]), mode == "mixed")
        gbs = sb / (ms / args.steps / 1e3) / 1e9
        out[mode] = dict(setup_s=setup_s, nnz=int(res["nnz"]), ms_per_step=ms / args.steps,
                         node_steps_per_s=case["n"] * args.steps / (ms / 1e3), clocks=clocks, status=int(st),
                         end_state=end, device_bytes=m.device_bytes(),
                         roofline=dict(bound="hbm", scope="whole NSNI step", achieved=gbs, peak=peak, unit="GB/s",
                                       frac=gbs / peak, algorithmic_bytes_per_step=sb,
                                       hbm_floor_ms=sb / (peak * 1e9) * 1e3))
        m.close()
    if "end_state" in out.get("fp64", {}) and "end_state" in out.get("mixed", {}):
        ref, mix = out["fp64"]["end_state"], out["mixed"]["end_state"]
        out["mixed_rel_err"] = rel_err(mix, ref)
        for eps_v, key in ((1.0e-12, "fp64_perturbed_1e-12_rel_change"), (1.0e-7, "fp64_perturbed_1e-7_rel_change")):
            cp = dict(case)
            cp["vinit"] = np.asarray(case["vinit"]) * (1.0 + eps_v)
            q = mega.Mega(cp, p)
            q.search_and_shapes()
            q.step(args.nsni_steps, dt, mode="fp64", allow_status=True)
            pert = cases.bar_metrics(case, q.download(_lib.F_COO_CURRENT), q.download(_lib.F_EPS))
            q.close()
            out[key] = rel_err(pert, ref)
    # direct nodal integration over the same steps, for its status
    d = mega.Mega(case, _lib.params(**cases.param_kwargs(case)))
    d.search_and_shapes()
    out["dni_fp64_status"] = int(d.step(args.nsni_steps, dt, mode="fp64", allow_status=True))
    out["dni_fp64_end_state"] = cases.bar_metrics(case, d.download(_lib.F_COO_CURRENT), d.download(_lib.F_EPS))
    d.close()
    return out


def pre_model_run(args):
    """Mesh pre-processing (windows, volumes, smoothing cells) of a jittered
    hexahedral box through the C ABI from host arrays, against the oracle's
    vectorised CPU restatement of the same loops."""
    from taylor_b200 import cases, mega
    sys.path.insert(0, ROOT)
    from oracle import premodel as P
    k = args.pre_nodes
    coo, elems = cases.hex_box(k, k, k, 0.1e-3, jitter=0.05, seed=3)
    mega.pre_model_hex(coo, elems, norm_win=2.0)  # warm-up (same sizes)
    t0 = time.perf_counter()
    got = mega.pre_model_hex(coo, elems, norm_win=2.0)
    gpu_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    w, v = P.hex_windows_and_volumes(coo, elems)
    P.smoothing_lengths(v, w)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(got["win_raw"], w) and np.array_equal(got["vol"], v))
    return dict(workload=f"hex box {k}^3 nodes, h=0.1mm, 5% jitter", nodes=len(coo), elements=len(elems),
                gpu_s_with_copies=gpu_s, cpu_numpy_s=cpu_s, windows_and_volumes_bit_exact=same)


RATE_LAW = (90e6, 292e6, 0.31, 0.025, 1.0)  # A, B, n, C, epsdot0 of the power-law rate-dependent hardening


def learned_runs(args, rank):
    """Rate-dependent bar: plain FP64, plain mixed, mixed with the textbook
    Newton start (perfectly plastic estimate, Newton in dgamma) and mixed +
    learned start, from impact for the same steps.  The plain solver starts
    Newton in ln(dgamma) from the upper bound of the multiplier.  The learned
    context logs return-mapping samples during the first quarter (plain
    Newton), trains the network on them on the device, then continues with
    the learned start; the others run plain throughout.  Times cover the last
    three quarters."""
    from taylor_b200 import _lib, cases, mega
    case = cases.taylor_bar(h=args.rate_h, rate_law=RATE_LAW, seed=7 + rank)
    n = case["n"]
    p = _lib.params(**cases.param_kwargs(case, newton_max_iter=60, newton_rtol=1e-10))
    p_textbook = _lib.params(**cases.param_kwargs(case, newton_max_iter=60, newton_rtol=1e-10, rate_solver=1))
    total = args.rate_steps
    first = total // 4
    rest = total - first
    runs = {}
    dt = None
    for name, mode, learn, pp in (("fp64", "fp64", False, p), ("mixed", "mixed", False, p),
                                  ("mixed_textbook_newton", "mixed", False, p_textbook),
                                  ("mixed_learned", "mixed", True, p)):
        m = mega.Mega(case, pp)
        m.search_and_shapes()
        if dt is None:
            nb = m.search_and_shapes(download=True)
            dt = cases.stable_dt(case, nb["gn"], nb["gstart"], nb["gstack"])
            del nb
        m.autotune(dt, mode=mode, reps=3)  # as every timed run: variants and (mixed) the banked record layout
        info = {}
        if learn:
            m.log_rate_samples(cap=10_000_000, stride=4, seed=3)
        st_first = m.step(first, dt, mode=mode, allow_status=True)
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
        ms = m.step_timed(rest, dt, mode=mode, learned=learn, allow_status=True)
        info["clocks"] = clk.stop()
        info["status"] = int(st_first | m.last_status)
        s1 = m.scalars()
        it = s1["newton_iters_total"] - s0["newton_iters_total"]
        pl = s1["plastic_nodes_total"] - s0["plastic_nodes_total"]
        try:
            kt = m.kernel_times(3, dt, mode=mode, learned=learn)
        except Exception:
            kt = [float("nan")] * 3
        end = cases.bar_metrics(case, m.download(_lib.F_COO_CURRENT), m.download(_lib.F_EPS))
        m.close()
        info.update(ms_per_step=ms / rest, node_steps_per_s=n * rest / (ms / 1e3), newton_iters=int(it),
                    plastic_updates=int(pl), iters_per_plastic_update=it / max(pl, 1),
                    stress_kernel_ms=float(kt[1]), end_state=end)
        runs[name] = info
    ref = runs["fp64"]["end_state"]
    for name in ("mixed", "mixed_textbook_newton", "mixed_learned"):
        e = runs[name]["end_state"]
        runs[name]["rel_err_vs_fp64"] = rel_err(e, ref)
    return dict(workload=f"rate-dependent taylor_bar h={args.rate_h*1e3:.3g}mm", nodes=n, dt=dt, steps=total,
                timed_steps=rest, rate_law=dict(A=RATE_LAW[0], B=RATE_LAW[1], n=RATE_LAW[2], C=RATE_LAW[3],
                                                epsdot0=RATE_LAW[4]), newton_rtol=1e-10, runs=runs,
                mixed_learned_over_fp64=runs["fp64"]["ms_per_step"] / runs["mixed_learned"]["ms_per_step"],
                iteration_reduction_vs_plain=1.0 - runs["mixed_learned"]["iters_per_plastic_update"]
                / runs["mixed"]["iters_per_plastic_update"],
                iteration_reduction_vs_textbook=1.0 - runs["mixed_learned"]["iters_per_plastic_update"]
                / runs["mixed_textbook_newton"]["iters_per_plastic_update"])


def pmb_run(args):
    """Bond-based PMB plate (400 x 400 x 16 particles at 0.25 mm, horizon
    3.015 h, pre-notch cut on the device, the notch-side edge halves driven
    apart at a sustained +-5 m/s): the mixed run (float bond force, double
    positions) steps the whole job, the FP64 run a tenth of it; broken bonds
    and the crack tip (from the particles' local damage) are reported."""
    from taylor_b200 import cases, mega
    nz = max(4, args.pmb_nx // 25)
    case = cases.pd_plate(nx=args.pmb_nx, ny=args.pmb_nx, nz=nz, notch=20e-3 * args.pmb_nx / 400)
    n = case["n"]
    dt = 0.5 * case["h"] / np.sqrt(72e9 / case["rho"])
    out = dict(workload=f"pmb plate {args.pmb_nx}x{args.pmb_nx}x{nz} h=0.25mm", particles=n, dt=dt)
    peak, _ = measured_peak()
    for mode, steps in (("mixed", args.pmb_steps), ("fp64", max(10, args.pmb_steps // 10))):
        t0 = time.perf_counter()
        p = mega.Pmb(case, None, fixed=case["fixed"], mode=mode)
        init_s = time.perf_counter() - t0
        ncut = p.cut(*cases.notch_rect(case))
        p.step(3, dt)
        clk = Clocks()
        clk.start()
        ms = p.step(steps, dt, timed=True)
        clocks = clk.stop()
        dmg, nbroken = p.download(4)
        tip = cases.crack_tip(case, dmg)
        bonds = p.nnz
        # per step: bond column index and broken bit; per particle u in/out,
        # velocity and acceleration read+write, X, volume, fixity
        algo = bonds * (4 + 1 / 8) + n * (24 + 24 + 48 + 48 + 24 + 8 + 1)
        gbs = algo / (ms / steps / 1e3) / 1e9
        out[mode] = dict(steps=steps, ms_per_step=ms / steps, particle_steps_per_s=n * steps / (ms / 1e3),
                         bonds=bonds, notch_bonds=ncut, broken_bond_entries=nbroken, init_s=init_s,
                         crack_tip_x_m=tip, crack_growth_m=None if tip is None else tip - case["notch"],
                         damaged_particles=int(np.count_nonzero(dmg > 0.35)),
                         roofline=dict(bound="hbm", achieved=gbs, peak=peak, unit="GB/s", frac=gbs / peak,
                                       algorithmic_bytes_per_step=algo),
                         clocks=clocks)
        p.close()
    return out


def batch_run(args):
    """Many bars of uneven size (spacing uniform in 0.15-0.6 mm, v0 in
    100-300 m/s, sigma_y in 200-600 MPa, H = 100 MPa, one seed) stepped as
    one context, every step one CUDA-graph replay over all bars, each bar
    with its own stable step (mega_set_instance_dt), against the same bars
    stepped one context after another.  Mixed precision, --batch-steps steps
    of every bar timed.  Then the same bars with the power-law
    rate-dependent law (A = sigma_y) log return-mapping samples on the batch
    path and train the surrogate on them on the device."""
    from taylor_b200 import _lib, cases, mega
    b = cases.batch_bars(args.batch_bars)
    n = b["n"]
    p = _lib.params(**cases.param_kwargs(b, dist_max=tuple(float(v) for v in b["dist_max"].max(axis=0)),
                                         ql_len=b["ql_len"]))
    dts = b["dt"]
    K_steps = args.batch_steps
    t0 = time.perf_counter()
    m = mega.Mega(b, p)
    m.set_instances(b["counts"], b["dist_max"])
    m.set_precisions(fp64=False, mixed=True)
    m.search_and_shapes()
    m.set_instance_dt(dts)
    init_s = time.perf_counter() - t0
    m.step(3, float(dts.min()), mode="mixed")
    clk = Clocks()
    clk.start()
    ms = m.step_timed(K_steps, float(dts.min()), mode="mixed", allow_status=True)
    clocks = clk.stop()
    status = int(m.last_status)
    xb = m.download(_lib.F_COO_CURRENT)
    dev_bytes = m.device_bytes()
    m.close()
    off = np.concatenate([[0], np.cumsum(b["counts"])])
    finite_bars = int(sum(np.all(np.isfinite(xb[off[k]:off[k + 1]])) for k in range(len(b["bars"]))))
    seq_ms = 0.0
    t0 = time.perf_counter()
    for k, bar in enumerate(b["bars"]):
        pk = _lib.params(**cases.param_kwargs(bar, dist_max=tuple(float(v) for v in b["dist_max"][k]),
                                              ql_len=b["ql_len"]))
        s = mega.Mega(bar, pk)
        s.set_precisions(fp64=False, mixed=True)
        s.search_and_shapes()
        s.step(3, float(dts[k]), mode="mixed")
        seq_ms += s.step_timed(K_steps, float(dts[k]), mode="mixed", allow_status=True)
        s.close()
    seq_wall = time.perf_counter() - t0
    # the rate-dependent batch generates the surrogate's training data
    rb = cases.batch_bars(args.batch_bars, rate_law=RATE_LAW[1:])
    pr = _lib.params(**cases.param_kwargs(rb, dist_max=tuple(float(v) for v in rb["dist_max"].max(axis=0)),
                                          ql_len=rb["ql_len"], newton_max_iter=60, newton_rtol=1e-10))
    q = mega.Mega(rb, pr)
    q.set_instances(rb["counts"], rb["dist_max"])
    q.set_precisions(fp64=False, mixed=True)
    q.search_and_shapes()
    q.set_instance_dt(rb["dt"])
    q.log_rate_samples(cap=10_000_000, stride=4, seed=11)
    log_steps = max(1, K_steps // 5)
    t1 = time.perf_counter()
    rst = q.step(log_steps, float(rb["dt"].min()), mode="mixed", allow_status=True)
    log_s = time.perf_counter() - t1
    held = _held_count(q)
    t1 = time.perf_counter()
    _, loss = q.train_surrogate(mega.mlp_init(5), epochs=6, batch=8192, lr=2e-3, seed=9)
    train_s = time.perf_counter() - t1
    q.close()
    return dict(workload=f"{args.batch_bars} Taylor bars, h in 0.15-0.6 mm", bars=args.batch_bars, nodes=n,
                nodes_min=int(b["counts"].min()), nodes_max=int(b["counts"].max()),
                dt_min=float(dts.min()), dt_max=float(dts.max()), steps=K_steps, per_instance_dt=True,
                batched=dict(ms_per_step=ms / K_steps, node_steps_per_s=n * K_steps / (ms / 1e3), init_s=init_s,
                             device_bytes=dev_bytes, clocks=clocks, status=status, bars_finite=finite_bars),
                sequential=dict(ms_per_step=seq_ms / K_steps, node_steps_per_s=n * K_steps / (seq_ms / 1e3),
                                wall_s_with_init=seq_wall),
                batched_over_sequential=seq_ms / ms,
                surrogate_data=dict(law="power-law rate-dependent, A = sigma_y of each bar", steps=log_steps,
                                    samples=int(held), log_s=log_s, status=int(rst), train_s=train_s,
                                    loss_first_epoch=float(loss[0]), loss_last_epoch=float(loss[-1])))


def _held_count(m):
    import ctypes as C
    from taylor_b200 import _lib
    k = C.c_int64(0)
    _lib.check(_lib.lib().mega_rate_samples(m.h, None, 0, C.byref(k)), "rate_samples")
    return k.value


def cpu_baseline(case, steps, nthreads, warmup=1):
    """The oracle (C++ OpenMP restatement of MEGA with the reference's
    per-thread FINT_TEMP buffers) on the host cores: step 0, `warmup`
    untimed steps, then `steps` timed steps of the same bar."""
    from oracle import oracle as O
    from taylor_b200 import cases
    p = O.params(**cases.param_kwargs(case))
    r = O.Run(case, p, nthreads=nthreads)
    dt = cases.stable_dt(case, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    r.step(max(1, warmup), dt)
    t0 = time.perf_counter()
    r.step(steps, dt)
    el = time.perf_counter() - t0
    return case["n"] * steps / el, el


def main():
    args = parse()
    if args.impl == "reference":
        if int(os.environ.get("RANK", 0)) != 0:  # rank 0 alone times the host cores; no process group
            return
        from taylor_b200 import cases
        case = cases.taylor_bar(h=args.h, seed=1)
        nthreads = os.cpu_count() or 1
        steps = args.steps
        val, el = cpu_baseline(case, steps, nthreads, warmup=args.warmup)
        sample = (f"{steps} timed explicit steps of the {case['n']}-node bar after step 0 and {args.warmup} "
                  f"untimed ones, C++ OpenMP restatement of MEGA with per-thread FINT_TEMP buffers on "
                  f"{nthreads} threads of {cpu_model()} (the Fortran reference cannot be compiled here)")
        line = dict(metric=METRIC, value=val, unit=UNIT, n_gpus=args.gpus, steps=steps, warmup=args.warmup,
                    ms_per_step=1e3 * el / steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64", data="synthetic (seeded jittered lattice of the 0.1 mm copper bar)",
                    impl="reference",
                    config=dict(workload=workload_name(args.h, case["n"]), nodes=case["n"], sample=sample),
                    cpu_baseline=dict(value=val, unit=UNIT, cores=nthreads, kind="port", cpu=cpu_model(),
                                      sample=sample),
                    e2e=dict(value=val, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line))
        return

    rank, world, dist = dist_setup(args.gpus)
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
        steps = args.cpu_steps or args.steps
        val, el = cpu_baseline(r["case"], steps, nthreads)
        cpu = dict(value=val, unit=UNIT, cores=nthreads, kind="port", cpu=cpu_model(), seconds=el,
                   sample=f"{steps} timed explicit steps of the same {n}-node bar after step 0 and one untimed "
                          f"step, C++ OpenMP restatement of MEGA with per-thread FINT_TEMP buffers on {nthreads} "
                          f"threads of {cpu_model()} (the Fortran reference cannot be compiled here)")
    e2e_val = world * n * K / r["e2e_s"]
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=K, warmup=args.warmup,
        ms_per_step=mix["ms"] / K, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32+f64",
        data="synthetic (seeded jittered lattice of the 0.1 mm copper bar, random-free material data)",
        config=dict(workload=workload_name(args.h, n), nodes=n, nnz=nnz, mean_neighbours=nnz / n,
                    dt=r["dt"], parallelism=f"replicas{world}", l2="inputs larger than L2 (no flush needed)",
                    step0_search_shapes_s=r["step0_s"], device_bytes=r["dev_bytes"], autotuned=r["tuned"]),
        fp64_value=fp64_value, fp64_ms_per_step=f64["ms"] / K, mixed_over_fp64=value / fp64_value,
        roofline=roof, cpu_baseline=cpu,
        e2e=dict(value=e2e_val, unit=UNIT, h2d_bytes_per_step=r["h2d"] / K, d2h_bytes_per_step=r["d2h"] / K,
                 note="model upload + step 0 + K steps with per-step scalar readback + end-state download, "
                      "after one untimed job of the same size",
                 parts=r["e2e_parts"]),
        gpu_launches=mix["launches"], clocks=mix["clocks"], clocks_fp64=f64["clocks"],
        newton_iters_last_step=r["scalars"]["newton_iters"], plastic_nodes_last_step=r["scalars"]["plastic_nodes"],
        accuracy=r["accuracy"], learned=r["learned"], peridynamics=r["pmb"], nsni=r["nsni"],
        pre_model=r["pre_model"], batch=r["batch"])
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
