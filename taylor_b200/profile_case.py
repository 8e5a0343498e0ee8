"""Small, fixed workloads for profiling one kernel family under ncu.

    python -m taylor_b200.profile_case step  [--h 0.2e-3] [--mode mixed] [--steps 6] [--variant V]
    python -m taylor_b200.profile_case nsni  [--h 0.2e-3] [--mode mixed] [--steps 6] [--variant V]
    python -m taylor_b200.profile_case pmb   [--nx 200]   [--mode mixed] [--steps 6]
    python -m taylor_b200.profile_case learned [--h 0.16e-3] [--steps 6]

Each builds its case, runs the set-up, then `--steps` explicit steps one
launch sequence at a time (no graph replay, so `ncu -k <kernel> -s <skip>`
sees every launch), and prints one line with the case size.  The default
sizes keep the packed records above the 126 MB L2 while the whole run holds
a few GB at most, as a capture with many metric passes needs.
"""
import argparse
import sys
import time

from taylor_b200 import _lib, cases, mega


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["step", "nsni", "pmb", "learned"])
    ap.add_argument("--h", type=float, default=0.2e-3)
    ap.add_argument("--nx", type=int, default=200)
    ap.add_argument("--mode", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--variant", type=int, default=-1, help="pin both gathers' launch variant (-1: autotune)")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    if a.what == "pmb":
        case = cases.pd_plate(nx=a.nx, ny=a.nx, nz=max(4, a.nx // 25), notch=20e-3 * a.nx / 400)
        p = mega.Pmb(case, None, fixed=case["fixed"], mode=a.mode)
        p.cut(*cases.notch_rect(case))
        dt = 0.5 * case["h"] / (72e9 / case["rho"]) ** 0.5
        for _ in range(a.steps):
            p.step(1, dt)
        _, nb = p.download(3)
        print(f"pmb plate {a.nx}x{a.nx}: {case['n']} particles, {p.nnz} bonds, {nb} broken, "
              f"{time.perf_counter() - t0:.1f} s")
        p.close()
        return 0
    if a.what == "learned":
        case = cases.taylor_bar(h=a.h if a.h != 0.2e-3 else 0.16e-3, rate_law=(90e6, 292e6, 0.31, 0.025, 1.0))
        p = _lib.params(**cases.param_kwargs(case, newton_max_iter=60, newton_rtol=1e-10))
    else:
        case = cases.taylor_bar(h=a.h)
        p = _lib.params(**cases.param_kwargs(case, itype_int=2 if a.what == "nsni" else 0))
    m = mega.Mega(case, p)
    info = m.search_and_shapes()
    dt = 0.5 * 0.9 * case["h"] / 4590.0
    # the tuner also lays the float records out for the gathers' banks (its
    # first mixed call), as a production run has them; --variant then pins
    # both gathers
    m.autotune(dt, mode=a.mode, reps=3)
    if a.variant >= 0:
        m.set_variants(a.variant, a.variant, mode=a.mode)
    learned = a.what == "learned"
    if learned:
        m.log_rate_samples(cap=2_000_000, stride=2, seed=3)
        m.step(200, dt, mode=a.mode, allow_status=True)     # impact first: plastic nodes to learn from
        m.train_surrogate(mega.mlp_init(5), epochs=3, batch=8192, lr=2e-3, seed=9)
        m.log_rate_samples(0)
    for _ in range(a.steps):
        m.step(1, dt, mode=a.mode, learned=learned, allow_status=True)
    print(f"{a.what} bar h={case['h']*1e3:.3g}mm: {case['n']} nodes, {info['nnz']} entries, {a.mode}, "
          f"{time.perf_counter() - t0:.1f} s")
    m.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
