"""Drive the step kernel for a profiler: build one problem, then run a few
steps so that the profiler can skip the warm-up launches and capture the rest.

    python 2dradiation_b200/profile_step.py --form fp32 --nx 400 --dirs 64 --fourier 16 --steps 6

The default problem is the curved-scattering workload at full size (about
250 MB on the device in the FP32 form, 660 MB in FP64), larger than L2.
"""
import argparse
import importlib
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--form", choices=["fp32", "fp64"], default="fp32")
    p.add_argument("--workload", default="curved_scatter")
    p.add_argument("--nx", type=int, default=400)
    p.add_argument("--dirs", type=int, default=64)
    p.add_argument("--fourier", type=int, default=16)
    p.add_argument("--steps", type=int, default=6)
    a = p.parse_args()
    G = importlib.import_module("2dradiation_b200")
    kw = dict(nx_=a.nx, ny_=a.nx, n_dir=a.dirs, steps=a.steps)
    if a.workload != "flat_beam":
        kw["n_fourier"] = a.fourier
    case = G.workloads.make_case(a.workload, **kw)
    with G.prepare(case, G.PRECISION_FP32 if a.form == "fp32" else G.PLAIN_FP64) as r:
        for _ in range(a.steps):
            r.step(1)
        print("profile_step:", a.form, a.workload, a.nx, a.dirs, "E sum", float(r.moments_if()["E"].sum()))


if __name__ == "__main__":
    main()
