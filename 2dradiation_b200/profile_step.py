"""Drive the step kernel for a profiler: build one problem, then run a few
steps so that the profiler can skip the warm-up launches and capture the rest.

    python 2dradiation_b200/profile_step.py --form fp32 --nx 400 --dirs 64 --fourier 16 --steps 6
    python 2dradiation_b200/profile_step.py --form fp64 --adaptive --steps 4   # adaptive streaming
    python 2dradiation_b200/profile_step.py --batch 16 --steps 4               # batched form
    python 2dradiation_b200/profile_step.py --adjoint --steps 12               # adjoint workload

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
    p.add_argument("--adaptive", action="store_true", help="the adaptive streaming type (plain form)")
    p.add_argument("--batch", type=int, default=0,
                   help="instead: this many uneven problems of the batched form (seed 10)")
    p.add_argument("--adjoint", action="store_true",
                   help="instead: the adjoint workload (256^2 x 48), forward and one backward of --steps steps")
    a = p.parse_args()
    G = importlib.import_module("2dradiation_b200")
    if a.batch:
        probs = [G.prepare(c, G.PRECISION_FP32) for c in G.workloads.batch_instances(count=a.batch, seed=10)]
        with G.Batch(probs) as b:
            for _ in range(a.steps):
                b.step(1)
        print("profile_step: batch of", a.batch, "E sum", float(sum(r.moments_if()["E"].sum() for r in probs)))
        for r in probs:
            r.close()
        return
    if a.adjoint:
        import numpy as np
        r = G.prepare(G.workloads.adjoint_case(steps=a.steps), G.PLAIN_FP64)
        with G.Adjoint(r, 20) as adj:
            r.set_intensity(np.zeros(r.nxy * r.nd))
            adj.forward(a.steps)
            g = adj.backward(r.moments_if()["E"])
        print("profile_step: adjoint", a.steps, "steps, |dL/deta|", float(np.linalg.norm(g["eta"])))
        r.close()
        return
    kw = dict(nx_=a.nx, ny_=a.nx, n_dir=a.dirs, steps=a.steps)
    if a.workload != "flat_beam":
        kw["n_fourier"] = a.fourier
    case = G.workloads.make_case(a.workload, **kw)
    if a.adaptive:
        W = G.workloads
        case["streaming_type"] = W.FLAT_ADAPTIVE if case["streaming_type"] == W.FLAT_FIXED else W.CURVED_ADAPTIVE
    with G.prepare(case, G.PRECISION_FP32 if a.form == "fp32" else G.PLAIN_FP64) as r:
        for _ in range(a.steps):
            r.step(1)
        print("profile_step:", a.form, a.workload, a.nx, a.dirs, "E sum", float(r.moments_if()["E"].sum()))


if __name__ == "__main__":
    main()
