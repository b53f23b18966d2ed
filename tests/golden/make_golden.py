"""Generate the golden vectors in this directory from the reference itself.

Runs each case of cases.py through the reference compiled from its own
sources (oracle/Makefile target `ref`, which needs the reference tree at
/root/reference) and stores inputs and outputs as compressed .npz files:
  ref_strict_*  the reference built with IEEE semantics (no -ffast-math);
                the oracle restatement must reproduce these bit for bit;
  ref_fast_*    the reference built with its own flags (-O3 -ffast-math);
                kept to document how far its fast-math build drifts.
Usage:  python tests/golden/make_golden.py
"""
import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE))

import oracle as O  # noqa: E402
from cases import golden_cases  # noqa: E402

W = importlib.import_module("2dradiation_b200.workloads")
# metric arrays are stored for one case per metric class (they are large)
METRIC_PINS = ("curved_shell", "moving_schwarzschild", "moving_flat")
KEYS = ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy", "E_LF", "Fx_LF", "Fy_LF", "Pxx_LF", "Pxy_LF", "Pyy_LF",
        "F_LF", "I", "coefS", "coefX", "coefY", "coefCx", "coefCy", "st_w", "st_phi", "st_cx", "st_cy",
        "ig_index", "ig_weight", "ss_phi", "ss_w")


def main():
    O.build(with_reference=True)
    for name, case in golden_cases(W).items():
        strict = O.run(case, "ref_strict", want_metric=True)
        fast = O.run(case, "ref_fast")
        out = {}
        for k in KEYS:
            out["ref_strict_" + k] = strict[k]
        for k in ("E", "Fx", "Fy", "I"):
            out["ref_fast_" + k] = fast[k]
        if name in METRIC_PINS:
            out["ref_strict_metric_arrays"] = strict["metric_arrays"]
        out["ref_strict_max_iterations"] = np.array(strict["max_iterations"])
        out["ref_strict_average_iterations"] = np.array(strict["average_iterations"])
        for k, v in case["fields"].items():
            out["field_" + k] = v
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, "written", {k: v.shape for k, v in list(out.items())[:3]})


if __name__ == "__main__":
    main()
