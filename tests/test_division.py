"""The plain FP64 step divides by a per-cell constant through a reciprocal
and a Markstein correction instead of a division per direction (div_rn in
2dradiation_b200/csrc/kernels_plain.cu); the bitwise contract holds only if
that routine returns the IEEE quotient.  Its operations are IEEE multiply,
fma and reciprocal, which the host performs identically, so the check runs
on the CPU over tens of millions of operand pairs, including the step's own
operand range and adversarial mantissas."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_markstein_division_matches_ieee(tmp_path):
    exe = tmp_path / "division_check"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-o", str(exe),
                    str(HERE / "division_check.c"), "-lm"], check=True)
    for seed in (1, 2):
        out = subprocess.run([str(exe), "20000000", str(seed)], check=True, capture_output=True,
                             text=True).stdout.strip().splitlines()
        assert out[-1] == "0", out
