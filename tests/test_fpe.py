"""No invalid operation, division by zero or overflow on the test inputs: the
oracle and the kernels' own column and point code (host builds) run with
those floating-point exceptions trapping, the analogue of the reference's
debug build (-ffpe-trap=invalid,zero,overflow, ifs-source/cmake/
compile_flags.cmake:359-393).  Each case runs in a child process on one
thread; a trap ends the child with SIGFPE."""
import os
import subprocess
import sys

import pytest

from tests import util

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, sys
import numpy as np
from openifs_b200 import inputs
from tests import util
kind, case = sys.argv[1], sys.argv[2]
p, po = util.params()
arrs = inputs.generate(24, 32, p, seed=4)
if case != "default":
    arrs = util.apply_case(arrs, case)
ngptot = 24 * 32 - 5
if kind.startswith("satadj") or kind.startswith("sltend"):
    sat = inputs.generate_satadj(24, 32, p, seed=4) if kind.startswith("satadj") else \
        inputs.generate_sltend(24, 32, p, seed=4)
if kind.startswith("diag"):
    q = util.opt_params(p, "all+budgets")
    qo = util.opt_params(po, "all+budgets")
    from openifs_b200 import fields
    diag = inputs.generate_diag(arrs, 32, fields.budget_fields_needed(q), seed=4)
libm = ctypes.CDLL("libm.so.6")
libm.feenableexcept(0x01 | 0x04 | 0x08)  # FE_INVALID | FE_DIVBYZERO | FE_OVERFLOW
if kind in ("oracle_glibc", "oracle_plibm"):
    util.run_oracle(po, arrs, 32, 24, ngptot, nthreads=1, libm=kind.split("_")[1])
elif kind in ("kernel_fp64", "kernel_mixed"):
    util.run_hostemu(p, arrs, 32, 24, ngptot, precision=0 if kind == "kernel_fp64" else 1)
elif kind == "satadj_oracle":
    util.run_oracle_satadj(po, sat, 32, 24, ngptot)
elif kind == "satadj_kernel":
    util.run_hostemu_satadj(p, sat, 32, 24, ngptot)
elif kind == "sltend_oracle":
    util.run_oracle_sltend(po, sat, 32, 24, ngptot)
elif kind == "sltend_kernel":
    util.run_hostemu_sltend(p, sat, 32, 24, ngptot)
elif kind == "diag_oracle":
    util.run_oracle_diag(qo, arrs, diag, 32, 24, ngptot)
elif kind == "diag_kernel":
    util.run_hostemu_diag(q, arrs, diag, 32, 24, ngptot)
libm.fedisableexcept(0x01 | 0x04 | 0x08)
print("ok")
"""

KINDS = ["oracle_glibc", "oracle_plibm", "kernel_fp64", "kernel_mixed", "satadj_oracle", "satadj_kernel",
         "sltend_oracle", "sltend_kernel", "diag_oracle", "diag_kernel"]


def _run(kind, case):
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""),
               OMP_NUM_THREADS="1")
    r = subprocess.run([sys.executable, "-c", CHILD, kind, case], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), (
        f"{kind}/{case}: exit {r.returncode} (SIGFPE is -8)\n{r.stderr[-2000:]}")


@pytest.mark.parametrize("kind", KINDS)
def test_no_fp_exceptions(built, kind):
    _run(kind, "default")


@pytest.mark.parametrize("case", util.EDGE_CASES)
def test_no_fp_exceptions_edge_cases(built, case):
    _run("oracle_glibc", case)
    _run("kernel_fp64", case)
