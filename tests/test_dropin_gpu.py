"""The drop-in boundary, exercised by the reference's own tests.

oracle/Makefile (`make -C oracle dropin`) builds the reference's
tests/test_factorization.cpp, tests/test_equilibration.cpp,
tests/test_symbolic.cpp and tests/test_assembly.cpp against its kept sources
with src/factorization.cpp and src/assembly.cpp replaced by
hybrid-aphi-solver_b200/dropin/factorization_b200.cpp and
hybrid-aphi-solver_b200/dropin/assembly_b200.cpp, which define every function
of include/aphi_solver/factorization.hpp and include/aphi_solver/assembly.hpp
over the aphi_b200 C ABI (the element fill and scatter of refill and the
factorization, solves and refinement run on the device). Each program prints "<passed>/<checks> checks passed" and
exits 0 only if every check passed; here they run on the B200."""
import re
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "oracle" / "_ref" / "dropin"


@pytest.mark.parametrize("name", ["test_factorization", "test_equilibration", "test_symbolic", "test_assembly"])
def test_reference_tests_pass_through_the_dropin(name, cuda):
    exe = DROPIN / name
    if not exe.exists():
        pytest.skip(f"{exe} not built (make -C oracle dropin needs the reference tree at build time)")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    m = re.search(r"(\d+)/(\d+) checks passed", r.stdout)
    assert m, (r.stdout[-2000:], r.stderr[-2000:])
    assert r.returncode == 0 and m.group(1) == m.group(2), (r.stdout[-3000:], r.stderr[-3000:])
    assert int(m.group(2)) > 0
    # the program used this repository's library
    maps = subprocess.run(["ldd", str(exe)], capture_output=True, text=True).stdout
    assert "libaphi_b200.so" in maps
