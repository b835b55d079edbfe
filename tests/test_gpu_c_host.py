"""A compiled C host evaluates through the C ABI on the GPU.

The program is what a C, C++ or Fortran bind(C) caller of the reference does
(api.f90:1038-1111): dftd3_new_structure, dftd3_new_d3_model, a damping
constructor, dftd3_get_dispersion with energy, gradient and sigma, and the
generic delete.  It is compiled against include/s-dftd3.h, linked with the
library, and run on the reference's validation geometries 06 (OLYP-D3(BJ),
gradient and virial) and 07 (M06L-D3(0) with ATM); its printed results are
compared with the values stored in the reference's validation files (abs
1e-6, test/validation/tester.py:61) and with the FP64 oracle (1e-12).
"""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "simple-dftd3_b200" / "lib"
GOLDEN = Path(__file__).resolve().parent / "golden"

PROGRAM = r"""
#include <stdio.h>
#include "s-dftd3.h"

static const int numbers[NAT] = {NUMBERS};
static const double xyz[3 * NAT] = {XYZ};

int main(void)
{
    dftd3_error error = dftd3_new_error();
    dftd3_structure mol = dftd3_new_structure(error, NAT, numbers, xyz, NULL, NULL);
    if (dftd3_check_error(error)) return 2;
    dftd3_model disp = dftd3_new_d3_model(error, mol);
    if (dftd3_check_error(error)) return 3;
    dftd3_param param = CONSTRUCTOR;
    if (dftd3_check_error(error)) return 4;
    double energy = 0.0, gradient[3 * NAT], sigma[9];
    dftd3_get_dispersion(error, mol, disp, param, &energy, gradient, sigma);
    if (dftd3_check_error(error)) {
        char msg[512];
        dftd3_get_error(error, msg, NULL);
        fprintf(stderr, "%s\n", msg);
        return 5;
    }
    printf("%.17g\n", energy);
    for (int k = 0; k < 3 * NAT; k++) printf("%.17g\n", gradient[k]);
    for (int k = 0; k < 9; k++) printf("%.17g\n", sigma[k]);
    dftd3_delete(param);
    dftd3_delete(disp);
    dftd3_delete(mol);
    dftd3_delete(error);
    return 0;
}
"""


def _case(name):
    for c in json.loads((GOLDEN / "validation.json").read_text()):
        if c["name"] == name:
            return c
    raise KeyError(name)


def _program(numbers, xyz, par):
    if par["damping"] == "rational":
        ctor = (f"dftd3_new_rational_damping(error, {par['s6']!r}, {par['s8']!r}, {par['s9']!r}, "
                f"{par['a1']!r}, {par['a2']!r}, {par['alp']!r})")
    else:
        ctor = (f"dftd3_new_zero_damping(error, {par['s6']!r}, {par['s8']!r}, {par['s9']!r}, "
                f"{par['rs6']!r}, {par['rs8']!r}, {par['alp']!r})")
    return (PROGRAM.replace("NAT", str(len(numbers)))
            .replace("NUMBERS", ", ".join(str(int(z)) for z in numbers))
            .replace("XYZ", ", ".join(repr(float(x)) for x in np.ravel(xyz)))
            .replace("CONSTRUCTOR", ctor))


@pytest.mark.parametrize("name", ["06-gradient-d3-bj", "07-gradient-d3-zero"])
def test_c_host_evaluates_validation_set(tmp_path, name):
    import oracle_ref
    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    case = _case(name)
    numbers = np.array(case["numbers"], dtype=np.int32)
    xyz = np.array(case["positions"], dtype=float)
    if case["unit"] == "angstrom":
        xyz = xyz * oracle_ref.AATOAU
    par = case["param"]
    src = tmp_path / "host.c"
    src.write_text(_program(numbers, xyz, par))
    exe = tmp_path / "host"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                    "-L", str(LIB), "-lsdftd3_b200", f"-Wl,-rpath,{LIB}"], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    vals = np.array([float(x) for x in out.stdout.split()])
    nat = len(numbers)
    assert vals.size == 1 + 3 * nat + 9
    energy, gradient, sigma = vals[0], vals[1:1 + 3 * nat].reshape(nat, 3), vals[1 + 3 * nat:].reshape(3, 3)
    # the reference's stored results (tester.py:61)
    assert abs(energy - case["energy"]) <= case["tol_abs"]
    assert np.abs(gradient - np.reshape(case["gradient"], (nat, 3))).max() <= case["tol_abs"]
    assert np.abs(sigma - np.reshape(case["virial"], (3, 3))).max() <= case["tol_abs"]
    # and the FP64 oracle at the parity tolerance
    ref = oracle_ref.dispersion(numbers, xyz, par)
    assert abs(energy - ref["energy"]) <= 1e-12 * abs(ref["energy"])
    assert np.abs(gradient - ref["gradient"]).max() <= 1e-12 * np.abs(ref["gradient"]).max()
    assert np.abs(sigma - ref["virial"]).max() <= 1e-12 * np.abs(ref["virial"]).max()
