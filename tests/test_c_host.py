"""A C and a C++ host compiled against include/s-dftd3.h and
include/dftd3_b200.h and linked with the library, as the integration notes
describe (CPU only: structure, model and parameter handles, the parameter
database, error messages and the generic delete; no evaluation)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "simple-dftd3_b200" / "lib"

PROGRAM = r"""
#include <stdio.h>
#include "s-dftd3.h"
#include "dftd3_b200.h"

int main(void)
{
    dftd3_error error = dftd3_new_error();
    int numbers[3] = {8, 1, 1};
    double xyz[9] = {0.0, 0.0, -0.7, 0.0, 1.4, 0.4, 0.0, -1.4, 0.4};
    dftd3_structure mol = dftd3_new_structure(error, 3, numbers, xyz, NULL, NULL);
    if (dftd3_check_error(error)) return 2;
    dftd3_model disp = dftd3_new_d3_model(error, mol);
    if (dftd3_check_error(error)) return 3;
    char method[] = "pbe0";
    dftd3_param param = dftd3_load_rational_damping(error, method, true);
    if (dftd3_check_error(error)) return 4;
    int kind = -1;
    double v[9];
    dftd3_b200_get_param_values(error, param, &kind, v);
    printf("version %d kind %d s6 %.4f s8 %.4f s9 %.1f a1 %.4f a2 %.4f\n", dftd3_get_version(), kind, v[0], v[1],
           v[2], v[3], v[4]);
    char unknown[] = "no-such-method";
    dftd3_param bad = dftd3_load_rational_damping(error, unknown, false);
    char msg[256];
    int len = 256;
    if (dftd3_check_error(error)) {
        dftd3_get_error(error, msg, &len);
        printf("error: %s\n", msg);
    }
    DELETE_ALL
    printf("deleted %d %d %d %d %d\n", param == NULL, disp == NULL, mol == NULL, error == NULL, bad == NULL);
    return 0;
}
"""

C_DELETE = "dftd3_delete(param); dftd3_delete(disp); dftd3_delete(mol); dftd3_delete(error);"
CXX_DELETE = ("dftd3_delete_param(&param); dftd3_delete_model(&disp); dftd3_delete_structure(&mol); "
              "dftd3_delete_error(&error);")


def _build_and_run(tmp_path, compiler, suffix, delete, std):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    src = tmp_path / f"host.{suffix}"
    src.write_text(PROGRAM.replace("DELETE_ALL", delete))
    exe = tmp_path / f"host_{suffix}"
    subprocess.run([compiler, std, "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                    "-L", str(LIB), "-lsdftd3_b200", f"-Wl,-rpath,{LIB}"], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    return out.stdout


@pytest.mark.parametrize("compiler,suffix,delete,std", [("gcc", "c", C_DELETE, "-std=c11"),
                                                        ("g++", "cpp", CXX_DELETE, "-std=c++17")])
def test_host_program(tmp_path, compiler, suffix, delete, std):
    out = _build_and_run(tmp_path, compiler, suffix, delete, std)
    lines = out.splitlines()
    # PBE0-D3(BJ): s6 = 1, s8 = 1.2177, a1 = 0.4145, a2 = 4.8593; s9 = 1 with ATM
    assert lines[0] == "version 10600 kind 0 s6 1.0000 s8 1.2177 s9 1.0 a1 0.4145 a2 4.8593", lines[0]
    assert lines[1].startswith("error: ") and "no-such-method" in lines[1], lines[1]
    assert lines[2] == "deleted 1 1 1 1 1", lines[2]
