"""The relink recipe for reference programs (drop-in use of the library): the
reference's FFTSVDpbeAPI.c compiled with its three drop-in definitions renamed,
linked with the other reference objects and libfftsvd_b200.so, binds
solveSurfaceOperator, generateRHS and collectPotentials to the library, and the
library's references to the reference's process globals (errortolerance,
innerdielectric, addcoulombic) to the program.  The unmodified FFTSVDpbeAPI.o
would keep the reference's own definitions: a definition inside the executable
takes precedence over a shared library's.  CPU only (the program runs no device
code); needs the reference sources and the oracle's objects."""
import glob
import os
import subprocess

import pytest

import ref  # oracle: the reference tree location

from fftsvd_b200.lib import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = ref.REFERENCE_TREE
OBJ32 = os.path.join(ROOT, "oracle", "_ref", "obj32")
DROPIN = ["solveSurfaceOperator", "generateRHS", "collectPotentials"]
GLOBALS = ["errortolerance", "innerdielectric", "addcoulombic"]

MAIN = r"""
#include "FFTSVDpbeAPI.h"
unsigned int num_GMRES_iter;
void* volatile sink[3];
int main(void) {
   sink[0] = (void*)solveSurfaceOperator;
   sink[1] = (void*)generateRHS;
   sink[2] = (void*)collectPotentials;
   return 0;
}
"""


def _cflags():
    return ["-O2", "-w", "-std=gnu99", "-include", "assert.h", "-D_MALLOC", "-DPWD=\"/nonexistent\"",
            "-I" + os.path.join(ROOT, "oracle", "shim"), "-I" + REFERENCE]


@pytest.mark.skipif(not (os.path.isdir(REFERENCE) and os.path.isdir(OBJ32)),
                    reason="reference sources or oracle objects not present")
def test_relinked_reference_program_binds_the_library(tmp_path):
    main_c = tmp_path / "main.c"
    main_c.write_text(MAIN)
    subprocess.run(["gcc", *_cflags(), "-c", str(main_c), "-o", str(tmp_path / "main.o")], check=True)
    renames = [f"-D{name}=reference_{name}" for name in DROPIN]
    api = str(tmp_path / "api_renamed.o")
    subprocess.run(["gcc", *_cflags(), "-fopenmp", "-DOMP", *renames, "-c",
                    os.path.join(REFERENCE, "FFTSVDpbeAPI.c"), "-o", api], check=True)
    objs = [o for o in sorted(glob.glob(os.path.join(OBJ32, "*.o")))
            if os.path.basename(o) not in ("ref_driver.o", "FFTSVDpbeAPI.o")]
    libdir = os.path.dirname(LIB_PATH)
    exe = str(tmp_path / "prog")
    subprocess.run(["gcc", "-o", exe, str(tmp_path / "main.o"), *objs, api, "-L" + libdir, "-lfftsvd_b200",
                    "-Wl,-rpath," + libdir, "-lm", "-fopenmp"], check=True)
    undefined = subprocess.run(["nm", "-u", exe], capture_output=True, text=True, check=True).stdout.split()
    assert all(name in undefined for name in DROPIN)
    env = dict(os.environ, LD_DEBUG="bindings")
    out = subprocess.run([exe], env=env, capture_output=True, text=True, check=True).stderr
    lib = os.path.basename(LIB_PATH)
    for name in DROPIN:
        lines = [l for l in out.splitlines() if f"`{name}'" in l and "binding file" in l]
        assert lines and all(lib in l.split(" to ")[1] for l in lines), name
    for name in GLOBALS:
        lines = [l for l in out.splitlines() if f"`{name}'" in l and "binding file" in l]
        assert lines and all(lib in l.split(" to ")[0] and "prog" in l.split(" to ")[1] for l in lines), name
