"""The drop-in entry points read a caller's reference-built structures through
the mirrors in fftsvd_b200/csrc/refabi.h.  This compares, field by field, the
offsets and sizes of those mirrors with the reference's own declarations
(Vector3D.h, Panel.h, FlatPanel.h, Charge.h, Tree.h, Cube.h, SurfaceOperator.h,
Preconditioner.h, FFTSVDpbeAPI.h:23-42), compiled with the configuration the
oracle builds the reference in.  CPU only; needs the reference sources."""
import os
import subprocess

import pytest

import ref  # oracle: the reference tree location

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = ref.REFERENCE_TREE

# (reference type, mirror type, fields, compare sizeof)
STRUCTS = [
    ("_Vector3D", "Vec3", ["x", "y", "z"], True),
    ("_Panel", "Panel", ["centroid", "normal", "area", "maxedgelength", "numdirectquadpoints", "directquadpoints",
                         "directquadnormals", "directquadweights", "type", "realpanel"], True),
    ("_FlatPanel", "FlatPanel", ["vertex"], False),
    ("_Charge", "Charge", ["numcharges", "globalindexstart", "points", "charges"], True),
    ("_Tree", "Tree", ["panels", "numpanels", "points", "normals", "numpoints", "maxpanelsperfinestcube",
                       "partitioningdepth", "kerneltype", "parameters", "gridpoints", "gridpointsperlevel",
                       "quadraturepoints", "numquadraturepoints", "pinv_Q2Sgridpoints", "epsilon", "layertype",
                       "Tprecomputed", "root", "minimumcubesize"], True),
    ("_Cube", "Cube", ["level", "indices", "bounds", "center", "parent", "leaf", "panelindices", "numpanelindices",
                       "pointindices", "numpointindices", "localcubes", "numlocalcubes", "interactingcubes",
                       "numinteractingcubes", "children", "drows", "dcolumns", "rowrank", "columnrank", "VTsrc",
                       "Udest", "D_single", "D_double", "FFT_PV_VT_q", "sum_T_FFT_PV_VT_q", "FFT_UTIT_UT_q",
                       "sum_T_FFT_UTIT_UT_q", "UTI", "PV_single", "PV_double", "P_single", "P_double", "I_",
                       "I_double", "tree"], True),
    ("_SurfaceOperator", "SurfaceOperator", ["kernel", "epsilon", "kappa", "mynumpanels", "startphi", "startdphi",
                                             "tree", "M3", "numchildren", "children", "resultInternal",
                                             "resultExternal", "parent", "charges"], True),
    ("PreconditionerElement", "PreconditionerElement", ["row", "value"], True),
    ("_Preconditioner", "Preconditioner", ["rows", "columns", "nnz", "P", "numelements"], False),
    ("PDBentry", "PDBentry", ["record", "atomnumber", "atomname", "alternatelocation", "residuename", "chain",
                              "residuenumber", "residueinsertion", "x", "y", "z", "occupancy", "temperature",
                              "footnotenumber", "radius", "charge", "potential"], True),
]


def _program(prefix: str) -> str:
    lines = []
    for ref_t, mirror_t, fields, size in STRUCTS:
        t = ref_t if prefix == "" else prefix + mirror_t
        key = mirror_t
        for f in fields:
            lines.append(f'   printf("{key}.{f} %zu %zu\\n", offsetof({t}, {f}), sizeof((({t}*)0)->{f}));')
        if size:
            lines.append(f'   printf("{key} sizeof %zu\\n", sizeof({t}));')
    return "\n".join(lines)


def _run(cmd, src, tmp_path, name):
    path = tmp_path / name
    path.write_text(src)
    exe = tmp_path / (name + ".bin")
    subprocess.run(cmd + [str(path), "-o", str(exe)], check=True, capture_output=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="reference sources not present")
def test_refabi_mirrors_match_reference_layout(tmp_path):
    ref_src = ("#include <stddef.h>\n#include <stdio.h>\n#include \"FFTSVDpbeAPI.h\"\nint main(void) {\n"
               + _program("") + "\n   return 0;\n}\n")
    ref_cmd = ["gcc", "-std=gnu99", "-w", "-include", "assert.h", "-D_MALLOC", "-DPWD=\"/nonexistent\"",
               "-I" + os.path.join(ROOT, "oracle", "shim"), "-I" + REFERENCE]
    mirror_src = ("#include <cstddef>\n#include <cstdio>\n#include \"refabi.h\"\nint main() {\n"
                  + _program("fftsvd::ref::") + "\n   return 0;\n}\n")
    mirror_cmd = ["g++", "-std=c++17", "-Wno-invalid-offsetof", "-I" + os.path.join(ROOT, "fftsvd_b200", "csrc")]
    ref_lines = _run(ref_cmd, ref_src, tmp_path, "ref_layout.c")
    mirror_lines = _run(mirror_cmd, mirror_src, tmp_path, "mirror_layout.cc")
    assert len(ref_lines) == len(mirror_lines) > 100
    diff = [(a, b) for a, b in zip(ref_lines, mirror_lines) if a != b]
    assert not diff, diff


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="reference sources not present")
def test_public_header_compiles_after_the_reference_api_header(tmp_path):
    """A C file of the reference side (the oracle driver is one) may include the
    reference's FFTSVDpbeAPI.h and then this library's header."""
    src = tmp_path / "both.c"
    src.write_text('#include "FFTSVDpbeAPI.h"\n#include "fftsvd_b200.h"\nint main(void) { return 0; }\n')
    subprocess.run(["gcc", "-std=gnu99", "-fsyntax-only", "-Werror", "-include", "assert.h", "-D_MALLOC",
                    "-DPWD=\"/nonexistent\"", "-I" + os.path.join(ROOT, "oracle", "shim"), "-I" + REFERENCE,
                    "-I" + os.path.join(ROOT, "include"), str(src)], check=True, capture_output=True)
