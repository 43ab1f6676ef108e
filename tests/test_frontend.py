"""Input front end (fftsvd_b200.frontend) against the reference's own readers.

The reference's readers (FFTSVDpbeAPI.c, VertFace.c, compiled unchanged into the oracle)
parse the same synthetic files; every field must agree exactly. The files are written here:
made-up atoms, radius and charge tables, and icosphere meshes in the vert/face layout, with
the edge cases the readers handle (lower-case records, a truncated record that reads stale
buffer bytes, comment lines, zero-area and non-cap faces, cavities read without the flip)."""
import ctypes as C
import os
import warnings

import numpy as np
import pytest

import ref  # oracle
from fftsvd_b200 import frontend as F
from fftsvd_b200 import meshes

pytestmark = pytest.mark.skipif(not ref.available(False), reason="oracle/_ref is not built")


class CPDB(C.Structure):
    _fields_ = [("record", C.c_char * 7), ("atomnumber", C.c_uint), ("atomname", C.c_char * 5),
                ("alternatelocation", C.c_char), ("residuename", C.c_char * 4), ("chain", C.c_char),
                ("residuenumber", C.c_uint), ("residueinsertion", C.c_char), ("x", C.c_double), ("y", C.c_double),
                ("z", C.c_double), ("occupancy", C.c_double), ("temperature", C.c_double),
                ("footnotenumber", C.c_uint), ("radius", C.c_double), ("charge", C.c_double),
                ("potential", C.c_double)]


class CSIZ(C.Structure):
    _fields_ = [("atomlabel", C.c_char * 7), ("residuelabel", C.c_char * 4), ("radius", C.c_double)]


class CCRG(C.Structure):
    _fields_ = [("atomlabel", C.c_char * 7), ("residuelabel", C.c_char * 4), ("residuenumber", C.c_uint),
                ("chain", C.c_char), ("charge", C.c_double)]


@pytest.fixture(scope="module")
def lib():
    L = ref._lib(False)
    L.readPDB.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.POINTER(CPDB))]
    L.readSIZ.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.POINTER(CSIZ))]
    L.readCRG.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.POINTER(CCRG))]
    L.assignRadiiCharges.argtypes = [C.POINTER(CPDB), C.c_uint, C.POINTER(CSIZ), C.c_uint, C.POINTER(CCRG), C.c_uint]
    L.readParams.argtypes = [C.c_char_p]
    L.oref_flat_panels.restype = C.c_uint
    L.oref_flat_panels.argtypes = [C.c_char_p, C.c_uint, C.c_uint, C.c_uint, C.POINTER(C.c_double), C.c_uint]
    L.oref_read_srf.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.c_uint,
                                C.POINTER(C.c_double), C.c_uint]
    return L


def _ch(b: bytes) -> str:
    return "" if b in (b"", b"\x00") else b.decode("latin-1")


def _pdb_line(rec, serial, name, alt, res, chain, resseq, icode, x, y, z, occ, temp):
    s = f"{rec:<6}{serial:5d} {name:<4}{alt:1}{res:>3} {chain:1}{resseq:4d}{icode:1}   {x:8.3f}{y:8.3f}{z:8.3f}" \
        f"{occ:6.2f}{temp:6.2f}"
    return s.ljust(80) + "\n"


def _write_molecule(d):
    pdb = os.path.join(d, "mol.pdb")
    lines = ["REMARK synthetic molecule for the reader tests\n",
             _pdb_line("ATOM", 1, " N", "", "ALA", "A", 1, "", 1.25, -2.5, 3.125, 1.0, 10.5),
             _pdb_line("ATOM", 2, " CA", "B", "ALA", "A", 1, "", 2.0, -1.75, 3.5, 0.5, 11.0),
             _pdb_line("ATOM", 3, " C", "", "ALA", "A", 1, "", 3.5, -1.0, 3.0, 1.0, 12.25),
             _pdb_line("ATOM", 4, " O", "", "ALA", "A", 1, "", 4.0, -0.25, 2.5, 1.0, 13.0),
             _pdb_line("atom", 5, " CB", "", "GLY", "C", 7, "X", -3.0, 0.5, 1.0, 1.0, 9.0),
             "ATOM      7  H   ALA A   2\n",  # truncated: later columns are whatever the buffer holds
             _pdb_line("HETATM", 6, "NA", "", "ION", "B", 2, "", 0.0, 0.0, 0.0, 1.0, 20.0),
             "TER\n",
             _pdb_line("ATOM", 8, " OXT", "", "ALA", " ", 1, "", -1.5, 2.25, -0.5, 1.0, 8.0),
             "END\n"]
    with open(pdb, "w") as f:
        f.writelines(lines)
    siz = os.path.join(d, "radii.siz")
    with open(siz, "w") as f:
        f.write("atom__res_radius_\n")
        f.write("! element defaults\n")
        for atom, res, r in [("N", "", 1.65), ("C", "", 1.76), ("O", "", 1.40), ("H", "", 1.0), ("CA", "ALA", 1.87),
                             ("NA", "ION", 1.2)]:
            f.write(f"{atom:<6}{res:<3}{r:8.3f}\n")
    crg = os.path.join(d, "charges.crg")
    with open(crg, "w") as f:
        f.write("atom__resnumbc_charge_\n")
        f.write("! comment\n")
        for atom, res, num, chain, q in [("N", "ALA", "   1", "A", -0.3), ("CA", "ALA", "    ", " ", 0.1),
                                         ("C", "ALA", "   1", " ", 0.55), ("O", "", "    ", " ", -0.5),
                                         ("NA", "ION", "   2", "B", 1.0), ("CB", "", "   7", "C", -0.05),
                                         ("OXT", "ALA", "    ", " ", -0.8)]:
            f.write(f"{atom:<6}{res:<3}{num:>4}{chain:1}{q:8.3f}\n")
    return pdb, siz, crg


def _ref_pdb(lib, path):
    n = C.c_uint()
    p = C.POINTER(CPDB)()
    with ref.stdout_to_stderr():
        lib.readPDB(path.encode(), C.byref(n), C.byref(p))
    return n.value, p


def test_pdb_siz_crg_and_assignment_match_the_reference(lib, tmp_path):
    pdb, siz, crg = _write_molecule(str(tmp_path))
    n, rp = _ref_pdb(lib, pdb)
    ours = F.readPDB(pdb)
    assert len(ours) == n == 8
    for i, e in enumerate(ours):
        r = rp[i]
        assert e.record == r.record.decode() and e.atomnumber == r.atomnumber, i
        assert e.atomname == r.atomname.decode() and e.residuename == r.residuename.decode(), i
        assert (e.alternatelocation, e.chain, e.residueinsertion) == (
            _ch(r.alternatelocation), _ch(r.chain), _ch(r.residueinsertion)), i
        assert e.residuenumber == r.residuenumber and e.footnotenumber == r.footnotenumber, i
        assert (e.x, e.y, e.z, e.occupancy, e.temperature) == (r.x, r.y, r.z, r.occupancy, r.temperature), i
    # the truncated record takes its coordinates from the bytes the previous record left
    assert ours[5].atomname == "H" and (ours[5].x, ours[5].y, ours[5].z) == (-3.0, 0.5, 1.0)

    ns, sp = C.c_uint(), C.POINTER(CSIZ)()
    nc, cp = C.c_uint(), C.POINTER(CCRG)()
    with ref.stdout_to_stderr():
        lib.readSIZ(siz.encode(), C.byref(ns), C.byref(sp))
        lib.readCRG(crg.encode(), C.byref(nc), C.byref(cp))
    S, Q = F.readSIZ(siz), F.readCRG(crg)
    assert len(S) == ns.value == 6 and len(Q) == nc.value == 7
    for i, s in enumerate(S):
        assert (s.atomlabel, s.residuelabel, s.radius) == (sp[i].atomlabel.decode(), sp[i].residuelabel.decode(),
                                                           sp[i].radius), i
    for i, c in enumerate(Q):
        assert (c.atomlabel, c.residuelabel, c.residuenumber, c.chain, c.charge) == (
            cp[i].atomlabel.decode(), cp[i].residuelabel.decode(), cp[i].residuenumber, _ch(cp[i].chain),
            cp[i].charge), i

    with ref.stdout_to_stderr():
        lib.assignRadiiCharges(rp, n, sp, ns, cp, nc)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        F.assignRadiiCharges(ours, S, Q)
    for i, e in enumerate(ours):
        assert (e.radius, e.charge) == (rp[i].radius, rp[i].charge), (i, e.atomname)
    assert ours[1].radius == 1.87 and ours[6].charge == 1.0  # full matches
    assert ours[4].radius == 1.76  # atom-name prefix "C" of CB


def test_first_record_reads_the_counting_pass_leftovers(lib, tmp_path):
    """readPDB counts records, rewinds and reads again through the same buffer: a truncated
    first record takes its missing columns from the file's last full line."""
    path = str(tmp_path / "short.pdb")
    with open(path, "w") as f:
        f.write("HETATM    1 CL   ION X   9\n")
        f.write(_pdb_line("ATOM", 2, " N", "", "GLY", "A", 3, "", 7.5, -8.25, 9.0, 1.0, 4.5))
    n, rp = _ref_pdb(lib, path)
    ours = F.readPDB(path)
    assert n == len(ours) == 2
    for i, e in enumerate(ours):
        assert (e.atomname, e.x, e.y, e.z, e.temperature) == (rp[i].atomname.decode(), rp[i].x, rp[i].y, rp[i].z,
                                                             rp[i].temperature), i
    assert (ours[0].x, ours[0].y, ours[0].z) == (7.5, -8.25, 9.0)


def test_crd_xyzr_and_modpdb_match_the_reference(lib, tmp_path):
    crd = str(tmp_path / "mol.crd")
    with open(crd, "w") as f:
        f.write("* synthetic coordinates\n*\n    3\n")
        for num, resn, res, atom, x, y, z, seg, temp in [(1, 1, "ALA", "N", 1.5, -2.0, 0.25, "PROA", 0.0),
                                                         (2, 1, "ALA", "CA", 2.5, -1.0, 0.75, "PROA", 1.5),
                                                         (3, 2, "GLY", "O", -0.5, 3.0, -1.25, "PROB", 2.0)]:
            f.write(f"{num:5d}{resn:5d} {res:<4} {atom:<4}{x:10.5f}{y:10.5f}{z:10.5f} {seg:<4} {resn:<4} {temp:10.5f}\n")
    xyzr = str(tmp_path / "mol.xyzr")
    with open(xyzr, "w") as f:
        f.write("1.0 2.0 3.0 1.5\n-4.25 0.5e1 6 2\n7.5 8.5\n")
    lib.readCRD.argtypes = lib.readXYZR.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.POINTER(CPDB))]
    lib.writeMODPDB.argtypes = [C.c_char_p, C.POINTER(CPDB), C.c_uint]
    for reader, ours in ((lib.readCRD, F.readCRD(crd)), (lib.readXYZR, F.readXYZR(xyzr))):
        n, p = C.c_uint(), C.POINTER(CPDB)()
        with ref.stdout_to_stderr():
            reader((crd if reader is lib.readCRD else xyzr).encode(), C.byref(n), C.byref(p))
        assert n.value == len(ours)
        for i, e in enumerate(ours):
            r = p[i]
            assert (e.atomnumber, e.residuenumber, e.residuename, e.atomname, e.chain) == (
                r.atomnumber, r.residuenumber, r.residuename.decode(), r.atomname.decode(), _ch(r.chain)), i
            assert (e.x, e.y, e.z, e.temperature, e.radius) == (r.x, r.y, r.z, r.temperature, r.radius), i
    pdb, siz, crg = _write_molecule(str(tmp_path))
    n, rp = _ref_pdb(lib, pdb)
    ours = F.readPDB(pdb)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        F.assignRadiiCharges(ours, F.readSIZ(siz), F.readCRG(crg))
    for i, e in enumerate(ours):
        rp[i].radius, rp[i].charge = e.radius, e.charge
    out_ref, out_ours = str(tmp_path / "ref.pdb"), str(tmp_path / "ours.pdb")
    with ref.stdout_to_stderr():
        lib.writeMODPDB(out_ref.encode(), rp, n)
    F.writeMODPDB(out_ours, ours)
    with open(out_ref, "rb") as a, open(out_ours, "rb") as b:
        assert a.read() == b.read()
    # site potentials: the FRC writer with the reference's parameter globals
    params = F.Params(innerdielectric=4.0, outerdielectric=80.0, ionicstrength=0.145, ionexclusionradius=2.0,
                      proberadius=1.4)
    for nm in ("innerdielectric", "outerdielectric", "ionicstrength", "ionexclusionradius", "proberadius"):
        C.c_double.in_dll(lib, nm).value = getattr(params, nm)
    for i, e in enumerate(ours):
        e.potential = rp[i].potential = 0.125 * (i + 1) - 0.3
    lib.writeFRC.argtypes = [C.c_char_p, C.POINTER(CPDB), C.c_uint]
    with ref.stdout_to_stderr():
        lib.writeFRC(out_ref.encode(), rp, n)
    F.writeFRC(out_ours, ours, params)
    with open(out_ref, "rb") as a, open(out_ours, "rb") as b:
        assert a.read() == b.read()


def test_params_match_the_reference(lib, tmp_path):
    path = str(tmp_path / "param.prm")
    with open(path, "w") as f:
        f.write("INDI=4.0\nexdi = 80.0\nSALT=0.145\nIONRAD=0\nPRBRAD=1.4\nDE=1e-6\nENERGY(g)\nOUT(MODPDB)\n"
                "OUT(phi)\nADDCOUL=yes\nDVERT=2.5\nSVERT=1.5\nCURVED=no\n")
    names = ["innerdielectric", "outerdielectric", "ionicstrength", "ionexclusionradius", "proberadius",
             "errortolerance", "dielectricvertexdensity", "saltvertexdensity"]
    for nm in names:
        C.c_double.in_dll(lib, nm).value = 0.0
    for nm in ("outputmodpdb", "addcoulombic", "usecurved"):
        C.c_uint.in_dll(lib, nm).value = 0
    with ref.stdout_to_stderr():
        lib.readParams(path.encode())
    p = F.readParams(path)
    for nm in names:
        assert getattr(p, nm) == C.c_double.in_dll(lib, nm).value, nm
    assert p.energycalculation == C.c_char.in_dll(lib, "energycalculation").value.decode() == "G"
    assert p.outputmodpdb == C.c_uint.in_dll(lib, "outputmodpdb").value == 1
    assert p.addcoulombic == C.c_uint.in_dll(lib, "addcoulombic").value == 1
    assert p.usecurved == C.c_uint.in_dll(lib, "usecurved").value == 0
    F.checkParams(p)
    assert abs(p.kappa - np.sqrt(0.145) / 3.047) < 1e-15


def test_param_errors_raise(tmp_path):
    path = str(tmp_path / "bad.prm")
    with open(path, "w") as f:
        f.write("INDI=4\nEXDI=80\nDE=1e-6\nENERGY(G)\nSALT=-1\n")
    with pytest.raises(F.FrontEndError):
        F.checkParams(F.readParams(path))
    with open(path, "w") as f:
        f.write("ADDCOUL=maybe\n")
    with pytest.raises(F.FrontEndError):
        F.readParams(path)
    with pytest.raises(F.FrontEndError):
        F.readPDB(str(tmp_path / "missing.pdb"))


def _mesh_files(d, name, level=2, radius=10.0, extra_degenerate=True, genus_mod=None):
    v, f = meshes.icosphere_mesh(level, radius)
    genus = np.ones(len(f), dtype=np.int64)
    if genus_mod:
        genus[::genus_mod] = 2  # non-cap faces, dropped from accessible surfaces
    if extra_degenerate:  # zero-area faces, dropped everywhere
        f = np.concatenate([f, [[0, 0, 1], [3, 5, 3]]])
        genus = np.concatenate([genus, [1, 1]])
    base = os.path.join(d, name)
    F.write_vert_face(base, v, f, genus)
    return base, v, f


@pytest.mark.parametrize("accessible,cavity,genus_mod", [(0, 0, None), (1, 0, 3), (0, 1, None), (1, 1, 4)])
def test_flat_panels_match_the_reference(lib, tmp_path, accessible, cavity, genus_mod):
    base, v, f = _mesh_files(str(tmp_path), "surf", genus_mod=genus_mod)
    ours = F.getFlatPanels(base, accessible, cavity)
    out = np.zeros((len(f), 9))
    with ref.stdout_to_stderr():
        n = lib.oref_flat_panels(base.encode(), accessible, cavity, 0, out.ctypes.data_as(C.POINTER(C.c_double)),
                                 len(f))
    assert ours.shape == (n, 9)
    assert np.array_equal(ours, out[:n])
    if not accessible and not cavity:  # written flipped, read flipped: the icosphere's own corner order
        assert np.array_equal(ours, meshes.icosphere(2, 10.0))


def test_srf_matches_the_reference(lib, tmp_path):
    d = str(tmp_path)
    _mesh_files(d, "diel", level=2, radius=10.0)
    _mesh_files(d, "salt", level=1, radius=14.0, genus_mod=5)
    _mesh_files(d, "cav", level=1, radius=3.0, extra_degenerate=False)
    srf = os.path.join(d, "operator.srf")
    with open(srf, "w") as f:
        f.write("f\nf\nsalt\ndiel\ncav\n\n0\n0\n\n")
    s = F.readSRF(srf)
    counts = (C.c_uint * 5)()
    layer_n = (C.c_uint * 8)()
    parents = (C.c_uint * 8)()
    out = np.zeros((4000, 9))
    with ref.stdout_to_stderr():
        lib.oref_read_srf(srf.encode(), counts, layer_n, parents, 8, out.ctypes.data_as(C.POINTER(C.c_double)), 4000)
    assert (len(s.salts), len(s.dielectrics), len(s.dielectriccavities), len(s.saltcavities), s.numtotalpanels) == \
        tuple(counts)
    ours = s.salts + s.dielectrics + s.dielectriccavities + s.saltcavities
    assert [len(p) for p in ours] == list(layer_n[:len(ours)])
    assert np.array_equal(np.concatenate(ours), out[:sum(len(p) for p in ours)])
    assert s.dielectricparent + s.dielectriccavityparent + s.saltcavityparent == list(parents[:2])


def _born_inputs(d, salt=0.0):
    _mesh_files(d, "sphere", level=3, radius=10.0, extra_degenerate=False)
    with open(os.path.join(d, "operator.srf"), "w") as f:
        f.write("f\nf\n\nsphere\n\n\n0\n\n\n")
    with open(os.path.join(d, "p.prm"), "w") as f:
        f.write(f"INDI=1\nEXDI=80\nSALT={salt}\nDE=1e-6\nENERGY(G)\n")
    with open(os.path.join(d, "ion.pdb"), "w") as f:
        f.write(_pdb_line("HETATM", 1, "NA", "", "ION", "A", 1, "", 0.0, 0.0, 0.0, 1.0, 0.0))
    with open(os.path.join(d, "r.siz"), "w") as f:
        f.write(f"header\n{'NA':<6}{'ION':<3}{1.2:8.3f}\n")
    with open(os.path.join(d, "c.crg"), "w") as f:
        f.write(f"header\n{'NA':<6}{'ION':<3}{1:4d}A{1.0:8.3f}\n")
    return [os.path.join(d, n) for n in ("p.prm", "ion.pdb", "r.siz", "c.crg", "operator.srf")]


def test_born_ion_from_files_through_the_reference_solve(tmp_path):
    """The whole input sequence on a Born ion: files -> system -> the reference's own CPU
    solve, against the analytic Born energy."""
    sysm = F.pbe_system(*_born_inputs(str(tmp_path)))
    assert sysm.panels.shape == (1280, 9) and sysm.charge.tolist() == [1.0]
    rs = ref.RefSystem(sysm.panels, sysm.charge_pos, sysm.charge, sysm.params.innerdielectric,
                       sysm.params.outerdielectric, sysm.kappa, svd_tol=1e-4)
    with ref.stdout_to_stderr():
        sol, _ = rs.solve(rs.rhs(), sysm.params.errortolerance)
        e = rs.energy(rs.reaction(sol))
    rs.close()
    born = -332.112 / (2 * 10.0) * (1 - 1 / 80.0)
    assert abs(e - born) < 1e-2 * abs(born), (e, born)


def test_unsupported_topologies_raise(tmp_path):
    d = str(tmp_path)
    paths = _born_inputs(d)
    with open(paths[0], "w") as f:
        f.write("INDI=1\nEXDI=80\nSALT=0.1\nIONRAD=2.0\nDE=1e-6\nENERGY(G)\n")
    with pytest.raises(F.FrontEndError, match="Stern"):
        F.pbe_system(*paths)


@pytest.mark.gpu
def test_born_ion_from_files_on_the_gpu(gpu, tmp_path):
    """The same inputs through the library's own setup and GPU solve."""
    from fftsvd_b200.surface import Surface
    sysm = F.pbe_system(*_born_inputs(str(tmp_path)))
    s = Surface.from_problem(sysm.panels, sysm.charge_pos, sysm.charge, sysm.params.innerdielectric,
                             sysm.params.outerdielectric, sysm.kappa, svd_tol=1e-4)
    r = s.solve(s.rhs(), precision="mixed", tol=sysm.params.errortolerance)
    e = s.energy(s.reaction_potentials(r.solution))
    born = -332.112 / (2 * 10.0) * (1 - 1 / 80.0)
    assert abs(e - born) < 1e-2 * abs(born), (e, born)
