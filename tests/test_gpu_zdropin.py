"""The drop-in entry points on operators built by the reference's
generateSurfaceOperator: collectPotentials (FFTSVDpbeAPI.c:1896-1922) against
the reference's own collectPotentials on the same solution, and the operator
cache of solveSurfaceOperator when a second operator is passed.

Tolerance: the reaction potentials are the same FP64 panel integrals summed in
another order (the library's reaction-potential test holds them to 1e-11), and
the Coulomb sum is the same FP64 arithmetic, so the collected potentials agree
to 1e-11 relative.

The GPU tests of this file call ref.export_api_globals(), which makes the
compiled reference's process globals visible to the library for the rest of the
process; the file is collected after the other GPU test files."""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F
import ref
from helpers import make_case, rel


def _lib():
    lib = F.load()
    lib.collectPotentials.restype = None
    lib.collectPotentials.argtypes = [C.c_void_p, C.c_uint, C.c_void_p, C.c_uint, C.c_void_p,
                                      C.POINTER(C.c_double)]
    return lib


def _collect(lib, rs, collect, inputs, sol):
    sol = np.ascontiguousarray(sol, dtype=np.float64)
    lib.collectPotentials(C.cast(collect, C.c_void_p), len(collect), C.cast(inputs, C.c_void_p), len(inputs),
                          C.c_void_p(rs.surface_operator), sol.ctypes.data_as(C.POINTER(C.c_double)))


def _potentials(entries):
    return np.array([e.potential for e in entries])


@pytest.fixture(scope="module")
def api_case():
    tri, qpos, q, c = make_case("blob3")
    with ref.stdout_to_stderr():
        rs = ref.RefSystem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], via_api=True, gmres_tol=1e-6)
    sol = np.random.default_rng(21).standard_normal(2 * len(tri))
    # the charges, then three extra collection points inside the surface
    extra = qpos[:3] * 0.5
    collect_pos = np.vstack([qpos, extra])
    chains = [b"A", b"X", b"B", b"x", b"A"] * (len(q) // 5) + [b"A"] * (len(q) % 5)
    return rs, c, tri, qpos, q, sol, collect_pos, chains


def test_collect_rejects_bad_calls_and_leaves_entries(api_case):
    """Errors are reported and change no entry (the reference would write past
    a collect array shorter than its charges, or exit)."""
    rs, c, tri, qpos, q, sol, collect_pos, chains = api_case
    lib = _lib()
    short = ref.pdb_entries(qpos[:5], potential=7.0)
    inputs = ref.pdb_entries(qpos, q)
    _collect(lib, rs, short, inputs, sol)
    assert np.all(_potentials(short) == 7.0)
    assert b"beyond the collected entries" in lib.fftsvd_b200_last_error()
    full = ref.pdb_entries(collect_pos, potential=7.0)
    lib.collectPotentials(C.cast(full, C.c_void_p), len(full), C.cast(inputs, C.c_void_p), len(inputs),
                          C.c_void_p(rs.surface_operator), None)
    assert np.all(_potentials(full) == 7.0)
    assert b"null argument" in lib.fftsvd_b200_last_error()


def test_collect_reads_the_reference_globals(api_case):
    """innerdielectric is taken from the reference's process global once that is
    in the global symbol scope: a zero value is rejected before any device work."""
    rs, c, tri, qpos, q, sol, collect_pos, chains = api_case
    lib = _lib()
    ref.export_api_globals()
    inner = C.c_double.in_dll(rs.lib, "innerdielectric")
    assert C.c_double.in_dll(C.CDLL(None), "innerdielectric").value == inner.value == c["eps_in"]
    entries = ref.pdb_entries(collect_pos, potential=7.0)
    try:
        inner.value = 0.0
        _collect(lib, rs, entries, ref.pdb_entries(qpos, q), sol)
    finally:
        inner.value = c["eps_in"]
    assert np.all(_potentials(entries) == 7.0)
    assert b"innerdielectric must be positive" in lib.fftsvd_b200_last_error()


def test_dropin_solve_without_device_returns_null(api_case):
    """Without a CUDA device the drop-in solve reads the caller's operator
    (layout walk and cache signature), then reports the missing device and
    leaves the solution NULL."""
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a CUDA device is present; the GPU tests cover the solve")
    rs, c, tri, qpos, q, sol, collect_pos, chains = api_case
    lib = F.load()
    lib.solveSurfaceOperator.restype = None
    lib.solveSurfaceOperator.argtypes = [C.POINTER(C.POINTER(C.c_double)), C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_double), C.c_uint]
    rhs = np.ascontiguousarray(rs.rhs())
    out = C.POINTER(C.c_double)()
    lib.solveSurfaceOperator(C.byref(out), C.c_void_p(rs.surface_operator), C.c_void_p(rs.preconditioner),
                             rhs.ctypes.data_as(C.POINTER(C.c_double)), len(tri))
    assert not out
    assert lib.fftsvd_b200_last_error()


@pytest.mark.gpu
def test_collect_matches_reference_without_coulomb(api_case, gpu):
    rs, c, tri, qpos, q, sol, collect_pos, chains = api_case
    lib = _lib()
    inputs = ref.pdb_entries(qpos, q, chain=chains)
    ours = ref.pdb_entries(collect_pos, potential=7.0)
    theirs = ref.pdb_entries(collect_pos)
    _collect(lib, rs, ours, inputs, sol)
    with ref.stdout_to_stderr():
        rs.collect_potentials(theirs, inputs, sol, addcoulombic=0)
    p, p_ref = _potentials(ours), _potentials(theirs)
    assert np.all(p[len(q):] == 0.0) and np.all(p_ref[len(q):] == 0.0)
    assert rel(p, p_ref) < 1e-11
    assert rel(p[:len(q)], 561.0 * rs.reaction(sol) / c["eps_in"]) < 1e-11


@pytest.mark.gpu
def test_collect_matches_reference_with_coulomb_and_globals(api_case, gpu):
    """With the reference's globals visible: addcoulombic adds the Coulomb sum
    over input entries whose chain is not 'X' (either case), and innerdielectric
    scales every potential."""
    rs, c, tri, qpos, q, sol, collect_pos, chains = api_case
    lib = _lib()
    ref.export_api_globals()
    coul = C.c_uint.in_dll(rs.lib, "addcoulombic")
    inner = C.c_double.in_dll(rs.lib, "innerdielectric")
    assert inner.value == c["eps_in"]
    inputs = ref.pdb_entries(qpos, q, chain=chains)
    try:
        coul.value = 1
        ours = ref.pdb_entries(collect_pos)
        _collect(lib, rs, ours, inputs, sol)
        theirs = ref.pdb_entries(collect_pos)
        with ref.stdout_to_stderr():
            rs.collect_potentials(theirs, inputs, sol, addcoulombic=1)
        assert rel(_potentials(ours), _potentials(theirs)) < 1e-11
        coul.value = 0
        plain = ref.pdb_entries(collect_pos)
        _collect(lib, rs, plain, inputs, sol)
        keep = np.array([ch.upper() != b"X" for ch in chains])
        d = np.linalg.norm(collect_pos[:, None, :] - qpos[None, keep, :], axis=2)
        with np.errstate(divide="ignore"):
            terms = np.where(d > 0, 561.0 * q[keep][None, :] / (c["eps_in"] * d), 0.0)
        coulomb = _potentials(ours) - _potentials(plain)
        assert rel(coulomb, terms.sum(axis=1)) < 1e-11
        coul.value = 1
        inner.value = 2.0 * c["eps_in"]
        halved = ref.pdb_entries(collect_pos)
        _collect(lib, rs, halved, inputs, sol)
        assert rel(_potentials(halved), 0.5 * _potentials(ours)) < 1e-13
    finally:
        coul.value = 0
        inner.value = c["eps_in"]


@pytest.mark.gpu
def test_dropin_solve_rebuilds_for_another_operator_at_same_addresses(gpu):
    """Operators freed and rebuilt (here: the same mesh with another kappa, then
    another mesh) may reuse the addresses of the previous ones; every solve must
    still match the reference solve of the operator it was given."""
    lib = F.load()
    lib.solveSurfaceOperator.restype = None
    lib.solveSurfaceOperator.argtypes = [C.POINTER(C.POINTER(C.c_double)), C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_double), C.c_uint]
    tri3, qpos3, q3, c3 = make_case("blob3")
    born, bpos, bq, cb = make_case("born3")
    systems = [(tri3, qpos3, q3, c3["eps_in"], c3["eps_out"], c3["kappa"]),
               (tri3, qpos3, q3, c3["eps_in"], c3["eps_out"], 0.3),
               (born, bpos, bq, cb["eps_in"], cb["eps_out"], cb["kappa"])]
    for tri, qpos, q, eps_in, eps_out, kappa in systems:
        with ref.stdout_to_stderr():
            rs = ref.RefSystem(tri, qpos, q, eps_in, eps_out, kappa, via_api=True, gmres_tol=1e-6)
        rhs = np.ascontiguousarray(rs.rhs())
        out = C.POINTER(C.c_double)()
        lib.solveSurfaceOperator(C.byref(out), C.c_void_p(rs.surface_operator), C.c_void_p(rs.preconditioner),
                                 rhs.ctypes.data_as(C.POINTER(C.c_double)), len(tri))
        assert out
        x = np.ctypeslib.as_array(out, shape=(2 * len(tri),)).copy()
        C.CDLL(None).free(out)
        x_ref, _ = rs.solve(rhs, 1e-6)
        e, e_ref = rs.energy(rs.reaction(x)), rs.energy(rs.reaction(x_ref))
        assert abs(e - e_ref) < 2e-6 * abs(e_ref), (kappa, e, e_ref)
        rs.close()
