"""Input front end: the reference's readers for parameters, molecules and surface meshes
(FFTSVDpbeAPI.c, VertFace.c), so that PDB-derived systems run through the solver.

Names and results follow the reference functions; the C parsing rules are kept where they
decide what is read:

- Lines are read as C ``fgets`` reads them into a fixed buffer: at most size - 1 characters
  at a time (longer lines arrive in pieces). A field past the end of a short line reads
  what an earlier, longer line left in the buffer; readers that count their records first
  start their second pass with the file's last line in it.
- Numbers are converted with the prefix rules of C ``atof``, ``atoi`` and ``sscanf``.
- Text fields lose all whitespace (``removeWhitespace``, FFTSVDpbeAPI.c:64-80).

Where the reference calls ``error()`` and exits (FFTSVDpbeAPI.c:38-50), these functions raise
``FrontEndError``; ``warning()`` becomes a Python warning. Where the reference's behaviour
is undefined (face indices outside the vertex list, more CRD records than the count line
declares), these functions raise as well.

Only flat panels and the two-region (or salt-free) topology are built by the library's own
setup: ``pbe_system`` rejects salt-layer (Stern), cavity and curved-panel inputs.
"""
from __future__ import annotations

import dataclasses
import math
import warnings

import numpy as np

KT_CONVERSION = 561.0   # FFTSVDpbeAPI.h: kT units, for compatibility with DelPhi
DEBYE_CONSTANT = 3.047  # FFTSVDpbeAPI.h: kappa = sqrt(ionic strength) / 3.047 (FFTSVDpbeAPI.c:1060)


class FrontEndError(ValueError):
    """An input the reference rejects with error() and exit(-1)."""


# ------------------------------------------------------------------ C text semantics

_SPACE = b" \t\n\v\f\r"


class _LineBuffer:
    """A char buffer filled by C fgets(buf, size, file): each read stores at most size - 1
    bytes (up to and including a newline) and a terminating NUL; bytes after the NUL keep
    what earlier reads left there."""

    def __init__(self, data: bytes, size: int):
        self.data, self.size, self.pos = data, size, 0
        self.buf = bytearray(size)

    def next(self) -> bool:
        if self.pos >= len(self.data):
            return False
        end = self.pos
        limit = min(len(self.data), self.pos + self.size - 1)
        while end < limit:
            end += 1
            if self.data[end - 1] == 0x0A:
                break
        chunk = self.data[self.pos:end]
        self.buf[:len(chunk)] = chunk
        self.buf[len(chunk)] = 0
        self.pos = end
        return True

    def rewind(self) -> "_LineBuffer":
        """Read to the end and start again, as the readers that count their records first do
        (the buffer then holds the file's last piece)."""
        while self.next():
            pass
        self.pos = 0
        return self

    def cstr(self, off: int = 0) -> bytes:
        """The NUL-terminated string starting at off."""
        end = self.buf.find(0, off)
        return bytes(self.buf[off:end if end >= 0 else len(self.buf)])

    def strncpy(self, off: int, n: int) -> bytes:
        """strncpy(dst, buf + off, n) into a zeroed destination: the bytes up to n or a NUL."""
        return self.cstr(off)[:n]

    def char(self, off: int) -> bytes:
        return bytes(self.buf[off:off + 1])


def _remove_ws(b: bytes) -> str:
    return bytes(c for c in b if c not in _SPACE).decode("latin-1")


def _strtod_prefix(s: bytes, i: int = 0):
    """C strtod on s[i:]: (value, end index); end == i when nothing converts."""
    n = len(s)
    j = i
    while j < n and s[j] in _SPACE:
        j += 1
    k = j
    if k < n and s[k] in b"+-":
        k += 1
    low = s[k:k + 8].lower()
    for word in (b"infinity", b"inf", b"nan"):
        if low.startswith(word):
            sign = -1.0 if s[j:j + 1] == b"-" else 1.0
            return (sign * math.inf if word != b"nan" else math.nan), k + len(word)
    m = k
    digits = 0
    while m < n and 0x30 <= s[m] <= 0x39:
        m += 1
        digits += 1
    if m < n and s[m] == 0x2E:
        m += 1
        while m < n and 0x30 <= s[m] <= 0x39:
            m += 1
            digits += 1
    if digits == 0:
        return 0.0, i
    if m < n and s[m] in b"eE":
        e = m + 1
        if e < n and s[e] in b"+-":
            e += 1
        if e < n and 0x30 <= s[e] <= 0x39:
            while e < n and 0x30 <= s[e] <= 0x39:
                e += 1
            m = e
    return float(s[j:m]), m


def _atof(s: bytes) -> float:
    return _strtod_prefix(s)[0]


def _strtol_prefix(s: bytes, i: int = 0):
    n = len(s)
    j = i
    while j < n and s[j] in _SPACE:
        j += 1
    k = j
    if k < n and s[k] in b"+-":
        k += 1
    m = k
    while m < n and 0x30 <= s[m] <= 0x39:
        m += 1
    if m == k:
        return 0, i
    return int(s[j:m]), m


def _atoi(s: bytes) -> int:
    return _strtol_prefix(s)[0]


def _uint(v: int) -> int:
    return v & 0xFFFFFFFF  # assignment of an int to an unsigned int field


def _sscanf(s: bytes, count: int, conv) -> list:
    """sscanf with `count` numeric conversions separated by spaces: the values converted
    before the first failure."""
    out, i = [], 0
    for _ in range(count):
        v, e = conv(s, i)
        if e == i:
            break
        out.append(v)
        i = e
    return out


def _read(path: str) -> bytes:
    try:
        with open(path, "rb") as f:
            return f.read()
    except OSError as e:
        raise FrontEndError(f"Could not open {path}: {e.strerror}") from e


# ------------------------------------------------------------------ parameters

@dataclasses.dataclass
class Params:
    """The reference's parameter globals (FFTSVDpbeAPI.c:18-36), all zero before readParams."""
    dielectricvertexdensity: float = 0.0
    saltvertexdensity: float = 0.0
    innerdielectric: float = 0.0
    outerdielectric: float = 0.0
    ionicstrength: float = 0.0
    ionexclusionradius: float = 0.0
    proberadius: float = 0.0
    errortolerance: float = 0.0
    energycalculation: str = "\0"
    outputmodpdb: int = 0
    outputfrc: int = 0
    addcoulombic: int = 0
    usequalocation: int = 0
    usecurved: int = 0
    inftydielectric: float = 0.0
    # lambda in the reference; a Python keyword here
    lambda_: float = 0.0

    @property
    def kappa(self) -> float:
        """Inverse Debye length (1/A) from the ionic strength (FFTSVDpbeAPI.c:1060)."""
        return math.sqrt(self.ionicstrength) / DEBYE_CONSTANT


def _yesno(s: bytes) -> int:
    """FFTSVDpbeAPI.c:82-93."""
    t = s.split(b"\0")[0].decode("latin-1").lower()
    if len(t) == 0:
        return 0
    if t in ("t", "y", "true", "yes", "1"):
        return 1
    if t in ("f", "n", "false", "no", "0"):
        return 0
    raise FrontEndError("Invalid parameter boolean expression")


def readParams(path: str, params: Params | None = None) -> Params:
    """DelPhi-style parameter file, one `COMMAND=value` per line (FFTSVDpbeAPI.c:95-175)."""
    p = params if params is not None else Params()
    buf = _LineBuffer(_read(path), 81)
    while buf.next():
        line = _remove_ws(buf.cstr()).encode("latin-1")
        cmd = b""
        while len(cmd) < len(line) and (0x41 <= line[len(cmd)] <= 0x5A or 0x61 <= line[len(cmd)] <= 0x7A):
            cmd += line[len(cmd):len(cmd) + 1]
        command = cmd.decode("latin-1").upper()
        nxt = line[len(cmd) + 1:]
        simple = {"DVERT": "dielectricvertexdensity", "SVERT": "saltvertexdensity", "INDI": "innerdielectric",
                  "EXDI": "outerdielectric", "INFTYDI": "inftydielectric", "LAMBDA": "lambda_",
                  "SALT": "ionicstrength", "IONRAD": "ionexclusionradius", "PRBRAD": "proberadius",
                  "DE": "errortolerance"}
        flags = {"ADDCOUL": "addcoulombic", "USEQUAL": "usequalocation", "CURVED": "usecurved"}
        if command in simple:
            setattr(p, simple[command], _atof(nxt))
        elif command in flags:
            if _yesno(nxt):
                setattr(p, flags[command], 1)
        elif command == "ENERGY":
            rest = line[len(cmd):]
            if len(rest) >= 2 and rest[0:1] == b"(":
                p.energycalculation = chr(rest[1]).upper()
        elif command == "OUT":
            rest = line[len(cmd):]
            if rest[0:1] == b"(" and len(rest) > 1 and rest[1:2] != b")":
                sub = rest[1:].split(b")")[0].decode("latin-1")
                if sub.lower() == "modpdb":
                    p.outputmodpdb = 1
                elif sub.lower() == "frc":
                    p.outputfrc = 1
                elif sub.lower() != "phi":
                    warnings.warn(f"Unknown OUT parameter subcommand {sub}")
        else:
            warnings.warn(f"Unknown parameter command {command}")
    return p


def checkParams(p: Params) -> None:
    """FFTSVDpbeAPI.c:177-200."""
    if p.dielectricvertexdensity < 0.0:
        raise FrontEndError("Dielectric vertex density must be > 0.0")
    if p.saltvertexdensity < 0.0:
        raise FrontEndError("Salt vertex density must be > 0.0")
    if p.innerdielectric < 1.0:
        raise FrontEndError("Inner dielectric must be >= 1.0")
    if p.outerdielectric < 1.0:
        raise FrontEndError("Outer dielectric must be >= 1.0")
    if p.innerdielectric > p.outerdielectric:
        warnings.warn("Inner dielectric is greater than outer dielectric")
    if p.ionicstrength < 0.0:
        raise FrontEndError("Ionic strength must be >= 0.0")
    if p.ionexclusionradius < 0.0:
        raise FrontEndError("Ionic exclusion radius must be >= 0.0")
    if p.proberadius < 0.0:
        raise FrontEndError("Probe radius must be >= 0.0")
    if p.errortolerance <= 0.0:
        raise FrontEndError("Error tolerance must be >= 0.0")
    if p.energycalculation != "G":
        raise FrontEndError("Only energy calculation 'G' is currently supported")
    if p.usequalocation and p.ionicstrength > 0.0:
        raise FrontEndError("Qualocation does not work with ionic strength > 0.0")


# ------------------------------------------------------------------ molecules

@dataclasses.dataclass
class PDBentry:
    """FFTSVDpbeAPI.h PDBentry; char fields as str ('' for NUL)."""
    record: str = ""
    atomnumber: int = 0
    atomname: str = ""
    alternatelocation: str = ""
    residuename: str = ""
    chain: str = ""
    residuenumber: int = 0
    residueinsertion: str = ""
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0
    occupancy: float = 0.0
    temperature: float = 0.0
    footnotenumber: int = 0
    radius: float = 0.0
    charge: float = 0.0
    potential: float = 0.0


@dataclasses.dataclass
class SIZentry:
    atomlabel: str = ""
    residuelabel: str = ""
    radius: float = 0.0


@dataclasses.dataclass
class CRGentry:
    atomlabel: str = ""
    residuelabel: str = ""
    residuenumber: int = 0
    chain: str = ""
    charge: float = 0.0


def _ch(b: bytes) -> str:
    return "" if b in (b"", b"\0") else b.decode("latin-1")


def _unsigned_from_double(v: float) -> int:
    """C conversion of a double to unsigned int (values in range)."""
    return _uint(int(v)) if math.isfinite(v) else 0


def readPDB(path: str) -> list[PDBentry]:
    """ATOM and HETATM records by fixed columns (FFTSVDpbeAPI.c:202-278)."""
    buf = _LineBuffer(_read(path), 81).rewind()
    out = []
    while buf.next():
        line = buf.cstr()
        if not (line[:4].upper() == b"ATOM" or line[:6].upper() == b"HETATM"):
            continue
        e = PDBentry()
        e.record = _remove_ws(buf.strncpy(0, 6))
        e.atomnumber = _uint(_atoi(buf.strncpy(6, 5)))
        e.atomname = _remove_ws(buf.strncpy(12, 4))
        e.alternatelocation = _ch(buf.char(16))
        e.residuename = _remove_ws(buf.strncpy(17, 3))
        e.chain = _ch(buf.char(21))
        e.residuenumber = _uint(_atoi(buf.strncpy(22, 4)))
        e.residueinsertion = _ch(buf.char(26))
        e.x = _atof(buf.strncpy(30, 8))
        e.y = _atof(buf.strncpy(38, 8))
        e.z = _atof(buf.strncpy(46, 8))
        e.occupancy = _atof(buf.strncpy(54, 6))
        e.temperature = _atof(buf.strncpy(60, 6))
        e.footnotenumber = _unsigned_from_double(_atof(buf.strncpy(67, 3)))
        out.append(e)
    return out


def readCRD(path: str) -> list[PDBentry]:
    """CHARMM CRD: '*' header lines, an atom count, then fixed-column records
    (FFTSVDpbeAPI.c:280-341)."""
    buf = _LineBuffer(_read(path), 81)
    count = None
    while buf.next():
        if buf.cstr()[:1] != b"*":
            count = _atoi(buf.cstr())
            break
    if count is None:
        count = _atoi(buf.cstr())
    out = [PDBentry() for _ in range(max(count, 0))]
    k = 0
    while buf.next():
        if k >= len(out):
            raise FrontEndError(f"{path}: more CRD records than the declared {count}")
        e = out[k]
        e.atomnumber = _uint(_atoi(buf.strncpy(0, 5)))
        e.residuenumber = _uint(_atoi(buf.strncpy(5, 5)))
        e.residuename = _remove_ws(buf.strncpy(11, 3))
        e.atomname = _remove_ws(buf.strncpy(16, 4))
        e.x = _atof(buf.strncpy(20, 10))
        e.y = _atof(buf.strncpy(30, 10))
        e.z = _atof(buf.strncpy(40, 10))
        e.chain = _ch(buf.char(51))
        e.temperature = _atof(buf.strncpy(61, 10))
        k += 1
    return out


def readXYZR(path: str) -> list[PDBentry]:
    """'x y z radius' per line (FFTSVDpbeAPI.c:343-381)."""
    buf = _LineBuffer(_read(path), 81).rewind()
    out = []
    while buf.next():
        v = _sscanf(buf.cstr(), 4, _strtod_prefix)
        e = PDBentry()
        for name, val in zip(("x", "y", "z", "radius"), v):
            setattr(e, name, val)
        out.append(e)
    return out


def _table_lines(path: str):
    buf = _LineBuffer(_read(path), 81).rewind()
    buf.next()  # first line is junk
    while buf.next():
        line = buf.cstr()
        if line[:1] != b"!" and len(line) > 0:
            yield buf


def readSIZ(path: str) -> list[SIZentry]:
    """DelPhi radius table (FFTSVDpbeAPI.c:383-437)."""
    out = []
    for buf in _table_lines(path):
        out.append(SIZentry(_remove_ws(buf.strncpy(0, 6)), _remove_ws(buf.strncpy(6, 3)), _atof(buf.strncpy(9, 8))))
    return out


def readCRG(path: str) -> list[CRGentry]:
    """DelPhi charge table (FFTSVDpbeAPI.c:439-507)."""
    out = []
    for buf in _table_lines(path):
        out.append(CRGentry(_remove_ws(buf.strncpy(0, 6)), _remove_ws(buf.strncpy(6, 3)),
                            _uint(_atoi(buf.strncpy(9, 4))), _ch(buf.char(13)), _atof(buf.strncpy(14, 8))))
    return out


def assignRadiiCharges(pdb: list[PDBentry], siz: list[SIZentry], crg: list[CRGentry]) -> None:
    """Radius and charge of every atom by the reference's match levels (FFTSVDpbeAPI.c:569-674):
    radii by atom and residue name, else atom-name prefix, else element letter; charges by
    the most specific of eight combinations of chain, residue number, residue and atom name."""
    for a in pdb:
        level = 0
        for r in siz:
            if a.atomname == r.atomlabel and a.residuename == r.residuelabel:
                a.radius = r.radius
                level = 3
                break
            if len(r.residuelabel) == 0 and a.atomname[:len(r.atomlabel)] == r.atomlabel:
                if level < 2:
                    a.radius = r.radius
                    level = 2
            elif (len(r.residuelabel) == 0 and a.atomname[:1] == r.atomlabel[:1] and len(r.atomlabel) == 1
                  and len(a.atomname) > 0):
                if level < 1:
                    a.radius = r.radius
                    level = 1
        if level == 0:
            warnings.warn(f"Atom {a.atomnumber} {a.atomname} {a.residuename} {a.chain} has no radius entry, "
                          "defaulting to 0.0")
            a.radius = 0.0
        elif level == 1:
            warnings.warn(f"Atom {a.atomnumber} {a.atomname} {a.residuename} {a.chain} using default element "
                          f"radius of {a.radius:f}")
        level = 0
        for c in crg:
            same_name = a.atomname == c.atomlabel
            same_res = a.residuename == c.residuelabel
            same_chain = c.chain == a.chain
            same_num = c.residuenumber == a.residuenumber
            if same_chain and same_num and same_res and same_name:
                a.charge = c.charge
                level = 8
                break
            for lev, cond in ((7, same_num and same_res and same_name), (6, same_chain and same_res and same_name),
                              (5, same_res and same_name), (4, same_chain and same_num and same_name),
                              (3, same_num and same_name), (2, same_chain and same_name), (1, same_name)):
                if cond:
                    if level < lev:
                        a.charge = c.charge
                        level = lev
                    break
        if level == 0 and len(crg) > 0:
            warnings.warn(f"Atom {a.atomnumber} {a.atomname} {a.residuename} {a.chain} has no charge entry, "
                          "defaulting to 0.0")
            a.charge = 0.0


# ------------------------------------------------------------------ surfaces

def _read_vert(path: str) -> np.ndarray:
    """VertFace_readvert (VertFace.c:26-51): every 127-byte fgets piece is a vertex."""
    buf = _LineBuffer(_read(path), 128).rewind()
    verts = []
    while buf.next():
        v = _sscanf(buf.cstr(), 3, _strtod_prefix)
        verts.append(v + [0.0] * (3 - len(v)))
    return np.array(verts, dtype=np.float64).reshape(-1, 3)


def _scan_uint(s: bytes, i: int):
    v, e = _strtol_prefix(s, i)
    return _uint(v), e


def _read_face(path: str, flip: bool) -> tuple[np.ndarray, np.ndarray]:
    """VertFace_readface / _readface_flip (VertFace.c:53-101): 1-based 'a b c genus';
    the flipped reader stores the second index as the third corner and vice versa."""
    buf = _LineBuffer(_read(path), 128).rewind()
    faces, genus = [], []
    while buf.next():
        v = _sscanf(buf.cstr(), 4, _scan_uint)
        v = v + [0] * (4 - len(v))
        a, b, c = ((x - 1) & 0xFFFFFFFF for x in v[:3])
        faces.append((a, c, b) if flip else (a, b, c))
        genus.append(v[3])
    return np.array(faces, dtype=np.int64).reshape(-1, 3), np.array(genus, dtype=np.int64)


def _distance(u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Vector3D_distance (Vector3D.c:64-68), same operation order."""
    d = u - v
    return np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])


def getFlatPanels(basename: str, accessible: int = 0, cavity: int = 0, usequalocation: int = 0) -> np.ndarray:
    """Flat panels of basename.vert / basename.face (FFTSVDpbeAPI.c:676-712): faces are read
    flipped unless the surface is a cavity (without qualocation); faces of zero area are dropped,
    and on an accessible surface every face whose genus is not 1. Returns (panels, 9): the three
    corners of each panel in the order of FlatPanel_allocate (the library's triangle layout)."""
    verts = _read_vert(basename + ".vert")
    faces, genus = _read_face(basename + ".face", flip=not (cavity and not usequalocation))
    if faces.size and (faces.max() >= len(verts)):
        raise FrontEndError(f"{basename}.face: vertex index outside the {len(verts)} vertices")
    vx, vy, vz = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
    d1, d2, d3 = _distance(vx, vy), _distance(vy, vz), _distance(vz, vx)
    s = 0.5 * (d1 + d2 + d3)
    with np.errstate(invalid="ignore"):
        area = np.sqrt(s * (s - d1) * (s - d2) * (s - d3))
    keep = area > 0.0
    if accessible:
        keep &= genus == 1
    return np.ascontiguousarray(np.concatenate([vx[keep], vy[keep], vz[keep]], axis=1))


@dataclasses.dataclass
class SRF:
    """readSRF output (FFTSVDpbeAPI.c:776-1032): panel sets per layer and the parents."""
    salttype: str
    dielectrictype: str
    salts: list
    dielectrics: list
    dielectriccavities: list
    saltcavities: list
    dielectricparent: list
    dielectriccavityparent: list
    saltcavityparent: list
    numtotalpanels: int


def _srf_names(line: bytes) -> list[bytes]:
    """The file names of one SRF line: as many strsep(" \\n") tokens, in order, as the
    line has non-empty tokens."""
    toks = line.replace(b"\n", b" ").split(b" ")
    count = sum(1 for t in toks if len(t) > 0)
    return toks[:count]


def readSRF(path: str, usequalocation: int = 0) -> SRF:
    """The SRF surface list (FFTSVDpbeAPI.c:776-1032): salt and dielectric panel types, then
    the salt, dielectric, dielectric-cavity and salt-cavity surface base names, then the
    parents of dielectrics, dielectric cavities and salt cavities. Relative names are taken
    relative to the SRF file's directory."""
    buf = _LineBuffer(_read(path), 1024)
    lines = []
    for _ in range(9):
        lines.append(buf.cstr() if buf.next() else b"")
    salttype = chr(lines[0][0]) if lines[0] else "\0"
    dielectrictype = chr(lines[1][0]) if lines[1] else "\0"
    slash = path.rfind("/")
    base = path[:slash + 1] if slash >= 0 else ""

    def load(line, kind, accessible, cavity):
        sets = []
        for tok in _srf_names(line):
            name = tok.decode("latin-1")
            if not name.startswith("/"):
                name = base + name
            if kind == "f":
                sets.append(getFlatPanels(name, accessible, cavity, usequalocation))
            elif kind == "c":
                raise FrontEndError("curved panels are not supported by this library's setup")
            else:
                sets.append(np.zeros((0, 9)))
        return sets

    salts = load(lines[2], salttype, 1, 0)
    diel = load(lines[3], dielectrictype, 0, 0)
    dcav = load(lines[4], dielectrictype, 0, 1)
    scav = load(lines[5], salttype, 1, 1)
    total = sum(len(p) for p in salts + diel + dcav + scav)

    def parents(line, n):
        toks = line.replace(b"\n", b" ").split(b" ")
        return [_uint(_atoi(toks[i] if i < len(toks) else b"")) for i in range(n)]

    dpar = parents(lines[6], len(diel))
    dcpar = parents(lines[7], len(dcav))
    scpar = parents(lines[8], len(scav))
    for i, p in enumerate(dcpar):
        if p == 999:  # marked as bad by the mesher
            total -= len(dcav[i])
    for i, p in enumerate(scpar):
        if p == 999:
            total -= len(scav[i])
    return SRF(salttype, dielectrictype, salts, diel, dcav, scav, dpar, dcpar, scpar, total)


# ------------------------------------------------------------------ the whole input

@dataclasses.dataclass
class PBESystem:
    """A molecule and its dielectric surface, ready for fftsvd_b200.surface.Surface.from_problem."""
    params: Params
    atoms: list
    panels: np.ndarray        # (n, 9) flat panel corners
    charge_pos: np.ndarray    # (nq, 3) charged atoms
    charge: np.ndarray        # (nq,)

    @property
    def kappa(self) -> float:
        return self.params.kappa


def pbe_system(params_path: str, pdb_path: str, siz_path: str, crg_path: str, srf_path: str) -> PBESystem:
    """The FFTSVDpbe input sequence (FFTSVDpbe.c:115-158): parameters, molecule, radii and
    charges, surfaces. Supports one flat dielectric surface without salt layers or cavities:
    the single-molecule topology of the library's setup (Laplace inside, Yukawa or Laplace
    outside with kappa = sqrt(ionic strength) / 3.047)."""
    p = readParams(params_path)
    checkParams(p)
    atoms = readPDB(pdb_path)
    siz = readSIZ(siz_path)
    crg = readCRG(crg_path)
    assignRadiiCharges(atoms, siz, crg)
    srf = readSRF(srf_path, p.usequalocation)
    if p.usecurved or srf.dielectrictype != "f":
        raise FrontEndError("curved panels are not supported by this library's setup")
    if p.ionicstrength > 0.0 and p.ionexclusionradius > 1e-6:
        raise FrontEndError("the Stern-layer topology (salt > 0 with an ion exclusion radius) is not supported")
    if len(srf.dielectrics) != 1 or srf.dielectriccavities or srf.saltcavities:
        raise FrontEndError("exactly one dielectric surface and no cavities are supported")
    pos = np.array([[a.x, a.y, a.z] for a in atoms], dtype=np.float64).reshape(-1, 3)
    q = np.array([a.charge for a in atoms], dtype=np.float64)
    return PBESystem(p, atoms, srf.dielectrics[0], pos, q)


def pbe_surface(system: PBESystem, svd_tol: float = 1e-5, **kwargs):
    """The device surface of a system read by pbe_system: the library's own setup with the
    system's dielectrics and kappa, the SVD tolerance of the reference API (SVD_ERROR 1e-5,
    FFTSVDpbeAPI.h) by default."""
    from .surface import Surface
    return Surface.from_problem(system.panels, system.charge_pos, system.charge, system.params.innerdielectric,
                                system.params.outerdielectric, system.kappa, svd_tol=svd_tol, **kwargs)


def write_vert_face(basename: str, vertices: np.ndarray, faces: np.ndarray, genus=None, flip: bool = True) -> None:
    """Write a triangle mesh as basename.vert / basename.face in the layout getFlatPanels
    reads (1-based indices). With flip (the default), the second and third corners are
    swapped on output, so that the flipped reader restores the given corner order."""
    vertices = np.asarray(vertices, dtype=np.float64)
    faces = np.asarray(faces, dtype=np.int64)
    g = np.ones(len(faces), dtype=np.int64) if genus is None else np.asarray(genus)
    with open(basename + ".vert", "w") as f:
        for v in vertices:
            f.write(f"{v[0]:.17g} {v[1]:.17g} {v[2]:.17g}\n")
    with open(basename + ".face", "w") as f:
        for (a, b, c), gg in zip(faces, g):
            if flip:
                b, c = c, b
            f.write(f"{a + 1} {b + 1} {c + 1} {gg}\n")


def writeMODPDB(path: str, atoms: list[PDBentry]) -> None:
    """The atoms with their radii and charges (FFTSVDpbeAPI.c:509-533)."""
    with open(path, "w") as f:
        f.write("HEADER output from FFTSVDpbe\n")
        f.write("HEADER atom radii in columns 55-60\n")
        f.write("HEADER atom charges in columns 61-67\n")
        for a in atoms:
            f.write("%-6s%5d %4s%1s%3s %1s%4d%1s   %8.3f%8.3f%8.3f%6.2f%7.3f\n" % (
                a.record, a.atomnumber, a.atomname, a.alternatelocation or "\0", a.residuename,
                a.chain or "\0", a.residuenumber, a.residueinsertion or "\0", a.x, a.y, a.z, a.radius, a.charge))


def writeFRC(path: str, atoms: list[PDBentry], params: Params) -> None:
    """Site potentials of the atoms (their `potential` fields) in the DelPhi FRC layout
    (FFTSVDpbeAPI.c:535-567)."""
    with open(path, "w") as f:
        f.write("FFTSVDpbe SITE POTENTIAL FILE\n")
        f.write("grid size,percent fill: %3d %8f\n" % (0, 0.0))
        f.write("inner,outer dielectric: %8f %8f\n" % (params.innerdielectric, params.outerdielectric))
        f.write("ionic strength (M): %8f\n" % params.ionicstrength)
        f.write("ion excl., probe radius: %8f %8f\n" % (params.ionexclusionradius, params.proberadius))
        f.write("linear, nolinear iterations: %8d %8d\n" % (0, 0))
        f.write("boundary condition: %2d\n" % 0)
        f.write("Data Output: COORDINATES CHARGE POTENTIALS FIELDS\n")
        f.write("title: FFTSVDpbe: BEM PBE Solver\n")
        f.write("\n")
        f.write("\n")
        f.write("    ATOM COORDINATES (X,Y,Z)     CHARGE   GRID PT.    GRID FIELDS: (Ex, Ey, Ez)\n")
        for a in atoms:
            f.write("%9.3f%9.3f%9.3f%8.4f%15.6f  %9.4f%9.4f%9.4f\n" % (a.x, a.y, a.z, a.charge, a.potential, 0.0, 0.0,
                                                                     0.0))
        f.write("total energy =   %6f  kt\n" % 0.0)


__all__ = ["FrontEndError", "Params", "PDBentry", "SIZentry", "CRGentry", "SRF", "PBESystem", "readParams",
           "checkParams", "readPDB", "readCRD", "readXYZR", "readSIZ", "readCRG", "assignRadiiCharges",
           "getFlatPanels", "readSRF", "pbe_system", "pbe_surface", "write_vert_face", "writeMODPDB", "writeFRC", "KT_CONVERSION",
           "DEBYE_CONSTANT"]
