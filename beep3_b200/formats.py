"""libBEEP's on-disk inputs, read on the host above the C ABI.

* :func:`read_gts` -- GTS surfaces (vertices with optional normals, edges,
  faces as edge triples), as ``GTS_Surface::read_mesh_from_file``
  (src/bem/gts_utils.h:32-113); :func:`write_gts` writes the same layout
  (``write_mesh_to_file``, :115-155).
* :func:`read_off` -- OFF / nOFF / header-less OFF triangle meshes
  (``OFF_Surface::read_mesh_from_file``, src/bem/off_utils.h:26-185).
* :func:`read_xyzqr` -- charges ``x y z q r [hydrophobicity sigma epsilon]``
  per line (``Charge::read_charges_from_file``, src/common/charge.h:105-140).
* :class:`MeshTarball` -- ``.mtz`` mesh tarballs: an archive holding
  ``definition.xml`` (root ``<contents>``) that names the mesh, xyzqr,
  centre and energies files and optional ones (``MeshTarball``,
  src/bem/mesh_tarball.h:28-105, src/bem/mesh_tarball.cpp:33-240).
* :func:`load_mesh` -- a :class:`~beep3_b200.beep.Mesh` from a tarball or a
  GTS/OFF file plus an xyzqr file (``Mesh::init`` and the file constructor,
  src/bem/mesh.cpp:55-300): curved meshes from a tarball take their energy
  coefficients from its energies file, as the reference does.
* :class:`ConfigFile` -- the ``<BEM_Config>`` XML run description (solvent,
  output, mesh library, layout of instances; ``ConfigFile::init``,
  src/bem/config_file.cpp:32-247), and :func:`beep_from_config`, which sets
  up a :class:`~beep3_b200.beep.BEEP` scenario from it (``BEEP::init``,
  src/beep/beep.cpp:114-195).

Vertex normals: the GTS reader keeps supplied unit normals and the mesh
computes those given as zero (src/bem/mesh.cpp:1006-1019); OFF normals are
always recomputed (src/bem/off_utils.h:160-185).  Default qualocation /
quadrature rules are the reference's DEFAULT_QUALS 4 and DEFAULT_QUADS 0
(src/beep/beep.h:58-59).
"""
from __future__ import annotations

import os
import shutil
import tarfile
import tempfile
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

DEFAULT_QUALS = 4
DEFAULT_QUADS = 0


class FormatError(ValueError):
    """A file does not follow the format its reader expects."""


def _data_lines(path):
    """Lines of a text file without those that start with '#' or '!'."""
    with open(path) as f:
        for ln in f:
            if ln.startswith(("#", "!")):
                continue
            yield ln


# --------------------------------------------------------------------------- GTS
def read_gts(path) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(vertices (V, 3), vertex normals (V, 3; zero rows where the file gives
    none), triangles (T, 3) 0-based) of a GTS surface.  A face is three
    1-based edge indices; its vertices are, in order, the vertex shared by
    edges 1 and 2, by edges 2 and 3 and by edges 3 and 1."""
    it = _data_lines(path)
    try:
        head = next(it).split()
        nv, ne, nf = int(head[0]), int(head[1]), int(head[2])
    except (StopIteration, ValueError, IndexError) as e:
        raise FormatError(f"{path}: expected 'num_vertices num_edges num_faces'") from e
    if ne != 3 * nf // 2:
        raise FormatError(f"{path}: {ne} edges for {nf} faces is not a closed triangle mesh")
    verts = np.zeros((nv, 3))
    normals = np.zeros((nv, 3))
    edges = np.zeros((ne, 2), np.int64)
    tris = np.zeros((nf, 3), np.int64)
    try:
        for k in range(nv):
            f = next(it).split()
            verts[k] = [float(v) for v in f[:3]]
            if len(f) >= 6:
                normals[k] = [float(v) for v in f[3:6]]
        for k in range(ne):
            f = next(it).split()
            edges[k] = [int(f[0]) - 1, int(f[1]) - 1]
        for k in range(nf):
            f = next(it).split()
            e = [int(v) - 1 for v in f[:3]]
            for i, (a, b) in enumerate(((0, 1), (1, 2), (2, 0))):
                common = set(edges[e[a]].tolist()) & set(edges[e[b]].tolist())
                if len(common) != 1:
                    raise FormatError(f"{path}: face {k + 1}: edges {e[a] + 1} and {e[b] + 1} share no vertex")
                tris[k, i] = common.pop()
    except StopIteration as e:
        raise FormatError(f"{path}: file ends early") from e
    except (ValueError, IndexError) as e:
        raise FormatError(f"{path}: malformed line") from e
    if edges.size and (edges.min() < 0 or edges.max() >= nv):
        raise FormatError(f"{path}: edge vertex index out of range")
    return verts, normals, tris.astype(np.int32)


def write_gts(path, vertices, triangles, vertex_normals=None) -> None:
    """GTS surface of a closed triangle mesh: vertices (with normals when
    given), edges low-high, faces as the edges (v1 v2), (v2 v3), (v3 v1)."""
    V = np.asarray(vertices, float)
    T = np.asarray(triangles, np.int64)
    N = np.zeros_like(V) if vertex_normals is None else np.asarray(vertex_normals, float)
    index: dict[tuple[int, int], int] = {}
    edges: list[tuple[int, int]] = []
    faces = []
    for tri in T.tolist():
        fe = []
        for a, b in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
            key = (min(a, b), max(a, b))
            if key not in index:
                index[key] = len(edges)
                edges.append(key)
            fe.append(index[key])
        faces.append(fe)
    with open(path, "w") as f:
        f.write(f"{len(V)} {len(edges)} {len(faces)} GtsSurface GtsFace GtsEdge GtsVertex\n")
        for v, n in zip(V, N):
            f.write(" ".join(repr(float(x)) for x in (*v, *n)) + "\n")
        for a, b in edges:
            f.write(f"{a + 1} {b + 1}\n")
        for fe in faces:
            f.write(" ".join(str(e + 1) for e in fe) + "\n")


# --------------------------------------------------------------------------- OFF
def read_off(path) -> tuple[np.ndarray, np.ndarray]:
    """(vertices (V, 3), triangles (T, 3) 0-based) of an OFF or nOFF file, or
    of one whose header keyword is missing (first line 'nv nf ne').  Faces
    must be triangles ('3 a b c')."""
    it = _data_lines(path)
    try:
        first = next(it).strip()
        if first in ("OFF", "nOFF"):
            first = next(it).strip()
        nv, nf = (int(v) for v in first.split()[:2])
    except (StopIteration, ValueError) as e:
        raise FormatError(f"{path}: first line should read OFF or nOFF, or 'num_vertices num_faces num_edges'") from e
    verts = np.zeros((nv, 3))
    tris = np.zeros((nf, 3), np.int32)
    try:
        for k in range(nv):
            verts[k] = [float(v) for v in next(it).split()[:3]]
        for k in range(nf):
            f = next(it).split()
            if int(f[0]) != 3:
                raise FormatError(f"{path}: face {k + 1} has {f[0]} vertices; triangles are required")
            tris[k] = [int(v) for v in f[1:4]]
    except StopIteration as e:
        raise FormatError(f"{path}: expected {nv} vertices and {nf} faces, the file ends early") from e
    except (ValueError, IndexError) as e:
        raise FormatError(f"{path}: malformed line") from e
    if tris.size and (tris.min() < 0 or tris.max() >= nv):
        raise FormatError(f"{path}: face vertex index out of range")
    return verts, tris


def write_off(path, vertices, triangles) -> None:
    V = np.asarray(vertices, float)
    T = np.asarray(triangles, np.int64)
    with open(path, "w") as f:
        f.write(f"OFF\n{len(V)} {len(T)} {3 * len(T) // 2}\n")
        for v in V:
            f.write(" ".join(repr(float(x)) for x in v) + "\n")
        for t in T:
            f.write(f"3 {t[0]} {t[1]} {t[2]}\n")


# --------------------------------------------------------------------------- charges
def read_xyzqr(path, skip_zeroes: bool = False) -> np.ndarray:
    """Charges as rows x y z q r hydrophobicity sigma epsilon (the last three
    0 when absent).  A charge of zero is skipped when ``skip_zeroes``, and
    always when it also has no hydrophobicity and no Lennard-Jones pair
    (sigma or epsilon zero): such lines are solvent or hetero atoms."""
    rows = []
    with open(path) as f:
        for n, ln in enumerate(f, 1):
            fields = ln.split()
            if not fields:
                continue
            if len(fields) < 5:
                raise FormatError(f"{path}:{n}: expected x y z q r")
            try:
                vals = [float(v) for v in fields[:8]]
            except ValueError as e:
                raise FormatError(f"{path}:{n}: not a number") from e
            vals += [0.0] * (8 - len(vals))
            q, hyd, sig, eps = vals[3], vals[5], vals[6], vals[7]
            if skip_zeroes and q == 0.0:
                continue
            if q == 0.0 and hyd == 0.0 and (sig == 0.0 or eps == 0.0):
                continue
            rows.append(vals)
    return np.asarray(rows, float).reshape(-1, 8)


def write_xyzqr(path, charges, radius: float = 1.0) -> None:
    """x y z q r lines from rows x y z q (r = ``radius``) or x y z q r ..."""
    C = np.asarray(charges, float)
    with open(path, "w") as f:
        for row in C:
            r = row[4] if len(row) > 4 else radius
            f.write(" ".join(repr(float(v)) for v in (*row[:4], r, *row[5:8])) + "\n")


def read_centre(path) -> np.ndarray:
    with open(path) as f:
        vals = f.read().split()
    if len(vals) < 3:
        raise FormatError(f"{path}: expected x y z")
    return np.array([float(v) for v in vals[:3]])


@dataclass
class EnergyPrecalcs:
    """Per node patch: energy coefficients f and h, force coefficients f and
    h (3 each), hydrophobicity, charge index (src/bem/mesh.cpp:927-960)."""
    coef_f: np.ndarray
    coef_h: np.ndarray
    force_f: np.ndarray
    force_h: np.ndarray
    hydrophobicity: np.ndarray
    charge_index: np.ndarray


def read_energies(path, n_patches: int) -> EnergyPrecalcs:
    vals = np.zeros((n_patches, 10))
    with open(path) as f:
        for k in range(n_patches):
            ln = f.readline()
            if not ln:
                raise FormatError(f"{path}: {k} lines for {n_patches} node patches")
            fields = ln.split()
            try:
                row = [float(v) for v in fields[:10]]
            except ValueError as e:
                raise FormatError(f"{path}:{k + 1}: not a number") from e
            vals[k, :len(row)] = row
    return EnergyPrecalcs(vals[:, 0].copy(), vals[:, 1].copy(), vals[:, 2:5].copy(), vals[:, 5:8].copy(),
                          vals[:, 8].copy(), vals[:, 9].astype(np.int64))


def write_energies(path, coef_f, coef_h) -> None:
    with open(path, "w") as f:
        for cf, ch in zip(coef_f, coef_h):
            f.write(f"{float(cf)!r} {float(ch)!r} 0 0 0 0 0 0 0 0\n")


# --------------------------------------------------------------------------- tarballs
class MeshTarball:
    """A ``.mtz`` mesh tarball extracted to a private temporary folder (removed
    by :meth:`close` or on leaving a ``with`` block).  ``definition.xml`` at
    the archive's top names the files: mandatory ``mesh``, ``xyzqr``,
    ``centre``, ``energies``; optional ``pdb``, ``pqr``, ``vertex_normals``,
    ``fh``, ``diffusion_tensor``, ``ellipsoid``, ``ecm``, ``mesh2``,
    ``energies2``.  A missing mandatory tag or a repeated tag is an error."""

    DEFINITION = "definition.xml"
    ROOT = "contents"
    MANDATORY = ("xyzqr", "mesh", "energies", "centre")
    OPTIONAL = ("pdb", "pqr", "vertex_normals", "fh", "diffusion_tensor", "ellipsoid", "ecm", "mesh2", "energies2")

    def __init__(self, path):
        self.path = Path(path)
        self.work_dir = Path(tempfile.mkdtemp(prefix="beep-"))
        try:
            self._extract()
            self.files = self._parse_definition()
        except BaseException:
            self.close()
            raise

    def _extract(self) -> None:
        try:
            with tarfile.open(self.path, "r:*") as tar:
                for m in tar.getmembers():
                    dest = (self.work_dir / m.name).resolve()
                    if not str(dest).startswith(str(self.work_dir.resolve()) + os.sep) or not (m.isfile() or m.isdir()):
                        raise FormatError(f"{self.path}: archive member {m.name!r} escapes the archive or is not a "
                                          f"plain file")
                tar.extractall(self.work_dir, filter="data")
        except tarfile.TarError as e:
            raise FormatError(f"{self.path}: not a readable archive") from e

    def _parse_definition(self) -> dict[str, Path]:
        xml = self.work_dir / self.DEFINITION
        if not xml.exists():
            raise FormatError(f"{self.path}: no {self.DEFINITION}")
        try:
            root = ET.parse(xml).getroot()
        except ET.ParseError as e:
            raise FormatError(f"{self.DEFINITION} ({self.path}): not well-formed XML") from e
        if root.tag != self.ROOT:
            raise FormatError(f"{self.DEFINITION} ({self.path}): root element should be <{self.ROOT}>")
        files: dict[str, Path] = {}
        for tag in self.MANDATORY + self.OPTIONAL:
            found = root.findall(tag)
            if len(found) > 1:
                raise FormatError(f"{self.DEFINITION} ({self.path}): multiple <{tag}> tags")
            if not found:
                if tag in self.MANDATORY:
                    raise FormatError(f"{self.DEFINITION} ({self.path}): missing mandatory <{tag}> tag")
                continue
            files[tag] = self.work_dir / (found[0].text or "").strip()
        return files

    def get(self, tag: str) -> Path | None:
        return self.files.get(tag)

    def close(self) -> None:
        shutil.rmtree(self.work_dir, ignore_errors=True)

    def __enter__(self) -> "MeshTarball":
        return self

    def __exit__(self, *exc) -> None:
        self.close()


def write_mtz(path, vertices, triangles, charges, centre, coef_f=None, coef_h=None, mesh_format: str = "gts") -> None:
    """A mesh tarball (gzip-compressed tar) with definition.xml, the mesh, the
    charges, the centre and, when given, the energy coefficients."""
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        mesh_name = f"mesh.{mesh_format}"
        (write_gts if mesh_format == "gts" else write_off)(td / mesh_name, vertices, triangles)
        write_xyzqr(td / "charges.xyzqr", charges)
        (td / "centre.txt").write_text(" ".join(repr(float(v)) for v in centre) + "\n")
        n = len(np.asarray(vertices))
        write_energies(td / "energies.txt", np.zeros(n) if coef_f is None else coef_f,
                       np.zeros(n) if coef_h is None else coef_h)
        (td / MeshTarball.DEFINITION).write_text(
            f"<contents><mesh>{mesh_name}</mesh><xyzqr>charges.xyzqr</xyzqr><centre>centre.txt</centre>"
            f"<energies>energies.txt</energies></contents>\n")
        with tarfile.open(path, "w:gz") as tar:
            for name in (MeshTarball.DEFINITION, mesh_name, "charges.xyzqr", "centre.txt", "energies.txt"):
                tar.add(td / name, arcname=name)


# --------------------------------------------------------------------------- meshes
def read_mesh_file(path) -> tuple[np.ndarray, np.ndarray | None, np.ndarray]:
    """(vertices, vertex normals or None, triangles) of a .gts or .off file
    (the extension decides, src/bem/mesh.cpp:235-257)."""
    p = Path(path)
    if p.suffix == ".gts":
        V, N, T = read_gts(p)
        return V, N, T
    if p.suffix == ".off":
        V, T = read_off(p)
        return V, None, T
    raise FormatError(f"mesh filename {p} does not have either a GTS or OFF extension")


def _vertex_normals(V, N, T):
    """Supplied unit normals where given; the area-weighted mean of the
    adjacent triangles' planar normals where a row is zero."""
    if N is None:
        return None
    N = np.asarray(N, float)
    zero = ~np.any(N != 0.0, axis=1)
    if zero.all():
        return None
    bad = ~zero & (np.abs(np.linalg.norm(N, axis=1) - 1.0) > 1e-6)
    if bad.any():
        raise FormatError(f"supplied vertex normal {int(np.nonzero(bad)[0][0])} is not a unit vector")
    if zero.any():
        a, b, c = (V[T[:, i]] for i in range(3))
        cr = np.cross(b - a, c - a)  # 2 x area x planar normal
        acc = np.zeros_like(V)
        for i in range(3):
            np.add.at(acc, T[:, i], cr)
        acc /= np.linalg.norm(acc, axis=1, keepdims=True)
        N = np.where(zero[:, None], acc, N)
    return N


def load_mesh(path, xyzqr=None, planar: bool = False, qual_rule: int = DEFAULT_QUALS,
              quad_rule: int = DEFAULT_QUADS, skip_zeroes: bool = False):
    """A library mesh from a ``.mtz`` tarball, or from a ``.gts`` / ``.off``
    file and an xyzqr file.  From a tarball: the centre file sets the mesh
    centre, and a curved mesh takes its energy coefficients from the
    energies file (src/bem/mesh.cpp:100-140); a planar one, or a mesh from
    loose files, has them computed by the engine."""
    from .beep import Mesh
    p = Path(path)
    if p.suffix == ".mtz" or tarfile.is_tarfile(p):
        with MeshTarball(p) as mt:
            V, N, T = read_mesh_file(mt.get("mesh"))
            ch = read_xyzqr(mt.get("xyzqr"), skip_zeroes)
            centre = read_centre(mt.get("centre"))
            mesh = Mesh(V, T, ch[:, :4], planar=planar, qual_rule=qual_rule, quad_rule=quad_rule, centre=centre,
                        vertex_normals=_vertex_normals(V, N, T))
            if not planar:
                e = read_energies(mt.get("energies"), mesh.n_patches)
                mesh._energy_coef = (e.coef_f, e.coef_h)
            return mesh
    if xyzqr is None:
        raise FormatError(f"{p}: a mesh file needs an xyzqr charge file")
    V, N, T = read_mesh_file(p)
    ch = read_xyzqr(xyzqr, skip_zeroes)
    return Mesh(V, T, ch[:, :4], planar=planar, qual_rule=qual_rule, quad_rule=quad_rule,
                vertex_normals=_vertex_normals(V, N, T))


# --------------------------------------------------------------------------- XML config
@dataclass
class InstanceLayout:
    instance_id: int
    mesh_id: int
    dielectric: float
    offset: np.ndarray
    rotation: np.ndarray  # unit quaternion (a, b, c, d)
    quad: int  # -1: the default
    qual: int


@dataclass
class ConfigFile:
    """``<BEM_Config quad= qual=>`` with ``<solvent dielectric= kappa=>``,
    ``<output>``, ``<library><mesh id=>path</mesh>...`` (ids in order) and
    ``<layout><instance instance_id= mesh_id= dielectric= x= y= z= [a= b= c=
    d=] [quad= qual=]/>...`` (ids in order; the rotation is a unit
    quaternion, identity when absent)."""
    path: Path
    solvent_dielectric: float = 80.0
    solvent_kappa: float = 0.0
    output_file: str = ""
    default_quad: int = -1
    default_qual: int = -1
    mesh_library: list = field(default_factory=list)
    layout: list = field(default_factory=list)

    ROOT = "BEM_Config"

    @classmethod
    def read(cls, path) -> "ConfigFile":
        path = Path(path)
        try:
            root = ET.parse(path).getroot()
        except (ET.ParseError, OSError) as e:
            raise FormatError(f"failed to load file: {path}") from e
        if root.tag != cls.ROOT:
            raise FormatError(f"root element should be: {cls.ROOT} (got: {root.tag})")
        cfg = cls(path)

        def num(el, key, conv=float, required=True, default=None):
            v = el.get(key)
            if v is None:
                if required:
                    raise FormatError(f"{path}: missing {key} attribute in <{el.tag}>")
                return default
            try:
                return conv(v)
            except ValueError as e:
                raise FormatError(f"{path}: bad {key} attribute in <{el.tag}>") from e

        cfg.default_quad = num(root, "quad", int, False, -1)
        cfg.default_qual = num(root, "qual", int, False, -1)
        solvent = root.find("solvent")
        if solvent is None:
            raise FormatError(f"{path}: failed to find <solvent> tag (in which solvent dielectric & kappa are required)")
        cfg.solvent_dielectric = num(solvent, "dielectric")
        cfg.solvent_kappa = num(solvent, "kappa")
        out = root.find("output")
        if out is None:
            raise FormatError(f"{path}: failed to find an output tag")
        cfg.output_file = (out.text or "").strip()
        lib = root.find("library")
        for el in (list(lib) if lib is not None else []):
            if el.tag != "mesh":
                raise FormatError(f"{path}: expected <mesh> tags within <library> block")
            mid = num(el, "id", int)
            if mid != len(cfg.mesh_library):
                raise FormatError(f"{path}: mesh id's must correspond to ordering within <library> block")
            cfg.mesh_library.append((el.text or "").strip())
        lay = root.find("layout")
        if lay is None:
            raise FormatError(f"{path}: no <layout> block")
        for el in lay:
            if el.tag != "instance":
                raise FormatError(f"{path}: expected <instance> tags within <layout> block")
            iid, mid = num(el, "instance_id", int), num(el, "mesh_id", int)
            diel = num(el, "dielectric")
            xyz = np.array([num(el, k) for k in "xyz"])
            q = [num(el, k, float, False) for k in "abcd"]
            if any(v is None for v in q):
                q = [1.0, 0.0, 0.0, 0.0]
            if all(v == 0.0 for v in q):
                q[0] = 1.0
            q = np.array(q)
            if abs(np.linalg.norm(q) - 1.0) > 1e-3:
                raise FormatError(f"{path}: quaternion is not close to being a unit quaternion")
            q = q / np.linalg.norm(q)
            if iid != len(cfg.layout):
                raise FormatError(f"{path}: instance id's must correspond to ordering within <layout> block")
            if mid >= len(cfg.mesh_library):
                raise FormatError(f"{path}: invalid mesh_id in <instance>")
            cfg.layout.append(InstanceLayout(iid, mid, diel, xyz, q, num(el, "quad", int, False, cfg.default_quad),
                                             num(el, "qual", int, False, cfg.default_qual)))
        return cfg


def beep_from_config(cfg: ConfigFile, nbsize: int | None = None, precision: str = "fp64", device: int = 0,
                     planar: bool = False):
    """A BEEP scenario with the configuration's meshes and instances.  Mesh
    paths are relative to the configuration file; each (mesh, quadrature
    rules) pair is loaded once."""
    from .beep import BEEP, DEFAULT_NBSIZE
    bp = BEEP(eps_solvent=cfg.solvent_dielectric, kappa=cfg.solvent_kappa,
              nbsize=DEFAULT_NBSIZE if nbsize is None else nbsize, precision=precision, device=device)
    loaded = {}
    for inst in cfg.layout:
        qual = DEFAULT_QUALS if inst.qual < 0 else inst.qual
        quad = DEFAULT_QUADS if inst.quad < 0 else inst.quad
        key = (inst.mesh_id, qual, quad)
        if key not in loaded:
            mp = Path(cfg.mesh_library[inst.mesh_id])
            if not mp.is_absolute():
                mp = cfg.path.parent / mp
            loaded[key] = load_mesh(mp, planar=planar, qual_rule=qual, quad_rule=quad)
        bp.insert_mesh_instance(loaded[key], offset=inst.offset, rotation=inst.rotation, eps_protein=inst.dielectric)
    return bp
