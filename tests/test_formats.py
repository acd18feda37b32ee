"""The reference's on-disk inputs (GTS / OFF surfaces, xyzqr charges, .mtz
mesh tarballs, the BEM_Config XML run description) read on the host.  The
reference ships no sample files, so the cases are written here: by the
writers (round trips), and by hand where a format has variants the writers
do not produce (comments, header-less OFF, missing normals, optional
fields)."""
import tarfile

import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200 import formats as F


def cyc_equal(T1, T2):
    """Triangle lists equal up to a cyclic rotation of each triangle."""
    if T1.shape != T2.shape:
        return False
    for t1, t2 in zip(T1.tolist(), T2.tolist()):
        if t1 not in (t2, t2[1:] + t2[:1], t2[2:] + t2[:2]):
            return False
    return True


def test_gts_round_trip_and_patches(tmp_path):
    V, T = b.icosphere(2, 10.0)
    F.write_gts(tmp_path / "s.gts", V, T)
    V2, N2, T2 = F.read_gts(tmp_path / "s.gts")
    assert np.array_equal(V2, V) and cyc_equal(T2, T) and not N2.any()
    ch = b.charges_in_sphere(5, 6.0, seed=1)
    m1 = b.Mesh(V, T, ch)
    m2 = F.load_mesh(tmp_path / "s.gts", xyzqr=_xyzqr(tmp_path, ch))
    assert np.allclose(m2.patches.area, m1.patches.area, rtol=1e-14)
    assert np.allclose(m2.patches.qual, m1.patches.qual, rtol=1e-13, atol=1e-13)


def _xyzqr(tmp_path, ch):
    F.write_xyzqr(tmp_path / "c.xyzqr", ch)
    return tmp_path / "c.xyzqr"


def test_gts_by_hand_comments_and_normals(tmp_path):
    # a tetrahedron: edges 1-2 1-3 1-4 2-3 2-4 3-4, faces as edge triples
    text = """# comment
! another comment
4 6 4 GtsSurface GtsFace GtsEdge GtsVertex
0 0 0 -0.5773502691896258 -0.5773502691896258 -0.5773502691896258
1 0 0
0 1 0
0 0 1
1 2
1 3
1 4
2 3
2 4
3 4
2 1 4
1 3 5
4 6 5
3 6 2
"""
    (tmp_path / "t.gts").write_text(text)
    V, N, T = F.read_gts(tmp_path / "t.gts")
    assert V.shape == (4, 3) and T.shape == (4, 3)
    assert np.allclose(N[0], -np.ones(3) / np.sqrt(3)) and not N[1:].any()
    # face (2 1 4): edges (1 3), (1 2), (2 3) share 1, then 2, then 3
    assert T[0].tolist() == [0, 1, 2]
    assert sorted(map(tuple, np.sort(T, axis=1).tolist())) == [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
    # supplied normals are kept, zero ones computed
    Nm = F._vertex_normals(V, N, T)
    assert np.allclose(Nm[0], N[0]) and np.allclose(np.linalg.norm(Nm, axis=1), 1.0)


def test_gts_errors(tmp_path):
    (tmp_path / "bad.gts").write_text("4 5 4\n")
    with pytest.raises(F.FormatError):
        F.read_gts(tmp_path / "bad.gts")
    (tmp_path / "short.gts").write_text("4 6 4\n0 0 0\n")
    with pytest.raises(F.FormatError):
        F.read_gts(tmp_path / "short.gts")


@pytest.mark.parametrize("header", ["OFF\n", "nOFF\n", ""])
def test_off_variants(tmp_path, header):
    V, T = b.icosphere(1, 3.0)
    body = f"{len(V)} {len(T)} {3 * len(T) // 2}\n" + "".join(
        " ".join(repr(float(x)) for x in v) + "\n" for v in V) + "# a comment line\n" + "".join(
        f"3 {t[0]} {t[1]} {t[2]}\n" for t in T)
    (tmp_path / "s.off").write_text("# made by hand\n" + header + body)
    V2, T2 = F.read_off(tmp_path / "s.off")
    assert np.array_equal(V2, V) and np.array_equal(T2, T)


def test_off_rejects_non_triangles(tmp_path):
    (tmp_path / "q.off").write_text("OFF\n4 1 4\n0 0 0\n1 0 0\n1 1 0\n0 1 0\n4 0 1 2 3\n")
    with pytest.raises(F.FormatError):
        F.read_off(tmp_path / "q.off")
    with pytest.raises(F.FormatError):
        F.read_mesh_file(tmp_path / "q.ply")


def test_xyzqr_rules(tmp_path):
    (tmp_path / "c.xyzqr").write_text(
        "1 2 3 0.5 1.8\n"            # plain charge
        "0 0 0 0.0 1.5\n"            # zero charge, no other parameters: skipped
        "4 5 6 0.0 1.2 0.3\n"        # zero charge with a hydrophobicity: kept
        "7 8 9 0.0 1.2 0 3.1 0.2\n"  # zero charge with a Lennard-Jones pair: kept
        "\n"
        "1 1 1 -1 2.0 0.1 3.0 0.0\n")
    ch = F.read_xyzqr(tmp_path / "c.xyzqr")
    assert ch.shape == (4, 8)
    assert ch[:, 3].tolist() == [0.5, 0.0, 0.0, -1.0]
    assert ch[1, 5] == 0.3 and ch[2, 6] == 3.1
    assert F.read_xyzqr(tmp_path / "c.xyzqr", skip_zeroes=True)[:, 3].tolist() == [0.5, -1.0]
    (tmp_path / "bad.xyzqr").write_text("1 2 3\n")
    with pytest.raises(F.FormatError):
        F.read_xyzqr(tmp_path / "bad.xyzqr")


def test_mtz_round_trip(tmp_path):
    V, T = b.icosphere(2, 10.0)
    ch = b.charges_in_sphere(5, 6.0, seed=2)
    centre = np.array([0.1, -0.2, 0.3])
    cf, chh = np.linspace(0, 1, len(V)), np.linspace(1, 2, len(V))
    for fmt in ("gts", "off"):
        F.write_mtz(tmp_path / f"m_{fmt}.mtz", V, T, ch, centre, cf, chh, mesh_format=fmt)
        mesh = F.load_mesh(tmp_path / f"m_{fmt}.mtz")
        assert np.array_equal(mesh.centre, centre)
        assert np.allclose(mesh.charges, ch)
        # curved meshes take their energy coefficients from the tarball
        assert np.array_equal(mesh._energy_coef[0], cf) and np.array_equal(mesh._energy_coef[1], chh)
        ref = b.Mesh(V, T, ch, centre=centre)
        assert np.allclose(mesh.patches.area, ref.patches.area, rtol=1e-14)
        planar = F.load_mesh(tmp_path / f"m_{fmt}.mtz", planar=True)
        assert planar._energy_coef is None


def _tarball(path, files: dict):
    with tarfile.open(path, "w:gz") as tar:
        for name, text in files.items():
            p = path.parent / ("_" + name)
            p.write_text(text)
            tar.add(p, arcname=name)


def test_mtz_definition_errors(tmp_path):
    good = "<contents><mesh>m.gts</mesh><xyzqr>c</xyzqr><centre>x</centre><energies>e</energies></contents>"
    _tarball(tmp_path / "ok.mtz", {"definition.xml": good, "m.gts": "", "c": "", "x": "0 0 0", "e": ""})
    with F.MeshTarball(tmp_path / "ok.mtz") as mt:
        assert mt.get("mesh").name == "m.gts" and mt.get("fh") is None
        work = mt.work_dir
    assert not work.exists()  # the temporary folder is removed
    missing = "<contents><mesh>m.gts</mesh><xyzqr>c</xyzqr><centre>x</centre></contents>"
    _tarball(tmp_path / "missing.mtz", {"definition.xml": missing})
    with pytest.raises(F.FormatError, match="energies"):
        F.MeshTarball(tmp_path / "missing.mtz")
    twice = good.replace("</contents>", "<mesh>n.gts</mesh></contents>")
    _tarball(tmp_path / "twice.mtz", {"definition.xml": twice})
    with pytest.raises(F.FormatError, match="multiple"):
        F.MeshTarball(tmp_path / "twice.mtz")
    _tarball(tmp_path / "root.mtz", {"definition.xml": "<stuff/>"})
    with pytest.raises(F.FormatError, match="root"):
        F.MeshTarball(tmp_path / "root.mtz")


CONFIG = """<?xml version="1.0"?>
<BEM_Config qual="4" quad="0">
  <solvent dielectric="80.0" kappa="0.1"/>
  <output>out.txt</output>
  <library>
    <mesh id="0">a.mtz</mesh>
    <mesh id="1">b.mtz</mesh>
  </library>
  <layout>
    <instance instance_id="0" mesh_id="0" dielectric="2.0" x="0" y="0" z="0"/>
    <instance instance_id="1" mesh_id="1" dielectric="4.0" x="30" y="0" z="5" a="0.7071067811865476" b="0" c="0.7071067811865476" d="0"/>
    <instance instance_id="2" mesh_id="0" dielectric="2.0" x="-30" y="1" z="0" a="0" b="0" c="0" d="0" qual="1"/>
  </layout>
</BEM_Config>
"""


def test_config_file_and_scenario(tmp_path):
    for name, k, seed in (("a.mtz", 1, 3), ("b.mtz", 2, 4)):
        V, T = b.icosphere(k, 5.0)
        F.write_mtz(tmp_path / name, V, T, b.charges_in_sphere(3, 3.0, seed=seed), np.zeros(3))
    (tmp_path / "run.xml").write_text(CONFIG)
    cfg = F.ConfigFile.read(tmp_path / "run.xml")
    assert cfg.solvent_dielectric == 80.0 and cfg.solvent_kappa == 0.1 and cfg.output_file == "out.txt"
    assert cfg.mesh_library == ["a.mtz", "b.mtz"] and len(cfg.layout) == 3
    assert np.allclose(cfg.layout[1].rotation, [0.7071067811865476, 0, 0.7071067811865476, 0])
    assert cfg.layout[2].rotation.tolist() == [1.0, 0.0, 0.0, 0.0]  # an all-zero quaternion means no rotation
    assert cfg.layout[2].qual == 1 and cfg.layout[0].qual == 4
    bp = F.beep_from_config(cfg)
    assert len(bp.instances) == 3 and bp.kappa == 0.1 and bp.eps_solvent == 80.0
    assert bp.instances[1].eps_protein == 4.0 and np.allclose(bp.instances[1].offset, [30, 0, 5])
    # mesh 0 is loaded twice: once per quadrature rule
    assert bp.instances[0].mesh is not bp.instances[2].mesh
    assert bp.num_patches == 2 * 42 + 162


@pytest.mark.parametrize("edit, match", [
    (lambda s: s.replace('<solvent dielectric="80.0" kappa="0.1"/>', ""), "solvent"),
    (lambda s: s.replace('<mesh id="1">', '<mesh id="2">'), "ordering"),
    (lambda s: s.replace('instance_id="2"', 'instance_id="5"'), "ordering"),
    (lambda s: s.replace('a="0.7071067811865476"', 'a="0.9"'), "unit quaternion"),
    (lambda s: s.replace('mesh_id="1"', 'mesh_id="7"'), "mesh_id"),
    (lambda s: s.replace("BEM_Config", "Config"), "root element"),
])
def test_config_file_errors(tmp_path, edit, match):
    (tmp_path / "run.xml").write_text(edit(CONFIG))
    with pytest.raises(F.FormatError, match=match):
        F.ConfigFile.read(tmp_path / "run.xml")
