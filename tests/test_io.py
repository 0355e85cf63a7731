"""Scene ingestion and image files (host only): the Mitsuba XML subset and
OBJ loaders, the built-in scene, and the PPM / HDR / EXR writers and the HDR
reader.  The loader cases restate the reference's own tests
(src/mitsuba.rs:599-838)."""
from __future__ import annotations

import math
import os
import struct
from pathlib import Path

import numpy as np
import pytest

from tinypt_b200 import _abi, io, scenes
from tinypt_b200.scene import Material, RenderConfig, Transform

CFG = RenderConfig(width=16, height=9)


def load(tmp_path, xml, cfg=CFG):
    p = tmp_path / "scene.xml"
    p.write_text(xml)
    ls, c = io.LoadedScene.from_xml(str(p), cfg)
    with ls:
        return ls.to_scene(), c, ls.warnings


def test_parses_shapes_and_materials(tmp_path):
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <sensor type="perspective">
        <float name="fov" value="40"/>
        <string name="fov_axis" value="y"/>
        <transform name="to_world"><lookat origin="0,1.2,4" target="0,0.5,0" up="0,1,0"/></transform>
      </sensor>
      <shape type="sphere">
        <point name="center" x="-1" y="0.5" z="0"/><float name="radius" value="0.5"/>
        <bsdf type="diffuse"><srgb name="reflectance" value="0.8,0.3,0.3"/></bsdf>
      </shape>
      <shape type="sphere">
        <point name="center" x="0" y="0.5" z="0"/><float name="radius" value="0.5"/>
        <bsdf type="roughconductor"><string name="distribution" value="ggx"/>
          <float name="alpha" value="0.25"/><rgb name="specular_reflectance" value="0.9,0.7,0.3"/></bsdf>
      </shape>
      <shape type="sphere">
        <point name="center" x="0" y="3" z="-1"/><float name="radius" value="0.8"/>
        <emitter type="area"><rgb name="radiance" value="8,7,5"/></emitter>
      </shape>
    </scene>""")
    assert len(scene.world.spheres) == 3 and len(scene.mats) == 3
    assert scene.mats[0].kind == _abi.TPT_MAT_LAMBERT
    assert scene.mats[1].kind == _abi.TPT_MAT_GGX and abs(scene.mats[1].param - 0.25) < 1e-12
    assert scene.mats[2].kind == _abi.TPT_MAT_DIFFUSE_LIGHT and scene.mats[2].rgb == (8.0, 7.0, 5.0)
    assert scene.cam.kind == _abi.TPT_CAMERA_LOOK_AT_DOF and scene.cam.fov_y_deg == 40.0
    assert scene.cam.eye == (0.0, 1.2, 4.0) and scene.cam.target == (0.0, 0.5, 0.0)
    assert scene.cam.aspect == 16 / 9


def test_srgb_tag_gamma_decodes_but_rgb_is_linear(tmp_path):
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <shape type="sphere"><bsdf type="diffuse"><srgb name="reflectance" value="0.8,0.8,0.8"/></bsdf></shape>
      <shape type="sphere"><bsdf type="diffuse"><rgb name="reflectance" value="0.8,0.8,0.8"/></bsdf></shape>
    </scene>""")
    srgb, lin = scene.mats[0].rgb[0], scene.mats[1].rgb[0]
    assert srgb == ((0.8 + 0.055) / 1.055) ** 2.4 and lin == 0.8 and srgb < lin


def test_reads_film_sampler_integrator_into_config(tmp_path):
    _, c, _ = load(tmp_path, """<scene version="3.0.0">
      <integrator type="path"><integer name="max_depth" value="12"/><integer name="rr_depth" value="5"/></integrator>
      <sampler type="independent"><integer name="sample_count" value="256"/></sampler>
      <film type="hdrfilm"><integer name="width" value="800"/><integer name="height" value="600"/></film>
      <shape type="sphere"><bsdf type="diffuse"/></shape>
    </scene>""")
    assert (c.width, c.height, c.spp, c.max_bounces, c.rr_start) == (800, 600, 256, 12, 5)


def test_parses_parametric_shapes(tmp_path):
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <shape type="rectangle"><bsdf type="diffuse"/></shape>
      <shape type="cube"><bsdf type="diffuse"/></shape>
      <shape type="disk"><bsdf type="diffuse"/></shape>
    </scene>""")
    assert [m.n_tris for m in scene.world.meshes] == [2, 12, 64]
    assert len(scene.world.instances) == 3
    # same vertices as the Python restatements of the canonical shapes
    for got, want in zip(scene.world.meshes, (scenes.unit_rectangle(0), scenes.unit_cube(1), scenes.unit_disk(2))):
        g = got.positions[got.indices].reshape(-1, 3, 3)
        w = want.positions[want.indices].reshape(-1, 3, 3)
        assert np.array_equal(g, w)


def test_parses_obj_mesh_with_transform(tmp_path):
    (tmp_path / "m.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <shape type="obj"><string name="filename" value="m.obj"/>
        <transform name="to_world"><translate x="10" y="0" z="0"/></transform>
        <bsdf type="diffuse"><rgb name="reflectance" value="0.5,0.5,0.5"/></bsdf></shape>
    </scene>""")
    assert len(scene.world.meshes) == 1 and scene.world.meshes[0].n_tris == 1 and len(scene.mats) == 1
    assert scene.world.instances[0].xform.apply_point([0.0, 0.0, 0.0]) == [10.0, 0.0, 0.0]


def test_constant_emitter_and_scale(tmp_path):
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <emitter type="constant"><rgb name="radiance" value="0.1,0.2,0.4"/></emitter>
      <shape type="sphere"><bsdf type="diffuse"/></shape></scene>""")
    assert scene.env.width == 1 and np.array_equal(scene.env.data.ravel(), [0.1, 0.2, 0.4])
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <emitter type="constant"><rgb name="radiance" value="1,1,1"/><float name="scale" value="3"/></emitter>
    </scene>""")
    assert np.array_equal(scene.env.data.ravel(), [3.0, 3.0, 3.0])


def test_no_env_emitter_defaults_to_black_background(tmp_path):
    scene, _, _ = load(tmp_path, '<scene version="3.0.0"><shape type="sphere"><bsdf type="diffuse"/></shape></scene>')
    assert scene.env is not None and np.all(scene.env.data == 0.0)


def test_unknown_bsdf_falls_back_to_diffuse(tmp_path):
    scene, _, warn = load(tmp_path, """<scene version="3.0.0">
      <shape type="sphere"><bsdf type="plastic"><rgb name="reflectance" value="0.2,0.4,0.6"/></bsdf></shape>
    </scene>""")
    assert len(scene.mats) == 1 and scene.mats[0].kind == _abi.TPT_MAT_LAMBERT
    assert scene.mats[0].rgb == (0.2, 0.4, 0.6)
    assert any("plastic" in w for w in warn)


def test_envmap_file_loads(tmp_path):
    img = np.random.default_rng(1).uniform(0.01, 4.0, (8, 16, 3))
    io.write_image(str(tmp_path / "env.hdr"), img)
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <emitter type="envmap"><string name="filename" value="env.hdr"/><float name="scale" value="2"/></emitter>
    </scene>""")
    assert (scene.env.width, scene.env.height) == (16, 8)
    assert np.allclose(scene.env.data, 2.0 * io.read_hdr(str(tmp_path / "env.hdr")))


def test_transforms_match_the_oracle(tmp_path, oracle_mod):
    """Instance transforms composed from translate / rotate / scale / matrix
    ops equal the oracle's restatement of src/transform.rs bit for bit."""
    scene, _, _ = load(tmp_path, """<scene version="3.0.0">
      <shape type="cube"><transform name="to_world">
        <translate x="0.9" y="0.5" z="0"/><rotate x="0.3" y="1" z="0.2" angle="35"/><scale x="0.6" y="1.0" z="0.6"/>
      </transform><bsdf type="diffuse"/></shape>
      <shape type="cube"><transform name="to_world">
        <translate x="-0.9" y="0.4" z="0"/><rotate x="0" y="1" z="0" angle="30"/><scale value="0.8"/>
      </transform><bsdf type="diffuse"/></shape>
      <shape type="cube"><transform name="to_world">
        <matrix value="1 0 0 2  0 0 -1 3  0 1 0 4  0 0 0 1"/><rotate x="1" angle="90"/>
      </transform><bsdf type="diffuse"/></shape>
    </scene>""")
    ops = [
        [(0, (0.9, 0.5, 0.0, 0, 0)), (2, (0.3, 1.0, 0.2, 35.0, 0)), (1, (0.6, 1.0, 0.6, 0, 0))],
        [(0, (-0.9, 0.4, 0.0, 0, 0)), (2, (0.0, 1.0, 0.0, 30.0, 0)), (1, (0.8, 0.8, 0.8, 0, 0))],
    ]
    for inst, op in zip(scene.world.instances, ops):
        _, at = oracle_mod.transform(op, 0, [0.0, 0.0, 0.0])
        assert np.array_equal(np.array(inst.xform.a).ravel(), at[:9]) and np.array_equal(inst.xform.t, at[9:])
    m = scene.world.instances[2].xform
    want = Transform.from_affine([[1, 0, 0], [0, 0, -1], [0, 1, 0]], [2, 3, 4]).compose(
        Transform.rotate((1.0, 0.0, 0.0), 90.0))
    assert np.array_equal(np.array(m.a), np.array(want.a)) and m.t == want.t


def test_obj_faces_indices_and_polygons(tmp_path):
    (tmp_path / "p.obj").write_text(
        "# comment\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\nvt 0 0\n"
        "f 1/1/1 2/1/1 3/1/1 4/1/1\nf -4 -2 -1\nf 1 2\nf 9 1 2 3\n")
    m = io.load_obj_via_xml(str(tmp_path / "p.obj"))
    # quad fan (2), negative indices (1), too short (0), out-of-range index dropped -> (1 2 3) fan (1)
    assert m.indices.tolist() == [[0, 1, 2], [0, 2, 3], [0, 2, 3], [0, 1, 2]]


@pytest.mark.parametrize("xml, message", [
    ("", "empty XML"),
    ("this is not xml <<<", "bad XML tag"),
    ("<scene version='3.0.0'><shape type='sphere'></scene>", "unbalanced XML"),
    ("<scene version='3.0.0'><shape type='sphere'>", "unbalanced XML"),
    ("<foo/>", "root element is not <scene>"),
])
def test_malformed_xml_is_an_error(tmp_path, xml, message):
    """src/mitsuba.rs:137-141, 262-300: a file that does not parse, or whose
    root is not <scene>, fails the load (InvalidData)."""
    with pytest.raises(_abi.TinyptError, match=message):
        load(tmp_path, xml)
    with pytest.raises(_abi.TinyptError, match="cannot open"):
        io.LoadedScene.from_xml(str(tmp_path / "absent.xml"), CFG)


def test_missing_files_and_bad_ops_are_warnings(tmp_path):
    """What the reference only warns about (src/mitsuba.rs:226-250, 376-398,
    496-540): a missing OBJ or env map file, an OBJ shape without a filename,
    an unknown shape type, a matrix without 16 values and a rotation about a
    zero axis are skipped and the scene still loads."""
    scene, _, warn = load(tmp_path, """<scene version="3.0.0">
      <emitter type="envmap"><string name="filename" value="nope.hdr"/></emitter>
      <shape type="obj"><string name="filename" value="nope.obj"/><bsdf type="diffuse"/></shape>
      <shape type="obj"><bsdf type="diffuse"/></shape>
      <shape type="teapot"><bsdf type="diffuse"/></shape>
      <shape type="cube"><bsdf type="diffuse"/>
        <transform name="to_world"><matrix value="1 0 0"/><rotate x="0" y="0" z="0" angle="30"/>
          <translate x="1"/></transform></shape>
    </scene>""")
    text = "\n".join(warn)
    for w in ("failed to load envmap", "failed to load obj", "obj shape without filename",
              "unsupported shape type 'teapot', skipped", "matrix expects 16 values, got 3; ignored",
              "rotate with zero axis; ignored"):
        assert w in text, w
    # only the cube is left, translated by the one valid op; the env is black
    assert len(scene.world.meshes) == 1 and len(scene.world.instances) == 1
    m = scene.world.instances[0].xform
    assert np.array_equal(np.array(m.a), np.eye(3)) and tuple(m.t) == (1.0, 0.0, 0.0)
    assert scene.env is not None and float(np.max(np.abs(scene.env.data))) == 0.0


def test_malformed_obj_lines_follow_the_reference(tmp_path):
    """src/obj_loader.rs:11-53: unparsable coordinates read as 0, lines are
    trimmed and need "v " / "f " prefixes, an index resolves against the
    vertices read so far (negative ones relative to them), invalid indices
    are dropped and a face left with fewer than 3 is skipped."""
    (tmp_path / "m.obj").write_text(
        "  v 1 2\n\tv\t3 4 5\nv a b c\nf 1 2 7\nf x y z\nf 1 2 3 4\nv 0 1 0\nf -3 -2 -1\n")
    m = io.load_obj_via_xml(str(tmp_path / "m.obj"))
    assert m.positions.reshape(-1, 3).tolist() == [[1, 2, 0], [0, 0, 0], [0, 1, 0]]
    assert m.indices.reshape(-1, 3).tolist() == [[0, 1, 2]]


def test_default_scene_matches_the_python_restatement():
    cfg = RenderConfig(width=320, height=180)
    with io.LoadedScene.default(cfg) as ls:
        got = ls.to_scene()
    want = scenes.build_scene(320, 180)
    assert [(m.kind, m.rgb, m.param) for m in got.mats] == [(m.kind, m.rgb, m.param) for m in want.mats]
    assert [(s.c, s.r, s.mat_id) for s in got.world.spheres] == [(tuple(s.c), s.r, s.mat_id) for s in want.world.spheres]
    assert got.env is None
    c, w = got.cam, want.cam
    assert (c.kind, c.eye, c.target, c.up, c.fov_y_deg, c.aspect) == (w.kind, w.eye, w.target, w.up, w.fov_y_deg,
                                                                     w.aspect)
    assert math.isclose(c.focus_dist, w.focus_dist, rel_tol=0, abs_tol=0) and c.aperture == w.aperture


_SAMPLES_ENV = os.environ.get("TINYPT_REFERENCE_SAMPLES", "")
REF_SAMPLES = Path(_SAMPLES_ENV) if _SAMPLES_ENV else None


@pytest.mark.skipif(REF_SAMPLES is None or not REF_SAMPLES.is_dir(),
                    reason="TINYPT_REFERENCE_SAMPLES does not name the reference's sample/ directory")
def test_reference_sample_scenes_load():
    counts = {}
    for name in ("default.xml", "cornell.xml", "env_scene.xml", "mesh.xml"):
        ls, cfg = io.LoadedScene.from_xml(str(REF_SAMPLES / name), CFG)
        with ls:
            s = ls.to_scene()
            counts[name] = (len(s.world.spheres), [m.n_tris for m in s.world.meshes], len(s.mats))
    assert counts["default.xml"][0] == 6
    assert counts["mesh.xml"][1] == [12, 12]          # two instances of sample/cube.obj
    assert counts["cornell.xml"][1].count(2) == 6 and counts["cornell.xml"][1].count(12) == 2


# ---- images -------------------------------------------------------------------------------------
def _srgb8(x):
    x = min(max(x, 0.0), 1.0)
    v = 12.92 * x if x <= 0.0031308 else 1.055 * x ** (1.0 / 2.4) - 0.055
    return int(v * 255.0 + 0.5)


def test_ppm_pipeline(tmp_path):
    img = np.array([[[0.0, 0.5, 2.0], [0.02, 0.18, 1.0]]])
    for tm, ev in (("none", 0.0), ("aces", 1.0)):
        p = tmp_path / f"o_{tm}.ppm"
        io.write_image(str(p), img, exposure=ev, tonemap=tm)
        lines = p.read_text().split("\n")
        assert lines[:3] == ["P3", "2 1", "255"]
        vals = [int(v) for v in lines[3].split()]

        def tone(x):
            x *= 2.0 ** ev
            if tm == "aces":
                x = max(x, 0.0)
                x = min(max((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0), 1.0)
            return _srgb8(x)
        assert vals == [tone(v) for v in img.ravel()]


def test_hdr_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    for w in (5, 40):  # flat and run-length scanlines
        img = rng.lognormal(0.0, 2.0, (7, w, 3))
        img[0, :] = 0.0
        img[1, :] = 1.5                  # long runs
        p = tmp_path / f"x{w}.hdr"
        io.write_image(str(p), img)
        back = io.read_hdr(str(p))
        assert back.shape == img.shape
        assert np.all(back[0] == 0.0)
        m = img.max(axis=2, keepdims=True)
        assert np.all(np.abs(back - img) <= m / 128.0)    # 8-bit shared-exponent mantissas


def test_reference_output_unit_tests(tmp_path):
    """src/output.rs:134-200 restated: the format follows the extension,
    case-insensitively, with PPM for anything else; PPM applies the exact
    sRGB curve even at exposure 0 without tonemap (0 -> 0, 1 -> 255, 2
    clamps); the RGBE round trip of the reference's 2x2 image stays within
    pmax/128 + 1e-6 per channel."""
    img = np.array([[[0.25, 0.5, 1.0], [2.0, 0.1, 0.0]], [[0.0, 0.0, 0.0], [8.0, 4.0, 2.0]]])
    for name, head in (("out.exr", b"\x76\x2f\x31\x01"), ("OUT.EXR", b"\x76\x2f\x31\x01"),
                       ("out.hdr", b"#?RADIANCE"), ("out.HDR", b"#?RADIANCE"),
                       ("out.ppm", b"P3"), ("out.txt", b"P3"), ("out", b"P3")):
        io.write_image(str(tmp_path / name), img, tonemap="none")
        assert (tmp_path / name).read_bytes().startswith(head), name
    p = tmp_path / "s.ppm"
    io.write_image(str(p), np.array([[[0.5, 0.0, 1.0], [2.0, 0.5, 0.5]]]), exposure=0.0, tonemap="none")
    vals = [int(v) for v in p.read_text().split("\n")[3].split()]
    assert vals[:4] == [_srgb8(0.5), 0, 255, 255]
    p = tmp_path / "r.hdr"
    io.write_image(str(p), img)
    back = io.read_hdr(str(p))
    assert back.shape == (2, 2, 3)
    pmax = img.max(axis=2, keepdims=True)
    assert np.all(np.abs(back - img) <= pmax / 128.0 + 1e-6)


def test_exr_layout_and_acescg(tmp_path):
    img = np.array([[[1.0, 1.0, 1.0], [1.0, 0.0, 0.0]], [[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]])
    p = tmp_path / "o.exr"
    io.write_image(str(p), img)
    b = p.read_bytes()
    assert struct.unpack("<II", b[:8]) == (20000630, 2)
    assert b"channels\0chlist\0" in b and b"dataWindow\0box2i\0" in b and b"compression\0compression\0" in b
    hdr_end = b.index(b"screenWindowWidth\0float\0") + len(b"screenWindowWidth\0float\0") + 4 + 4 + 1
    offs = struct.unpack("<2Q", b[hdr_end:hdr_end + 16])
    rows = []
    for o in offs:
        y, n = struct.unpack("<ii", b[o:o + 8])
        f = np.frombuffer(b[o + 8:o + 8 + n], dtype="<f4").reshape(3, 2)   # B, G, R planes
        rows.append(f[::-1].T)                                             # -> (x, rgb)
    got = np.stack(rows)
    # white stays white; the primaries map to the columns of the sRGB -> ACEScg matrix
    assert np.allclose(got[0, 0], 1.0, atol=2e-3)
    m = np.stack([got[0, 1], got[1, 0], got[1, 1]], 1)
    want = np.array([[0.6131, 0.3395, 0.0474], [0.0702, 0.9164, 0.0134], [0.0206, 0.1096, 0.8698]])
    assert np.allclose(m, want, atol=2e-3)


# ---- checkpoints ----------------------------------------------------------------------------
def test_film_tiles_match_the_oracle(oracle_mod):
    for w, h, t, m in ((40, 23, 16, True), (64, 64, 8, True), (50, 10, 16, False), (1, 1, 16, True)):
        assert np.array_equal(io.film_tiles(w, h, t, m), oracle_mod.tile_order(w, h, t, m))


def test_checkpoint_roundtrip_and_format(tmp_path):
    w, h = 7, 5
    rng = np.random.default_rng(2)
    acc, acc_w = rng.standard_normal((w * h, 3)), rng.integers(0, 9, w * h).astype(np.float64)
    p = tmp_path / "checkpoint_0000000000000001.bin"
    io.save_checkpoint(str(p), 0x4859503000000001, w, h, 11, acc, acc_w)
    b = p.read_bytes()
    assert b[:8] == b"HYPCKPT\0"
    assert struct.unpack("<IQIIQ", b[8:36]) == (1, 0x4859503000000001, w, h, 11)
    assert len(b) == 36 + 8 * 4 * w * h
    assert np.array_equal(np.frombuffer(b[36:36 + 24 * w * h], "<f8").reshape(-1, 3), acc)
    nid, a2, w2 = io.load_checkpoint(str(p), 0x4859503000000001, w, h)
    assert nid == 11 and np.array_equal(a2, acc) and np.array_equal(w2, acc_w)
    # another scene, size or version is not resumed (src/checkpoint.rs:86-138)
    assert io.load_checkpoint(str(p), 0x4859503000000002, w, h) is None
    assert io.load_checkpoint(str(p), 0x4859503000000001, w + 1, h) is None
    assert io.load_checkpoint(str(tmp_path / "absent.bin"), 1, w, h) is None
    bad = bytearray(b)
    bad[8] = 2
    (tmp_path / "v2.bin").write_bytes(bytes(bad))
    assert io.load_checkpoint(str(tmp_path / "v2.bin"), 0x4859503000000001, w, h) is None
    bad = bytearray(b)
    bad[0] = ord("X")
    (tmp_path / "magic.bin").write_bytes(bytes(bad))
    assert io.load_checkpoint(str(tmp_path / "magic.bin"), 0x4859503000000001, w, h) is None


@pytest.mark.parametrize("keep", [0, 3, 8, 20, 35, 36, 36 + 24 * 35, 36 + 32 * 35 - 1])
def test_truncated_checkpoint_is_an_io_error(tmp_path, keep):
    """A checkpoint that ends early -- in the magic, the header or the film
    -- is an I/O error, as read_exact makes it in src/checkpoint.rs:86-138
    (a file that matches up to where it ends is not mistaken for 'absent')."""
    w, h = 7, 5
    acc, acc_w = np.ones((w * h, 3)), np.ones(w * h)
    p = tmp_path / "ck.bin"
    io.save_checkpoint(str(p), 9, w, h, 3, acc, acc_w)
    b = p.read_bytes()
    assert len(b) == 36 + 32 * w * h
    p.write_bytes(b[:keep])
    with pytest.raises(RuntimeError, match="truncated checkpoint"):
        io.load_checkpoint(str(p), 9, w, h)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [_abi.TPT_MODE_PLAIN_F64, _abi.TPT_MODE_WAVEFRONT_FP32])
def test_resume_from_partial_checkpoint(gpu, tmp_path, mode):
    """A checkpoint holding the first k tiles (as the reference's renderer
    leaves one mid-frame) resumes to the whole-film render, and the final
    checkpoint lists every tile."""
    from tinypt_b200.render import DeviceScene

    cfg = RenderConfig(width=40, height=24, spp=8, max_bounces=6, rr_start=3, seed=4, tile=8, mode=mode)
    scene = scenes.sphere_scene(cfg.width, cfg.height)
    tiles = io.film_tiles(cfg.width, cfg.height, 8, True)
    k = len(tiles) // 3
    with DeviceScene(scene) as ds:
        full = ds.render(cfg)
        part_a = np.zeros_like(full.acc)
        part_w = np.zeros_like(full.acc_w)
        for x0, y0, x1, y1 in tiles[:k]:
            for y in range(y0, y1):
                sl = slice(y * cfg.width + x0, y * cfg.width + x1)
                part_a[sl], part_w[sl] = full.acc[sl], full.acc_w[sl]
        p = tmp_path / "ck.bin"
        io.save_checkpoint(str(p), 77, cfg.width, cfg.height, k, part_a, part_w)
        out = ds.render_resume(cfg, str(p), 77)
    assert np.array_equal(out.acc, full.acc) and np.array_equal(out.acc_w, full.acc_w)
    nid, a, w = io.load_checkpoint(str(p), 77, cfg.width, cfg.height)
    assert nid == len(tiles) and np.array_equal(a, full.acc)


@pytest.mark.gpu
def test_resume_ignores_an_unreadable_checkpoint_and_a_failed_save(gpu, tmp_path, capfd):
    """src/render.rs:56-68 resumes only on Ok(Some(..)): a truncated file is
    rendered over from scratch and replaced by the final checkpoint; a final
    save that fails is reported on stderr and the film still comes back
    (src/render.rs:268-272)."""
    from tinypt_b200.render import DeviceScene

    cfg = RenderConfig(width=40, height=24, spp=4, max_bounces=4, rr_start=3, seed=5, tile=8,
                       mode=_abi.TPT_MODE_WAVEFRONT_FP32)
    scene = scenes.sphere_scene(cfg.width, cfg.height)
    n_tiles = len(io.film_tiles(cfg.width, cfg.height, 8, True))
    p = tmp_path / "ck.bin"
    io.save_checkpoint(str(p), 5, cfg.width, cfg.height, 2, np.full((cfg.width * cfg.height, 3), 9.0),
                       np.full(cfg.width * cfg.height, 9.0))
    p.write_bytes(p.read_bytes()[:100])
    with DeviceScene(scene) as ds:
        full = ds.render(cfg)
        out = ds.render_resume(cfg, str(p), 5)
        assert np.array_equal(out.acc, full.acc) and np.array_equal(out.acc_w, full.acc_w)
        nid, a, _ = io.load_checkpoint(str(p), 5, cfg.width, cfg.height)
        assert nid == n_tiles and np.array_equal(a, full.acc)
        out = ds.render_resume(cfg, str(tmp_path / "no_such_dir" / "ck.bin"), 5)
    assert np.array_equal(out.acc, full.acc)
    assert "Final checkpoint save failed" in capfd.readouterr().err
