"""The command-line renderer (tinypt_b200/bin/tinypt, the reference's flags):
its flag parsing against src/main.rs:16-140 (on the CPU, through --dry-run),
and a Mitsuba XML scene rendered on the GPU and written as PPM / HDR,
identical to the same render through the Python API."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from tinypt_b200 import io
from tinypt_b200.build import CLI
from tinypt_b200.scene import RenderConfig

XML = """<scene version="3.0.0">
  <integrator type="path"><integer name="max_depth" value="6"/></integrator>
  <sampler type="independent"><integer name="sample_count" value="4"/></sampler>
  <film type="hdrfilm"><integer name="width" value="48"/><integer name="height" value="27"/></film>
  <sensor type="perspective"><float name="fov" value="40"/><string name="fov_axis" value="y"/>
    <transform name="to_world"><lookat origin="0,1.2,4" target="0,0.5,0" up="0,1,0"/></transform></sensor>
  <shape type="sphere"><point name="center" x="0" y="-1000" z="0"/><float name="radius" value="1000"/>
    <bsdf type="diffuse"><srgb name="reflectance" value="0.5,0.5,0.5"/></bsdf></shape>
  <shape type="cube"><transform name="to_world"><translate x="-0.8" y="0.4" z="0"/>
    <rotate x="0" y="1" z="0" angle="30"/><scale value="0.4"/></transform>
    <bsdf type="roughconductor"><float name="alpha" value="0.2"/></bsdf></shape>
  <shape type="sphere"><point name="center" x="0.8" y="0.5" z="0"/><float name="radius" value="0.5"/>
    <bsdf type="dielectric"/></shape>
  <shape type="rectangle"><transform name="to_world"><translate x="0" y="3" z="0"/>
    <rotate x="1" angle="90"/><scale value="0.5"/></transform>
    <emitter type="area"><rgb name="radiance" value="10,10,10"/></emitter></shape>
  <emitter type="constant"><rgb name="radiance" value="0.1,0.1,0.15"/></emitter>
</scene>"""


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["wavefront", "plain"])
def test_cli_renders_xml_scene(gpu, tmp_path, mode):
    from tinypt_b200 import _abi
    from tinypt_b200.render import DeviceScene

    assert CLI.exists(), "build() links the command-line renderer"
    xml = tmp_path / "s.xml"
    xml.write_text(XML)
    for ext in ("ppm", "hdr"):
        out = tmp_path / f"o_{mode}.{ext}"
        r = subprocess.run([str(CLI), "--scene", str(xml), "-o", str(out), "--seed", "3", "--mode", mode,
                            "--no-denoise"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert "Done in" in r.stderr
    # the same render through the Python API writes the same bytes
    ls, cfg = io.LoadedScene.from_xml(str(xml), RenderConfig(width=16, height=9, seed=3))
    cfg.mode = _abi.TPT_MODE_WAVEFRONT_FP32 if mode == "wavefront" else _abi.TPT_MODE_PLAIN_F64
    with ls, DeviceScene(ls.to_scene()) as ds:
        assert (cfg.width, cfg.height, cfg.spp, cfg.max_bounces) == (48, 27, 4, 6)
        o = ds.render(cfg)
    px = (o.acc / np.maximum(o.acc_w, 1.0)[:, None]).reshape(27, 48, 3)
    assert np.all(o.acc_w == 4) and px.max() > 0.0
    mine = tmp_path / f"py_{mode}.ppm"
    io.write_image(str(mine), px)
    assert mine.read_bytes() == (tmp_path / f"o_{mode}.ppm").read_bytes()
    hdr = io.read_hdr(str(tmp_path / f"o_{mode}.hdr"))
    assert hdr.shape == (27, 48, 3) and np.allclose(hdr, px, rtol=1.0 / 64, atol=1e-6)


# RenderConfig::default (src/config.rs:67-92) and main.rs's own defaults
DEFAULTS = dict(width="1920", height="1080", spp="512", max_bounces="8", rr_start="3", tile="16", adaptive="0",
                adaptive_min_spp="8", adaptive_threshold="0.02", morton="1", seed="0", mode="wavefront",
                denoise="1", tonemap="aces", exposure="0", out="out.ppm", env="-", scene="-")


def dry_run(*args):
    r = subprocess.run([str(CLI), "--dry-run", *args], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return dict(kv.split("=", 1) for kv in r.stdout.split())


def test_cli_defaults_are_the_reference_defaults():
    assert dry_run() == DEFAULTS


@pytest.mark.parametrize("args, changed", [
    (["--spp", "0"], {"spp": "1"}),                       # n.max(1)
    (["--spp", "+7"], {"spp": "7"}),                      # usize::from_str takes a '+'
    (["--spp", "-5"], {}),                                # not a usize: ignored
    (["--spp", " 7"], {}),                                # no surrounding spaces
    (["--spp", "99999999999999999999999"], {}),           # overflow: ignored
    (["--spp"], {}),                                      # flag without a value
    (["--adaptive", "--adaptive-min-spp", "0"], {"adaptive": "1", "adaptive_min_spp": "1"}),
    (["--adaptive-threshold", "-1"], {"adaptive_threshold": "0"}),
    (["--adaptive-threshold", "nan"], {"adaptive_threshold": "0"}),   # f64::max(NaN, 0.0) = 0
    (["--adaptive-threshold", "1e-3"], {"adaptive_threshold": "0.001"}),
    (["--adaptive-threshold", "0x1p-3"], {}),             # no hex floats in Rust
    (["--seed", "18446744073709551615"], {"seed": "18446744073709551615"}),
    (["--seed", "18446744073709551616"], {}),
    (["--tonemap", "none", "--exposure", "-1.5"], {"tonemap": "none", "exposure": "-1.5"}),
    (["--tonemap", "reinhard"], {}),                      # Tonemap::from_str: none | aces
    (["--no-denoise", "--no-morton", "-o", "x.hdr"], {"denoise": "0", "morton": "0", "out": "x.hdr"}),
    (["--bogus", "3", "--adaptive"], {"adaptive": "1"}),  # unknown flags are ignored
    (["--no-adaptive"], {}),
    (["--mode", "plain"], {"mode": "plain"}),
])
def test_cli_flag_parsing_follows_the_reference(args, changed):
    assert dry_run(*args) == {**DEFAULTS, **changed}


def test_cli_env_flags_and_missing_env_map(tmp_path):
    """--no-env clears an earlier --env; a missing env map leaves the
    built-in scene's sky with a warning (src/scene.rs:82-90)."""
    assert dry_run("--env", "a.hdr", "--no-env")["env"] == "-"
    r = subprocess.run([str(CLI), "--dry-run", "--env", str(tmp_path / "absent.hdr")], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0 and "env map load failed" in r.stderr


def test_cli_scene_file_settings_and_spp_override(tmp_path):
    """The XML's film / sampler / integrator set the config, an explicit
    --spp wins over the file's sample_count, and --env is not read when
    --scene is given (src/main.rs:110-121)."""
    p = tmp_path / "s.xml"
    p.write_text(XML)
    got = dry_run("--scene", str(p), "--env", str(tmp_path / "absent.hdr"))
    assert (got["width"], got["height"], got["spp"], got["max_bounces"]) == ("48", "27", "4", "6")
    got = dry_run("--spp", "9", "--scene", str(p))
    assert got["spp"] == "9" and got["width"] == "48"
    r = subprocess.run([str(CLI), "--dry-run", "--scene", str(tmp_path / "absent.xml")], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode != 0 and "load scene" in r.stderr
