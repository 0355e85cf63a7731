"""The command-line renderer (tinypt_b200/bin/tinypt, the reference's flags):
a Mitsuba XML scene rendered on the GPU and written as PPM / HDR, identical
to the same render through the Python API."""
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
