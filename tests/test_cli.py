"""The gr-renderer command line (crates/gr-renderer/src/main.rs) and the PNG
files it writes.

CPU: argument names and defaults equal the reference's clap fields; the
scene main.rs builds (camera, metric, disk, sky, supersampling); unknown
metric / scene / unreadable sky map end with status 1; PNG encode / decode
round trips (every filter type on the read side, CRC checked).  GPU: the
CLI's PNG holds exactly the frame of the library call, and equals the
oracle's frame.
"""
from __future__ import annotations

import math
import struct
import zlib

import numpy as np
import pytest

from gargantua_b200 import abi, cli, hdr, png, workloads
from gargantua_b200.curved import AccretionDisk, HdriSky, ProceduralSky
from gargantua_b200.gr_core import Kerr, Schwarzschild


def test_defaults_match_the_reference():  # main.rs:19-74
    a = cli.parser().parse_args([])
    assert (a.metric, a.mass, a.spin, a.width, a.height) == ("schwarzschild", 1.0, 0.9, 800, 600)
    assert (a.disk, a.scene, a.r_inner, a.r_outer, a.scale_height) == (False, "none", 6.0, 20.0,
                                                                       1.0)
    assert (a.samples, a.quiet, a.hdri, a.hdri_intensity, a.output) == (1, False, None, 1.0,
                                                                        "out.png")


def test_scene_of_arguments(tmp_path):
    s = cli.build_scene(cli.parser().parse_args([]))
    assert isinstance(s.metric, Schwarzschild) and s.disk is None
    assert s.camera.position == (0.0, 30.0, math.pi / 2.0, 0.0)
    assert s.camera.look_at == (-1.0, 0.0, 0.0) and s.camera.up == (0.0, 0.0, 1.0)
    assert s.camera.aspect == 800 / 600 and s.camera.fov_y_radians == math.radians(60.0)
    assert isinstance(s.options.sky, ProceduralSky) and s.options.samples_per_axis == 1
    ref = workloads.reference_cli(800, 600)
    assert s.camera == ref.camera
    path = tmp_path / "sky.hdr"
    hdr.write_hdr(path, np.ones((4, 8, 3), np.float32))
    s = cli.build_scene(cli.parser().parse_args(
        ["--metric", "kerr", "--spin", "0.5", "--disk", "--r-inner", "7", "--r-outer", "25",
         "--scale-height", "2", "--samples", "0", "--hdri", str(path), "--hdri-intensity",
         "3"]))
    assert isinstance(s.metric, Kerr) and s.metric.spin == 0.5
    assert isinstance(s.disk, AccretionDisk)
    assert (s.disk.r_inner, s.disk.r_outer, s.disk.scale_height) == (7.0, 25.0, 2.0)
    assert s.options.samples_per_axis == 1  # args.samples.max(1)
    assert isinstance(s.options.sky, HdriSky) and s.options.sky.intensity == 3.0
    s = cli.build_scene(cli.parser().parse_args(["--precision", "mixed"]))
    assert s.integrator_c().precision == abi.GG_PREC_MIXED
    assert s.integrator_c().stepper == abi.GG_STEPPER_DP45


@pytest.mark.parametrize("argv", [["--metric", "minkowski"], ["--scene", "teapot"],
                                  ["--hdri", "/nonexistent.hdr"]])
def test_bad_arguments_exit_1(argv, capsys, tmp_path):
    assert cli.main(argv + ["--output", str(tmp_path / "x.png")]) == 1
    assert capsys.readouterr().err
    assert not (tmp_path / "x.png").exists()


@pytest.mark.parametrize("h,w", [(1, 1), (7, 5), (64, 33)])
def test_png_round_trip(tmp_path, h, w):
    rng = np.random.default_rng(h * w)
    img = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    img[:, : w // 2] = img[:, :1]  # rows where Sub wins
    path = tmp_path / "f.png"
    png.write_png(path, img)
    assert np.array_equal(png.read_png(path), img)


def _png_with_filter(img, ft):
    """A PNG of img whose every row uses filter type ft (written here, the
    specification's filter definitions, section 9)."""
    h, w, c = img.shape
    stride = w * c
    rows = img.reshape(h, stride).astype(np.int32)
    raw = bytearray()
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        cur = rows[y]
        out = np.zeros(stride, np.int32)
        for x in range(stride):
            a = int(cur[x - c]) if x >= c else 0
            b = int(prev[x])
            cc = int(prev[x - c]) if x >= c else 0
            pred = (0, a, b, (a + b) >> 1, png._paeth(a, b, cc))[ft]
            out[x] = (int(cur[x]) - pred) & 255
        raw.append(ft)
        raw += bytes(out.astype(np.uint8))
        prev = cur
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 2 if c == 3 else 6, 0, 0, 0)
    return (png._SIG + png._chunk(b"IHDR", ihdr) + png._chunk(b"IDAT", zlib.compress(bytes(raw)))
            + png._chunk(b"IEND", b""))


@pytest.mark.parametrize("ft", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("c", [3, 4])
def test_png_decoder_filters(ft, c):
    rng = np.random.default_rng(ft * 10 + c)
    img = rng.integers(0, 256, (6, 5, c), dtype=np.uint8)
    assert np.array_equal(png.decode_png(_png_with_filter(img, ft)), img)


def test_png_rejects_corruption():
    data = bytearray(png.encode_png(np.zeros((2, 2, 3), np.uint8)))
    data[20] ^= 1  # inside IHDR
    with pytest.raises(ValueError):
        png.decode_png(bytes(data))
    with pytest.raises(ValueError):
        png.encode_png(np.zeros((2, 2), np.uint8))


@pytest.mark.gpu
@pytest.mark.parametrize("argv,metric,disk", [
    (["--width", "96", "--height", "72"], "schwarzschild", False),
    (["--width", "64", "--height", "48", "--metric", "kerr", "--disk", "--samples", "2"], "kerr",
     True),
])
def test_cli_png_equals_library_and_oracle(renderer, oracle_mod, tmp_path, capsys, argv, metric,
                                           disk):
    out = tmp_path / "out.png"
    assert cli.main(argv + ["--quiet", "--output", str(out)], renderer=renderer) == 0
    line = capsys.readouterr().out.strip()
    w, h = int(argv[1]), int(argv[3])
    assert line.startswith(f"Rendered {w}x{h} ({metric}{'+disk' if disk else ''}) in ")
    assert line.endswith(f"s → {out}")
    got = png.read_png(out)
    scene = cli.build_scene(cli.parser().parse_args(argv))
    img, _ = renderer.render(scene)
    assert np.array_equal(got, img)
    oimg, _ = oracle_mod.render(scene, rays=False)
    # the hashed starfield keys on the f64 bits of the final direction:
    # only star placement may differ (as in the procedural-sky parity test),
    # at most the ~3/512 star rate on each side
    assert (got == oimg).all(axis=2).mean() > 0.97


@pytest.mark.gpu
def test_cli_hdri_and_mixed(renderer, tmp_path):
    sky = tmp_path / "sky.hdr"
    rng = np.random.default_rng(1)
    hdr.write_hdr(sky, rng.random((16, 32, 3)).astype(np.float32))
    out = tmp_path / "m.png"
    argv = ["--width", "80", "--height", "60", "--metric", "kerr", "--hdri", str(sky),
            "--hdri-intensity", "0.5", "--precision", "mixed", "--output", str(out)]
    assert cli.main(argv, renderer=renderer) == 0
    img = png.read_png(out)
    assert img.shape == (60, 80, 3) and img.any()
    fp64 = tmp_path / "d.png"
    assert cli.main(argv[:-4] + ["--output", str(fp64)], renderer=renderer) == 0
    # the two forms trace different steppers; the sky map must agree wherever
    # both escape, so the frames are close
    d = np.abs(png.read_png(fp64).astype(int) - img.astype(int)).max(axis=2)
    assert (d <= 2).mean() > 0.98
