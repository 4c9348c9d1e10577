"""Postprocessing and export (host code, sprout_b200/csrc/postprocess.cpp) on the CPU:

* every tonemapper of the reference's pipeline (Linear, ACES, Generic, Piecewise, with fixed and
  automatic exposure) against the reference's own implementation, compiled from its sources
  (oracle/_ref/ref_post), on the same HDR pixels;
* the half conversion against numpy's IEEE binary16 rounding (nearest even), every class of
  value included;
* EXR files (ZIP compressed half RGB) read back by the reference's own EXR reader, and parsed
  here by the format's definition; RGBE files decoded here.
"""

import pathlib
import shutil
import struct
import subprocess
import zlib

import numpy as np
import pytest

import oracle

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
REF_POST = oracle.HERE / "_ref" / "ref_post"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = tmp_path_factory.mktemp("post") / "postprocess_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", str(HERE / "postprocess_check.cpp"),
                    str(ROOT / "sprout_b200" / "csrc" / "postprocess.cpp"), "-I", str(ROOT / "sprout_b200" / "csrc"),
                    "-o", str(exe), "-lz"], check=True)
    return exe


def hdr_image(w=37, h=21, seed=3):
    rng = np.random.default_rng(seed)
    img = np.exp(rng.normal(-1.0, 2.0, size=(h, w, 4))).astype(np.float32)
    img[0, :4, :3] = [[0, 0, 0], [1e-6, 2e-6, 3e-6], [50, 60, 70], [0.18, 0.18, 0.18]]
    img[..., 3] = rng.uniform(0, 1, size=(h, w))
    return img


CASES = [
    ("Linear", 0, 0.0, (0, 0, 0, 0, 0)),
    ("Linear", 0, 1.5, (0, 0, 0, 0, 0)),
    ("Linear", 1, 0.0, (0, 0, 0, 0, 0)),
    ("ACES", 0, 0.0, (0, 0, 0, 0, 0)),
    ("ACES", 1, 0.0, (0, 0, 0, 0, 0)),
    ("ACES", 0, -1.0, (0, 0, 0, 0, 0)),
    ("Generic", 0, 0.0, (1.15, 0.99, 0.18, 0.18, 1.0)),
    ("Generic", 0, 0.5, (1.3, 0.95, 0.2, 0.22, 8.0)),
    ("Piecewise", 0, 0.0, (0.1, 0.5, 2.0, 0.5, 0.5)),
    ("Piecewise", 1, 0.0, (0.3, 0.4, 1.5, 0.6, 0.2)),
]


@pytest.mark.parametrize("kind,auto,exposure,params", CASES)
def test_tonemappers_match_the_reference(driver, tmp_path, kind, auto, exposure, params):
    if not REF_POST.exists():
        pytest.skip("oracle/_ref/ref_post not built")
    img = hdr_image()
    h, w = img.shape[:2]
    src = tmp_path / "in.bin"
    img.tofile(src)
    args = [kind, str(auto), repr(exposure)] + [repr(float(p)) for p in params] + [str(w), str(h), str(src)]
    subprocess.run([str(driver), "tonemap"] + args + [str(tmp_path / "mine.bin")], check=True)
    subprocess.run([str(REF_POST), "tonemap"] + args + [str(tmp_path / "ref.bin")], check=True)
    mine = np.fromfile(tmp_path / "mine.bin", np.float32).reshape(h, w, 4)
    ref = np.fromfile(tmp_path / "ref.bin", np.float32).reshape(h, w, 4)
    ok = np.isfinite(ref)
    assert np.array_equal(ok, np.isfinite(mine))
    # float rounding differs only in the order of a few operations (and the automatic exposure's
    # mean is summed in double here, in float chunks by the reference); the reference evaluates
    # the Piecewise curve's power segments with its own polynomial exp and log (math/exp.hpp),
    # this code with the C library's, whose results differ by a few 1e-5 relative in the toe
    rtol = 5e-4 if kind == "Piecewise" else 1e-4
    assert np.allclose(mine[ok], ref[ok], rtol=rtol, atol=1e-6), np.max(np.abs(mine[ok] - ref[ok]))
    assert np.array_equal(mine[..., 3], img[..., 3])  # alpha untouched


def test_half_conversion_rounds_to_nearest_even(driver, tmp_path):
    rng = np.random.default_rng(7)
    values = np.concatenate([
        rng.normal(0, 1, 20000), np.exp(rng.uniform(-25, 12, 20000)) * rng.choice([-1, 1], 20000),
        [0.0, -0.0, 65504.0, 65519.9, 65520.0, 1e6, -1e6, 2.0 ** -24, 2.0 ** -25, 1.5 * 2.0 ** -25,
         2.0 ** -14, 2.0 ** -14 * (1 - 2 ** -11), np.inf, -np.inf]]).astype(np.float32)
    values.tofile(tmp_path / "in.bin")
    subprocess.run([str(driver), "half", str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], check=True)
    mine = np.fromfile(tmp_path / "out.bin", np.uint16)
    with np.errstate(over="ignore"):
        want = values.astype(np.float16).view(np.uint16)
    assert np.array_equal(mine, want), np.nonzero(mine != want)[0][:5]
    nan = np.array([np.nan], np.float32)
    nan.tofile(tmp_path / "nan.bin")
    subprocess.run([str(driver), "half", str(tmp_path / "nan.bin"), str(tmp_path / "nan_out.bin")], check=True)
    assert np.isnan(np.fromfile(tmp_path / "nan_out.bin", np.uint16).view(np.float16)[0])


def parse_exr(data):
    """The OpenEXR single-part scanline layout, ZIP blocks of 16 lines, half channels."""
    assert struct.unpack_from("<I", data, 0)[0] == 20000630 and struct.unpack_from("<I", data, 4)[0] == 2
    pos, attrs = 8, {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\0", end + 1)
        size = struct.unpack_from("<i", data, tend + 1)[0]
        attrs[name] = data[tend + 5: tend + 5 + size]
        pos = tend + 5 + size
    pos += 1
    assert attrs["compression"] == b"\x03"
    x0, y0, x1, y1 = struct.unpack("<4i", attrs["dataWindow"])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    channels = [c.decode() for c in attrs["channels"].split(b"\0") if c and c[0:1].isalpha() and len(c) == 1]
    offsets = struct.unpack_from(f"<{(h + 15) // 16}Q", data, pos)
    img = np.zeros((h, w, len(channels)), np.float32)
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        lines = min(16, h - y)
        raw_len = lines * w * len(channels) * 2
        block = data[off + 8: off + 8 + size]
        if size < raw_len:
            t = bytearray(zlib.decompress(block))
            for i in range(1, len(t)):
                t[i] = (t[i - 1] + t[i] - 128) & 0xFF
            half = (len(t) + 1) // 2
            raw = bytearray(len(t))
            raw[0::2], raw[1::2] = t[:half], t[half:]
        else:
            raw = block
        rows = np.frombuffer(bytes(raw), np.float16).reshape(lines, len(channels), w)
        img[y: y + lines] = rows.transpose(0, 2, 1).astype(np.float32)
    return channels, img


def test_exr_is_read_back_by_the_reference_and_by_the_format(driver, tmp_path):
    img = hdr_image(w=53, h=37)  # 37 rows: two full 16-line blocks and a partial one
    img.tofile(tmp_path / "in.bin")
    exr = tmp_path / "out.exr"
    subprocess.run([str(driver), "exr", "53", "37", str(tmp_path / "in.bin"), str(exr)], check=True)
    want = img[..., :3].astype(np.float16).astype(np.float32)
    channels, parsed = parse_exr(exr.read_bytes())
    assert channels == ["B", "G", "R"]
    assert np.array_equal(parsed[..., ::-1], want)
    if not REF_POST.exists():
        pytest.skip("oracle/_ref/ref_post not built")
    res = subprocess.run([str(REF_POST), "read_exr", str(exr), str(tmp_path / "ref.bin")], check=True,
                         capture_output=True, text=True)
    assert res.stdout.split() == ["53", "37"]
    ref = np.fromfile(tmp_path / "ref.bin", np.float32).reshape(37, 53, 3)
    assert np.array_equal(ref, want)


def test_rgbe_decodes_to_the_image(driver, tmp_path):
    img = hdr_image(w=19, h=11)
    img.tofile(tmp_path / "in.bin")
    out = tmp_path / "out.hdr"
    subprocess.run([str(driver), "rgbe", "19", "11", str(tmp_path / "in.bin"), str(out)], check=True)
    data = out.read_bytes()
    header, pixels = data.split(b"\n\n", 1)
    assert header.startswith(b"#?RADIANCE") and b"FORMAT=32-bit_rle_rgbe" in header
    size_line, body = pixels.split(b"\n", 1)
    assert size_line == b"-Y 11 +X 19"
    rgbe = np.frombuffer(body, np.uint8).reshape(11, 19, 4).astype(np.float64)
    scale = np.where(rgbe[..., 3:] > 0, np.ldexp(1.0, (rgbe[..., 3:] - 136).astype(int)), 0.0)
    decoded = (rgbe[..., :3] + 0.5) * scale
    v = np.max(img[..., :3], axis=2, keepdims=True)
    # 8-bit mantissas relative to the largest channel: within 1/128 of it
    assert np.all(np.abs(decoded - img[..., :3]) <= v / 128 + 1e-30)
