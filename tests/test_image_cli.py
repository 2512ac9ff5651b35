"""Image output (pbrt_write_png: the reference's image_write, src/renderers/mt.rs:152-167) and
the command-line renderer's argument handling (src/main.rs, src/config.rs:131-170). No GPU."""
from __future__ import annotations

import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

import pbrt_b200 as pb
from conftest import ROOT

CLI = os.path.join(ROOT, "pbrt_b200", "pbrt")


def read_png(path):
    """A minimal PNG reader: RGBA8, filter 0 (what the writer produces), checking every CRC."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, ihdr = 8, b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(typ + body) == crc
        if typ == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype, _, _, interlace = ihdr
    assert (depth, ctype, interlace) == (8, 6, 0)
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    assert np.all(rows[:, 0] == 0)
    return rows[:, 1:].reshape(h, w, 4)


@pytest.mark.parametrize("w,h", [(1, 1), (7, 3), (300, 200)])
def test_png_round_trip(tmp_path, w, h):
    rgba = np.random.default_rng(w * h).integers(0, 256, (h, w, 4), dtype=np.uint8)
    p = str(tmp_path / "x.png")
    pb.write_png(p, rgba)
    np.testing.assert_array_equal(read_png(p), rgba)


def test_film_to_png(tmp_path):
    film = np.random.default_rng(1).random((20, 30, 3)) * 1.5
    p = str(tmp_path / "f.png")
    pb.film_to_png(film, p)
    got = read_png(p)
    np.testing.assert_array_equal(got, pb.film_to_rgba8(film))
    assert np.all(got[..., 3] == 255)


def test_png_rejects_bad_arguments(tmp_path):
    with pytest.raises(pb.PbrtError):
        pb.write_png(str(tmp_path / "no_such_dir" / "x.png"), np.zeros((2, 2, 4), np.uint8))


@pytest.mark.parametrize("args,msg", [
    (["--input"], "trailing parameter"),
    (["--bogus", "1"], "Unknown option"),
    (["--output", "x.png"], "--input is required"),
    (["--input", "/nonexistent.stage"], "cannot read"),
    (["--input", "x", "--samples_ppx", "-3"], "bad value"),
])
def test_cli_argument_errors(args, msg):
    r = subprocess.run([CLI] + args, capture_output=True, text=True)
    assert r.returncode == 1 and msg in r.stderr
