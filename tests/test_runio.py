"""Run and bed files in the reference's formats (docs/data-format.md), CPU only."""
import json
import os

import numpy as np
import pytest

from wavesim_b200.runio import FormatError, Run, RunWriter, read_bed, remove_run, write_bed


def test_bed_round_trip_and_rejections(tmp_path):
    elev = np.linspace(-20, 5, 12, dtype=np.float32).reshape(3, 4)
    p = str(tmp_path / "spot.json")
    write_bed(p, "spot", elev, 3.0, 3.0)
    h, e = read_bed(p)
    assert h["format"] == "wavesim-bed" and h["version"] == 1 and (h["nx"], h["ny"]) == (4, 3)
    assert np.array_equal(e, elev)
    raw = np.fromfile(tmp_path / "spot.f32", dtype="<f4")
    raw[5] = np.nan
    raw.tofile(tmp_path / "spot.f32")
    with pytest.raises(FormatError):
        read_bed(p)
    raw[:11].tofile(tmp_path / "spot.f32")
    with pytest.raises(FormatError):
        read_bed(p)
    h["version"] = 2
    (tmp_path / "spot.json").write_text(json.dumps(h))
    with pytest.raises(FormatError):
        read_bed(p)


def test_run_round_trip_reads_like_the_documented_reader(tmp_path):
    d = str(tmp_path / "run")
    ny, nx = 5, 7
    bed = np.arange(nx * ny, dtype=np.float32).reshape(ny, nx) - 20
    w = RunWriter(d, "test", bed, 2.0, 2.0, fields=("breaking", "eta"), waves={"height_m": 2.0})
    frames = []
    for k in range(3):
        eta = np.full((ny, nx), k + 0.5, dtype=np.float32)
        brk = np.full((ny, nx), 0.1 * k, dtype=np.float32)
        w.write_frame(10.0 + k, [brk, eta])
        frames.append((eta, brk))
    assert not os.path.exists(os.path.join(d, "run.json"))  # the header comes last
    w.write_stats(["eta_max"], [frames[-1][0]], 10.0, 12.0)
    w.finish()
    # docs/data-format.md "Reading a run", as a viewer does it
    h = json.load(open(os.path.join(d, "run.json")))
    mm = np.memmap(os.path.join(d, "frames.f32"), dtype="<f4", mode="r",
                   shape=(h["frame_count"], len(h["fields"]), h["ny"], h["nx"]))
    assert np.array_equal(mm[1, h["fields"].index("eta")], frames[1][0])
    r = Run(d)
    assert r.header["times"] == [10.0, 11.0, 12.0] and r.header["waves"]["height_m"] == 2.0
    assert np.array_equal(r.field("eta", 2), frames[2][0]) and np.array_equal(r.field("breaking", 1), frames[1][1])
    assert np.array_equal(r.bed, bed) and np.array_equal(r.stat("eta_max"), frames[2][0])
    assert r.field("depth", 0) is None


def test_run_writer_checks_and_replaces_an_old_run(tmp_path):
    d = str(tmp_path / "run")
    bed = np.zeros((2, 3), dtype=np.float32)
    with pytest.raises(FormatError):
        RunWriter(d, "x", bed, 1.0, 1.0, fields=("breaking",))
    w = RunWriter(d, "x", bed, 1.0, 1.0)
    with pytest.raises(FormatError):
        w.write_frame(0.0, [bed])
    with pytest.raises(FormatError):
        w.write_frame(0.0, [bed, np.zeros(5, dtype=np.float32)])
    w.write_frame(0.0, [bed, bed])
    w.finish()
    (tmp_path / "run" / "keep.txt").write_text("other files stay")
    RunWriter(d, "y", bed, 1.0, 1.0)  # a new run removes the old one's files first
    assert not os.path.exists(os.path.join(d, "run.json")) and os.path.exists(os.path.join(d, "keep.txt"))
    remove_run(d)
    assert sorted(os.listdir(d)) == ["keep.txt"]


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run_tiny")


def test_writer_reproduces_the_reference_golden_run_byte_for_byte(tmp_path):
    """The run the reference's `write_tiny` writes (crates/waveio/tests/golden.rs:18-78), built
    the same way here: a 6 x 4 bed rising 0.75 m per cell from -2 m and four frames of eta and
    breaking, every value a multiple of 1/16 (exact in FP32). The reference compares its writer's
    output with the committed fixture byte for byte (golden.rs:80-104); so does this test."""
    nx, ny = 6, 4
    n = np.arange(nx * ny)
    elev = (np.float32(-2.0) + np.float32(0.75) * (n % nx).astype(np.float32)).astype(np.float32)
    w = RunWriter(str(tmp_path), "tiny", elev.reshape(ny, nx), 3.0, 2.0, fields=("eta", "breaking"),
                  frame={"crs": "EPSG:32604", "origin_easting": 1000.0, "origin_northing": 2000.0,
                         "x_bearing_deg": 130.0, "note": "fixture"},
                  waves={"wave_height_m": 1.0, "wave_period_s": 14.0, "tide_m": 0.0, "maker_x_m": 6.0,
                         "sponge_offshore_cells": 2, "sponge_side_cells": 1},
                  source={"name": "Synthetic fixture", "attribution": "none"})
    for k in range(4):
        wave = (np.float32(0.125) * np.float32(k) + np.float32(0.0625) * (n % nx).astype(np.float32)
                - np.float32(0.25)).astype(np.float32)
        eta = np.where(elev < 0, np.maximum(wave, elev), elev).astype(np.float32)
        breaking = np.where(elev < 0, np.float32(0.25) * ((n + k) % 4).astype(np.float32), 0.0).astype(np.float32)
        w.write_frame(2.0 * k, [eta, breaking])
    w.finish()
    for name in ("run.json", "bed.f32", "frames.f32"):
        with open(os.path.join(GOLDEN, name), "rb") as f:
            want = f.read()
        with open(tmp_path / name, "rb") as f:
            got = f.read()
        assert got == want, name
    r = Run(GOLDEN)
    assert r.header["frame_count"] == 4 and np.array_equal(r.field("breaking", 3).ravel()[:3], [0.75, 0.0, 0.25])
