"""Run and bed files: the formats the reference's tools and viewer read (docs/data-format.md).

A **bed** (`wavesim-bed`, version 1) is a JSON header beside `nx * ny` little-endian FP32
elevations, row-major with y outer (crates/waveio/src/bed.rs:10-80). A **run** (`wavesim-run`,
version 1) is a directory: `bed.f32`, `frames.f32` (every frame's fields back to back, each a
block of `nx * ny` values laid out like the bed), optionally `stats.f32`, and `run.json`, written
last so that a run that stopped part-way has no header (crates/waveio/src/run.rs:10-300). This
module writes and reads both, so runs of this build feed the reference's viewer and tools
unchanged; `record_frame` and `record_stats` take the frame and the statistics from the device
(`Solver.frame`, `Recorder.read`).
"""
from __future__ import annotations

import json
import os

import numpy as np

RUN_FORMAT, RUN_VERSION = "wavesim-run", 1
BED_FORMAT, BED_VERSION = "wavesim-bed", 1
RUN_FILES = ("run.json", "bed.f32", "frames.f32", "stats.f32")  # run.rs:56
LAYOUT_BED = "row-major, y outer (increasing), x inner (increasing)"
LAYOUT_RUN = ("per frame: one block per field, in `fields` order; each block row-major, y outer "
              "(increasing), x inner (increasing)")


FRAME_KEYS = ("crs", "origin_easting", "origin_northing", "x_bearing_deg", "note")  # bed.rs:16-24


class FormatError(ValueError):
    pass


def _sorted_json(v):
    """A JSON value with every object's keys sorted, recursively."""
    if isinstance(v, dict):
        return {k: _sorted_json(v[k]) for k in sorted(v)}
    if isinstance(v, list):
        return [_sorted_json(x) for x in v]
    return v


def default_frame() -> dict:
    """A frame with no map placement (bed.rs:16-24)."""
    return {"crs": "", "origin_easting": 0.0, "origin_northing": 0.0, "x_bearing_deg": 0.0, "note": ""}


# ---- bed files ---------------------------------------------------------------------------------

def write_bed(header_path: str, name: str, elevation: np.ndarray, dx: float, dy: float, frame: dict | None = None,
              description: str = "", source=None) -> None:
    """A bed file: `<name>.json` at header_path and its `.f32` data beside it."""
    elevation = np.asarray(elevation)
    ny, nx = elevation.shape
    data = os.path.splitext(os.path.basename(header_path))[0] + ".f32"
    e32 = np.ascontiguousarray(elevation, dtype="<f4")
    if not np.all(np.isfinite(e32)):
        raise FormatError("bed elevations must be finite")
    e32.tofile(os.path.join(os.path.dirname(os.path.abspath(header_path)), data))
    header = {"format": BED_FORMAT, "version": BED_VERSION, "name": name, "description": description,
              "nx": nx, "ny": ny, "dx": float(dx), "dy": float(dy), "data": data, "dtype": "f32-le",
              "layout": LAYOUT_BED, "units": "metres above mean sea level; negative is underwater",
              "frame": frame or default_frame(),
              "stats": {"min": float(e32.min()), "max": float(e32.max())}, "source": source or {}}
    with open(header_path, "w") as f:
        f.write(json.dumps(header, indent=2) + "\n")


def read_bed(header_path: str):
    """(header, elevation (ny, nx) float32); rejects another format or version, a data file of
    the wrong length and NaN or infinite values (bed.rs:57-80)."""
    with open(header_path) as f:
        header = json.load(f)
    if header.get("format") != BED_FORMAT or header.get("version") != BED_VERSION:
        raise FormatError(f"{header_path}: not a {BED_FORMAT} version {BED_VERSION}")
    path = os.path.join(os.path.dirname(os.path.abspath(header_path)), header["data"])
    raw = np.fromfile(path, dtype="<f4")
    nx, ny = int(header["nx"]), int(header["ny"])
    if raw.size != nx * ny:
        raise FormatError(f"{path}: {raw.size} values, expected {nx * ny}")
    if not np.all(np.isfinite(raw)):
        raise FormatError(f"{path}: NaN or infinite elevation")
    return header, raw.reshape(ny, nx)


# ---- runs ---------------------------------------------------------------------------------------

def remove_run(directory: str) -> None:
    """A run's own files in `directory`, and nothing else (run.rs:58-76)."""
    for name in RUN_FILES:
        p = os.path.join(directory, name)
        if os.path.exists(p):
            os.remove(p)


class RunWriter:
    """run.rs:78-215: create the directory (removing an old run's files first), copy the bed,
    append frames, optionally write statistics, and write the header last."""

    def __init__(self, directory: str, name: str, bed: np.ndarray, dx: float, dy: float,
                 fields=("eta", "breaking"), frame: dict | None = None, waves: dict | None = None, source=None):
        if "eta" not in fields:
            raise FormatError("a run's fields must include eta")
        os.makedirs(directory, exist_ok=True)
        remove_run(directory)
        bed = np.asarray(bed)
        ny, nx = bed.shape
        np.ascontiguousarray(bed, dtype="<f4").tofile(os.path.join(directory, "bed.f32"))
        self.dir = directory
        self._frames = open(os.path.join(directory, "frames.f32"), "wb")
        self.header = {"format": RUN_FORMAT, "version": RUN_VERSION, "name": name, "nx": nx, "ny": ny,
                       "dx": float(dx), "dy": float(dy), "bed": "bed.f32", "frames": "frames.f32",
                       "fields": list(fields), "dtype": "f32-le", "layout": LAYOUT_RUN, "frame_count": 0,
                       "times": [], "frame": frame or default_frame(), "waves": dict(waves or {}),
                       "source": source or {}}

    def note(self, key: str, value) -> None:
        self.header["waves"][key] = value

    def write_frame(self, time: float, fields) -> None:
        if len(fields) != len(self.header["fields"]):
            raise FormatError(f"frame has {len(fields)} fields, expected {len(self.header['fields'])}")
        want = self.header["nx"] * self.header["ny"]
        for f in fields:
            if np.asarray(f).size != want:
                raise FormatError(f"a field has {np.asarray(f).size} values, expected {want}")
        for f in fields:
            np.ascontiguousarray(f, dtype="<f4").ravel().tofile(self._frames)
        self.header["times"].append(float(time))
        self.header["frame_count"] += 1

    def write_stats(self, fields, blocks, start: float, end: float) -> None:
        want = self.header["nx"] * self.header["ny"]
        if len(fields) != len(blocks) or any(np.asarray(b).size != want for b in blocks):
            raise FormatError(f"stats must be {len(fields)} blocks of {want} values")
        with open(os.path.join(self.dir, "stats.f32"), "wb") as f:
            for b in blocks:
                np.ascontiguousarray(b, dtype="<f4").ravel().tofile(f)
        self.header["stats"] = {"file": "stats.f32", "fields": list(fields), "from_s": float(start), "to_s": float(end)}

    def finish(self) -> str:
        """Close the frames and write run.json (run.rs:200-212) as the reference's serializer
        does: two-space pretty JSON and a newline, the header's and the frame's keys in their
        declaration order (run.rs:14-43, bed.rs:16-24), the free-form `waves` and `source`
        objects with their keys sorted at every depth, as serde_json's maps keep them."""
        self._frames.close()
        path = os.path.join(self.dir, "run.json")
        h = dict(self.header)
        h["frame"] = {k: h["frame"][k] for k in FRAME_KEYS if k in h["frame"]}
        h["waves"] = _sorted_json(h["waves"])
        h["source"] = _sorted_json(h["source"])
        with open(path, "w") as f:
            f.write(json.dumps(h, indent=2) + "\n")
        return path


class Run:
    """A finished run read back (run.rs:217-300): checks the format, version and file lengths."""

    def __init__(self, directory: str):
        path = os.path.join(directory, "run.json")
        with open(path) as f:
            h = json.load(f)
        if h.get("format") != RUN_FORMAT or h.get("version") != RUN_VERSION:
            raise FormatError(f"{path}: not a {RUN_FORMAT} version {RUN_VERSION}")
        self.header = h
        nx, ny = int(h["nx"]), int(h["ny"])
        self.bed = self._read(os.path.join(directory, h["bed"]), nx * ny).reshape(ny, nx)
        n = int(h["frame_count"]) * len(h["fields"]) * nx * ny
        self.frames = self._read(os.path.join(directory, h["frames"]), n)
        self.stats = None
        if h.get("stats"):
            st = h["stats"]
            self.stats = self._read(os.path.join(directory, st["file"]), len(st["fields"]) * nx * ny)

    @staticmethod
    def _read(path: str, count: int) -> np.ndarray:
        raw = np.fromfile(path, dtype="<f4")
        if raw.size != count:
            raise FormatError(f"{path}: {raw.size} values, expected {count}")
        return raw

    def field(self, name: str, k: int):
        """Field `name` of frame k as (ny, nx), looked up by name (never by position)."""
        h = self.header
        if name not in h["fields"]:
            return None
        f, n = h["fields"].index(name), h["nx"] * h["ny"]
        start = (k * len(h["fields"]) + f) * n
        return self.frames[start:start + n].reshape(h["ny"], h["nx"])

    def stat(self, name: str):
        st = self.header.get("stats")
        if not st or name not in st["fields"]:
            return None
        n = self.header["nx"] * self.header["ny"]
        f = st["fields"].index(name)
        return self.stats[f * n:(f + 1) * n].reshape(self.header["ny"], self.header["nx"])


# ---- from the device ----------------------------------------------------------------------------

def record_frame(writer: RunWriter, solver, time: float, tide: float = 0.0) -> float:
    """Append the solver's resident state as a frame (eta, breaking; lib.rs:1348-1380); returns
    the highest surface above `tide` over wet cells."""
    eta, breaking, rise = solver.frame(tide)
    fields = {"eta": eta, "breaking": breaking}
    writer.write_frame(time, [fields[f] for f in writer.header["fields"]])
    return rise


def record_stats(writer: RunWriter, recorder, start: float, end: float) -> None:
    """stats.f32 from a device recorder, in the reference's field order (lib.rs:1489-1505)."""
    out = recorder.read()
    names = ["break_fraction", "eta_max", "eta_min"]
    blocks = [out["breaking_fraction"], out["eta_max"], out["eta_min"]]
    if out["wave_height"] is not None:
        names.append("wave_height")
        blocks.append(out["wave_height"])
        writer.note("waves_recorded", out["waves"])
        if out["unsettled"] is not None:
            writer.note("unsettled_per_period", out["unsettled"])
        if out["harmonic"] is not None:
            names += ["harmonic_re", "harmonic_im"]
            blocks += [out["harmonic"].real, out["harmonic"].imag]
    writer.write_stats(names, blocks, start, end)
