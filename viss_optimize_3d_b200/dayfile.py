"""Binary day, sky and image files of the streaming day loop (bin/vissgen_stream).

They replace the reference's per-day text files (uvw/xyza/xyzb/bll
{d}day1M.txt, vissgen3d_blockage.cu:309-391) and its 6-digit text image
(C{d}day1M.txt, :542-553) with the same values as raw little-endian arrays
behind one 64-byte header (layout in host/dayfile.h):

  VISSDAY  float32 uvw[n][3], xyza[n][3], xyzb[n][3], bll[n]
  VISSSKY  float32 B[npix], theta[npix], phi[npix]
  VISSIMG  image[npix], float32 per day or float64 for a day sum

`observation_rows` builds a day's rows (unique samples, then their conjugate
mirrors) from a synthetic observation, as the reference's inputs hold them.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("elem_bytes", "<u4"), ("count", "<i8"),
                   ("day", "<i8"), ("frequency", "<f8"), ("days", "<i8"), ("reserved", "<i8", (2,))])
assert HEADER.itemsize == 64
VERSION = 1


@dataclasses.dataclass
class DayRows:
    uvw: np.ndarray    # (n, 3) float32, wavelengths
    xyza: np.ndarray   # (n, 3) float32, metres
    xyzb: np.ndarray   # (n, 3) float32, metres
    bll: np.ndarray    # (n,) float32


def _header(magic: bytes, elem: int, count: int, day: int = 1, frequency: float = 0.0,
            days: int = 1) -> np.ndarray:
    h = np.zeros((), HEADER)
    h["magic"], h["version"], h["elem_bytes"], h["count"] = magic, VERSION, elem, count
    h["day"], h["frequency"], h["days"] = day, frequency, days
    return h


def _read(path: str, magic: bytes, per_item: int):
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < HEADER.itemsize:
        raise ValueError(f"{path}: shorter than a header")
    h = raw[:HEADER.itemsize].view(HEADER)[0]
    if h["magic"] != magic or h["version"] != VERSION or h["elem_bytes"] not in (4, 8):
        raise ValueError(f"{path}: not a version-{VERSION} {magic.decode()} file")
    dt = np.float32 if h["elem_bytes"] == 4 else np.float64
    want = HEADER.itemsize + int(h["count"]) * per_item * int(h["elem_bytes"])
    if raw.size != want:
        raise ValueError(f"{path}: size {raw.size} bytes, header says {want}")
    return h, raw[HEADER.itemsize:].view(dt)


def write_day(path: str, rows: DayRows, day: int = 1, frequency: float = 0.0) -> None:
    n = rows.uvw.shape[0]
    parts = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
             for a in (rows.uvw, rows.xyza, rows.xyzb, rows.bll)]
    if [p.size for p in parts] != [3 * n, 3 * n, 3 * n, n]:
        raise ValueError("uvw, xyza, xyzb must be (n, 3) and bll (n,)")
    with open(path, "wb") as f:
        _header(b"VISSDAY", 4, n, day, frequency).tofile(f)
        for p in parts:
            p.tofile(f)


def read_day(path: str):
    h, a = _read(path, b"VISSDAY", 10)
    n = int(h["count"])
    rows = DayRows(a[:3 * n].reshape(n, 3), a[3 * n:6 * n].reshape(n, 3),
                   a[6 * n:9 * n].reshape(n, 3), a[9 * n:])
    return rows, int(h["day"]), float(h["frequency"])


def write_sky(path: str, B, theta, phi) -> None:
    B, theta, phi = (np.ascontiguousarray(x, dtype=np.float32).reshape(-1) for x in (B, theta, phi))
    if not (B.size == theta.size == phi.size):
        raise ValueError("B, theta, phi must have npix values each")
    with open(path, "wb") as f:
        _header(b"VISSSKY", 4, B.size).tofile(f)
        for x in (B, theta, phi):
            x.tofile(f)


def read_sky(path: str):
    h, a = _read(path, b"VISSSKY", 3)
    n = int(h["count"])
    return a[:n], a[n:2 * n], a[2 * n:]


def write_image(path: str, image, day: int = 1, days: int = 1, frequency: float = 0.0) -> None:
    """float32 for one day's image, float64 for a day sum (as the loop writes them)."""
    image = np.ascontiguousarray(image).reshape(-1)
    if image.dtype not in (np.float32, np.float64):
        raise ValueError("image must be float32 or float64")
    with open(path, "wb") as f:
        _header(b"VISSIMG", image.dtype.itemsize, image.size, day, frequency, days).tofile(f)
        image.astype(image.dtype.newbyteorder("<"), copy=False).tofile(f)


def read_image(path: str):
    """(image, first day, days summed)."""
    h, a = _read(path, b"VISSIMG", 1)
    return a, int(h["day"]), int(h["days"])


def observation_rows(obs, f_hz: float, lam: float | None = None) -> DayRows:
    """A synthetic observation day as the reference's files hold it: the unique
    baselines (snapshot-major) then their mirrors (u -> -u, same positions and
    bll), FP32.  lam defaults to c / f."""
    from .synth import C_LIGHT
    lam = C_LIGHT / f_hz if lam is None else lam
    P = np.asarray(obs.positions, dtype=np.float64)
    pairs = np.asarray(obs.pairs)
    Pa = P[:, pairs[:, 0], :].reshape(-1, 3)
    Pb = P[:, pairs[:, 1], :].reshape(-1, 3)
    u = ((Pa - Pb) / lam).astype(np.float32)
    bll = np.linalg.norm(u.astype(np.float64), axis=1).astype(np.float32)
    return DayRows(np.concatenate([u, -u]), np.concatenate([Pa, Pa]).astype(np.float32),
                   np.concatenate([Pb, Pb]).astype(np.float32), np.concatenate([bll, bll]))


def day_path(directory: str, day: int) -> str:
    return os.path.join(directory, f"day{day}.vday")
