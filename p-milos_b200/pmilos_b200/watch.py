"""Real-time directory mode on the scan server.

The reference's real-time loop (pmilos.c:2047-2440) waits for data cubes to
appear in the directory of its observed-profiles path: it lists the directory in
alphabetical order (scandir + alphasort), takes the first regular file it has not
read yet whose name contains neither "_mod_" nor "_stokes_", polls every 5 s,
and gives up after TIMEOUT_FILE = 600 s without a new cube (defines.h:303); each
cube is inverted and its models written next to it.

Here each new cube is ingested on the GPU (``ingest_fits``: raw data block to
the device, reorder kernel) and submitted to a ``Server`` as a device-resident
scan, so that cubes arriving while others are being inverted overlap on the GPU;
the models of each cube are written as ``<name>_mod_gpu.fits`` in the layout of
the reference's writeFitsImageModels (utilsFits.c:1706-1830): float32 planes
eta0, B, vlos, dopp, aa, gamma, azimuth, S0, S1, mac, alpha, iterations, chi^2,
each [columns][rows] in pixel order (NAXIS1 = rows, NAXIS2 = columns, NAXIS3 =
13).
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import Server, fits_header, ingest_fits

SKIP = ("_mod_", "_stokes_")
POLL_S = 5.0
TIMEOUT_S = 600.0


def new_cubes(directory: str, seen: set) -> list[str]:
    """Files of ``directory`` not in ``seen``, in the reference's order and
    filter; hidden names (leading '.') are skipped too, so that a writer can
    stage a cube under a hidden name and rename it into place when complete."""
    out = []
    for name in sorted(os.listdir(directory)):
        path = os.path.join(directory, name)
        if name.startswith(".") or any(s in name for s in SKIP) or os.path.isdir(path) or path in seen:
            continue
        out.append(path)
    return out


def models_fits_bytes(models: np.ndarray, iters: np.ndarray, chisq: np.ndarray, rows: int, cols: int) -> bytes:
    """The model cube of one inversion as a FITS file (see the module docstring)."""
    planes = np.empty((13, rows * cols), dtype=np.float32)
    planes[:11] = models.T
    planes[11] = iters
    planes[12] = chisq
    cards = ["SIMPLE  =                    T", "BITPIX  =                  -32", "NAXIS   =                    3",
             f"NAXIS1  = {rows:20d}", f"NAXIS2  = {cols:20d}", f"NAXIS3  = {13:20d}", "END"]
    hdr = "".join(c.ljust(80) for c in cards).encode("ascii")
    hdr += b" " * (-len(hdr) % 2880)
    body = planes.astype(">f4").tobytes()
    body += b"\0" * (-len(body) % 2880)
    return hdr + body


class DirectoryStream:
    """Serve every cube that appears in ``directory`` on ``grid`` of ``server``.

    ``run()`` returns when no new cube has appeared for ``timeout_s`` (after
    finishing the cubes in flight) and gives the output paths in arrival order."""

    def __init__(self, server: Server, grid: int, directory: str, poll_s: float = POLL_S,
                 timeout_s: float = TIMEOUT_S, on_done=None):
        self.server, self.grid, self.dir = server, grid, directory
        self.poll_s, self.timeout_s, self.on_done = poll_s, timeout_s, on_done
        self.seen: set = set()

    def run(self) -> list[str]:
        written, inflight = [], []
        last_new = time.monotonic()
        while True:
            fresh = new_cubes(self.dir, self.seen)
            for path in fresh:
                self.seen.add(path)
                with open(path, "rb") as f:
                    raw = f.read()
                hdr = fits_header(raw)
                cube = ingest_fits(raw)
                inflight.append((path, hdr, cube, self.server.submit(self.grid, cube)))
            if fresh:
                last_new = time.monotonic()
            # write what has finished, in arrival order
            while inflight:
                path, hdr, cube, sid = inflight[0]
                try:
                    r = self.server.wait(sid, timeout=0.0 if len(inflight) > 1 or fresh else self.poll_s)
                except TimeoutError:
                    break
                inflight.pop(0)
                out = os.path.splitext(path)[0] + "_mod_gpu.fits"
                with open(out, "wb") as f:
                    f.write(models_fits_bytes(r["models"], r["iters"], r["chisq"], hdr["nrows"], hdr["ncols"]))
                written.append(out)
                if self.on_done:
                    self.on_done(path, out, r)
            if not inflight and time.monotonic() - last_new >= self.timeout_s:
                return written
            if not fresh and not inflight:
                time.sleep(self.poll_s)
