"""Minimal reader of single-HDU FITS float32 images (test helper; no CFITSIO here)."""
from __future__ import annotations

import numpy as np


def read_fits_f32(path: str):
    """Returns (header dict, [NAXIS1, NAXIS2, ...], flat float32 data in file order)."""
    raw = open(path, "rb").read()
    hdr, off = {}, 0
    while True:
        block = raw[off:off + 2880]
        off += 2880
        end = False
        for i in range(36):
            card = block[i * 80:(i + 1) * 80].decode("ascii")
            key = card[:8].strip()
            if key == "END":
                end = True
                break
            if card[8:10] == "= ":
                hdr[key] = card[10:].split("/")[0].strip().strip("'").strip()
        if end:
            break
    if int(hdr["BITPIX"]) != -32:
        raise ValueError("only BITPIX = -32 images are supported")
    dims = [int(hdr[f"NAXIS{i + 1}"]) for i in range(int(hdr["NAXIS"]))]
    n = int(np.prod(dims))
    return hdr, dims, np.frombuffer(raw[off:off + 4 * n], dtype=">f4").astype(np.float32)
