"""Build-time extraction of the Vioreanu-Rokhlin simplex nodes and weights.

The discretisation nodes for triangular patches (iptype = 1) are the
Vioreanu-Rokhlin nodes of orders 0..20, which fmm3dbie compiles in from two
data files (``src/tria_routs/koorn-uvs-dat.txt`` and ``koorn-wts-dat.txt``,
``INCLUDE``d by ``get_vioreanu_nodes`` / ``get_vioreanu_wts`` at
``src/tria_routs/koornexps.f90:57,90``).  Those files carry their own licence
notice, so they are not copied into this repository: this script parses them
from a reference checkout at build time and writes a binary cache
``_data/vioreanu_rokhlin.bin`` next to the package (git-ignored, shipped with
the built shared library).

Binary layout (little endian):
    magic   : 8 bytes  b"BIEVR001"
    nmax    : int32    (= 20)
    for norder in 0..nmax:
        npols : int32  (= (norder+1)(norder+2)/2)
        uvs   : float64[2*npols]   (u0, v0, u1, v1, ...)
        wts   : float64[npols]
"""
from __future__ import annotations

import os
import re
import struct
import sys

MAGIC = b"BIEVR001"
NMAX = 20
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_data")
TABLE_PATH = os.path.join(DATA_DIR, "vioreanu_rokhlin.bin")

_BLOCK = re.compile(r"if\s*\(\s*norder\s*\.eq\.\s*(\d+)\s*\)\s*then(.*?)endif",
                    re.S | re.I)
_UV = re.compile(r"uvs\(\s*(\d+)\s*,\s*(\d+)\s*\)\s*=\s*([-+0-9.DdEe]+)")
_W = re.compile(r"wts\(\s*(\d+)\s*\)\s*=\s*([-+0-9.DdEe]+)")


def _fnum(s: str) -> float:
    return float(s.replace("D", "E").replace("d", "e"))


def parse(uvs_text: str, wts_text: str):
    """Return {norder: (uvs list[2*npols], wts list[npols])}."""
    out = {}
    uv_blocks = {int(m.group(1)): m.group(2) for m in _BLOCK.finditer(uvs_text)}
    w_blocks = {int(m.group(1)): m.group(2) for m in _BLOCK.finditer(wts_text)}
    for n in range(NMAX + 1):
        npols = (n + 1) * (n + 2) // 2
        uvs = [0.0] * (2 * npols)
        wts = [0.0] * npols
        seen_uv = 0
        for m in _UV.finditer(uv_blocks[n]):
            c, i, val = int(m.group(1)), int(m.group(2)), _fnum(m.group(3))
            uvs[2 * (i - 1) + (c - 1)] = val
            seen_uv += 1
        seen_w = 0
        for m in _W.finditer(w_blocks[n]):
            i, val = int(m.group(1)), _fnum(m.group(2))
            wts[i - 1] = val
            seen_w += 1
        if seen_uv != 2 * npols or seen_w != npols:
            raise ValueError(f"order {n}: parsed {seen_uv} node coords, {seen_w} weights")
        out[n] = (uvs, wts)
    return out


def write_table(table, path: str = TABLE_PATH) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path + ".tmp", "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<i", NMAX))
        for n in range(NMAX + 1):
            uvs, wts = table[n]
            f.write(struct.pack("<i", len(wts)))
            f.write(struct.pack(f"<{len(uvs)}d", *uvs))
            f.write(struct.pack(f"<{len(wts)}d", *wts))
    os.replace(path + ".tmp", path)


def read_table(path: str = TABLE_PATH):
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError("bad Vioreanu-Rokhlin table file")
    (nmax,) = struct.unpack_from("<i", data, 8)
    off = 12
    out = {}
    for n in range(nmax + 1):
        (npols,) = struct.unpack_from("<i", data, off)
        off += 4
        uvs = list(struct.unpack_from(f"<{2 * npols}d", data, off))
        off += 16 * npols
        wts = list(struct.unpack_from(f"<{npols}d", data, off))
        off += 8 * npols
        out[n] = (uvs, wts)
    return out


def generate(reference_root: str, path: str = TABLE_PATH) -> str:
    """Parse the node/weight tables from a reference checkout into ``path``."""
    d = os.path.join(reference_root, "src", "tria_routs")
    with open(os.path.join(d, "koorn-uvs-dat.txt")) as f:
        uvs_text = f.read()
    with open(os.path.join(d, "koorn-wts-dat.txt")) as f:
        wts_text = f.read()
    write_table(parse(uvs_text, wts_text), path)
    return path


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FMM3DBIE_REFERENCE")
    if not root:
        sys.exit("usage: python -m fmm3dbie_b200.tables REFERENCE_DIR "
                 "(or set FMM3DBIE_REFERENCE to a reference checkout)")
    print(generate(root))
