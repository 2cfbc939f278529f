"""Convert the reference's compiled-in parity-check tables into `.ldpc` data files.

The reference bakes each LDPC code into C sources: the macros of
``src/matrix/<code>/constantes_gpu.h`` (``_N``, ``_K`` = number of checks,
``_M`` = number of edges, ``NB_DEGRES``, ``DEG_1``, ``DEG_2``,
``DEG_1_COMPUTATIONS``, ``DEG_2_COMPUTATIONS``) and the flattened
check-major variable-index list ``PosNoeudsVariable[_M]`` of
``src/matrix/<code>/constantes_decoder.h`` (e.g. ``4000x2000/constantes_decoder.h:3``).
Rows of degree ``DEG_1`` come first, then the ``DEG_2`` rows; the row order is
the decoder's layer order, so it is preserved exactly.

This script runs once, in a checkout that has the reference tree, and writes
the binary files that ship in this directory; nothing reads the reference at
run time.  The file format is the project's own (see ``codes.py``):

    char[8]  magic  "LDPCH001"
    u32      n_vars, n_checks, n_edges, n_groups, col_bytes, reserved
    u32[2]   (degree, count) per row group, in row order
    u16/u32  cols[n_edges]   (col_bytes = 2 when n_vars <= 65536)

Usage: python import_reference_tables.py <reference>/src/matrix
"""
import os
import re
import struct
import sys

MAGIC = b"LDPCH001"


def _macros(text):
    out = {}
    for m in re.finditer(r"^\s*#define\s+(\w+)\s+([0-9]+)\b", text, re.M):
        out[m.group(1)] = int(m.group(2))
    return out


def _table(text):
    body = text[text.index("{") + 1: text.rindex("}")]
    body = re.sub(r"/\*.*?\*/", " ", body, flags=re.S)
    return [int(x) for x in re.findall(r"[0-9]+", body)]


def convert(code_dir, out_path):
    gpu = open(os.path.join(code_dir, "constantes_gpu.h")).read()
    dec = open(os.path.join(code_dir, "constantes_decoder.h")).read()
    mac = _macros(gpu)
    n, k, m = mac["_N"], mac["_K"], mac["_M"]
    groups = [(mac["DEG_1"], mac["DEG_1_COMPUTATIONS"])]
    if mac.get("NB_DEGRES", 1) > 1:
        groups.append((mac["DEG_2"], mac["DEG_2_COMPUTATIONS"]))
    cols = _table(dec)
    assert len(cols) == m, (code_dir, len(cols), m)
    assert sum(d * c for d, c in groups) == m, (code_dir, groups, m)
    assert sum(c for _, c in groups) == k, (code_dir, groups, k)
    assert max(cols) < n
    cb = 2 if n <= 65536 else 4
    with open(out_path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<6I", n, k, m, len(groups), cb, 0))
        for d, c in groups:
            f.write(struct.pack("<2I", d, c))
        f.write(struct.pack("<%d%s" % (m, "H" if cb == 2 else "I"), *cols))
    return n, k, m, groups


def main(matrix_dir):
    here = os.path.dirname(os.path.abspath(__file__))
    for name in sorted(os.listdir(matrix_dir)):
        d = os.path.join(matrix_dir, name)
        if not (os.path.isdir(d) and os.path.exists(os.path.join(d, "constantes_decoder.h"))):
            continue
        info = convert(d, os.path.join(here, name + ".ldpc"))
        print(name, info)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python import_reference_tables.py <reference src/matrix directory>")
    main(sys.argv[1])
