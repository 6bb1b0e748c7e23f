"""Extract the BC1 cluster-fit ordering tables into ``bc1_order_tables.bin``.

The ordering tables are trained data inherited by the reference from rgbcx
(public domain): they cannot be derived, and the encoder is bit-exact only
with the very same tables. This script reads them from the reference sources

  quicktex/s3tc/bc1/OrderTable.cpp   OrderTable<3>::Orders      (:47-60,  153 x 3)
                                     OrderTable<4>::Orders      (:64-162, 969 x 4)
                                     OrderTable<3>::BestOrders  (:165-320, 153 x 32)
  quicktex/s3tc/bc1/OrderTable4.cpp  OrderTable<4>::BestOrders  (:996-1965, 969 x 128,
                                     the default, non-RGBCX_USE_SMALLER_TABLES, branch)

and writes them in this package's own layout (little endian):

  offset  size            content
  0       4               magic b"QTOT"
  4       4               u32 version (1)
  8       969*4           u8  orders4[969][4]   selector histogram of each 4-colour ordering
  3884    153*3           u8  orders3[153][3]   selector histogram of each 3-colour ordering
  4343    1 (pad to 4352) zero
  4352    969*128*2       u16 best4[969][128]   ranked candidate orderings per start ordering
  252416  153*32*2        u16 best3[153][32]

Usage:  python oracle/gen_order_tables.py REFERENCE_ROOT

(REFERENCE_ROOT is the root of the reference source tree; QT_REFERENCE_ROOT
in the environment is used when the argument is omitted.)
"""

from __future__ import annotations

import os
import re
import struct
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "quicktex_b200", "data",
                   "bc1_order_tables.bin")

N4, N3, B4, B3 = 969, 153, 128, 32
OFF_ORDERS4 = 8
OFF_ORDERS3 = OFF_ORDERS4 + N4 * 4
OFF_BEST4 = 4352
OFF_BEST3 = OFF_BEST4 + N4 * B4 * 2
TOTAL = OFF_BEST3 + N3 * B3 * 2


def _ints(text: str) -> list[int]:
    return [int(x) for x in re.findall(r"\d+", text)]


def _region(text: str, start_pat: str, end_pat: str = r"\}\};") -> str:
    m = re.search(start_pat, text)
    if not m:
        raise ValueError(f"pattern not found: {start_pat}")
    body = text[m.end():]
    e = re.search(end_pat, body)
    return body[: e.start()]


def extract(ref_root: str) -> dict[str, np.ndarray]:
    bc1 = os.path.join(ref_root, "quicktex", "s3tc", "bc1")
    ot = open(os.path.join(bc1, "OrderTable.cpp")).read()
    ot4 = open(os.path.join(bc1, "OrderTable4.cpp")).read()

    orders3 = _ints(_region(ot, r"OrderTable<3>::OrderArray OrderTable<3>::Orders\s*=\s*\{"))
    orders4 = _ints(_region(ot, r"OrderTable<4>::OrderArray OrderTable<4>::Orders\s*=\s*\{"))
    best3 = _ints(_region(ot, r"OrderTable<3>::BestOrderArray OrderTable<3>::BestOrders\s*=\s*\{"))
    # the full-size table is the #else branch of RGBCX_USE_SMALLER_TABLES
    best4_all = _region(ot4, r"OrderTable<4>::BestOrderArray OrderTable<4>::BestOrders\s*=\s*\{\{")
    best4 = _ints(best4_all.split("#else", 1)[1].split("#endif", 1)[0])

    tabs = {
        "orders4": np.array(orders4, np.uint8).reshape(N4, 4),
        "orders3": np.array(orders3, np.uint8).reshape(N3, 3),
        "best4": np.array(best4, np.uint16).reshape(N4, B4),
        "best3": np.array(best3, np.uint16).reshape(N3, B3),
    }
    # structural checks: every histogram sums to 16 and each table is a permutation of all compositions
    assert (tabs["orders4"].sum(1) == 16).all() and len({tuple(r) for r in tabs["orders4"]}) == N4
    assert (tabs["orders3"].sum(1) == 16).all() and len({tuple(r) for r in tabs["orders3"]}) == N3
    assert tabs["best4"].max() < N4 and tabs["best3"].max() < N3
    return tabs


def pack(tabs: dict[str, np.ndarray]) -> bytes:
    buf = bytearray(TOTAL)
    buf[0:8] = b"QTOT" + struct.pack("<I", 1)
    buf[OFF_ORDERS4:OFF_ORDERS4 + N4 * 4] = tabs["orders4"].tobytes()
    buf[OFF_ORDERS3:OFF_ORDERS3 + N3 * 3] = tabs["orders3"].tobytes()
    buf[OFF_BEST4:OFF_BEST4 + N4 * B4 * 2] = tabs["best4"].astype("<u2").tobytes()
    buf[OFF_BEST3:OFF_BEST3 + N3 * B3 * 2] = tabs["best3"].astype("<u2").tobytes()
    return bytes(buf)


def load(path: str = OUT) -> dict[str, np.ndarray]:
    raw = open(path, "rb").read()
    assert raw[:4] == b"QTOT" and len(raw) == TOTAL
    return {
        "orders4": np.frombuffer(raw, np.uint8, N4 * 4, OFF_ORDERS4).reshape(N4, 4),
        "orders3": np.frombuffer(raw, np.uint8, N3 * 3, OFF_ORDERS3).reshape(N3, 3),
        "best4": np.frombuffer(raw, "<u2", N4 * B4, OFF_BEST4).reshape(N4, B4),
        "best3": np.frombuffer(raw, "<u2", N3 * B3, OFF_BEST3).reshape(N3, B3),
    }


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QT_REFERENCE_ROOT")
    if not root:
        raise SystemExit("usage: python oracle/gen_order_tables.py REFERENCE_ROOT (or set QT_REFERENCE_ROOT)")
    data = pack(extract(root))
    with open(OUT, "wb") as f:
        f.write(data)
    print(f"wrote {OUT} ({len(data)} bytes)")
