"""Writes hosek_rgb.npy, the Hosek-Wilkie sky model's RGB coefficient and
radiance tables, from the text of the reference's vendored data header.

    python noor_b200/data/make_hosek_data.py <reference tree>

reads <tree>/noor/external/ArHosekSkyModelData_RGB.h (datasetRGB1..3: 1080
coefficients each, datasetRGBRad1..3: 120 radiances each) and stores them as
one float32 array of 3 x 1080 + 3 x 120 values, in that order -- the layout
noor_hosek_fit takes.  The tables are (c) 2012-2013 Lukas Hosek and
Alexander Wilkie under the 3-clause BSD license (HOSEK_WILKIE_LICENSE here).
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "hosek_rgb.npy"


def parse(text: str, name: str, count: int) -> np.ndarray:
    m = re.search(r"float\s+" + name + r"\[\]\s*=\s*\{(.*?)\};", text, re.S)
    if not m:
        raise ValueError(f"{name} not found")
    body = re.sub(r"//[^\n]*", "", m.group(1))
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    vals = [float(v) for v in body.replace("\n", " ").split(",") if v.strip()]
    if len(vals) != count:
        raise ValueError(f"{name}: {len(vals)} values, expected {count}")
    return np.array(vals, np.float32)


def main() -> None:
    tree = Path(sys.argv[1]) if len(sys.argv) > 1 else None
    if tree is None:
        raise SystemExit("usage: make_hosek_data.py <reference tree>")
    text = (tree / "noor" / "external" / "ArHosekSkyModelData_RGB.h").read_text()
    parts = [parse(text, f"datasetRGB{c}", 1080) for c in (1, 2, 3)]
    parts += [parse(text, f"datasetRGBRad{c}", 120) for c in (1, 2, 3)]
    np.save(OUT, np.concatenate(parts))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
