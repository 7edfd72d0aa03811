"""Copies the reference's own test inputs into tests/golden/fixtures/ and extracts the
marching-cubes case table of the reference as a golden array.

NANOSHAPER_REFERENCE names the root of a NanoShaper source checkout (read only).  Written:
  * fixtures/1crn.xyzr, fixtures/1crn_ses_conf.prm   (tests/1crn_ses of the reference)
  * fixtures/1crn_skin_conf.prm                      (tests/1crn_skin of the reference)
  * fixtures/6xm4.xyzr.gz, fixtures/6xm4_skin_conf.prm (tests/6xm4_skin of the reference)
  * fixtures/mc_tritable.npy: triTable of src/tools.h:181 as an int16 (256, 16) array, -1 padded
Run:  NANOSHAPER_REFERENCE=<checkout> python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import gzip
import os
import re
import shutil
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "fixtures"


def tri_table(tools_h: Path) -> np.ndarray:
    text = tools_h.read_text()
    start = text.index("triTable[256][16]")
    body = text[start:text.index("};", start)]
    rows = re.findall(r"\{([^{}]*)\}", body)
    tab = np.array([[int(v) for v in r.split(",") if v.strip()] for r in rows], np.int16)
    assert tab.shape == (256, 16), tab.shape
    return tab


def main() -> None:
    ref = Path(os.environ["NANOSHAPER_REFERENCE"])
    OUT.mkdir(exist_ok=True)
    t = ref / "tests"
    shutil.copyfile(t / "1crn_ses" / "1crn.xyzr", OUT / "1crn.xyzr")
    shutil.copyfile(t / "1crn_ses" / "1crn_ses_conf.prm", OUT / "1crn_ses_conf.prm")
    shutil.copyfile(t / "1crn_skin" / "1crn_skin_conf.prm", OUT / "1crn_skin_conf.prm")
    shutil.copyfile(t / "6xm4_skin" / "6xm4_skin_conf.prm", OUT / "6xm4_skin_conf.prm")
    with open(t / "6xm4_skin" / "6xm4.xyzr", "rb") as f, open(OUT / "6xm4.xyzr.gz", "wb") as raw:
        with gzip.GzipFile(fileobj=raw, mode="wb", mtime=0) as g:
            shutil.copyfileobj(f, g)
    np.save(OUT / "mc_tritable.npy", tri_table(ref / "src" / "tools.h"))
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
