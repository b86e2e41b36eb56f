"""Host generators of the synthetic inputs (CPU): the rectangle list the device
generator is given reproduces the host block mask, and the struct mirror of
the device generators' descriptor matches the C header's field order."""

from __future__ import annotations

import ctypes
import re

import numpy as np

from conftest import REPO


def test_urban_rects_reproduce_the_block_mask():
    from hybrid_flood_b200.workloads import urban, urban_rects

    rows, cols = 120, 200
    w = urban(rows, cols, seed=7)
    rects = urban_rects(rows, cols, seed=7)
    blocks = np.zeros((rows, cols), bool)
    covered = 0
    for r0, c0, h, wd in rects:
        patch = blocks[r0:r0 + h, c0:c0 + wd]
        covered += int(patch.size - patch.sum())
        patch[...] = True
    assert covered >= 0.3 * rows * cols
    x = (np.arange(cols) + 0.5) * 1.0
    plane = 0.003 * (cols * 1.0 - x)[None, :] * np.ones((rows, 1))
    np.testing.assert_array_equal((plane + np.where(blocks, 10.0, -0.2)).astype(np.float32), w.bed)


def test_urban_desc_mirrors_the_header():
    from hybrid_flood_b200 import _lib

    text = (REPO / "include" / "swe_b200.h").read_text()
    body = text[text.index("typedef struct {\n    int32_t rows, cols;\n    double dx;"):]
    body = body[:body.index("} swe_urban_desc;")]
    names = []
    for line in body.splitlines()[1:]:
        m = re.match(r"\s*(?:const\s+)?[a-z0-9_]+\s+\**\s*([a-z0-9_, *]+);", line)
        if m:
            names += [n.strip(" *") for n in m.group(1).split(",")]
    assert names == [f[0] for f in _lib.UrbanDesc._fields_]
    # 2 int32 + 3 double + 2 int32 + 5 double + uint64 + int32 (+4 padding) + pointer
    assert ctypes.sizeof(_lib.UrbanDesc) == 104
