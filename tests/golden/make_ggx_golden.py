"""Generates tests/golden/ggx_integral_reference.npz: the reference's generated GGX
directional-albedo table E[32][32] (source/core/scene/material/ggx/ggx_integral.inl, written by
the reference's ggx_integrate.cpp:199-230), read as text from the reference sources.

    SPROUT_REFERENCE=<reference checkout> python tests/golden/make_ggx_golden.py
"""

from __future__ import annotations

import os
import pathlib
import re

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REFERENCE = pathlib.Path(os.environ.get("SPROUT_REFERENCE", "/root/reference"))


def main():
    src = REFERENCE / "source" / "core" / "scene" / "material" / "ggx" / "ggx_integral.inl"
    text = src.read_text()
    body = text[text.index("E[32][32]"):]
    body = body[: body.index("};")]
    table = np.array([float(x) for x in re.findall(r"([0-9.]+(?:e[-+]?[0-9]+)?)f", body)][:1024], np.float32)
    assert table.size == 1024
    np.savez_compressed(HERE / "ggx_integral_reference.npz", E=table.reshape(32, 32),
                        source=np.frombuffer(b"source/core/scene/material/ggx/ggx_integral.inl E[32][32]", np.uint8))
    print("wrote", HERE / "ggx_integral_reference.npz")


if __name__ == "__main__":
    main()
