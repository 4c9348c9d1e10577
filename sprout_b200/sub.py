"""Writes 3-D density images in the reference renderer's SUB format (the format its
Volumetric materials read through "density": {"file": ...}; image::encoding::sub::Reader,
sub_image_reader.cpp): "SUB\\0", the JSON header's length as uint64, the JSON header, then
the binary part -- all voxels, or for a sparse image a topology bitfield (32-bit words,
voxel i at bit 31 - i % 32 of word i / 32) followed by the values of the marked voxels."""

from __future__ import annotations

import json
import pathlib

import numpy as np


def write_sub(path, density, byte: bool = False, sparse: bool = False) -> None:
    """density: (nz, ny, nx) array, x fastest in memory; byte: store Byte1 (values in [0, 1]
    quantised to 1/255), else Float1; sparse: store only the nonzero voxels behind a topology."""
    d = np.ascontiguousarray(density)
    nz, ny, nx = d.shape
    flat = d.reshape(-1)
    values = np.round(np.clip(flat, 0.0, 1.0) * 255.0).astype(np.uint8) if byte else flat.astype(np.float32)
    binary = bytearray()
    image = {"description": {"dimensions": [nx, ny, nz], "type": "Byte1" if byte else "Float1"}}
    if sparse:
        mask = values != 0
        words = np.zeros((flat.size + 31) // 32, np.uint32)
        idx = np.nonzero(mask)[0]
        np.bitwise_or.at(words, idx >> 5, (np.uint32(0x80000000) >> (idx % 32).astype(np.uint32)).astype(np.uint32))
        image["topology"] = {"binary": {"offset": 0, "size": int(words.nbytes)}}
        binary += words.tobytes()
        stored = values[mask]
    else:
        stored = values
    image["pixels"] = {"binary": {"offset": len(binary), "size": int(stored.nbytes)}}
    binary += stored.tobytes()
    header = json.dumps({"image": image}).encode()
    pathlib.Path(path).write_bytes(b"SUB\0" + np.uint64(len(header)).tobytes() + header + bytes(binary))
