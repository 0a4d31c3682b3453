"""Generates the golden fixtures under tests/golden/ from the reference tree.

Run where the reference is present (it is read, never modified):
    python tests/golden/make_golden.py /path/to/RenderingEngine
    (or with the path in $RE_REFERENCE_ROOT)

Outputs:
  * cornell_256x256_64spp_seed1.json -- the identity/count fields of the
    reference's golden CPU Cornell report
    (rt/cpu/references/wave1/cornell-256x256-64spp-seed1.json).
  * cornell_256x256_64spp_seed1.npz -- the linear RGB image of the golden EXR
    (same directory), decoded with a minimal OpenEXR scanline reader written
    here (ZIP/ZIPS compression, HALF/FLOAT channels).
"""
from __future__ import annotations

import json
import struct
import sys
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _read_header(buf: bytes):
    assert struct.unpack_from("<I", buf, 0)[0] == 20000630, "not an OpenEXR file"
    pos = 8
    attrs = {}
    while buf[pos] != 0:
        end = buf.index(b"\0", pos)
        name = buf[pos:end].decode()
        pos = end + 1
        end = buf.index(b"\0", pos)
        typ = buf[pos:end].decode()
        pos = end + 1
        size = struct.unpack_from("<i", buf, pos)[0]
        pos += 4
        attrs[name] = (typ, buf[pos:pos + size])
        pos += size
    return attrs, pos + 1


def _channels(raw: bytes):
    chans = []
    pos = 0
    while raw[pos] != 0:
        end = raw.index(b"\0", pos)
        name = raw[pos:end].decode()
        pos = end + 1
        ptype = struct.unpack_from("<i", raw, pos)[0]
        pos += 16
        chans.append((name, ptype))
    return chans


def decode_exr(path: Path) -> np.ndarray:
    buf = path.read_bytes()
    attrs, pos = _read_header(buf)
    comp = attrs["compression"][1][0]
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    chans = _channels(attrs["channels"][1])
    lines_per_block = {0: 1, 2: 1, 3: 16}[comp]
    nblocks = (h + lines_per_block - 1) // lines_per_block
    offsets = struct.unpack_from(f"<{nblocks}Q", buf, pos)
    out = {name: np.zeros((h, w), np.float32) for name, _ in chans}
    for off in offsets:
        y, size = struct.unpack_from("<ii", buf, off)
        data = buf[off + 8: off + 8 + size]
        nl = min(lines_per_block, y1 - y + 1)
        bytes_per_px = sum(2 if t == 1 else 4 for _, t in chans)
        expected = nl * w * bytes_per_px
        if comp in (2, 3) and size < expected:
            raw = np.frombuffer(zlib.decompress(data), np.uint8).astype(np.int32)
            # Undo the predictor, then the byte interleave (OpenEXR ZIP scheme).
            d = np.cumsum(raw - 128 + np.r_[128, np.zeros(len(raw) - 1, np.int32)]) & 0xFF
            d[0] = raw[0]
            d = d.astype(np.uint8)
            half = (len(d) + 1) // 2
            inter = np.empty_like(d)
            inter[0::2] = d[:half]
            inter[1::2] = d[half:]
            data = inter.tobytes()
        p = 0
        for ly in range(nl):
            for name, t in chans:
                n = w * (2 if t == 1 else 4)
                arr = np.frombuffer(data[p:p + n], np.float16 if t == 1 else np.float32)
                out[name][y - y0 + ly] = arr.astype(np.float32)
                p += n
    return np.stack([out["R"], out["G"], out["B"]], axis=-1)


def main(ref: Path) -> None:
    src = ref / "rt" / "cpu" / "references" / "wave1"
    report = json.loads((src / "cornell-256x256-64spp-seed1.json").read_text())
    keep = {k: report[k] for k in ("width", "height", "spp", "max_bounces", "seed",
                                   "ray_count", "shadow_ray_count", "non_finite_count", "elapsed_ms")}
    keep["scene_hash"] = report["scene_hash_fnv1a64"]
    keep["linear_rgb_hash"] = report["linear_rgb_hash_fnv1a64"]
    keep["source"] = "rt/cpu/references/wave1/cornell-256x256-64spp-seed1.json"
    (HERE / "cornell_256x256_64spp_seed1.json").write_text(json.dumps(keep, indent=2) + "\n")
    img = decode_exr(src / "cornell-256x256-64spp-seed1.exr")
    np.savez_compressed(HERE / "cornell_256x256_64spp_seed1.npz", rgb=img.astype(np.float32))
    print("wrote golden fixtures", img.shape, float(img.mean()))


if __name__ == "__main__":
    import os
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RE_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py /path/to/RenderingEngine (or set RE_REFERENCE_ROOT)")
    main(Path(root))
