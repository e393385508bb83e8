"""Generates tests/golden/params_reference.json from the reference's own
.params files (data/*.params of the reference project): the raw bytes and
their fields decoded in the order of scene::loadParameters
(sources/scene/scene.cpp:1183-1250).

    python tests/golden/make_params_golden.py <reference_root>

(reference_root: the reference project's root, or $MLODS_REF_ROOT)
"""
import json
import os
import struct
import sys
from pathlib import Path

# field, struct code, count -- scene.cpp:1183-1250
LAYOUT = [("cam_quat", "f", 4), ("cam_translation", "f", 3), ("cam_dist", "f", 1), ("sigma", "f", 1),
          ("fixed_sigmas", "f", 5), ("beginning_sigma", "f", 1), ("factor", "f", 1), ("constant_shift", "f", 1),
          ("exponent", "f", 1), ("cutoff", "f", 1), ("n_computed_sigmas", "I", 1), ("max_iterations", "I", 1),
          ("max_depth", "I", 1), ("min_depth", "I", 1), ("fast_method", "I", 1), ("kernel_type", "i", 1),
          ("computed_sigma", "B", 1), ("cut", "B", 1), ("n_points", "I", 1), ("max_upsamples", "I", 1),
          ("offset", "f", 6)]


def decode(raw: bytes) -> dict:
    out, off = {}, 0
    for name, code, n in LAYOUT:
        vals = struct.unpack_from("<" + code * n, raw, off)
        off += struct.calcsize("<" + code * n)
        out[name] = list(vals) if n > 1 else vals[0]
    assert off == len(raw) == 134, (off, len(raw))
    return out


def main():
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MLODS_REF_ROOT")
    if not arg:
        sys.exit("usage: make_params_golden.py <reference_root> (or set MLODS_REF_ROOT)")
    root = Path(arg)
    files = sorted((root / "data").glob("*.params"))
    data = {f.stem: {"hex": f.read_bytes().hex(), "fields": decode(f.read_bytes())} for f in files}
    out = Path(__file__).with_name("params_reference.json")
    out.write_text(json.dumps(data, indent=1, sort_keys=True))
    print(f"wrote {out} ({len(data)} files)")


if __name__ == "__main__":
    main()
