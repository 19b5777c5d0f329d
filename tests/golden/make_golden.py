"""Regenerate the golden fixtures in this directory from the reference tree.

Run where the reference source is available:
    python tests/golden/make_golden.py /path/to/oxideav-render-vulkan

It reads the reference's own known-answer tests as text (nothing is
compiled or executed) and writes:
  * f16_kat.json      — f32_to_f16 vectors of `f16_conversion_known_values`
                         (src/scene.rs:496-510), expected bits per input;
  * furnace.json      — the `white_furnace` test's setup and expected value
                         (tests/pathtrace.rs:169-180, 295-317);
  * pt_constants.json — path-tracer constants the reference fixes in code:
                         PATHS_PER_DISPATCH etc. (src/pathtrace.rs:83-98),
                         the per-slot colour spaces and material word layout
                         (src/pathtrace.rs:1042-1096, 1338-1423), PSNR floors
                         of the parity tests (tests/pathtrace.rs:319-418).
"""
from __future__ import annotations

import json
import re
import struct
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent


def f16_vectors(scene_rs: str):
    body = scene_rs[scene_rs.index("fn f16_conversion_known_values"):]
    body = body[: body.index("\n    }\n")]
    exact, masked = [], []
    for m in re.finditer(r"assert_eq!\(f32_to_f16\(([^)]*?)\)\s*(&\s*0x[0-9a-f]+)?\s*,\s*(0x[0-9a-f]+)\)", body):
        arg, mask, want = m.group(1).strip(), m.group(2), int(m.group(3), 16)
        if arg == "f32::INFINITY":
            bits = 0x7F800000
        elif arg == "f32::NAN":
            bits = 0x7FC00000
        else:
            expr = arg.replace("_", "")
            val = eval(expr, {"__builtins__": {}})  # numeric literal or a/b only
            bits = struct.unpack("<I", struct.pack("<f", float(val)))[0]
        entry = {"source": arg, "f32_bits": bits, "f16": want}
        if mask:
            entry["mask"] = int(mask.replace("&", "").strip(), 16)
            masked.append(entry)
        else:
            exact.append(entry)
    return {"from": "src/scene.rs:496-510", "exact": exact, "masked": masked}


def furnace(tests_rs: str):
    m = re.search(r"furnace_scene\(([\d.]+),\s*([\d.]+)\)", tests_rs)
    o = re.search(r"let mut o = opts\((\d+),\s*(\d+),\s*(\d+),\s*(\d+)\);\s*o\.ambient = ([\d.]+);", tests_rs)
    tol = re.search(r"\(c - ([\d.]+)\)\.abs\(\) < ([\d.]+)", tests_rs)
    cam = re.search(r"add_camera\(&mut scene, \[([^\]]+)\], \[([^\]]+)\], ([\d.]+)\);\s*scene\s*\}\s*\n\s*/// Floor", tests_rs)
    return {
        "from": "tests/pathtrace.rs:169-180, 295-317",
        "rho": float(m.group(1)), "le": float(m.group(2)),
        "width": int(o.group(1)), "height": int(o.group(2)), "spp": int(o.group(3)), "bounces": int(o.group(4)),
        "ambient": float(o.group(5)),
        "expected": float(tol.group(1)), "tolerance": float(tol.group(2)),
        "camera": {"eye": [float(x) for x in cam.group(1).split(",")],
                   "target": [float(x) for x in cam.group(2).split(",")], "yfov": float(cam.group(3))},
        "strategies": ["Mis", "LightOnly", "BsdfOnly"],
    }


def constants(pt_rs: str, tests_rs: str):
    def const(name):
        m = re.search(rf"const {name}: \w+ = ([^;]+);", pt_rs)
        v = m.group(1).strip()
        if v.startswith("1 <<"):
            return 1 << int(v.split("<<")[1])
        return int(v, 0) if not v.startswith("u32") else 0xFFFFFFFF
    floors = {}
    for m in re.finditer(r'parity\(\s*"([a-z]+)",[^;]*?,\s*([\d.]+),\s*\);', tests_rs, re.S):
        floors[m.group(1)] = float(m.group(2))
    return {
        "from": "src/pathtrace.rs:83-98; tests/pathtrace.rs:319-418",
        "MAX_LAYER": const("MAX_LAYER"), "PATHS_PER_DISPATCH": const("PATHS_PER_DISPATCH"),
        "PATHS_PER_SUBMIT": const("PATHS_PER_SUBMIT"), "MAT_STRIDE": const("MAT_STRIDE"),
        "MAT_SLOTS": const("MAT_SLOTS"), "psnr_floors_db": floors,
    }


def main(ref: Path):
    scene_rs = (ref / "src/scene.rs").read_text()
    pt_rs = (ref / "src/pathtrace.rs").read_text()
    tests_rs = (ref / "tests/pathtrace.rs").read_text()
    (OUT / "f16_kat.json").write_text(json.dumps(f16_vectors(scene_rs), indent=1) + "\n")
    (OUT / "furnace.json").write_text(json.dumps(furnace(tests_rs), indent=1) + "\n")
    (OUT / "pt_constants.json").write_text(json.dumps(constants(pt_rs, tests_rs), indent=1) + "\n")
    print("wrote", *(p.name for p in OUT.glob("*.json")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the oxideav-render-vulkan source tree>")
    main(Path(sys.argv[1]))
