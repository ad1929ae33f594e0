"""Extract the reference's own known-answer vectors into reference_vectors.json.

The reference (tombh/total-viewsheds, Rust) cannot be built in this
environment (no cargo), so its unit tests cannot run.  Their expected values
are the golden vectors that pin the oracle.  This script reads them, as text,
from the reference sources and writes them to ``reference_vectors.json`` beside
this file.  Run it where a reference checkout is present, naming its root
(the argument, or the TVS_REFERENCE_ROOT environment variable):

    python tests/golden/extract_reference_vectors.py REFERENCE_ROOT

Sources (paths inside the reference repository):
  crates/total-viewsheds/src/axes.rs:216-333         5x5 axes at 0 and 135 degrees
  crates/total-viewsheds/src/band_of_sight.rs:230-315  9x9 band shapes at 0/15/90/135
  crates/total-viewsheds/src/cache.rs:87-105        9x9 shape at 35 degrees
  crates/total-viewsheds/src/compute.rs:276-416      9x9 DEMs, totals, ASCII viewsheds
"""

import json
import re
import sys
from pathlib import Path

SRC = Path("crates/total-viewsheds/src")
OUT = Path(__file__).resolve().parent / "reference_vectors.json"

NUM = r"-?\d+(?:\.\d+)?(?:e-?\d+)?"


def fn_body(text, name):
    """Return the source of `fn name(...) { ... }` (brace matched)."""
    m = re.search(r"fn\s+" + re.escape(name) + r"\s*\([^)]*\)[^{]*\{", text)
    if not m:
        raise KeyError(name)
    depth, i = 1, m.end()
    while depth:
        c = text[i]
        depth += c == "{"
        depth -= c == "}"
        i += 1
    return text[m.end():i - 1]


def bracket_groups(body):
    """Top-level [...] groups in order of appearance (nested groups kept inside).
    Attributes such as #[rustfmt::skip] are not data and are skipped."""
    out, depth, start = [], 0, None
    for i, c in enumerate(body):
        if c == "[":
            if depth == 0:
                start = i
            depth += 1
        elif c == "]":
            depth -= 1
            if depth == 0 and not (start > 0 and body[start - 1] == "#"):
                out.append(body[start:i + 1])
    return out


def numbers(group):
    return [float(x) if re.search(r"[.e]", x) else int(x) for x in re.findall(NUM, group)]


def rows(group):
    """[[a, b], [c, d]] -> [[a, b], [c, d]]"""
    return [numbers(g) for g in re.findall(r"\[([^\[\]]*)\]", group[1:-1])]


def strings(group):
    return re.findall(r'"([^"]*)"', group)


def main(root):
    src = root / SRC
    axes = (src / "axes.rs").read_text()
    bos = (src / "band_of_sight.rs").read_text()
    cache = (src / "cache.rs").read_text()
    compute = (src / "compute.rs").read_text()

    vectors = {"source": "tombh/total-viewsheds unit tests", "axes": {}, "band_of_sight": {},
               "cache": {}, "compute": {}}

    for name, angle in (("at_0_degrees", 0), ("at_135_degrees", 135)):
        g = bracket_groups(fn_body(axes, name))
        vectors["axes"][str(angle)] = {
            "width": 5,
            "angle": angle,
            "distances": numbers(g[0]),
            "sight_order": numbers(g[1]),
            "sector_ordered": numbers(g[2]),
        }

    for angle in (0, 15, 90, 135):
        g = bracket_groups(fn_body(bos, f"sector_at_{angle}_degrees"))
        vectors["band_of_sight"][str(angle)] = {
            "width": 9, "scale": 1.0, "max_line_of_sight": 3, "angle": angle,
            "bands": rows(g[0]),
            "distances": numbers(g[1]),
        }

    body = fn_body(cache, "saves_and_loads")
    deltas = re.search(r"vec!\[([^\]]*)\]", body).group(1)
    vectors["cache"] = {
        "width": 9, "scale": 1.0, "max_line_of_sight": 3, "angle": 35,
        "band_deltas": [int(x) for x in re.findall(r"-?\d+(?=i32)", deltas)],
        "distances_len": int(re.search(r"distances\.len\(\),\s*(\d+)", body).group(1)),
        "distance_40": float(re.search(r"distances\[40\],\s*(" + NUM + ")", body).group(1)),
        "distance_last": float(re.search(r"&(" + NUM + r")\)", body).group(1)),
    }

    single = numbers(bracket_groups(fn_body(compute, "single_peak_dem"))[0])
    double = numbers(bracket_groups(fn_body(compute, "double_peak_dem"))[0])
    c = vectors["compute"]
    c["width"], c["scale"], c["max_line_of_sight"], c["rings_per_km"] = 9, 1.0, 3, 5000.0
    c["observer_height"] = 1.8  # compute.rs:41 hard-codes it
    c["dems"] = {"single_peak": single, "double_peak": double}
    c["totals"] = {
        "single_peak": numbers(bracket_groups(fn_body(compute, "single_peak_totals"))[0]),
        "double_peak": numbers(bracket_groups(fn_body(compute, "double_peak_totals"))[0]),
    }
    c["viewsheds"] = {}
    for name in ("summit", "off_summit", "double_peak"):
        body = fn_body(compute, name)
        call = re.search(r"create_viewshed\(&super::(\w+)\(\),\s*(\d+)\)", body)
        c["viewsheds"][name] = {
            "dem": call.group(1).replace("_dem", ""),
            "pov_id": int(call.group(2)),
            "rows": strings(bracket_groups(body)[-1]),
        }

    OUT.write_text(json.dumps(vectors, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    import os
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TVS_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: extract_reference_vectors.py REFERENCE_ROOT "
                 "(or set TVS_REFERENCE_ROOT)")
    main(Path(root))
