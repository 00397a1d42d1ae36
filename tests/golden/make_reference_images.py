"""Copies the reference's own rendered images of its synthetic `dual-eclipse`
benchmark fixture into tests/golden/, with their provenance.

The reference publishes these PNGs beside its benchmark results
(benchmarks/m4pro-2026-10-15/current/dual-eclipse-spp{1,32}.png, rendered on
an Apple M4 Pro; the same images rendered on a Radeon RX 7600 XT, in
benchmarks/optimizations/rx7600xt-2026-10-04/, differ from them by 0.08/255
display MAE on the bodies). They are the only outputs of the reference's
integrator in the repository, so they pin the oracle and the CUDA path to the
reference itself. The fixture scene is defined in code at
src/render_benchmark.rs:339-362; the request that rendered them is
benchmarks/optimizations/rx7600xt-2026-10-04/request.json (1280x720 display,
75% trace scale, 4 bounces, 32 image samples).

Run it in the container that holds the reference checkout:
    python tests/golden/make_reference_images.py /path/to/reference
"""
from __future__ import annotations

import hashlib
import json
import shutil
import sys
from pathlib import Path

GOLDEN = Path(__file__).resolve().parent
SOURCE = "benchmarks/m4pro-2026-10-15/current"
CROSS_CHECK = "benchmarks/optimizations/rx7600xt-2026-10-04"


def main(reference: Path) -> None:
    record = {"fixture": "src/render_benchmark.rs:339-362 (dual-eclipse, step 0)",
              "request": f"{CROSS_CHECK}/request.json", "images": {}}
    for spp in (1, 32):
        src = reference / SOURCE / f"dual-eclipse-spp{spp}.png"
        dst = GOLDEN / f"reference_dual_eclipse_spp{spp}.png"
        shutil.copyfile(src, dst)
        other = reference / CROSS_CHECK / f"dual-eclipse-spp{spp}.png"
        record["images"][dst.name] = {
            "source": f"{SOURCE}/{src.name}",
            "sha256": hashlib.sha256(dst.read_bytes()).hexdigest(),
            "cross_check": f"{CROSS_CHECK}/{other.name}",
            "cross_check_sha256": hashlib.sha256(other.read_bytes()).hexdigest(),
        }
    (GOLDEN / "reference_images.json").write_text(json.dumps(record, indent=1) + "\n")


if __name__ == "__main__":
    main(Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
