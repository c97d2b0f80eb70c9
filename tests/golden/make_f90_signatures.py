"""Writes f90_signatures.json: the dummy-argument lists of the reference
subroutines that include/picard_f90.h restates, read from the reference's
Fortran sources (subroutine headers, continuation lines joined).

usage: python tests/golden/make_f90_signatures.py [REFERENCE_DIR]
(default REFERENCE_DIR: /root/reference).  The JSON is committed; the tests
read only the JSON.
"""
from __future__ import annotations

import json
import os
import re
import sys

SOURCES = {
    "CalcDistance": "CalcDistance.f90",
    "ParticlesInitialize": "ParticlesInitialize.f90",
    "BCinflow": "BCinflow.f90",
    "AdvancePosition": "AdvancePosition.f90",
    "ParticlesProduce": "ParticlesProduce.f90",
    "BCoutflow": "BCoutflow.f90",
    "ParticlesTransfer": "ParticlesTransfer.f90",
    "ParticlesGridify": "ParticlesGridify.f90",
    "ParticlesGridifyAll": "ParticlesGridifyAll.f90",
    "BCpotentials": "BCpotentials.f90",
    "CalcEpotential": "CalcEpotential.f90",
    "CalcEfield": "CalcEfield.f90",
    "BCfields": "BCfields.f90",
    "AdvanceVelocity": "AdvanceVelocity.f90",
    "AdvanceVelocityExp": "AdvanceVelocity.f90",
    "AdvanceVelocityImp": "AdvanceVelocity.f90",
    "DumpParticles": "Write.f90",
    "DumpFields": "Write.f90",
}


def header(text: str, name: str) -> tuple[int, list[str]]:
    lines = text.splitlines()
    for n, line in enumerate(lines):
        m = re.match(r"\s*subroutine\s+(\w+)\s*\((.*)$", line, re.I)
        if not m or m.group(1).lower() != name.lower():
            continue
        body = m.group(2)
        k = n
        while body.rstrip().endswith("&"):
            k += 1
            body = body.rstrip()[:-1] + lines[k].strip().lstrip("&")
        args = body.split(")")[0]
        return n + 1, [a.strip() for a in args.split(",") if a.strip()]
    raise KeyError(name)


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = {}
    for name, src in SOURCES.items():
        with open(os.path.join(ref, src)) as f:
            line, args = header(f.read(), name)
        out[name] = {"source": f"{src}:{line}", "args": args}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "f90_signatures.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"wrote {path}: {len(out)} subroutines")


if __name__ == "__main__":
    main()
