"""Regenerates the golden fixtures in tests/golden from the reference sources.

Run in a checkout that has the illcrawl sources at /root/reference:
    python tests/golden/make_golden.py
Writes:
  spiral_table.txt  -- the 8 x 125 char4 offsets of
                       particle_grid_iteration_order.cl:25-1048 (dx dy dz per line,
                       subcell-major), parsed from the reference file;
  gaunt_factor.sha256 -- sha256 and shape of the reference's gaunt_factor.dat,
                       which illcrawl_b200/data/gaunt_factor.dat must equal.
"""
import hashlib
import os
import re

REF = "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    src = open(os.path.join(REF, "particle_grid_iteration_order.cl")).read()
    ents = re.findall(r"\(char4\)\(\s*(-?\d+),\s*(-?\d+),\s*(-?\d+),\s*(-?\d+)\)", src)
    assert len(ents) == 1000, len(ents)
    with open(os.path.join(HERE, "spiral_table.txt"), "w") as f:
        f.write("# particle_grid_iteration_order.cl:25-1048, subcell-major, dx dy dz\n")
        for a, b, c, _ in ents:
            f.write(f"{a} {b} {c}\n")
    raw = open(os.path.join(REF, "gaunt_factor.dat"), "rb").read()
    rows = [l for l in raw.decode().splitlines() if l and not l.startswith("#")]
    with open(os.path.join(HERE, "gaunt_factor.sha256"), "w") as f:
        f.write(f"{hashlib.sha256(raw).hexdigest()} {len(rows)} {len(rows[0].split())}\n")


if __name__ == "__main__":
    main()
