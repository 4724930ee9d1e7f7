"""Regenerates the golden fixtures in tests/golden from the reference sources.

Run with the illcrawl sources checked out somewhere:
    python tests/golden/make_golden.py <illcrawl source directory>
or with the directory in the ILLCRAWL_REFERENCE environment variable.
Writes:
  spiral_table.txt  -- the 8 x 125 char4 offsets of
                       particle_grid_iteration_order.cl:25-1048 (dx dy dz per line,
                       subcell-major), parsed from the reference file;
  gaunt_factor.sha256 -- sha256 and shape of the reference's gaunt_factor.dat,
                       which illcrawl_b200/data/gaunt_factor.dat must equal;
  chandra_arf.txt   -- the first 1024 entries of chandra.cpp's arf_data table
                       (the entries the arf constructor hands to its
                       tabulated_function, chandra.cpp:1073-1079) as float32 bit
                       patterns, with the constructor's x range start and step.
"""
import decimal
import hashlib
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_dir(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("ILLCRAWL_REFERENCE")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("usage: make_golden.py <illcrawl source directory> "
                         "(or set ILLCRAWL_REFERENCE)")
    return ref


def float32_of_literal(text):
    """The float32 a C++ compiler makes of the literal: the float nearest to
    its exact decimal value (ties to even). Parsing through a double first can
    round twice, so the neighbours of that first guess are compared exactly."""
    exact = decimal.Decimal(text)
    guess = np.float32(float(text))
    best = None
    for c in (np.nextafter(guess, np.float32(-np.inf)), guess,
              np.nextafter(guess, np.float32(np.inf))):
        d = abs(decimal.Decimal(float(c)) - exact)
        even = (int(np.array(c, np.float32).view(np.uint32)) & 1) == 0
        if best is None or d < best[0] or (d == best[0] and even):
            best = (d, c)
    return np.float32(best[1])


def chandra_arf(ref):
    src = open(os.path.join(ref, "chandra.cpp")).read()
    body = src[src.index("arf_data [] = {"):]
    body = body[body.index("{") + 1:body.index("};")]
    lits = re.findall(r"([-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?)f", body)
    ctor = re.search(r"arf_data\s*\+\s*(\d+),.*?\n\s*([0-9.eE+-]+)f,.*?\n\s*([0-9.eE+-]+)f\}",
                     src, re.S)
    n, x0, dx = int(ctor.group(1)), ctor.group(2), ctor.group(3)
    assert len(lits) >= n, (len(lits), n)
    vals = [float32_of_literal(t) for t in lits[:n]]
    return n, x0, dx, vals


def main(argv):
    ref = reference_dir(argv)
    src = open(os.path.join(ref, "particle_grid_iteration_order.cl")).read()
    ents = re.findall(r"\(char4\)\(\s*(-?\d+),\s*(-?\d+),\s*(-?\d+),\s*(-?\d+)\)", src)
    assert len(ents) == 1000, len(ents)
    with open(os.path.join(HERE, "spiral_table.txt"), "w") as f:
        f.write("# particle_grid_iteration_order.cl:25-1048, subcell-major, dx dy dz\n")
        for a, b, c, _ in ents:
            f.write(f"{a} {b} {c}\n")
    raw = open(os.path.join(ref, "gaunt_factor.dat"), "rb").read()
    rows = [l for l in raw.decode().splitlines() if l and not l.startswith("#")]
    with open(os.path.join(HERE, "gaunt_factor.sha256"), "w") as f:
        f.write(f"{hashlib.sha256(raw).hexdigest()} {len(rows)} {len(rows[0].split())}\n")
    n, x0, dx, vals = chandra_arf(ref)
    with open(os.path.join(HERE, "chandra_arf.txt"), "w") as f:
        f.write("# chandra.cpp arf_data[0:%d] as float32 bits (hex), one per line; "
                "chandra.cpp:1073-1079 x_min and dx follow\n" % n)
        f.write(f"x_min {x0}\ndx {dx}\n")
        for v in vals:
            f.write("%08x\n" % int(np.array(v, np.float32).view(np.uint32)))


if __name__ == "__main__":
    main(sys.argv)
