"""Scene generator for the reference's .boid scene descriptions.

Reads a .boid file (ParticleDistance, LowerDomain, UpperDomain, then
StartCuboid/Cuboid2/Cyboid/Cyboid2/Recboid/Recboid2 ... End<shape> blocks)
and emits the particles in the order and with the floating-point arithmetic
of the reference generator (generator/generator.cpp: readfile :129-184, the
block readers :187-656, genparticle :660-897, writefile :908-931), so that the
written .grid is byte-identical to the reference generator's output.  All
blocks of one shape are emitted before the next shape, in the order Cuboid,
Cuboid2, Cyboid, Cyboid2, Recboid, Recboid2, as in genparticle.

Quirks kept:
* Cuboid lattices run from lower + 0.5 h to upper - 0.49 h with the spacing
  accumulated by repeated addition.
* Cuboid2 starts at lower + 0.01 h, runs to upper (exclusive), and rotates
  about the block centre by `Angle` interpreted in RADIANS (:712-713).
* Cyboid ignores Spacing and Ratio: it places the centres of a
  floor(w * sqrt(3) / min(w)) grid per axis (:719-750).
* Cyboid2 is a conical shell: rings of max(6, (int)(2 pi r / Spacing))
  particles at every level from lower + 0.5 s to upper - 0.49 s with the
  radius interpolated from R1 * Ratio (bottom) to R1 (top), R1 = mean of the
  x and y half-widths, then one ring at the top face and one at the bottom
  face (:786-850).
* Recboid keeps the Cuboid2 lattice points with tan(Angle * 3.1415 / 180) >
  y / x (IEEE division: x = 0 gives +-inf or NaN) (:854-876); Recboid2
  rotates the Cuboid2 lattice about the ORIGIN by Angle * 3.1415 / 180
  (:878-895).
"""
import math
import warnings

import numpy as np


def _c_round(x):
    """C round(): half away from zero"""
    a = abs(x)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1
    return int(math.copysign(r, x)) if x < 0 else int(r)


_SHAPES = ("StartCuboid", "StartCuboid2", "StartCyboid", "StartCyboid2", "StartRecboid", "StartRecboid2")
_BASE = {"Spacing", "Type", "Lower", "Upper", "Velocity"}
# the fields each block reader accepts and those it requires (:187-656):
# Cuboid2 takes no Enthalpy and needs an Angle
_ACCEPTED = {"Cuboid": _BASE | {"Enthalpy"}, "Cuboid2": _BASE | {"Angle"},
             "Cyboid": _BASE | {"Enthalpy", "Ratio"}, "Cyboid2": _BASE | {"Enthalpy", "Ratio"},
             "Recboid": _BASE | {"Enthalpy", "Angle"}, "Recboid2": _BASE | {"Enthalpy", "Angle"}}
_REQUIRED = {"Cuboid": _BASE, "Cuboid2": _BASE | {"Angle"},
             "Cyboid": _BASE | {"Enthalpy", "Ratio"}, "Cyboid2": _BASE | {"Enthalpy", "Ratio"},
             "Recboid": _BASE | {"Enthalpy", "Angle"}, "Recboid2": _BASE | {"Enthalpy", "Angle"}}


def _c_div(a, b):
    """IEEE double division as C does it (b = 0 gives +-inf or NaN)"""
    if b != 0.0:
        return a / b
    if a == 0.0 or math.isnan(a):
        return math.nan
    return math.copysign(math.inf, a) * math.copysign(1.0, b)


def _lattice2(blk):
    """the Cuboid2 / Recboid lattice (:697-709, :861-863): x and y from
    lower + 0.01 h up to upper (exclusive), z from lower + 0.5 h to
    upper - 0.49 h, spacing accumulated by repeated addition"""
    lo, up = blk["lower"], blk["upper"]
    width = [up[d] - lo[d] for d in range(3)]
    cnt = [_c_round(width[d] / blk["space"]) for d in range(3)]
    h = [width[d] / cnt[d] for d in range(3)]
    px = lo[0] + 0.01 * h[0]
    while px < up[0] - 0.0 * h[0]:
        py = lo[1] + 0.01 * h[1]
        while py < up[1] - 0.0 * h[1]:
            pz = lo[2] + 0.5 * h[2]
            while pz < up[2] - 0.49 * h[2]:
                yield px, py, pz
                pz += h[2]
            py += h[1]
        px += h[0]


def parse_boid(text):
    tokens = []
    for line in text.splitlines():
        if line.startswith("#"):
            # readfile skips '#' lines; inside a block fscanf reads raw tokens,
            # but commented blocks only ever start with '#Start...' in practice
            tokens.append(("#", line))
            continue
        tokens.append(("L", line))
    dom = {"ParticleDistance": None, "LowerDomain": None, "UpperDomain": None}
    blocks = []
    i = 0
    while i < len(tokens):
        kind, line = tokens[i]
        i += 1
        if kind == "#":
            continue
        w = line.split()
        if not w:
            continue
        if w[0] == "ParticleDistance":
            dom["ParticleDistance"] = float(w[1])
        elif w[0] in ("LowerDomain", "UpperDomain"):
            dom[w[0]] = [float(s) for s in w[1:4]]
        elif w[0] in _SHAPES:
            shape = w[0][5:]
            end = "End" + shape
            blk = {"shape": shape, "angle": 0.0, "ratio": 0.0, "enthalpy": 0.0, "velocity": [0.0, 0.0, 0.0],
                   "lower": [0.0, 0.0, 0.0], "upper": [0.0, 0.0, 0.0], "type": 0}
            # the block body is read token by token with fscanf (whitespace
            # separated, comment lines included as tokens)
            words = []
            while i < len(tokens):
                _, l2 = tokens[i]
                i += 1
                words += l2.split()
                if end in words:
                    break
            seen = set()
            k = 0
            bad = None
            while k < len(words) and words[k] != end:
                t = words[k]
                if t not in _ACCEPTED[shape]:
                    bad = "no such indication: %s" % t
                    break
                if t == "Spacing":
                    blk["space"] = float(words[k + 1]); k += 2
                elif t == "Type":
                    blk["type"] = int(words[k + 1]); k += 2
                elif t in ("Lower", "Upper", "Velocity"):
                    blk[t.lower()] = [float(s) for s in words[k + 1:k + 4]]; k += 4
                else:  # Angle, Ratio, Enthalpy
                    blk[t.lower()] = float(words[k + 1]); k += 2
                seen.add(t)
            missing = _REQUIRED[shape] - seen
            if bad is None and missing:
                bad = "%s block without %s" % (shape, ", ".join(sorted(missing)))
            if bad is not None:
                # the reference's block reader fails, the block is dropped and
                # readfile stops there; the blocks read so far are generated
                # (:152-175, :180-183)
                warnings.warn("boid: %s; the rest of the file is ignored" % bad)
                break
            blocks.append(blk)
        # any other line (unknown keywords and shapes included) is ignored
    return dom, blocks


def generate(dom, blocks):
    typ, pos, vel = [], [], []
    for blk in [b for b in blocks if b["shape"] == "Cuboid"]:
        lo, up = blk["lower"], blk["upper"]
        width = [up[d] - lo[d] for d in range(3)]
        cnt = [_c_round(width[d] / blk["space"]) for d in range(3)]
        h = [width[d] / cnt[d] for d in range(3)]
        px = lo[0] + 0.5 * h[0]
        while px < up[0] - 0.49 * h[0]:
            py = lo[1] + 0.5 * h[1]
            while py < up[1] - 0.49 * h[1]:
                pz = lo[2] + 0.5 * h[2]
                while pz < up[2] - 0.49 * h[2]:
                    typ.append(blk["type"]); pos.append((px, py, pz)); vel.append(tuple(blk["velocity"]))
                    pz += h[2]
                py += h[1]
            px += h[0]
    for blk in [b for b in blocks if b["shape"] == "Cuboid2"]:
        lo, up = blk["lower"], blk["upper"]
        width = [up[d] - lo[d] for d in range(3)]
        cnt = [_c_round(width[d] / blk["space"]) for d in range(3)]
        h = [width[d] / cnt[d] for d in range(3)]
        c = [(up[d] + lo[d]) / 2 for d in range(3)]
        ca, sa = math.cos(blk["angle"]), math.sin(blk["angle"])
        px = lo[0] + 0.01 * h[0]
        while px < up[0] - 0.0 * h[0]:
            py = lo[1] + 0.01 * h[1]
            while py < up[1] - 0.0 * h[1]:
                pz = lo[2] + 0.5 * h[2]
                while pz < up[2] - 0.49 * h[2]:
                    nx = (px - c[0]) * ca - (py - c[1]) * sa + c[0]
                    ny = (px - c[0]) * sa + (py - c[1]) * ca + c[1]
                    typ.append(blk["type"]); pos.append((nx, ny, pz)); vel.append(tuple(blk["velocity"]))
                    pz += h[2]
                py += h[1]
            px += h[0]
    for blk in [b for b in blocks if b["shape"] == "Cyboid"]:
        lo, up = blk["lower"], blk["upper"]
        width = [up[d] - lo[d] for d in range(3)]
        side = min(width[0], min(width[1], width[2])) / math.sqrt(3.0)
        nt = [int(math.floor(width[d] / side)) for d in range(3)]
        h = [width[d] / nt[d] for d in range(3)]
        for i in range(nt[0]):
            for j in range(nt[1]):
                for k in range(nt[2]):
                    p = (lo[0] + (i + 0.5) * h[0], lo[1] + (j + 0.5) * h[1], lo[2] + (k + 0.5) * h[2])
                    typ.append(blk["type"]); pos.append(p); vel.append(tuple(blk["velocity"]))
    for blk in [b for b in blocks if b["shape"] == "Cyboid2"]:
        lo, up = blk["lower"], blk["upper"]
        width = [up[d] - lo[d] for d in range(3)]
        c = [0.5 * (up[d] + lo[d]) for d in range(3)]
        s = blk["space"]
        height = width[2]
        R1 = 0.5 * (width[0] + width[1]) * 0.5
        R2 = R1 * blk["ratio"]

        def ring(pz, radius):
            n = max(6, int(2.0 * math.pi * radius / s))
            for ith in range(n):
                th = (2.0 * math.pi * ith) / n
                typ.append(blk["type"])
                pos.append((c[0] + radius * math.cos(th), c[1] + radius * math.sin(th), pz))
                vel.append(tuple(blk["velocity"]))

        pz = lo[2] + 0.5 * s
        while pz < up[2] - 0.49 * s:
            ratio_z = (pz - lo[2]) / height
            ring(pz, R2 + (R1 - R2) * ratio_z)
            pz += s
        ring(up[2], R1)
        ring(lo[2], R2)
    for blk in [b for b in blocks if b["shape"] == "Recboid"]:
        t = math.tan(blk["angle"] * 3.1415 / 180)
        for px, py, pz in _lattice2(blk):
            if t > _c_div(py, px):
                typ.append(blk["type"]); pos.append((px, py, pz)); vel.append(tuple(blk["velocity"]))
    for blk in [b for b in blocks if b["shape"] == "Recboid2"]:
        a = blk["angle"] * 3.1415 / 180
        ca, sa = math.cos(a), math.sin(a)
        for px, py, pz in _lattice2(blk):
            typ.append(blk["type"]); pos.append((px * ca - py * sa, px * sa + py * ca, pz))
            vel.append(tuple(blk["velocity"]))
    return (np.array(typ, np.int32), np.array(pos, np.float64).reshape(-1, 3),
            np.array(vel, np.float64).reshape(-1, 3))


def grid_text(dom, typ, x, v):
    """The reference generator's writefile layout (generator/generator.cpp:948-971)."""
    lo, up = dom["LowerDomain"], dom["UpperDomain"]
    out = ["%f\n" % 0.0,
           "%d %e  %e %e %e  %e %e %e\n" % (len(typ), dom["ParticleDistance"], lo[0], up[0], lo[1], up[1], lo[2], up[2])]
    out += ["%d    %e %e %e  %e %e %e \n" % (typ[i], x[i, 0], x[i, 1], x[i, 2], v[i, 0], v[i, 1], v[i, 2])
            for i in range(len(typ))]
    return "".join(out)


def boid_to_grid(boid_path, grid_path):
    with open(boid_path) as f:
        dom, blocks = parse_boid(f.read())
    typ, x, v = generate(dom, blocks)
    with open(grid_path, "w") as f:
        f.write(grid_text(dom, typ, x, v))
    return len(typ)


def main(argv=None):
    """The reference generator's command line (generator.cpp:117-127):
    `python -m dem_mph_b200.generator [NAME]` reads NAME.boid and writes
    NAME.grid in the current directory (sample.boid / sample.grid without an
    argument)."""
    import sys
    args = sys.argv[1:] if argv is None else argv
    name = args[0] if args else "sample"
    n = boid_to_grid(name + ".boid", name + ".grid")
    sys.stderr.write("%d particles were generated\n" % n)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
