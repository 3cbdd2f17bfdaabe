"""Scene generator for the reference's .boid scene descriptions.

Reads a .boid file (ParticleDistance, LowerDomain, UpperDomain, then
StartCuboid ... EndCuboid and StartCuboid2 ... EndCuboid2 blocks) and emits
the particles in the order and with the floating-point arithmetic of the
reference generator (generator/generator.cpp: readfile :127-184, genparticle
:658-739 for Cuboid and Cuboid2, writefile :948-971), so that the written
.grid is byte-identical to the reference generator's output.  All Cuboid
blocks are emitted first, then all Cuboid2 blocks, as in genparticle.

Quirks kept: Cuboid lattices run from lower + 0.5 h to upper - 0.49 h with
the spacing accumulated by repeated addition; Cuboid2 starts at
lower + 0.01 h, runs to upper (exclusive), and rotates about the block
centre by `Angle` interpreted in RADIANS (generator/generator.cpp:712-713).
"""
import math

import numpy as np


def _c_round(x):
    """C round(): half away from zero"""
    a = abs(x)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1
    return int(math.copysign(r, x)) if x < 0 else int(r)


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
        elif w[0] in ("StartCuboid", "StartCuboid2"):
            end = "EndCuboid" if w[0] == "StartCuboid" else "EndCuboid2"
            blk = {"shape": w[0][5:], "angle": 0.0, "velocity": [0.0, 0.0, 0.0]}
            # the block body is read token by token with fscanf (whitespace
            # separated, comment lines included as tokens)
            words = []
            while i < len(tokens):
                _, l2 = tokens[i]
                i += 1
                words += l2.split()
                if end in words:
                    break
            k = 0
            while k < len(words) and words[k] != end:
                t = words[k]
                if t == "Spacing":
                    blk["space"] = float(words[k + 1]); k += 2
                elif t == "Type":
                    blk["type"] = int(words[k + 1]); k += 2
                elif t in ("Lower", "Upper", "Velocity"):
                    blk[t.lower()] = [float(s) for s in words[k + 1:k + 4]]; k += 4
                elif t == "Angle":
                    blk["angle"] = float(words[k + 1]); k += 2
                elif t == "Enthalpy":
                    k += 2
                else:
                    raise ValueError("no such indication: %s" % t)
            blocks.append(blk)
        elif w[0].startswith("Start"):
            raise NotImplementedError("shape %s is not supported by this generator" % w[0])
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
