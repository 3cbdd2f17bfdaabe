"""Readers and writers of the reference's text formats, for Python callers.

- dem.data: keyword lines read with the reference's sscanf patterns
  (readDataFile, source/DEM-MPH.cpp:621-679).  As with sscanf, a keyword line
  with too few numbers still assigns the ones it has, and the line is then
  reported as invalid.
- .grid / .prof: line 1 Time, line 2 ``N dx xmin xmax ymin ymax zmin zmax``,
  then N rows ``type x y z vx vy vz`` (readGridFile :681-851, writeProfFile
  :853-877, generator/generator.cpp:948-971).

The C++ executable reads the same formats through libdmph.so
(dmph_read_data_file / dmph_read_grid_file); both are checked against each
other in tests/test_files.py.
"""
import re

import numpy as np

from .abi import Params, TYPE_COUNT, default_params

_FLOAT = re.compile(
    r"[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)", re.IGNORECASE)

# (format, target) in the reference's order of attempts (:634-660)
_SCALARS = ["Dt", "DEMDt", "OutputInterval", "VtkOutputInterval", "EndTime",
            "RadiusRatioA", "RadiusRatioP", "RadiusRatioV"]
_SCALAR_FIELD = {"Dt": "dt", "DEMDt": "dem_dt", "OutputInterval": "output_interval",
                 "VtkOutputInterval": "vtk_output_interval", "EndTime": "end_time",
                 "RadiusRatioA": "radius_ratio_a", "RadiusRatioP": "radius_ratio_p",
                 "RadiusRatioV": "radius_ratio_v"}
_ARRAYS_A = [("Density", "density"), ("BulkModulus", "bulk_modulus"),
             ("BulkViscosity", "bulk_viscosity"), ("ShearViscosity", "shear_viscosity"),
             ("SurfaceTension", "surface_tension")]
_ARRAYS_B = [("YoungModulus", "young_modulus"), ("PoissonRatio", "poisson_ratio"),
             ("RestitutionCoefficient", "restitution_coefficient"),
             ("ViscousFrictionCoefficient", "viscous_friction_coefficient")]


def _scan(line, items):
    """Emulate sscanf with a format made of literal words (str, each preceded by
    a whitespace directive) and runs of %lf (int = how many).  Returns the
    parsed values (a prefix when a number is missing, as sscanf assigns them
    one by one) or None when a literal before the first number did not
    match."""
    pos = 0
    vals = []
    for it in items:
        if isinstance(it, str):
            while pos < len(line) and line[pos].isspace():
                pos += 1
            if not line.startswith(it, pos):
                return vals if vals else None
            pos += len(it)
        else:
            for _ in range(it):
                while pos < len(line) and line[pos].isspace():
                    pos += 1
                m = _FLOAT.match(line, pos)
                if not m:
                    return vals
                vals.append(float(m.group(0)))
                pos = m.end()
    return vals


def parse_data_text(text, params=None, invalid=None):
    """Parse dem.data text into a Params (see module docstring)."""
    p = params if params is not None else default_params()
    for raw in text.splitlines(keepends=True):
        if raw.startswith("#"):
            continue
        done = False
        for key in _SCALARS:
            v = _scan(raw, [key, 1])
            if v:
                setattr(p, _SCALAR_FIELD[key], v[0])
                done = True
                break
        if done:
            continue

        def try_array(key, field, arr=None):
            v = _scan(raw, key.split() + [TYPE_COUNT])
            if v is None:
                return False
            tgt = arr if arr is not None else getattr(p, field)
            for k, x in enumerate(v):
                tgt[k] = x
            return len(v) == TYPE_COUNT

        for key, field in _ARRAYS_A:
            if try_array(key, field):
                done = True
                break
        if not done:
            for t in range(TYPE_COUNT):
                if try_array("InteractionRatio(Type%d)" % t, None, p.interaction_ratio[t]):
                    done = True
                    break
        if not done:
            v = _scan(raw, ["Gravity", 3])
            if v is not None:
                for k, x in enumerate(v):
                    p.gravity[k] = x
                done = len(v) == 3
        if not done:
            for key, field in _ARRAYS_B:
                if try_array(key, field):
                    done = True
                    break
        if not done:
            for w in (4, 5):
                vals = _scan(raw, ["Wall%d" % w, "Center", 3, "Velocity", 3, "Omega", 3])
                if vals is not None:
                    for k, x in enumerate(vals):
                        tgt = (p.wall_center, p.wall_velocity, p.wall_omega)[k // 3]
                        tgt[w][k % 3] = x
                    if len(vals) == 9:
                        done = True
                        break
        if not done and invalid is not None:
            invalid.append(raw)
    return p


def read_data_file(path, params=None, invalid=None):
    with open(path, "r") as f:
        return parse_data_text(f.read(), params, invalid)


def read_grid(path, params=None):
    """Read a .grid/.prof file.  Returns (params, type[int32], x[N,3], v[N,3]);
    params gets time, particle_spacing and the domain from the header."""
    p = params if params is not None else default_params()
    with open(path, "r") as f:
        t = float(f.readline().split()[0])
        head = f.readline().split()
        n = int(head[0])
        vals = [float(s) for s in head[1:8]]
        data = np.loadtxt(f, dtype=np.float64, max_rows=n, ndmin=2)
    p.time = t
    p.particle_spacing = vals[0]
    p.domain_min[0], p.domain_max[0] = vals[1], vals[2]
    p.domain_min[1], p.domain_max[1] = vals[3], vals[4]
    p.domain_min[2], p.domain_max[2] = vals[5], vals[6]
    if data.shape[0] != n:
        raise ValueError("%s: header says %d particles, found %d rows" % (path, n, data.shape[0]))
    typ = data[:, 0].astype(np.int32)
    x = np.ascontiguousarray(data[:, 1:4])
    v = np.ascontiguousarray(data[:, 4:7])
    return p, typ, x, v


def write_grid(path, params, typ, x, v, time=0.0, prof=False):
    """Write a .grid (generator layout, generator/generator.cpp:948-971) or,
    with prof=True, a .prof (writeProfFile layout, source/DEM-MPH.cpp:853-877)."""
    n = len(typ)
    with open(path, "w") as f:
        if prof:
            f.write("%e\n" % time)
            f.write("%d %e %e %e %e %e %e %e\n" % (
                n, params.particle_spacing, params.domain_min[0], params.domain_max[0],
                params.domain_min[1], params.domain_max[1], params.domain_min[2], params.domain_max[2]))
            fmt = "%d %e %e %e  %e %e %e\n"
        else:
            f.write("%f\n" % time)
            f.write("%d %e  %e %e %e  %e %e %e\n" % (
                n, params.particle_spacing, params.domain_min[0], params.domain_max[0],
                params.domain_min[1], params.domain_max[1], params.domain_min[2], params.domain_max[2]))
            fmt = "%d    %e %e %e  %e %e %e \n"
        rows = [fmt % (int(typ[i]), x[i, 0], x[i, 1], x[i, 2], v[i, 0], v[i, 1], v[i, 2])
                for i in range(n)]
        f.write("".join(rows))


def write_data_file(path, p):
    """Write a dem.data the reference (and dmph_read_data_file) can read."""
    def row(name, arr):
        return "%-28s %s\n" % (name, " ".join("%.17g" % arr[k] for k in range(TYPE_COUNT)))
    s = ["# written by dem_mph_b200.files.write_data_file\n"]
    for key in _SCALARS:
        s.append("%-28s %.17g\n" % (key, getattr(p, _SCALAR_FIELD[key])))
    for key, field in _ARRAYS_A:
        s.append(row(key, getattr(p, field)))
    for t in range(TYPE_COUNT):
        s.append(row("InteractionRatio(Type%d)" % t, p.interaction_ratio[t]))
    s.append("%-28s %.17g %.17g %.17g\n" % ("Gravity", p.gravity[0], p.gravity[1], p.gravity[2]))
    for key, field in _ARRAYS_B:
        s.append(row(key, getattr(p, field)))
    for w in (4, 5):
        c, v, o = p.wall_center[w], p.wall_velocity[w], p.wall_omega[w]
        s.append("Wall%d  Center %.17g %.17g %.17g Velocity %.17g %.17g %.17g Omega %.17g %.17g %.17g\n"
                 % (w, c[0], c[1], c[2], v[0], v[1], v[2], o[0], o[1], o[2]))
    with open(path, "w") as f:
        f.write("".join(s))
