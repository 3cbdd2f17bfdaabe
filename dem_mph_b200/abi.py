"""ctypes mirror of include/dmph.h (the C ABI of libdmph.so).

`Params` has the exact layout of `dmph_params`; the constants are those of the
header.  Only plain ctypes is used here, so this module imports without a GPU
and without the CUDA library.
"""
import ctypes as C

TYPE_COUNT = 6
FLUID_BEGIN, FLUID_END = 0, 2
SOLID_BEGIN, SOLID_END = 2, 4
WALL_BEGIN, WALL_END = 4, 6

OK = 0
EINVAL, ECUDA, ENOMEM, EIO, ENAN, ETIMEOUT, ERANGE = -1, -2, -3, -4, -5, -6, -7

PRECISION_FP64 = 0
PRECISION_FP32_SPLIT = 1

FLAG_SURFACE_TENSION_ON = 1 << 0
FLAG_SURFACE_TENSION_OFF = 1 << 1
FLAG_WALL_DEM_COEFFS = 1 << 2
FLAG_RIGID_CLUMPS = 1 << 3
FLAG_ALL_NEIGHBOR_COUNTS = 1 << 4
FLAG_LIST_REUSE = 1 << 5

# dmph_field ids and (dtype, components)
FIELDS = {
    "Force": (0, "f8", 3),
    "VolStrainP": (1, "f8", 1),
    "DivergenceP": (2, "f8", 1),
    "PressureP": (3, "f8", 1),
    "DensityA": (4, "f8", 1),
    "GravityCenter": (5, "f8", 3),
    "PressureA": (6, "f8", 1),
    "NormalSpringConstant": (7, "f8", 1),
    "NormalViscousDampingConstant": (8, "f8", 1),
    "TangentialSpringConstant": (9, "f8", 1),
    "TangentialViscousDampingConstant": (10, "f8", 1),
    "alpha": (11, "f8", 1),
    "DragC": (12, "f8", 1),
    "NeighborCount": (13, "i4", 1),
    "SolidNeighborCount": (14, "i4", 1),
    "CellIndex": (15, "i4", 1),
    "Mass": (16, "f8", 1),
    "VirialPressure": (17, "f8", 1),
}

_D6 = C.c_double * TYPE_COUNT
_D3 = C.c_double * 3


class Params(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("precision", C.c_int32),
        ("flags", C.c_uint32),
        ("reserved0", C.c_int32),
        ("dt", C.c_double),
        ("dem_dt", C.c_double),
        ("output_interval", C.c_double),
        ("vtk_output_interval", C.c_double),
        ("end_time", C.c_double),
        ("radius_ratio_a", C.c_double),
        ("radius_ratio_p", C.c_double),
        ("radius_ratio_v", C.c_double),
        ("density", _D6),
        ("bulk_modulus", _D6),
        ("bulk_viscosity", _D6),
        ("shear_viscosity", _D6),
        ("surface_tension", _D6),
        ("interaction_ratio", _D6 * TYPE_COUNT),
        ("gravity", _D3),
        ("young_modulus", _D6),
        ("poisson_ratio", _D6),
        ("restitution_coefficient", _D6),
        ("viscous_friction_coefficient", _D6),
        ("wall_center", _D3 * TYPE_COUNT),
        ("wall_velocity", _D3 * TYPE_COUNT),
        ("wall_omega", _D3 * TYPE_COUNT),
        ("time", C.c_double),
        ("particle_spacing", C.c_double),
        ("domain_min", _D3),
        ("domain_max", _D3),
    ]

    def copy(self):
        out = Params()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(Params))
        return out


class Info(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("n_fluid", C.c_int32),
        ("n_solid", C.c_int32),
        ("n_wall", C.c_int32),
        ("cell_count", C.c_int32 * 3),
        ("total_cell_count", C.c_int32),
        ("power_count", C.c_int32),
        ("dem_substeps", C.c_int32),
        ("steps", C.c_int64),
        ("rebuilds", C.c_int64),
        ("time", C.c_double),
        ("cell_width", C.c_double * 3),
        ("n0a", C.c_double),
        ("n0p", C.c_double),
        ("r2g", C.c_double),
        ("max_radius", C.c_double),
        ("num_bodies", C.c_int32),
        ("surface_tension", C.c_int32),
        ("kernel_launches", C.c_int64),
    ]


class SurrogateParams(C.Structure):
    """dmph_surrogate_params"""
    _fields_ = [
        ("substeps", C.c_int32),
        ("check_interval", C.c_int32),
        ("tolerance", C.c_double),
        ("fallback_blocks", C.c_int32),
        ("train_iters_per_block", C.c_int32),
        ("batch", C.c_int32),
        ("pool_rows", C.c_int32),
        ("learning_rate", C.c_float),
        ("seed", C.c_uint64),
        ("residual", C.c_int32),
        ("front_tolerance", C.c_double),
    ]


class SurrogateStats(C.Structure):
    """dmph_surrogate_stats"""
    _fields_ = [
        ("calls", C.c_int64),
        ("plain_blocks", C.c_int64),
        ("judged", C.c_int64),
        ("fallbacks", C.c_int64),
        ("samples", C.c_int64),
        ("train_iters", C.c_int64),
        ("pool_rows", C.c_int64),
        ("in_fallback", C.c_int32),
        ("last_error", C.c_double),
        ("last_error_v", C.c_double),
        ("last_loss", C.c_double),
        ("last_front_dev", C.c_double),
        ("front_estimate", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


MLP_IN, MLP_OUT, MLP_FEATURES, MLP_TARGETS = 64, 16, 52, 6


def default_params():
    """The reference's static initialisers (source/DEM-MPH.cpp:61-75): Dt and
    DEMDt 1e100, everything else zero; dim 3."""
    p = Params()
    p.dim = 3
    p.dt = 1.0e100
    p.dem_dt = 1.0e100
    return p
