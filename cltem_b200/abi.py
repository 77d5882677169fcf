"""ctypes mirror of include/mslice.h (structs, status codes, constants).

The layouts must match the C header field for field; tests/test_abi.py checks the sizes against
the library's own view of them.
"""
import ctypes as C

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_STATE = 3
ERR_CANCELLED = 4
ERR_OOM = 5
ERR_UNSUPPORTED = 6

MODE_CTEM = 1
MODE_STEM = 2
MODE_CBED = 3

KIRKLAND = 0
PENG = 1
LOBATO = 2

MAX_DETECTORS = 16


class Aberration(C.Structure):
    _fields_ = [("mag", C.c_double), ("ang", C.c_double)]


class Detector(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("inner", C.c_double), ("outer", C.c_double),
                ("xcentre", C.c_double), ("ycentre", C.c_double)]


class Config(C.Structure):
    _fields_ = [
        ("mode", C.c_int),
        ("double_precision", C.c_int),
        ("resolution", C.c_int),
        ("allow_any_resolution", C.c_int),
        ("slice_thickness", C.c_double),
        ("slice_offset", C.c_double),
        ("padding_xy", C.c_double),
        ("padding_z", C.c_double),
        ("full3d", C.c_int),
        ("full3d_integrals", C.c_int),
        ("inverse_limit_factor", C.c_double),
        ("struct_limits", C.c_double * 6),
        ("voltage", C.c_double),
        ("C10", C.c_double), ("C12", Aberration), ("C21", Aberration), ("C23", Aberration),
        ("C30", C.c_double), ("C32", Aberration), ("C34", Aberration), ("C41", Aberration),
        ("C43", Aberration), ("C45", Aberration),
        ("C50", C.c_double), ("C52", Aberration), ("C54", Aberration), ("C56", Aberration),
        ("cond_ap", C.c_double), ("cond_ap_smooth", C.c_double),
        ("obj_ap", C.c_double), ("obj_ap_smooth", C.c_double),
        ("beam_tilt", C.c_double), ("beam_azimuth", C.c_double),
        ("alpha", C.c_double), ("delta", C.c_double),
        ("ctem_area", C.c_double * 4),
        ("stem_area", C.c_double * 4),
        ("stem_pixels_x", C.c_int), ("stem_pixels_y", C.c_int),
        ("stem_padding", C.c_double),
        ("cbed_x", C.c_double), ("cbed_y", C.c_double), ("cbed_padding", C.c_double),
        ("n_detectors", C.c_int),
        ("detectors", Detector * MAX_DETECTORS),
        ("intermediate_slices", C.c_int),
        ("ctem_image", C.c_int),
        ("probe_batch", C.c_int),
        ("iterations", C.c_int),
        ("mixed_static", C.c_int),
        ("stem_moving_frame", C.c_int),
        ("stem_job_pixels", C.c_int),
        ("chromatic", C.c_int),
        ("chromatic_cc", C.c_double),
        ("chromatic_hwhm_neg", C.c_double), ("chromatic_hwhm_pos", C.c_double),
        ("source_size", C.c_int),
        ("source_fwhm", C.c_double),
        ("seed", C.c_ulonglong),
        ("plasmon", C.c_int),
        ("plasmon_individual", C.c_int),
        ("plasmon_mfp", C.c_double),
        ("plasmon_char_angle", C.c_double),
        ("plasmon_crit_angle", C.c_double),
    ]


class Geometry(C.Structure):
    _fields_ = [
        ("sim_x", C.c_double * 2), ("sim_y", C.c_double * 2),
        ("full_x", C.c_double * 2), ("full_y", C.c_double * 2),
        ("z_lims", C.c_double * 2), ("padding_z", C.c_double * 2),
        ("real_scale", C.c_double), ("inverse_scale", C.c_double), ("angle_scale", C.c_double),
        ("wavelength", C.c_double), ("wavenumber", C.c_double),
        ("sigma", C.c_double), ("wavevector", C.c_double * 3),
        ("k_max", C.c_double), ("dz", C.c_double),
        ("n_slices", C.c_int), ("pre_slices", C.c_int),
        ("blocks_x", C.c_int), ("blocks_y", C.c_int),
        ("load_blocks_x", C.c_int), ("load_blocks_y", C.c_int), ("load_blocks_z", C.c_int),
        ("block_scale_x", C.c_double), ("block_scale_y", C.c_double),
        ("crop", C.c_uint * 4),
        ("n_outputs", C.c_int),
    ]


def geometry_dict(g: Geometry) -> dict:
    out = {}
    for name, typ in Geometry._fields_:
        v = getattr(g, name)
        out[name] = list(v) if hasattr(v, "__len__") else v
    return out


def config_defaults() -> Config:
    """A Config holding SimulationManager's defaults (src/simulation/simulationmanager.cpp:8-50,
    src/simulation/structure/simulationcell.cpp:7-13, commonstructs.h:210-215)."""
    c = Config()
    c.mode = MODE_CTEM
    c.double_precision = 0
    c.resolution = 256
    c.slice_thickness = 1.0
    c.slice_offset = 0.0
    c.padding_xy = 8.0
    c.padding_z = 3.0
    c.full3d = 0
    c.full3d_integrals = 20
    c.inverse_limit_factor = 2.0 / 3.0
    c.voltage = 200.0
    c.C30 = 10000.0
    c.cond_ap = 20.0
    c.obj_ap = 100.0
    c.alpha = 0.3
    c.delta = 30.0
    c.ctem_area[:] = [0.0, 10.0, 0.0, 10.0]
    c.stem_area[:] = [0.0, 10.0, 0.0, 10.0]
    c.stem_pixels_x = 64
    c.stem_pixels_y = 64
    # PlasmonScattering defaults (plasmon.h: 10 nm, 1 mrad, 0.1 mrad, type full)
    c.plasmon_mfp = 100.0
    c.plasmon_char_angle = 1.0
    c.plasmon_crit_angle = 0.1
    return c
