"""ctypes mirrors of the plain-C records in include/aero3d.h (no library is loaded here)."""
import ctypes as C

A3D_MAX_ENGINES = 2
A3D_MAX_EXITS = 2
A3D_ENV_N = 300

A3D_OK = 0
STATUS_NAMES = {0: "A3D_OK", 1: "A3D_ERR_ARG", 2: "A3D_ERR_CUDA", 3: "A3D_ERR_NOMEM",
                4: "A3D_ERR_NONFINITE", 5: "A3D_ERR_STATE", 6: "A3D_ERR_BUDGET",
                7: "A3D_ERR_TIMEOUT", 8: "A3D_ERR_NODEVICE"}


class a3d_surface(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("x0", "z0", "semi", "cr", "ct", "tanL", "tanD_pt", "tanI_pt",
                                          "tanD_deg", "tanI_deg", "tcR", "tcT", "camber", "sA")] + \
               [("bb", C.c_double * 4)]


class a3d_engine(C.Structure):
    _fields_ = [("x0", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("internal", C.c_int32), ("env_n", C.c_int32), ("env_xmax", C.c_double),
                ("env_R", C.c_float * (A3D_ENV_N + 1)), ("pad_", C.c_float)]


class a3d_exit(C.Structure):
    _fields_ = [("type", C.c_int32), ("pad_", C.c_int32), ("x", C.c_double), ("R", C.c_double),
                ("Rin", C.c_double)]


class a3d_shape(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("fus_L", "fus_R0", "fus_Ln", "fus_Lt", "fus_xt0", "fus_Re",
                                          "fus_noseP", "fus_tailUp")] + \
               [("wing", a3d_surface), ("htail", a3d_surface), ("vtail", a3d_surface),
                ("ref_b", C.c_double), ("view_Rmax", C.c_double), ("lip_x", C.c_double), ("lip_r", C.c_double),
                ("n_engines", C.c_int32), ("n_exits", C.c_int32),
                ("engines", a3d_engine * A3D_MAX_ENGINES), ("exits", a3d_exit * A3D_MAX_EXITS)]
