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


class a3d_server_config(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_double), ("residual_drop", C.c_double), ("max_active", C.c_int32),
                ("chunk_iters", C.c_int32), ("max_iters", C.c_int32), ("device", C.c_int32),
                ("warm_start", C.c_int32), ("kz", C.c_int32), ("sequence", C.c_int32),
                ("sequence_max_iters", C.c_int32), ("sequence_drop", C.c_double)]


class a3d_request(C.Structure):
    _fields_ = [("shape", a3d_shape), ("cells", C.c_double), ("M", C.c_double), ("alpha_deg", C.c_double),
                ("delta_deg", C.c_double), ("F", C.c_double * 5), ("fix", C.c_double * 15),
                ("ref_S", C.c_double), ("ref_xcg", C.c_double), ("ref_zcg", C.c_double), ("ref_c", C.c_double),
                ("xT", C.c_double), ("geometry_key", C.c_uint64)]


class a3d_result(C.Structure):
    _fields_ = [("status", C.c_int32), ("warm", C.c_int32), ("iterations", C.c_int64),
                ("CL", C.c_double), ("CD", C.c_double), ("Cm", C.c_double), ("CDi", C.c_double),
                ("residual", C.c_double), ("res0", C.c_double),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("coarse_iterations", C.c_int64)]
