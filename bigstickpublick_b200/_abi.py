"""ctypes mirror of include/bsg.h and include/bsg_host.h.

Field order and types match the C structs exactly; the libraries are loaded
from the package directory (built in-tree), never from a system path.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))

i8p = C.POINTER(C.c_int8)
i16p = C.POINTER(C.c_int16)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
u64p = C.POINTER(C.c_uint64)

BSG_OK = 0
STATUS_NAMES = {
    0: "BSG_OK", 1: "BSG_ERR_BAD_TABLE", 2: "BSG_ERR_OOB_INDEX", 3: "BSG_ERR_CUDA",
    4: "BSG_ERR_NOMEM", 5: "BSG_ERR_TIMEOUT", 6: "BSG_ERR_NAN", 7: "BSG_ERR_ARG",
    8: "BSG_ERR_UNSUPPORTED", 9: "BSG_ERR_NOT_CONVERGED",
}
BSG_OP_SPE, BSG_OP_PP, BSG_OP_NN, BSG_OP_PN = 1, 2, 3, 4
BSG_PREC_FP32, BSG_PREC_FP64 = 4, 8
BSG_ACCUMULATE, BSG_DEVICE_PTRS = 1, 2


class BsgTables(C.Structure):
    _fields_ = [
        ("dimbasis", C.c_int64), ("nsd_p", C.c_int64), ("nsd_n", C.c_int64),
        ("pstart", i64p), ("nstart", i64p),
        ("np1b", C.c_int64), ("p1b_isd", i64p), ("p1b_fsd", i64p),
        ("p1b_cop", i16p), ("p1b_dop", i16p), ("p1b_phase", i8p),
        ("nn1b", C.c_int64), ("n1b_isd", i64p), ("n1b_fsd", i64p),
        ("n1b_cop", i16p), ("n1b_dop", i16p), ("n1b_phase", i8p),
        ("np2b", C.c_int64), ("p2b_isd", i64p), ("p2b_fsd", i64p),
        ("p2b_op", i32p), ("p2b_phase", i8p),
        ("nn2b", C.c_int64), ("n2b_isd", i64p), ("n2b_fsd", i64p),
        ("n2b_op", i32p), ("n2b_phase", i8p),
        ("nmatpp", C.c_int64), ("nmatnn", C.c_int64), ("nmatpn", C.c_int64),
        ("hmatpp", f32p), ("hmatnn", f32p), ("hmatpn", f32p),
        ("nhsps_pl", C.c_int32), ("nhsps_pr", C.c_int32),
        ("nhsps_nl", C.c_int32), ("nhsps_nr", C.c_int32),
        ("cpnpair", i64p), ("dpnpair", i64p),
        ("call_spe", C.c_int32), ("pspe_h", f32p), ("nspe_h", f32p),
        ("nbundles", C.c_int64), ("optype", i32p), ("hchar", i32p),
        ("pxstart", i64p), ("pxend", i64p), ("nxstart", i64p), ("nxend", i64p),
        ("cstride", i64p),
    ]


class BsgConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_nb", C.c_int32),
                ("validate", C.c_int32), ("pn_table_max", C.c_int32)]


class BsgLanczosParams(C.Structure):
    _fields_ = [
        ("nkeep", C.c_int32), ("niter", C.c_int32), ("nthick_add", C.c_int32),
        ("max_restarts", C.c_int32), ("nb", C.c_int32), ("matvec_prec", C.c_int32),
        ("fixed_iter", C.c_int32), ("ncheck", C.c_int32), ("converge_tol", C.c_double),
        ("want_vectors", C.c_int32), ("pivot", C.c_int32), ("seed", C.c_uint64),
        ("lanc_prec", C.c_int32), ("reserved", C.c_int32),
    ]


class BsgSpecies(C.Structure):
    _fields_ = [
        ("nsps", C.c_int32), ("nl", C.c_int32), ("m2", C.POINTER(C.c_int32)), ("par", C.POINTER(C.c_int32)),
        ("nsd", C.c_int64), ("sd_bits", C.POINTER(C.c_uint64)), ("xstart", C.POINTER(C.c_int64)),
        ("nsectors", C.c_int32), ("sector_start", C.POINTER(C.c_int64)), ("sector_end", C.POINTER(C.c_int64)),
    ]


class BsgReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("total_iterations", C.c_int32),
        ("restarts", C.c_int32), ("random_restarts", C.c_int32),
        ("matvecs", C.c_int32), ("converged", C.c_int32),
        ("t_matvec_ms", C.c_double), ("t_reorth_ms", C.c_double),
        ("t_eig_ms", C.c_double), ("t_total_ms", C.c_double),
    ]


class BsgStats(C.Structure):
    _fields_ = [
        ("n_ops_pp", C.c_int64), ("n_ops_nn", C.c_int64), ("n_ops_pn", C.c_int64),
        ("n_ops_spe", C.c_int64), ("jump_bytes", C.c_int64), ("derived_bytes", C.c_int64),
        ("n_rows", C.c_int64), ("n_contrib", C.c_int64),
        ("kernel_launches_per_matvec", C.c_int32), ("reserved", C.c_int32),
        ("density_ms", C.c_double), ("density_rows", C.c_int64),
        ("density_launches", C.c_int32), ("reserved2", C.c_int32),
        ("apply1b_ms", C.c_double), ("grad_ms", C.c_double),
        ("n_ops_ppp", C.c_int64), ("n_ops_nnn", C.c_int64), ("n_ops_ppn", C.c_int64), ("n_ops_pnn", C.c_int64),
    ]


class BsgTables3(C.Structure):
    _fields_ = [
        ("p2b_cop", i32p), ("p2b_dop", i32p), ("n2b_cop", i32p), ("n2b_dop", i32p),
        ("np3b", C.c_int64), ("p3b_isd", i64p), ("p3b_fsd", i64p), ("p3b_op", i32p), ("p3b_phase", i8p),
        ("nn3b", C.c_int64), ("n3b_isd", i64p), ("n3b_fsd", i64p), ("n3b_op", i32p), ("n3b_phase", i8p),
        ("nmatppp", C.c_int64), ("nmatnnn", C.c_int64), ("nmatppn", C.c_int64), ("nmatpnn", C.c_int64),
        ("hmatppp", f32p), ("hmatnnn", f32p), ("hmatppn", f32p), ("hmatpnn", f32p),
        ("npairs_p", C.c_int32), ("npairs_n", C.c_int32),
        ("cppntriplet", i32p), ("dppntriplet", i32p), ("cpnntriplet", i32p), ("dpnntriplet", i32p),
    ]


class BsgModel3Spec(C.Structure):
    _fields_ = [("w2", C.c_double), ("w3", C.c_double), ("seed", C.c_uint64)]


class BsgOrbit(C.Structure):
    _fields_ = [("nr", C.c_int32), ("l", C.c_int32), ("j2", C.c_int32), ("w", C.c_int32)]


class BsgTbme(C.Structure):
    _fields_ = [("a", C.c_int32), ("b", C.c_int32), ("c", C.c_int32), ("d", C.c_int32),
                ("J", C.c_int32), ("T", C.c_int32), ("v", C.c_double)]


class BsgModelSpec(C.Structure):
    _fields_ = [
        ("norb", C.c_int32), ("orbits", C.POINTER(BsgOrbit)),
        ("np", C.c_int32), ("nn", C.c_int32), ("jz2", C.c_int32), ("parity", C.c_int32),
        ("ntbme", C.c_int32), ("tbme", C.POINTER(BsgTbme)), ("spe", f64p),
        ("spe_scale", C.c_double), ("tbme_scale", C.c_double),
    ]


class BsgDensityTables(C.Structure):
    _fields_ = [
        ("np1b", C.c_int64), ("p1b_isd", i64p), ("p1b_fsd", i64p),
        ("p1b_cop", i16p), ("p1b_dop", i16p), ("p1b_phase", i8p),
        ("nn1b", C.c_int64), ("n1b_isd", i64p), ("n1b_fsd", i64p),
        ("n1b_cop", i16p), ("n1b_dop", i16p), ("n1b_phase", i8p),
        ("nbundles", C.c_int64), ("optype", i32p), ("hchar", i32p),
        ("pxstart", i64p), ("pxend", i64p), ("nxstart", i64p), ("nxend", i64p), ("cstride", i64p),
    ]


class BsgHostTables(C.Structure):
    _fields_ = [
        ("t", BsgTables),
        ("nsectors_p", C.c_int32), ("nsectors_n", C.c_int32),
        ("psector_start", i64p), ("psector_end", i64p),
        ("psector_jz2", i32p), ("psector_par", i32p),
        ("nsector_start", i64p), ("nsector_end", i64p),
        ("nsector_jz2", i32p), ("nsector_par", i32p),
        ("psector_conj", i32p),
        ("nhsps_p", C.c_int32), ("nhsps_n", C.c_int32),
        ("sp_orb_p", i32p), ("sp_m2_p", i32p), ("sp_orb_n", i32p), ("sp_m2_n", i32p),
        ("sd_bits_p", u64p), ("sd_bits_n", u64p),
        ("npairs_pp", C.c_int64), ("npairs_nn", C.c_int64), ("npairs_pn", C.c_int64),
        ("priv", C.c_void_p),
        ("dt", BsgDensityTables),
        ("t3", C.POINTER(BsgTables3)),
    ]


def lib_path(name):
    return os.path.join(_HERE, name)


_host = None
_gpu = None


def host_lib():
    """libbsghost.so: the CPU table builder (stand-in for the Fortran host)."""
    global _host
    if _host is None:
        path = lib_path("libbsghost.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() first")
        lib = C.CDLL(path)
        lib.bsg_host_build.argtypes = [C.POINTER(BsgModelSpec), C.POINTER(C.POINTER(BsgHostTables))]
        lib.bsg_host_build.restype = C.c_int
        lib.bsg_host_build3.argtypes = [C.POINTER(BsgModelSpec), C.POINTER(BsgModel3Spec),
                                        C.POINTER(C.POINTER(BsgHostTables))]
        lib.bsg_host_build3.restype = C.c_int
        lib.bsg_host_free.argtypes = [C.POINTER(BsgHostTables)]
        lib.bsg_host_free.restype = None
        lib.bsg_host_last_error.argtypes = []
        lib.bsg_host_last_error.restype = C.c_char_p
        lib.bsg_host_me_jacobian.argtypes = [C.POINTER(BsgHostTables), C.c_int, f64p, f64p]
        lib.bsg_host_me_jacobian.restype = C.c_int
        _host = lib
    return _host


def gpu_lib():
    """libbsgpu.so: the sm_100a engine.  Raises when it is missing: there is no
    CPU fallback for the product path."""
    global _gpu
    if _gpu is None:
        path = lib_path("libbsgpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: the CUDA engine must be built "
                               "(__graft_entry__.build()); there is no CPU fallback")
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.bsg_create.argtypes = [C.POINTER(BsgTables), C.POINTER(BsgConfig), C.POINTER(vp)]
        lib.bsg_create.restype = C.c_int
        lib.bsg_create3.argtypes = [C.POINTER(BsgTables), C.POINTER(BsgTables3), C.POINTER(BsgConfig), C.POINTER(vp)]
        lib.bsg_create3.restype = C.c_int
        lib.bsg_destroy.argtypes = [vp]
        lib.bsg_destroy.restype = C.c_int
        lib.bsg_strerror.argtypes = [C.c_int]
        lib.bsg_strerror.restype = C.c_char_p
        lib.bsg_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        lib.bsg_last_error.restype = C.c_int
        lib.bsg_applyh.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int]
        lib.bsg_applyh.restype = C.c_int
        lib.bsg_applyh_stream.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, vp]
        lib.bsg_applyh_stream.restype = C.c_int
        lib.bsg_lanczos.argtypes = [vp, C.POINTER(BsgLanczosParams), f64p, f64p, f64p,
                                    C.POINTER(BsgReport)]
        lib.bsg_lanczos.restype = C.c_int
        lib.bsg_grad.argtypes = [vp, f64p, C.c_int, f64p, f64p, f64p, f64p, f64p]
        lib.bsg_grad.restype = C.c_int
        lib.bsg_density1b.argtypes = [vp, C.POINTER(BsgDensityTables), f64p, C.c_int, f64p, f64p]
        lib.bsg_density1b.restype = C.c_int
        lib.bsg_apply1b.argtypes = [vp, C.POINTER(BsgDensityTables), f64p, f64p, f64p, f64p, C.c_int]
        lib.bsg_apply1b.restype = C.c_int
        lib.bsg_get_stats.argtypes = [vp, C.POINTER(BsgStats)]
        lib.bsg_get_stats.restype = C.c_int
        lib.bsg_validate_tables.argtypes = [C.POINTER(BsgTables), C.c_char_p, C.c_size_t]
        lib.bsg_validate_tables.restype = C.c_int
        lib.bsg_validate_tables3.argtypes = [C.POINTER(BsgTables), C.POINTER(BsgTables3), C.c_char_p, C.c_size_t]
        lib.bsg_validate_tables3.restype = C.c_int
        lib.bsg_applyh_noalloc.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int]
        lib.bsg_applyh_noalloc.restype = C.c_int
        lib.bsg_batch_create.argtypes = [C.c_int, C.POINTER(C.POINTER(BsgTables)), C.POINTER(BsgConfig), C.POINTER(vp)]
        lib.bsg_batch_create.restype = C.c_int
        lib.bsg_batch_destroy.argtypes = [vp]
        lib.bsg_batch_destroy.restype = C.c_int
        lib.bsg_batch_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        lib.bsg_batch_last_error.restype = C.c_int
        lib.bsg_batch_dims.argtypes = [vp, i64p]
        lib.bsg_batch_dims.restype = C.c_int
        lib.bsg_batch_system.argtypes = [vp, C.c_int, C.POINTER(vp)]
        lib.bsg_batch_system.restype = C.c_int
        lib.bsg_batch_applyh.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.c_int, vp]
        lib.bsg_batch_applyh.restype = C.c_int
        lib.bsg_batch_autotune.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        lib.bsg_batch_autotune.restype = C.c_int
        lib.bsg_batch_set_tuning.argtypes = [vp, C.c_int, C.c_int]
        lib.bsg_batch_set_tuning.restype = C.c_int
        lib.bsg_batch_lanczos.argtypes = [vp, C.POINTER(BsgLanczosParams), f64p, C.POINTER(f64p), C.POINTER(BsgReport)]
        lib.bsg_batch_lanczos.restype = C.c_int
        lib.bsg_batch_grad.argtypes = [vp, C.POINTER(f64p), C.c_int, C.POINTER(f64p), C.POINTER(f64p),
                                       C.POINTER(f64p), C.POINTER(f64p), C.POINTER(f64p), C.POINTER(C.c_double)]
        lib.bsg_batch_grad.restype = C.c_int
        lib.bsg_jumpgen_create.argtypes = [C.c_int, C.POINTER(BsgSpecies), C.POINTER(vp)]
        lib.bsg_jumpgen_create.restype = C.c_int
        lib.bsg_jumpgen_destroy.argtypes = [vp]
        lib.bsg_jumpgen_destroy.restype = C.c_int
        lib.bsg_jumpgen_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        lib.bsg_jumpgen_last_error.restype = C.c_int
        lib.bsg_jumpgen_one.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_double)]
        lib.bsg_jumpgen_one.restype = C.c_int
        lib.bsg_jumpgen_two.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_double)]
        lib.bsg_jumpgen_two.restype = C.c_int
        lib.bsg_jumpgen_sort1.argtypes = [vp, C.c_int, vp, vp, C.c_int, C.c_int64, vp, vp, vp, vp, vp,
                                          C.POINTER(C.c_double)]
        lib.bsg_jumpgen_sort1.restype = C.c_int
        _gpu = lib
    return _gpu
