"""Python host binding of libopenqcd_b200.so (ctypes).

Mirrors the C interface in include/openqcd_b200.h: the reference-named
drop-in calls (Dw_dble, Dw, Dwee_dble, ..., apply_sw_dble, sap, sap_gcr) take
numpy arrays in the reference's storage order; the b200_dev_* calls take
device pointers (ints) to fields in the library's own layout.

The library must have been built (build.py); importing this module on a
machine without it raises, there is no fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("B200_LIB", os.path.join(HERE, "libopenqcd_b200.so"))

_lib = None

# transport callbacks of the domain decomposition (b200_dd_setup)
DD_EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                             C.c_void_p)
DD_ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_void_p)


class Qflt(C.Structure):
    _fields_ = [("q", C.c_double * 2)]


class ComplexQflt(C.Structure):
    _fields_ = [("re", Qflt), ("im", Qflt)]


class ComplexF(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class ComplexD(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


DOP_T = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)
MOP_T = C.CFUNCTYPE(None, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)

DIRAC_OPS = {"Dw": 0, "Dwee": 1, "Dwoo": 2, "Dwoe": 3, "Dweo": 4, "Dwhat": 5}

_SIGS = {
    "b200_set_device": (C.c_int, [C.c_int]),
    "b200_geometry": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_set_lat_parms": (C.c_int, [C.c_double]),
    "b200_set_sw_type": (C.c_int, [C.c_int]),
    "b200_set_bc_parms": (C.c_int, [C.c_int]),
    "b200_set_bc_theta": (C.c_int, [C.c_void_p]),
    "b200_links12_active": (C.c_int, []),
    "b200_set_sw_parms": (C.c_int, [C.c_double]),
    "b200_set_tm_parms": (C.c_int, [C.c_int]),
    "b200_set_sap_parms": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "b200_upload_ud": (C.c_int, [C.c_void_p]),
    "b200_download_ud": (C.c_int, [C.c_void_p]),
    "b200_upload_swd": (C.c_int, [C.c_void_p]),
    "b200_download_swd": (C.c_int, [C.c_void_p, C.c_int]),
    "b200_sw_term": (C.c_int, []),
    "b200_random_ud": (C.c_int, [C.c_double, C.c_ulonglong]),
    "b200_host_alloc": (C.c_void_p, [C.c_size_t]),
    "b200_host_free": (None, [C.c_void_p]),
    "b200_dev_alloc": (C.c_void_p, [C.c_size_t]),
    "b200_memcpy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "b200_last_error": (C.c_char_p, []),
    "b200_set_fatal": (None, [C.c_int]),
    "b200_sync": (C.c_int, []),
    "b200_volume": (C.c_int, []),
    "Dw_dble": (None, [C.c_double, C.c_void_p, C.c_void_p]),
    "Dwee_dble": (None, [C.c_double, C.c_void_p, C.c_void_p]),
    "Dwoo_dble": (None, [C.c_double, C.c_void_p, C.c_void_p]),
    "Dwoe_dble": (None, [C.c_void_p, C.c_void_p]),
    "Dweo_dble": (None, [C.c_void_p, C.c_void_p]),
    "Dwhat_dble": (None, [C.c_double, C.c_void_p, C.c_void_p]),
    "Dw": (None, [C.c_float, C.c_void_p, C.c_void_p]),
    "Dwee": (None, [C.c_float, C.c_void_p, C.c_void_p]),
    "Dwoo": (None, [C.c_float, C.c_void_p, C.c_void_p]),
    "Dwoe": (None, [C.c_void_p, C.c_void_p]),
    "Dweo": (None, [C.c_void_p, C.c_void_p]),
    "Dwhat": (None, [C.c_float, C.c_void_p, C.c_void_p]),
    "apply_sw_dble": (None, [C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    "apply_sw": (None, [C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    "apply_swinv_dble": (C.c_int, [C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sap": (None, [C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "sap_gcr": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_void_p]),
    "b200_set_nthread": (C.c_int, [C.c_int]),
    "spinor_prod_dble": (ComplexQflt, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "spinor_prod_re_dble": (Qflt, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "norm_square_dble": (Qflt, [C.c_int, C.c_int, C.c_void_p]),
    "mulc_spinor_add_dble": (None, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, ComplexD]),
    "mulr_spinor_add_dble": (None, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double]),
    "scale_dble": (None, [C.c_int, C.c_int, C.c_double, C.c_void_p]),
    "normalize_dble": (C.c_double, [C.c_int, C.c_int, C.c_void_p]),
    "spinor_prod": (ComplexF, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "spinor_prod_re": (C.c_float, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "norm_square": (C.c_float, [C.c_int, C.c_int, C.c_void_p]),
    "mulc_spinor_add": (None, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, ComplexF]),
    "mulr_spinor_add": (None, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_float]),
    "scale": (None, [C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "normalize": (C.c_float, [C.c_int, C.c_int, C.c_void_p]),
    "fgcr": (C.c_double, [C.c_int, DOP_T, MOP_T, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                          C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_clear_error": (None, []),
    "b200_set_sap_prec": (C.c_int, [C.c_int]),
    "b200_set_sap_link12": (C.c_int, [C.c_int]),
    "b200_set_dw_staged": (C.c_int, [C.c_int]),
    "Aweeinv_dble": (None, [C.c_void_p, C.c_void_p]),
    "Awooinv_dble": (None, [C.c_void_p, C.c_void_p]),
    "Awoe_dble": (None, [C.c_void_p, C.c_void_p]),
    "Aweo_dble": (None, [C.c_void_p, C.c_void_p]),
    "Aw": (None, [C.c_void_p, C.c_void_p]),
    "Awhat": (None, [C.c_void_p, C.c_void_p]),
    "Aweeinv": (None, [C.c_void_p, C.c_void_p]),
    "Awooinv": (None, [C.c_void_p, C.c_void_p]),
    "Awoe": (None, [C.c_void_p, C.c_void_p]),
    "Aweo": (None, [C.c_void_p, C.c_void_p]),
    "set_ltl_modes": (C.c_int, []),
    "ltl_matrix": (C.c_void_p, []),
    "dfl_Lvd": (None, [C.c_void_p]),
    "dfl_LRvd": (None, [C.c_void_p, C.c_void_p]),
    "dfl_RLvd": (None, [C.c_void_p, C.c_void_p]),
    "dfl_Lv": (None, [C.c_void_p]),
    "b200_set_ltl_solver": (C.c_int, [C.c_int]),
    "b200_rhs_tiles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_set_rhs_tiles": (C.c_int, [C.c_void_p, C.c_void_p]),
    "b200_dfl_set_lmode": (C.c_int, [C.c_int, C.c_void_p]),
    "b200_set_cuda_graphs": (C.c_int, [C.c_int]),
    "b200_set_pipeline": (C.c_int, [C.c_int]),
    "b200_pipeline_slabs": (C.c_int, []),
    "b200_pipeline_pieces": (C.c_int, []),
    "b200_pipeline_used": (C.c_int, []),
    "b200_pipeline_plan": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_graphs_cached": (C.c_int, []),
    "tmcg": (C.c_double, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                          C.c_void_p]),
    "tmcgeo": (C.c_double, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p]),
    "b200_dev_tmcg": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "tmcgm": (None, [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                     C.c_void_p]),
    "b200_dev_tmcgm": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "export_cnfg": (None, [C.c_char_p]),
    "import_cnfg": (None, [C.c_char_p, C.c_int]),
    "export_sfld": (None, [C.c_char_p, C.c_int, C.c_void_p]),
    "import_sfld": (None, [C.c_char_p, C.c_int, C.c_void_p]),
    "b200_plaq_sum": (C.c_double, []),
    "b200_dev_dirac_multi": (C.c_int, [C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_profiler": (C.c_int, [C.c_int]),
    "b200_sap_tuning": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_set_dfl_parms": (C.c_int, [C.c_void_p, C.c_int]),
    "b200_set_dfl_pro_parms": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double]),
    "b200_set_dfl_gen_parms": (C.c_int, [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
    "b200_dfl_nv": (C.c_int, []),
    "b200_dfl_profile": (C.c_int, [C.c_int, C.c_void_p]),
    "b200_dev_gcr_batch": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_release_workspace": (C.c_int, []),
    "b200_dev_point_source": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "b200_net_nweights": (C.c_int, []),
    "b200_net_init": (C.c_int, [C.c_ulonglong, C.c_float]),
    "b200_net_set_weights": (C.c_int, [C.c_void_p]),
    "b200_net_get_weights": (C.c_int, [C.c_void_p]),
    "b200_net_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "b200_net_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_net_batch_grad": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_net_adam_step": (C.c_int, [C.c_void_p, C.c_float]),
    "b200_net_train": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_ulonglong,
                                 C.c_void_p]),
    "b200_net_make_pairs": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_ulonglong]),
    "b200_set_precond": (C.c_int, [C.c_int]),
    "b200_dfl_time": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "b200_dfl_s2vd_multi": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "b200_Awhat_dble_multi": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "b200_dfl_vd2s_multi": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "b200_dfl_set_basis": (C.c_int, [C.c_int, C.c_void_p]),
    "b200_dfl_get_basis": (C.c_int, [C.c_int, C.c_void_p]),
    "dfl_modes": (None, [C.c_void_p, C.c_void_p]),
    "b200_dev_dfl_modes": (C.c_int, [C.c_ulonglong, C.c_void_p, C.c_void_p]),
    "dfl_subspace": (None, [C.c_void_p]),
    "dfl_s2vd": (None, [C.c_void_p, C.c_void_p]),
    "dfl_vd2s": (None, [C.c_void_p, C.c_void_p]),
    "set_Aw": (None, [C.c_double]),
    "set_Awhat": (C.c_int, [C.c_double]),
    "Aw_dble": (None, [C.c_void_p, C.c_void_p]),
    "Awhat_dble": (None, [C.c_void_p, C.c_void_p]),
    "ltl_gcr": (C.c_double, [C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dfl_sap_gcr": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "dfl_sap_gcr2": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    "b200_dev_dfl_sap_gcr": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_dev_alloc_spinor": (C.c_void_p, [C.c_int]),
    "b200_dev_free": (None, [C.c_void_p]),
    "b200_dev_random_spinor": (C.c_int, [C.c_int, C.c_void_p, C.c_double, C.c_ulonglong]),
    "b200_dev_from_ref": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "b200_dev_to_ref": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "b200_dev_dirac": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "b200_dev_sap": (C.c_int, [C.c_float, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "b200_dev_sap_gcr": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
    "b200_dev_norm2": (C.c_double, [C.c_int, C.c_void_p]),
    "b200_dev_Dwhat_dble_noalloc": (C.c_int, [C.c_double, C.c_void_p, C.c_void_p]),
    "b200_dev_time_dirac": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "b200_dev_time_sap": (C.c_int, [C.c_float, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_void_p]),
    "b200_set_block_order": (C.c_int, [C.c_int]),
    "b200_tune_block_order": (C.c_int, [C.c_void_p]),
    "b200_dd_setup": (C.c_int, [C.c_int, C.c_int, DD_EXCHANGE_FN, DD_ALLGATHER_FN, C.c_void_p]),
    "b200_dd_info": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "b200_dd_global_sum": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "b200_set_sap_variant": (C.c_int, [C.c_int]),
    "b200_net_make_sap_pairs": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                          C.c_ulonglong]),
    "b200_dfl_set_start_fields": (C.c_int, [C.c_void_p]),
    "b200_tune_block_shape": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p]),
    "b200_selfcheck_bounded_wait": (C.c_int, [C.c_int]),
    "b200_time_Dw_dble_host": (C.c_int, [C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
}

EXPORTED = list(_SIGS)


def lib():
    """Load the shared library (once) and declare the prototypes."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libopenqcd_b200.so is not built (run openqcd-2.4.2_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L.b200_set_fatal(0)
        _lib = L
    return _lib


class B200Error(RuntimeError):
    pass


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if isinstance(a, np.ndarray) else a


def check(rc):
    if rc is not None and rc < 0:
        raise B200Error(lib().b200_last_error().decode())
    return rc


def set_device(dev):
    return check(lib().b200_set_device(dev))


def even_first_ipt(L):
    """An ipt[] table in the reference's convention (ipt[lexicographic index]
    = storage index, even sites first), ordering each parity
    lexicographically."""
    L = tuple(L)
    x = np.indices(L).reshape(4, -1)
    par = x.sum(axis=0) & 1
    order = np.argsort(par, kind="stable")
    ipt = np.empty(order.size, dtype=np.int32)
    ipt[order] = np.arange(order.size, dtype=np.int32)
    return ipt


def geometry(L, bs, ipt=None):
    Lc = np.ascontiguousarray(L, dtype=np.int32)
    bc = np.ascontiguousarray(bs, dtype=np.int32)
    ip = None if ipt is None else np.ascontiguousarray(ipt, dtype=np.int32)
    return check(lib().b200_geometry(_ptr(Lc), _ptr(bc), None if ip is None else _ptr(ip)))


def set_parms(csw, m0, eoflg=0, bc=3, isw=0):
    L = lib()
    check(L.b200_set_lat_parms(csw))
    check(L.b200_set_sw_type(isw))
    check(L.b200_set_bc_parms(bc))
    check(L.b200_set_sw_parms(m0))
    check(L.b200_set_tm_parms(eoflg))


def set_bc_theta(theta):
    """spatial phase angles of set_bc_parms (applied to fields made on the
    device or read from files)"""
    t = np.ascontiguousarray(theta, dtype=np.float64)
    return check(lib().b200_set_bc_theta(_ptr(t)))


def set_sap_parms(bs, isolv, nmr, ncy):
    b = np.ascontiguousarray(bs, dtype=np.int32)
    return check(lib().b200_set_sap_parms(_ptr(b), isolv, nmr, ncy))


def set_sap_prec(bits):
    return check(lib().b200_set_sap_prec(bits))


def set_sap_link12(on):
    return check(lib().b200_set_sap_link12(1 if on else 0))


def links12_active():
    """True when the FP32 operators read 12-real links for the current field"""
    return check(lib().b200_links12_active()) == 1


def set_cuda_graphs(on):
    """SAP preconditioner as CUDA graphs (default on); returns the previous
    setting"""
    return lib().b200_set_cuda_graphs(1 if on else 0)


def set_pipeline(on):
    """pipelined host transfers of Dw / Dw_dble (default on); returns the
    previous setting"""
    return lib().b200_set_pipeline(1 if on else 0)


def pipeline_slabs():
    """block rows of the host pipeline (0: no pipeline)"""
    return lib().b200_pipeline_slabs()


def pipeline_pieces():
    """transfer pieces of the host pipeline (0: no pipeline)"""
    return lib().b200_pipeline_pieces()


def pipeline_plan(L, bs, ipt):
    """(pieces, block rows) of the host pipeline for lattice L, blocks bs and
    storage order ipt (host code; no device needed)"""
    Lc = np.ascontiguousarray(L, dtype=np.int32)
    bc = np.ascontiguousarray(bs, dtype=np.int32)
    ip = np.ascontiguousarray(ipt, dtype=np.int32)
    npc, nsl = C.c_int(0), C.c_int(0)
    check(lib().b200_pipeline_plan(_ptr(Lc), _ptr(bc), _ptr(ip), C.byref(npc), C.byref(nsl)))
    return npc.value, nsl.value


def pipeline_used():
    """1 if the last host Dw / Dw_dble call ran the pipeline, 0 if it copied
    the fields whole"""
    return lib().b200_pipeline_used()


def graphs_cached():
    return lib().b200_graphs_cached()


def set_dw_staged(mode):
    """FP64 operators: 1 SW matrices staged in shared memory (default), 0
    read directly; returns the previous mode"""
    return lib().b200_set_dw_staged(int(mode))


def set_block_order(kind):
    """traversal order of the blocks in the full-lattice kernels; returns the
    previous kind"""
    return check(lib().b200_set_block_order(int(kind)))


def tune_block_order():
    """time Dw_dble under every block order, keep the fastest; returns
    (kind, [ms per launch for each kind])"""
    ms = np.zeros(5, dtype=np.float32)
    k = check(lib().b200_tune_block_order(_ptr(ms)))
    return k, [float(x) for x in ms]


def sap_tuning(prec):
    v, t, ms = C.c_int(0), C.c_int(0), C.c_float(0.0)
    check(lib().b200_sap_tuning(prec, C.byref(v), C.byref(t), C.byref(ms)))
    return v.value, t.value, ms.value


def upload_ud(ud):
    return check(lib().b200_upload_ud(_ptr(np.ascontiguousarray(ud, dtype=np.float64))))


def download_ud(vol):
    out = np.zeros(4 * vol * 18)
    check(lib().b200_download_ud(_ptr(out)))
    return out


def upload_swd(swd):
    return check(lib().b200_upload_swd(_ptr(np.ascontiguousarray(swd, dtype=np.float64))))


def download_swd(vol, which=0):
    out = np.zeros(2 * vol * 36)
    check(lib().b200_download_swd(_ptr(out), which))
    return out


def sw_term():
    return check(lib().b200_sw_term())


def random_ud(eps, seed):
    return check(lib().b200_random_ud(eps, seed))


def _err_after():
    e = lib().b200_last_error()
    return e.decode() if e else ""


def _void(f, *args):
    """Call a void entry point and raise if it recorded an error."""
    lib().b200_clear_error()
    f(*args)
    e = _err_after()
    if e:
        raise B200Error(e)


def dirac_ref(op, prec, mu, s, r=None):
    """Apply a reference-named operator to reference-layout numpy arrays."""
    L = lib()
    dt = np.float64 if prec == 64 else np.float32
    s = np.ascontiguousarray(s, dtype=dt)
    r = np.zeros_like(s) if r is None else np.array(r, dtype=dt, copy=True)
    name = op + ("_dble" if prec == 64 else "")
    f = getattr(L, name)
    before = _err_after()
    if op in ("Dwoe", "Dweo"):
        f(_ptr(s), _ptr(r))
    else:
        f(mu, _ptr(s), _ptr(r))
    after = _err_after()
    if after and after != before:
        raise B200Error(after)
    return r


class DevField:
    """A spinor field resident on the device in the library's layout."""

    def __init__(self, prec):
        self.prec = prec
        self.ptr = lib().b200_dev_alloc_spinor(prec)
        if not self.ptr:
            raise B200Error(_err_after())

    def free(self):
        if self.ptr:
            lib().b200_dev_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def from_ref(self, q):
        dt = np.float64 if self.prec == 64 else np.float32
        q = np.ascontiguousarray(q, dtype=dt)
        check(lib().b200_dev_from_ref(self.prec, _ptr(q), self.ptr))
        return self

    def to_ref(self, vol):
        dt = np.float64 if self.prec == 64 else np.float32
        out = np.zeros(vol * 24, dtype=dt)
        check(lib().b200_dev_to_ref(self.prec, self.ptr, _ptr(out)))
        return out

    def random(self, sigma, seed):
        check(lib().b200_dev_random_spinor(self.prec, self.ptr, sigma, seed))
        return self

    def point(self, x, spin, colour):
        xs = np.ascontiguousarray(x, dtype=np.int32)
        check(lib().b200_dev_point_source(self.prec, self.ptr, _ptr(xs), spin, colour))
        return self

    def norm2(self):
        return lib().b200_dev_norm2(self.prec, self.ptr)


def dev_dirac_multi(mu, ss, rs, subs=None):
    n = len(ss)
    sp = (C.c_void_p * n)(*[x.ptr for x in ss])
    rp = (C.c_void_p * n)(*[x.ptr for x in rs])
    up = (C.c_void_p * n)(*[x.ptr for x in subs]) if subs else None
    return check(lib().b200_dev_dirac_multi(n, mu, sp, rp, up))


def dev_dirac(op, mu, s, r):
    return check(lib().b200_dev_dirac(s.prec, DIRAC_OPS[op], mu, s.ptr, r.ptr))


def dev_sap(mu, isolv, nmr, ncy, psi, rho):
    return check(lib().b200_dev_sap(mu, isolv, nmr, ncy, psi.ptr, rho.ptr))


def dev_sap_gcr(nkv, nmx, istop, res, mu, eta, psi):
    ifail = C.c_int(0)
    status = C.c_int(0)
    rho = lib().b200_dev_sap_gcr(nkv, nmx, istop, res, mu, eta.ptr, psi.ptr, C.byref(ifail), C.byref(status))
    if rho < 0:
        raise B200Error(_err_after())
    return rho, ifail.value, status.value


def dev_dfl_sap_gcr(nkv, nmx, istop, res, mu, eta, psi):
    ifail = C.c_int(0)
    status = (C.c_int * 3)()
    lib().b200_clear_error()
    rho = lib().b200_dev_dfl_sap_gcr(nkv, nmx, istop, res, mu, eta.ptr, psi.ptr, C.byref(ifail), status)
    if rho < 0:
        raise B200Error(_err_after())
    return rho, ifail.value, list(status)


def dev_gcr_batch(nkv, nmx, istop, res, mus, etas, psis, dfl=False):
    """Solve len(etas) systems together (device fields); returns per-system
    (rho, ifail, status[, little steps])."""
    n = len(etas)
    mu = (C.c_double * n)(*mus)
    ep = (C.c_void_p * n)(*[e.ptr for e in etas])
    pp = (C.c_void_p * n)(*[p.ptr for p in psis])
    rho = (C.c_double * n)()
    ifail = (C.c_int * n)()
    status = (C.c_int * (2 * n))()
    check(lib().b200_dev_gcr_batch(n, 1 if dfl else 0, nkv, nmx, istop, res, mu, ep, pp, rho, ifail, status))
    return list(rho), list(ifail), list(status[:n]), list(status[n:])


def release_workspace():
    return check(lib().b200_release_workspace())


def sap_gcr(nkv, nmx, istop, res, mu, eta):
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = np.zeros_like(eta)
    ifail = C.c_int(0)
    status = C.c_int(0)
    rho = lib().sap_gcr(nkv, nmx, istop, res, mu, _ptr(eta), _ptr(psi), C.byref(ifail), C.byref(status))
    if rho < 0:
        raise B200Error(_err_after())
    return psi, rho, ifail.value, status.value


def tmcgm(nmx, istop, res, mu, eta, psi0=None):
    """tmcgm on reference-layout arrays: res and mu are sequences of equal
    length; returns (list of solutions, ifail, status).  Only the even sites
    of the solutions are computed; their odd sites are those of psi0."""
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    res = np.ascontiguousarray(res, dtype=np.float64)
    nmu = len(mu)
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = [np.zeros_like(eta) if psi0 is None else np.array(psi0[k], dtype=np.float64, copy=True)
           for k in range(nmu)]
    ptrs = (C.c_void_p * max(nmu, 1))(*[_ptr(p) for p in psi])
    ifail = C.c_int(0)
    status = C.c_int(0)
    lib().b200_clear_error()
    lib().tmcgm(nmx, istop, _ptr(res), nmu, _ptr(mu), _ptr(eta), ptrs, C.byref(ifail), C.byref(status))
    err = _err_after()
    if err:
        raise B200Error(err)
    return psi, ifail.value, status.value


def sap_ref(mu, isolv, nmr, psi, rho):
    psi = np.array(psi, dtype=np.float32, copy=True)
    rho = np.array(rho, dtype=np.float32, copy=True)
    before = _err_after()
    lib().sap(mu, isolv, nmr, _ptr(psi), _ptr(rho))
    after = _err_after()
    if after and after != before:
        raise B200Error(after)
    return psi, rho


def apply_sw_dble(vol, mu, m, s):
    s = np.ascontiguousarray(s, dtype=np.float64)
    r = np.zeros_like(s)
    lib().apply_sw_dble(vol, mu, _ptr(np.ascontiguousarray(m, dtype=np.float64)), _ptr(s), _ptr(r))
    return r


def apply_sw(vol, mu, m, s):
    s = np.ascontiguousarray(s, dtype=np.float32)
    r = np.zeros_like(s)
    lib().apply_sw(vol, mu, _ptr(np.ascontiguousarray(m, dtype=np.float32)), _ptr(s), _ptr(r))
    return r


def apply_swinv_dble(vol, mu, m, s):
    s = np.ascontiguousarray(s, dtype=np.float64)
    r = np.zeros_like(s)
    f = lib().apply_swinv_dble(vol, mu, _ptr(np.ascontiguousarray(m, dtype=np.float64)), _ptr(s), None, _ptr(r))
    return r, f


class HostArray:
    """Page-locked host buffer exposed as a numpy array."""

    def __init__(self, n, dtype=np.float64):
        dt = np.dtype(dtype)
        self.ptr = lib().b200_host_alloc(n * dt.itemsize)
        if not self.ptr:
            raise B200Error(_err_after())
        buf = (C.c_char * (n * dt.itemsize)).from_address(self.ptr)
        self.a = np.frombuffer(buf, dtype=dt, count=n)

    def free(self):
        if self.ptr:
            self.a = None
            lib().b200_host_free(self.ptr)
            self.ptr = None


def time_dirac(prec, op, mu, s, r, n):
    ms = C.c_float(0.0)
    check(lib().b200_dev_time_dirac(prec, DIRAC_OPS[op], mu, s.ptr, r.ptr, n, C.byref(ms)))
    return ms.value


def time_sap(mu, isolv, nmr, ncy, psi, rho, n):
    ms = C.c_float(0.0)
    check(lib().b200_dev_time_sap(mu, isolv, nmr, ncy, psi.ptr, rho.ptr, n, C.byref(ms)))
    return ms.value


def time_Dw_dble_host(mu, s, r, n):
    ms = C.c_float(0.0)
    check(lib().b200_time_Dw_dble_host(mu, _ptr(s), _ptr(r), n, C.byref(ms)))
    return ms.value


# ------------------------------------------------------------------ deflation
def set_dfl_parms(bs, Ns):
    b = np.ascontiguousarray(bs, dtype=np.int32)
    check(lib().b200_set_dfl_parms(_ptr(b), Ns))
    return lib().b200_dfl_nv()


def set_dfl_pro_parms(nkv, nmx, res, nmx_gcr, res_gcr):
    return check(lib().b200_set_dfl_pro_parms(nkv, nmx, res, nmx_gcr, res_gcr))


def set_dfl_gen_parms(kappa, mu, ninv, nmr, ncy):
    return check(lib().b200_set_dfl_gen_parms(kappa, mu, ninv, nmr, ncy))


DFL_PHASES = ["sap_smoothing", "gram_schmidt", "little_setup", "little_solve", "sap", "other"]


def dfl_profile(on):
    """Switch the deflation phase timers on or off; returns the sums so far."""
    out = np.zeros(6)
    check(lib().b200_dfl_profile(1 if on else 0, _ptr(out)))
    return dict(zip(DFL_PHASES, out.tolist()))


def dfl_time(what, n):
    """Device ms per call of a deflation kernel (0 restrict, 1 prolong,
    2 Awhat_dble, 3 Aw_dble, 4 ltl_gcr) and the last solve's GCR steps."""
    ms, its = C.c_float(0.0), C.c_int(0)
    check(lib().b200_dfl_time(what, n, C.byref(ms), C.byref(its)))
    return ms.value / n, its.value


def dfl_set_basis(l, field):
    return check(lib().b200_dfl_set_basis(l, _ptr(np.ascontiguousarray(field, dtype=np.float32))))


def dfl_get_basis(l, vol):
    out = np.zeros(vol * 24, dtype=np.float32)
    check(lib().b200_dfl_get_basis(l, _ptr(out)))
    return out


def dfl_modes(seed=1):
    ifail = C.c_int(0)
    status = (C.c_int * 2)()
    check(lib().b200_dev_dfl_modes(seed, C.byref(ifail), status))
    return ifail.value, list(status)


def dfl_set_start_fields(fields):
    """start fields of the next dfl_modes (Ns FP32 reference-layout fields)"""
    f = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float32).reshape(-1) for x in fields]))
    return check(lib().b200_dfl_set_start_fields(_ptr(f)))


def dfl_subspace(modes):
    arrs = [np.ascontiguousarray(m, dtype=np.float32) for m in modes]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    _void(lib().dfl_subspace, ptrs)


def dfl_s2vd(s, nv):
    s = np.ascontiguousarray(s, dtype=np.float32)
    vd = np.zeros(2 * nv)
    _void(lib().dfl_s2vd, _ptr(s), _ptr(vd))
    return vd


def dfl_s2vd_multi(fields, nv):
    """batched dfl_s2vd of several FP32 fields (reference layout)"""
    fs = [np.ascontiguousarray(f, dtype=np.float32) for f in fields]
    vds = [np.zeros(2 * nv) for _ in fs]
    pf = (C.c_void_p * len(fs))(*[f.ctypes.data for f in fs])
    pv = (C.c_void_p * len(fs))(*[v.ctypes.data for v in vds])
    check(lib().b200_dfl_s2vd_multi(len(fs), pf, pv))
    return vds


def Awhat_multi(vs, ws=None):
    """batched Awhat_dble of several little vectors (set_Awhat done before)"""
    vs = [np.ascontiguousarray(v, dtype=np.float64) for v in vs]
    ws = [np.zeros_like(v) for v in vs] if ws is None else [np.array(w, dtype=np.float64, copy=True) for w in ws]
    pv = (C.c_void_p * len(vs))(*[v.ctypes.data for v in vs])
    pw = (C.c_void_p * len(ws))(*[w.ctypes.data for w in ws])
    check(lib().b200_Awhat_dble_multi(len(vs), pv, pw))
    return ws


def dfl_vd2s_multi(vds, vol):
    """batched dfl_vd2s of several little vectors"""
    vs = [np.ascontiguousarray(v, dtype=np.float64) for v in vds]
    fs = [np.zeros(vol * 24, dtype=np.float32) for _ in vs]
    pv = (C.c_void_p * len(vs))(*[v.ctypes.data for v in vs])
    pf = (C.c_void_p * len(vs))(*[f.ctypes.data for f in fs])
    check(lib().b200_dfl_vd2s_multi(len(vs), pv, pf))
    return fs


def dfl_vd2s(vd, vol):
    vd = np.ascontiguousarray(vd, dtype=np.float64)
    s = np.zeros(vol * 24, dtype=np.float32)
    _void(lib().dfl_vd2s, _ptr(vd), _ptr(s))
    return s


def little(which, mu, v, w=None):
    """which 0: set_Aw(mu), Aw_dble(v, w); 1: set_Awhat(mu), Awhat_dble."""
    v = np.ascontiguousarray(v, dtype=np.float64)
    w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float64, copy=True)
    f = 0
    if which == 0:
        _void(lib().set_Aw, mu)
        _void(lib().Aw_dble, _ptr(v), _ptr(w))
    else:
        f = check(lib().set_Awhat(mu))
        _void(lib().Awhat_dble, _ptr(v), _ptr(w))
    return w, f


LITTLE_EO = {"Aweeinv_dble": 2, "Awooinv_dble": 3, "Awoe_dble": 4, "Aweo_dble": 5}


def little_eo(name, mu, v, w=None):
    """set_Awhat(mu), then one of Aweeinv_dble, Awooinv_dble, Awoe_dble,
    Aweo_dble (little vectors of nv complex doubles)."""
    v = np.ascontiguousarray(v, dtype=np.float64)
    w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float64, copy=True)
    f = check(lib().set_Awhat(mu))
    _void(getattr(lib(), name), _ptr(v), _ptr(w))
    return w, f


LITTLE32 = ["Aw", "Awhat", "Aweeinv", "Awooinv", "Awoe", "Aweo"]


def little32(which, mu, v, w=None):
    """FP32 little operators: 0 set_Aw(mu), Aw; 1..5 set_Awhat(mu), then
    Awhat, Aweeinv, Awooinv, Awoe, Aweo (little vectors of nv complex floats
    as float32 arrays)."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float32, copy=True)
    if which == 0:
        _void(lib().set_Aw, mu)
    else:
        check(lib().set_Awhat(mu))
    _void(getattr(lib(), LITTLE32[which]), _ptr(v), _ptr(w))
    return w


def set_ltl_modes():
    return check(lib().set_ltl_modes())


def ltl_matrix(ns):
    p = lib().ltl_matrix()
    if not p:
        raise B200Error(_err_after() or "little modes are not set")
    return np.ctypeslib.as_array((C.c_double * (2 * ns * ns)).from_address(p)).copy()


def dfl_proj(which, v, w=None):
    """0 dfl_Lvd(v), 1 dfl_LRvd(v, w), 2 dfl_RLvd(v, w); returns (v, w)"""
    v = np.array(v, dtype=np.float64, copy=True)
    w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float64, copy=True)
    if which == 0:
        _void(lib().dfl_Lvd, _ptr(v))
    elif which == 1:
        _void(lib().dfl_LRvd, _ptr(v), _ptr(w))
    else:
        _void(lib().dfl_RLvd, _ptr(v), _ptr(w))
    return v, w


def dfl_Lv(v):
    v = np.array(v, dtype=np.float32, copy=True)
    _void(lib().dfl_Lv, _ptr(v))
    return v


def rhs_tiles():
    """autotuned fields per pass of the batched restriction and prolongation
    (0: not tuned yet), whether the four-field pass runs on the tensor cores,
    and the times of four fields with 1, 2, 4 fields per pass on the CUDA
    cores and 4 on the tensor cores"""
    t = np.zeros(2, dtype=np.int32)
    tc = np.zeros(2, dtype=np.int32)
    ms = np.zeros(8, dtype=np.float32)
    check(lib().b200_rhs_tiles(_ptr(t), _ptr(tc), _ptr(ms)))
    return {"restrict": int(t[0]), "prolong": int(t[1]), "restrict_tc": bool(tc[0]), "prolong_tc": bool(tc[1]),
            "restrict_ms": ms[:4].tolist(), "prolong_ms": ms[4:].tolist()}


def set_rhs_tiles(restrict, prolong, restrict_tc=True, prolong_tc=True):
    """fix the fields per pass of the batched restriction and prolongation
    (1, 2 or 4; 0 hands the choice back to the autotuner) and whether four
    fields run on the tensor cores"""
    t = np.array([restrict, prolong], dtype=np.int32)
    tc = np.array([int(restrict_tc), int(prolong_tc)], dtype=np.int32)
    check(lib().b200_set_rhs_tiles(_ptr(t), _ptr(tc)))


def set_ltl_solver(kind):
    """0 the device GCR, 1 the reference's fgcr4vd + gcr4v with global-mode
    deflation; returns the previous choice"""
    return check(lib().b200_set_ltl_solver(int(kind)))


def dfl_set_lmode(l, v):
    return check(lib().b200_dfl_set_lmode(l, _ptr(np.ascontiguousarray(v, dtype=np.float32))))


def ltl_gcr(mu, eta):
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = np.zeros_like(eta)
    ifail = C.c_int(0)
    status = (C.c_int * 2)()
    lib().b200_clear_error()
    rho = lib().ltl_gcr(mu, _ptr(eta), _ptr(psi), C.byref(ifail), status)
    if rho < 0:
        raise B200Error(_err_after())
    return psi, rho, ifail.value, list(status)


def dfl_sap_gcr(nkv, nmx, istop, res, mu, eta):
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = np.zeros_like(eta)
    ifail = C.c_int(0)
    status = (C.c_int * 3)()
    lib().b200_clear_error()
    rho = lib().dfl_sap_gcr(nkv, nmx, istop, res, mu, _ptr(eta), _ptr(psi), C.byref(ifail), status)
    if rho < 0:
        raise B200Error(_err_after())
    return psi, rho, ifail.value, list(status)


def dfl_sap_gcr2(nkv, nmx, istop, res, mu, eta):
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = np.zeros_like(eta)
    ifail = (C.c_int * 2)()
    status = (C.c_int * 6)()
    lib().b200_clear_error()
    rho = lib().dfl_sap_gcr2(nkv, nmx, istop, res, mu, _ptr(eta), _ptr(psi), ifail, status)
    if rho < 0:
        raise B200Error(_err_after())
    return psi, rho, list(ifail), list(status)


# ------------------------------------------------------ learned preconditioner
def net_nweights():
    return lib().b200_net_nweights()


def net_init(seed=1, scale=0.25):
    return check(lib().b200_net_init(seed, scale))


def net_set_weights(w):
    w = np.ascontiguousarray(w, dtype=np.float32)
    return check(lib().b200_net_set_weights(_ptr(w)))


def net_get_weights():
    w = np.zeros(net_nweights(), dtype=np.float32)
    check(lib().b200_net_get_weights(_ptr(w)))
    return w


def net_apply(inp, out, half=True):
    return check(lib().b200_net_apply(inp.ptr, out.ptr, 1 if half else 0))


def net_grad(r, e):
    loss = C.c_double(0.0)
    g = np.zeros(net_nweights(), dtype=np.float32)
    check(lib().b200_net_grad(r.ptr, e.ptr, C.byref(loss), _ptr(g)))
    return loss.value, g


def net_batch_grad(rs, es):
    """mean loss and mean gradient over the pairs (rs[k], es[k])"""
    n = len(rs)
    rp = (C.c_void_p * n)(*[x.ptr for x in rs])
    ep = (C.c_void_p * n)(*[x.ptr for x in es])
    loss = C.c_double(0.0)
    g = np.zeros(net_nweights(), dtype=np.float32)
    check(lib().b200_net_batch_grad(n, rp, ep, C.byref(loss), _ptr(g)))
    return loss.value, g


def net_adam_step(grad, lr):
    g = np.ascontiguousarray(grad, dtype=np.float32)
    return check(lib().b200_net_adam_step(_ptr(g), lr))


def data_parallel_steps(grad_fn, step_fn, npairs, steps, batch, lr, seed, allreduce, world):
    """The loop of data-parallel training, independent of where the
    gradients come from.  Per step this rank draws `batch` of its own
    npairs pairs (generator seeded with `seed`, which differs between
    ranks), grad_fn(indices) -> (mean loss, mean gradient); the loss and
    gradient are summed over the ranks by allreduce (a float64 vector in,
    the sum out) and divided by `world`, and step_fn(gradient, lr) applies
    the same optimiser step on every rank, so the weights stay identical.
    Returns the per-step mean loss over all ranks."""
    rng = np.random.default_rng(seed)
    hist = []
    for _ in range(steps):
        idx = rng.integers(0, npairs, size=batch)
        loss, g = grad_fn(idx)
        buf = np.concatenate([[loss], np.asarray(g, dtype=np.float64)])
        buf = np.asarray(allreduce(buf), dtype=np.float64) / world
        step_fn(buf[1:].astype(np.float32), lr)
        hist.append(float(buf[0]))
    return hist


def net_train_data_parallel(rs, es, steps, batch, lr, seed=1, group=None):
    """Data-parallel training of the network over the ranks of a
    torch.distributed process group (one process per GPU): every rank holds
    its own training pairs (e.g. from its own gauge field) and draws its
    minibatches with the seed seed + rank; the gradients are all-reduced
    (SUM, then divided by the number of ranks) and every rank applies the
    same Adam step.  Without an initialised process group it is plain
    training on this rank's pairs.  Returns the per-step mean loss."""
    try:
        import torch
        import torch.distributed as dist
        on = dist.is_available() and dist.is_initialized()
    except ImportError:
        on = False
    rank = dist.get_rank(group) if on else 0
    world = dist.get_world_size(group) if on else 1

    def allreduce(v):
        if not on:
            return v
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()

    def grad_fn(idx):
        return net_batch_grad([rs[i] for i in idx], [es[i] for i in idx])

    return data_parallel_steps(grad_fn, net_adam_step, len(rs), steps, batch, lr, seed + rank, allreduce, world)


def net_train(rs, es, steps, batch, lr, seed=1):
    n = len(rs)
    rp = (C.c_void_p * n)(*[x.ptr for x in rs])
    ep = (C.c_void_p * n)(*[x.ptr for x in es])
    hist = np.zeros(max(steps, 1), dtype=np.float32)
    check(lib().b200_net_train(n, rp, ep, steps, batch, lr, seed, _ptr(hist)))
    return hist[:steps]


def net_make_pairs(rs, es, mu, res, seed=1):
    n = len(rs)
    rp = (C.c_void_p * n)(*[x.ptr for x in rs])
    ep = (C.c_void_p * n)(*[x.ptr for x in es])
    return check(lib().b200_net_make_pairs(n, rp, ep, mu, res, seed))


def net_make_sap_pairs(rs, es, mu, res, seed=1):
    """(residual, SAP-error) training pairs: es[k] = Dw^-1 rs[k] - M_sap rs[k]"""
    n = len(rs)
    rp = (C.c_void_p * n)(*[x.ptr for x in rs])
    ep = (C.c_void_p * n)(*[x.ptr for x in es])
    return check(lib().b200_net_make_sap_pairs(n, rp, ep, mu, res, seed))


def set_precond(kind):
    """0 SAP, 1 network, 2 network then SAP, 3 none, 4 SAP plus the network"""
    return check(lib().b200_set_precond(kind))


# ------------------------------------------------------------------- archives
def export_cnfg(path):
    _void(lib().export_cnfg, path.encode())


def import_cnfg(path, mask=0):
    _void(lib().import_cnfg, path.encode(), mask)


def export_sfld(path, eo, sd):
    sd = np.ascontiguousarray(sd, dtype=np.float64)
    _void(lib().export_sfld, path.encode(), eo, _ptr(sd))


def import_sfld(path, eo, sd):
    sd = np.array(sd, dtype=np.float64, copy=True)
    _void(lib().import_sfld, path.encode(), eo, _ptr(sd))
    return sd


def plaq_sum():
    v = lib().b200_plaq_sum()
    if v < -1e299:
        raise B200Error(_err_after())
    return v


# ------------------------------------------------------- CG, normal equations
def tmcg(nmx, istop, res, mu, eta, eo=False, psi0=None):
    """tmcg (eo False) or tmcgeo (eo True) on reference-layout arrays."""
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = np.zeros_like(eta) if psi0 is None else np.array(psi0, dtype=np.float64, copy=True)
    ifail = C.c_int(0)
    status = C.c_int(0)
    f = lib().tmcgeo if eo else lib().tmcg
    lib().b200_clear_error()
    rho = f(nmx, istop, res, mu, _ptr(eta), _ptr(psi), C.byref(ifail), C.byref(status))
    if rho < 0:
        raise B200Error(_err_after())
    return psi, rho, ifail.value, status.value


# ------------------------------------------------------------------------
# Domain decomposition along x0: the transport the library calls back.

class DomainDecomposition:
    """Ranks of a torch.distributed group holding consecutive x0-slabs
    (b200_dd_setup).  transport "host": the exchange synchronises the
    library's stream, copies the two send faces to host memory, moves them
    with point-to-point messages of the group's backend (gloo) and copies
    the received faces back; "nccl": the faces move between the device
    buffers with NCCL (torch's batch_isend_irecv), no host copy.  The
    all-gather of the reduction partials goes through the same group.

    memcpy(dst, src, nbytes) moves bytes between the library's buffers and
    host memory (default: the library's own b200_memcpy); a test on CPU can
    pass a host-only copy.  Call install() before b200_geometry."""

    def __init__(self, group=None, transport="host", memcpy=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.np = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.transport = transport
        self.memcpy = memcpy or (lambda dst, src, n: check(lib().b200_memcpy(dst, src, n)))
        self.sync_stream = memcpy is None      # a host-only copy (CPU test) has no stream to wait for
        self._xfn = DD_EXCHANGE_FN(self._exchange)
        self._gfn = DD_ALLGATHER_FN(self._allgather)
        self.error = None

    def install(self):
        return check(lib().b200_dd_setup(self.np, self.rank, self._xfn, self._gfn, None))

    def _peer(self, d):
        return self.dist.get_global_rank(self.group, (self.rank + d) % self.np) if self.group is not None \
            else (self.rank + d) % self.np

    def _exchange(self, send_dn, send_up, recv_up, recv_dn, nbytes, stream, user):
        try:
            self.exchange(send_dn, send_up, recv_up, recv_dn, nbytes)
            return 0
        except Exception as e:          # reported to the library, which fails the call
            self.error = e
            return -1

    def exchange(self, send_dn, send_up, recv_up, recv_dn, nbytes):
        torch, dist = self.torch, self.dist
        dn, up = self._peer(-1), self._peer(+1)
        if self.transport == "nccl":
            lib().b200_sync()
            t = {k: _device_bytes(torch, p, nbytes) for k, p in
                 (("sd", send_dn), ("su", send_up), ("ru", recv_up), ("rd", recv_dn))}
            ops = [dist.P2POp(dist.isend, t["sd"], dn, self.group), dist.P2POp(dist.irecv, t["ru"], up, self.group),
                   dist.P2POp(dist.isend, t["su"], up, self.group), dist.P2POp(dist.irecv, t["rd"], dn, self.group)]
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            torch.cuda.current_stream().synchronize()
            return
        hs = [torch.empty(nbytes, dtype=torch.uint8) for _ in range(4)]
        if self.sync_stream:
            lib().b200_sync()
        self.memcpy(hs[0].data_ptr(), send_dn, nbytes)
        self.memcpy(hs[1].data_ptr(), send_up, nbytes)
        # tag 1: faces moving down (send_dn -> the lower rank's recv_up);
        # tag 2: faces moving up (send_up -> the upper rank's recv_dn)
        reqs = [dist.isend(hs[0], dn, self.group, tag=1), dist.isend(hs[1], up, self.group, tag=2),
                dist.irecv(hs[2], up, self.group, tag=1), dist.irecv(hs[3], dn, self.group, tag=2)]
        for r in reqs:
            r.wait()
        self.memcpy(recv_up, hs[2].data_ptr(), nbytes)
        self.memcpy(recv_dn, hs[3].data_ptr(), nbytes)

    def _allgather(self, inp, out, n, user):
        try:
            torch, dist = self.torch, self.dist
            x = torch.tensor([inp[k] for k in range(n)], dtype=torch.float64)
            if self.transport == "nccl":
                x = x.cuda()
            parts = [torch.empty_like(x) for _ in range(self.np)]
            dist.all_gather(parts, x, group=self.group)
            k = 0
            for p in parts:
                for v in p.cpu().tolist():
                    out[k] = v
                    k += 1
            return 0
        except Exception as e:
            self.error = e
            return -1


class _CudaBytes:
    """A device byte range torch can wrap without copying."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (int(ptr), False), "version": 3}


def _device_bytes(torch, ptr, n):
    return torch.as_tensor(_CudaBytes(ptr, n), device="cuda")


def dd_info():
    bufs = (C.c_void_p * 4)()
    nb = C.c_size_t(0)
    nx = C.c_longlong(0)
    npr = lib().b200_dd_info(bufs, C.byref(nb), C.byref(nx))
    return npr, [b for b in bufs], nb.value, nx.value


def dd_global_sum(pairs):
    """the library's global double-double sum of (hi, lo) pairs over the ranks"""
    a = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1)
    out = np.zeros_like(a)
    check(lib().b200_dd_global_sum(_ptr(a), _ptr(out), a.size // 2))
    return out


def dd_off():
    """back to one rank (takes effect at the next geometry call)"""
    return check(lib().b200_dd_setup(1, 0, DD_EXCHANGE_FN(0), DD_ALLGATHER_FN(0), None))


def tune_block_shape(candidates, nsteps=8, mu=0.0, Ns=0):
    """the block-shape autotuner: returns (the best shape, the score of every
    candidate: residual reduction ln(|eta|/|r|) per second, -1 if it does
    not fit); Ns > 0 scores the deflated solver with an Ns-mode subspace per
    candidate; the best shape stays in force"""
    c = np.ascontiguousarray(np.asarray(candidates, dtype=np.int32).reshape(-1, 4))
    sc = np.zeros(len(c), dtype=np.float32)
    k = check(lib().b200_tune_block_shape(_ptr(c), len(c), nsteps, mu, Ns, _ptr(sc)))
    return tuple(int(v) for v in c[k]), [float(v) for v in sc]


def set_sap_variant(v):
    return check(lib().b200_set_sap_variant(int(v)))
