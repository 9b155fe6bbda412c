"""ctypes binding of libmolsim_gpu.so (the C-ABI declared in include/molsim_gpu.h)."""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmolsim_gpu.so")
_LIB = None

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)

MSG_OK = 0
MSG_PREC_FP64 = 0
MSG_PREC_MIXED = 1
MSG_TUNE_PAIR_LANES = 1
MSG_TUNE_PAIR_KERNEL = 2
MSG_TUNE_PAIR_UNROLL = 3
MSG_TUNE_OVERLAP = 4
MSG_TUNE_PAIR_BLOCKS = 5
MSG_TUNE_CONV_BLOCKS = 6
STATUS = {0: "ok", 1: "r2 < r2umin", 2: "table interval overrun", 3: "neighbour capacity exceeded",
          4: "CUDA error", 5: "device timeout", 6: "invalid argument", 7: "non-finite force",
          8: "hard-core overlap"}


class MsgParams(C.Structure):
    _fields_ = [("np", C.c_int32), ("npt", C.c_int32), ("boxlen", C.c_double * 3), ("rcut", C.c_double),
                ("drnlist", C.c_double), ("iptpn", i32p), ("az", f64p), ("masspt", f64p), ("ubuf", f64p),
                ("nbuf", C.c_int32), ("iubuflow", i32p), ("r2umin", f64p), ("r2atat", f64p),
                ("lewald", C.c_int32), ("order", C.c_int32), ("nmesh", C.c_int32), ("lsurf", C.c_int32),
                ("ualpha", C.c_double), ("epsi_four_pi", C.c_double), ("nbond", C.c_int32),
                ("bond_ij", i32p), ("bond_k", f64p), ("bond_eq", f64p), ("bond_p", i32p),
                ("tstep", C.c_double), ("bd_fac1", f64p), ("bd_fac2", f64p), ("maxnneigh", C.c_int32),
                ("ncut", C.c_int32), ("ncutregion", C.c_int32), ("lewald2dlc", C.c_int32),
                ("inlist", C.c_int32), ("lvlistllist", C.c_int32)]


class MsgEnergy(C.Structure):
    _fields_ = [("utot", C.c_double), ("utwob0", C.c_double), ("utwob", C.c_double * 10),
                ("urec", C.c_double), ("ubond", C.c_double), ("virial", C.c_double), ("ekin", C.c_double)]

    def as_dict(self, natat=10):
        return dict(utot=self.utot, utwob=[self.utwob0] + list(self.utwob)[:natat], urec=self.urec,
                    ubond=self.ubond, virial=self.virial, ekin=self.ekin)


class MsgMcParams(C.Structure):
    _fields_ = [("beta", C.c_double), ("dtran", f64p), ("isamp", C.c_int32), ("pad", C.c_int32)]


class MsgMcAllParams(C.Structure):
    _fields_ = [("beta", C.c_double), ("dtranall", f64p)]


class MsgSiteEwald(C.Structure):
    _fields_ = [("lewald", C.c_int32), ("order", C.c_int32), ("nmesh", C.c_int32), ("ncut", C.c_int32),
                ("ncutregion", C.c_int32), ("lsurf", C.c_int32), ("ualpha", C.c_double),
                ("epsi_four_pi", C.c_double), ("az", f64p)]


class MsgTabParams(C.Structure):
    _fields_ = [("npt", C.c_int32), ("zat", f64p), ("sigat", f64p), ("epsat", f64p), ("rcut", C.c_double),
                ("ualpha", C.c_double), ("epsi_four_pi", C.c_double), ("lewald", C.c_int32),
                ("lljcut", C.c_int32), ("ljrcut", C.c_double), ("ljushift", C.c_double),
                ("r2uminin", C.c_double), ("utoltab", C.c_double), ("ftoltab", C.c_double),
                ("umaxtab", C.c_double), ("fmaxtab", C.c_double), ("rumaxfac", C.c_double)]


# Every entry point of include/molsim_gpu.h with (restype, argtypes).
SIGNATURES = {
    "msg_create": (C.c_int, [C.POINTER(MsgParams), C.c_int32, C.POINTER(C.c_void_p)]),
    "msg_create_batch": (C.c_int, [C.POINTER(MsgParams), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "msg_destroy": (None, [C.c_void_p]),
    "msg_last_error": (C.c_char_p, [C.c_void_p]),
    "msg_nsys": (C.c_int32, [C.c_void_p]),
    "msg_set_state": (C.c_int, [C.c_void_p, C.c_int32, f64p, f64p, f64p]),
    "msg_nlist_before_macrostep": (C.c_int, [C.c_void_p]),
    "msg_set_state_all": (C.c_int, [C.c_void_p, f64p, f64p, f64p]),
    "msg_get_state": (C.c_int, [C.c_void_p, C.c_int32, f64p, f64p, f64p]),
    "msg_build_nlist": (C.c_int, [C.c_void_p, C.c_int32, i32p, i32p, C.c_int32, C.POINTER(C.c_int64)]),
    "msg_utotal": (C.c_int, [C.c_void_p, C.c_int32, f64p, f64p, C.POINTER(MsgEnergy)]),
    "msg_get_linacc": (C.c_int, [C.c_void_p]),
    "msg_mc_seed": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "msg_velver_p": (C.c_int, [C.c_int32] * 5 + [f64p, C.c_double, C.c_double, C.c_int32, C.c_double] + [f64p] * 7 +
                     [i32p] * 4 + [f64p, C.c_int32, f64p, f64p, i32p, i32p, C.c_int32, f64p, C.c_int32, i32p, f64p,
                                   f64p, f64p, C.POINTER(C.c_float)]),
    "msg_velver_p_ewald": (C.c_int, [C.c_int32] * 5 + [f64p, C.c_double, C.c_double, C.c_int32, C.c_double] +
                           [f64p] * 7 + [i32p] * 4 + [f64p, C.c_int32, f64p, f64p, i32p, i32p, C.c_int32, f64p,
                                                      C.c_int32, i32p, f64p, C.POINTER(MsgSiteEwald), f64p, f64p,
                                                      f64p, C.POINTER(C.c_float)]),
    "msg_utwobody_p": (C.c_int, [C.c_int32] * 4 + [f64p, C.c_double, f64p, f64p] + [i32p] * 6 +
                       [C.c_int32, f64p, C.c_int32, i32p, f64p, f64p, f64p, f64p, C.POINTER(C.c_float)]),
    "msg_uewald_sites": (C.c_int, [C.c_int32, f64p, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_double, f64p,
                                   f64p, C.c_int32, i32p, i32p, i32p, C.c_int32, f64p, f64p, f64p,
                                   C.POINTER(C.c_float)]),
    "msg_uewald_sites_spm": (C.c_int, [C.c_int32, f64p, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                       f64p, f64p, C.c_int32, i32p, i32p, i32p, C.c_int32, f64p, f64p, f64p,
                                       C.POINTER(C.c_float)]),
    "msg_mcall_pass": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(MsgMcAllParams), C.POINTER(C.c_int64), C.c_int32,
                                 C.POINTER(MsgEnergy)]),
    "msg_random_jump": (C.c_int, [C.c_int32, C.c_int32, C.c_uint32, C.POINTER(C.c_int32)]),
    "msg_mc_pass": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(MsgMcParams), C.POINTER(C.c_int64),
                              C.POINTER(C.c_int64), C.c_int32, C.POINTER(MsgEnergy)]),
    "msg_get_forces": (C.c_int, [C.c_void_p, C.c_int32, f64p, f64p]),
    "msg_tune": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "msg_velver": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MsgEnergy)]),
    "msg_velver_async": (C.c_int, [C.c_void_p, C.c_int32]),
    "msg_velver_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, f64p, f64p, f64p, C.POINTER(MsgEnergy)]),
    "msg_bd_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_uint64, C.c_int32, f64p, f64p, C.POINTER(MsgEnergy)]),
    "msg_nrebuild": (C.c_int64, [C.c_void_p, C.c_int32]),
    "msg_put_state": (C.c_int, [C.c_void_p, C.c_int32, f64p, f64p, f64p, C.c_int32]),
    "msg_estimate_bytes": (C.c_int, [C.POINTER(MsgParams), C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    "msg_device_bytes": (C.c_int64, [C.c_void_p]),
    "msg_pending": (C.c_int, [C.c_void_p]),
    "msg_get_energy": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(MsgEnergy)]),
    "msg_trim_caches": (C.c_int, []),
    "msg_stream": (C.c_void_p, [C.c_void_p]),
    "msg_launch_count": (C.c_int64, [C.c_void_p]),
    "msg_set_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "msg_ntimers": (C.c_int32, []),
    "msg_kernel_time": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_char_p), f64p, C.POINTER(C.c_int64)]),
    "msg_utwobody_noalloc": (C.c_int, [C.c_int32, C.c_int32, f64p, C.c_double, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                                       i32p, f64p, f64p, C.c_void_p, C.c_void_p, C.c_void_p, i32p,
                                       C.c_void_p]),
    "msg_rcut_to_alpha": (C.c_double, [C.c_double] * 5 + [i32p]),
    "msg_alpha_to_ncut": (C.c_int32, [C.c_double] * 5 + [i32p]),
    "msg_pot_tab": (C.c_int, [C.POINTER(MsgTabParams), f64p, C.c_int32, i32p, i32p, f64p, i32p]),
}


def lib():
    """Load the in-tree library.  There is no fallback: a missing or stale build is an error."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libmolsim_gpu.so is not built; run `python -m molsim_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB
