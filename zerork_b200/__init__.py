"""zerork_b200 -- sm_100a kernels for Zero-RK's batched stiff-reactor path.

Python host-side mirror of the C ABI in include/zerork_b200.h (mechanism
level) and include/zerork_cfd_plugin.h (the cfd_plugin reactor solver).  The
compute path is the in-tree shared library lib/libzerork_b200.so; there is no
CPU fallback: on a machine without the library or without a GPU the compute
entry points raise.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libzerork_b200.so")

_lib = None


class ZeroRKError(RuntimeError):
    """A nonzero status from the shared library (message from zrk_last_error)."""

    def __init__(self, code, msg):
        super().__init__(f"[zerork_b200 error {code}] {msg}")
        self.code = code


def lib():
    """The loaded shared library (built by zerork_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ZeroRKError(-1, f"{LIB_PATH} is missing; run `python zerork_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.zrk_last_error.restype = C.c_char_p
        L.zrk_mech_create.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(vp)]
        L.zrk_mech_parse.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(vp)]
        L.zrk_mech_free.argtypes = [vp]
        L.zrk_mech_sizes.argtypes = [vp, ip, ip, ip, ip]
        L.zrk_mech_table.argtypes = [vp, C.c_char_p, vp, C.c_long, C.POINTER(C.c_long), ip]
        L.zrk_mech_species_name.restype = C.c_char_p
        L.zrk_mech_species_name.argtypes = [vp, C.c_int]
        L.zrk_mech_jac_pattern.argtypes = [vp, vp, vp]
        L.zrk_mech_set_double_option.argtypes = [vp, C.c_char_p, C.c_double]
        L.zrk_mech_get_double_option.argtypes = [vp, C.c_char_p, dp]
        L.zrk_mech_set_launch.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.zrk_mech_get_launch.argtypes = [vp, ip, ip, ip, ip, ip]
        L.zrk_mech_autotune.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp,
                                        C.POINTER(C.c_float)]
        L.zrk_rates_jac_dev.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.zrk_rates_jac_host.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
        L.zrk_rates_tc_dev.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
        L.zrk_rates_tc_host.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.zrk_measure_fp64.argtypes = [dp, dp]
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise ZeroRKError(rc, lib().zrk_last_error().decode())
    return rc


def _ptr(x):
    """Raw address of a numpy array or torch tensor (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return C.c_void_p(x.ctypes.data)
    return C.c_void_p(x.data_ptr())


def measure_fp64():
    """(FP64 FMA GFLOP/s, double exp G/s) measured on the current device."""
    a, b = C.c_double(), C.c_double()
    check(lib().zrk_measure_fp64(C.byref(a), C.byref(b)))
    return a.value, b.value


TABLE_NAMES = ("mw", "thermo", "step_rxn", "step_dir", "reac_ptr", "reac_spc", "prod_ptr",
               "prod_spc", "arr_step", "arr_lnA", "arr_n", "arr_Ta", "keq_step", "keq_fwd",
               "keq_dn", "tb_fwd", "tb_rev", "tb_ptr", "tb_spc", "tb_alpha", "fo_fwd", "fo_rev",
               "fo_type", "fo_spc", "fo_ptr", "fo_eff_spc", "fo_alpha", "fo_par", "plog_step",
               "plog_pt_ptr", "plog_ln_ptr", "plog_p", "plog_lnp", "plog_lnA", "plog_sgn", "plog_n",
               "plog_Ta")


class Mechanism:
    """A CHEMKIN mechanism on the GPU (mirrors zerork::mechanism / mechanism_cuda).

    ``device=False`` parses only (tables and Jacobian pattern, no GPU needed).
    """

    def __init__(self, mech_file, therm_file, device=True):
        L = lib()
        h = C.c_void_p()
        fn = L.zrk_mech_create if device else L.zrk_mech_parse
        check(fn(str(mech_file).encode(), str(therm_file).encode(), C.byref(h)))
        self._h = h
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(L.zrk_mech_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        self.nsp, self.nrxn, self.nstep, self.nnz = a.value, b.value, c.value, d.value
        self.species = [L.zrk_mech_species_name(h, i).decode() for i in range(self.nsp)]
        self.files = (str(mech_file), str(therm_file))

    def close(self):
        if getattr(self, "_h", None):
            lib().zrk_mech_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def table(self, name):
        L = lib()
        cnt, isd = C.c_long(), C.c_int()
        check(L.zrk_mech_table(self._h, name.encode(), None, 0, C.byref(cnt), C.byref(isd)))
        out = np.zeros(cnt.value, dtype=np.float64 if isd.value else np.int32)
        check(L.zrk_mech_table(self._h, name.encode(), out.ctypes.data_as(C.c_void_p),
                               cnt.value, C.byref(cnt), C.byref(isd)))
        return out

    def tables(self):
        d = {n: self.table(n) for n in TABLE_NAMES}
        d.update(nsp=self.nsp, nrxn=self.nrxn, nstep=self.nstep)
        return d

    def jac_pattern(self):
        cp = np.zeros(self.nsp + 2, dtype=np.int32)
        ri = np.zeros(self.nnz, dtype=np.int32)
        check(lib().zrk_mech_jac_pattern(self._h, cp.ctypes.data_as(C.c_void_p),
                                         ri.ctypes.data_as(C.c_void_p)))
        return cp, ri

    def set_option(self, name, value):
        check(lib().zrk_mech_set_double_option(self._h, name.encode(), float(value)))

    def get_option(self, name):
        v = C.c_double()
        check(lib().zrk_mech_get_double_option(self._h, name.encode(), C.byref(v)))
        return v.value

    def set_launch(self, ts=0, v=1, warps=8, global_ws=False, grid=0, stage=False, two_ctas=False):
        flags = (1 if global_ws else 0) | (2 if stage else 0) | (4 if two_ctas else 0)
        check(lib().zrk_mech_set_launch(self._h, ts, v, warps, flags, grid))

    def get_launch(self):
        a, b, c, d, e = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().zrk_mech_get_launch(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d),
                                        C.byref(e)))
        return dict(ts=a.value, v=b.value, warps=c.value, global_ws=bool(d.value & 1), grid=e.value,
                    stage=bool(d.value & 2), two_ctas=bool(d.value & 4))

    def autotune(self, T, P, Y, wdot, jac=None, n=None, stream=None):
        """Time every tile/warp mapping on a device sample; keep the fastest."""
        ld = Y.shape[1]
        n = ld if n is None else n
        s = None if stream is None else C.c_void_p(stream)
        ms = C.c_float()
        check(lib().zrk_mech_autotune(self._h, n, ld, _ptr(T), _ptr(P), _ptr(Y), _ptr(wdot),
                                      _ptr(jac), s, C.byref(ms)))
        return self.get_launch(), ms.value

    def rates_jac(self, T, P, Y, wdot, jac=None, ydot=None, n=None, stream=None):
        """Device tensors, species-major: Y[nsp, ld], wdot[nsp, ld], jac[nnz, ld]."""
        ld = Y.shape[1]
        n = ld if n is None else n
        s = None if stream is None else C.c_void_p(stream)
        check(lib().zrk_rates_jac_dev(self._h, n, ld, _ptr(T), _ptr(P), _ptr(Y), _ptr(wdot),
                                      _ptr(jac), _ptr(ydot), s))

    def rates_tc(self, T, conc, step_limiter=None, stream=None):
        """Rates from temperature and concentrations (mechanism_cuda's
        getReactionRates(Limiter)_CUDA_mr_dev): device tensors T[n],
        C[nsp, n] (species-major); returns device tensors (net, create,
        destroy [nsp, n], rop [nstep, n])."""
        import torch
        n = T.shape[0]
        ld = conc.shape[1]
        kw = dict(dtype=torch.float64, device=conc.device)
        net, cre, des = (torch.empty((self.nsp, ld), **kw) for _ in range(3))
        rop = torch.empty((self.nstep, ld), **kw)
        s = None if stream is None else C.c_void_p(stream)
        check(lib().zrk_rates_tc_dev(self._h, n, ld, _ptr(T), _ptr(conc), _ptr(step_limiter), _ptr(net),
                                     _ptr(cre), _ptr(des), _ptr(rop), s))
        return net, cre, des, rop

    def rates_tc_host(self, T, conc, step_limiter=None):
        """Host arrays T[n], C[nsp, n] (species-major); the host-side
        getReactionRates(Limiter) for n states.  Returns numpy (net, create,
        destroy, rop)."""
        T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
        n = T.shape[0]
        Cm = np.ascontiguousarray(conc, dtype=np.float64).reshape(self.nsp, n)
        lim = None if step_limiter is None else np.ascontiguousarray(step_limiter, dtype=np.float64)
        net, cre, des = (np.zeros((self.nsp, n)) for _ in range(3))
        rop = np.zeros((self.nstep, n))
        check(lib().zrk_rates_tc_host(self._h, n, _ptr(T), _ptr(Cm), _ptr(lim), _ptr(net), _ptr(cre),
                                      _ptr(des), _ptr(rop)))
        return net, cre, des, rop

    def rates_jac_host(self, T, P, Y, want_jac=True):
        """Host numpy arrays (species-major Y[nsp, n]); returns (wdot, jac)."""
        T = np.ascontiguousarray(T, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        n = T.shape[0]
        wdot = np.zeros((self.nsp, n))
        jac = np.zeros((self.nnz, n)) if want_jac else None
        check(lib().zrk_rates_jac_host(self._h, n, _ptr(T), _ptr(P), _ptr(Y), _ptr(wdot), _ptr(jac)))
        return wdot, jac
