"""Python mirror of the cfd_plugin C ABI (include/zerork_cfd_plugin.h).

Same calls and status codes as the reference's zerork_cfd_plugin.h
(applications/cfd_plugin/zerork_cfd_plugin.h:11-87); the solve runs the
sm_100a batched integrator in lib/libzerork_b200.so.
"""
import ctypes as C

import numpy as np

from . import lib as _lib

STATUS = ["SUCCESS", "INVALID_HANDLE", "INVALID_FILENAME", "INVALID_FIELD_NAME",
          "INVALID_POINTER", "FAILED_MECHANISM_PARSE", "FAILED_OPTIONS_PARSE", "FAILED_SOLVE",
          "OPTION_NOT_DEFINED"]
FIELDS = {"DPDT": 0, "COST": 1, "GPU": 2, "Y_SRC": 3, "E_SRC": 4, "IGNITION_TIME": 5,
          "TEMPERATURE_DELTA": 6}


def status_name(code):
    return STATUS[code] if 0 <= code < len(STATUS) else ("UNKNOWN_ERROR" if code == 99 else str(code))


class PluginError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what}: {status_name(code)}")
        self.code = code


_bound = False

# zerork_callback_fn (applications/cfd_plugin/zerork_cfd_plugin.h:44-46)
CALLBACK = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                       C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p)


def plugin_lib():
    global _bound
    L = _lib()
    if not _bound:
        vp, cp = C.c_void_p, C.c_char_p
        L.zerork_reactor_init.restype = vp
        L.zerork_reactor_read_options_file.argtypes = [cp, vp]
        L.zerork_reactor_set_mechanism_files.argtypes = [cp, cp, vp]
        L.zerork_reactor_load_mechanism.argtypes = [vp]
        L.zerork_reactor_solve.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, vp, vp, vp, vp]
        L.zerork_reactor_set_aux_field_pointer.argtypes = [C.c_int, vp, vp]
        L.zerork_reactor_set_int_option.argtypes = [cp, C.c_int, vp]
        L.zerork_reactor_set_double_option.argtypes = [cp, C.c_double, vp]
        L.zerork_reactor_set_string_option.argtypes = [cp, cp, vp]
        L.zerork_reactor_get_int_option.argtypes = [cp, C.POINTER(C.c_int), vp]
        L.zerork_reactor_get_double_option.argtypes = [cp, C.POINTER(C.c_double), vp]
        L.zerork_reactor_get_string_option.argtypes = [cp, C.POINTER(C.c_char_p), C.c_int, vp]
        L.zerork_reactor_set_reactor_ids.argtypes = [vp, vp]
        L.zerork_reactor_set_callback_fn.argtypes = [CALLBACK, vp, vp]
        L.zrk_plugin_num_species.argtypes = [vp]
        L.zerork_reactor_free.argtypes = [vp]
        L.zrk_plugin_last_stats.argtypes = [vp, C.POINTER(C.c_long), C.POINTER(C.c_float)]
        L.zrk_plugin_set_predictor.argtypes = [vp, vp, vp, vp, vp, vp]
        L.zrk_plugin_graph_stats.argtypes = [vp, C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.zrk_plugin_krylov_iterations.argtypes = [vp, C.POINTER(C.c_long)]
        L.zrk_plugin_group_stats.argtypes = [vp, C.POINTER(C.c_long)]
        L.zrk_plugin_autotune.argtypes = [vp, C.c_int, C.c_double, vp, vp, vp, C.POINTER(C.c_int),
                                          C.POINTER(C.c_float)]
        _bound = True
    return L


class Plugin:
    """One plugin handle (not thread-safe, like the reference's)."""

    def __init__(self, mech=None, therm=None, **options):
        self.L = plugin_lib()
        self.h = self.L.zerork_reactor_init()
        if not self.h:
            raise PluginError(99, "zerork_reactor_init")
        self._keep = {}
        if mech:
            self.check(self.L.zerork_reactor_set_mechanism_files(
                str(mech).encode(), None if therm is None else str(therm).encode(), self.h),
                "set_mechanism_files")
        for k, v in options.items():
            self.set_option(k, v)

    def check(self, rc, what):
        if rc != 0:
            raise PluginError(rc, what)
        return rc

    def close(self):
        if self.h:
            self.L.zerork_reactor_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, name, value):
        n = name.encode()
        if isinstance(value, bool) or isinstance(value, (int, np.integer)):
            rc = self.L.zerork_reactor_set_int_option(n, int(value), self.h)
        elif isinstance(value, float):
            rc = self.L.zerork_reactor_set_double_option(n, value, self.h)
        else:
            rc = self.L.zerork_reactor_set_string_option(n, str(value).encode(), self.h)
        self.check(rc, f"set {name}")

    def get_int(self, name):
        v = C.c_int()
        self.check(self.L.zerork_reactor_get_int_option(name.encode(), C.byref(v), self.h), name)
        return v.value

    def get_double(self, name):
        v = C.c_double()
        self.check(self.L.zerork_reactor_get_double_option(name.encode(), C.byref(v), self.h), name)
        return v.value

    def get_string(self, name, length=256):
        buf = C.create_string_buffer(length)
        p = C.c_char_p(C.addressof(buf))
        self.check(self.L.zerork_reactor_get_string_option(name.encode(), C.byref(p), length, self.h),
                   name)
        return buf.value.decode()

    def read_options_file(self, path):
        self.check(self.L.zerork_reactor_read_options_file(str(path).encode(), self.h),
                   "read_options_file")

    def load_mechanism(self):
        self.check(self.L.zerork_reactor_load_mechanism(self.h), "load_mechanism")

    def set_aux_field(self, field, array):
        a = np.ascontiguousarray(array, dtype=np.float64)
        self._keep[field] = a
        self.check(self.L.zerork_reactor_set_aux_field_pointer(FIELDS[field], a.ctypes.data, self.h),
                   f"aux {field}")
        return a

    def set_callback(self, fn):
        """Per-step callback fn(reactor_id, steps, time, dt, y, dy) -> int,
        y and dy float64 arrays of nsp + 1 (mass fractions, T / Tref) valid
        during the call; a nonzero return ends that reactor's integration at
        that step (zerork_reactor_set_callback_fn, solver_cvode.cpp:247-257)."""
        nv = [None]

        def tramp(rid, steps, t, dt, y, dy, _data):
            if nv[0] is None:
                nv[0] = self.L.zrk_plugin_num_species(self.h) + 1
            n = nv[0]
            return int(fn(rid, steps, t, dt, np.ctypeslib.as_array(y, (n,)),
                          np.ctypeslib.as_array(dy, (n,))))

        cfn = CALLBACK(tramp)
        self._keep["callback"] = cfn
        self.check(self.L.zerork_reactor_set_callback_fn(cfn, None, self.h), "set_callback_fn")

    def set_reactor_ids(self, ids):
        a = np.ascontiguousarray(ids, dtype=np.int32)
        self._keep["reactor_ids"] = a
        self.check(self.L.zerork_reactor_set_reactor_ids(a.ctypes.data, self.h), "set_reactor_ids")
        return a

    def solve(self, dt, T, P, Y, n_cycle=0, time=0.0, raise_on_fail=True):
        """In place on float64 arrays T[n], P[n], Y[n, nsp] (reactor-major)."""
        for a in (T, P, Y):
            assert a.dtype == np.float64 and a.flags.c_contiguous
        rc = self.L.zerork_reactor_solve(n_cycle, time, dt, T.shape[0], T.ctypes.data, P.ctypes.data,
                                         Y.ctypes.data, self.h)
        if rc != 0 and (raise_on_fail or rc != 7):
            raise PluginError(rc, "zerork_reactor_solve")
        return rc

    def set_predictor(self, net, x_scaler=None, t_scaler=None):
        """Attach a trained predictor network (zerork_b200.predictor.Mlp) with
        its input/target standardisation; net=None detaches it."""
        if net is None:
            self.check(self.L.zrk_plugin_set_predictor(self.h, None, None, None, None, None),
                       "set_predictor")
            self._keep.pop("predictor", None)
            return
        arrs = [np.ascontiguousarray(a, dtype=np.float32)
                for a in (x_scaler.mu, x_scaler.sd, t_scaler.mu, t_scaler.sd)]
        self._keep["predictor"] = (net, arrs)
        rc = self.L.zrk_plugin_set_predictor(self.h, net.h, *[a.ctypes.data for a in arrs])
        if rc != 0:
            raise PluginError(99, "set_predictor: " + _lib().zrk_last_error().decode())

    def graph_stats(self):
        c, l = C.c_long(), C.c_long()
        self.L.zrk_plugin_graph_stats(self.h, C.byref(c), C.byref(l))
        return {"captures": c.value, "launches": l.value}

    def autotune(self, dt, T, P, Y):
        """Tune the integrator launch mapping on a sample of these reactors;
        returns (best setting, kernel ms)."""
        T = np.ascontiguousarray(T, np.float64)
        P = np.ascontiguousarray(P, np.float64)
        Y = np.ascontiguousarray(Y, np.float64)
        b, ms = C.c_int(), C.c_float()
        rc = self.L.zrk_plugin_autotune(self.h, T.shape[0], dt, T.ctypes.data, P.ctypes.data,
                                        Y.ctypes.data, C.byref(b), C.byref(ms))
        if rc != 0:
            raise PluginError(99, "autotune: " + _lib().zrk_last_error().decode())
        return b.value, ms.value

    def last_stats(self):
        t = (C.c_long * 7)()
        ms = C.c_float()
        self.L.zrk_plugin_last_stats(self.h, t, C.byref(ms))
        keys = ("nsteps", "nrej", "nnewt", "njac", "nlu", "nrhs", "nfailed")
        d = {k: int(t[i]) for i, k in enumerate(keys)}
        d["kernel_ms"] = ms.value
        k = C.c_long()
        self.L.zrk_plugin_krylov_iterations(self.h, C.byref(k))
        d["nkry"] = k.value
        g = (C.c_long * 6)()
        self.L.zrk_plugin_group_stats(self.h, g)
        for i, key in enumerate(("groups", "group_steps", "group_newton", "launches", "syncs",
                                 "group_status")):
            d[key] = int(g[i])
        return d
