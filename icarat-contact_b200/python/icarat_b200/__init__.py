"""ctypes binding of libicarat_b200.so (the C ABI in include/icarat_b200.h).

This is the thin layer the tests, the smoke check and bench.py drive the
library through; every call goes through the exported C entry points.  There
is no fallback: if the shared library is missing or no CUDA device is present
the calls raise.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(os.path.dirname(_HERE))  # icarat-contact_b200/
LIB_PATH = os.path.join(PKG_DIR, "lib", "libicarat_b200.so")
HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "icarat_b200.h")

FP64, MIXED, TF32, MIXED_REFINE = 0, 1, 2, 3
JACOBI, GMG = 0, 1
PLANE_STRESS, PLANE_STRAIN, THREE_D = 0, 1, 2
JOB_OC, JOB_MMA = 0, 1
FILTER_HELMHOLTZ, FILTER_CONE = 0, 1
STATUS = {0: "OK", -1: "BAD_ARG", -2: "OOM", -3: "BREAKDOWN", -4: "MAXITER", -5: "TIMEOUT",
          -6: "NAN", -7: "CUDA", -8: "STATE", -9: "REJECTED"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)
_llp = C.POINTER(C.c_longlong)


class GridDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("state", C.c_int), ("young1", C.c_double), ("young2", C.c_double),
                ("poisson", C.c_double), ("penalty", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("precond", C.c_int), ("tol", C.c_double),
                ("maxit", C.c_int), ("inner_tol", C.c_double), ("mg_smooth", C.c_int),
                ("mg_coarse_dofs", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("matvecs", C.c_int), ("outer", C.c_int),
                ("relres", C.c_double), ("true_relres", C.c_double), ("seconds", C.c_double),
                ("status", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


STEP_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_double, _dp, _dp, _dp)


class LoopOpts(C.Structure):
    _fields_ = [("nsteps", C.c_int), ("filter_radius", C.c_double), ("move_limit", C.c_double),
                ("use_threshold", C.c_int), ("volume_ref", C.c_double), ("solve", SolveOpts),
                ("iter_seconds", _dp), ("filter_type", C.c_int), ("nondesign", _u8p),
                ("volume_set", _u8p), ("on_step", STEP_CB), ("step_user", C.c_void_p),
                ("conv_eps", C.c_double), ("conv_min_steps", C.c_int), ("steps_done", _ip),
                ("resume", C.c_void_p), ("checkpoint", C.c_void_p)]


class JobDesc(C.Structure):
    _fields_ = [("grid", GridDesc), ("kind", C.c_int), ("loop", LoopOpts),
                ("fixed", _u8p), ("load", _dp), ("rho0", _dp)]


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("end_s", C.c_double), ("bytes", C.c_longlong),
                ("nsteps", C.c_int)]


class IcbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None

# exported symbol -> (restype, argtypes); every name declared in the header
_SIGS = {
    "icb_last_error": (C.c_char_p, []),
    "icb_version": (C.c_char_p, []),
    "icb_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "icb_ctx_destroy": (C.c_int, [C.c_void_p]),
    "icb_ctx_stream": (C.c_void_p, [C.c_void_p]),
    "icb_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "icb_problem_create": (C.c_int, [C.c_void_p, C.POINTER(GridDesc), C.POINTER(C.c_void_p)]),
    "icb_problem_destroy": (C.c_int, [C.c_void_p]),
    "icb_dirichlet_box": (C.c_int, [C.c_void_p, _ip, _dp, _dp]),
    "icb_dirichlet_mask": (C.c_int, [C.c_void_p, _u8p, _dp]),
    "icb_traction_box": (C.c_int, [C.c_void_p, _dp, _dp]),
    "icb_nodal_load": (C.c_int, [C.c_void_p, C.c_longlong, _dp]),
    "icb_finalize": (C.c_int, [C.c_void_p, _llp]),
    "icb_count_dof": (C.c_int, [C.c_void_p, _ip, C.POINTER(C.c_longlong)]),
    "icb_get_dof_map": (C.c_int, [C.c_void_p, _ip]),
    "icb_von_mises": (C.c_int, [C.c_void_p, _dp, _dp]),
    "icb_heat_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "icb_heat_destroy": (C.c_int, [C.c_void_p]),
    "icb_heat_dirichlet_box": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _dp]),
    "icb_heat_flux_box": (C.c_int, [C.c_void_p, C.c_double, _dp]),
    "icb_heat_nodal_source": (C.c_int, [C.c_void_p, C.c_longlong, C.c_double]),
    "icb_heat_finalize": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "icb_heat_set_density": (C.c_int, [C.c_void_p, _dp]),
    "icb_heat_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "icb_heat_get_temperature": (C.c_int, [C.c_void_p, _dp]),
    "icb_heat_objective": (C.c_int, [C.c_void_p, _dp]),
    "icb_heat_sensitivity": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "icb_run_heat": (C.c_int, [C.c_void_p, C.c_void_p, _dp, _dp, _dp]),
    "icb_gcmma_create": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.POINTER(C.c_void_p)]),
    "icb_gcmma_destroy": (C.c_int, [C.c_void_p]),
    "icb_gcmma_outer": (C.c_int, [C.c_void_p, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp, _dp]),
    "icb_gcmma_inner": (C.c_int, [C.c_void_p, _dp, C.c_double, _dp, _dp, C.c_double, _dp, _dp,
                                  _dp, _dp, _dp]),
    "icb_gcmma_concheck": (C.c_int, [C.c_void_p, C.c_double, _dp, _ip]),
    "icb_run_gcmma": (C.c_int, [C.c_void_p, C.c_void_p, _dp, _dp, _ip, _dp]),
    "icb_reactions": (C.c_int, [C.c_void_p, _dp]),
    "icb_get_load": (C.c_int, [C.c_void_p, _dp]),
    "icb_problem_sizes": (C.c_int, [C.c_void_p, _llp, _llp, _llp, _llp]),
    "icb_get_K0": (C.c_int, [C.c_void_p, _dp]),
    "icb_element_volume": (C.c_int, [C.c_void_p, _dp]),
    "icb_set_density": (C.c_int, [C.c_void_p, _dp]),
    "icb_set_density_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "icb_solve": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    "icb_get_displacement": (C.c_int, [C.c_void_p, _dp]),
    "icb_get_node_values": (C.c_int, [C.c_void_p, _dp]),
    "icb_compliance": (C.c_int, [C.c_void_p, _dp]),
    "icb_sensitivity": (C.c_int, [C.c_void_p, _dp, _dp]),
    "icb_sensitivity_device": (C.c_void_p, [C.c_void_p]),
    "icb_matvec": (C.c_int, [C.c_void_p, _dp, _dp]),
    "icb_diagonal": (C.c_int, [C.c_void_p, _dp]),
    "icb_soa_length": (C.c_longlong, [C.c_void_p]),
    "icb_operator_apply_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "icb_smoother_apply_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_double, C.c_double]),
    "icb_launch_count": (C.c_longlong, []),
    "icb_solve_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                    C.POINTER(SolveInfo)]),
    "icb_noalloc_max_soa": (C.c_longlong, []),
    "icb_loop_checkpoint_bytes": (C.c_longlong, [C.c_void_p, C.c_int]),
    "icb_set_option": (C.c_int, [C.c_char_p, C.c_longlong]),
    "icb_run_batch": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), _ip, C.POINTER(LoopOpts),
                                C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), C.c_int, _ip]),
    "icb_job_footprint": (C.c_longlong, [C.POINTER(GridDesc), C.c_int]),
    "icb_server_create": (C.c_int, [C.c_int, C.c_longlong, C.c_int, C.POINTER(C.c_void_p)]),
    "icb_server_submit": (C.c_int, [C.c_void_p, C.POINTER(JobDesc), _llp]),
    "icb_server_wait": (C.c_int, [C.c_void_p, C.c_longlong, C.c_double, C.POINTER(JobInfo)]),
    "icb_server_result": (C.c_int, [C.c_void_p, C.c_longlong, _dp, _dp, _dp]),
    "icb_server_cancel": (C.c_int, [C.c_void_p, C.c_longlong]),
    "icb_server_forget": (C.c_int, [C.c_void_p, C.c_longlong]),
    "icb_server_destroy": (C.c_int, [C.c_void_p]),
    "icb_get_option": (C.c_longlong, [C.c_char_p]),
    "icb_cone_create": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_void_p)]),
    "icb_cone_destroy": (C.c_int, [C.c_void_p]),
    "icb_cone_filter": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    "icb_cone_filter_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "icb_threshold": (C.c_int, [C.c_void_p, C.c_longlong, _dp, C.c_double, C.c_double, _dp, _dp]),
    "icb_helm_create": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_void_p)]),
    "icb_helm_destroy": (C.c_int, [C.c_void_p]),
    "icb_helm_filter": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    "icb_oc_update": (C.c_int, [C.c_void_p, C.c_void_p, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                C.c_double, C.c_double, C.c_double, _ip]),
    "icb_mma_create": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.POINTER(C.c_void_p)]),
    "icb_mma_destroy": (C.c_int, [C.c_void_p]),
    "icb_mma_update": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]),
    "icb_run_oc": (C.c_int, [C.c_void_p, C.POINTER(LoopOpts), _dp, _dp, _dp]),
    "icb_run_mma": (C.c_int, [C.c_void_p, C.POINTER(LoopOpts), _dp, _dp, _dp]),
}


def lib():
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built: run python icarat-contact_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def set_option(name, value):
    check(lib().icb_set_option(name.encode(), int(value)))


def get_option(name):
    return lib().icb_get_option(name.encode())


def launch_count():
    return lib().icb_launch_count()


def header_symbols():
    """Function names declared in include/icarat_b200.h."""
    import re
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(icb_[a-z0-9_]+)\s*\(", txt)))


def check(rc):
    if rc != 0:
        raise IcbError(rc, lib().icb_last_error().decode())
    return rc


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Context:
    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib().icb_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def stream(self):
        return lib().icb_ctx_stream(self.h)

    def synchronize(self):
        check(lib().icb_ctx_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.icb_ctx_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


class Problem:
    """A structured SIMP problem on the device (the LinearAnalysis equivalent)."""

    def __init__(self, ctx, dim, nx, ny, nz=1, lx=None, ly=None, lz=None, state=None,
                 young=(1e-9, 1.0), nu=0.3, penal=3.0):
        self.ctx = ctx
        self.dim = dim
        self.desc = GridDesc(dim, nx, ny, nz if dim == 3 else 1,
                             float(nx if lx is None else lx), float(ny if ly is None else ly),
                             float((nz if dim == 3 else 1) if lz is None else lz),
                             (THREE_D if dim == 3 else PLANE_STRESS) if state is None else state,
                             float(young[0]), float(young[1]), float(nu), float(penal))
        h = C.c_void_p()
        check(lib().icb_problem_create(ctx.h, C.byref(self.desc), C.byref(h)))
        self.h = h
        nel, nn, neq, ne = C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(lib().icb_problem_sizes(self.h, C.byref(nel), C.byref(nn), C.byref(neq), C.byref(ne)))
        self.nel, self.nnode, self.neq = nel.value, nn.value, neq.value
        self.numeq = None

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.icb_problem_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    # set-up -------------------------------------------------------------
    def dirichlet_box(self, flag, val, rng):
        f = np.asarray(list(flag) + [0] * (6 - len(flag)), np.int32)
        v = np.asarray(list(val) + [0.0] * (6 - len(val)), np.float64)
        r = np.asarray(rng, np.float64).reshape(6)
        check(lib().icb_dirichlet_box(self.h, _p(f, _ip), _p(v), _p(r)))

    def dirichlet_mask(self, fixed, val=None):
        f = np.ascontiguousarray(fixed, np.uint8)
        v = None if val is None else _p(np.ascontiguousarray(val, np.float64))
        check(lib().icb_dirichlet_mask(self.h, _p(f, _u8p), v))

    def traction_box(self, val, rng):
        v = np.zeros(3)
        v[:len(val)] = val
        r = np.asarray(rng, np.float64).reshape(6)
        check(lib().icb_traction_box(self.h, _p(v), _p(r)))

    def nodal_load(self, node, f):
        v = np.zeros(3)
        v[:len(f)] = f
        check(lib().icb_nodal_load(self.h, int(node), _p(v)))

    def finalize(self):
        ne = C.c_longlong()
        check(lib().icb_finalize(self.h, C.byref(ne)))
        self.numeq = ne.value
        return self.numeq

    def dof_map(self):
        d = np.zeros(self.neq, np.int32)
        check(lib().icb_get_dof_map(self.h, _p(d, _ip)))
        return d

    def load(self):
        f = np.zeros(self.numeq)
        check(lib().icb_get_load(self.h, _p(f)))
        return f

    def K0(self):
        nd = self.dim * (4 if self.dim == 2 else 8)
        K = np.zeros((nd, nd))
        check(lib().icb_get_K0(self.h, _p(K)))
        return K

    def element_volume(self):
        v = C.c_double()
        check(lib().icb_element_volume(self.h, C.byref(v)))
        return v.value

    # analysis -----------------------------------------------------------
    def set_density(self, rho):
        r = np.ascontiguousarray(rho, np.float64)
        assert r.size == self.nel
        check(lib().icb_set_density(self.h, _p(r)))

    def set_density_device(self, ptr):
        check(lib().icb_set_density_device(self.h, C.c_void_p(ptr)))

    def solve(self, precision=FP64, precond=JACOBI, tol=1e-10, maxit=10000, inner_tol=0.0,
              mg_smooth=0, mg_coarse_dofs=0, raise_on_error=True):
        o = SolveOpts(precision, precond, tol, maxit, inner_tol, mg_smooth, mg_coarse_dofs)
        info = SolveInfo()
        rc = lib().icb_solve(self.h, C.byref(o), C.byref(info))
        if raise_on_error:
            check(rc)
        d = info.as_dict()
        d["rc"] = rc
        return d

    def displacement(self):
        u = np.zeros(self.numeq)
        check(lib().icb_get_displacement(self.h, _p(u)))
        return u

    def node_values(self):
        v = np.zeros(self.neq)
        check(lib().icb_get_node_values(self.h, _p(v)))
        return v

    def compliance(self):
        c = C.c_double()
        check(lib().icb_compliance(self.h, C.byref(c)))
        return c.value

    def sensitivity(self, with_dv=False):
        dc = np.zeros(self.nel)
        dv = np.zeros(self.nel) if with_dv else None
        check(lib().icb_sensitivity(self.h, _p(dc), None if dv is None else _p(dv)))
        return (dc, dv) if with_dv else dc

    def von_mises(self, with_stress=False):
        m = np.zeros(self.nel)
        v = 3 if self.dim == 2 else 6
        st = np.zeros(self.nel * v) if with_stress else None
        check(lib().icb_von_mises(self.h, _p(m), None if st is None else _p(st)))
        return (m, st.reshape(self.nel, v)) if with_stress else m

    def reactions(self):
        r = np.zeros(self.neq)
        check(lib().icb_reactions(self.h, _p(r)))
        return r

    def matvec(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.numeq)
        check(lib().icb_matvec(self.h, _p(x), _p(y)))
        return y

    def soa_length(self):
        return lib().icb_soa_length(self.h)

    def operator_apply_device(self, x_ptr, y_ptr, precision=FP64):
        check(lib().icb_operator_apply_device(self.h, precision, C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def smoother_apply_device(self, u_ptr, y_ptr, b_ptr, dinv_ptr, c1, c2, precision=FP64):
        """one fused Chebyshev step y <- u + c2 D^-1 (b - K u) + c1 (u - y) on
        device SoA vectors (icb_smoother_apply_device)"""
        check(lib().icb_smoother_apply_device(self.h, precision, C.c_void_p(u_ptr),
                                              C.c_void_p(y_ptr), C.c_void_p(b_ptr),
                                              C.c_void_p(dinv_ptr), float(c1), float(c2)))

    def diagonal(self):
        d = np.zeros(self.numeq)
        check(lib().icb_diagonal(self.h, _p(d)))
        return d


# ------------------------------------------------------ optimisation side --
class Cone:
    """Filter<E,N> density filter on the device."""

    def __init__(self, prob, radius):
        self.p = prob
        h = C.c_void_p()
        check(lib().icb_cone_create(prob.h, radius, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().icb_cone_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def apply(self, x, sens=False):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(self.p.nel)
        check(lib().icb_cone_filter(self.h, _p(x), _p(out), int(sens)))
        return out


class Helmholtz:
    """FilterHelmholtz on the device."""

    def __init__(self, prob, radius):
        self.p = prob
        h = C.c_void_p()
        check(lib().icb_helm_create(prob.h, radius, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().icb_helm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def apply(self, x, sens=False):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(self.p.nel)
        check(lib().icb_helm_filter(self.h, _p(x), _p(out), int(sens)))
        return out


def threshold(ctx, x, beta, T=0.5):
    x = np.ascontiguousarray(x, np.float64)
    a, b = np.zeros_like(x), np.zeros_like(x)
    check(lib().icb_threshold(ctx.h, x.size, _p(x), beta, T, _p(a), _p(b)))
    return a, b


def oc_update(prob, cone, x, dfdx, g, dgdx, xmin, xmax, move, beta=0.0, T=0.5):
    x = np.array(x, np.float64)
    steps = C.c_int()
    args = [np.ascontiguousarray(v, np.float64) for v in (dfdx, dgdx, xmin, xmax)]
    check(lib().icb_oc_update(prob.h, None if cone is None else cone.h, _p(x), _p(args[0]),
                              float(g), _p(args[1]), _p(args[2]), _p(args[3]), move, beta, T,
                              C.byref(steps)))
    return x, steps.value


class HeatDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("cond1", C.c_double * 6), ("cond2", C.c_double * 6), ("penalty", C.c_double)]


class Heat:
    """icb_heat: steady heat conduction with SIMP conductivity (LinearHeat)."""

    def __init__(self, ctx, dim, nx, ny, nz=1, lx=None, ly=None, lz=None,
                 cond1=(1.0, 1.0, 1.0, 0, 0, 0), cond2=(1e-3, 1e-3, 1e-3, 0, 0, 0), penal=3.0):
        self.desc = HeatDesc(dim, nx, ny, nz if dim == 3 else 1, float(lx or nx), float(ly or ny),
                             float((lz or nz) if dim == 3 else 1.0), (C.c_double * 6)(*cond1),
                             (C.c_double * 6)(*cond2), penal)
        h = C.c_void_p()
        check(lib().icb_heat_create(ctx.h, C.byref(self.desc), C.byref(h)))
        self.h, self.ctx, self.dim = h, ctx, dim
        self.nel = nx * ny * (nz if dim == 3 else 1)
        self.nnode = (nx + 1) * (ny + 1) * ((nz + 1) if dim == 3 else 1)

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.icb_heat_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def dirichlet_box(self, flag, val, rng):
        check(lib().icb_heat_dirichlet_box(self.h, int(flag), float(val), _p(np.asarray(rng, np.float64))))

    def flux_box(self, q, rng):
        check(lib().icb_heat_flux_box(self.h, float(q), _p(np.asarray(rng, np.float64))))

    def nodal_source(self, node, q):
        check(lib().icb_heat_nodal_source(self.h, int(node), float(q)))

    def finalize(self):
        n = C.c_longlong()
        check(lib().icb_heat_finalize(self.h, C.byref(n)))
        self.numeq = n.value
        return n.value

    def set_density(self, rho):
        check(lib().icb_heat_set_density(self.h, _p(np.ascontiguousarray(rho, np.float64))))

    def solve(self, tol=1e-10, maxit=10000):
        o = SolveOpts(FP64, JACOBI, tol, maxit, 0.0, 0, 0)
        info = SolveInfo()
        check(lib().icb_heat_solve(self.h, C.byref(o), C.byref(info)))
        return info.as_dict()

    def temperature(self):
        t = np.zeros(self.nnode)
        check(lib().icb_heat_get_temperature(self.h, _p(t)))
        return t

    def objective(self):
        f = C.c_double()
        check(lib().icb_heat_objective(self.h, C.byref(f)))
        return f.value

    def sensitivity(self, rho):
        dc = np.zeros(self.nel)
        check(lib().icb_heat_sensitivity(self.h, _p(np.ascontiguousarray(rho, np.float64)), _p(dc),
                                         None))
        return dc

    def run(self, rho0, nsteps, radius, tol=1e-10, maxit=100000):
        o = LoopOpts(nsteps, radius, 0.15, 1, 0.0, SolveOpts(FP64, JACOBI, tol, maxit, 0.0, 0, 0),
                     None)
        hist, x = np.zeros(nsteps), np.zeros(self.nel)
        check(lib().icb_run_heat(self.h, C.byref(o), _p(np.ascontiguousarray(rho0, np.float64)),
                                 _p(hist), _p(x)))
        return hist, x


class GCMMA:
    """icb_gcmma: GCMMASolver's outer / inner updates and ConCheck (m = 1)."""

    def __init__(self, ctx, n, m=1):
        h = C.c_void_p()
        check(lib().icb_gcmma_create(ctx.h, n, m, C.byref(h)))
        self.h, self.n = h, n

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.icb_gcmma_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def outer(self, xval, f0x, df0dx, fx, dfdx, xmin, xmax):
        xm = np.zeros(self.n)
        a = [np.ascontiguousarray(v, np.float64) for v in (xval, df0dx, np.atleast_1d(fx), dfdx,
                                                           xmin, xmax)]
        check(lib().icb_gcmma_outer(self.h, _p(xm), _p(a[0]), float(f0x), *[_p(v) for v in a[1:]]))
        return xm

    def inner(self, xmma, f0xnew, fxnew, xval, f0x, df0dx, fx, dfdx, xmin, xmax):
        xm = np.array(xmma, np.float64)
        a = [np.ascontiguousarray(v, np.float64) for v in (np.atleast_1d(fxnew), xval, df0dx,
                                                           np.atleast_1d(fx), dfdx, xmin, xmax)]
        check(lib().icb_gcmma_inner(self.h, _p(xm), float(f0xnew), _p(a[0]), _p(a[1]), float(f0x),
                                    *[_p(v) for v in a[2:]]))
        return xm

    def concheck(self, f0xnew, fxnew):
        ok = C.c_int()
        fx = np.ascontiguousarray(np.atleast_1d(fxnew), np.float64)
        check(lib().icb_gcmma_concheck(self.h, float(f0xnew), _p(fx), C.byref(ok)))
        return bool(ok.value)


def run_gcmma(prob, rho0, nsteps, radius, precision=FP64, precond=GMG, tol=1e-8, maxit=20000):
    """icb_run_gcmma: (compliance history, inner iterations per step, design)."""
    o = LoopOpts(nsteps, radius, 0.15, 1, 0.0, SolveOpts(precision, precond, tol, maxit, 0.0, 0, 0),
                 None)
    hist, inner, x = np.zeros(nsteps), np.zeros(nsteps, np.int32), np.zeros(prob.nel)
    rho0 = np.ascontiguousarray(rho0, np.float64)
    check(lib().icb_run_gcmma(prob.h, C.byref(o), _p(rho0), _p(hist), _p(inner, _ip), _p(x)))
    return hist, inner, x


class MMA:
    def __init__(self, ctx, n, m=1):
        h = C.c_void_p()
        check(lib().icb_mma_create(ctx.h, n, m, C.byref(h)))
        self.h, self.n = h, n

    def close(self):
        if getattr(self, "h", None):
            lib().icb_mma_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def update(self, x, dfdx, gx, dgdx, xmin, xmax):
        x = np.array(x, np.float64)
        a = [np.ascontiguousarray(v, np.float64) for v in (dfdx, np.atleast_1d(gx), dgdx, xmin, xmax)]
        check(lib().icb_mma_update(self.h, _p(x), *[_p(v) for v in a]))
        return x


def run_loop(prob, kind, rho0, nsteps, radius, move=0.15, use_threshold=True, volume_ref=0.0,
             precision=FP64, precond=GMG, tol=1e-8, maxit=20000, filter_type=0, nondesign=None,
             volume_set=None, on_step=None, conv_eps=0.0, conv_min_steps=0, steps_done=None,
             resume=None, checkpoint=None):
    """icb_run_oc (kind "oc") or icb_run_mma (kind "mma"): compliance history, design.
    on_step(step, compliance, rho_phys, nodeval, mises) receives numpy copies;
    conv_eps > 0 applies the apps' isConvergence(conv_eps, conv_min_steps)
    stop rule, steps_done (a one-element int32 array) receives the steps run;
    resume (bytes-like) continues a run from its checkpoint, checkpoint (a
    writable uint8 array of checkpoint_bytes(prob, kind)) receives one."""
    o = LoopOpts(nsteps, radius, move, int(use_threshold), volume_ref,
                 SolveOpts(precision, precond, tol, maxit, 0.0, 0, 0), None)
    if resume is not None:
        rbuf = np.frombuffer(bytes(resume), np.uint8).copy()
        o.resume = rbuf.ctypes.data
    if checkpoint is not None:
        assert checkpoint.dtype == np.uint8 and checkpoint.size >= checkpoint_bytes(prob, kind)
        o.checkpoint = checkpoint.ctypes.data
    o.filter_type = filter_type
    o.conv_eps = conv_eps
    o.conv_min_steps = conv_min_steps
    if steps_done is not None:
        o.steps_done = _p(steps_done, _ip)
    keep = []
    for name, m in (("nondesign", nondesign), ("volume_set", volume_set)):
        if m is not None:
            a = np.ascontiguousarray(m, np.uint8)
            keep.append(a)
            setattr(o, name, _p(a, _u8p))
    if on_step is not None:
        nel, neq = prob.nel, prob.neq

        def _cb(_u, step, comp, rho, nv, mi):
            on_step(step, comp, np.ctypeslib.as_array(rho, (nel,)).copy(),
                    np.ctypeslib.as_array(nv, (neq,)).copy(),
                    np.ctypeslib.as_array(mi, (nel,)).copy())
        o.on_step = STEP_CB(_cb)
        keep.append(o.on_step)
    hist = np.zeros(nsteps)
    x = np.zeros(prob.nel)
    rho0 = None if rho0 is None else np.ascontiguousarray(rho0, np.float64)
    f = lib().icb_run_oc if kind == "oc" else lib().icb_run_mma
    check(f(prob.h, C.byref(o), None if rho0 is None else _p(rho0), _p(hist), _p(x)))
    return hist, x


def checkpoint_bytes(prob, kind):
    """icb_loop_checkpoint_bytes for kind "oc" or "mma"."""
    return lib().icb_loop_checkpoint_bytes(prob.h, 0 if kind == "oc" else 1)


# ------------------------------------------------------------ batch/serve --
def loop_opts(nsteps, radius, move=0.15, use_threshold=True, volume_ref=0.0, precision=FP64,
              precond=GMG, tol=1e-8, maxit=20000):
    return LoopOpts(nsteps, radius, move, int(use_threshold), volume_ref,
                    SolveOpts(precision, precond, tol, maxit, 0.0, 0, 0), None)


def run_batch(probs, kinds, opts, rho0s, nworkers):
    """icb_run_batch: returns (hists, xs, statuses)."""
    n = len(probs)
    H = [np.zeros(o.nsteps) for o in opts]
    X = [np.zeros(p.nel) for p in probs]
    R = [np.ascontiguousarray(r, np.float64) for r in rho0s]
    ph = (C.c_void_p * n)(*[p.h.value for p in probs])
    kk = np.asarray(kinds, np.int32)
    oo = (LoopOpts * n)(*opts)
    rr = (_dp * n)(*[_p(r) for r in R])
    hh = (_dp * n)(*[_p(h) for h in H])
    xx = (_dp * n)(*[_p(x) for x in X])
    st = np.zeros(n, np.int32)
    rc = lib().icb_run_batch(n, ph, _p(kk, _ip), oo, rr, hh, xx, nworkers, _p(st, _ip))
    check(rc)
    return H, X, st


def job_footprint(grid, kind):
    """icb_job_footprint: device bytes one run of this grid needs."""
    return lib().icb_job_footprint(C.byref(grid), kind)


def shard_by_footprint(footprints, nshards):
    """Split jobs over GPUs with no exchange between them: longest-first
    greedy assignment to the least-loaded shard (by device footprint, a proxy
    for work).  Returns one sorted index list per shard; every rank computes
    the same split from the same list."""
    loads = [0] * nshards
    shards = [[] for _ in range(nshards)]
    for i in sorted(range(len(footprints)), key=lambda k: (-footprints[k], k)):
        r = min(range(nshards), key=lambda k: (loads[k], k))
        shards[r].append(i)
        loads[r] += footprints[i]
    return [sorted(s) for s in shards]


class Server:
    """icb_server: continuous batching of app-loop jobs on one GPU."""

    def __init__(self, device=0, budget_bytes=150 << 30, slots=8):
        h = C.c_void_p()
        check(lib().icb_server_create(device, int(budget_bytes), slots, C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, grid, kind, loop, fixed, load, rho0):
        fixed = np.ascontiguousarray(fixed, np.uint8)
        load = np.ascontiguousarray(load, np.float64)
        rho0 = np.ascontiguousarray(rho0, np.float64)
        jd = JobDesc(grid, kind, loop, _p(fixed, _u8p), _p(load), _p(rho0))
        jid = C.c_longlong()
        check(lib().icb_server_submit(self.h, C.byref(jd), C.byref(jid)))
        self._keep[jid.value] = (loop.nsteps, grid)
        return jid.value

    def wait(self, jid, timeout=-1.0):
        info = JobInfo()
        rc = lib().icb_server_wait(self.h, jid, timeout, C.byref(info))
        return rc, info

    def result(self, jid):
        nsteps, grid = self._keep[jid]
        nel = grid.nx * grid.ny * (grid.nz if grid.dim == 3 else 1)
        hist, x, it = np.zeros(nsteps), np.zeros(nel), np.zeros(nsteps)
        check(lib().icb_server_result(self.h, jid, _p(hist), _p(x), _p(it)))
        return hist, x, it

    def cancel(self, jid):
        return lib().icb_server_cancel(self.h, jid)

    def forget(self, jid):
        self._keep.pop(jid, None)
        return lib().icb_server_forget(self.h, jid)

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.icb_server_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()
