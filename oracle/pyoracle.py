"""ctypes front-end of the oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/lib/liboracle.so`` (the CPU restatement of ICARAT's SIMP step,
see ``oracle.cpp``) and, when it was built, ``oracle/_ref/libref_opt.so``
(ICARAT's own OC/MMA compiled from its sources).  Only the tests, the smoke
check and the CPU-baseline legs of ``bench.py`` import this module, always as
the checker; the product library never does.

Parity status: the FEM solve is unpinned by reference-run outputs (ICARAT's
solve needs Eigen/toml11, absent here); it is pinned by published closed-form
element matrices and independent quadratures (elastic and heat), a direct
factorisation and ICARAT's own finite-difference procedure.  OC, MMA and GCMMA
are pinned against ICARAT's own sources.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_opt.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)
_i64p = C.POINTER(C.c_int64)
VOLUME_CB = C.CFUNCTYPE(C.c_double, _dp, C.c_void_p)


class OrcGrid(C.Structure):
    """Mirror of ``struct OrcGrid`` in oracle.cpp."""
    _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("state", C.c_int), ("young1", C.c_double), ("young2", C.c_double),
                ("nu", C.c_double), ("penal", C.c_double)]


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        G = C.POINTER(OrcGrid)
        sig = {
            "orc_numnp": (C.c_int64, [G]),
            "orc_nelx": (C.c_int64, [G]),
            "orc_K0": (None, [G, _dp]),
            "orc_element_volume": (C.c_double, [G]),
            "orc_dirichlet_box": (None, [G, _ip, _dp, _dp, _u8p, _dp]),
            "orc_count_dof": (C.c_int64, [G, _u8p, _ip]),
            "orc_traction_box": (None, [G, _dp, _dp, _ip, C.c_int64, _dp]),
            "orc_simp": (None, [G, _dp, _dp]),
            "orc_csr_assemble": (C.c_void_p, [G, _ip, C.c_int64, _dp]),
            "orc_csr_free": (None, [C.c_void_p]),
            "orc_csr_nnz": (C.c_int64, [C.c_void_p]),
            "orc_csr_export": (None, [C.c_void_p, _i64p, _ip, _dp]),
            "orc_csr_spmv": (None, [C.c_void_p, _dp, _dp]),
            "orc_csr_pcg": (C.c_int, [C.c_void_p, _dp, _dp, C.c_double, C.c_int, _ip, _dp, _ip]),
            "orc_csr_pcg_fixed": (C.c_double, [C.c_void_p, _dp, _dp, C.c_int]),
            "orc_linear_solve": (C.c_int, [G, _u8p, _dp, _ip, C.c_int64, _dp, _dp, C.c_double,
                                           C.c_int, _dp, _dp, _dp, _ip, _dp, _ip]),
            "orc_sensitivity": (None, [G, _dp, _dp, _dp]),
            "orc_cone_create": (C.c_void_p, [G, C.c_double]),
            "orc_cone_free": (None, [C.c_void_p]),
            "orc_cone_size": (C.c_int, [C.c_void_p]),
            "orc_cone_apply": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
            "orc_cone_bruteforce_counts": (C.c_int64, [G, C.c_double, _ip]),
            "orc_threshold": (None, [C.c_int64, _dp, C.c_double, C.c_double, _dp]),
            "orc_threshold_deriv": (None, [C.c_int64, _dp, C.c_double, C.c_double, _dp]),
            "orc_helmholtz": (C.c_int, [G, C.c_double, _dp, _dp, C.c_int, C.c_double, _ip]),
            "orc_oc_update": (C.c_int, [C.c_int64, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                        C.c_double, VOLUME_CB, C.c_void_p]),
            "orc_mma_create": (C.c_void_p, [C.c_int64, C.c_int, C.c_double, C.c_double, C.c_double]),
            "orc_mma_free": (None, [C.c_void_p]),
            "orc_mma_update": (None, [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_oc_loop": (C.c_int, [G, _u8p, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double,
                                      C.c_int, C.c_double, _dp, _dp, _ip]),
            "orc_mma_loop": (C.c_int, [G, _u8p, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double,
                                       C.c_double, _dp, _dp]),
            "orc_von_mises": (None, [G, _dp, _dp, _dp, _dp]),
            "orc_reactions": (None, [G, _dp, _dp, _dp]),
            "orc_mma_cone_loop": (C.c_int, [G, _u8p, _dp, _dp, _dp, C.c_int, C.c_double, _u8p,
                                            _u8p, C.c_double, _dp, _dp]),
            "orc_gcmma_create": (C.c_void_p, [C.c_int64, C.c_int, C.c_double, C.c_double,
                                              C.c_double]),
            "orc_gcmma_free": (None, [C.c_void_p]),
            "orc_gcmma_outer": (None, [C.c_void_p, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp, _dp]),
            "orc_gcmma_inner": (None, [C.c_void_p, _dp, C.c_double, _dp, _dp, C.c_double, _dp, _dp,
                                       _dp, _dp, _dp]),
            "orc_gcmma_concheck": (C.c_int, [C.c_void_p, C.c_double, _dp]),
            "orc_gcmma_loop": (C.c_int, [G, _u8p, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double,
                                         _dp, _ip, _dp]),
            "orc_heat_Ke": (None, [G, _dp, _dp, _dp, _dp]),
            "orc_heat_solve": (C.c_int, [G, _dp, _dp, _u8p, _dp, _dp, _dp, C.c_double, _dp, _dp,
                                         _ip]),
            "orc_heat_sensitivity": (None, [G, _dp, _dp, _dp, _dp, _dp]),
            "orc_heat_loop": (C.c_int, [G, _dp, _dp, _u8p, _dp, _dp, _dp, C.c_int, C.c_double,
                                        C.c_double, _dp, _dp]),
            "orc_ebe_pcg_time": (C.c_double, [G, _u8p, _dp, _dp, C.c_int, _dp]),
            "orc_num_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    """ICARAT's own OC/MMA (compiled from its sources into oracle/_ref)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref not built (needs the ICARAT source tree)")
        L = C.CDLL(REF_PATH)
        L.ref_oc_update.restype = None
        L.ref_oc_update.argtypes = [C.c_int, _dp, _dp, C.c_double, _dp, _dp, _dp, C.c_double,
                                    VOLUME_CB, C.c_void_p]
        L.ref_mma_create.restype = C.c_void_p
        L.ref_mma_create.argtypes = [C.c_int, C.c_int]
        L.ref_mma_update.restype = None
        L.ref_mma_update.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_mma_free.restype = None
        L.ref_mma_free.argtypes = [C.c_void_p]
        L.ref_gcmma_create.restype = C.c_void_p
        L.ref_gcmma_create.argtypes = [C.c_int, C.c_int]
        L.ref_gcmma_outer.restype = None
        L.ref_gcmma_outer.argtypes = [C.c_void_p, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp, _dp]
        L.ref_gcmma_inner.restype = None
        L.ref_gcmma_inner.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp, C.c_double, _dp, _dp,
                                      _dp, _dp, _dp]
        L.ref_gcmma_concheck.restype = C.c_int
        L.ref_gcmma_concheck.argtypes = [C.c_void_p, C.c_double, _dp]
        L.ref_gcmma_free.restype = None
        L.ref_gcmma_free.argtypes = [C.c_void_p]
        _ref = L
    return _ref


# ----------------------------------------------------------------- helpers --
class Problem:
    """A structured SIMP problem held as numpy arrays for the oracle.

    ``fixed``/``dval``: per DOF (node-major, interleaved) Dirichlet flag/value.
    ``fext_full``: full-grid nodal load (node-major, interleaved); loads on
    constrained DOFs are dropped when mapped to the numeq vector, as
    SurfaceLoad::generate does.
    """

    def __init__(self, dim, nx, ny, nz=1, lx=None, ly=None, lz=None, state=None,
                 young=(1e-9, 1.0), nu=0.3, penal=3.0):
        self.g = OrcGrid(dim, nx, ny, nz if dim == 3 else 1,
                         float(lx if lx is not None else nx), float(ly if ly is not None else ny),
                         float(lz if lz is not None else (nz if dim == 3 else 1)),
                         (2 if dim == 3 else 0) if state is None else state,
                         float(young[0]), float(young[1]), float(nu), float(penal))
        self.dim = dim
        self.nnode = int(lib().orc_numnp(C.byref(self.g)))
        self.nel = int(lib().orc_nelx(C.byref(self.g)))
        self.dofnp = 1 if state == 3 else dim  # heat conduction: one DOF per node
        self.neq = self.nnode * self.dofnp
        self.fixed = np.zeros(self.neq, np.uint8)
        self.dval = np.zeros(self.neq)
        self.fext_full = np.zeros(self.neq)
        self._extra_numeq_load = []

    # boundary conditions ------------------------------------------------
    def dirichlet_box(self, flag, val, rng):
        f = np.asarray(list(flag) + [0] * (6 - len(flag)), np.int32)
        v = np.asarray(list(val) + [0.0] * (6 - len(val)), np.float64)
        r = np.asarray(rng, np.float64).reshape(6)
        lib().orc_dirichlet_box(C.byref(self.g), _ptr(f, _ip), _ptr(v), _ptr(r),
                                _ptr(self.fixed, _u8p), _ptr(self.dval))

    def traction_box(self, val, rng):
        self._extra_numeq_load.append((np.asarray(val, np.float64), np.asarray(rng, np.float64).reshape(6)))

    def dofs(self):
        dof = np.zeros(self.neq, np.int32)
        numeq = int(lib().orc_count_dof(C.byref(self.g), _ptr(self.fixed, _u8p), _ptr(dof, _ip)))
        return dof, numeq

    def fext(self):
        """numeq load vector: nodal loads on free DOFs plus traction boxes."""
        dof, numeq = self.dofs()
        f = np.zeros(numeq)
        free = dof < numeq
        np.add.at(f, dof[free], self.fext_full[free])
        for val, rng in self._extra_numeq_load:
            v3 = np.zeros(3)
            v3[:len(val)] = val
            lib().orc_traction_box(C.byref(self.g), _ptr(v3), _ptr(rng), _ptr(dof, _ip),
                                   numeq, _ptr(f))
        return f

    # operators ----------------------------------------------------------
    def K0(self):
        nd = self.dim * (4 if self.dim == 2 else 8)
        K = np.zeros((nd, nd))
        lib().orc_K0(C.byref(self.g), _ptr(K))
        return K

    def element_volume(self):
        return lib().orc_element_volume(C.byref(self.g))

    def assemble(self, rho):
        dof, numeq = self.dofs()
        rho = np.ascontiguousarray(rho, np.float64)
        h = lib().orc_csr_assemble(C.byref(self.g), _ptr(dof, _ip), numeq, _ptr(rho))
        nnz = lib().orc_csr_nnz(h)
        rp = np.zeros(numeq + 1, np.int64)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        lib().orc_csr_export(h, _ptr(rp, _i64p), _ptr(col, _ip), _ptr(val))
        lib().orc_csr_free(h)
        return rp, col, val

    def solve(self, rho, tol=1e-8, maxit=100000):
        dof, numeq = self.dofs()
        f = self.fext()
        rho = np.ascontiguousarray(rho, np.float64)
        u = np.zeros(numeq)
        nv = np.zeros(self.neq)
        comp = C.c_double()
        it = C.c_int()
        rr = C.c_double()
        mv = C.c_int()
        rc = lib().orc_linear_solve(C.byref(self.g), _ptr(self.fixed, _u8p), _ptr(self.dval),
                                    _ptr(dof, _ip), numeq, _ptr(f), _ptr(rho), tol, maxit,
                                    _ptr(u), _ptr(nv), C.byref(comp), C.byref(it), C.byref(rr),
                                    C.byref(mv))
        return dict(u=u, nodeval=nv, compliance=comp.value, iters=it.value, relres=rr.value,
                    matvecs=mv.value, rc=rc, dof=dof, numeq=numeq, f=f)

    def sensitivity(self, rho, nodeval):
        dc = np.zeros(self.nel)
        lib().orc_sensitivity(C.byref(self.g), _ptr(np.ascontiguousarray(rho, np.float64)),
                              _ptr(np.ascontiguousarray(nodeval)), _ptr(dc))
        return dc

    def simp(self, rho):
        E = np.zeros(self.nel)
        lib().orc_simp(C.byref(self.g), _ptr(np.ascontiguousarray(rho, np.float64)), _ptr(E))
        return E

    def helmholtz(self, R, x, sens=False, tol=1e-10):
        out = np.zeros(self.nel)
        it = C.c_int()
        lib().orc_helmholtz(C.byref(self.g), R, _ptr(np.ascontiguousarray(x, np.float64)),
                            _ptr(out), int(sens), tol, C.byref(it))
        return out

    def oc_loop(self, rho0, nsteps, rfil, movelimit, use_beta=True, tol=1e-8):
        hist = np.zeros(nsteps)
        x = np.zeros(self.nel)
        tot = C.c_int()
        lib().orc_oc_loop(C.byref(self.g), _ptr(self.fixed, _u8p), _ptr(self.dval),
                          _ptr(self.fext()), _ptr(np.ascontiguousarray(rho0, np.float64)), nsteps,
                          rfil, movelimit, int(use_beta), tol, _ptr(hist), _ptr(x), C.byref(tot))
        return hist, x, tot.value

    def von_mises(self, rho, nodeval, with_stress=False):
        """Element von Mises stress (and the nel x voigt stress) of a solution."""
        m = np.zeros(self.nel)
        v = 3 if self.dim == 2 else 6
        st = np.zeros(self.nel * v) if with_stress else None
        lib().orc_von_mises(C.byref(self.g), _ptr(np.ascontiguousarray(rho, np.float64)),
                            _ptr(np.ascontiguousarray(nodeval, np.float64)), _ptr(m),
                            None if st is None else _ptr(st))
        return (m, st.reshape(self.nel, v)) if with_stress else m

    def reactions(self, rho, nodeval):
        """Internal force sum_e Ke u_e at every DOF, node-major (neq)."""
        r = np.zeros(self.neq)
        lib().orc_reactions(C.byref(self.g), _ptr(np.ascontiguousarray(rho, np.float64)),
                            _ptr(np.ascontiguousarray(nodeval, np.float64)), _ptr(r))
        return r

    def mma_cone_loop(self, rho0, nsteps, rfil, nondesign=None, volset=None, tol=1e-8):
        hist = np.zeros(nsteps)
        x = np.zeros(self.nel)
        nd = None if nondesign is None else np.ascontiguousarray(nondesign, np.uint8)
        vs = None if volset is None else np.ascontiguousarray(volset, np.uint8)
        lib().orc_mma_cone_loop(C.byref(self.g), _ptr(self.fixed, _u8p), _ptr(self.dval),
                                _ptr(self.fext()), _ptr(np.ascontiguousarray(rho0, np.float64)),
                                nsteps, rfil, None if nd is None else _ptr(nd, _u8p),
                                None if vs is None else _ptr(vs, _u8p), tol, _ptr(hist), _ptr(x))
        return hist, x

    def ebe_pcg_time(self, rho, nit):
        """Seconds of nit matrix-free Jacobi-PCG iterations on the host cores."""
        rr = C.c_double()
        t = lib().orc_ebe_pcg_time(C.byref(self.g), _ptr(self.fixed, _u8p),
                                   _ptr(np.ascontiguousarray(rho, np.float64)),
                                   _ptr(np.ascontiguousarray(self.fext_full, np.float64)), nit,
                                   C.byref(rr))
        return t, rr.value

    # heat conduction (state 3) ------------------------------------------
    def heat_Ke(self, cond1, cond2):
        ne = 4 if self.dim == 2 else 8
        K1, K2 = np.zeros((ne, ne)), np.zeros((ne, ne))
        lib().orc_heat_Ke(C.byref(self.g), _ptr(np.asarray(cond1, np.float64)),
                          _ptr(np.asarray(cond2, np.float64)), _ptr(K1), _ptr(K2))
        return K1, K2

    def heat_solve(self, cond1, cond2, rho, tol=1e-10):
        nv = np.zeros(self.nnode)
        obj = C.c_double()
        it = C.c_int()
        rc = lib().orc_heat_solve(C.byref(self.g), _ptr(np.asarray(cond1, np.float64)),
                                  _ptr(np.asarray(cond2, np.float64)), _ptr(self.fixed, _u8p),
                                  _ptr(self.dval), _ptr(self.fext()),
                                  _ptr(np.ascontiguousarray(rho, np.float64)), tol, _ptr(nv),
                                  C.byref(obj), C.byref(it))
        return {"nodeval": nv, "objective": obj.value, "iters": it.value, "rc": rc}

    def heat_sensitivity(self, cond1, cond2, rho, nodeval):
        dc = np.zeros(self.nel)
        lib().orc_heat_sensitivity(C.byref(self.g), _ptr(np.asarray(cond1, np.float64)),
                                   _ptr(np.asarray(cond2, np.float64)),
                                   _ptr(np.ascontiguousarray(rho, np.float64)),
                                   _ptr(np.ascontiguousarray(nodeval, np.float64)), _ptr(dc))
        return dc

    def heat_loop(self, cond1, cond2, rho0, nsteps, R, tol=1e-10):
        hist, x = np.zeros(nsteps), np.zeros(self.nel)
        lib().orc_heat_loop(C.byref(self.g), _ptr(np.asarray(cond1, np.float64)),
                            _ptr(np.asarray(cond2, np.float64)), _ptr(self.fixed, _u8p),
                            _ptr(self.dval), _ptr(self.fext()),
                            _ptr(np.ascontiguousarray(rho0, np.float64)), nsteps, R, tol,
                            _ptr(hist), _ptr(x))
        return hist, x

    def gcmma_loop(self, rho0, nsteps, rfil, tol=1e-8):
        hist = np.zeros(nsteps)
        inner = np.zeros(nsteps, np.int32)
        x = np.zeros(self.nel)
        lib().orc_gcmma_loop(C.byref(self.g), _ptr(self.fixed, _u8p), _ptr(self.dval),
                             _ptr(self.fext()), _ptr(np.ascontiguousarray(rho0, np.float64)),
                             nsteps, rfil, tol, _ptr(hist), _ptr(inner, _ip), _ptr(x))
        return hist, inner, x

    def mma_loop(self, rho0, nsteps, R, Vref=0.0, tol=1e-8):
        hist = np.zeros(nsteps)
        x = np.zeros(self.nel)
        lib().orc_mma_loop(C.byref(self.g), _ptr(self.fixed, _u8p), _ptr(self.dval),
                           _ptr(self.fext()), _ptr(np.ascontiguousarray(rho0, np.float64)), nsteps,
                           R, Vref, tol, _ptr(hist), _ptr(x))
        return hist, x


class Cone:
    """Filter<E,N> density filter with its cached ``aa`` (forward then adjoint)."""

    def __init__(self, prob, r):
        self.p = prob
        self.h = lib().orc_cone_create(C.byref(prob.g), r)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_cone_free(self.h)
            self.h = None

    def size(self):
        return lib().orc_cone_size(self.h)

    def apply(self, x, sens=False):
        out = np.zeros(self.p.nel)
        lib().orc_cone_apply(self.h, _ptr(np.ascontiguousarray(x, np.float64)), _ptr(out), int(sens))
        return out


def threshold(x, beta, T=0.5):
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros_like(x)
    lib().orc_threshold(x.size, _ptr(x), beta, T, _ptr(out))
    return out


def threshold_deriv(x, beta, T=0.5):
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros_like(x)
    lib().orc_threshold_deriv(x.size, _ptr(x), beta, T, _ptr(out))
    return out


def oc_update(x, dfdx, g, dgdx, xmin, xmax, movelimit, volume_fn, use_ref=False):
    """One OC update; ``volume_fn(xkp1: ndarray) -> float`` is the callback."""
    n = x.size
    x = np.array(x, np.float64)

    def _cb(p, _ud):
        return float(volume_fn(np.ctypeslib.as_array(p, shape=(n,)).copy()))

    cb = VOLUME_CB(_cb)
    args = (_ptr(x), _ptr(np.ascontiguousarray(dfdx, np.float64)), float(g),
            _ptr(np.ascontiguousarray(dgdx, np.float64)), _ptr(np.ascontiguousarray(xmin, np.float64)),
            _ptr(np.ascontiguousarray(xmax, np.float64)), float(movelimit), cb, None)
    if use_ref:
        ref().ref_oc_update(n, *args)
    else:
        lib().orc_oc_update(n, *args)
    return x


class MMA:
    """MMA update; ``use_ref`` selects ICARAT's own MMASolver (oracle/_ref)."""

    def __init__(self, n, m=1, use_ref=False):
        self.n, self.m, self.use_ref = n, m, use_ref
        if use_ref:
            self.h = ref().ref_mma_create(n, m)
        else:
            self.h = lib().orc_mma_create(n, m, 0.0, 1e5, 0.0)

    def __del__(self):
        if getattr(self, "h", None):
            (ref().ref_mma_free if self.use_ref else lib().orc_mma_free)(self.h)
            self.h = None

    def update(self, x, dfdx, gx, dgdx, xmin, xmax):
        x = np.array(x, np.float64)
        a = [np.ascontiguousarray(v, np.float64) for v in (dfdx, np.atleast_1d(gx), dgdx, xmin, xmax)]
        f = ref().ref_mma_update if self.use_ref else lib().orc_mma_update
        f(self.h, _ptr(x), *[_ptr(v) for v in a])
        return x


class GCMMA:
    """GCMMA outer / inner updates and ConCheck; ``use_ref`` selects ICARAT's
    own GCMMASolver (oracle/_ref)."""

    def __init__(self, n, m=1, use_ref=False):
        self.n, self.m, self.use_ref = n, m, use_ref
        self.h = ref().ref_gcmma_create(n, m) if use_ref else lib().orc_gcmma_create(
            n, m, 0.0, 1000.0, 0.0)

    def __del__(self):
        if getattr(self, "h", None):
            (ref().ref_gcmma_free if self.use_ref else lib().orc_gcmma_free)(self.h)
            self.h = None

    def _L(self):
        return ref() if self.use_ref else lib()

    def outer(self, xval, f0x, df0dx, fx, dfdx, xmin, xmax):
        xmma = np.zeros(self.n)
        a = [np.ascontiguousarray(v, np.float64) for v in (xval, df0dx, np.atleast_1d(fx), dfdx,
                                                           xmin, xmax)]
        f = self._L().ref_gcmma_outer if self.use_ref else lib().orc_gcmma_outer
        f(self.h, _ptr(xmma), _ptr(a[0]), float(f0x), *[_ptr(v) for v in a[1:]])
        return xmma

    def inner(self, xmma, f0xnew, fxnew, xval, f0x, df0dx, fx, dfdx, xmin, xmax):
        xmma = np.array(xmma, np.float64)
        a = [np.ascontiguousarray(v, np.float64) for v in (np.atleast_1d(fxnew), xval, df0dx,
                                                           np.atleast_1d(fx), dfdx, xmin, xmax)]
        f = self._L().ref_gcmma_inner if self.use_ref else lib().orc_gcmma_inner
        f(self.h, _ptr(xmma), float(f0xnew), _ptr(a[0]), _ptr(a[1]), float(f0x),
          *[_ptr(v) for v in a[2:]])
        return xmma

    def concheck(self, f0xnew, fxnew):
        fx = np.ascontiguousarray(np.atleast_1d(fxnew), np.float64)
        f = self._L().ref_gcmma_concheck if self.use_ref else lib().orc_gcmma_concheck
        return bool(f(self.h, float(f0xnew), _ptr(fx)))
