"""ctypes wrapper of the oracle libraries -- TEST INFRASTRUCTURE ONLY.

Oracle(...)      oracle/_build/libemu_oracle.so  (C restatement, emu_oracle.c)
RefHarness(nf)   oracle/_ref/libemuref<nf>.so    (the reference's generated
                                                 kernel bodies, ref_harness.cpp)
RefInit()        oracle/_ref/libemurefinit.so    (the reference's direction-set
                                                 and Minerbo helpers)

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libemu_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libemuref%d.so")

_D = ctypes.POINTER(ctypes.c_double)


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("nflavors", ctypes.c_int), ("shape_order", ctypes.c_int), ("ncell", ctypes.c_int * 3),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
        ("rho", ctypes.c_double), ("Ye", ctypes.c_double), ("T", ctypes.c_double),
        ("mass1", ctypes.c_double), ("mass2", ctypes.c_double), ("mass3", ctypes.c_double),
        ("theta12", ctypes.c_double), ("theta13", ctypes.c_double), ("theta23", ctypes.c_double),
        ("alpha1", ctypes.c_double), ("alpha2", ctypes.c_double), ("deltaCP", ctypes.c_double),
        ("cfl_factor", ctypes.c_double), ("flavor_cfl_factor", ctypes.c_double),
        ("max_adaptive_speedup", ctypes.c_double), ("maxError", ctypes.c_double),
    ]


def oracle_params(p):
    """OracleParams from an emu_b200.api.EmuParams (or any object with the
    same field names)."""
    o = OracleParams()
    o.nflavors = p.nflavors
    o.shape_order = p.shape_order
    for i in range(3):
        o.ncell[i] = p.ncell[i]
    o.Lx, o.Ly, o.Lz = p.Lx, p.Ly, p.Lz
    o.rho, o.Ye, o.T = p.rho_in, p.Ye_in, p.T_in
    o.mass1, o.mass2, o.mass3 = p.mass1, p.mass2, p.mass3
    o.theta12, o.theta13, o.theta23 = p.theta12, p.theta13, p.theta23
    o.alpha1, o.alpha2, o.deltaCP = p.alpha1, p.alpha2, p.deltaCP
    o.cfl_factor, o.flavor_cfl_factor = p.cfl_factor, p.flavor_cfl_factor
    o.max_adaptive_speedup, o.maxError = p.max_adaptive_speedup, p.maxError
    return o


def _ptr(a):
    return a.ctypes.data_as(_D)


class _Base:
    prefix = "oracle_"

    def __init__(self, path, params):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with `python oracle/build_oracle.py`)")
        self.lib = ctypes.CDLL(path)
        self.P = oracle_params(params)
        self.nf = params.nflavors
        self.nreal = 3 + 8 + 2 * (2 + self.nf * self.nf)
        self.ncomp = 3 + 8 * self.nf * self.nf
        self.ncells = params.ncell[0] * params.ncell[1] * params.ncell[2]

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def new_mesh(self):
        m = np.zeros(self.ncomp * self.ncells)
        nc = self.ncells
        m[0:nc] = self.P.rho
        m[nc:2 * nc] = self.P.T
        m[2 * nc:3 * nc] = self.P.Ye
        return m

    def deposit(self, parts, nthreads=1, mesh=None):
        parts = np.ascontiguousarray(parts, dtype=np.float64)
        mesh = self.new_mesh() if mesh is None else mesh
        f = self._f("deposit")
        f.argtypes = [ctypes.POINTER(OracleParams), _D, ctypes.c_int64, _D, ctypes.c_int]
        f(ctypes.byref(self.P), _ptr(parts), parts.shape[0], _ptr(mesh), nthreads)
        return mesh

    def interpolate_rhs(self, mesh, parts, nthreads=1):
        parts = np.ascontiguousarray(parts, dtype=np.float64)
        out = np.zeros_like(parts)
        f = self._f("interpolate_rhs")
        f.argtypes = [ctypes.POINTER(OracleParams), _D, _D, ctypes.c_int64, _D, ctypes.c_int]
        f(ctypes.byref(self.P), _ptr(mesh), _ptr(parts), parts.shape[0], _ptr(out), nthreads)
        return out

    def renormalize(self, parts):
        parts = np.array(parts, dtype=np.float64, copy=True)
        bad = ctypes.c_int64(-1)
        f = self._f("renormalize")
        f.argtypes = [ctypes.POINTER(OracleParams), _D, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        f.restype = ctypes.c_int
        st = f(ctypes.byref(self.P), _ptr(parts), parts.shape[0], ctypes.byref(bad))
        return parts, st, bad.value

    def compute_dt(self, mesh, vvac_max):
        dt = ctypes.c_double(0)
        f = self._f("compute_dt")
        f.argtypes = [ctypes.POINTER(OracleParams), _D, ctypes.c_double, _D]
        f.restype = ctypes.c_int
        st = f(ctypes.byref(self.P), _ptr(mesh), vvac_max, ctypes.byref(dt))
        return dt.value, st

    def vvac_max(self, parts):
        parts = np.ascontiguousarray(parts, dtype=np.float64)
        f = self._f("vvac_max")
        f.argtypes = [ctypes.POINTER(OracleParams), _D, ctypes.c_int64]
        f.restype = ctypes.c_double
        return f(ctypes.byref(self.P), _ptr(parts), parts.shape[0])

    def rk_step(self, parts, dt, rk_type=4, nthreads=1):
        """One integrator step in place; returns (mesh after the step, status, bad)."""
        assert parts.flags.c_contiguous and parts.dtype == np.float64
        mesh = self.new_mesh()
        scratch = np.zeros(5 * parts.size)
        bad = ctypes.c_int64(-1)
        f = self._f("rk_step")
        f.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int, _D, ctypes.c_int64, ctypes.c_double, _D, _D,
                      ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
        f.restype = ctypes.c_int
        st = f(ctypes.byref(self.P), rk_type, _ptr(parts), parts.shape[0], dt, _ptr(mesh), _ptr(scratch),
               nthreads, ctypes.byref(bad))
        return mesh, st, bad.value

    def evolve(self, parts, nsteps, end_time=float("inf"), rk_type=4, nthreads=1, start_time=0.0):
        """The evolve_flavor loop (main.cpp:118-213): deposit, dt from the
        initial mesh, then steps with dt from each step's last stage mesh and
        the step clipped to land on end_time.  Returns (parts, t, dts, status)."""
        parts = np.array(parts, dtype=np.float64, copy=True)
        vmax = self.vvac_max(parts)
        mesh = self.deposit(parts, nthreads)
        dt, st = self.compute_dt(mesh, vmax)
        t = start_time
        dts = []
        status = st
        for _ in range(nsteps):
            last = False
            if end_time - t < dt:
                dt = end_time - t
                last = True
            mesh, s, _ = self.rk_step(parts, dt, rk_type, nthreads)
            status |= s
            t = t + dt
            dts.append(dt)
            if last:
                break
            dt, s = self.compute_dt(mesh, vmax)
            status |= s
        return parts, t, np.array(dts), status


class Oracle(_Base):
    prefix = "oracle_"

    def __init__(self, params):
        super().__init__(ORACLE_LIB, params)

    def shape(self, delta, order):
        first = ctypes.c_int(0)
        w = (ctypes.c_double * 3)()
        self.lib.oracle_shape.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.c_double * 3]
        self.lib.oracle_shape(delta, order, ctypes.byref(first), w)
        return first.value, np.array(list(w))

    def finish_step(self, parts):
        """end of step in place: periodic wrap + position sync, then
        Renormalize (main.cpp:163-170); returns the Renormalize status"""
        assert parts.flags.c_contiguous and parts.dtype == np.float64
        self.lib.oracle_wrap.argtypes = [ctypes.POINTER(OracleParams), _D, ctypes.c_int64]
        self.lib.oracle_wrap(ctypes.byref(self.P), _ptr(parts), parts.shape[0])
        bad = ctypes.c_int64(-1)
        f = self._f("renormalize")
        f.argtypes = [ctypes.POINTER(OracleParams), _D, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        f.restype = ctypes.c_int
        return f(ctypes.byref(self.P), _ptr(parts), parts.shape[0], ctypes.byref(bad))

    def vvac(self, pupt):
        V = np.zeros(2 * self.nf * self.nf)
        self.lib.oracle_vvac.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_double, _D]
        self.lib.oracle_vvac(ctypes.byref(self.P), pupt, _ptr(V))
        return V

    def su_length(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self.lib.oracle_su_length.argtypes = [ctypes.c_int, _D]
        self.lib.oracle_su_length.restype = ctypes.c_double
        return self.lib.oracle_su_length(self.nf, _ptr(f))


class RefHarness(_Base):
    prefix = "ref_"

    def __init__(self, params):
        super().__init__(REF_LIB % params.nflavors, params)
        self.lib.ref_nflavors.restype = ctypes.c_int
        assert self.lib.ref_nflavors() == params.nflavors

    def set_trace_length(self, parts):
        parts = np.array(parts, dtype=np.float64, copy=True)
        self.lib.ref_set_trace_length.argtypes = [_D, ctypes.c_int64]
        self.lib.ref_set_trace_length(_ptr(parts), parts.shape[0])
        return parts


def have_ref(nf):
    return os.path.exists(REF_LIB % nf)


REF_INIT_LIB = os.path.join(HERE, "_ref", "libemurefinit.so")


class RefInit:
    """The reference's initial-condition helpers (uniform_sphere_xyz,
    minerbo_Z, minerbo_closure of FlavoredNeutrinoContainerInit.cpp),
    compiled where they lie into oracle/_ref/libemurefinit.so."""

    def __init__(self):
        self.lib = ctypes.CDLL(REF_INIT_LIB)
        self.lib.refinit_uniform_sphere_xyz.argtypes = [ctypes.c_int, _D, ctypes.c_int]
        self.lib.refinit_uniform_sphere_xyz.restype = ctypes.c_int
        self.lib.refinit_minerbo_Z.argtypes = [ctypes.c_double]
        self.lib.refinit_minerbo_Z.restype = ctypes.c_double
        self.lib.refinit_minerbo_closure.argtypes = [ctypes.c_double, ctypes.c_double]
        self.lib.refinit_minerbo_closure.restype = ctypes.c_double

    def uniform_sphere_xyz(self, nphi):
        n = self.lib.refinit_uniform_sphere_xyz(nphi, ctypes.cast(None, _D), 0)
        out = np.zeros((n, 3))
        self.lib.refinit_uniform_sphere_xyz(nphi, _ptr(out), n)
        return out

    def minerbo_Z(self, fluxfac):
        return self.lib.refinit_minerbo_Z(fluxfac)

    def minerbo_closure(self, Z, mu):
        return self.lib.refinit_minerbo_closure(Z, mu)


def have_ref_init():
    return os.path.exists(REF_INIT_LIB)
