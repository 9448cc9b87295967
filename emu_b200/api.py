"""Python binding of the C ABI in include/emu_b200.h (ctypes, numpy).

The library is the CUDA implementation; there is no CPU fallback.  Loading
fails loudly when libemu_b200.so is missing, and every device call raises
EmuError when the library reports a failure.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libemu_b200.so")

EMU_OK = 0
EMU_ERR_TRACE = 1
EMU_ERR_NEGDIAG = 2
EMU_ERR_LENGTH = 4
EMU_ERR_DT = 8
EMU_ERR_ARG = 16
EMU_ERR_CUDA = 32
EMU_ERR_STATE = 64
EMU_ERR_IO = 128
EMU_ERR_PARSE = 256
EMU_ERR_NOMEM = 512
EMU_ERR_LIMIT = 1024
EMU_ERR_TIMEOUT = 2048

PREC_FP64 = 0
PREC_MIXED = 1

# physical constants of Source/Constants.H
EV = 1.60218e-12
CLIGHT = 2.99792458e10
HBAR = 1.05457266e-27
MP = 1.6726219e-24
HBARC = HBAR * CLIGHT
GF = 1.1663787e-5 / (1e9 * 1e9 * EV * EV) * HBARC * HBARC * HBARC


class EmuParams(ctypes.Structure):
    """Mirror of struct emu_params (include/emu_b200.h)."""
    _fields_ = [
        ("nflavors", ctypes.c_int), ("shape_order", ctypes.c_int), ("precision", ctypes.c_int),
        ("integration_type", ctypes.c_int), ("rk_type", ctypes.c_int),
        ("ncell", ctypes.c_int * 3), ("nppc", ctypes.c_int * 3), ("nphi_equator", ctypes.c_int),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
        ("max_grid_size", ctypes.c_int), ("nsteps", ctypes.c_int), ("end_time", ctypes.c_double),
        ("write_plot_every", ctypes.c_int), ("write_plot_particles_every", ctypes.c_int),
        ("rho_in", ctypes.c_double), ("Ye_in", ctypes.c_double), ("T_in", ctypes.c_double),
        ("simulation_type", ctypes.c_int),
        ("cfl_factor", ctypes.c_double), ("flavor_cfl_factor", ctypes.c_double),
        ("max_adaptive_speedup", ctypes.c_double),
        ("do_restart", ctypes.c_int), ("restart_dir", ctypes.c_char * 512),
        ("maxError", ctypes.c_double),
        ("mass1", ctypes.c_double), ("mass2", ctypes.c_double), ("mass3", ctypes.c_double),
        ("theta12", ctypes.c_double), ("theta13", ctypes.c_double), ("theta23", ctypes.c_double),
        ("alpha1", ctypes.c_double), ("alpha2", ctypes.c_double), ("deltaCP", ctypes.c_double),
        ("st3_wavelength_fraction_of_domain", ctypes.c_int), ("st3_amplitude", ctypes.c_double),
        ("st4_ndens", ctypes.c_double), ("st4_theta", ctypes.c_double), ("st4_phi", ctypes.c_double),
        ("st4_fluxfac", ctypes.c_double),
        ("st4_ndensbar", ctypes.c_double), ("st4_thetabar", ctypes.c_double), ("st4_phibar", ctypes.c_double),
        ("st4_fluxfacbar", ctypes.c_double), ("st4_amplitude", ctypes.c_double),
        ("st5_nnue", ctypes.c_double), ("st5_nnua", ctypes.c_double), ("st5_nnux", ctypes.c_double),
        ("st5_fxnue", ctypes.c_double), ("st5_fxnua", ctypes.c_double), ("st5_fxnux", ctypes.c_double),
        ("st5_fynue", ctypes.c_double), ("st5_fynua", ctypes.c_double), ("st5_fynux", ctypes.c_double),
        ("st5_fznue", ctypes.c_double), ("st5_fznua", ctypes.c_double), ("st5_fznux", ctypes.c_double),
        ("st5_amplitude", ctypes.c_double),
        ("direction_generator", ctypes.c_int), ("ndirections", ctypes.c_int),
        ("seed", ctypes.c_uint64), ("resort_interval", ctypes.c_int), ("fused", ctypes.c_int),
    ]

    def copy(self):
        c = EmuParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(EmuParams))
        return c


class EmuRunInfo(ctypes.Structure):
    _fields_ = [("steps_done", ctypes.c_int), ("status", ctypes.c_int), ("bad_particle", ctypes.c_int64),
                ("time", ctypes.c_double), ("dt_next", ctypes.c_double)]


class EmuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("emu_b200 error %d: %s" % (code, msg))
        self.code = code


_P = ctypes.POINTER
_D = ctypes.POINTER(ctypes.c_double)
_lib = None

# every symbol declared in include/emu_b200.h with its ctypes signature
SIGNATURES = {
    "emu_abi_version": (ctypes.c_int, []),
    "emu_nattribs": (ctypes.c_int, [ctypes.c_int]),
    "emu_nreal": (ctypes.c_int, [ctypes.c_int]),
    "emu_ncomp": (ctypes.c_int, [ctypes.c_int]),
    "emu_params_default": (None, [_P(EmuParams)]),
    "emu_parse_inputs": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _P(ctypes.c_char_p), _P(EmuParams),
                                         ctypes.c_char_p, ctypes.c_size_t]),
    "emu_init_particles": (ctypes.c_int, [_P(EmuParams), _D, ctypes.c_int64, _P(ctypes.c_int64)]),
    "emu_vvac_max": (ctypes.c_int, [_P(EmuParams), _D, ctypes.c_int64, _D]),
    "emu_create": (ctypes.c_int, [_P(EmuParams), _P(ctypes.c_void_p)]),
    "emu_destroy": (None, [ctypes.c_void_p]),
    "emu_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "emu_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "emu_load_particles": (ctypes.c_int, [ctypes.c_void_p, _D, ctypes.c_int64]),
    "emu_get_particles": (ctypes.c_int, [ctypes.c_void_p, _D, ctypes.c_int64]),
    "emu_num_particles": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_int64)]),
    "emu_deposit": (ctypes.c_int, [ctypes.c_void_p]),
    "emu_get_mesh": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "emu_interpolate_rhs": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "emu_renormalize": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_int64)]),
    "emu_compute_dt": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "emu_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _P(ctypes.c_int64)]),
    "emu_evolve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  _P(EmuRunInfo)]),
    "emu_evolve_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "emu_evolve_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "emu_evolve_end": (ctypes.c_int, [ctypes.c_void_p, _P(EmuRunInfo)]),
    "emu_flush_l2": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]),
    "emu_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "emu_profile_step": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_float), ctypes.c_int, _P(ctypes.c_int)]),
    "emu_write_plotfile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int]),
    "emu_write_plotfile_host": (ctypes.c_int, [_P(EmuParams), ctypes.c_char_p, ctypes.c_double, ctypes.c_int,
                                               _D, _D, ctypes.c_int64]),
    "emu_read_particles": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _D, ctypes.c_int64,
                                          _P(ctypes.c_int64), _D, _P(ctypes.c_int)]),
    "emu_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "emu_deposit_noalloc": (ctypes.c_int, [_P(EmuParams), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "emu_init_particles_device": (ctypes.c_int, [ctypes.c_void_p]),
    "emu_comm_id": (ctypes.c_int, [ctypes.c_char_p]),
    "emu_attach_comm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "emu_local_group_create": (ctypes.c_int, [ctypes.c_int, _P(ctypes.c_void_p)]),
    "emu_attach_local": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "emu_local_group_destroy": (None, [ctypes.c_void_p]),
    "emu_adjoint_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, _D,
                                           _P(EmuRunInfo)]),
    "emu_adjoint_objective": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D]),
    "emu_adjoint_reserve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int)]),
    "emu_adjoint_backward": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D, _D]),
}


COMM_ID_BYTES = 128


class LocalGroup:
    """Ranks of the sharded schedule that are contexts of this process
    (emu_local_group_create): each rank's context is driven from its own
    thread.  Destroy (close) after every member context is closed."""

    def __init__(self, nranks):
        self.lib = load_library()
        h = ctypes.c_void_p()
        _check(self.lib.emu_local_group_create(int(nranks), ctypes.byref(h)), None, "emu_local_group_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.emu_local_group_destroy(self.h)
            self.h = None


_nccl_preloaded = False


def _preload_nccl():
    """Load the NCCL of the nvidia-nccl wheel (the one PyTorch links) before
    the library opens NCCL by its soname, so that one NCCL serves both: a
    system libnccl.so.2 found first would satisfy PyTorch's later load of the
    same soname and lack symbols PyTorch needs.  EMU_NCCL_LIBRARY names
    another NCCL explicitly."""
    global _nccl_preloaded
    if _nccl_preloaded:
        return
    _nccl_preloaded = True
    path = os.environ.get("EMU_NCCL_LIBRARY")
    if not path:
        import importlib.util
        try:
            spec = importlib.util.find_spec("nvidia.nccl")
        except (ImportError, ValueError):
            spec = None
        for d in (spec.submodule_search_locations if spec and spec.submodule_search_locations else []):
            cand = os.path.join(d, "lib", "libnccl.so.2")
            if os.path.exists(cand):
                path = cand
                break
    if path:
        ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)


def comm_id():
    """a new communicator id (bytes) for Context.attach_comm"""
    _preload_nccl()
    lib = load_library()
    buf = ctypes.create_string_buffer(COMM_ID_BYTES)
    _check(lib.emu_comm_id(buf), None, "emu_comm_id")
    return buf.raw


def load_library(path=None):
    """Load libemu_b200.so (built by emu_b200.build).  Raises if missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError("libemu_b200.so not found at %s; build it with `python -m emu_b200.build`" % p)
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _dptr(a):
    return a.ctypes.data_as(_D)


def last_error(ctx=None):
    lib = load_library()
    buf = ctypes.create_string_buffer(1024)
    lib.emu_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")


def _check(code, ctx=None, what=""):
    if code != EMU_OK:
        raise EmuError(code, (what + ": " if what else "") + last_error(ctx))
    return code


def default_params(**kw):
    """emu_params with the defaults of emu_params_default, set here without
    loading the library (the host-only benchmark legs build their workloads
    from these; tests pin the two byte for byte)."""
    p = EmuParams()
    ctypes.memset(ctypes.byref(p), 0, ctypes.sizeof(EmuParams))
    p.nflavors, p.shape_order, p.precision = 2, 2, PREC_FP64
    p.integration_type, p.rk_type = 1, 4
    for d in range(3):
        p.ncell[d] = 1
        p.nppc[d] = 1
    p.nphi_equator = 1
    p.Lx = p.Ly = p.Lz = 1.0
    p.max_grid_size = 64
    p.nsteps = 1
    p.end_time = 1.0
    p.write_plot_every = p.write_plot_particles_every = 1
    p.T_in, p.Ye_in = 10.0, 1.0
    p.cfl_factor = p.flavor_cfl_factor = 0.5
    p.maxError = 1e-6
    p.direction_generator, p.ndirections, p.seed = 0, 0, 0
    p.resort_interval, p.fused = -1, 1
    for k, v in kw.items():
        set_param(p, k, v)
    return p


def library_default_params():
    """emu_params_default of the library itself"""
    lib = load_library()
    p = EmuParams()
    lib.emu_params_default(ctypes.byref(p))
    return p


def set_param(p, key, value):
    if key in ("ncell", "nppc"):
        arr = getattr(p, key)
        for i in range(3):
            arr[i] = int(value[i])
    elif key == "restart_dir":
        p.restart_dir = value.encode() if isinstance(value, str) else value
    else:
        setattr(p, key, value)


def parse_inputs(path, overrides=()):
    lib = load_library()
    p = EmuParams()
    n = len(overrides)
    arr = (ctypes.c_char_p * max(n, 1))(*[o.encode() for o in overrides])
    err = ctypes.create_string_buffer(512)
    code = lib.emu_parse_inputs(path.encode() if path else None, n, arr, ctypes.byref(p), err, 512)
    if code != EMU_OK:
        raise EmuError(code, err.value.decode())
    return p


def nreal(nf):
    return 3 + 8 + 2 * (2 + nf * nf)


def ncomp(nf):
    return 3 + 8 * nf * nf


def init_particles(p):
    """InitParticles on the host: (n, nreal) FP64 particle records."""
    lib = load_library()
    n = ctypes.c_int64(0)
    _check(lib.emu_init_particles(ctypes.byref(p), None, 0, ctypes.byref(n)), None, "emu_init_particles")
    out = np.zeros((n.value, nreal(p.nflavors)), dtype=np.float64)
    _check(lib.emu_init_particles(ctypes.byref(p), _dptr(out), n.value, ctypes.byref(n)), None,
           "emu_init_particles")
    return out


def vvac_max(p, records):
    lib = load_library()
    out = ctypes.c_double(0)
    r = np.ascontiguousarray(records, dtype=np.float64)
    _check(lib.emu_vvac_max(ctypes.byref(p), _dptr(r), r.shape[0], ctypes.byref(out)))
    return out.value


def read_particles(plotfile_dir, nf):
    lib = load_library()
    n = ctypes.c_int64(0)
    t = ctypes.c_double(0)
    st = ctypes.c_int(0)
    _check(lib.emu_read_particles(plotfile_dir.encode(), nf, None, 0, ctypes.byref(n), None, None))
    out = np.zeros((n.value, nreal(nf)))
    _check(lib.emu_read_particles(plotfile_dir.encode(), nf, _dptr(out), n.value, ctypes.byref(n),
                                  ctypes.byref(t), ctypes.byref(st)))
    return out, t.value, st.value


class Context:
    """A device context: FlavoredNeutrinoContainer + mesh + integrator on one GPU."""

    def __init__(self, params):
        self.lib = load_library()
        self.params = params.copy()
        self.nf = params.nflavors
        h = ctypes.c_void_p()
        _check(self.lib.emu_create(ctypes.byref(self.params), ctypes.byref(h)), None, "emu_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.emu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, code, what):
        return _check(code, self.h, what)

    def set_stream(self, stream_handle):
        self._ck(self.lib.emu_set_stream(self.h, ctypes.c_void_p(stream_handle)), "emu_set_stream")

    def synchronize(self):
        self._ck(self.lib.emu_synchronize(self.h), "emu_synchronize")

    def load_particles(self, records):
        r = np.ascontiguousarray(records, dtype=np.float64)
        assert r.ndim == 2 and r.shape[1] == nreal(self.nf)
        self._ck(self.lib.emu_load_particles(self.h, _dptr(r), r.shape[0]), "emu_load_particles")

    def load_particles_ptr(self, ptr, n):
        """Load from a raw host pointer (pinned buffers)."""
        self._ck(self.lib.emu_load_particles(self.h, ctypes.cast(ptr, _D), n), "emu_load_particles")

    def get_particles_ptr(self, ptr, n):
        self._ck(self.lib.emu_get_particles(self.h, ctypes.cast(ptr, _D), n), "emu_get_particles")

    def num_particles(self):
        n = ctypes.c_int64(0)
        self._ck(self.lib.emu_num_particles(self.h, ctypes.byref(n)), "emu_num_particles")
        return n.value

    def get_particles(self):
        n = self.num_particles()
        out = np.empty((n, nreal(self.nf)))
        self._ck(self.lib.emu_get_particles(self.h, _dptr(out), n), "emu_get_particles")
        return out

    def deposit(self):
        self._ck(self.lib.emu_deposit(self.h), "emu_deposit")

    def get_mesh(self):
        p = self.params
        nc = p.ncell[0] * p.ncell[1] * p.ncell[2]
        out = np.empty(ncomp(self.nf) * nc)
        self._ck(self.lib.emu_get_mesh(self.h, _dptr(out)), "emu_get_mesh")
        return out

    def interpolate_rhs(self):
        n = self.num_particles()
        out = np.empty((n, nreal(self.nf)))
        self._ck(self.lib.emu_interpolate_rhs(self.h, _dptr(out)), "emu_interpolate_rhs")
        return out

    def renormalize(self):
        bad = ctypes.c_int64(-1)
        code = self.lib.emu_renormalize(self.h, ctypes.byref(bad))
        return code, bad.value

    def compute_dt(self):
        dt = ctypes.c_double(0)
        code = self.lib.emu_compute_dt(self.h, ctypes.byref(dt))
        if code & ~EMU_ERR_DT:
            self._ck(code, "emu_compute_dt")
        return dt.value, code

    def step(self, dt, raise_on_error=True):
        bad = ctypes.c_int64(-1)
        code = self.lib.emu_step(self.h, float(dt), ctypes.byref(bad))
        if code and raise_on_error:
            self._ck(code, "emu_step")
        return code, bad.value

    def evolve(self, nsteps, start_time=0.0, end_time=float("inf")):
        info = EmuRunInfo()
        code = self.lib.emu_evolve(self.h, int(nsteps), float(start_time), float(end_time), ctypes.byref(info))
        if code & ~(EMU_ERR_TRACE | EMU_ERR_NEGDIAG | EMU_ERR_LENGTH | EMU_ERR_DT):
            self._ck(code, "emu_evolve")
        return info

    def init_particles_device(self):
        """InitParticles on the device, loaded into this context"""
        self._ck(self.lib.emu_init_particles_device(self.h), "emu_init_particles_device")

    def attach_local(self, group, rank):
        """join rank `rank` of a LocalGroup (before load_particles)"""
        self._ck(self.lib.emu_attach_local(self.h, group.h, int(rank)), "emu_attach_local")

    def attach_comm(self, comm_id, rank, nranks):
        """join a particle-sharding communicator (before load_particles)"""
        assert len(comm_id) == COMM_ID_BYTES
        _preload_nccl()
        self._ck(self.lib.emu_attach_comm(self.h, comm_id, int(rank), int(nranks)), "emu_attach_comm")

    # ---- discrete adjoint (FP64 RK4) ----
    def adjoint_reserve(self, nsteps, checkpoint_interval):
        """Allocate a recorded run's storage up front; returns (device bytes,
        stage-state storage: 2 every step of the run (no recompute), 1 per
        segment, 0 per step; sub-checkpoint spacing or 0)."""
        b, st, sub = ctypes.c_int64(0), ctypes.c_int(0), ctypes.c_int(0)
        self._ck(self.lib.emu_adjoint_reserve(self.h, int(nsteps), int(checkpoint_interval), ctypes.byref(b),
                                              ctypes.byref(st), ctypes.byref(sub)), "emu_adjoint_reserve")
        return int(b.value), int(st.value), int(sub.value)

    def adjoint_forward(self, nsteps, checkpoint_interval, start_time=0.0):
        """Recorded run of nsteps from the loaded state; returns (dts, info)."""
        dts = np.zeros(int(nsteps))
        info = EmuRunInfo()
        self._ck(self.lib.emu_adjoint_forward(self.h, int(nsteps), int(checkpoint_interval), float(start_time),
                                              _dptr(dts), ctypes.byref(info)), "emu_adjoint_forward")
        return dts, info

    def adjoint_objective(self, gradient=True):
        """(J, dJ/df [n, 2nf^2], dJ/d(N, Nbar) [n, 2]) of the current state, load order."""
        n = self.num_particles()
        J = np.zeros(1)
        lf = np.zeros((n, 2 * self.nf * self.nf)) if gradient else None
        lN = np.zeros((n, 2)) if gradient else None
        null = ctypes.cast(None, _D)
        self._ck(self.lib.emu_adjoint_objective(self.h, _dptr(J), _dptr(lf) if gradient else null,
                                                _dptr(lN) if gradient else null), "emu_adjoint_objective")
        return float(J[0]), lf, lN

    def adjoint_backward(self, lam_f_final, lam_N_final=None):
        """(dJ/df0 [n, 2nf^2], dJ/d(N, Nbar) [n, 2]) of the recorded run's initial state."""
        n = self.num_particles()
        lf = np.ascontiguousarray(lam_f_final, dtype=np.float64).reshape(n, 2 * self.nf * self.nf)
        lN = None if lam_N_final is None else np.ascontiguousarray(lam_N_final, dtype=np.float64).reshape(n, 2)
        out_f = np.zeros_like(lf)
        out_N = np.zeros((n, 2))
        self._ck(self.lib.emu_adjoint_backward(self.h, _dptr(lf), ctypes.cast(None, _D) if lN is None else _dptr(lN),
                                               _dptr(out_f), _dptr(out_N)), "emu_adjoint_backward")
        return out_f, out_N

    def evolve_begin(self, start_time, end_time, max_steps):
        self._ck(self.lib.emu_evolve_begin(self.h, float(start_time), float(end_time), int(max_steps)),
                 "emu_evolve_begin")

    def evolve_steps(self, n):
        self._ck(self.lib.emu_evolve_steps(self.h, int(n)), "emu_evolve_steps")

    def evolve_end(self):
        info = EmuRunInfo()
        self.lib.emu_evolve_end(self.h, ctypes.byref(info))
        return info

    def profile_step(self):
        """per-kernel CUDA-event durations (ms) of one device-resident step"""
        buf = (ctypes.c_float * 16)()
        nk = ctypes.c_int(0)
        self._ck(self.lib.emu_profile_step(self.h, buf, 16, ctypes.byref(nk)), "emu_profile_step")
        return [buf[i] for i in range(nk.value)]

    def set_wait_limit(self, polls):
        """limit of the cooperative kernels' grid-barrier waits (polls; < 0:
        the default)"""
        self._ck(self.lib.emu_set_wait_limit(self.h, int(polls)), "emu_set_wait_limit")

    def flush_l2(self, ptr, nbytes):
        self._ck(self.lib.emu_flush_l2(self.h, ctypes.c_void_p(ptr), int(nbytes)), "emu_flush_l2")

    def write_plotfile(self, path, time, step, write_particles=True):
        self._ck(self.lib.emu_write_plotfile(self.h, path.encode(), float(time), int(step),
                                             1 if write_particles else 0), "emu_write_plotfile")


def write_plotfile_host(p, path, time, step, mesh, records=None):
    """Write pltNNNNN-style output from host arrays (no GPU)."""
    lib = load_library()
    m = np.ascontiguousarray(mesh, dtype=np.float64)
    r = None if records is None else np.ascontiguousarray(records, dtype=np.float64)
    _check(lib.emu_write_plotfile_host(ctypes.byref(p), path.encode(), float(time), int(step), _dptr(m),
                                       None if r is None else _dptr(r), 0 if r is None else r.shape[0]),
           None, "emu_write_plotfile_host")
