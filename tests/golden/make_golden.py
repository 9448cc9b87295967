"""Generate the golden fixtures tests/golden/golden_<case>.npz.

Each fixture holds a small seeded particle set, its run parameters, and the
outputs of the reference's own per-particle arithmetic (the kernel bodies of
Scripts/symbolic_hermitians/generate_code.py compiled into
oracle/_ref/libemuref<N>.so by oracle/build_oracle.py):

  mesh0      deposit_to_mesh of the particles (GIdx planes)
  rhs0       interpolate_rhs_from_mesh on mesh0 (particle records)
  dt0        compute_dt on mesh0 (with Vvac_max of the particles)
  step_<k>   particles after one step of integrator k (0 FE, 2 trapezoid,
             3 SSPRK3, 4 RK4) with dt0, and mesh_<k> the last stage mesh
  renorm_in / renorm_out / renorm_status   Renormalize of perturbed states

Run from the repository root with the reference tree present:
    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from emu_b200 import api  # noqa: E402
from oracle import build_oracle  # noqa: E402
from oracle.oracle import RefHarness  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

PARAM_FIELDS = [f[0] for f in api.EmuParams._fields_ if f[0] != "restart_dir"]


def params_to_json(p):
    d = {}
    for k in PARAM_FIELDS:
        v = getattr(p, k)
        if k in ("ncell", "nppc"):
            v = [int(x) for x in v]
        d[k] = v
    return json.dumps(d)


def params_from_json(s):
    d = json.loads(s)
    p = api.default_params()
    for k, v in d.items():
        api.set_param(p, k, v)
    return p


def _case(name, nf, ncell, order, L, ndirs, seed, rho=0.0, jitter=0.45, masses=None, **extra):
    p = api.default_params(nflavors=nf, shape_order=order, ncell=ncell, Lx=L[0], Ly=L[1], Lz=L[2],
                           simulation_type=4, st4_ndens=4.89e32, st4_ndensbar=3.1e32, st4_fluxfac=0.1,
                           st4_fluxfacbar=1.0 / 3.0, st4_theta=0.3, st4_phi=0.2, st4_thetabar=0.1,
                           st4_amplitude=1e-2, direction_generator=1, ndirections=ndirs, seed=seed,
                           rho_in=rho, Ye_in=0.45, cfl_factor=0.5, flavor_cfl_factor=0.4)
    for k, v in extra.items():
        api.set_param(p, k, v)
    m = masses or (-0.008596511, 0.0, 0.049487372)
    ev_g = api.EV / api.CLIGHT ** 2
    p.mass1, p.mass2, p.mass3 = m[0] * ev_g, m[1] * ev_g, m[2] * ev_g
    p.theta12, p.theta13, p.theta23, p.deltaCP = 0.59, 0.84, 0.15, 3.87
    parts = api.init_particles(p)
    rng = np.random.default_rng(seed)
    dx = np.array([L[i] / ncell[i] for i in range(3)])
    parts[:, 0:3] = (parts[:, 0:3] + rng.uniform(-jitter, jitter, (len(parts), 3)) * dx) % np.array(L)
    # a few particles exactly on cell faces and on the domain edge
    parts[0, 0:3] = 0.0
    if len(parts) > 2:
        parts[1, 2] = dx[2] * (ncell[2] // 2)
        parts[2, 0] = dx[0]
    parts[:, 4:7] = parts[:, 0:3]
    return name, p, parts


CASES = [
    lambda: _case("nf2_1d", 2, (1, 1, 16), 2, (1.0, 1.0, 8.0), 8, 11),
    lambda: _case("nf3_3d", 3, (4, 3, 5), 2, (2.0, 1.5, 2.5), 6, 12, rho=3e9),
    lambda: _case("nf2_cic", 2, (3, 3, 3), 1, (1.5, 1.5, 1.5), 5, 13, rho=1e10),
    lambda: _case("nf3_ngp", 3, (1, 1, 1), 0, (1.0, 1.0, 1.0), 7, 14, rho=1.3e9),
    # compute_dt's adaptive branch (Evolve.cpp:68-74) with the translation
    # limit off: dt_flavor = min(speedup dt_stupid, dt_adaptive); the cap
    # binds at speedup 3, the adaptive potential at 10
    lambda: _case("nf2_adaptive", 2, (1, 1, 16), 2, (1.0, 1.0, 8.0), 8, 15, rho=2e9, cfl_factor=-1.0,
                  max_adaptive_speedup=3.0),
    lambda: _case("nf3_adaptive_3d", 3, (3, 4, 3), 2, (1.5, 2.0, 1.5), 5, 16, rho=2e9, cfl_factor=-1.0,
                  max_adaptive_speedup=10.0),
]


def make(name, p, parts):
    r = RefHarness(p)
    out = {"params": np.array(params_to_json(p)), "parts": parts}
    mesh0 = r.deposit(parts)
    out["mesh0"] = mesh0
    out["rhs0"] = r.interpolate_rhs(mesh0, parts)
    vmax = r.vvac_max(parts)
    dt0, st = r.compute_dt(mesh0, vmax)
    out["vvac_max"] = np.array(vmax)
    out["dt0"] = np.array(dt0)
    for k in (0, 2, 3, 4):
        q = parts.copy()
        mesh, s, bad = r.rk_step(q, dt0, rk_type=k)
        out["step_%d" % k] = q
        out["mesh_%d" % k] = mesh
        out["status_%d" % k] = np.array(s)
    # Renormalize on perturbed states: small trace and length errors (fixed),
    # a large trace error (flagged), a negative diagonal (clamped / flagged)
    rng = np.random.default_rng(99)
    q = parts.copy()
    nh = p.nflavors ** 2
    f = 3 + 10
    fb = 3 + 12 + nh
    q[:, f] += rng.uniform(-5e-6, 5e-6, len(q))
    q[:, fb:fb + nh] *= 1.0 + rng.uniform(-3e-6, 3e-6, (len(q), 1))
    q[1, f] += 2e-3            # trace error > 100*maxError
    q[2, fb] = -5e-6           # diagonal below -maxError: clamped
    out["renorm_in"] = q.copy()
    qq, s, bad = r.renormalize(q)
    out["renorm_out"] = qq
    out["renorm_status"] = np.array(s)
    out["renorm_bad"] = np.array(bad)
    np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % name), **out)
    return out


def main(only=None):
    build_oracle.build_ref()
    for c in CASES:
        name, p, parts = c()
        if only and name not in only:
            continue
        make(name, p, parts)
        print(name, parts.shape)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
