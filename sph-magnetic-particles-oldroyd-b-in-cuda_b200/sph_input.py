"""Writers for the reference's text input formats.

`input`               key/value lines parsed by class_system::read_input
                      (reference src/system_read_input.cpp:102-269); `coll_x` lines must
                      follow `N_colloids`, as the reference reads them in file order.
`input_particles.in`  the restart file of new_sim = 1
                      (src/system_initialize_particles_old_sim.cpp:36,48): 2D columns
                      x y vx vy mass type cxx cxy cyy, 3D columns
                      x y z vx vy vz mass type cxx cxy cyy cxz cyz czz.  The reference
                      parses every column as float, so values are written float-exact.
"""
import numpy as np

DEFAULTS = dict(
    N=(64, 64), L=(1.0, 1.0), dim=2, dt=5e-5, t0=0.0, Nsteps=2000, overlap=4.0,
    rho=1.0, c=10.0, P0=0.0, eta=0.1, zeta=0.0, np=100.0, kT=0.01, tau=1.0,
    ext_force_type=0, ext_force=(0.0, 0.0), freq_micro=10**9, freq_macro=10**9,
    freq_walls=10**9, freq_colloids=10**9, wall=0, Vwall_top=0.0, Vwall_bottom=0.0,
    N_colloids=0, coll_R=1.0, coll_rho=1.0, coll_move=0, coll_x=(),
    coll_repulsion_cuton=0.0, F0_repulsion=1.0, tau_repulsion=1.0, cutoff_magnetic=0.1,
    F0_magnetic=1.0, omega_magnetic=0.0, new_sim=0,
)

_ORDER = [
    "N", "L", "dim", "dt", "t0", "Nsteps", "overlap", "rho", "c", "P0", "eta", "zeta", "np",
    "kT", "tau", "ext_force_type", "ext_force", "freq_micro", "freq_macro", "freq_walls",
    "freq_colloids", "wall", "Vwall_bottom", "Vwall_top", "N_colloids", "coll_R", "coll_rho",
    "coll_move", "coll_x", "coll_repulsion_cuton", "F0_repulsion", "tau_repulsion",
    "cutoff_magnetic", "F0_magnetic", "omega_magnetic", "new_sim",
]


def _fmt(v):
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def make_input(**kw):
    """Return the text of a reference `input` file; unspecified keys take DEFAULTS."""
    p = dict(DEFAULTS)
    unknown = set(kw) - set(p)
    if unknown:
        raise KeyError("unknown input keys: %s" % sorted(unknown))
    p.update(kw)
    lines = ["# SPH input (reference format)"]
    for k in _ORDER:
        v = p[k]
        if k == "coll_x":
            for c in v:
                lines.append("coll_x " + " ".join(_fmt(float(t)) for t in c))
            continue
        if isinstance(v, (tuple, list, np.ndarray)):
            lines.append(k + " " + " ".join(_fmt(t) for t in v))
        else:
            lines.append(k + " " + _fmt(v))
    return "\n".join(lines) + "\n"


def write_input(path, **kw):
    with open(path, "w") as f:
        f.write(make_input(**kw))
    return path


def write_particles(path, dim, x, y, z, vx, vy, vz, mass, type_, cxx, cxy, cyy,
                    cxz=None, cyz=None, czz=None):
    """Write a restart file; every value is rounded to float32 first so that the file
    holds exactly what the reference's float parser will read."""
    f32 = lambda a: np.asarray(a, dtype=np.float32)
    if dim == 2:
        cols = [f32(x), f32(y), f32(vx), f32(vy), f32(mass), f32(type_), f32(cxx), f32(cxy), f32(cyy)]
    else:
        cols = [f32(x), f32(y), f32(z), f32(vx), f32(vy), f32(vz), f32(mass), f32(type_),
                f32(cxx), f32(cxy), f32(cyy), f32(cxz), f32(cyz), f32(czz)]
    data = np.stack(cols, axis=1)
    # %.9g round-trips every float32 exactly
    np.savetxt(path, data, fmt="%.9g")
    return path
