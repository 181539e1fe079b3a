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


def suspension_centres(n, R, rcut, seed, L=(1.0, 1.0, 1.0), min_dist=2.2, tries=100000):
    """n colloid centres for a 3D box with walls normal to y, drawn uniformly from `seed`:
    x over the periodic box, y at least R + rcut from both walls, z in [R, L - R]; every
    pair at least min_dist * R apart (x and z periodic).  Two rules keep the input one the
    reference accepts: each pair passes its overlap check as it is written,
    sqrt(dx^2 + dy^2 + dy^2) >= 2R with dx periodic (src/system_read_input.cpp:482-500
    takes the z difference from the y coordinates); and z stays R clear of the box faces,
    because the reference places the poles of a colloid's particle shells at z +- r without
    the periodic wrap (src/system_initialize_particles_new_sim.cpp:196-199,239-242), and a
    pole below z = 0 hashes outside the cell grid at the first search.  Raises if a centre
    finds no place in `tries` draws."""
    rng = np.random.default_rng(seed)
    lo, hi = R + rcut, L[1] - R - rcut
    out = []
    for _ in range(n):
        for _ in range(tries):
            c = (rng.uniform(0.0, L[0]), rng.uniform(lo, hi), rng.uniform(R, L[2] - R))
            ok = True
            for p in out:
                dx = c[0] - p[0]
                dx -= L[0] * round(dx / L[0])
                dy = c[1] - p[1]
                dz = c[2] - p[2]
                dz -= L[2] * round(dz / L[2])
                if dx * dx + dy * dy + dz * dz < (min_dist * R) ** 2 or \
                        dx * dx + 2.0 * dy * dy < (2.0 * R) ** 2:
                    ok = False
                    break
            if ok:
                out.append(c)
                break
        else:
            raise ValueError("no place for colloid %d of %d" % (len(out) + 1, n))
    return tuple(out)


def suspension_spec(N=96, n_colloids=32, seed=11, nsteps=2000, tau_repulsion=1.0,
                    F0_repulsion=10.0, F0_magnetic=5.0):
    """The 3D suspension of rotating magnetic colloids between walls at rest: N^3 lattice,
    L = 1, overlap 3, Oldroyd-B (tau 1, np 100, kT 0.01, eta 0.1, rho 1, c 10, P0 0),
    n_colloids colloids of radius 4 dx (density 1, moving), repulsion cut-on 2.05 R
    (the reference's cut-on is the surface-to-surface gap, 0.05 R), F0_repulsion 10,
    magnetic cutoff 6 R, F0_magnetic 5, omega 2 pi, dt 2e-5.  tau_repulsion defaults to 1:
    the reference rejects 0.01 here (its repulsion cutoff 2R + 5R/tau_rep would exceed the
    box, src/system_initialize.cpp:161,225-247), and 1 is the smallest round value it
    accepts."""
    dx = 1.0 / N
    R = 4.0 * dx
    rcut = 3.0 * dx
    return dict(N=(N, N, N), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1, Vwall_bottom=0.0,
                Vwall_top=0.0, rho=1.0, c=10.0, P0=0.0, eta=0.1, zeta=0.0, np=100.0, kT=0.01,
                tau=1.0, dt=2e-5, Nsteps=nsteps, N_colloids=n_colloids, coll_R=R,
                coll_rho=1.0, coll_move=0,
                coll_x=suspension_centres(n_colloids, R, rcut, seed),
                coll_repulsion_cuton=0.05 * R, F0_repulsion=F0_repulsion,
                tau_repulsion=tau_repulsion, cutoff_magnetic=6.0 * R, F0_magnetic=F0_magnetic,
                omega_magnetic=2.0 * np.pi)
