"""Python host API of the B200 SPH engine (ctypes over lib/libsph_b200.so).

The class `System` mirrors the reference's `class_system` step methods
(src/class_system.h:344-650): neighbours_search, calculate_density, calculate_pressure,
calculate_vel_gradient, calculate_forces, calculate_external_forces,
calculate_force_walls, calculate_force_colloids, V_Verlet_step1, V_Verlet_step2; plus
`step(n)`, the driver loop of src/main.cu:358-467 replayed as a CUDA graph.  Arrays come
back in the reference's original particle order.

There is no CPU fallback: importing works anywhere, but creating a System needs the
compiled library and a CUDA device, and raises otherwise.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SPH_B200_LIB selects another build of the engine library (e.g. a tuning variant)
LIB_PATH = os.environ.get("SPH_B200_LIB") or os.path.join(HERE, "lib", "libsph_b200.so")

FIELDS = [
    "x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "dens", "press", "mass",
    "cxx", "cxy", "cyy", "cxz", "cyz", "czz", "dcdt_xx", "dcdt_xy", "dcdt_yy",
    "dcdt_xz", "dcdt_yz", "dcdt_zz", "gxx", "gxy", "gxz", "gyx", "gyy", "gyz", "gzx",
    "gzy", "gzz",
]
COLLOID_FIELDS = [
    "coll_x", "coll_y", "coll_z", "coll_vx", "coll_vy", "coll_vz", "coll_omegax",
    "coll_omegay", "coll_omegaz", "coll_theta", "coll_quat0", "coll_quatx", "coll_quaty",
    "coll_quatz", "fx_colloid", "fy_colloid", "fz_colloid", "tx_colloid", "ty_colloid",
    "tz_colloid",
]
STATUS = {
    0: "SPH_OK", 1: "SPH_ERR_BAD_INPUT", 2: "SPH_ERR_CUDA", 3: "SPH_ERR_CELL_RANGE",
    4: "SPH_ERR_NAN", 5: "SPH_ERR_TIMEOUT", 6: "SPH_ERR_STATE", 7: "SPH_ERR_NOMEM",
    8: "SPH_ERR_CAPACITY", 9: "SPH_ERR_IO",
}
PRECISION = {"fp64": 0, "mixed": 1}

# every symbol include/sph_capi.h declares
EXPORTS = [
    "sph_read_input", "sph_create", "sph_create_ensemble", "sph_destroy", "sph_get_info",
    "sph_last_error", "sph_status_string", "sph_neighbours_search", "sph_calculate_density",
    "sph_calculate_pressure", "sph_calculate_vel_gradient", "sph_calculate_forces",
    "sph_calculate_external_forces", "sph_calculate_force_walls",
    "sph_calculate_force_colloids", "sph_vv_step1", "sph_vv_step2", "sph_initial_forces",
    "sph_step", "sph_synchronize", "sph_read_field", "sph_write_field",
    "sph_read_field_device", "sph_read_type", "sph_read_colloid_field",
    "sph_read_wall_forces", "sph_export_cells", "sph_export_colloid_cells",
    "sph_kinetic_energy", "sph_last_step_ms", "sph_kernel_launches", "sph_host_setup",
    "sph_profile_phases", "sph_phase_name", "sph_save_checkpoint", "sph_load_checkpoint",
    "sph_observe", "sph_observables", "sph_reset_observables", "sph_get_tuning",
    "sph_set_tuning", "sph_autotune", "sph_neighbours_search_noalloc", "sph_neighbour_lists",
    "sph_write_restart",
]
OBSERVABLES = ["wall_stress", "N1", "chain_order", "kinetic_energy"]

c_int, c_double, c_void_p, c_char_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p
PD = ctypes.POINTER(ctypes.c_double)
PI = ctypes.POINTER(ctypes.c_int)


class SphInput(ctypes.Structure):
    _fields_ = [
        ("N", c_int * 3), ("L", c_double * 3), ("dim", c_int), ("dt", c_double),
        ("t0", c_double), ("Nsteps", c_int), ("overlap", c_double), ("rho", c_double),
        ("c", c_double), ("P0", c_double), ("eta", c_double), ("zeta", c_double),
        ("np", c_double), ("kT", c_double), ("tau", c_double), ("ext_force_type", c_int),
        ("ext_force", c_double * 3), ("freq_micro", c_int), ("freq_macro", c_int),
        ("freq_walls", c_int), ("freq_colloids", c_int), ("wall", c_int),
        ("Vwall_top", c_double), ("Vwall_bottom", c_double), ("N_colloids", c_int),
        ("coll_R", c_double), ("coll_rho", c_double), ("coll_xyz", PD), ("coll_move", c_int),
        ("coll_repulsion_cuton", c_double), ("F0_repulsion", c_double),
        ("tau_repulsion", c_double), ("cutoff_magnetic", c_double), ("F0_magnetic", c_double),
        ("omega_magnetic", c_double), ("new_sim", c_int),
    ]


class SphOptions(ctypes.Structure):
    _fields_ = [("precision", c_int), ("device", c_int), ("use_graph", c_int),
                ("nbr_capacity", c_int), ("init_on_device", c_int)]


class SphTuning(ctypes.Structure):
    _fields_ = [("list_threads_per_cell", c_int), ("density_block", c_int)]


class SphInfo(ctypes.Structure):
    _fields_ = [
        ("N", c_int), ("dim", c_int), ("wall", c_int), ("Ncells", c_int * 3),
        ("Ntotal_cells", c_int), ("Nwalls", c_int), ("Nlist_walls", c_int),
        ("N_colloids", c_int), ("Nlist_colloids", c_int), ("Ncells_colloids", c_int * 3),
        ("Ntotal_cells_colloids", c_int), ("step", c_int), ("nboxes", c_int),
        ("precision", c_int),
        ("rcut", c_double), ("rcutsq", c_double), ("cw", c_double), ("c_gradw", c_double),
        ("csq", c_double), ("rho0", c_double), ("a", c_double), ("b", c_double),
        ("nkT", c_double), ("tau", c_double), ("dt", c_double), ("cell_size", c_double * 3),
        ("wall_width", c_double), ("y_bottom", c_double), ("y_top", c_double),
        ("V_bottom", c_double), ("V_top", c_double), ("coll_R", c_double),
        ("coll_mass", c_double), ("coll_I", c_double), ("L", c_double * 3), ("t0", c_double),
        ("omega_magnet", c_double),
        ("Nmax", c_int), ("ext_force_type", c_int),
        ("rcut_inv", c_double), ("c", c_double), ("rho", c_double), ("P0", c_double),
        ("ky", c_double), ("beta_max", c_double), ("ext_force", c_double * 3),
        ("coll_rho", c_double), ("coll_rep_cuton", c_double), ("coll_rep_cutoff", c_double),
        ("rcuton_coll_rep", c_double), ("rcutoff_coll_rep", c_double),
        ("rcuton_coll_rep_sq", c_double), ("rcutoff_coll_rep_sq", c_double),
        ("rcutoff_coll", c_double), ("rcutoff_coll_sq", c_double), ("F0_rep", c_double),
        ("tau_rep", c_double), ("r0_magnet", c_double), ("r0_magnet_sq", c_double),
        ("F0_magnet", c_double), ("cell_colloids_size", c_double * 3),
    ]


_lib = None


class SphError(RuntimeError):
    def __init__(self, status, msg):
        self.status = STATUS.get(status, str(status))
        super().__init__("%s: %s" % (self.status, msg))


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    """Load the engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("engine library missing: %s (run make in %s)" % (LIB_PATH, HERE))
        L = ctypes.CDLL(LIB_PATH)
        L.sph_read_input.argtypes = [c_char_p, ctypes.POINTER(SphInput), PD, c_int, c_char_p, ctypes.c_size_t]
        L.sph_create.argtypes = [ctypes.POINTER(SphInput), c_char_p, ctypes.POINTER(SphOptions), ctypes.POINTER(c_void_p)]
        L.sph_create_ensemble.argtypes = [c_int, ctypes.POINTER(SphInput), ctypes.POINTER(c_char_p),
                                          ctypes.POINTER(SphOptions), ctypes.POINTER(c_void_p)]
        L.sph_destroy.argtypes = [c_void_p]
        L.sph_destroy.restype = None
        L.sph_get_info.argtypes = [c_void_p, c_int, ctypes.POINTER(SphInfo)]
        L.sph_last_error.argtypes = [c_void_p]
        L.sph_last_error.restype = c_char_p
        L.sph_status_string.argtypes = [c_int]
        L.sph_status_string.restype = c_char_p
        for n in ["sph_neighbours_search", "sph_calculate_density", "sph_calculate_pressure",
                  "sph_calculate_vel_gradient", "sph_calculate_external_forces",
                  "sph_calculate_force_walls", "sph_vv_step1", "sph_vv_step2",
                  "sph_initial_forces", "sph_synchronize"]:
            getattr(L, n).argtypes = [c_void_p]
        L.sph_calculate_forces.argtypes = [c_void_p, PD]
        L.sph_calculate_force_colloids.argtypes = [c_void_p, PD]
        L.sph_step.argtypes = [c_void_p, c_int]
        L.sph_read_field.argtypes = [c_void_p, c_int, PD]
        L.sph_write_field.argtypes = [c_void_p, c_int, PD]
        L.sph_read_field_device.argtypes = [c_void_p, c_int, c_void_p]
        L.sph_read_type.argtypes = [c_void_p, PI]
        L.sph_read_colloid_field.argtypes = [c_void_p, c_int, PD]
        L.sph_read_wall_forces.argtypes = [c_void_p, PD]
        L.sph_export_cells.argtypes = [c_void_p, PI, PI, PI, PI]
        L.sph_export_colloid_cells.argtypes = [c_void_p, PI, PI, PI, PI]
        L.sph_kinetic_energy.argtypes = [c_void_p, PD]
        L.sph_save_checkpoint.argtypes = [c_void_p, c_char_p]
        L.sph_get_tuning.argtypes = [c_void_p, ctypes.POINTER(SphTuning)]
        L.sph_set_tuning.argtypes = [c_void_p, ctypes.POINTER(SphTuning)]
        L.sph_autotune.argtypes = [c_void_p, c_char_p, ctypes.POINTER(SphTuning)]
        L.sph_observe.argtypes = [c_void_p]
        L.sph_observables.argtypes = [c_void_p, PD, ctypes.POINTER(ctypes.c_longlong)]
        L.sph_reset_observables.argtypes = [c_void_p]
        L.sph_load_checkpoint.argtypes = [c_void_p, c_char_p]
        L.sph_last_step_ms.argtypes = [c_void_p, PD]
        L.sph_kernel_launches.argtypes = [c_void_p, ctypes.POINTER(ctypes.c_longlong)]
        _lib = L
    return _lib


def read_input(path):
    """Parse a reference `input` file with the engine's parser; returns (SphInput, coll)."""
    inp = SphInput()
    coll = np.zeros(3 * 1000, dtype=np.float64)
    msg = ctypes.create_string_buffer(256)
    st = lib().sph_read_input(path.encode(), ctypes.byref(inp), coll.ctypes.data_as(PD), 1000, msg, 256)
    if st != 0:
        raise SphError(st, msg.value.decode())
    return inp, coll


class SphHostState(ctypes.Structure):
    _fields_ = [(n, PD) for n in ["x", "y", "z", "vx", "vy", "vz", "mass", "cxx", "cxy", "cyy",
                                  "cxz", "cyz", "czz"]] + [
        ("type", PI), ("walls_list", PI), ("walls_start", PI), ("colloids_list", PI),
        ("colloids_start", PI), ("x_center", PD), ("y_center", PD), ("z_center", PD)]


def host_setup(input_path, particles_path=None):
    """Initial state as the engine's host set-up builds it (no GPU needed): the arrays the
    reference's class_system holds on the host after constructor + initialize."""
    L = lib()
    L.sph_host_setup.argtypes = [ctypes.POINTER(SphInput), c_char_p, c_int,
                                 ctypes.POINTER(SphHostState), PI, ctypes.POINTER(SphInfo)]
    inp, coll = read_input(str(input_path))
    inp.coll_xyz = coll.ctypes.data_as(PD)
    pp = particles_path.encode() if particles_path else None
    n = c_int(0)
    info = SphInfo()
    st = L.sph_host_setup(ctypes.byref(inp), pp, 0, None, ctypes.byref(n), ctypes.byref(info))
    if st != 0:
        raise SphError(st, "sph_host_setup failed (see stderr)")
    cap = max(n.value, 1)
    out = {k: np.zeros(cap) for k in ["x", "y", "z", "vx", "vy", "vz", "mass", "cxx", "cxy",
                                     "cyy", "cxz", "cyz", "czz", "x_center", "y_center", "z_center"]}
    for k in ["type", "walls_list", "colloids_list", "colloids_start"]:
        out[k] = np.zeros(cap, dtype=np.int32)
    out["walls_start"] = np.zeros(2, dtype=np.int32)
    hs = SphHostState()
    for name, typ in SphHostState._fields_:
        setattr(hs, name, out[name].ctypes.data_as(typ))
    st = L.sph_host_setup(ctypes.byref(inp), pp, cap, ctypes.byref(hs), ctypes.byref(n), ctypes.byref(info))
    if st != 0:
        raise SphError(st, "sph_host_setup failed (see stderr)")
    res = {}
    for name, _ in SphInfo._fields_:
        v = getattr(info, name)
        res[name] = list(v) if isinstance(v, ctypes.Array) else v
    N, nl, nw, nc = info.N, info.Nlist_colloids, info.Nlist_walls, info.N_colloids
    arrays = {k: out[k][:N] for k in ["x", "y", "z", "vx", "vy", "vz", "mass", "cxx", "cxy",
                                     "cyy", "cxz", "cyz", "czz", "type"]}
    arrays.update(walls_list=out["walls_list"][:nw], walls_start=out["walls_start"],
                  colloids_list=out["colloids_list"][:nl], colloids_start=out["colloids_start"][:nc],
                  x_center=out["x_center"][:nl], y_center=out["y_center"][:nl],
                  z_center=out["z_center"][:nl])
    return arrays, res


def write_restart(path, dim, a):
    """Write `a` (the arrays host_setup returns: x, y, z, vx, vy, vz, mass, type, cxx ... czz)
    as the reference's restart file input_particles.in (include/sph_io.h: sph_write_restart),
    every value rounded to float as the reference reads it.  Formatted on all host cores."""
    L = lib()
    L.sph_write_restart.argtypes = [c_char_p, c_int, c_int] + [PD] * 7 + [PI] + [PD] * 6
    n = len(a["x"])
    d = {k: np.ascontiguousarray(a[k], dtype=np.float64)
         for k in ["x", "y", "z", "vx", "vy", "vz", "mass", "cxx", "cxy", "cyy", "cxz", "cyz", "czz"]}
    t = np.ascontiguousarray(a["type"], dtype=np.int32)
    P = lambda k: d[k].ctypes.data_as(PD)
    st = L.sph_write_restart(str(path).encode(), int(dim), n, P("x"), P("y"), P("z"), P("vx"),
                             P("vy"), P("vz"), P("mass"), t.ctypes.data_as(PI), P("cxx"),
                             P("cxy"), P("cyy"), P("cxz"), P("cyz"), P("czz"))
    if st != 0:
        raise SphError(st, "sph_write_restart failed for %s" % path)


def write_seeded_start(workdir, spec, seed, vmax):
    """A lattice box started from seeded random fluid velocities, the way the reference can
    take one: new_sim = 1 with a restart file (src/system_initialize_particles_old_sim.cpp).
    Positions, masses, types and c = I are the lattice state the reference builds for
    new_sim = 0 (the engine's host set-up, no GPU needed); every fluid velocity component is
    drawn uniform in [-vmax, vmax] from `seed`; walls and colloid particles stay at rest, as
    the lattice start has them.  Writes `workdir`/input (new_sim = 1) and
    `workdir`/input_particles.in; returns (input path, particles path, N)."""
    import sph_input

    spec = dict(spec)
    spec.pop("new_sim", None)
    lattice_in = os.path.join(workdir, "input_lattice")
    sph_input.write_input(lattice_in, **spec)
    a, info = host_setup(lattice_in)
    n = len(a["x"])
    rng = np.random.default_rng(seed)
    v = rng.uniform(-vmax, vmax, size=(3, n))
    v[:, a["type"] != 0] = 0.0
    if info["dim"] == 2:
        v[2] = 0.0
    a = dict(a, vx=v[0], vy=v[1], vz=v[2])
    pp = os.path.join(workdir, "input_particles.in")
    write_restart(pp, info["dim"], a)
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, new_sim=1, **spec)
    return inp, pp, n


class SphGrid(ctypes.Structure):
    _fields_ = [("dim", c_int), ("wall", c_int), ("Ncells", c_int * 3),
                ("cell_size", c_double * 3), ("wall_width", c_double)]


def neighbours_search_noalloc(x, y, z, n, grid, particle_cell, particle_index, cell_start,
                              cell_end, stream=None):
    """Allocation-free neighbour search on caller-owned device arrays (device pointers as
    ints).  For callers that cannot allocate device memory; returns the raw status code."""
    L = lib()
    L.sph_neighbours_search_noalloc.argtypes = [c_void_p, c_void_p, c_void_p, c_int,
                                                ctypes.POINTER(SphGrid), c_void_p, c_void_p,
                                                c_void_p, c_void_p, c_void_p]
    return L.sph_neighbours_search_noalloc(x, y, z, int(n), ctypes.byref(grid), particle_cell,
                                           particle_index, cell_start, cell_end, stream)


class System:
    """One or more simulation boxes on the GPU (the reference's class_system)."""

    def __init__(self, input_paths, particles_paths=None, precision="fp64", use_graph=True,
                 device=0, nbr_capacity=0, init_on_device=True):
        """init_on_device: lattice boxes are built on the GPU (bit-identical to the host
        set-up, 4-20x faster to create); colloid shells and restart files are still built
        on the host.  False builds every box on the host."""
        if isinstance(input_paths, (str, os.PathLike)):
            input_paths = [input_paths]
        n = len(input_paths)
        self._keep = []
        arr = (SphInput * n)()
        for b, path in enumerate(input_paths):
            inp, coll = read_input(str(path))
            self._keep.append(coll)
            arr[b] = inp
            arr[b].coll_xyz = coll.ctypes.data_as(PD)
        paths = (c_char_p * n)()
        for b in range(n):
            p = particles_paths[b] if particles_paths else None
            paths[b] = p.encode() if p else None
        opt = SphOptions(PRECISION[precision], device, 1 if use_graph else 0, nbr_capacity,
                         1 if init_on_device else 0)
        h = c_void_p()
        st = lib().sph_create_ensemble(n, arr, paths, ctypes.byref(opt), ctypes.byref(h))
        if st != 0:
            raise SphError(st, "sph_create failed (see stderr)")
        self._h = h
        self.nboxes = n
        self.precision = precision
        self._info = [self.info(b) for b in range(n)]
        self.N = sum(i["N"] for i in self._info)
        self.ncoll = sum(i["N_colloids"] for i in self._info)

    def close(self):
        if getattr(self, "_h", None):
            lib().sph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, st):
        if st != 0:
            raise SphError(st, lib().sph_last_error(self._h).decode())

    def info(self, box=0):
        o = SphInfo()
        self._ok(lib().sph_get_info(self._h, box, ctypes.byref(o)))
        out = {}
        for name, _ in SphInfo._fields_:
            v = getattr(o, name)
            out[name] = list(v) if isinstance(v, ctypes.Array) else v
        return out

    # --- class_system methods ---
    def neighbours_search(self):
        self._ok(lib().sph_neighbours_search(self._h))

    def calculate_density(self):
        self._ok(lib().sph_calculate_density(self._h))

    def calculate_pressure(self):
        self._ok(lib().sph_calculate_pressure(self._h))

    def calculate_vel_gradient(self):
        self._ok(lib().sph_calculate_vel_gradient(self._h))

    @staticmethod
    def _m(m):
        if m is None:
            return None
        a = np.ascontiguousarray(m, dtype=np.float64)
        return a

    def calculate_forces(self, m=None):
        a = self._m(m)
        self._ok(lib().sph_calculate_forces(self._h, a.ctypes.data_as(PD) if a is not None else None))

    def calculate_external_forces(self):
        self._ok(lib().sph_calculate_external_forces(self._h))

    def calculate_force_walls(self):
        self._ok(lib().sph_calculate_force_walls(self._h))

    def calculate_force_colloids(self, m=None):
        a = self._m(m)
        self._ok(lib().sph_calculate_force_colloids(self._h, a.ctypes.data_as(PD) if a is not None else None))

    def V_Verlet_step1(self):
        self._ok(lib().sph_vv_step1(self._h))

    def V_Verlet_step2(self):
        self._ok(lib().sph_vv_step2(self._h))

    def initial_forces(self):
        self._ok(lib().sph_initial_forces(self._h))

    def step(self, n=1):
        self._ok(lib().sph_step(self._h, int(n)))

    def synchronize(self):
        self._ok(lib().sph_synchronize(self._h))

    def last_step_ms(self):
        v = c_double()
        self._ok(lib().sph_last_step_ms(self._h, ctypes.byref(v)))
        return v.value

    def neighbour_lists(self):
        """{'capacity', 'max_used', 'grown'}: candidate chunks a particle's list holds, the
        most chunks a particle has needed so far, and how many times the lists have grown."""
        cap, used, grown = c_int(0), c_int(0), c_int(0)
        lib().sph_neighbour_lists.argtypes = [c_void_p, PI, PI, PI]
        self._ok(lib().sph_neighbour_lists(self._h, ctypes.byref(cap), ctypes.byref(used),
                                           ctypes.byref(grown)))
        return {"capacity": cap.value, "max_used": used.value, "grown": grown.value}

    def kernel_launches(self):
        v = ctypes.c_longlong()
        self._ok(lib().sph_kernel_launches(self._h, ctypes.byref(v)))
        return v.value

    def profile_phases(self, nsteps=5):
        """Mean device milliseconds per phase of a step (CUDA events on the engine's stream)."""
        L = lib()
        L.sph_profile_phases.argtypes = [c_void_p, c_int, PD]
        L.sph_phase_name.argtypes = [c_int]
        L.sph_phase_name.restype = c_char_p
        n = 11
        out = np.zeros(n)
        self._ok(L.sph_profile_phases(self._h, int(nsteps), out.ctypes.data_as(PD)))
        return {L.sph_phase_name(k).decode(): float(out[k]) for k in range(n)}

    # --- state ---
    def field(self, name):
        out = np.empty(self.N, dtype=np.float64)
        self._ok(lib().sph_read_field(self._h, FIELDS.index(name), out.ctypes.data_as(PD)))
        return out

    def set_field(self, name, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        assert a.shape == (self.N,)
        self._ok(lib().sph_write_field(self._h, FIELDS.index(name), a.ctypes.data_as(PD)))

    def type(self):
        out = np.empty(self.N, dtype=np.int32)
        self._ok(lib().sph_read_type(self._h, out.ctypes.data_as(PI)))
        return out

    def colloid_field(self, name):
        out = np.zeros(max(self.ncoll, 0), dtype=np.float64)
        if self.ncoll:
            self._ok(lib().sph_read_colloid_field(self._h, COLLOID_FIELDS.index(name), out.ctypes.data_as(PD)))
        return out

    def wall_forces(self):
        """(nboxes, 2 walls, 3) wall forces."""
        out = np.zeros(6 * self.nboxes, dtype=np.float64)
        self._ok(lib().sph_read_wall_forces(self._h, out.ctypes.data_as(PD)))
        return out.reshape(self.nboxes, 2, 3)

    def export_cells(self):
        i0 = self._info[0]
        pc = np.empty(i0["N"], dtype=np.int32)
        pi = np.empty(i0["N"], dtype=np.int32)
        cs = np.empty(i0["Ntotal_cells"], dtype=np.int32)
        ce = np.empty(i0["Ntotal_cells"], dtype=np.int32)
        self._ok(lib().sph_export_cells(self._h, pc.ctypes.data_as(PI), pi.ctypes.data_as(PI),
                                        cs.ctypes.data_as(PI), ce.ctypes.data_as(PI)))
        return dict(particle_cell=pc, particle_index=pi, cell_start=cs, cell_end=ce)

    def export_colloid_cells(self):
        i0 = self._info[0]
        n, m = i0["N_colloids"], i0["Ntotal_cells_colloids"]
        a = [np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(m, np.int32), np.zeros(m, np.int32)]
        self._ok(lib().sph_export_colloid_cells(self._h, *[x.ctypes.data_as(PI) for x in a]))
        return dict(coll_cell=a[0], coll_index=a[1], coll_cell_start=a[2], coll_cell_end=a[3])

    def kinetic_energy(self):
        out = np.zeros(self.nboxes, dtype=np.float64)
        self._ok(lib().sph_kinetic_energy(self._h, out.ctypes.data_as(PD)))
        return out

    def tuning(self):
        t = SphTuning()
        self._ok(lib().sph_get_tuning(self._h, ctypes.byref(t)))
        return {"list_threads_per_cell": t.list_threads_per_cell, "density_block": t.density_block}

    def set_tuning(self, list_threads_per_cell=32, density_block=128):
        t = SphTuning(list_threads_per_cell, density_block)
        self._ok(lib().sph_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, cache_path=None):
        """Pick the fastest launch geometry (cached per GPU, dim, overlap and size when a
        cache file is given); returns it.  The simulation state is not changed."""
        t = SphTuning()
        self._ok(lib().sph_autotune(self._h, os.fsencode(cache_path) if cache_path else None,
                                    ctypes.byref(t)))
        return {"list_threads_per_cell": t.list_threads_per_cell, "density_block": t.density_block}

    def observe(self):
        """Add one sample of every box's observables (asynchronous)."""
        self._ok(lib().sph_observe(self._h))

    def observables(self):
        """(nboxes x 4 time averages in OBSERVABLES order, number of samples)."""
        out = np.zeros((self.nboxes, len(OBSERVABLES)), dtype=np.float64)
        n = ctypes.c_longlong(0)
        self._ok(lib().sph_observables(self._h, out.ctypes.data_as(PD), ctypes.byref(n)))
        return out, n.value

    def reset_observables(self):
        self._ok(lib().sph_reset_observables(self._h))

    def save_checkpoint(self, path):
        """Binary checkpoint of the full state (bit-exact restart)."""
        self._ok(lib().sph_save_checkpoint(self._h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Restore a checkpoint written by a system built from the same input."""
        self._ok(lib().sph_load_checkpoint(self._h, os.fsencode(path)))
