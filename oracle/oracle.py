"""ctypes binding of the CPU FP64 oracle (oracle/sph_oracle.c) -- test infrastructure.

Only the tests, the smoke check and the CPU-baseline leg of bench.py use this module, as
the checker or as the timed CPU baseline.  It also reads the binary dumps written by the
reference program's own CUDA build (oracle/ref_harness.cu).
"""
import ctypes
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ref_sph")

# double-field ids, same order as the enum in sph_oracle.c
DFIELDS = [
    "x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "dens", "press", "mass",
    "cxx", "cxy", "cyy", "cxz", "cyz", "czz", "dcdt_xx", "dcdt_xy", "dcdt_yy",
    "dcdt_xz", "dcdt_yz", "dcdt_zz", "gxx", "gxy", "gxz", "gyx", "gyy", "gyz",
    "gzx", "gzy", "gzz", "coll_x", "coll_y", "coll_z", "coll_vx", "coll_vy",
    "coll_vz", "coll_omegax", "coll_omegay", "coll_omegaz", "coll_theta",
    "coll_quat0", "coll_quatx", "coll_quaty", "coll_quatz", "fx_colloid",
    "fy_colloid", "fz_colloid", "tx_colloid", "ty_colloid", "tz_colloid",
    "fx_wall", "fy_wall", "fz_wall", "x_center", "y_center", "z_center",
]
IFIELDS = [
    "type", "particle_cell", "particle_index", "cell_start", "cell_end", "walls_list",
    "walls_start", "colloids_list", "colloids_start", "coll_cell", "coll_index",
    "coll_cell_start", "coll_cell_end",
]
INFO_INTS = [
    "N", "dim", "wall", "Ncells0", "Ncells1", "Ncells2", "Ntotal_cells", "Nwalls",
    "Nlist_walls", "N_colloids", "Nlist_colloids", "Ncells_colloids0", "Ncells_colloids1",
    "Ncells_colloids2", "Ntotal_cells_colloids", "step",
]
INFO_DBLS = [
    "rcut", "rcutsq", "rcut_inv", "cw", "c_gradw", "csq", "rho0", "a", "b", "nkT", "tau",
    "dt", "cell_size0", "cell_size1", "cell_size2", "wall_width", "y_bottom", "y_top",
    "V_bottom", "V_top", "coll_R", "coll_mass", "coll_I", "rcuton_coll_rep_sq",
    "rcutoff_coll_rep_sq", "r0_magnet_sq", "F0_rep", "tau_rep", "F0_magnet",
    "omega_magnet", "ky", "beta_max", "L0", "L1", "L2", "cell_colloids_size0",
    "cell_colloids_size1", "cell_colloids_size2", "t0", "kinetic_energy",
]

_lib = None


def build():
    """Compile liboracle.so (gcc, OpenMP, -ffp-contract=off)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE, "_build/liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, cp, sz = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t
        L.orc_create_from_file.restype = vp
        L.orc_create_from_file.argtypes = [cp, cp, cp, sz]
        L.orc_destroy.argtypes = [vp]
        for name in ["orc_calculate_density", "orc_calculate_pressure",
                     "orc_calculate_vel_gradient", "orc_kernel_forces",
                     "orc_calculate_external_forces", "orc_kernel_dcdt",
                     "orc_calculate_force_walls", "orc_vv_step1", "orc_vv_step2"]:
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        L.orc_neighbours_search.argtypes = [vp]
        L.orc_neighbours_search.restype = ctypes.c_int
        L.orc_calculate_forces.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.orc_calculate_force_colloids.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.orc_run.argtypes = [vp, ctypes.c_int]
        L.orc_run.restype = ctypes.c_int
        L.orc_dfield.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_dfield.argtypes = [vp, ctypes.c_int]
        L.orc_field_len.argtypes = [vp, ctypes.c_int]
        L.orc_ifield.restype = ctypes.POINTER(ctypes.c_int)
        L.orc_ifield.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.orc_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        L.orc_W.argtypes = [vp, ctypes.c_double]
        L.orc_W.restype = ctypes.c_double
        L.orc_gradW.argtypes = [vp, ctypes.c_double]
        L.orc_gradW.restype = ctypes.c_double
        L.orc_kinetic_energy.argtypes = [vp]
        L.orc_kinetic_energy.restype = ctypes.c_double
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_set_threads.restype = ctypes.c_int
        L.orc_magnetic_mom.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_magnetic_mom.argtypes = [vp]
        _lib = L
    return _lib


def set_threads(n):
    return lib().orc_set_threads(int(n))


class Oracle:
    """One simulation box held by the CPU oracle (the reference's class_system state)."""

    def __init__(self, input_path, particles_path=None):
        msg = ctypes.create_string_buffer(256)
        p = particles_path.encode() if particles_path else None
        self._h = lib().orc_create_from_file(input_path.encode(), p, msg, 256)
        if not self._h:
            raise ValueError("oracle setup failed: " + msg.value.decode())

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- step methods (class_system names) ---
    def neighbours_search(self):
        return lib().orc_neighbours_search(self._h)

    def calculate_density(self):
        lib().orc_calculate_density(self._h)

    def calculate_pressure(self):
        lib().orc_calculate_pressure(self._h)

    def calculate_vel_gradient(self):
        lib().orc_calculate_vel_gradient(self._h)

    def kernel_forces(self):
        lib().orc_kernel_forces(self._h)

    def calculate_external_forces(self):
        lib().orc_calculate_external_forces(self._h)

    def kernel_dcdt(self):
        lib().orc_kernel_dcdt(self._h)

    def calculate_force_walls(self):
        lib().orc_calculate_force_walls(self._h)

    def magnetic_moment(self, t):
        w = self.info()["omega_magnet"]
        return np.array([np.cos(w * t), np.sin(w * t), 0.0])

    def calculate_force_colloids(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        lib().orc_calculate_force_colloids(self._h, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def calculate_forces(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        lib().orc_calculate_forces(self._h, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def vv_step1(self):
        lib().orc_vv_step1(self._h)

    def vv_step2(self):
        lib().orc_vv_step2(self._h)

    def run(self, nsteps):
        """main.cu loop: first call also does the initial search + forces (step 0)."""
        return lib().orc_run(self._h, int(nsteps))

    def W(self, r):
        return lib().orc_W(self._h, float(r))

    def gradW(self, r):
        return lib().orc_gradW(self._h, float(r))

    def kinetic_energy(self):
        return lib().orc_kinetic_energy(self._h)

    # --- state access (copies) ---
    def field(self, name):
        k = DFIELDS.index(name)
        n = lib().orc_field_len(self._h, k)
        p = lib().orc_dfield(self._h, k)
        if n <= 0 or not p:
            return np.zeros(0)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def ifield(self, name):
        k = IFIELDS.index(name)
        n = ctypes.c_int(0)
        p = lib().orc_ifield(self._h, k, ctypes.byref(n))
        if n.value <= 0 or not p:
            return np.zeros(0, dtype=np.int32)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def set_field(self, name, values):
        k = DFIELDS.index(name)
        n = lib().orc_field_len(self._h, k)
        p = lib().orc_dfield(self._h, k)
        np.ctypeslib.as_array(p, shape=(n,))[:] = np.asarray(values, dtype=np.float64)

    def info(self):
        iv = (ctypes.c_int * 16)()
        dv = (ctypes.c_double * 40)()
        lib().orc_info(self._h, iv, dv)
        out = dict(zip(INFO_INTS, list(iv)))
        out.update(dict(zip(INFO_DBLS, list(dv))))
        return out


def read_ref_dump(path):
    """Read one binary dump of the reference build (ref_harness.cu `put` records)."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        name = data[off:off + 32].split(b"\0", 1)[0].decode()
        code, esz, n = struct.unpack_from("<iiq", data, off + 32)
        off += 48
        nb = n * esz
        dt = {(0, 8): np.float64, (0, 4): np.float32, (1, 4): np.int32}[(code, esz)]
        out[name] = np.frombuffer(data[off:off + nb], dtype=dt).copy()
        off += nb
    return out
