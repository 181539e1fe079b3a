"""Output writers (include/sph_io.h) against the C library's own printf: every file is
byte-identical to what the reference's fprintf loops write (src/system_print_particles.cpp,
system_print_walls.cpp, system_print_colloids.cpp, system_print_particles_gradv.cpp,
system_print_macro_vars.cu).  Host code only: no GPU."""
import ctypes
import math
import os

import numpy as np
import pytest

import sph_b200

libc = ctypes.CDLL(None)
libc.snprintf.restype = ctypes.c_int

REAL = b"%.8lf"


def c_format(fmt, *args):
    buf = ctypes.create_string_buffer(8192)
    cargs = [ctypes.c_double(a) if isinstance(a, float) else ctypes.c_int(a) for a in args]
    n = libc.snprintf(buf, len(buf), fmt, *cargs)
    assert 0 <= n < len(buf)
    return buf.value.decode()


def P(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def I(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int))


@pytest.fixture(scope="module")
def lib():
    L = sph_b200.lib()
    L.sph_format_fixed8.restype = ctypes.c_int
    L.sph_format_fixed8.argtypes = [ctypes.c_double, ctypes.c_char_p]
    for name in ("sph_write_micro", "sph_write_walls", "sph_write_colloids", "sph_write_gradv",
                 "sph_append_macro"):
        getattr(L, name).restype = ctypes.c_int
    return L


def fixed8(lib, x):
    buf = ctypes.create_string_buffer(400)
    n = lib.sph_format_fixed8(ctypes.c_double(x), buf)
    assert n == len(buf.value)
    return buf.value.decode()


def edge_values():
    vals = [0.0, -0.0, 1.0, -1.0, 0.5, 1e-9, -1e-9, 5e-9, -5e-9, 4.999999999e-9, 1.5e-8,
            2.5e-8, 0.123456785, 0.123456775, 2.0 ** -9, 3 * 2.0 ** -9, -(2.0 ** -9),
            2.0 ** -30, 5e-324, -5e-324, 2.2250738585072014e-308, 8.99999999e10, 9.0e10,
            -9.0e10, 1e15, 1.7976931348623157e308, -1.7976931348623157e308, math.inf,
            -math.inf, math.nan, 123456.78901234567, 0.999999995, 0.999999994999,
            1.000000005, 99999999.999999995]
    # exact ties at the ninth decimal: k / 2^9 has nine decimals ending in 5
    vals += [k / 512.0 for k in range(-2048, 2048, 7)]
    return vals


def test_fixed8_matches_printf_on_edges(lib):
    for x in edge_values():
        assert fixed8(lib, x) == c_format(b"%.8f", x), x


def test_fixed8_matches_printf_random(lib):
    rng = np.random.default_rng(3)
    mant = rng.uniform(-1.0, 1.0, 20000)
    expo = rng.integers(-40, 40, 20000)
    xs = np.ldexp(mant, expo)
    # random bit patterns too (finite ones)
    bits = rng.integers(0, 2 ** 63, 5000, dtype=np.int64).view(np.float64)
    xs = np.concatenate([xs, bits[np.isfinite(bits)]])
    for x in xs:
        assert fixed8(lib, float(x)) == c_format(b"%.8f", float(x)), repr(float(x))


def micro_reference(dim, cols, type_):
    n = len(type_)
    if dim == 2:
        fmt = b"%d " + b" ".join([REAL] * 7) + b" %d " + b" ".join([REAL] * 3) + b" \n"
        order = ["x", "y", "vx", "vy", "mass", "dens", "press", "T", "cxx", "cxy", "cyy"]
    else:
        fmt = b"%d " + b" ".join([REAL] * 9) + b" %d " + b" ".join([REAL] * 6) + b"\n"
        order = ["x", "y", "z", "vx", "vy", "vz", "mass", "dens", "press", "T", "cxx", "cxy",
                 "cyy", "cxz", "cyz", "czz"]
    out = []
    for i in range(n):
        args = [i] + [int(type_[i]) if k == "T" else float(cols[k][i]) for k in order]
        out.append(c_format(fmt, *args))
    return "".join(out)


@pytest.mark.parametrize("dim,n", [(2, 700), (3, 500), (3, 70000)])
def test_micro_file(lib, tmp_path, dim, n):
    rng = np.random.default_rng(dim * 100 + n)
    names = ["x", "y", "z", "vx", "vy", "vz", "mass", "dens", "press", "cxx", "cxy", "cyy",
             "cxz", "cyz", "czz"]
    cols = {k: rng.normal(0, 10.0 ** rng.integers(-6, 4), n) for k in names}
    cols["x"][:3] = [-0.0, 2.0 ** -9, 1e12]
    type_ = rng.integers(0, 40, n).astype(np.int32)
    path = str(tmp_path / "micro-7.dat")
    st = lib.sph_write_micro(path.encode(), dim, n, *[P(cols[k]) for k in names[:9]], I(type_),
                             *[P(cols[k]) for k in names[9:]])
    assert st == 0
    got = open(path).read()
    if n > 5000:  # spot-check the chunk seams of a large file against printf row by row
        lines = got.splitlines(keepends=True)
        assert len(lines) == n
        for i in [0, 1, 32767, 32768, 32769, 65535, 65536, n - 1]:
            sub = {k: v[i:i + 1] for k, v in cols.items()}
            ref = micro_reference(dim, sub, type_[i:i + 1]).split(" ", 1)[1]
            assert lines[i] == "%d %s" % (i, ref)
    else:
        assert got == micro_reference(dim, cols, type_)


@pytest.mark.parametrize("dim", [2, 3])
def test_walls_colloids_gradv_files(lib, tmp_path, dim):
    rng = np.random.default_rng(dim)
    # walls: "i fx fy [fz]"
    w = [rng.normal(size=2) for _ in range(3)]
    p = str(tmp_path / "walls-3.dat")
    assert lib.sph_write_walls(p.encode(), dim, 2, P(w[0]), P(w[1]), P(w[2])) == 0
    fmt = b"%d " + b" ".join([REAL] * dim) + b"\n"
    ref = "".join(c_format(fmt, i, *[float(w[k][i]) for k in range(dim)]) for i in range(2))
    assert open(p).read() == ref
    # colloids: 15 columns in the 3D order, 2D subset x y vx vy omegaz fx fy tz
    nc = 5
    cols = [rng.normal(size=nc) for _ in range(15)]
    arr = (ctypes.POINTER(ctypes.c_double) * 15)(*[P(c) for c in cols])
    p = str(tmp_path / "colloids-3.dat")
    assert lib.sph_write_colloids(p.encode(), dim, nc, arr) == 0
    pick = [0, 1, 3, 4, 8, 9, 10, 14] if dim == 2 else list(range(15))
    fmt = b"%d " + b" ".join([REAL] * len(pick)) + b"\n"
    ref = "".join(c_format(fmt, i, *[float(cols[k][i]) for k in pick]) for i in range(nc))
    assert open(p).read() == ref
    # gradv
    n = 9
    xyz = [rng.normal(size=n) for _ in range(3)]
    g = [rng.normal(size=n) for _ in range(9)]
    garr = (ctypes.POINTER(ctypes.c_double) * 9)(*[P(c) for c in g])
    p = str(tmp_path / "gradv-3.dat")
    assert lib.sph_write_gradv(p.encode(), dim, n, P(xyz[0]), P(xyz[1]), P(xyz[2]), garr) == 0
    gp = [0, 1, 3, 4] if dim == 2 else list(range(9))
    fmt = b"%d " + b" ".join([REAL] * (dim + len(gp))) + b"\n"
    ref = "".join(c_format(fmt, i, *[float(xyz[k][i]) for k in range(dim)],
                           *[float(g[k][i]) for k in gp]) for i in range(n))
    assert open(p).read() == ref


def test_macro_file(lib, tmp_path):
    p = str(tmp_path / "macro.dat")
    lib.sph_append_macro.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_double]
    assert lib.sph_append_macro(p.encode(), 0, 0.25) == 0
    assert lib.sph_append_macro(p.encode(), 5, 1.0 / 3.0) == 0
    assert open(p).read() == c_format(b"%d %f\n", 0, 0.25) + c_format(b"%d %f\n", 5, 1.0 / 3.0)
    assert lib.sph_append_macro(p.encode(), 0, 2.0) == 0  # step 0 truncates
    assert open(p).read() == c_format(b"%d %f\n", 0, 2.0)


def test_writer_rejects_bad_arguments(lib, tmp_path):
    p = str(tmp_path / "x.dat").encode()
    z = np.zeros(1)
    assert lib.sph_write_walls(p, 4, 1, P(z), P(z), P(z)) != 0
    assert lib.sph_write_walls(str(tmp_path / "no" / "dir.dat").encode(), 2, 1, P(z), P(z),
                               P(z)) == 9  # SPH_ERR_IO


@pytest.mark.parametrize("dim,n", [(2, 900), (3, 40000)])
def test_restart_file_writer(tmp_path, dim, n):
    """sph_write_restart writes the same bytes as the reference-format writer in
    sph_input.write_particles (every value rounded to float, "%.9g"), and the engine's own
    restart reader (host set-up, no GPU) reads back exactly those floats."""
    import sph_input

    rng = np.random.default_rng(dim * 7 + n)
    a = {k: rng.normal(0, 10.0 ** rng.integers(-7, 3), n)
         for k in ["x", "y", "z", "vx", "vy", "vz", "mass", "cxx", "cxy", "cyy", "cxz", "cyz",
                   "czz"]}
    a["x"] = rng.uniform(0.0, 1.0, n)
    a["y"] = rng.uniform(0.0, 1.0, n)
    a["z"] = rng.uniform(0.0, 1.0, n) if dim == 3 else np.zeros(n)
    a["mass"] = np.full(n, 1.0 / n)
    a["type"] = np.zeros(n, dtype=np.int32)
    a["vx"][:4] = [-0.0, 1e-45, 3.4e38, 0.1]
    p_c = str(tmp_path / "c.in")
    p_py = str(tmp_path / "py.in")
    sph_b200.write_restart(p_c, dim, a)
    sph_input.write_particles(p_py, dim, a["x"], a["y"], a["z"], a["vx"], a["vy"], a["vz"],
                              a["mass"], a["type"], a["cxx"], a["cxy"], a["cyy"], a["cxz"],
                              a["cyz"], a["czz"])
    assert open(p_c).read() == open(p_py).read()
    side = int(round(n ** (1.0 / dim)))
    inp = str(tmp_path / "input")
    sph_input.write_input(inp, N=(side,) * dim, L=(1.0,) * dim, dim=dim, overlap=3.0, new_sim=1)
    got, info = sph_b200.host_setup(inp, p_c)
    assert info["N"] == n
    f32 = lambda v: np.asarray(v, dtype=np.float32).astype(np.float64)
    for k in ["x", "y", "vx", "vy", "cxy"] + (["z", "vz", "czz"] if dim == 3 else []):
        assert np.array_equal(got[k], f32(a[k])), k


def test_seeded_start(tmp_path):
    """write_seeded_start: the lattice of new_sim = 0 with seeded fluid velocities in
    [-vmax, vmax], walls at rest, every value rounded to float as the reference reads it."""
    import sph_input

    spec = dict(N=(12, 12, 12), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1,
                Vwall_bottom=-0.5, Vwall_top=0.5, dt=2e-5)
    inp, pp, n = sph_b200.write_seeded_start(str(tmp_path), spec, seed=3, vmax=0.01)
    lattice, _ = sph_b200.host_setup(str(tmp_path / "input_lattice"))
    got, info = sph_b200.host_setup(inp, pp)
    assert info["N"] == n == len(lattice["x"])
    f32 = lambda v: np.asarray(v, dtype=np.float32).astype(np.float64)
    for k in ["x", "y", "z", "mass", "cxx", "cyy"]:
        assert np.array_equal(got[k], f32(lattice[k])), k
    assert np.array_equal(got["type"], lattice["type"])
    fluid = got["type"] == 0
    for k in ["vx", "vy", "vz"]:
        v = got[k]
        assert np.all(np.abs(v[fluid]) <= 0.01) and np.all(v[~fluid] == 0.0)
        assert np.std(v[fluid]) > 0.004
    other = tmp_path / "again"
    other.mkdir()
    sph_b200.write_seeded_start(str(other), spec, seed=3, vmax=0.01)
    assert open(pp).read() == open(str(other / "input_particles.in")).read()
    assert "new_sim 1" in open(inp).read() and sph_input.DEFAULTS["new_sim"] == 0
