"""The engine's host-side set-up against the oracle's, on the CPU.

Both restate class_system::read_input / constructor / initialize of the reference
(src/system_read_input.cpp, system_constructor.cpp, system_initialize.cpp,
system_initialize_particles_new_sim.cpp, system_initialize_particles_old_sim.cpp)
independently, in C++ (product) and C (oracle); the initial state and the derived
constants must agree bit for bit.  Also checks that both parsers accept and reject the
same input files, including the reference's own sample input.
"""
import os

import numpy as np
import pytest

import make_golden as mg
import oracle
import sph_b200
import sph_input

REF_SAMPLE = dict(  # the values of the reference's src/input (2D, 75^2, 2 colloids)
    N=(75, 75), L=(25.0, 25.0), dim=2, dt=0.0025, t0=0.0, Nsteps=1000000, overlap=4.0,
    rho=1.0, c=1.0, P0=0.9, eta=0.1, zeta=0.0, np=10.0, kT=0.001, tau=10.0,
    ext_force_type=0, ext_force=(1.0, 0.0), wall=0, Vwall_bottom=0.01, Vwall_top=-0.01,
    N_colloids=2, coll_R=1.0, coll_rho=1.0, coll_move=0, coll_x=((12.5, 12.5), (14.6, 12.5)),
    coll_repulsion_cuton=0.0, F0_repulsion=0.02115, tau_repulsion=1000.0,
    cutoff_magnetic=3.0, F0_magnetic=1.63, omega_magnetic=0.003, new_sim=0)

CASES = dict(mg.CASES)
CASES["ref_sample"] = REF_SAMPLE
CASES["walls3d_colloids"] = dict(N=(32, 32, 32), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0,
                                 wall=1, N_colloids=2, coll_R=3.0 / 32,
                                 coll_x=((0.3, 0.5, 0.5), (0.7, 0.5, 0.45)),
                                 tau_repulsion=4.0, cutoff_magnetic=0.3)
CASES["noninteger_overlap"] = dict(N=(40, 30), L=(1.0, 0.75), dim=2, overlap=3.5, wall=1)

INFO_KEYS = {"N": "N", "rcut": "rcut", "cw": "cw", "c_gradw": "c_gradw", "csq": "csq",
             "rho0": "rho0", "a": "a", "b": "b", "nkT": "nkT", "wall_width": "wall_width",
             "coll_mass": "coll_mass", "coll_I": "coll_I", "y_top": "y_top"}


def setup_case(name, workdir):
    spec = CASES[name]
    if name in mg.CASES:
        mg.case_dir(name, workdir)
    else:
        sph_input.write_input(os.path.join(workdir, "input"), **spec)
    pp = os.path.join(workdir, "input_particles.in")
    return os.path.join(workdir, "input"), (pp if os.path.exists(pp) else None)


@pytest.mark.parametrize("name", list(CASES))
def test_host_setup_matches_oracle(name, workdir):
    inp, pp = setup_case(name, workdir)
    arrays, info = sph_b200.host_setup(inp, pp)
    o = oracle.Oracle(inp, pp)
    oi = o.info()
    for k_e, k_o in INFO_KEYS.items():
        assert info[k_e] == oi[k_o], k_e
    assert info["Ncells"] == [oi["Ncells0"], oi["Ncells1"], oi["Ncells2"]]
    assert info["cell_size"] == [oi["cell_size0"], oi["cell_size1"], oi["cell_size2"]]
    dim = oi["dim"]
    for f in ["x", "y", "vx", "vy", "mass", "cxx", "cxy", "cyy"] + (
            ["z", "vz", "cxz", "cyz", "czz"] if dim == 3 else []):
        assert np.array_equal(arrays[f], o.field(f)), f
    assert np.array_equal(arrays["type"], o.ifield("type"))
    if oi["wall"]:
        assert np.array_equal(arrays["walls_list"], o.ifield("walls_list"))
        assert np.array_equal(arrays["walls_start"], o.ifield("walls_start"))
    if oi["N_colloids"]:
        assert np.array_equal(arrays["colloids_list"], o.ifield("colloids_list"))
        assert np.array_equal(arrays["colloids_start"], o.ifield("colloids_start"))
        for f in ["x_center", "y_center"] + (["z_center"] if dim == 3 else []):
            assert np.array_equal(arrays[f], o.field(f)), f


BAD = {
    "missing_key": lambda t: "\n".join(l for l in t.splitlines() if not l.startswith("tau ")),
    "dim_vs_N": lambda t: t.replace("dim 2", "dim 3"),
    "coll_count": lambda t: t.replace("N_colloids 2", "N_colloids 3"),
    "overlapping": lambda t: t.replace("coll_x 14.6 12.5", "coll_x 13.0 12.5"),
    "outside_box": lambda t: t.replace("coll_x 14.6 12.5", "coll_x 26.0 12.5"),
    "ext_type": lambda t: t.replace("ext_force_type 0", "ext_force_type 4"),
    "cells_too_big": lambda t: t.replace("overlap 4.0", "overlap 30.0"),
}


@pytest.mark.parametrize("case", list(BAD))
def test_both_parsers_reject_the_same_inputs(case, workdir):
    text = sph_input.make_input(**REF_SAMPLE)
    path = os.path.join(workdir, "input")
    with open(path, "w") as f:
        f.write(BAD[case](text))
    with pytest.raises(ValueError):
        oracle.Oracle(path)
    with pytest.raises(sph_b200.SphError):
        sph_b200.host_setup(path)


def test_reference_z_overlap_quirk(workdir):
    # the 3D overlap check takes the z separation from y (system_read_input.cpp:485):
    # colloids stacked in z with equal x, y are rejected by both parsers
    spec = dict(N=(32, 32, 32), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, N_colloids=2,
                coll_R=0.05, coll_x=((0.5, 0.5, 0.3), (0.5, 0.5, 0.7)), tau_repulsion=4.0,
                cutoff_magnetic=0.3)
    path = os.path.join(workdir, "input")
    sph_input.write_input(path, **spec)
    with pytest.raises(ValueError):
        oracle.Oracle(path)
    with pytest.raises(sph_b200.SphError):
        sph_b200.host_setup(path)


def test_suspension_spec_is_accepted(tmp_path):
    """The 96^3 suspension input: 32 seeded colloids the reference's own checks accept
    (overlap check as written, wall clearance, colloid coarse grid of >= 3 cells), every
    shell particle inside the cell grid at the first search, reproducible from its seed."""
    import sph_b200
    import sph_input

    spec = sph_input.suspension_spec()
    assert spec == sph_input.suspension_spec() and len(spec["coll_x"]) == 32
    path = str(tmp_path / "input")
    sph_input.write_input(path, **spec)
    a, info = sph_b200.host_setup(path)
    assert info["N_colloids"] == 32 and min(info["Ncells_colloids"]) >= 3
    cs, ww, nc = info["cell_size"], info["wall_width"], info["Ncells"]
    cx = np.floor(a["x"] / cs[0]).astype(int)
    cy = np.floor((a["y"] + ww) / cs[1]).astype(int)
    cz = np.floor(a["z"] / cs[2]).astype(int)
    cx[cx == nc[0]] -= 1
    cz[cz == nc[2]] -= 1
    cell = (cz * nc[1] + cy) * nc[0] + cx
    assert cell.min() >= 0 and cell.max() < info["Ntotal_cells"]
