"""input.json files for the C++ host tests: a Dirichlet box with a voxel cube,
electrons, ions and (optionally) photoelectrons, in the reference's schema."""
import json
import math
from pathlib import Path

from fopis_b200 import config


def write_input(dirpath, n=25, ppc=4, photo=True, steps=5, drift=(0.0, 0.0, 0.0), secondary=False, dielectric=None,
                em=False, courant=0.5):
    """dielectric: the materials map (texture index -> material name) of a dielectric
    cube whose +x face carries texture 2 and the other faces texture 1. em: an
    "EM" run (solver_type) with 5 keV electrons at 1e12 m^-3, dx = 0.5 m and
    dt = courant dx / c."""
    d = Path(dirpath)
    d.mkdir(parents=True, exist_ok=True)
    (d / "objects").mkdir(exist_ok=True)
    text = config.box_obj_text([((-2, -2, -2), (2, 2, 2))])
    if dielectric:
        # box_obj_text writes f a/1/n ...; the normal index n = 2 is the +x face
        text = "\n".join(l.replace("/1/2", "/2/2") if l.startswith("f ") else l for l in text.splitlines()) + "\n"
        text = text.replace("vt 0.5 0.5\n", "vt 0.5 0.5\nvt 0.25 0.5\n")
    (d / "objects" / "cube.obj").write_text(text)
    dx, dt = config.plasma_units()
    dens, te = 1.0e7, 1.0
    if em:
        dx, dens, te = 0.5, 1.0e12, 5.0e3
        dt = courant * dx / config.CLIGHT
    plasma = {
        "Electron": {"type": "ambient", "mass": 1.0, "charge": -1.0, "density": dens, "temperature": te,
                     "drift_velocity": list(drift), "particle_per_cell": ppc},
        "Ion": {"type": "ambient", "mass": 100.0, "charge": 1.0, "density": dens, "temperature": 1.0,
                "drift_velocity": [0.0, 0.0, 0.0], "particle_per_cell": ppc,
                "injection_axis": [True, True, False, True, True, True]},
    }
    emit = {}
    if photo:
        vbar = math.sqrt(8.0 * config.E / (math.pi * config.ME))
        plasma["Photo"] = {"type": "photoelectron", "mass": 1.0, "charge": -1.0, "density": 1.0e7, "temperature": 0.2,
                           "particle_per_cell": ppc, "current_density": 10.0 * config.E * 1.0e7 * vbar / 4.0}
        emit = {"Photo": {}}
    if secondary:
        plasma["Secondary"] = {"type": "secondary", "mass": 1.0, "charge": -1.0, "density": 1.0e7, "temperature": 2.0,
                               "particle_per_cell": ppc}
        emit["Secondary"] = {}
    js = {
        "Environment": {"max_timestep": steps, "job_type": "new", "solver_type": "EM" if em else "ES",
                        "boundary": "DDDDDD",
                        "dimension": "3D", "nx": n, "ny": n, "nz": n, "proc_x": 1, "proc_y": 1, "proc_z": 1,
                        "dx": dx, "dt": dt},
        "Plasma": plasma,
        "Field": {"static_bfield": [0.0, 0.0, 0.0], "shine_vector": [-1.0, 0.0, 0.0]},
        "Object": {"Spacecraft": {"file_name": "objects/cube.obj",
                                  "surface_type": "dielectric" if dielectric else "perfect", "emit_particles": emit,
                                  "is_potential_fixed": False, "fixed_potential": 0.0,
                                  "initial_potential_offset": 0.0, **({"materials": dielectric} if dielectric else {})}},
        "Options": {"use_existing_capacity_matrix": False},
        "IO": {"plot_energy_width": 1},
    }
    path = d / "input.json"
    path.write_text(json.dumps(js, indent=2))
    return path
