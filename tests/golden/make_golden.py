"""Generates the golden fixtures in tests/golden/ from the reference's own CPU code.

Run in a container where the reference sources are present:
    python tests/golden/make_golden.py            # every case
    python tests/golden/make_golden.py a b ...    # only the named cases (the others stay as they are)
It builds oracle/_ref/libcfdref.so from the reference's src/*.cpp (oracle/Makefile), builds the
meshes with the mesh layer, runs the reference loop (src/Solver.cpp:94-125) through the harness,
and stores inputs and outputs as compressed .npz.  The fixtures travel with the repository, so
tests that use them never need the reference itself.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import cfd_solver_withcuda_b200 as cb  # noqa: E402
from oracle import refpy  # noqa: E402

from cases import CASES, make_mesh, initial_state, ref_params  # noqa: E402

LAX_CASES = ("cyl_roe2_lts", "sod_roe1_rk3", "ramp_roe1_explicit")


def main(only=None):
    refpy.build_ref()
    mpath = os.path.join(HERE, "manifest.json")
    manifest = {}
    if only and os.path.exists(mpath):
        with open(mpath) as f:
            manifest = json.load(f)
    for name, case in CASES.items():
        if only and name not in only:
            continue
        mesh = make_mesh(case)
        U0 = initial_state(case, mesh)
        r = refpy.RefRun(mesh, ref_params(case))
        r.set_state(U0)
        # Single entry-point results after the first BC + flux evaluation.
        r.L.refh_apply_bc()
        r.L.refh_net_flux()
        first = r.state()
        r = refpy.RefRun(mesh, ref_params(case))
        r.set_state(U0)
        n = r.iterate(case["steps"], case.get("t_end", 0.0))
        st = r.state()
        out = {
            "U0": U0,
            "first_net_flux": first["net_flux"], "first_dt": first["dt"],
            "first_ghost_U": first["U"][mesh.n_physical:],
            "U": st["U"], "prim": st["prim"], "dt": st["dt"], "net_flux": st["net_flux"], "delU": st["delU"],
            "error": r.error(), "total_time": np.array([r.total_time()]), "iterations": np.array([n]),
            "min_dt": np.array([r.min_dt()]),
        }
        if case.get("amr"):
            out["grad_rho"] = r.gradient(0)
            out["grad_p"] = r.gradient(4)
            ind, tags = r.amr(case["amr"][0], case["amr"][1])
            out["amr_indicator"] = ind
            out["amr_tags"] = tags
        geo = r.geometry()
        for k in ("neighbours", "face_normals", "face_lengths", "center_distances", "area", "inv_area", "centers"):
            out["geo_" + k] = geo[k]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        manifest[name] = {"iterations": int(n), "np": mesh.n_physical, "ng": mesh.n_ghost}
        print(name, manifest[name])
    # Lax_Fedrichs (src/Numerical_Method.cpp:459-481) after Apply_Boundary_Conditions and the net
    # flux, on the final states of three quad-mesh cases (its sweep reads earlier cells' new values).
    if not only or "lax_friedrichs_reference" in only:
        out = {}
        for name in LAX_CASES:
            case = CASES[name]
            mesh = make_mesh(case)
            U = np.load(os.path.join(HERE, name + ".npz"))["U"]
            r = refpy.RefRun(mesh, ref_params(case))
            r.set_state(U)
            r.L.refh_apply_bc()
            r.L.refh_net_flux()
            r.L.refh_lax_friedrichs()
            out[name + "_U0"] = U
            out[name + "_U"] = r.state()["U"]
        np.savez_compressed(os.path.join(HERE, "lax_friedrichs_reference.npz"), **out)
        manifest["lax_friedrichs_reference"] = {"cases": list(LAX_CASES)}
    # Ausm_Flux (src/Ausm_Flux.cpp:5-205) on a non-uniform state of the mixed bump mesh: the final
    # state of the bump_roe2_rk3 case.
    if only and "ausm_reference" not in only:
        with open(mpath, "w") as f:
            json.dump(manifest, f, indent=1, sort_keys=True)
        return
    case = CASES["bump_roe2_rk3"]
    mesh = make_mesh(case)
    U = np.load(os.path.join(HERE, "bump_roe2_rk3.npz"))["U"]
    r = refpy.RefRun(mesh, ref_params(case))
    r.set_state(U)
    r.L.refh_ausm_net_flux()
    np.savez_compressed(os.path.join(HERE, "ausm_reference.npz"), U=U, net_flux=r.state()["net_flux"])
    manifest["ausm_reference"] = {"np": mesh.n_physical}
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)
