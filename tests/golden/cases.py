"""Parity cases shared by the fixture generator and the tests (seeded, small).

Each case names a mesh, an initial state and the reference's Solver_Config settings.  The sizes
are chosen so that the reference and the C oracle finish in well under a second.
"""
import numpy as np

import cfd_solver_withcuda_b200 as cb

GAMMA = 1.4

CASES = {
    # Sod shock tube on a reduced 100x4 box (full size 400x4 is in the GPU tests vs the oracle).
    "sod_roe1_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=3, is_second_order=0,
                         time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0, steps=80),
    "sod_roe2_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=3, is_second_order=1,
                         time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0, steps=80),
    "sod_llf1_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=1, is_second_order=0,
                         time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0, steps=80),
    "sod_roe2_explicit": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=3,
                              is_second_order=1, time_accurate=0, cfl=0.4, inlet_rho=1.0, inlet_p=1.0, steps=60),
    "sod_roe1_full_t02": dict(mesh=("box", 400, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=3,
                              is_second_order=0, time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0, steps=100000,
                              t_end=0.2),
    # Half cylinder O-grid, M=3 freestream, Roe-2O + reference MinMod, RK3 with local dt.
    "cyl_roe2_lts": dict(mesh=("half_cylinder", 48, 24, 1.0, 4.0, 1.005), ic="freestream", mach=3.0,
                         dissipation_type=3, is_second_order=1, time_accurate=1, local_time_stepping=1, cfl=0.8,
                         inlet_rho=1.0, inlet_p=1.0 / GAMMA, steps=40, amr=(0.05, 0.1)),
    # 15-degree ramp, bounding-box boundary classification, Roe-1O explicit.
    "ramp_roe1_explicit": dict(mesh=("ramp", 52, 18, 3.0, 1.0, 1.0, 15.0), ic="freestream", mach=2.0,
                               dissipation_type=3, is_second_order=0, time_accurate=0, cfl=0.5, inlet_rho=1.0,
                               inlet_p=1.0 / GAMMA, steps=40),
    # Mixed tri/quad bump channel (triangles take the reference's degenerate limiter path).
    "bump_roe2_rk3": dict(mesh=("bump", 40, 16, 3.0, 1.0, 0.1, 3, 0.3, 11, 1), ic="freestream", mach=1.6,
                          dissipation_type=3, is_second_order=1, time_accurate=1, cfl=0.5, inlet_rho=1.0,
                          inlet_p=1.0 / GAMMA, steps=30, amr=(0.1, 0.2)),
    # WENO path (src/WENO2D.cpp): component-wise on Sod with RK3, characteristic (Is_Char) on the
    # O-grid with local dt, and the explicit method on the mixed bump, where the reference falls
    # back to the 1O/2O residual because the mesh has triangles.
    "sod_weno_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=3, is_second_order=0,
                         time_accurate=1, cfl=0.4, inlet_rho=1.0, inlet_p=1.0, steps=6, weno=1),
    "pulse_weno_rk3": dict(mesh=("box", 40, 20, 0.0, 2.0, 0.0, 1.0), ic="pulse", mach=1.5, dissipation_type=3,
                           is_second_order=0, time_accurate=1, cfl=0.4, inlet_rho=1.0, inlet_p=1.0 / GAMMA, steps=18,
                           weno=1),
    "sod_weno_char_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=3,
                              is_second_order=0, time_accurate=1, local_time_stepping=1, cfl=0.4, inlet_rho=1.0,
                              inlet_p=1.0, steps=10, weno=1, weno_characteristic=1),
    "bump_weno_explicit_fallback": dict(mesh=("bump", 40, 16, 3.0, 1.0, 0.1, 3, 0.3, 11, 1), ic="freestream",
                                        mach=1.6, dissipation_type=3, is_second_order=1, time_accurate=0, cfl=0.4,
                                        inlet_rho=1.0, inlet_p=1.0 / GAMMA, steps=20, weno=1),
    # The reference's other dissipation types (src/Net_Flux.cpp:74-91,109-126): MOVERS and
    # MOVERS_2O with and without Is_MOVERS_1 / Enable_Entropy_Fix, RICCA and RICCA_2O,
    # MOVERS_NWSC and MOVERS_NWSC_2O, on Sod, the O-grid, the ramp and the mixed bump.
    "sod_movers1_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=2,
                            is_second_order=0, time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0, steps=60),
    "sod_movers1_single_efix_explicit": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=2,
                                             is_second_order=0, time_accurate=0, cfl=0.4, inlet_rho=1.0, inlet_p=1.0,
                                             steps=60, movers_single_alpha=1, movers_entropy_fix=1),
    "cyl_movers2_efix_lts": dict(mesh=("half_cylinder", 48, 24, 1.0, 4.0, 1.005), ic="freestream", mach=3.0,
                                 dissipation_type=2, is_second_order=1, time_accurate=1, local_time_stepping=1,
                                 cfl=0.8, inlet_rho=1.0, inlet_p=1.0 / GAMMA, steps=30, movers_entropy_fix=1),
    "ramp_ricca1_explicit": dict(mesh=("ramp", 52, 18, 3.0, 1.0, 1.0, 15.0), ic="freestream", mach=2.0,
                                 dissipation_type=4, is_second_order=0, time_accurate=0, cfl=0.5, inlet_rho=1.0,
                                 inlet_p=1.0 / GAMMA, steps=30),
    "cyl_ricca2_lts": dict(mesh=("half_cylinder", 48, 24, 1.0, 4.0, 1.005), ic="freestream", mach=3.0,
                           dissipation_type=4, is_second_order=1, time_accurate=1, local_time_stepping=1, cfl=0.8,
                           inlet_rho=1.0, inlet_p=1.0 / GAMMA, steps=30),
    "sod_nwsc1_rk3": dict(mesh=("box", 100, 4, 0.0, 1.0, 0.0, 0.01), ic="sod", dissipation_type=5,
                          is_second_order=0, time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0, steps=60),
    "bump_nwsc2_rk3": dict(mesh=("bump", 40, 16, 3.0, 1.0, 0.1, 3, 0.3, 11, 1), ic="freestream", mach=1.6,
                           dissipation_type=5, is_second_order=1, time_accurate=1, cfl=0.5, inlet_rho=1.0,
                           inlet_p=1.0 / GAMMA, steps=30),
    # Reference subsonic inlet (energy form of src/Inlet_Boundary_Conditions.cpp:32) and the
    # empty subsonic exit, LLF.
    "bump_llf1_subsonic": dict(mesh=("bump", 30, 12, 3.0, 1.0, 0.05, 2, 0.2, 5, 0), ic="freestream", mach=0.5,
                               dissipation_type=1, is_second_order=0, time_accurate=1, cfl=0.4, inlet_rho=1.0,
                               inlet_p=1.0 / GAMMA, inlet_bc=1, exit_bc=1, steps=30),
}


def make_mesh(case):
    kind, *args = case["mesh"]
    if kind == "box":
        return cb.Mesh.box(*args)
    if kind == "half_cylinder":
        return cb.Mesh.half_cylinder(*args)
    if kind == "ramp":
        return cb.Mesh.ramp(*args)
    if kind == "bump":
        nx, ny, length, height, thick, nql, jit, seed, tri = args
        return cb.Mesh.bump(nx, ny, length, height, thick, nql, jit, seed, bool(tri))
    raise ValueError(kind)


def initial_state(case, mesh):
    """Conserved variables for all cells, ghosts included (a ghost starts as a copy of its owner
    cell; BCs overwrite it except where the reference's subsonic exit is a no-op)."""
    NP = mesh.n_physical
    xc = mesh.centers[:NP, 0]
    if case["ic"] == "sod":
        left = xc < 0.5
        U = cb.conserved_from_primitive(np.where(left, 1.0, 0.125), 0 * xc, 0 * xc, np.where(left, 1.0, 0.1))
    elif case["ic"] == "pulse":
        # Uniform stream at the inlet state with a smooth density pulse at uniform pressure.
        rho0, p = case["inlet_rho"], case["inlet_p"]
        u = case["mach"] * np.sqrt(GAMMA * p / rho0)
        yc = mesh.centers[:NP, 1]
        rho = rho0 + 0.2 * np.exp(-((xc - 0.6) ** 2 + (yc - 0.5) ** 2) / 0.02)
        U = cb.conserved_from_primitive(rho, np.full(NP, u), np.zeros(NP), np.full(NP, p))
    else:
        rho, p = case["inlet_rho"], case["inlet_p"]
        a = np.sqrt(GAMMA * p / rho)
        u = case["mach"] * a
        U = cb.conserved_from_primitive(np.full(NP, rho), np.full(NP, u), np.zeros(NP), np.full(NP, p))
    full = np.zeros((mesh.n_total, 4))
    full[:NP] = U
    b = mesh.boundary
    full[b[:, 3]] = U[b[:, 1]]
    return full


def solver_config(case, **over):
    kw = dict(dissipation_type=case["dissipation_type"], is_second_order=case["is_second_order"],
              time_accurate=case["time_accurate"], local_time_stepping=case.get("local_time_stepping", 0),
              cfl=case["cfl"], limiter_zeta=case.get("limiter_zeta", 0.5), limiter_zeta1=case.get("limiter_zeta1", 0.5),
              inlet_rho=case["inlet_rho"], inlet_p=case["inlet_p"], inlet_bc=case.get("inlet_bc", 0),
              exit_bc=case.get("exit_bc", 0), weno=case.get("weno", 0),
              weno_characteristic=case.get("weno_characteristic", 0),
              movers_single_alpha=case.get("movers_single_alpha", 0),
              movers_entropy_fix=case.get("movers_entropy_fix", 0))
    kw.update(over)
    return cb.default_config(**kw)


def oracle_params(case, **over):
    kw = dict(dissipation_type=case["dissipation_type"], is_second_order=case["is_second_order"],
              time_accurate=case["time_accurate"], local_time_stepping=case.get("local_time_stepping", 0),
              cfl=case["cfl"], limiter_zeta=case.get("limiter_zeta", 0.5), limiter_zeta1=case.get("limiter_zeta1", 0.5),
              inlet_rho=case["inlet_rho"], inlet_p=case["inlet_p"], inlet_bc=case.get("inlet_bc", 0),
              exit_bc=case.get("exit_bc", 0), weno=case.get("weno", 0),
              weno_characteristic=case.get("weno_characteristic", 0),
              movers_single_alpha=case.get("movers_single_alpha", 0),
              movers_entropy_fix=case.get("movers_entropy_fix", 0))
    kw.update(over)
    return kw


def ref_params(case):
    """The case as the reference harness's named parameters (oracle/ref_harness.cpp refh_set_param)."""
    p = {"CFL": case["cfl"], "Time_Accurate": case["time_accurate"], "Dissipation_Type": case["dissipation_type"],
         "Is_Second_Order": case["is_second_order"], "Local_Time_Stepping": case.get("local_time_stepping", 0),
         "Limiter_Zeta": case.get("limiter_zeta", 0.5), "Limiter_Zeta1": case.get("limiter_zeta1", 0.5),
         "Inlet_Rho": case["inlet_rho"], "Inlet_P": case["inlet_p"],
         "Is_Inlet_SubSonic": 1 if case.get("inlet_bc", 0) == 1 else 0,
         "Is_Exit_SubSonic": 1 if case.get("exit_bc", 0) == 1 else 0,
         "Is_WENO": case.get("weno", 0), "Is_Char": case.get("weno_characteristic", 0),
         "Is_MOVERS_1": case.get("movers_single_alpha", 0), "Enable_Entropy_Fix": case.get("movers_entropy_fix", 0)}
    return p
