"""C ABI boundary on CPU: the library loads, exports every symbol include/cfd_b200.h declares, and
the host-only parts (config reader, error paths) behave; no kernel runs here."""
import os
import re

import pytest

import cfd_solver_withcuda_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cfd_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfd_[A-Za-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = cb.lib()
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) == set(cb.SIGNATURES), set(syms) ^ set(cb.SIGNATURES)


def test_only_c_abi_is_exported():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", cb.LIB_PATH], capture_output=True, text=True).stdout
    names = [l.split()[-1] for l in out.splitlines() if l.strip()]
    assert names and all(n.startswith("cfd_") for n in names), [n for n in names if not n.startswith("cfd_")][:5]


def test_config_json_reference_schema(tmp_path):
    p = tmp_path / "Solver_Config.json"
    p.write_text("""{
      "TestCase": {"Test_Case": 1, "Test_Case_Name": "Half_Cylinder"},
      "Simulation": {"Initialize_Type": 0, "Total_Iterations": 20000, "CFL": 0.8, "Terminating_Time": 1000.0},
      "Solver": {"Dissipation_Type": 3, "Is_Second_Order": true, "Time_Accurate": true,
                 "Local_Time_Stepping": true, "Limiter_Type": "VanLeer", "Integrator": "SSPRK3",
                 "Reconstruction": "Primitive"},
      "LimiterCoefficients": {"Limiter_Zeta": 0.5, "Limiter_Zeta1": 0.25
       // "Epsilon": 1.0e-6
      },
      "BoundaryConditions": {"Is_Inlet_SubSonic": false, "Inlet_Rho": 1.0, "Inlet_P": 0.714285714}
    }""")
    c = cb.read_config_json(str(p))
    assert c.dissipation_type == 3 and c.is_second_order == 1 and c.time_accurate == 1
    assert c.local_time_stepping == 1 and c.cfl == 0.8
    assert c.limiter == cb.LIM_VANLEER and c.integrator == cb.INT_SSPRK3 and c.reconstruct_primitive == 1
    assert c.limiter_zeta == 0.5 and c.limiter_zeta1 == 0.25
    assert c.inlet_bc == cb.INLET_SUPERSONIC and abs(c.inlet_p - 0.714285714) < 1e-15
    assert c.movers_single_alpha == 0 and c.movers_entropy_fix == 0


def test_config_json_movers_keys(tmp_path):
    """Is_MOVERS_1 and Enable_Entropy_Fix are read from the Solver block as the reference reads them
    (src/Configuration_Read.cpp:72-73); Flux_Scheme names the three MOVERS-family schemes."""
    p = tmp_path / "Solver_Config.json"
    p.write_text('{"Solver": {"Dissipation_Type": 2, "Is_Second_Order": false, "Is_MOVERS_1": true, '
                 '"Enable_Entropy_Fix": true}}')
    c = cb.read_config_json(str(p))
    assert c.dissipation_type == cb.DISS_MOVERS and c.movers_single_alpha == 1 and c.movers_entropy_fix == 1
    for name, diss in (("ricca", cb.DISS_RICCA), ("movers_nwsc", cb.DISS_MOVERS_NWSC), ("movers", cb.DISS_MOVERS)):
        p.write_text('{"Solver": {"Flux_Scheme": "%s"}}' % name)
        assert cb.read_config_json(str(p)).dissipation_type == diss, name


def test_config_json_errors(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("{ \"Solver\": { \"CFL\": }")
    with pytest.raises(cb.CfdError) as e:
        cb.read_config_json(str(p))
    assert e.value.status == 1
    with pytest.raises(cb.CfdError) as e:
        cb.read_config_json(str(tmp_path / "missing.json"))
    assert e.value.status == 8


def test_create_without_device_is_a_status_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    m = cb.Mesh.box(8, 2)
    with pytest.raises(cb.CfdError) as e:
        cb.Solver(m, cb.default_config())
    assert e.value.status == 9


def test_bad_configs_rejected_before_device_use():
    m = cb.Mesh.box(8, 2)
    for kw in (dict(dissipation_type=1, is_second_order=1), dict(limiter=9), dict(dissipation_type=9),
               dict(dissipation_type=0), dict(dissipation_type=4, is_second_order=1, muscl=1),
               dict(dissipation_type=5, is_second_order=1, reconstruct_primitive=1)):
        with pytest.raises(cb.CfdError) as e:
            cb.Solver(m, cb.default_config(**kw))
        assert e.value.status == 1, kw
