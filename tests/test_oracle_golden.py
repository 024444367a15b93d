"""The oracle (C restatement, oracle/cbs_oracle.c) against golden vectors
produced by the reference solver itself (tests/golden/make_golden.py).

Every array is compared bitwise: the restatement keeps the reference's
operation order and the fixtures were made with one OpenMP thread."""
import numpy as np
import pytest

from helpers import STAGED, bitwise, fixture_path, load_case, stage_step
from oracle import pyoracle

PRE = ["fedge", "detJ", "dNkdx", "annxf", "alen_e", "pdiagE", "gstifE", "color_ptr", "color_elem",
       "bc_list", "bc_values", "wall_node_list", "face_norm", "Mdiag_real", "elcoe_e"]


def _oracle(name):
    case, z = load_case(fixture_path(name))
    return pyoracle.Oracle(case), z


@pytest.mark.parametrize("name", STAGED)
def test_preprocess_bitwise(name):
    o, z = _oracle(name)
    for k in PRE:
        assert bitwise(o.get(k), z["ref_" + k]), k
    # iside: local face numbers assigned from sorted triplets
    assert bitwise(o.get("iside"), z["ref_iside"])
    assert bitwise(o.get("unkno"), z["ref_init_unkno"])
    assert bitwise(o.get("pres"), z["ref_init_pres"])
    assert bitwise(o.get("temperature"), z["ref_init_temperature"])


@pytest.mark.parametrize("name", STAGED)
def test_stages_bitwise(name):
    o, z = _oracle(name)
    k = stage_step(z)
    o.step(k - 1)
    o.stage("begin_step")
    o.iitime += 1
    assert bitwise(o.get("unkno"), z["ref_s0_unkno"])
    o.stage("time_step")
    assert bitwise(o.get("delte"), z["ref_s1_delte"])
    assert bitwise(o.get("dtreal"), z["ref_s1_dtreal"])
    o.stage("lhs")
    for a in ("elcoe2", "elcoe2p", "pdiag", "gstif", "pres"):
        assert bitwise(o.get(a), z["ref_s2_" + a]), a
    o.stage("step1")
    assert bitwise(o.get("rhs"), z["ref_s3_rhs"])
    assert bitwise(o.get("unkno"), z["ref_s3_unkno"])
    if case_param(z, "step2_check"):
        o.stage("dt_correction")
        o.stage("lhs")
    o.stage("step2_rhs")
    assert bitwise(o.get("rhs1"), z["ref_s4_rhs1"])
    assert bitwise(o.get("pdiag"), z["ref_s4_pdiag_in"])
    assert bitwise(o.get("gstif"), z["ref_s4_gstif"])
    assert bitwise(o.pressure_multiply(z["ref_s4_pres_in"]), z["ref_s4_Apres"])
    o.set("pres", z["ref_s4_pres_in"])
    o.set("pdiag", z["ref_s4_pdiag_in"])
    o.set("gstif", z["ref_s4_gstif"])
    o.stage("solve_pressure")
    assert bitwise(o.get("pres"), z["ref_s5_pres"])
    assert bitwise(o.get("cg"), z["ref_s5_cg"])
    assert bitwise(o.get("rhs1"), z["ref_s5_rhs1"])
    o.stage("step3")
    assert bitwise(o.get("unkno"), z["ref_s6_unkno"])
    assert bitwise(o.get("rhs"), z["ref_s6_rhs"])
    o.stage("step4")
    if "ref_s7_temperature" in z.files:
        assert bitwise(o.get("rhs1"), z["ref_s7_rhs1"])
        assert bitwise(o.get("temperature"), z["ref_s7_temperature"])
    o.stage("convergence")
    assert bitwise(o.get("hb"), z["ref_s8_hb"])
    assert bitwise(o.get("velocity"), z["ref_s8_velocity"])


def case_param(z, key):
    import json
    return json.loads(bytes(z["params_json"]).decode()).get(key, 0)


@pytest.mark.parametrize("name", STAGED)
def test_full_run_bitwise(name):
    o, z = _oracle(name)
    n = int(z["nsteps"][0])
    hist = []
    for _ in range(n):
        o.step(1)
        cg = o.get("cg")
        hist.append(np.concatenate([o.get("dtreal"), cg, o.get("hb")]))
    assert bitwise(np.concatenate(hist), z["ref_history"])
    assert bitwise(o.get("unkno"), z["ref_final_unkno"])
    assert bitwise(o.get("pres"), z["ref_final_pres"])
    assert bitwise(o.get("temperature"), z["ref_final_temperature"])


def test_c1_cavity16_first_100_steps_bitwise():
    """Config-1 cavity (16^3 x 6 tets, Re=100): the first 100 of 500 steps."""
    o, z = _oracle("c1_cavity16")
    assert bitwise(o.get("color_ptr"), z["ref_color_ptr"])
    assert o.get("color_ptr").size - 1 == 30
    o.step(100)
    assert bitwise(o.get("unkno"), z["ref_step100_unkno"])
    assert bitwise(o.get("pres"), z["ref_step100_pres"])
    hist = z["ref_history"].reshape(-1, 21)
    assert int(o.get("cg")[0]) == int(hist[99, 1])
