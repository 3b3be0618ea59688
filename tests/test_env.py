"""Environment files: the reference's parse rules and Bvh.* option handling (CPU only).

Mirrors environment/Environment.cpp:17-466 and environment/AppEnvironment.cpp:10-91.
"""
import pytest

import hippie_b200 as hp
from hippie_b200 import HPError

PLOC_ENV = """
Application {
    mode benchmark   # comment
}
Bvh {
    method ploc
    plocMortonCodeBits 60
    plocRadius 16
    plocAdaptive false
    plocMaxRadius 256
    layout bin
}
"""


def test_defaults():
    e = hp.Env()
    assert e.get_string("Bvh.method") == "lbvh"
    assert e.get_int("Bvh.lbvhMortonCodeBits") == 60
    assert e.get_float("Bvh.ct") == 3.0 and e.get_float("Bvh.ci") == 2.0
    assert e.get_bool("Bvh.adaptiveLeafSize") is True
    assert e.get_int("Bvh.atrTreeletSize") == 20
    p = e.build_params()
    assert p.method == hp.HP_METHOD_LBVH and p.morton_bits == 60 and p.max_leaf_size == 8


def test_benchmark_config_file(tmp_path):
    f = tmp_path / "ploc_radius16.env"
    f.write_text(PLOC_ENV)
    e = hp.Env().read_file(str(f))
    assert e.get_string("Application.mode") == "benchmark"
    p = e.build_params()
    assert p.method == hp.HP_METHOD_PLOC
    assert (p.ploc_radius, p.ploc_max_radius, p.ploc_adaptive, p.morton_bits) == (16, 256, 0, 60)


def test_unknown_key_fails():
    with pytest.raises(HPError) as ei:
        hp.Env().read_string("Bvh {\n insertionAnnealingSteps 3\n}\n")
    assert "unknown option" in str(ei.value)


def test_type_mismatch_fails():
    with pytest.raises(HPError):
        hp.Env().read_string("Bvh { maxLeafSize eight }")
    with pytest.raises(HPError):
        hp.Env().read_string("Bvh { adaptiveLeafSize maybe }")
    with pytest.raises(HPError):
        hp.Env().read_string("Camera { position 1 2 }")
    with pytest.raises(HPError):  # the value must be on the key's line
        hp.Env().read_string("Bvh {\n method\n lbvh\n}")


def test_unpaired_brace_fails():
    with pytest.raises(HPError):
        hp.Env().read_string("}\n")


def test_first_value_wins_and_bools():
    e = hp.Env().read_string("Bvh {\n maxLeafSize 4\n maxLeafSize 16\n adaptiveLeafSize OFF\n}")
    assert e.get_int("Bvh.maxLeafSize") == 4
    assert e.get_bool("Bvh.adaptiveLeafSize") is False
    for word, val in [("yes", True), ("on", True), ("TRUE", True), ("1", True), ("no", False), ("NO", False)]:
        assert hp.Env().read_string(f"Bvh {{ plocAdaptive {word} }}").get_bool("Bvh.plocAdaptive") is val


def test_float_values_keep_six_digits():
    # QString::number(float) keeps 6 significant digits
    e = hp.Env().read_string("Bvh { ct 3.14159265 }")
    import numpy as np
    assert e.get_float("Bvh.ct") == np.float32(3.14159)


def test_vector_option():
    e = hp.Env().read_string("Scene { light 0.48 0.08 0.17 }")
    assert e.get_string("Scene.light") == "0.48 0.08 0.17"


def test_out_of_range_keeps_default():
    p = hp.Env().read_string("Bvh { lbvhMortonCodeBits 70\n maxLeafSize 0\n atrIterations 40 }").build_params()
    assert p.morton_bits == 60 and p.max_leaf_size == 8 and p.atr_iterations == 2
    p = hp.Env().read_string("Bvh { method ploc\n plocRadius 600 }").build_params()
    assert p.ploc_radius == 1  # radius must not exceed plocMaxRadius (512)
    p = hp.Env().read_string("Bvh { ct -1.0 }").build_params()
    assert p.ct == 3.0


def test_method_and_layout_support():
    with pytest.raises(HPError) as ei:
        hp.Env().read_string("Bvh { method sbvh }").build_params()
    assert ei.value.status == 6
    # HLBVHBuilder: its own Morton bits and the SAH bits in [6,15], at most the Morton bits
    p = hp.Env().read_string("Bvh { method hlbvh\n hlbvhMortonCodeBits 30\n hlbvhMortonCodeSAHBits 9 }").build_params()
    assert (p.method, p.morton_bits, p.hlbvh_sah_bits) == (4, 30, 9)
    assert hp.Env().read_string("Bvh { method hlbvh }").build_params().hlbvh_sah_bits == 15
    for bad in ("hlbvhMortonCodeSAHBits 16", "hlbvhMortonCodeSAHBits 5",
                "hlbvhMortonCodeBits 12\n hlbvhMortonCodeSAHBits 15"):
        assert hp.Env().read_string("Bvh { method hlbvh\n %s }" % bad).build_params().hlbvh_sah_bits == 15
    # HipBVH: "bin", "quad", anything else Oct
    for text, want in (("bin", 2), ("quad", 4), ("oct", 8), ("octree", 8)):
        assert hp.Env().read_string("Bvh { layout %s }" % text).build_params().layout == want
    p = hp.Env().read_string("Bvh { method atr\n atrTreeletSize 9\n atrIterations 2 }").build_params()
    assert p.method == hp.HP_METHOD_ATR and p.atr_treelet == 9 and p.atr_iterations == 2
