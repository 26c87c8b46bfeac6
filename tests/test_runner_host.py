"""The host runtime's .config parser (libes_host.so, es_config_describe) against the
reference's parsing rules (src/SimulationConfiguration.h:79-228). No GPU needed."""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np
import pytest

from elasticscattering_b200 import _native as N
from elasticscattering_b200 import workloads

BASE = """num_samples 3
dimension 17
phi_steps 5
temperatures 0 2.5 10
magnetic_field_min 1
magnetic_field_max 4
magnetic_field_n 4
particle_speed 168000
clockwise 1
alpha 0.3
tau 1e-12
region_size 1e-6
region_extends 2e-6
impurity_density 1e15
impurity_radius 2e-9
start_seed 7
"""


def describe(path) -> dict:
    buf = C.create_string_buffer(1 << 16)
    st = N.host_lib().es_config_describe(str(path).encode(), buf, len(buf))
    if st != N.ES_OK:
        raise N.EsError(st, N.host_lib().es_host_last_error().decode())
    return json.loads(buf.value.decode())


def write(tmp_path, text, name="run.config"):
    p = tmp_path / name
    p.write_text(text)
    return p


def test_full_config_is_parsed_like_the_reference(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    d = describe(write(tmp_path, BASE))
    assert d["num_samples"] == 3 and d["dimension"] == 17 and d["phi_steps"] == 5
    assert d["magnetic_fields"] == [1.0, 2.0, 3.0, 4.0]
    assert d["temperatures"] == [2.5, 10.0]                   # T <= 0 is dropped
    assert d["sample_seeds"] == [(7 + 100) * (k + 1) for k in range(3)]
    assert d["target_cell_population"] == 15                  # the reference's default
    assert d["clockwise"] == 1 and d["alpha"] == 0.3 and d["tau"] == 1e-12
    assert d["output_type"] == "all" and d["output_directory"] == "ESLogs/Result_0"
    assert d["digits_in_sample_num"] == 1
    assert d["precision"] == N.ES_PRECISION_FP64 and d["batched"] == 0


def test_parser_quirks(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    text = ("# a comment\n://another\n\n" + BASE.replace("dimension 17", "dimension 17\ndimension 21")
            + "print_info\noutput_directory out dir\n")
    d = describe(write(tmp_path, text))
    assert d["dimension"] == 17                        # the first occurrence of a key wins
    assert d["print_info"] == 0                        # a key without a value maps to itself: atoi -> 0
    assert d["output_directory"] == "out dir/Result_0"  # the value is the rest of the line
    os.makedirs("out dir/Result_0")
    assert describe(write(tmp_path, text))["output_directory"] == "out dir/Result_1"
    d = describe(write(tmp_path, BASE + "output_type nothing\n"))
    assert d["output_type"] == "nothing" and d["output_directory"] == ""
    d = describe(write(tmp_path, BASE.replace("magnetic_field_min 1", "magnetic_field 6.5\nmagnetic_field_min 1")))
    assert d["magnetic_fields"] == [6.5]
    d = describe(write(tmp_path, BASE + "precision split\nbatched 1\ntarget_cell_population 9\n"))
    assert d["precision"] == N.ES_PRECISION_SPLIT and d["batched"] == 1 and d["target_cell_population"] == 9
    d = describe(write(tmp_path, BASE + "precision split_exact\n", "exact.config"))
    assert d["precision"] == N.ES_PRECISION_SPLIT_EXACT


@pytest.mark.parametrize("edit,message", [
    (("phi_steps 5", "phi_steps 4"), "Phi steps must be odd."),
    (("dimension 17", "dimension 16"), "Dimension must be odd."),
    (("num_samples 3", "num_samples 0"), "Samples must be greater than 0."),
    (("magnetic_field_n 4", "magnetic_field_n 1"), "magnetic field range with n<2"),
    (("tau 1e-12\n", ""), "missing config key 'tau'"),
])
def test_config_errors_are_reported(tmp_path, edit, message):
    p = write(tmp_path, BASE.replace(*edit))
    with pytest.raises(N.EsError, match=message.replace("(", r"\(").replace(")", r"\)")):
        describe(p)


def test_missing_file(tmp_path):
    with pytest.raises(N.EsError, match="Could not load config file"):
        describe(tmp_path / "nope.config")


def test_workload_config_text_round_trips(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    for w in (workloads.config0(), workloads.config3()):
        w.fields = [2.0, 4.5, 7.0] if w.name.startswith("config3") else w.fields
        d = describe(write(tmp_path, w.config_text()))
        assert d["dimension"] == w.dim and d["phi_steps"] == w.phi_steps
        assert np.allclose(d["magnetic_fields"], w.fields)
        assert d["target_cell_population"] == w.target_cell_population
        assert d["sample_seeds"] == [w.seed(0)]
        assert d["region_extends"] == w.region_extends and d["impurity_density"] == w.density
    # config 1's fields {1, 5, 10, 20, 40} are not a uniform range: a .config cannot hold them
    with pytest.raises(ValueError):
        workloads.config1().config_text()
