"""The per-pass results journal (config key `journal`, host/journal.cpp) on the
host: a sweep whose every pass is in the journal runs without a GPU, writes
T<j>.dat and Metrics.txt from the journal's sigmas and metrics, and skips torn
lines and lines of other runs; a sweep with a pass missing goes to the device
for it. The GPU side -- a sweep stopped by an injected failure and resumed --
is tests/test_gpu_runner.py's."""
from __future__ import annotations

import ctypes as C
import json

import numpy as np
import pytest

from elasticscattering_b200 import _native as N
from elasticscattering_b200 import journal
from elasticscattering_b200.batch import finish_results
from conftest import gpu_available

CONFIG = """num_samples 2
dimension 17
phi_steps 5
temperatures 2.5 10
magnetic_field_min 1
magnetic_field_max 3
magnetic_field_n 3
particle_speed 168000
clockwise 1
alpha 0.3
tau 1e-12
region_size 1e-6
region_extends 2e-6
impurity_density 1e15
impurity_radius 2e-9
start_seed 7
output_type results
"""


def describe(path) -> dict:
    buf = C.create_string_buffer(1 << 16)
    assert N.host_lib().es_config_describe(str(path).encode(), buf, len(buf)) == N.ES_OK
    return json.loads(buf.value.decode())


def run(path):
    out = C.create_string_buffer(4096)
    st = N.host_lib().es_run_config(str(path).encode(), out, len(out), 1)
    return st, out.value.decode()


def synthetic_sigma(s, coherent, i, t):
    """A distinct, deterministic sigma per (sample, sector, field, temperature)."""
    xx = 1.0e5 * (1.0 + 0.11 * s + 0.017 * i + 0.0031 * t + (0.5 if coherent else 0.0))
    xy = -3.0e3 * (1.0 + 0.07 * s - 0.013 * i + 0.0029 * t + (0.25 if coherent else 0.0))
    return xx, xy


def write_journal(cfg, path, skip=None, extra_lines=()):
    key = journal.run_key(cfg)
    lines = list(extra_lines[:1])
    for s, seed in enumerate(cfg["sample_seeds"]):
        for coherent in (True, False):
            for i, b in enumerate(cfg["magnetic_fields"]):
                if skip == (s, coherent, i):
                    continue
                sig = [synthetic_sigma(s, coherent, i, t) for t in range(len(cfg["temperatures"]))]
                met = {"cells_passed": 1000 + i, "impurities_tested": 5000 + s, "particles_inside_impurity": 7}
                lines.append(journal.format_entry(key, s, seed, coherent, b, sig, met, 17 * 17 * 20 - 7,
                                                  avg_particle_lifetime=1e-13, time_lifetimes=0.01))
    lines += list(extra_lines[1:])
    path.write_text("\n".join(lines) + "\n")
    return key


def read_rows(p):
    lines = p.read_text().splitlines()
    start = next(i for i, s in enumerate(lines) if s.startswith("B "))
    return np.array([[float(x) for x in s.split()] for s in lines[start + 1:] if s.strip()])


def test_run_key_matches_the_writer(tmp_path, monkeypatch):
    """The Python run key is the one host/journal.cpp writes: a journal made
    with it is taken whole (checked by the run below needing no device)."""
    monkeypatch.chdir(tmp_path)
    (tmp_path / "a.config").write_text(CONFIG)
    (tmp_path / "b.config").write_text(CONFIG.replace("tau 1e-12", "tau 2e-12"))
    (tmp_path / "c.config").write_text(CONFIG + "precision split\n")
    (tmp_path / "d.config").write_text(CONFIG + "batched 1\n")
    (tmp_path / "e.config").write_text(CONFIG.replace("start_seed 7", "start_seed 8"))
    keys = [journal.run_key(describe(tmp_path / n)) for n in ("a.config", "b.config", "c.config", "d.config",
                                                                "e.config")]
    assert len(set(keys[:4])) == 4
    assert keys[4] == keys[0]  # seeds are per entry, not part of the run


def test_whole_journal_runs_without_a_device(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    cfg_path = tmp_path / "run.config"
    cfg_path.write_text(CONFIG + "journal sweep.jsonl\n")
    cfg = describe(cfg_path)
    assert cfg["journal"] == "sweep.jsonl"
    other = journal.format_entry(12345, 0, cfg["sample_seeds"][0], True, 1.0, [(9.0, 9.0), (9.0, 9.0)], {}, 1)
    torn = journal.format_entry(journal.run_key(cfg), 1, cfg["sample_seeds"][1], False, 2.0,
                                [(9.0, 9.0), (9.0, 9.0)], {}, 1)[:-20]
    write_journal(cfg, tmp_path / "sweep.jsonl", extra_lines=(other, torn))
    before = (tmp_path / "sweep.jsonl").read_text()
    st, out_dir = run(cfg_path)
    assert st == N.ES_OK, N.host_lib().es_host_last_error()
    assert (tmp_path / "sweep.jsonl").read_text() == before  # nothing computed, nothing appended
    S, F, T = len(cfg["sample_seeds"]), len(cfg["magnetic_fields"]), len(cfg["temperatures"])
    coh = np.array([[[synthetic_sigma(s, True, i, t) for t in range(T)] for i in range(F)] for s in range(S)])
    inc = np.array([[[synthetic_sigma(s, False, i, t) for t in range(T)] for i in range(F)] for s in range(S)])
    fin = finish_results(coh, inc)
    for t in range(T):
        rows = read_rows(tmp_path / out_dir / f"T{t}.dat")
        assert rows.shape == (F, 6)
        for i, b in enumerate(cfg["magnetic_fields"]):
            expect = [fin["incoherent"][i, t, 0], fin["coherent"][i, t, 0], fin["incoherent"][i, t, 1],
                      fin["coherent"][i, t, 1]]
            assert rows[i, 0] == pytest.approx(b)
            assert np.allclose(rows[i, 1:5], expect, rtol=6e-7, atol=0), (t, i)
            assert rows[i, 5] == pytest.approx(fin["delta_xx"][i, t], rel=2e-3)
    metrics = (tmp_path / out_dir / "Metrics.txt").read_text()
    assert "Sample 1 Coherent" in metrics and metrics.count("Metric (Incoherent)") == 2


def test_torn_line_gets_a_newline_before_the_next_entry(tmp_path, monkeypatch):
    """A journal that ends in a torn line is closed with a newline when it is
    opened, so an appended entry starts on a line of its own."""
    monkeypatch.chdir(tmp_path)
    cfg_path = tmp_path / "run.config"
    cfg_path.write_text(CONFIG + "journal sweep.jsonl\n")
    cfg = describe(cfg_path)
    key = write_journal(cfg, tmp_path / "sweep.jsonl")
    with open(tmp_path / "sweep.jsonl", "a") as f:
        f.write('{"journal":1,"run":"')
    st, _ = run(cfg_path)
    assert st == N.ES_OK
    text = (tmp_path / "sweep.jsonl").read_text()
    assert text.endswith('{"journal":1,"run":"\n')
    assert len(journal.read(tmp_path / "sweep.jsonl", key)) == 2 * 2 * 3


@pytest.mark.skipif(gpu_available(), reason="checks that a missing pass needs the device")
def test_missing_pass_goes_to_the_device(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    cfg_path = tmp_path / "run.config"
    cfg_path.write_text(CONFIG + "journal sweep.jsonl\n")
    cfg = describe(cfg_path)
    write_journal(cfg, tmp_path / "sweep.jsonl", skip=(1, False, 2))
    st, _ = run(cfg_path)
    assert st != N.ES_OK
    assert "device" in N.host_lib().es_host_last_error().decode().lower()


def test_reader_skips_foreign_and_torn_lines(tmp_path):
    p = tmp_path / "j.jsonl"
    good = journal.format_entry(7, 0, 107, True, 2.5, [(1.0, 2.0)], {"cells_passed": 3}, 9)
    p.write_text("\n".join([good, journal.format_entry(8, 0, 107, True, 2.5, [(1.0, 2.0)], {}, 9), "not json",
                            good[:30]]) + "\n")
    assert len(journal.read(p)) == 2
    e = journal.read(p, key=7)
    assert len(e) == 1 and e[0]["sigma"] == [[1.0, 2.0]] and e[0]["metrics"]["cells_passed"] == 3
