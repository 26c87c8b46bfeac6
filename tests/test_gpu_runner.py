"""The host drop-in end to end: a reference .config through es_run_config (the
C ABI of the es_b200 runner) on the GPU, checked against the reference's own CPU
code (oracle/_ref) for the same samples and against the reference's folder layout
and file formats (src/SimulationRunner.cpp, src/Logger.cpp)."""
from __future__ import annotations

import ctypes as C
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O
from elasticscattering_b200 import _native as N
from elasticscattering_b200 import workloads

pytestmark = pytest.mark.gpu

DIM, PPQ, L, R_IMP, DENS, TCP = 17, 5, 1e-6, 2e-9, 2e15, 8
FIELDS = (10.0, 20.0)
TEMPS = (5.0, 40.0)
EXT = workloads.orbit_diameter(1.68e5, min(FIELDS))


def config_text(out_dir: Path, extra: str = "") -> str:
    return f"""# tiny sweep
num_samples 2
dimension {DIM}
phi_steps {PPQ}
temperatures 0 {TEMPS[0]} {TEMPS[1]}
magnetic_field_min {FIELDS[0]}
magnetic_field_max {FIELDS[1]}
magnetic_field_n 2
particle_speed 168000
clockwise 1
alpha 0.3
tau 1e-12
region_size {L}
region_extends {EXT!r}
impurity_density {DENS}
impurity_radius {R_IMP}
target_cell_population {TCP}
start_seed 0
output_directory {out_dir}
{extra}"""


def run_config(path: Path) -> Path:
    buf = C.create_string_buffer(4096)
    st = N.host_lib().es_run_config(str(path).encode(), buf, len(buf), 1)
    if st != N.ES_OK:
        raise N.EsError(st, N.host_lib().es_host_last_error().decode())
    return Path(buf.value.decode())


def reference_results():
    """Per (sample, sector, field): sigma per temperature from the reference's CPU code."""
    if not O.ref_available():
        pytest.skip("oracle/_ref was not built")
    lib = O.ref()
    out = {}
    for k in range(2):
        g = lib.ref_grid_new_seed((0 + 100) * (k + 1), L, EXT, DENS, R_IMP, TCP)
        for coh in (1, 0):
            sim = lib.ref_sim_new(g, DIM, PPQ, 1e-12, 0.3, 1, 1.68e5, L, EXT)
            lib.ref_sim_init_sample(sim, coh)
            for B in FIELDS:
                o = np.zeros(2 * len(TEMPS))
                m = (C.c_int * 7)()
                lib.ref_sim_sigmas(sim, B, np.array(TEMPS).ctypes.data, len(TEMPS), o.ctypes.data, m)
                out[(k, coh, B)] = o.reshape(-1, 2)
            lib.ref_sim_free(sim)
        lib.ref_grid_free(g)
    return out


def read_result_file(p: Path):
    rows = []
    lines = p.read_text().splitlines()
    start = next(i for i, s in enumerate(lines) if s.startswith("B "))
    for s in lines[start + 1:]:
        if s.strip():
            rows.append([float(x) for x in s.split()])
    return np.array(rows)


def png_pixels(p: Path):
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = 0
    while pos < len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(kind + body)
        if kind == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    assert len(raw) == h * (1 + 3 * w)
    return w, h


@pytest.mark.parametrize("extra", ["", "batched 1\n"])
def test_config_run_matches_reference_and_layout(tmp_path, cuda_device, extra):
    cfg = tmp_path / "tiny.config"
    cfg.write_text(config_text(tmp_path / "out", extra))
    out = run_config(cfg)
    assert out == tmp_path / "out" / "Result_0"
    assert (out / "tiny.config").read_text() == cfg.read_text()
    ref = reference_results()
    # T<j>.dat: per field the sample means of each sector, and delta_xx
    for j, T in enumerate(TEMPS):
        text = (out / f"T{j}.dat").read_text()
        assert text.startswith("# Elastic Scattering results summary.")
        assert f"Temperature {T:.4f}" in text and "Samples     2" in text and f"Positions   {DIM} x {DIM}" in text
        rows = read_result_file(out / f"T{j}.dat")
        assert rows.shape == (len(FIELDS), 6)
        for i, B in enumerate(FIELDS):
            coh = np.mean([ref[(k, 1, B)][j] for k in range(2)], axis=0)
            inc = np.mean([ref[(k, 0, B)][j] for k in range(2)], axis=0)
            assert rows[i, 0] == pytest.approx(B)
            expect = [inc[0], coh[0], inc[1], coh[1]]
            # printed with 7 significant digits
            assert np.allclose(rows[i, 1:5], expect, rtol=6e-7, atol=0), (B, rows[i, 1:5], expect)
            tot = [ref[(k, 1, B)][j][0] + ref[(k, 0, B)][j][0] for k in range(2)]
            mean = np.mean(tot)
            dxx = np.sqrt((np.mean(np.square(tot)) - mean * mean) / (2 - 1.0)) / mean
            assert rows[i, 5] == pytest.approx(dxx, rel=2e-3)
    metrics = (out / "Metrics.txt").read_text()
    assert metrics.startswith("# Metrics collected during particle lifetime computation.")
    assert "Sample 0 Coherent" in metrics and "Sample 1 Coherent" in metrics
    assert metrics.count("Metric (Incoherent)") == 2 and "Avg. particle lifetime" in metrics
    for k in range(2):
        sd = out / f"Sample {k}"
        assert (sd / "sample_results.dat").read_text().startswith("# Elastic Scattering sample results summary.")
        if not extra:
            for sector in ("Coherent", "Incoherent"):
                for j in range(len(TEMPS)):
                    for i in range(len(FIELDS)):
                        assert png_pixels(sd / sector / f"T{j} MF{i}.png") == (3 * DIM, DIM)


def test_second_run_takes_the_next_result_folder(tmp_path, cuda_device):
    cfg = tmp_path / "tiny.config"
    cfg.write_text(config_text(tmp_path / "out", "output_type results\n"))
    assert run_config(cfg).name == "Result_0"
    second = run_config(cfg)
    assert second.name == "Result_1"
    assert (second / "T0.dat").exists() and not (second / "Sample 0").exists()


CLI = Path(__file__).resolve().parent.parent / "elasticscattering_b200" / "es_b200"
TOTAL_PASSES = 2 * 2 * len(FIELDS)  # samples x sectors x fields


def run_cli(cfg: Path, fault: str | None = None):
    import os
    import subprocess

    env = dict(os.environ)
    env.pop("ES_FAULT_INJECT", None)
    if fault:
        env["ES_FAULT_INJECT"] = fault
    return subprocess.run([str(CLI), str(cfg)], capture_output=True, text=True, env=env, timeout=600)


def pass_counts(stdout: str):
    import re

    m = re.search(r"Passes: (\d+) computed, (\d+) from the journal", stdout)
    assert m, stdout
    return int(m.group(1)), int(m.group(2))


def result_rows(out: Path):
    return [read_result_file(out / f"T{j}.dat") for j in range(len(TEMPS))]


@pytest.mark.parametrize("extra", ["", "precision split\n"])
def test_sweep_stopped_by_a_failure_resumes_from_the_journal(tmp_path, cuda_device, extra):
    """A sweep stopped part way by an injected launch failure (ES_FAULT_INJECT,
    host-side) exits non-zero with the error; run again with the same journal it
    computes only the passes it had not finished, and its result files equal an
    uninterrupted run's."""
    from elasticscattering_b200 import journal

    clean = tmp_path / "clean.config"
    clean.write_text(config_text(tmp_path / "clean", "output_type results\n" + extra))
    ref = result_rows(run_config(clean))

    cfg = tmp_path / "sweep.config"
    jpath = tmp_path / "sweep.jsonl"
    cfg.write_text(config_text(tmp_path / "out", f"output_type results\njournal {jpath}\n" + extra))
    r = run_cli(cfg, fault="launch:12+")
    assert r.returncode != 0 and "launch" in r.stderr.lower(), (r.returncode, r.stderr)
    done = len(journal.read(jpath))
    assert 0 < done < TOTAL_PASSES, done

    r = run_cli(cfg)
    assert r.returncode == 0, r.stderr
    assert pass_counts(r.stdout) == (TOTAL_PASSES - done, done)
    assert len(journal.read(jpath)) == TOTAL_PASSES
    got = result_rows(sorted((tmp_path / "out").glob("Result_*"))[-1])
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_batched_sweep_computes_only_the_passes_missing_from_the_journal(tmp_path, cuda_device):
    from elasticscattering_b200 import journal

    cfg = tmp_path / "sweep.config"
    jpath = tmp_path / "sweep.jsonl"
    cfg.write_text(config_text(tmp_path / "out", f"output_type results\nbatched 1\nprecision split\njournal {jpath}\n"))
    r = run_cli(cfg)
    assert r.returncode == 0, r.stderr
    assert pass_counts(r.stdout) == (TOTAL_PASSES, 0)
    first = result_rows(tmp_path / "out" / "Result_0")
    lines = jpath.read_text().splitlines()
    jpath.write_text("\n".join(lines[:2] + lines[5:]) + "\n")  # three passes lost
    r = run_cli(cfg)
    assert r.returncode == 0, r.stderr
    assert pass_counts(r.stdout) == (3, TOTAL_PASSES - 3)
    assert len(journal.read(jpath)) == TOTAL_PASSES
    for a, b in zip(result_rows(tmp_path / "out" / "Result_1"), first):
        assert np.array_equal(a, b)
