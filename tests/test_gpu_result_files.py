"""Result files, byte for byte: one .config run through the reference's own
runner and writers on the CPU (oracle/_ref/libes_refrun.so: SimulationRunner,
Logger, SimulationCPU, Grid, unmodified) and through the B200 runner
(es_run_config) on the GPU. The results folders must hold the same files; the
copied config, every T<j>.dat and every sample_results.dat must be identical
bytes; Metrics.txt must be identical once its wall-clock timings are masked;
the PNG maps must hold the same pixels (at most a few one-level differences,
where a map value lies within 1e-9 of a pixel boundary). The reference's own
loader logic (reproduce_graphs/Reproduce SM figure 2/view_result.py:57-78,
restated in read_t_file) must read the B200 runner's T<j>.dat files into the
reference's numbers."""
from __future__ import annotations

import ctypes as C
import os
import re
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

import refrun_lib as RR
from elasticscattering_b200 import _native as N

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not RR.available(), reason="oracle/_ref/libes_refrun.so absent")]

CONFIG = """# a small sweep: 2 samples x 2 fields x 2 temperatures, images on
num_samples 2
dimension 17
phi_steps 5
temperatures 0 5 40
magnetic_field_min 10
magnetic_field_max 20
magnetic_field_n 2
particle_speed 168000
clockwise 1
alpha 0.3
tau 1e-12
region_size 1e-6
region_extends 4.776e-7
impurity_density 2e15
impurity_radius 2e-9
target_cell_population 8
start_seed 0
output_directory out
"""


def read_t_file(path: Path):
    """view_result.py's read_T0_file (reproduce_graphs/Reproduce SM figure
    2/view_result.py:57-78): the temperature line, the label line starting with
    'B' and holding 'sigma', then one row of floats per line."""
    data = []
    temperature = -1.0
    with open(path) as f:
        for line in f:
            if "Temperature" in line:
                temperature = float(line.split()[-1])
            if line.startswith("B") and "sigma" in line:
                break
        else:
            raise ValueError(f"No labels found in file {path}")
        assert temperature >= 0
        labels = line.split()
        for line in f:
            if line:
                data.append([float(x) for x in line.split()])
                assert len(data[-1]) == len(labels)
    return temperature, labels, np.array(data)


TIMING = re.compile(r"│[^│]*ms")


def mask_timings(text: str) -> str:
    out = []
    for line in text.splitlines():
        if line.startswith("Index time"):
            line = "Index time <t>ms"
        elif "Lifetimes" in line or "Temperatures" in line:
            line = TIMING.sub("│<t>ms", line)
        out.append(line)
    return "\n".join(out)


def png_rgb(p: Path) -> np.ndarray:
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 2
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), dtype=np.uint8).reshape(h, 1 + 3 * w)
    out = np.zeros((h, 3 * w), dtype=np.int32)
    prev = np.zeros(3 * w, dtype=np.int32)
    for y in range(h):  # undo the per-row PNG filters (types 0-4)
        f, line = raw[y, 0], raw[y, 1:].astype(np.int32)
        cur = np.zeros(3 * w, dtype=np.int32)
        for x in range(3 * w):
            a = cur[x - 3] if x >= 3 else 0
            b = prev[x]
            c = prev[x - 3] if x >= 3 else 0
            if f == 0:
                pr = 0
            elif f == 1:
                pr = a
            elif f == 2:
                pr = b
            elif f == 3:
                pr = (a + b) // 2
            else:
                p_ = a + b - c
                pa, pb, pc = abs(p_ - a), abs(p_ - b), abs(p_ - c)
                pr = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[x] = (line[x] + pr) & 0xFF
        out[y] = cur
        prev = cur
    return out


def run_ours(cfg: Path) -> Path:
    buf = C.create_string_buffer(4096)
    here = os.getcwd()
    os.chdir(cfg.parent)
    try:
        st = N.host_lib().es_run_config(cfg.name.encode(), buf, len(buf), 1)
    finally:
        os.chdir(here)
    if st != N.ES_OK:
        raise N.EsError(st, N.host_lib().es_host_last_error().decode())
    return cfg.parent / "out" / "Result_0"


def tree(d: Path) -> list:
    return sorted(str(p.relative_to(d)) for p in d.rglob("*"))


def test_results_folder_matches_the_reference_writers(tmp_path, cuda_device):
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    for d in (ref_dir, our_dir):
        d.mkdir()
        (d / "tiny.config").write_text(CONFIG)
    r = RR.run(ref_dir / "tiny.config", ref_dir)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    ref = ref_dir / "out" / "Result_0"
    ours = run_ours(our_dir / "tiny.config")
    assert tree(ours) == tree(ref)
    assert (ours / "tiny.config").read_bytes() == (ref / "tiny.config").read_bytes()
    t_files = sorted(p.name for p in ref.glob("T*.dat"))
    assert t_files == ["T0.dat", "T1.dat"]
    for name in t_files:
        assert (ours / name).read_bytes() == (ref / name).read_bytes(), name
        tr, lr, dr = read_t_file(ref / name)
        to, lo, do = read_t_file(ours / name)
        assert (to, lo) == (tr, lr) and np.array_equal(do, dr)
    for k in range(2):
        rel = Path(f"Sample {k}") / "sample_results.dat"
        assert (ours / rel).read_bytes() == (ref / rel).read_bytes(), rel
    assert mask_timings((ours / "Metrics.txt").read_text(encoding="utf-8")) == \
        mask_timings((ref / "Metrics.txt").read_text(encoding="utf-8"))
    differing = 0
    for png in sorted(ref.rglob("*.png")):
        a, b = png_rgb(png), png_rgb(ours / png.relative_to(ref))
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 1, png
        differing += int((a != b).sum())
    assert differing <= 8
